// pdl.cuh -- programmatic dependent launch.  Every kernel of the solve's
// loops starts with pdl_wait() (griddepcontrol.wait: block until the grid it
// depends on has completed and its memory is visible; immediate when the
// kernel was launched without a programmatic dependency) and then
// pdl_launch_dependents() (griddepcontrol.launch_dependents), so a kernel
// launched after it with programmatic stream serialisation is scheduled once
// all of this grid's blocks have started, and its launch latency overlaps
// this grid's tail.  Nothing a kernel reads or writes is touched before its
// wait, so the results are those of plain stream order.
#pragma once

namespace wgpu {

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

}  // namespace wgpu
