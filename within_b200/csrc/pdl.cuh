// pdl.cuh -- programmatic dependent launch.  Every kernel of the solve's
// loops starts with pdl_wait() (griddepcontrol.wait: block until the grid it
// depends on has completed and its memory is visible; immediate when the
// kernel was launched without a programmatic dependency), so a kernel
// launched after it with programmatic stream serialisation is scheduled as
// this grid's blocks finish (or, with c_pdl_early, once they have all
// started: pdl_launch_dependents, griddepcontrol.launch_dependents) and its
// launch latency overlaps this grid's tail.  Nothing a kernel reads or writes is touched before its
// wait, so the results are those of plain stream order.
#pragma once

namespace wgpu {

// 1: a kernel lets its dependent launch as soon as its blocks start
// (set per device by the host, WITHIN_PDL_EARLY); 0: when its blocks exit
__constant__ int c_pdl_early;

__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch_dependents() {
    if (c_pdl_early) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

}  // namespace wgpu
