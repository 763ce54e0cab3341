// segplan.hpp -- tile and split tables of the segmented-reduction engine
// (segreduce.cuh), shared by the host planner and the device kernel.
#pragma once
#include <cstdint>

namespace wgpu {

constexpr int SR_THREADS = 256;

struct SRTile {
    uint32_t problem;      // index of the problem (value functor context)
    uint32_t p0, p1;       // position range [p0, p1) inside the problem
    uint32_t own_lo, own_hi;  // segments whose first position lies in [p0, p1)
    int32_t cont_split;    // split id of the segment continuing into p0, or -1
    int32_t tail_split;    // split id of the owned segment that runs past p1, or -1
    uint32_t pad;
};

struct SRSplit {
    uint32_t problem, seg;
    uint32_t t0, t1;       // global tile ids: owner (tail) .. last tile (head)
};

}  // namespace wgpu
