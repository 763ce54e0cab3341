// segplan.hpp -- tile and split tables of the segmented-reduction engine
// (segreduce.cuh) and range tables of the warp-range segmented sweep
// (segsweep.cuh), shared by the host planners and the device kernels.
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

// Warp-range segmented sweep: one warp per range of consecutive positions of
// one problem.  Positions of a problem are [ptr[0], ptr[n_seg]); ranges start
// at ptr[0] + a multiple of SS_ALIGN positions, so that every chunk a warp
// reads starts on a 32-bit word of the segment-start bitmap.
constexpr int SS_THREADS = 256;
constexpr uint32_t SS_ALIGN = 128;
constexpr uint32_t SS_IDENTITY = 0xFFFFFFFFu;

struct SSRange {
    uint32_t problem;
    uint32_t p0, p1;       // positions [p0, p1)
    uint32_t word0;        // bitmap word of position p0
    uint32_t o0;           // ordinal (among the problem's non-empty segments) of the segment holding p0
    int32_t head_split;    // split id of the segment continuing into p0 from an earlier range, or -1
    int32_t tail_split;    // split id of the range's last segment when it runs past p1, or -1
    uint32_t e_lo, e_hi;   // empty segments this range emits: entries [e_lo, e_hi) of the empty list
    uint32_t nz_off;       // offset of the problem's non-empty segment ids, SS_IDENTITY = none empty
    uint32_t pad[2];
};

struct SSSplit {
    uint32_t problem, seg;
    uint32_t r0, r1;       // global range ids: the tail range (where the segment starts) .. the last head range
};

}  // namespace wgpu
