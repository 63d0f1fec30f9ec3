// Radius blocks of a work list for the persistent superposition kernels (forward
// and adjoint): the list holds each radius R in one block starting at
// BeamStateDev::rStart[R], the wide radii first, of which the first mergedR[R]
// items are live.
#pragma once

#include "pbs_types.h"

namespace pbs {

// Radius blocks of an instance: claim c of the instance is item c of the
// concatenated merged items of radii RHi, RHi - 1, ..., RLo.
template <int RLo, int RHi>
struct RadiusBlocks {
    int start[RHi - RLo + 1];
    int count[RHi - RLo + 1];
    int total;
};

template <int RLo, int RHi>
__device__ __forceinline__ void load_blocks(const BeamStateDev* beam, RadiusBlocks<RLo, RHi>& b) {
    const int t = threadIdx.x;
    if (t <= RHi - RLo) {
        const int R = RHi - t;
        const int end = R > 0 ? beam->rStart[R - 1] : beam->workCount;
        b.start[t] = beam->rStart[R];
        b.count[t] = max(min(beam->mergedR[R], end - beam->rStart[R]), 0);
    }
    __syncthreads();
    if (t == 0) {
        int n = 0;
        for (int i = 0; i <= RHi - RLo; ++i) n += b.count[i];
        b.total = n;
    }
}

template <int RLo, int RHi>
__device__ __forceinline__ int block_slot(const RadiusBlocks<RLo, RHi>& b, int c) {
#pragma unroll 1
    for (int i = 0; i <= RHi - RLo; ++i) {
        if (c < b.count[i]) return b.start[i] + c;
        c -= b.count[i];
    }
    return -1;
}

}  // namespace pbs
