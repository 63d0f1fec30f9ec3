// Tile-based Gaussian superposition of the per-ray IDD into the padded BEV dose.
//
// Work items come from the radius-sorted list built on the device; each item is one
// 32x8 tile of source rays at one step of one layer with its batched radius R
// (kernelSuperposition<R>, complete_superposition.cu:264-335). Every source s
// spreads idd_s * e_s(dy) * e_s(dx) over a (2R+1)^2 footprint, where
// e_s(0) = erf(r/2) and e_s(i) = (erf((i+1/2) r) - erf((i-1/2) r)) / 2.
//
// Register-blocked formulation (FP32 FMA pipe):
//   * a CTA owns one tile; warp w owns source row w of the tile;
//   * lanes are output columns (one 32-column chunk at a time); each lane keeps
//     the 2R+1 output rows its source row reaches in registers;
//   * per source, the lane factor idd_s * e_s(|dx|) is one shared-memory load and
//     the row factors e_s(0..R) are broadcast 16-byte loads, each reused for the
//     two symmetric rows R-k and R+k, feeding 2R+1 FMAs;
//   * the eight warps' partial rows are summed in a shared tile and the tile is
//     added to the BEV dose of its step (all layers share one BEV volume).
// A persistent grid pulls items from the list with an atomic counter.
#include "kernels.h"

namespace pbs {

namespace {

constexpr int kThreads = 256;
constexpr int kEStride = 36;                      // >= kMaxR + 1, multiple of 4 (16-byte rows)
constexpr int kOutH = kTileY + 2 * kMaxR;         // 72
constexpr int kOutW = kTileX + 2 * kMaxR;         // 96
constexpr size_t kSmemBytes = (2 * kThreads * kEStride + kOutH * kOutW) * sizeof(float);

template <int R>
__device__ __forceinline__ void superpose_rows(const float* __restrict__ E, const float* __restrict__ EW,
                                               float* __restrict__ out, int warp, int lane) {
    constexpr int N = 2 * R + 1;
    constexpr int Wo = kTileX + 2 * R;
    constexpr int kChunks = (Wo + 31) / 32;
    constexpr int kVec = (R + 1 + 3) / 4;
    const int sy = warp;
#pragma unroll 1
    for (int cc = 0; cc < kChunks; ++cc) {
        const int ox = cc * 32 + lane;
        float acc[N];
#pragma unroll
        for (int j = 0; j < N; ++j) acc[j] = 0.0f;
        const int sxLo = max(0, cc * 32 - 2 * R);
        const int sxHi = min(kTileX - 1, cc * 32 + 31);
        const float* eRow = E + (sy * kTileX) * kEStride;
        const float* wRow = EW + (sy * kTileX) * kEStride;
#pragma unroll 2
        for (int sx = sxLo; sx <= sxHi; ++sx) {
            const int d = ox - sx - R;  // column offset from the source, in [-R, R] when reached
            const int ad = d < 0 ? -d : d;
            const float w = (ad <= R) ? wRow[sx * kEStride + ad] : 0.0f;
            const float4* ev = reinterpret_cast<const float4*>(eRow + sx * kEStride);
#pragma unroll
            for (int q = 0; q < kVec; ++q) {
                const float4 v = ev[q];
                const float e4[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int k = 4 * q + c;
                    if (k <= R) {
                        acc[R + k] = fmaf(w, e4[c], acc[R + k]);
                        if (k > 0) acc[R - k] = fmaf(w, e4[c], acc[R - k]);
                    }
                }
            }
        }
        if (ox < Wo) {
#pragma unroll
            for (int j = 0; j < N; ++j)
                if (acc[j] != 0.0f) atomicAdd(out + (sy + j) * Wo + ox, acc[j]);
        }
    }
}

#define PBS_SUPERPOSE_CASE(R) \
    case R: superpose_rows<R>(E, EW, out, warp, lane); break;

__global__ void __launch_bounds__(kThreads, 2)
superpose_kernel(BeamGeomDev g, const float* __restrict__ idd, const float* __restrict__ rsig,
                 const int4* __restrict__ work, BeamStateDev* __restrict__ beam, float* __restrict__ bev) {
    extern __shared__ __align__(16) float sm[];
    float* E = sm;                               // [256][kEStride]  e_s(k), k = 0..R
    float* EW = sm + kThreads * kEStride;        // [256][kEStride]  idd_s * e_s(k)
    float* out = sm + 2 * kThreads * kEStride;   // [8+2R][32+2R]    tile footprint
    __shared__ int sItem;

    const int t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31;
    const int count = beam->workCount;
    const size_t padPlane = static_cast<size_t>(g.pitchX) * g.pitchY;
    const size_t layerStride = static_cast<size_t>(g.steps) * padPlane;
    const size_t bevPlane = static_cast<size_t>(g.bevX) * g.bevY;

    for (;;) {
        if (t == 0) sItem = atomicAdd(&beam->workNext, 1);
        __syncthreads();
        const int w = sItem;
        if (w >= count) break;
        const int4 it = work[w];
        const int lc = it.x, tile = it.y, zRel = it.z, R = it.w;
        const int tx = tile % g.tilesX, ty = tile / g.tilesX;
        const int Ho = kTileY + 2 * R, Wo = kTileX + 2 * R;

        // Source ray t of the tile: erf-difference table (complete_superposition.cu:298-307).
        {
            const int sy = t >> 5, sx = t & 31;
            const size_t src = lc * layerStride + zRel * padPlane + static_cast<size_t>(ty * kTileY + sy) * g.pitchX +
                               tx * kTileX + sx;
            const float dose = idd[src];
            const float rs = rsig[src];
            const bool live = dose > 0.0f;
            float erfNew = erff(rs * 0.5f);
            float erfOld = -erfNew;
            float* e = E + t * kEStride;
            float* ew = EW + t * kEStride;
            for (int i = 0; i <= R; ++i) {
                const float dv = 0.5f * (erfNew - erfOld);
                e[i] = dv;
                ew[i] = live ? dose * dv : 0.0f;
                erfOld = erfNew;
                erfNew = erff(rs * (float(i) + 1.5f));
            }
            for (int i = t; i < Ho * Wo; i += kThreads) out[i] = 0.0f;
        }
        __syncthreads();

        switch (R) {
            PBS_SUPERPOSE_CASE(0) PBS_SUPERPOSE_CASE(1) PBS_SUPERPOSE_CASE(2) PBS_SUPERPOSE_CASE(3)
            PBS_SUPERPOSE_CASE(4) PBS_SUPERPOSE_CASE(5) PBS_SUPERPOSE_CASE(6) PBS_SUPERPOSE_CASE(7)
            PBS_SUPERPOSE_CASE(8) PBS_SUPERPOSE_CASE(9) PBS_SUPERPOSE_CASE(10) PBS_SUPERPOSE_CASE(11)
            PBS_SUPERPOSE_CASE(12) PBS_SUPERPOSE_CASE(13) PBS_SUPERPOSE_CASE(14) PBS_SUPERPOSE_CASE(15)
            PBS_SUPERPOSE_CASE(16) PBS_SUPERPOSE_CASE(17) PBS_SUPERPOSE_CASE(18) PBS_SUPERPOSE_CASE(19)
            PBS_SUPERPOSE_CASE(20) PBS_SUPERPOSE_CASE(21) PBS_SUPERPOSE_CASE(22) PBS_SUPERPOSE_CASE(23)
            PBS_SUPERPOSE_CASE(24) PBS_SUPERPOSE_CASE(25) PBS_SUPERPOSE_CASE(26) PBS_SUPERPOSE_CASE(27)
            PBS_SUPERPOSE_CASE(28) PBS_SUPERPOSE_CASE(29) PBS_SUPERPOSE_CASE(30) PBS_SUPERPOSE_CASE(31)
            PBS_SUPERPOSE_CASE(32)
            default: break;
        }
        __syncthreads();

        float* dst = bev + static_cast<size_t>(zRel) * bevPlane + static_cast<size_t>(ty * kTileY - R + kMaxR) * g.bevX +
                     (tx * kTileX - R + kMaxR);
        for (int i = t; i < Ho * Wo; i += kThreads) {
            const float v = out[i];
            const int oy = i / Wo, ox = i - oy * Wo;
            if (v != 0.0f) atomicAdd(dst + static_cast<size_t>(oy) * g.bevX + ox, v);
        }
        // The next claim overwrites sItem only after every thread passed the sync below.
        __syncthreads();
    }
}

#undef PBS_SUPERPOSE_CASE

}  // namespace

cudaError_t launch_superpose(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                             BeamStateDev* beam, float* bev, int gridBlocks, cudaStream_t s) {
    cudaError_t e = cudaFuncSetAttribute(superpose_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(kSmemBytes));
    if (e != cudaSuccess) return e;
    superpose_kernel<<<gridBlocks, kThreads, kSmemBytes, s>>>(g, idd, rsigma, work, beam, bev);
    return cudaGetLastError();
}

}  // namespace pbs
