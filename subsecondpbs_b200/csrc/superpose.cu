// Tile-based Gaussian superposition of the per-ray IDD into the padded BEV dose.
//
// Work items come from the radius-sorted list built on the device; each item is one
// 32x8 tile of rays at one step of one layer with its batched radius R. A CTA
// builds the separable erf-difference weights of its 256 source rays in shared
// memory, then every thread gathers whole output pixels of the (8+2R) x (32+2R)
// footprint from the sources in reach and adds the pixel to the BEV dose of that
// step. All layers of the beam accumulate into the same BEV volume.
#include "kernels.h"

namespace pbs {

namespace {

constexpr int kSuperpThreads = 256;
constexpr int kTabStride = kMaxR + 1;  // erf-difference entries per source

__global__ void __launch_bounds__(kSuperpThreads)
superpose_kernel(BeamGeomDev g, const float* __restrict__ idd, const float* __restrict__ rsig,
                 const int4* __restrict__ work, const BeamStateDev* __restrict__ beam, float* __restrict__ bev) {
    extern __shared__ float sm[];
    float* E = sm;                                   // [256][kTabStride]  e_s(d)
    float* W = sm + kSuperpThreads * kTabStride;     // [256][kTabStride]  idd_s * e_s(d)

    const int count = beam->workCount;
    const int t = threadIdx.x;
    const size_t padPlane = static_cast<size_t>(g.pitchX) * g.pitchY;
    const size_t layerStride = static_cast<size_t>(g.steps) * padPlane;
    const size_t bevPlane = static_cast<size_t>(g.bevX) * g.bevY;

    for (int w = blockIdx.x; w < count; w += gridDim.x) {
        const int4 it = work[w];
        const int lc = it.x, tile = it.y, zRel = it.z, R = it.w;
        const int tx = tile % g.tilesX, ty = tile / g.tilesX;
        const int sy = t >> 5, sx = t & 31;
        const size_t src = lc * layerStride + zRel * padPlane + static_cast<size_t>(ty * kTileY + sy) * g.pitchX +
                           tx * kTileX + sx;
        const float dose = idd[src];
        const float rs = rsig[src];
        // erfDiffs of kernelSuperposition (complete_superposition.cu:298-307).
        {
            float erfNew = erff(rs * 0.5f);
            float erfOld = -erfNew;
            float* e = E + t * kTabStride;
            float* wv = W + t * kTabStride;
            for (int i = 0; i <= R; ++i) {
                const float d = 0.5f * (erfNew - erfOld);
                e[i] = d;
                wv[i] = dose * d;
                erfOld = erfNew;
                erfNew = erff(rs * (float(i) + 1.5f));
            }
        }
        __syncthreads();

        const int oh = kTileY + 2 * R, ow = kTileX + 2 * R;
        const int span = 2 * R;
        float* out = bev + static_cast<size_t>(zRel) * bevPlane + static_cast<size_t>(ty * kTileY - R + kMaxR) * g.bevX +
                     (tx * kTileX - R + kMaxR);
        for (int o = t; o < oh * ow; o += kSuperpThreads) {
            const int oy = o / ow, ox = o - oy * ow;
            const int syLo = max(0, oy - span), syHi = min(kTileY - 1, oy);
            const int sxLo = max(0, ox - span), sxHi = min(kTileX - 1, ox);
            float acc = 0.0f;
            for (int qy = syLo; qy <= syHi; ++qy) {
                const int dy = abs(oy - R - qy);
                const float* wrow = W + (qy * kTileX) * kTabStride + dy;
                const float* erow = E + (qy * kTileX) * kTabStride;
                for (int qx = sxLo; qx <= sxHi; ++qx) {
                    const int dx = abs(ox - R - qx);
                    acc += wrow[qx * kTabStride] * erow[qx * kTabStride + dx];
                }
            }
            if (acc != 0.0f) atomicAdd(out + static_cast<size_t>(oy) * g.bevX + ox, acc);
        }
        __syncthreads();
    }
}

}  // namespace

cudaError_t launch_superpose(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                             const BeamStateDev* beam, float* bev, int gridBlocks, cudaStream_t s) {
    const size_t smem = 2ull * kSuperpThreads * kTabStride * sizeof(float);
    cudaError_t e = cudaFuncSetAttribute(superpose_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         static_cast<int>(smem));
    if (e != cudaSuccess) return e;
    superpose_kernel<<<gridBlocks, kSuperpThreads, smem, s>>>(g, idd, rsigma, work, beam, bev);
    return cudaGetLastError();
}

}  // namespace pbs
