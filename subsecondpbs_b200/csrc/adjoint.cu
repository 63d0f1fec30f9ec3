// Adjoint of the dose with respect to the beam's ray weights: the transposes of
// the BEV -> dose transfer and of the tile superposition, followed by the IDD
// scaling. Dose is linear in the spot weights: for a live ray
//   idd[l][k][ray] = rayW[l][ray] * g[l][k][ray]      (idd_sigma.cu:194-201),
//   BEV = S(idd)  (tile superposition, complete_superposition.cu:264-335),
//   D  += T(BEV)  (divergent trilinear transfer, prim_transf_kernel.cu:11-44),
// so for a dose gradient Gd the ray-weight gradient is
//   rbar[l][ray] = sum_k g[l][k][ray] * (S^T T^T Gd)[l][k][ray]
//               = (sum_k idd[l][k][ray] * (S^T T^T Gd)[l][k][ray]) / rayW[l][ray].
// The tile radii, the live-ray mask and rSigmaEff do not depend on the weights'
// values, so they come from the same IDD and binning kernels as the forward pass.
#include <algorithm>

#include "device_util.cuh"
#include "work_blocks.cuh"
#include "kernels.h"
#include "launch_util.h"

namespace pbs {

namespace {

// T^T: every dose voxel of the transfer box spreads its gradient over the eight
// BEV texels its forward sample interpolated (bev_sample in transfer.cu), with the
// same weights. The forward adds a sample only where it is positive; a BEV sample
// is a sum of non-negative terms, so it is zero only where every texel's
// coefficient is zero and the linear transpose is exact.
// Items of one dose column and 8 consecutive z, x fastest, strided over by a
// persistent grid (the box is known only on the device; see transfer_kernel).
__global__ void __launch_bounds__(256)
transfer_adjoint_kernel(BeamGeomDev g, const double* __restrict__ gradDose, const BeamStateDev* __restrict__ beam,
                        float* __restrict__ gradBev) {
    if (!beam->transferValid) return;
    const int sx = beam->transferStart[0], sy = beam->transferStart[1], sz = beam->transferStart[2];
    const int mx = beam->transferMax[0], my = beam->transferMax[1], mz = beam->transferMax[2];
    const int nxCols = min(((mx - sx + 1 + 31) / 32) * 32, g.doseX - sx);
    const int nyCols = min(((my - sy + 1 + 7) / 8) * 8, g.doseY - sy);
    const int nzc = (mz - sz + 8) / 8;
    if (nxCols <= 0 || nyCols <= 0 || nzc <= 0) return;
    const long long items = static_cast<long long>(nxCols) * nyCols * nzc;
    const TransferParams T = beam->transfer;
    const float zShift = g.compatBevZShift ? float(beam->firstInside) : 0.0f;
    const size_t slice = static_cast<size_t>(g.doseX) * g.doseY;
    const int nx = g.bevX, ny = g.bevY, nz = g.steps;
    for (long long it = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; it < items;
         it += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = sx + static_cast<int>(it % nxCols);
        const long long r = it / nxCols;
        const int y = sy + static_cast<int>(r % nyCols);
        const int z0 = sz + static_cast<int>(r / nyCols) * 8;
        const int z1 = min(mz, z0 + 7);
        const V3 start = transfer_start(T, x, y);
        for (int z = z0; z <= z1; ++z) {
            const V3 f = transfer_fan_idx(T, start, z);
            if (f.x + 0.5f < 0.0f || f.y + 0.5f < 0.0f || f.z + 0.5f < 0.0f) continue;
            const float gd = float(gradDose[static_cast<size_t>(z) * slice + static_cast<size_t>(y) * g.doseX + x]);
            if (gd == 0.0f) continue;
            const float px = fminf(fmaxf(f.x, -2.0f), float(nx) + 1.0f);
            const float py = fminf(fmaxf(f.y, -2.0f), float(ny) + 1.0f);
            const float pz = fminf(fmaxf(f.z - zShift, -2.0f), float(nz) + 1.0f);
            const float fx = floorf(px), fy = floorf(py), fz = floorf(pz);
            const int x0 = int(fx), y0 = int(fy), z0i = int(fz);
            const float tx = px - fx, ty = py - fy, tz = pz - fz;
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const int xi = x0 + (c & 1), yi = y0 + ((c >> 1) & 1), zi = z0i + (c >> 2);
                if (xi < 0 || yi < 0 || zi < 0 || xi >= nx || yi >= ny || zi >= nz) continue;
                const float w =
                    ((c & 1) ? tx : 1.0f - tx) * (((c >> 1) & 1) ? ty : 1.0f - ty) * ((c >> 2) ? tz : 1.0f - tz);
                atomicAdd(gradBev + (static_cast<size_t>(zi) * ny + yi) * nx + xi, w * gd);
            }
        }
    }
}

constexpr int kAdjThreads = 256;
constexpr int kAdjOutFloats = (kTileY + 2 * kMaxR) * (kTileX + 2 * kMaxR);

// S^T for one tile at radius R: each source gathers the BEV gradient over its
// footprint with the forward's weights e(|dy|) e(|dx|) and adds idd * that sum to
// its ray's accumulator.
constexpr int kAdjEStride = kMaxR + 1;  // 33: odd, the threads' rows fall in distinct banks

template <int R>
__device__ __forceinline__ void superpose_adjoint_tile(const float* __restrict__ tileG, float* __restrict__ eRow,
                                                       float dose, float rs, float* __restrict__ rbarRay, int sy,
                                                       int sx) {
    constexpr int Wo = kTileX + 2 * R;
    float e[R + 1];
    superposition_row<R>(rs, e);
#pragma unroll
    for (int k = 0; k <= R; ++k) eRow[k] = e[k];
    // Rows R-k and R+k share the weight e[k]; within a row the columns R-j and
    // R+j share e[j] (kept in registers; the row weight comes from eRow).
    auto row_sum = [&](int i) {
        const float* row = tileG + (sy + i) * Wo + sx + R;
        float v = e[0] * row[0];
#pragma unroll
        for (int j = 1; j <= R; ++j) v = fmaf(e[j], row[-j] + row[j], v);
        return v;
    };
    float acc = e[0] * row_sum(R);
#pragma unroll 1
    for (int k = 1; k <= R; ++k) acc = fmaf(eRow[k], row_sum(R - k) + row_sum(R + k), acc);
    atomicAdd(rbarRay, dose * acc);
}

// S^T for one tile at radius R <= kSplitR, in the forward's (source column, |d|)
// pair form. A source's gradient is
//   sum_d e(d) P_d,  P_d = sum_k e(|k|) c_d[sy + R + k],
// where c_d is the sum of the footprint's gradient columns sx + R + d and
// sx + R - d (one column for d = 0), the same for the eight sources of the column.
// A lane is one (column, |d|) pair: it sums its two gradient columns once into
// registers, then forms P_d for the column's eight sources with their weights read
// as broadcast float4 chunks, and stores them; each source thread then sums
// e(d) P_d over d. The shared-memory reads per source drop from (2R+1)^2 scalars
// to about (2H + 8 Q)/8 per pair.
template <int R>
__device__ __forceinline__ void superpose_adjoint_pairs(const float* __restrict__ tileG, float4* __restrict__ E4,
                                                        float* __restrict__ P, float dose, float rs,
                                                        float* __restrict__ rbarRay) {
    constexpr int H = kTileY + 2 * R;
    constexpr int Wo = kTileX + 2 * R;
    constexpr int Q = (R + 1 + 3) / 4;
    constexpr int PS = (R + 1) | 1;             // odd row stride of P
    constexpr int M = R + 1;
    constexpr int G = 32 / M;                   // source columns per warp instruction
    constexpr int S = (32 + G - 1) / G;         // column spacing, units
    const int t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31;
    const bool live = rbarRay != nullptr;
    // Weights of source t = (sy, sx) = (warp, lane), chunk-major with the column
    // swizzle of the forward kernel.
    float e[4 * Q];
    if (live) {
        float row[R + 1];
        superposition_row<R>(rs, row);
#pragma unroll
        for (int k = 0; k <= R; ++k) e[k] = row[k];
    } else {
#pragma unroll
        for (int k = 0; k <= R; ++k) e[k] = 0.0f;
    }
#pragma unroll
    for (int k = R + 1; k < 4 * Q; ++k) e[k] = 0.0f;
    const int col = lane ^ ((lane >> 3) & 3);
#pragma unroll
    for (int q = 0; q < Q; ++q)
        E4[q * kAdjThreads + warp * kTileX + col] = make_float4(e[4 * q], e[4 * q + 1], e[4 * q + 2], e[4 * q + 3]);
    __syncthreads();
#pragma unroll 1
    for (int u = warp; u < S; u += kAdjThreads / 32) {
        const int g = lane / M;
        int d = lane - g * M;
        int sx = u + g * S;
        const bool valid = g < G && sx < kTileX;
        if (!valid) {
            sx = 0;
            d = 0;
        }
        float c[H];
        const float* ca = tileG + sx + R + d;
        const float* cb = tileG + sx + R - d;
#pragma unroll
        for (int i = 0; i < H; ++i) c[i] = ca[i * Wo] + (d > 0 ? cb[i * Wo] : 0.0f);
        const float4* eCol = E4 + (sx ^ ((sx >> 3) & 3));
#pragma unroll
        for (int sy = 0; sy < kTileY; ++sy) {
            float ev[4 * Q];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const float4 v = eCol[q * kAdjThreads + sy * kTileX];
                ev[4 * q] = v.x;
                ev[4 * q + 1] = v.y;
                ev[4 * q + 2] = v.z;
                ev[4 * q + 3] = v.w;
            }
            float pd = ev[0] * c[sy + R];
#pragma unroll
            for (int k = 1; k <= R; ++k) pd = fmaf(ev[k], c[sy + R - k] + c[sy + R + k], pd);
            if (valid) P[(sy * kTileX + sx) * PS + d] = pd;
        }
    }
    __syncthreads();
    if (live) {
        float acc = 0.0f;
#pragma unroll
        for (int k = 0; k <= R; ++k) acc = fmaf(e[k], P[t * PS + k], acc);
        atomicAdd(rbarRay, dose * acc);
    }
}

// Radii above kSplitR gather per source (superpose_adjoint_tile); the others run
// in pair form with every thread of the CTA (rbarRay null: no live source).
template <int R, int RHi>
__device__ __forceinline__ void adjoint_dispatch(int r, const float* tileG, float* eRow, float4* E4, float* P,
                                                 float dose, float rs, float* rbarRay, int sy, int sx) {
    if (r == R) {
        if constexpr (R <= kSplitR) {
            superpose_adjoint_pairs<R>(tileG, E4, P, dose, rs, rbarRay);
        } else {
            if (rbarRay) superpose_adjoint_tile<R>(tileG, eRow, dose, rs, rbarRay, sy, sx);
        }
        return;
    }
    if constexpr (R < RHi) adjoint_dispatch<R + 1, RHi>(r, tileG, eRow, E4, P, dose, rs, rbarRay, sy, sx);
}

// Shared memory of an instance for radii up to RHi: the tile's gradient footprint,
// then either the pair form's weight chunks and pair sums (RHi <= kSplitR) or each
// source's weight row.
template <int RHi>
struct AdjShape {
    static constexpr int kTile = (kTileY + 2 * RHi) * (kTileX + 2 * RHi);  // 16(4+R)(16+R) bytes: 16-byte aligned
    static constexpr bool kPairs = RHi <= kSplitR;
    static constexpr int kQ = (RHi + 1 + 3) / 4;
    static constexpr int kPS = (RHi + 1) | 1;
    static constexpr int kRest = kPairs ? kQ * kAdjThreads * 4 + kAdjThreads * kPS : kAdjThreads * kAdjEStride;
    static constexpr size_t kSmemBytes = size_t(kTile + kRest) * sizeof(float);
};

// Persistent CTAs over the radii RLo..RHi of the chunk's one-layer work list, taken
// radius block by radius block through the range's counter as in the forward
// superposition. The three instances of a beam overlap in the same way: each CTA
// lets the next instance launch at once (their items only add into the rays'
// accumulators) and waits for the previous instance before it exits.
template <int RLo, int RHi, int MinBlocks>
__global__ void __launch_bounds__(kAdjThreads, MinBlocks)
superpose_adjoint_kernel(BeamGeomDev g, const float* __restrict__ idd, const float* __restrict__ rsig,
                         const int4* __restrict__ work, BeamStateDev* __restrict__ beam, const float* __restrict__ gradBev,
                         float* __restrict__ rbar, int range) {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    extern __shared__ __align__(16) float adjSm[];
    using Sh = AdjShape<RHi>;
    float* tileG = adjSm;                        // [8+2R][32+2R] BEV gradient of the tile's footprint
    float* eS = adjSm + Sh::kTile;               // [256][kAdjEStride] each source's weights (R > kSplitR)
    float4* E4 = reinterpret_cast<float4*>(eS);  // pair form: weight chunks [Q][256] ...
    float* P = eS + Sh::kQ * kAdjThreads * 4;    // ... and pair sums [256][PS]
    __shared__ int sItem[2];
    __shared__ RadiusBlocks<RLo, RHi> sBlocks;
    const int t = threadIdx.x;
    int* counter = range == 0 ? &beam->workNext : (range == 1 ? &beam->workNextSmall : &beam->workNextTiny);
    const size_t padPlane = static_cast<size_t>(g.pitchX) * g.pitchY;
    const size_t layerStride = static_cast<size_t>(g.steps) * padPlane;
    const size_t bevPlane = static_cast<size_t>(g.bevX) * g.bevY;
    const size_t rayPlane = static_cast<size_t>(g.rayX) * g.rayY;
    load_blocks<RLo, RHi>(beam, sBlocks);
    if (t == 0) sItem[0] = atomicAdd(counter, 1);
    __syncthreads();
    int buf = 0;
    for (;;) {
        const int c = sItem[buf];
        if (c >= sBlocks.total) break;
        if (t == 0) sItem[buf ^ 1] = atomicAdd(counter, 1);
        const int4 it = work[block_slot<RLo, RHi>(sBlocks, c)];
        const int lc = it.x & 0xff, tile = it.y, zRel = it.z, R = it.w;
        const int tx = tile % g.tilesX, ty = tile / g.tilesX;
        const int Ho = kTileY + 2 * R, Wo = kTileX + 2 * R;
        const float* src = gradBev + static_cast<size_t>(zRel) * bevPlane +
                           static_cast<size_t>(ty * kTileY - R + kMaxR) * g.bevX + (tx * kTileX - R + kMaxR);
        for (int i = t; i < Ho * Wo; i += kAdjThreads) {
            const int oy = i / Wo, ox = i - oy * Wo;
            tileG[i] = src[static_cast<size_t>(oy) * g.bevX + ox];
        }
        __syncthreads();
        const int sy = t >> 5, sx = t & 31;
        const int ry = ty * kTileY + sy, rx = tx * kTileX + sx;
        const size_t s = lc * layerStride + zRel * padPlane + static_cast<size_t>(ry) * g.pitchX + rx;
        const float dose = idd[s];
        const bool live = dose > 0.0f && ry < g.rayY && rx < g.rayX;
        if (R >= RLo && R <= RHi)
            adjoint_dispatch<RLo, RHi>(R, tileG, eS + t * kAdjEStride, E4, P, dose, live ? rsig[s] : 0.0f,
                                       live ? rbar + lc * rayPlane + static_cast<size_t>(ry) * g.rayX + rx : nullptr,
                                       sy, sx);
        // Every thread is past the item (and has read sItem[buf]) before the next
        // claim lands in that slot.
        __syncthreads();
        buf ^= 1;
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <int RLo, int RHi, int MinBlocks>
cudaError_t launch_adjoint_range(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                                 BeamStateDev* beam, const float* gradBev, float* rbar, int numSMs, int range,
                                 bool overlap, cudaStream_t s) {
    auto k = superpose_adjoint_kernel<RLo, RHi, MinBlocks>;
    const size_t smem = AdjShape<RHi>::kSmemBytes;
    cudaError_t e = set_smem_limit(reinterpret_cast<const void*>(k), smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(numSMs * MinBlocks);
    cfg.blockDim = dim3(kAdjThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = overlap ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, g, idd, rsigma, work, beam, gradBev, rbar, range);
}

// Resident CTAs per SM of the adjoint instances (radii 16..32, 8..15, 0..7).
constexpr int kAdjWideBlocks = 3;
constexpr int kAdjMidBlocks = 4;
constexpr int kAdjNarrowBlocks = 6;

}  // namespace

cudaError_t launch_transfer_adjoint(const BeamGeomDev& g, const double* gradDose, const BeamStateDev* beam,
                                    float* gradBev, cudaStream_t s) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long long cap = (static_cast<long long>(g.doseX) * g.doseY * ((g.doseZ + 7) / 8) + 255) / 256;
    const int blocks = static_cast<int>(std::max<long long>(1, std::min<long long>(cap, sms * 8)));
    transfer_adjoint_kernel<<<blocks, 256, 0, s>>>(g, gradDose, beam, gradBev);
    return cudaGetLastError();
}

cudaError_t launch_superpose_adjoint(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                                     BeamStateDev* beam, const float* gradBev, float* rbar, int numSMs,
                                     cudaStream_t s) {
    cudaError_t e = launch_one_layer_list_view(beam, s);
    if (e != cudaSuccess) return e;
    e = launch_adjoint_range<kSplitR + 1, kMaxR, kAdjWideBlocks>(g, idd, rsigma, work, beam, gradBev, rbar, numSMs,
                                                                 0, false, s);
    if (e != cudaSuccess) return e;
    e = launch_adjoint_range<kSplitR2 + 1, kSplitR, kAdjMidBlocks>(g, idd, rsigma, work, beam, gradBev, rbar, numSMs,
                                                                   1, true, s);
    if (e != cudaSuccess) return e;
    return launch_adjoint_range<0, kSplitR2, kAdjNarrowBlocks>(g, idd, rsigma, work, beam, gradBev, rbar, numSMs, 2,
                                                               true, s);
}

}  // namespace pbs
