// Per-layer integrated depth dose and effective sigma along every ray, fused with the
// per-tile radius reduction, and the device-side radius histogram / batching that
// turns the tile codes into a radius-sorted superposition work list.
#include <float.h>
#include <limits.h>

#include "device_util.cuh"
#include "kernels.h"

namespace pbs {

namespace {

constexpr float kPInv = 0.5649718f;   // 1/p, p = 1.77 (raytracedicom_integration.h:22)
constexpr float kECoef = 8.639415f;   // (10 alpha)^(-1/p) (raytracedicom_integration.h:23)
constexpr float kSqrt2 = 1.41421356f;
constexpr float kERefSq = 198.81f;    // 14.1^2
constexpr float kSigmaDelta = 0.21f;
constexpr int kMaxChunkLayers = 64;

// One CTA = one 32x8 tile of rays for one layer. Each thread walks its ray from the
// beam's first-inside step to the layer's cut-off step; after every step the CTA
// reduces min(rSigmaEff) and any(idd > 0) over the tile and stores the radius bucket.
__global__ void __launch_bounds__(256)
idd_kernel(BeamGeomDev g, LutsDev luts, int layer0, const float* __restrict__ density,
           const float* __restrict__ wepl, const int* __restrict__ firstInside, const int* __restrict__ firstOutside,
           const float* __restrict__ rayW, const LayerParamsDev* __restrict__ lp, LayerStateDev* __restrict__ ls,
           const BeamStateDev* __restrict__ beam, float* __restrict__ iddOut, float* __restrict__ rsigOut,
           uint8_t* __restrict__ codes, int* __restrict__ firstPassiveOut) {
    extern __shared__ float ciddRow[];
    __shared__ float shMin[2][8];
    __shared__ int shLive[2][8];
    __shared__ int shPassive[8];

    const int lc = blockIdx.z;
    const int l = layer0 + lc;
    const int tx = blockIdx.x, ty = blockIdx.y;
    const int lane = threadIdx.x, warp = threadIdx.y;
    const int tid = warp * 32 + lane;
    const int x = tx * kTileX + lane, y = ty * kTileY + warp;
    const LayerParamsDev p = lp[l];
    const int first = beam->firstInside;
    const int afterLastL = ls[l].afterLast;

    // CIDD row of this layer's energy: the bilinear CIDD texture lookup at a fixed
    // energy coordinate is a depth lerp of the energy-interpolated row.
    {
        float eb = p.energyIdx;  // (energyIdx + 0.5) - 0.5 texel offset
        eb = fminf(fmaxf(eb, -1.0f), float(luts.nE));
        const float fl = floorf(eb);
        const float b = eb - fl;
        const int e0 = min(max(int(fl), 0), luts.nE - 1);
        const int e1 = min(max(int(fl) + 1, 0), luts.nE - 1);
        const float* r0 = luts.cidd + static_cast<size_t>(e0) * luts.nS;
        const float* r1 = luts.cidd + static_cast<size_t>(e1) * luts.nS;
        for (int d = tid; d < luts.nS; d += 256) {
            const float a0 = __ldg(r0 + d), a1 = __ldg(r1 + d);
            ciddRow[d] = a0 + (a1 - a0) * b;
        }
    }
    __syncthreads();

    const bool real = x < g.rayX && y < g.rayY;
    const size_t rayPlane = static_cast<size_t>(g.rayX) * g.rayY;
    const size_t padPlane = static_cast<size_t>(g.pitchX) * g.pitchY;
    const size_t layerStride = static_cast<size_t>(g.steps) * padPlane;
    float* iddL = iddOut + lc * layerStride;
    float* rsL = rsigOut + lc * layerStride;
    uint8_t* codeL = codes + static_cast<size_t>(lc) * g.steps * g.tilesX * g.tilesY;
    const size_t ridx = static_cast<size_t>(y) * g.rayX + x;

    int firstIn = 0;
    unsigned int afterLast = 0;
    float rayWeight = 0.0f;
    bool live = false;
    if (real) {
        firstIn = firstInside[ridx];
        afterLast = static_cast<unsigned int>(min(firstOutside[ridx], afterLastL));
        rayWeight = rayW[static_cast<size_t>(l) * rayPlane + ridx];
        live = true;
        if (rayWeight < 1e-6f || afterLast < static_cast<unsigned int>(first)) {
            live = false;
            afterLast = 0;
        }
    }

    const float stepLength = fabsf(g.fanDelta.z);
    const float quad = p.sigmaSqAirQuad;
    float cumulSpOld = 0.0f, cumulDoseOld = 0.0f;
    float incScat = 0.0f, incincScat = 0.0f;
    float incDiv = p.sigmaSqAirLin + (2.0f * float(first) - 1.0f) * quad;
    float sigmaSq = -incDiv;

    int buf = 0;
    for (int stepNo = first; stepNo < afterLastL; ++stepNo) {
        float res = 0.0f;
        float rSigmaEff = __int_as_float(0x7f800000);
        if (live) {
            const size_t idx = static_cast<size_t>(stepNo) * rayPlane + ridx;
            const float cumulSp = wepl[idx];
            const float cumulDose = lut_linear_clamp_smem(ciddRow, luts.nS, cumulSp * p.energyScaleFact + 0.5f);
            const float dens = density[idx];
            if (cumulSp < p.peakDepth) {
                const float resE = kECoef * powf(p.peakDepth - 0.5f * (cumulSp + cumulSpOld), kPInv);
                const float betaP = resE + 938.3f - 938.3f * 938.3f / (resE + 938.3f);
                const float rRl = dens * lut_linear_clamp(luts.rrl, luts.nRrl, dens * luts.rrlScale + 0.5f);
                const float thetaSq = kERefSq / (betaP * betaP) * stepLength * rRl;
                sigmaSq += incScat + incDiv;
                incincScat += 2.0f * thetaSq * stepLength * stepLength;
                incScat += incincScat;
                incDiv += 2.0f * quad;
            } else {
                sigmaSq -= 1.5f * (incScat + incDiv) * dens;
            }
            const float zk = g.fanCorner.z + float(stepNo) * g.fanDelta.z;
            const float vwx = g.fanDelta.x * (1.0f - zk / g.sourceDist.x);
            const float vwy = g.fanDelta.y * (1.0f - zk / g.sourceDist.y);
            rSigmaEff = 0.5f * (vwx + vwy) / (kSqrt2 * (sqrtf(sigmaSq) + kSigmaDelta));
            const unsigned int k = static_cast<unsigned int>(stepNo);
            const float stepVol = g.volConst + float(k) * g.volLin + float(k * k) * g.volSq;
            const float mass = dens * stepVol;
            if (mass > 1e-2f) res = rayWeight * (cumulDose - cumulDoseOld) / mass;
            cumulSpOld = cumulSp;
            cumulDoseOld = cumulDose;
            if (cumulSp > p.rangeStopDepth || static_cast<unsigned int>(stepNo) == afterLast) {
                live = false;
                afterLast = static_cast<unsigned int>(stepNo);
            }
        }
        if (!live || stepNo < firstIn - 1) {
            res = 0.0f;
            rSigmaEff = __int_as_float(0x7f800000);
        }
        const size_t o = static_cast<size_t>(stepNo - first) * padPlane + static_cast<size_t>(y) * g.pitchX + x;
        iddL[o] = res;
        rsL[o] = rSigmaEff;

        // Tile reduction: min rSigmaEff and whether any ray deposits.
        float m = rSigmaEff;
        for (int off = 16; off > 0; off >>= 1) m = fminf(m, __shfl_xor_sync(0xffffffffu, m, off));
        const int anyLive = __any_sync(0xffffffffu, res > 0.0f);
        if (lane == 0) {
            shMin[buf][warp] = m;
            shLive[buf][warp] = anyLive;
        }
        __syncthreads();
        if (tid == 0) {
            float tm = shMin[buf][0];
            int tl = shLive[buf][0];
            for (int w = 1; w < 8; ++w) {
                tm = fminf(tm, shMin[buf][w]);
                tl |= shLive[buf][w];
            }
            const int R = tile_radius_bucket(tm);
            codeL[static_cast<size_t>(stepNo - first) * g.tilesX * g.tilesY + ty * g.tilesX + tx] =
                static_cast<uint8_t>(R | (tl ? 0x80 : 0));
        }
        buf ^= 1;
    }

    int fp = real ? static_cast<int>(afterLast) : INT_MIN;
    if (real && firstPassiveOut) firstPassiveOut[static_cast<size_t>(lc) * rayPlane + ridx] = fp;
    for (int off = 16; off > 0; off >>= 1) fp = max(fp, __shfl_xor_sync(0xffffffffu, fp, off));
    if (lane == 0) shPassive[warp] = fp;
    __syncthreads();
    if (tid == 0) {
        int v = shPassive[0];
        for (int w = 1; w < 8; ++w) v = max(v, shPassive[w]);
        if (v != INT_MIN) atomicMax(&ls[l].maxFirstPassive, v);
    }
}

// Single CTA per layer chunk. Per layer: passive step clamp (wrapper.cu:4975-4990),
// radius histogram over [first, calcPassive), overflow merge into R=32
// (complete_superposition.cu:412-460), batching of sparse buckets into the next
// larger radius (complete_superposition.cu:476-483). Then a radius-descending work
// list of the live tiles for the whole chunk.
__global__ void __launch_bounds__(1024)
bin_plan_kernel(BeamGeomDev g, int layer0, int nLayers, const uint8_t* __restrict__ codes,
                LayerStateDev* __restrict__ ls, BeamStateDev* __restrict__ beam, int4* __restrict__ work,
                int workCapacity) {
    __shared__ int hist[kBuckets];
    __shared__ int mapR[kMaxChunkLayers][kBuckets];
    __shared__ int zCount[kMaxChunkLayers];
    __shared__ int countR[kMaxR + 1];
    __shared__ int offR[kMaxR + 1];
    __shared__ int liveL[kMaxChunkLayers];
    const int tid = threadIdx.x;
    const int first = beam->firstInside;
    const int tiles = g.tilesX * g.tilesY;

    if (tid <= kMaxR) countR[tid] = 0;
    for (int lc = 0; lc < nLayers; ++lc) {
        const int l = layer0 + lc;
        if (tid < kBuckets) hist[tid] = 0;
        if (tid == 0) {
            int calc = ls[l].maxFirstPassive;
            if (calc < first + 1) calc = first + 1;
            if (calc < 0) calc = first + 1;
            if (calc > ls[l].afterLast) calc = ls[l].afterLast;
            if (calc > g.steps) calc = g.steps;
            ls[l].calcPassive = calc;
            zCount[lc] = max(calc - first, 0);
            liveL[lc] = 0;
        }
        __syncthreads();
        const uint8_t* cl = codes + static_cast<size_t>(lc) * g.steps * tiles;
        const int n = zCount[lc] * tiles;
        for (int i = tid; i < n; i += blockDim.x) atomicAdd(&hist[cl[i] & 0x3f], 1);
        __syncthreads();
        if (tid == 0) {
            for (int i = 0; i < kBuckets; ++i) ls[l].hist[i] = hist[i];
            if (hist[kMaxR + 1] > 0) {
                hist[kMaxR] += hist[kMaxR + 1];
                hist[kMaxR + 1] = 0;
            }
            int layerMax = 0;
            for (int i = 0; i < kBuckets; ++i)
                if (hist[i] > 0) layerMax = i;
            int batched[kMaxR + 1];
            for (int i = 0; i <= kMaxR; ++i) batched[i] = 0;
            batched[0] = hist[0];
            mapR[lc][0] = 0;
            int recRad = layerMax;
            for (int rad = layerMax; rad > 0; --rad) {
                mapR[lc][rad] = recRad;
                batched[recRad] += hist[rad];
                if (batched[recRad] >= kMinTilesInBatch) recRad = rad - 1;
            }
            for (int rad = layerMax + 1; rad <= kMaxR; ++rad) mapR[lc][rad] = rad;
            mapR[lc][kMaxR + 1] = mapR[lc][kMaxR];
            for (int i = 0; i <= kMaxR; ++i) ls[l].batchedCounts[i] = batched[i];
            for (int i = 0; i < kBuckets; ++i) ls[l].batchedR[i] = mapR[lc][i];
        }
        __syncthreads();
        for (int i = tid; i < n; i += blockDim.x) {
            const int c = cl[i];
            if (c & 0x80) {
                atomicAdd(&countR[mapR[lc][c & 0x3f]], 1);
                atomicAdd(&liveL[lc], 1);
            }
        }
        __syncthreads();
    }
    if (tid == 0) {
        int acc = 0;
        long long fma = 0;
        for (int r = kMaxR; r >= 0; --r) {
            offR[r] = acc;
            acc += countR[r];
            fma += static_cast<long long>(countR[r]) * 256 * (2 * r + 1) * (2 * r + 1);
        }
        int total = acc;
        if (total > workCapacity) {
            atomicOr(&beam->errorFlags, 1);
            total = workCapacity;
        }
        beam->workCount = total;
        beam->workNext = 0;
        beam->liveTiles += acc;
        beam->superposeFma += fma;
        int mp = beam->maxCalcPassive;
        for (int lc = 0; lc < nLayers; ++lc) {
            ls[layer0 + lc].liveTiles = liveL[lc];
            mp = max(mp, ls[layer0 + lc].calcPassive);
        }
        beam->maxCalcPassive = mp;
    }
    __syncthreads();
    for (int lc = 0; lc < nLayers; ++lc) {
        const uint8_t* cl = codes + static_cast<size_t>(lc) * g.steps * tiles;
        const int n = zCount[lc] * tiles;
        for (int i = tid; i < n; i += blockDim.x) {
            const int c = cl[i];
            if (c & 0x80) {
                const int R = mapR[lc][c & 0x3f];
                const int slot = atomicAdd(&offR[R], 1);
                if (slot < workCapacity) work[slot] = make_int4(lc, i % tiles, i / tiles, R);
            }
        }
    }
}

}  // namespace

cudaError_t launch_idd(const BeamGeomDev& g, const LutsDev& luts, int layer0, int nLayers, const float* density,
                       const float* wepl, const int* firstInside, const int* firstOutside, const float* rayW,
                       const LayerParamsDev* lp, LayerStateDev* ls, const BeamStateDev* beam, float* idd,
                       float* rsigma, uint8_t* codes, int* firstPassive, cudaStream_t s) {
    dim3 grid(g.tilesX, g.tilesY, nLayers);
    dim3 block(32, 8);
    const size_t smem = static_cast<size_t>(luts.nS) * sizeof(float);
    idd_kernel<<<grid, block, smem, s>>>(g, luts, layer0, density, wepl, firstInside, firstOutside, rayW, lp, ls, beam,
                                         idd, rsigma, codes, firstPassive);
    return cudaGetLastError();
}

cudaError_t launch_bin_plan(const BeamGeomDev& g, int layer0, int nLayers, const uint8_t* codes, LayerStateDev* ls,
                            BeamStateDev* beam, int4* work, int workCapacity, cudaStream_t s) {
    if (nLayers > kMaxChunkLayers) return cudaErrorInvalidValue;
    bin_plan_kernel<<<1, 1024, 0, s>>>(g, layer0, nLayers, codes, ls, beam, work, workCapacity);
    return cudaGetLastError();
}

}  // namespace pbs
