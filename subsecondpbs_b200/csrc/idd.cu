// Per-layer integrated depth dose and effective sigma along every ray, fused with the
// per-tile radius reduction and the per-layer radius histogram, followed by the
// device-side batching (one small CTA) and the radius-sorted work-list scatter.
#include <float.h>
#include <limits.h>

#include <algorithm>

#include "device_util.cuh"
#include "kernels.h"
#include "launch_util.h"

namespace pbs {

namespace {

constexpr float kPInv = 0.5649718f;   // 1/p, p = 1.77 (raytracedicom_integration.h:22)
constexpr float kECoef = 8.639415f;   // (10 alpha)^(-1/p) (raytracedicom_integration.h:23)
constexpr float kSqrt2 = 1.41421356f;
constexpr int kMaxChunkLayers = 64;

// Divisions in the per-step walk use the approximate reciprocal (__fdividef, within
// 2 ulp): the IEEE quotient's range check and slow path cost more ALU and branch
// issue than the rest of a step's arithmetic. The tile radius bucket keeps its
// IEEE division (tile_radius_bucket).
//
// One CTA = one 32x8 tile of rays for one layer. Each thread walks its ray from the
// beam's first-inside step to the layer's cut-off step (fillIddAndSigmaKernel,
// idd_sigma.cu:46-259). After every step each warp reduces min(rSigmaEff) and
// any(idd > 0) over its 32 rays into shared memory; once the walk is done the CTA
// turns the eight warp partials of every step into the tile's radius bucket
// (tileRadCalc, complete_superposition.cu:198-255), stores the code and adds the
// tile's bucket counts to the layer histogram.
// Profile table value of channel c at a fractional depth and row index, both
// already clamped to the table: the linear filter of the reference's profile
// texture (wrapper.cu:2858-2860, unnormalised coordinates at texel centres) with
// exact weights.
__device__ __forceinline__ float profile_sample(const float* __restrict__ t, int depthN, int channels, int rows,
                                                int c, float depth, float row) {
    const float fd = floorf(depth), fr = floorf(row);
    const int d0 = int(fd), r0 = int(fr);
    const int d1 = min(d0 + 1, depthN - 1), r1 = min(r0 + 1, rows - 1);
    const float ad = depth - fd, ar = row - fr;
    auto at = [&](int r, int d) { return __ldg(t + (static_cast<size_t>(r) * depthN + d) * channels + c); };
    const float a0 = at(r0, d0), a1 = at(r0, d1), b0 = at(r1, d0), b1 = at(r1, d1);
    const float lo = a0 + (a1 - a0) * ad, hi = b0 + (b1 - b0) * ad;
    return lo + (hi - lo) * ar;
}

template <bool kNuclear, bool kProfile>
__global__ void __launch_bounds__(256)
idd_kernel(BeamGeomDev g, LutsDev luts, int layer0, const float* __restrict__ density,
           const float* __restrict__ wepl, const int* __restrict__ firstInside, const int* __restrict__ firstOutside,
           const float* __restrict__ rayW, const LayerParamsDev* __restrict__ lp, LayerStateDev* __restrict__ ls,
           const BeamStateDev* __restrict__ beam, float* __restrict__ iddOut, float* __restrict__ rsigOut,
           uint8_t* __restrict__ codes, int* __restrict__ firstPassiveOut, const int* __restrict__ rayToNuc,
           const float* __restrict__ lattice, float* __restrict__ nucIddOut, float* __restrict__ nucRsOut) {
    extern __shared__ float smem[];
    float* ciddRow = smem;                                    // [nS]
    float* nucWRow = ciddRow + luts.nS;                       // [nS] with the nuclear halo
    float* nucSRow = nucWRow + (kNuclear ? luts.nS : 0);      // [nS] with the nuclear halo
    float* rrlTab = nucSRow + (kNuclear ? luts.nS : 0);       // [nRrl]
    float* stepNum = rrlTab + luts.nRrl;                      // [steps] 0.5 (voxel width x + y)
    float* stepVolT = stepNum + g.steps;                      // [steps] step volume
    float* partMin = stepVolT + g.steps;                      // [steps][8]
    int* partLive = reinterpret_cast<int*>(partMin + g.steps * 8);  // [steps][8]
    __shared__ int shHist[kBuckets], shLive[kBuckets], shPassive[8];

    // Longest walks first: the layers are dispatched from the end of the chunk whose
    // cut-off step is deeper, so that the long CTAs do not form the grid's tail.
    const int nl = int(gridDim.z);
    const bool deepLast = ls[layer0].afterLast < ls[layer0 + nl - 1].afterLast;
    const int lc = deepLast ? nl - 1 - int(blockIdx.z) : int(blockIdx.z);
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
        if (kNuclear) {
            // Nuclear weight and sigma^2 tables share the CIDD axes (energy_reader.cpp:135-182).
            const float* w0 = luts.nucWeight + static_cast<size_t>(e0) * luts.nS;
            const float* w1 = luts.nucWeight + static_cast<size_t>(e1) * luts.nS;
            const float* q0 = luts.nucSqSigma + static_cast<size_t>(e0) * luts.nS;
            const float* q1 = luts.nucSqSigma + static_cast<size_t>(e1) * luts.nS;
            for (int d = tid; d < luts.nS; d += 256) {
                const float a0 = __ldg(w0 + d), a1 = __ldg(w1 + d);
                nucWRow[d] = a0 + (a1 - a0) * b;
                const float c0 = __ldg(q0 + d), c1 = __ldg(q1 + d);
                nucSRow[d] = c0 + (c1 - c0) * b;
            }
        }
        for (int d = tid; d < luts.nRrl; d += 256) rrlTab[d] = __ldg(luts.rrl + d);
        // Per-step voxel widths and volumes are the same for every ray of the step
        // (fill_idd_and_sigma_params.cuh:56-80).
        for (int k = tid; k < g.steps; k += 256) {
            const float zk = g.fanCorner.z + float(k) * g.fanDelta.z;
            const float vwx = g.fanDelta.x * (1.0f - zk / g.sourceDist.x);
            const float vwy = g.fanDelta.y * (1.0f - zk / g.sourceDist.y);
            stepNum[k] = 0.5f * (vwx + vwy);
            const unsigned int ku = static_cast<unsigned int>(k);
            stepVolT[k] = g.volConst + float(ku) * g.volLin + float(ku * ku) * g.volSq;
        }
        if (tid < kBuckets) {
            shHist[tid] = 0;
            shLive[tid] = 0;
        }
    }
    __syncthreads();

    const bool real = x < g.rayX && y < g.rayY;
    const size_t rayPlane = static_cast<size_t>(g.rayX) * g.rayY;
    const size_t padPlane = static_cast<size_t>(g.pitchX) * g.pitchY;
    const size_t layerStride = static_cast<size_t>(g.steps) * padPlane;
    float* iddL = iddOut + lc * layerStride;
    float* rsL = rsigOut + lc * layerStride;
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

    // Nuclear halo of this ray (idd_sigma.cu:88-98, 131-142): only rays under a
    // halo lattice cell carry a halo value; the cell's raw spot weight is its
    // weight. Every ray's primary dose keeps the (1 - nuclear weight) share.
    const bool nucOn = kNuclear && p.spotDist > 0.0f;
    int nucIdx = -1;
    float nucRayWeight = 0.0f;
    if (nucOn && real) {
        nucIdx = rayToNuc[ridx];
        if (nucIdx >= 0)
            nucRayWeight = lattice[(static_cast<size_t>(l) * g.latNy + nucIdx / g.nucX) * g.latNx + nucIdx % g.nucX];
    }
    const size_t nucPlane = static_cast<size_t>(g.nucX) * g.nucY;
    float* nucIddL = nucIddOut + lc * static_cast<size_t>(g.steps) * nucPlane;
    float* nucRsL = nucRsOut + lc * static_cast<size_t>(g.steps) * nucPlane;
    const float spotDist = p.spotDist;
    const float entrySigmaSq = ls[l].entrySigmaSq;
    const float eRefSq = nucOn ? g.eRefSq : 198.81f;
    const float sigmaDelta = nucOn ? g.sigmaDelta : 0.21f;
    const bool suppressDip = nucOn && g.suppressDistalDip;

    const float stepLength = fabsf(g.fanDelta.z);
    const float quad = p.sigmaSqAirQuad;
    float cumulSpOld = 0.0f, cumulDoseOld = 0.0f;
    float incScat = 0.0f, incincScat = 0.0f;
    float incDiv = p.sigmaSqAirLin + (2.0f * float(first) - 1.0f) * quad;
    float sigmaSq = -incDiv;

    // The next step's WEPL and density are loaded one step ahead.
    float nextSp = 0.0f, nextDens = 0.0f;
    if (live && first < afterLastL) {
        const size_t idx = static_cast<size_t>(first) * rayPlane + ridx;
        nextSp = wepl[idx];
        nextDens = density[idx];
    }
    float runMax = 0.0f;  // largest IDD of this ray (fixed-point range of the superposition)
    int stepNo = first;
    for (; stepNo < afterLastL; ++stepNo) {
        // Once no ray of the row is live, every later step is (0, +inf): the fill
        // below writes those without the per-step walk.
        if (!__any_sync(0xffffffffu, live)) break;
        float res = 0.0f;
        float rSigmaEff = __int_as_float(0x7f800000);
        float nucRes = 0.0f;
        float nucRSigmaEff = __int_as_float(0x7f800000);
        // WEPL of this step for the profile model (the reference reads the traced
        // value of every step, live or not).
        const float nextProfileSp = kProfile && real ? wepl[static_cast<size_t>(stepNo) * rayPlane + ridx] : 0.0f;
        if (live) {
            const float cumulSp = nextSp;
            const float dens = nextDens;
            if (stepNo + 1 < afterLastL) {
                const size_t idx = static_cast<size_t>(stepNo + 1) * rayPlane + ridx;
                nextSp = wepl[idx];
                nextDens = density[idx];
            }
            const float cumulDose = lut_linear_clamp_smem(ciddRow, luts.nS, cumulSp * p.energyScaleFact + 0.5f);
            if (cumulSp < p.peakDepth) {
                const float resE = kECoef * __powf(p.peakDepth - 0.5f * (cumulSp + cumulSpOld), kPInv);
                const float betaP = resE + 938.3f - __fdividef(938.3f * 938.3f, resE + 938.3f);
                const float rRl = dens * lut_linear_clamp_smem(rrlTab, luts.nRrl, dens * luts.rrlScale + 0.5f);
                const float thetaSq = __fdividef(eRefSq, betaP * betaP) * stepLength * rRl;
                sigmaSq += incScat + incDiv;
                incincScat += 2.0f * thetaSq * stepLength * stepLength;
                incScat += incincScat;
                incDiv += 2.0f * quad;
            } else if (!suppressDip) {
                sigmaSq -= 1.5f * (incScat + incDiv) * dens;
            }
            rSigmaEff = __fdividef(stepNum[stepNo], kSqrt2 * (sqrtf(sigmaSq) + sigmaDelta));
            const float mass = dens * stepVolT[stepNo];
            if (nucOn) {
                const float depthMidIdx = 0.5f * (cumulSp + cumulSpOld) * p.energyScaleFact + 0.5f;
                if (mass > 1e-2f) {
                    const float nucWeight = lut_linear_clamp_smem(nucWRow, luts.nS, depthMidIdx);
                    res = __fdividef((1.0f - nucWeight) * rayWeight * (cumulDose - cumulDoseOld), mass);
                    if (nucIdx >= 0)
                        nucRes = __fdividef(nucWeight * nucRayWeight * (cumulDose - cumulDoseOld), mass * spotDist * spotDist);
                }
                if (nucIdx >= 0) {
                    const float nucSqSigma = lut_linear_clamp_smem(nucSRow, luts.nS, depthMidIdx);
                    nucRSigmaEff = 0.5f * spotDist * (2.0f * stepNum[stepNo]) /
                                   (kSqrt2 * sqrtf(sigmaSq + nucSqSigma + entrySigmaSq));
                }
            } else if (mass > 1e-2f) {
                res = __fdividef(rayWeight * (cumulDose - cumulDoseOld), mass);
            }
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
            nucRes = 0.0f;
            nucRSigmaEff = __int_as_float(0x7f800000);
        }
        if (kProfile && real) {
            // CarbonPBS lateral profile model on the filled step, in the reference's
            // order: the sigma override (overrideRSigmaFromCarbonProfileKernel,
            // wrapper.cu:2080-2152), then the overall weight
            // (applyCarbonProfileOverallWeightKernel, wrapper.cu:2154-2187).
            const int nGauss = (g.profileChannels - 1) / 2;
            const float depthIdx = (nextProfileSp - g.profileDepth0) / g.profileDepthStep;
            const float dIdx = fminf(fmaxf(depthIdx, 0.0f), float(g.profileDepthN - 1));
            const float rIdx = p.profileRow;
            if (g.profileMode & 1) {
                if (!(res > 0.0f)) {
                    rSigmaEff = __int_as_float(0x7f800000);
                } else {
                    float sumW = 0.0f, sumS2 = 0.0f;
                    for (int gi = 0; gi < nGauss; ++gi) {
                        const float w = profile_sample(g.profile, g.profileDepthN, g.profileChannels, g.profileRows,
                                                       gi, dIdx, rIdx);
                        const float sr = profile_sample(g.profile, g.profileDepthN, g.profileChannels, g.profileRows,
                                                        gi + nGauss, dIdx, rIdx);
                        sumW += w;
                        sumS2 += w * sr * sr;
                    }
                    if (!(sumW > 1.0e-8f)) {
                        rSigmaEff = __int_as_float(0x7f800000);
                    } else {
                        // CarbonPBS geometric depth: distance from the virtual source along
                        // this divergent ray minus the source-to-beam-parameter distance.
                        const float sad = 0.5f * (g.sourceDist.x + g.sourceDist.y);
                        const float fanX = g.fanCorner.x + float(x) * g.fanDelta.x;
                        const float fanY = g.fanCorner.y + float(y) * g.fanDelta.y;
                        const float fanZ = g.fanCorner.z + float(stepNo) * g.fanDelta.z;
                        const float proj = (sad - fanZ) * sqrtf(1.0f + (fanX * fanX) / (g.sourceDist.x * g.sourceDist.x) +
                                                                (fanY * fanY) / (g.sourceDist.y * g.sourceDist.y));
                        const float phy = proj - (sad - g.beamParaPos);
                        const float initR2 = p.bp0 + 2.0f * p.bp1 * phy + p.bp2 * phy * phy;
                        const float axisSq = 0.5f * fmaxf(0.0f, initR2 + sumS2 / sumW);
                        const float axis = sqrtf(fmaxf(0.0f, axisSq));
                        rSigmaEff = 0.5f * stepNum[stepNo] / (kSqrt2 * (axis + 0.21f));
                    }
                }
            }
            if ((g.profileMode & 2) && res > 0.0f) {
                const float ow = profile_sample(g.profile, g.profileDepthN, g.profileChannels, g.profileRows,
                                                g.profileChannels - 1, dIdx, rIdx);
                res *= fmaxf(0.0f, ow);
            }
        }
        runMax = fmaxf(runMax, res);
        const int zr = stepNo - first;
        const size_t o = static_cast<size_t>(zr) * padPlane + static_cast<size_t>(y) * g.pitchX + x;
        iddL[o] = res;
        rsL[o] = rSigmaEff;
        if (nucIdx >= 0) {
            nucIddL[static_cast<size_t>(zr) * nucPlane + nucIdx] = nucRes;
            nucRsL[static_cast<size_t>(zr) * nucPlane + nucIdx] = nucRSigmaEff;
        }

        // Warp minimum on order-preserving unsigned keys of the floats; the device's
        // canonical NaN maps above +inf and drops out, as it does under fminf.
        const unsigned mk = __reduce_min_sync(0xffffffffu, float_order_key(rSigmaEff));
        const int anyLive = __any_sync(0xffffffffu, res > 0.0f);
        if (lane == 0) {
            partMin[zr * 8 + warp] = float_from_order_key(mk);
            partLive[zr * 8 + warp] = anyLive;
        }
    }
    // The row's remaining steps: no dose, rSigmaEff = +inf, nothing live.
    for (int k = stepNo; k < afterLastL; ++k) {
        const int zr = k - first;
        const size_t o = static_cast<size_t>(zr) * padPlane + static_cast<size_t>(y) * g.pitchX + x;
        iddL[o] = 0.0f;
        rsL[o] = __int_as_float(0x7f800000);
        if (nucIdx >= 0) {
            nucIddL[static_cast<size_t>(zr) * nucPlane + nucIdx] = 0.0f;
            nucRsL[static_cast<size_t>(zr) * nucPlane + nucIdx] = __int_as_float(0x7f800000);
        }
    }
    for (int zr = stepNo - first + lane; zr < afterLastL - first; zr += 32) {
        partMin[zr * 8 + warp] = __int_as_float(0x7f800000);
        partLive[zr * 8 + warp] = 0;
    }

    {
        const unsigned mb = __reduce_max_sync(0xffffffffu, __float_as_uint(fmaxf(runMax, 0.0f)));
        if (lane == 0 && mb) atomicMax(&ls[l].maxIddBits, mb);
    }
    int fp = real ? static_cast<int>(afterLast) : INT_MIN;
    if (real && firstPassiveOut) firstPassiveOut[static_cast<size_t>(lc) * rayPlane + ridx] = fp;
    for (int off = 16; off > 0; off >>= 1) fp = max(fp, __shfl_xor_sync(0xffffffffu, fp, off));
    if (lane == 0) shPassive[warp] = fp;
    __syncthreads();

    // Tile codes of every step and the tile's histogram contribution.
    const int nSteps = max(afterLastL - first, 0);
    uint8_t* codeL = codes + static_cast<size_t>(lc) * g.steps * g.tilesX * g.tilesY;
    const int tiles = g.tilesX * g.tilesY;
    for (int zr = tid; zr < nSteps; zr += 256) {
        float tm = partMin[zr * 8];
        int tl = partLive[zr * 8];
#pragma unroll
        for (int w = 1; w < 8; ++w) {
            tm = fminf(tm, partMin[zr * 8 + w]);
            tl |= partLive[zr * 8 + w];
        }
        const int R = tile_radius_bucket(tm);
        codeL[static_cast<size_t>(zr) * tiles + ty * g.tilesX + tx] = static_cast<uint8_t>(R | (tl ? 0x80 : 0));
        atomicAdd(&shHist[R], 1);
        if (tl) atomicAdd(&shLive[R], 1);
    }
    __syncthreads();
    if (tid < kBuckets) {
        if (shHist[tid]) atomicAdd(&ls[l].histAll[tid], shHist[tid]);
        if (shLive[tid]) atomicAdd(&ls[l].liveHist[tid], shLive[tid]);
    }
    if (tid == 0) {
        int v = shPassive[0];
        for (int w = 1; w < 8; ++w) v = max(v, shPassive[w]);
        if (v != INT_MIN) atomicMax(&ls[l].maxFirstPassive, v);
    }
}

// One thread per layer of the chunk: passive step (wrapper.cu:4975-4990), histogram
// over [first, calcPassive) (tiles at steps >= calcPassive hold only dead rays and
// fall in bucket 0), overflow merge into R=32 (complete_superposition.cu:412-460)
// and batching of sparse buckets into the radius above them
// (complete_superposition.cu:476-483). Thread 0 then lays out the chunk's work list
// in descending radius.
//
// With `primaryLs` set the kernel plans the nuclear halo of the chunk instead
// (performNuclearTileBasedSuperposition, complete_superposition.cu:558-708): the
// halo histogram already covers [first, calcPassive) of the primary layer, and a
// radius above 32 is an error (the reference throws) rather than a merge.
__global__ void __launch_bounds__(kMaxChunkLayers)
layer_plan_kernel(BeamGeomDev g, int layer0, int nLayers, LayerStateDev* __restrict__ ls,
                  BeamStateDev* __restrict__ beam, int workCapacity, const LayerStateDev* __restrict__ primaryLs,
                  const BeamStateDev* __restrict__ primaryBeam) {
    __shared__ int sLive[kMaxChunkLayers][kMaxR + 1];   // live items per layer and batched radius
    __shared__ int sCalc[kMaxChunkLayers];
    __shared__ int sWarpSum[kMaxChunkLayers / 32];
    __shared__ long long sWarpFma[kMaxChunkLayers / 32];
    __shared__ int sSplit[2];
    pdl_trigger();
    const int lc = threadIdx.x;
    const bool nuclear = primaryLs != nullptr;
    const int first = nuclear ? primaryBeam->firstInside : beam->firstInside;
    const int tiles = g.tilesX * g.tilesY;
    if (lc < 2) sSplit[lc] = 0;
    if (lc < nLayers) {
        LayerStateDev& st = ls[layer0 + lc];
        // Every input of the layer is read before its outputs are written: the outputs
        // go to the same struct through indexed stores, so a load placed after them
        // would wait for them to complete.
        int hist[kBuckets], liveHist[kBuckets];
        for (int i = 0; i < kBuckets; ++i) {
            hist[i] = st.histAll[i];
            liveHist[i] = st.liveHist[i];
        }
        const int afterLast = st.afterLast;
        const int maxFirstPassive = st.maxFirstPassive;
        int calc;
        if (nuclear) {
            calc = primaryLs[layer0 + lc].calcPassive;
            st.afterLast = calc;
            st.calcPassive = calc;
            if (hist[kMaxR + 1] > 0) atomicOr(&beam->errorFlags, 4);
        } else {
            calc = maxFirstPassive;
            if (calc < first + 1) calc = first + 1;
            if (calc < 0) calc = first + 1;
            if (calc > afterLast) calc = afterLast;
            if (calc > g.steps) calc = g.steps;
            st.calcPassive = calc;
            if (afterLast > calc && afterLast > first) hist[0] -= (afterLast - max(calc, first)) * tiles;
        }
        for (int i = 0; i < kBuckets; ++i) st.hist[i] = hist[i];
        if (hist[kMaxR + 1] > 0) {
            hist[kMaxR] += hist[kMaxR + 1];
            hist[kMaxR + 1] = 0;
        }
        int layerMax = 0;
        for (int i = 0; i < kBuckets; ++i)
            if (hist[i] > 0) layerMax = i;
        int batched[kMaxR + 1];
        int map[kBuckets];
        for (int i = 0; i <= kMaxR; ++i) batched[i] = 0;
        for (int i = 0; i < kBuckets; ++i) map[i] = i;
        batched[0] = hist[0];
        map[0] = 0;
        int recRad = layerMax;
        for (int rad = layerMax; rad > 0; --rad) {
            map[rad] = recRad;
            batched[recRad] += hist[rad];
            if (batched[recRad] >= kMinTilesInBatch) recRad = rad - 1;
        }
        map[kMaxR + 1] = map[kMaxR];
        int live = 0;
        for (int i = 0; i <= kMaxR; ++i) {
            st.batchedCounts[i] = batched[i];
            st.curR[i] = 0;
        }
        int liveR[kMaxR + 1];
        for (int i = 0; i <= kMaxR; ++i) liveR[i] = 0;
        for (int b = 0; b < kBuckets; ++b) {
            st.batchedR[b] = map[b];
            liveR[map[b]] += liveHist[b];
            live += liveHist[b];
        }
        for (int i = 0; i <= kMaxR; ++i) {
            st.liveR[i] = liveR[i];
            sLive[lc][i] = liveR[i];
        }
        st.liveTiles = live;
        sCalc[lc] = calc;
    }
    __syncthreads();

    // Work-list offsets: radius groups in descending radius, each with its layers in
    // order, i.e. position p = (kMaxR - r) * nLayers + q. Each thread sums a run of
    // positions, the block scans the runs, then each thread writes its offsets.
    const int total = (kMaxR + 1) * nLayers;
    const int per = (total + kMaxChunkLayers - 1) / kMaxChunkLayers;
    const int p0 = min(lc * per, total), p1 = min(p0 + per, total);
    int runSum = 0;
    long long runFma = 0;
    for (int p = p0; p < p1; ++p) {
        const int r = kMaxR - p / nLayers, q = p % nLayers;
        const int v = sLive[q][r];
        runSum += v;
        runFma += static_cast<long long>(v) * 256 * (2 * r + 1) * (2 * r + 1);
    }
    const int lane = lc & 31, warp = lc >> 5;
    int incl = runSum;
    for (int o = 1; o < 32; o <<= 1) {
        const int n = __shfl_up_sync(0xffffffffu, incl, o);
        if (lane >= o) incl += n;
    }
    long long wf = runFma;
    for (int o = 16; o > 0; o >>= 1) wf += __shfl_xor_sync(0xffffffffu, wf, o);
    if (lane == 31) sWarpSum[warp] = incl;
    if (lane == 0) sWarpFma[warp] = wf;
    __syncthreads();
    int acc = incl - runSum;
    for (int w = 0; w < warp; ++w) acc += sWarpSum[w];
    const int pSplit = (kMaxR - kSplitR) * nLayers, pSplit2 = (kMaxR - kSplitR2) * nLayers;
    for (int p = p0; p < p1; ++p) {
        const int r = kMaxR - p / nLayers, q = p % nLayers;
        if (p == pSplit) sSplit[0] = acc;
        if (p == pSplit2) sSplit[1] = acc;
        ls[layer0 + q].offR[r] = acc;
        if (q == 0) beam->rStart[r] = acc;
        acc += sLive[q][r];
    }
    __syncthreads();
    if (lc == 0) {
        if (nuclear) {
            // The halo transfer spans the same steps as the primary one.
            beam->firstInside = first;
            beam->maxCalcPassive = primaryBeam->maxCalcPassive;
        }
        acc = 0;
        long long fma = 0;
        for (int w = 0; w < kMaxChunkLayers / 32; ++w) {
            acc += sWarpSum[w];
            fma += sWarpFma[w];
        }
        const int split = sSplit[0], split2 = sSplit[1];
        int mp = beam->maxCalcPassive;
        for (int q = 0; q < nLayers; ++q) mp = max(mp, sCalc[q]);
        beam->maxCalcPassive = mp;
        if (acc > workCapacity) {
            atomicOr(&beam->errorFlags, 1);
            acc = workCapacity;
        }
        beam->workCount = acc;
        beam->workNext = 0;
        beam->workSplit = min(split, acc);
        beam->workNextSmall = 0;
        beam->workSplit2 = min(split2, acc);
        beam->workNextTiny = 0;
        for (int r = 0; r <= kMaxR; ++r) beam->mergedR[r] = 0;
        // Fixed-point range of the chunk's BEV: a cell sums at most `acc` tile
        // footprints (merged items sum several of them), each at most 256 x the
        // largest IDD of the chunk, so with that IDD below 2^ex every cell stays below
        // 2^(ex + 8 + ceil(log2 acc)); the shift puts that bound at 2^61.
        unsigned mb = 0;
        for (int q = 0; q < nLayers; ++q) mb = max(mb, ls[layer0 + q].maxIddBits);
        int ex = 0;
        frexpf(__uint_as_float(mb), &ex);
        int lg = 0;
        while ((1LL << lg) < static_cast<long long>(max(acc, 1))) ++lg;
        beam->fixedShift = mb ? min(61 - ex - 8 - lg, 120) : 0;
        beam->liveTiles += acc;
        beam->superposeFma += fma;
    }
}

// One thread per (layer, step, tile) code of the chunk: live tiles are written to
// their layer's radius group of the work list as one-layer items in the forward
// superposition's format (x = the chunk layer in the low byte, 0xff above it). Each
// layer's box of the cells its items can write (LayerStateDev::liveLo/liveHi) is
// reduced per warp (a warp's 32 consecutive codes span at most a few layers) before
// its atomics.
__global__ void work_scatter_kernel(BeamGeomDev g, int layer0, int nLayers, const uint8_t* __restrict__ codes,
                                    LayerStateDev* __restrict__ ls, const BeamStateDev* __restrict__ beam,
                                    int4* __restrict__ work, int workCapacity) {
    const int tiles = g.tilesX * g.tilesY;
    const int first = beam->firstInside;
    const size_t perLayer = static_cast<size_t>(g.steps) * tiles;
    const size_t total = perLayer * nLayers;
    const int lane = threadIdx.x & 31;
    // Warp-uniform trip count: every lane takes part in the reductions.
    for (size_t i0 = blockIdx.x * size_t(blockDim.x) + threadIdx.x - lane; i0 < total;
         i0 += size_t(gridDim.x) * blockDim.x) {
        const size_t i = i0 + lane;
        int key = -1, R = 0, tile = 0, zr = 0;
        if (i < total) {
            const int lc = int(i / perLayer);
            const int rem = int(i - size_t(lc) * perLayer);
            zr = rem / tiles;
            tile = rem - zr * tiles;
            LayerStateDev& st = ls[layer0 + lc];
            const int c = codes[i];
            if (zr < st.afterLast - first && (c & 0x80)) {
                R = st.batchedR[c & 0x3f];
                const int slot = st.offR[R] + atomicAdd(&st.curR[R], 1);
                if (slot < workCapacity)
                    work[slot] = make_int4(static_cast<int>(0xffffff00u | static_cast<unsigned>(lc)), tile, zr, R);
                key = lc;
            }
        }
        if (!__any_sync(0xffffffffu, key >= 0)) continue;
        const unsigned same = __match_any_sync(0xffffffffu, key);
        const int tx = tile % g.tilesX, ty = tile / g.tilesX;
        const int lo0 = key >= 0 ? tx * kTileX - R + kMaxR : INT_MAX;
        const int lo1 = key >= 0 ? ty * kTileY - R + kMaxR : INT_MAX;
        const int lo2 = key >= 0 ? zr : INT_MAX;
        const int hi0 = key >= 0 ? tx * kTileX + kTileX - 1 + R + kMaxR : INT_MIN;
        const int hi1 = key >= 0 ? ty * kTileY + kTileY - 1 + R + kMaxR : INT_MIN;
        const int hi2 = key >= 0 ? zr : INT_MIN;
        const int mlo0 = __reduce_min_sync(same, lo0), mlo1 = __reduce_min_sync(same, lo1);
        const int mlo2 = __reduce_min_sync(same, lo2);
        const int mhi0 = __reduce_max_sync(same, hi0), mhi1 = __reduce_max_sync(same, hi1);
        const int mhi2 = __reduce_max_sync(same, hi2);
        if (key >= 0 && lane == __ffs(same) - 1) {
            LayerStateDev& st = ls[layer0 + key];
            atomicMin(&st.liveLo[0], mlo0);
            atomicMin(&st.liveLo[1], mlo1);
            atomicMin(&st.liveLo[2], mlo2);
            atomicMax(&st.liveHi[0], mhi0);
            atomicMax(&st.liveHi[1], mhi1);
            atomicMax(&st.liveHi[2], mhi2);
        }
    }
}

// Appends a merged item to the block of its radius, [blockStart[R], blockStart[R - 1])
// (R = 0: up to blockStart[kMaxR + 1], the item count). Merging only joins items of one
// radius, so the merged items of R fit in the block its unmerged items occupy.
__device__ __forceinline__ void emit_merged(BeamStateDev* beam, const int* blockStart, int4* work, unsigned layers,
                                            int tile, int zr, int R) {
    const int begin = blockStart[R];
    const int end = R > 0 ? blockStart[R - 1] : blockStart[kMaxR + 1];
    const int slot = begin + atomicAdd(&beam->mergedR[R], 1);
    if (slot < end) work[slot] = make_int4(static_cast<int>(layers), tile, zr, R);
}

// The forward superposition's work list: one warp per (step, tile) of the chunk,
// a lane per chunk layer (two passes for chunks of more than 32 layers), takes the
// tile's live items at that step (the same items, radii and step ranges as
// work_scatter_kernel) and groups the layers with equal batched radius, in layer
// order, into items of up to kMergeLayers layers (x = the chunk layers as bytes,
// 0xff: none); radii above kSplitR stay one layer per item. Each item goes to the
// block of its radius (so the superposition's CTAs run one radius at a time); the
// order within a block is arbitrary, and the superposition's fixed-point BEV makes
// the dose independent of it.
__global__ void work_merge_kernel(BeamGeomDev g, int layer0, int nLayers, const uint8_t* __restrict__ codes,
                                  const LayerStateDev* __restrict__ ls, BeamStateDev* __restrict__ beam,
                                  int4* __restrict__ work) {
    // The block's extent of the cells its items write (min x, y, z; max x, y, z), and
    // the radius blocks of the list (read once: the claims below are atomics on the
    // same beam state, which later reads of it would wait behind).
    __shared__ int sExt[6];
    __shared__ int sStart[kMaxR + 2];
    pdl_wait();
    if (threadIdx.x < 6) sExt[threadIdx.x] = threadIdx.x < 3 ? INT_MAX : INT_MIN;
    if (threadIdx.x <= kMaxR) sStart[threadIdx.x] = beam->rStart[threadIdx.x];
    if (threadIdx.x == kMaxR + 1) sStart[kMaxR + 1] = beam->workCount;
    __syncthreads();
    const int lane = threadIdx.x & 31;
    const int tiles = g.tilesX * g.tilesY;
    const int first = beam->firstInside;
    const size_t perLayer = static_cast<size_t>(g.steps) * tiles;
    const size_t warps = (size_t(gridDim.x) * blockDim.x) >> 5;
    for (size_t i = (blockIdx.x * size_t(blockDim.x) + threadIdx.x) >> 5; i < perLayer; i += warps) {
        const int zr = int(i / tiles);
        const int tile = int(i - size_t(zr) * tiles);
        int rMax = -1;
        for (int base = 0; base < nLayers; base += 32) {
            const int lc = base + lane;
            int R = -1;
            if (lc < nLayers) {
                const LayerStateDev& st = ls[layer0 + lc];
                const int c = codes[size_t(lc) * perLayer + i];
                if (zr < st.afterLast - first && (c & 0x80)) R = st.batchedR[c & 0x3f];
            }
            rMax = max(rMax, R);
            const bool merge = R >= 0 && R <= kSplitR;
            const unsigned mergeLanes = __ballot_sync(0xffffffffu, merge);
            if (R > kSplitR) emit_merged(beam, sStart, work, 0xffffff00u | unsigned(lc), tile, zr, R);
            if (merge) {
                // Lanes with this radius; every kMergeLayers-th of them (in lane
                // order) writes the item of itself and the next ones.
                const unsigned same = __match_any_sync(mergeLanes, R);
                const unsigned below = (1u << lane) - 1u;
                const int rank = __popc(same & below);
                if (rank % kMergeLayers == 0) {
                    unsigned layers = 0xffffffffu;
                    unsigned rest = same & ~below;
                    for (int n = 0; n < kMergeLayers && rest; ++n) {
                        const int l = __ffs(rest) - 1;
                        rest &= rest - 1u;
                        layers = (layers & ~(0xffu << (8 * n))) | (unsigned(base + l) << (8 * n));
                    }
                    emit_merged(beam, sStart, work, layers, tile, zr, R);
                }
            }
        }
        rMax = __reduce_max_sync(0xffffffffu, rMax);
        if (lane == 0 && rMax >= 0) {
            const int tx = tile % g.tilesX, ty = tile / g.tilesX;
            atomicMin(&sExt[0], tx * kTileX - rMax + kMaxR);
            atomicMin(&sExt[1], ty * kTileY - rMax + kMaxR);
            atomicMin(&sExt[2], zr);
            atomicMax(&sExt[3], tx * kTileX + kTileX - 1 + rMax + kMaxR);
            atomicMax(&sExt[4], ty * kTileY + kTileY - 1 + rMax + kMaxR);
            atomicMax(&sExt[5], zr);
        }
    }
    __syncthreads();
    if (threadIdx.x < 3 && sExt[threadIdx.x] != INT_MAX) atomicMin(&beam->liveLo[threadIdx.x], sExt[threadIdx.x]);
    if (threadIdx.x >= 3 && threadIdx.x < 6 && sExt[threadIdx.x] != INT_MIN)
        atomicMax(&beam->liveHi[threadIdx.x - 3], sExt[threadIdx.x]);
}

// Halo cells start empty: IDD 0 and rSigmaEff +inf (wrapper.cu:4124-4135).
__global__ void nuc_fill_kernel(float* __restrict__ idd, float* __restrict__ rs, size_t n) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        idd[i] = 0.0f;
        rs[i] = __int_as_float(0x7f800000);
    }
}

// One warp per (layer, step, halo tile) over [first, calcPassive) of the layer:
// the tile's radius bucket and liveness (tileRadCalc, complete_superposition.cu:
// 198-255, on the halo grid), its code, and its count in the halo histogram.
__global__ void nuc_codes_kernel(BeamGeomDev gn, int layer0, int nLayers, const float* __restrict__ idd,
                                 const float* __restrict__ rs, const LayerStateDev* __restrict__ primaryLs,
                                 const BeamStateDev* __restrict__ primaryBeam, LayerStateDev* __restrict__ nucLs,
                                 uint8_t* __restrict__ codes) {
    const int lane = threadIdx.x & 31;
    const int tiles = gn.tilesX * gn.tilesY;
    const int first = primaryBeam->firstInside;
    const size_t plane = static_cast<size_t>(gn.pitchX) * gn.pitchY;
    const size_t perLayer = static_cast<size_t>(gn.steps) * tiles;
    const size_t total = perLayer * nLayers;
    const size_t warps = (size_t(gridDim.x) * blockDim.x) >> 5;
    for (size_t i = (blockIdx.x * size_t(blockDim.x) + threadIdx.x) >> 5; i < total; i += warps) {
        const int lc = int(i / perLayer);
        const int rem = int(i - size_t(lc) * perLayer);
        const int zr = rem / tiles, tile = rem - zr * tiles;
        if (zr >= primaryLs[layer0 + lc].calcPassive - first) continue;
        const int tx = tile % gn.tilesX, ty = tile / gn.tilesX;
        const float* ti = idd + (lc * static_cast<size_t>(gn.steps) + zr) * plane + size_t(ty * kTileY) * gn.pitchX +
                          tx * kTileX + lane;
        const float* tr = rs + (ti - idd);
        unsigned key = 0xffffffffu;
        bool live = false;
        float mx = 0.0f;
#pragma unroll
        for (int r = 0; r < kTileY; ++r) {
            key = min(key, float_order_key(tr[size_t(r) * gn.pitchX]));
            const float v = ti[size_t(r) * gn.pitchX];
            live |= v > 0.0f;
            mx = fmaxf(mx, v);
        }
        key = __reduce_min_sync(0xffffffffu, key);
        live = __any_sync(0xffffffffu, live);
        const unsigned mb = __reduce_max_sync(0xffffffffu, __float_as_uint(mx));
        if (lane == 0 && mb) atomicMax(&nucLs[layer0 + lc].maxIddBits, mb);
        if (lane == 0) {
            const int R = tile_radius_bucket(float_from_order_key(key));
            codes[i] = static_cast<uint8_t>(R | (live ? 0x80 : 0));
            atomicAdd(&nucLs[layer0 + lc].histAll[R], 1);
            if (live) atomicAdd(&nucLs[layer0 + lc].liveHist[R], 1);
        }
    }
}

}  // namespace

size_t idd_smem_bytes(const BeamGeomDev& g, const LutsDev& luts) {
    const size_t rows = static_cast<size_t>(luts.nS) * (g.nucOn ? 3 : 1);
    return (rows + luts.nRrl + 2 * static_cast<size_t>(g.steps)) * sizeof(float) +
           static_cast<size_t>(g.steps) * 8 * (sizeof(float) + sizeof(int));
}

cudaError_t launch_nuc_prepare(const BeamGeomDev& gn, int nLayers, float* idd, float* rsigma, cudaStream_t s) {
    const size_t n = static_cast<size_t>(nLayers) * gn.steps * gn.pitchX * gn.pitchY;
    const int blocks = int(std::min<size_t>((n + 255) / 256, 148 * 16));
    nuc_fill_kernel<<<blocks, 256, 0, s>>>(idd, rsigma, n);
    return cudaGetLastError();
}

cudaError_t launch_nuc_codes(const BeamGeomDev& gn, int layer0, int nLayers, const float* idd, const float* rsigma,
                             const LayerStateDev* primaryLs, const BeamStateDev* primaryBeam, LayerStateDev* nucLs,
                             uint8_t* codes, cudaStream_t s) {
    const size_t warps = static_cast<size_t>(nLayers) * gn.steps * gn.tilesX * gn.tilesY;
    const int blocks = int(std::min<size_t>((warps + 7) / 8, 148 * 16));
    nuc_codes_kernel<<<blocks, 256, 0, s>>>(gn, layer0, nLayers, idd, rsigma, primaryLs, primaryBeam, nucLs, codes);
    return cudaGetLastError();
}

cudaError_t launch_idd(const BeamGeomDev& g, const LutsDev& luts, int layer0, int nLayers, const float* density,
                       const float* wepl, const int* firstInside, const int* firstOutside, const float* rayW,
                       const LayerParamsDev* lp, LayerStateDev* ls, const BeamStateDev* beam, float* idd,
                       float* rsigma, uint8_t* codes, int* firstPassive, const int* rayToNuc, const float* lattice,
                       float* nucIdd, float* nucRsigma, cudaStream_t s) {
    dim3 grid(g.tilesX, g.tilesY, nLayers);
    dim3 block(32, 8);
    const size_t smem = idd_smem_bytes(g, luts);
    auto k = g.nucOn ? (g.profileMode ? idd_kernel<true, true> : idd_kernel<true, false>)
                     : (g.profileMode ? idd_kernel<false, true> : idd_kernel<false, false>);
    cudaError_t e = set_smem_limit(reinterpret_cast<const void*>(k), smem);
    if (e != cudaSuccess) return e;
    k<<<grid, block, smem, s>>>(g, luts, layer0, density, wepl, firstInside, firstOutside, rayW, lp, ls, beam, idd,
                                rsigma, codes, firstPassive, rayToNuc, lattice, nucIdd, nucRsigma);
    return cudaGetLastError();
}

cudaError_t launch_bin_plan(const BeamGeomDev& g, int layer0, int nLayers, const uint8_t* codes, LayerStateDev* ls,
                            BeamStateDev* beam, int4* work, int workCapacity, bool merged,
                            const LayerStateDev* primaryLs, const BeamStateDev* primaryBeam, cudaStream_t s) {
    if (nLayers > kMaxChunkLayers) return cudaErrorInvalidValue;
    layer_plan_kernel<<<1, kMaxChunkLayers, 0, s>>>(g, layer0, nLayers, ls, beam, workCapacity, primaryLs,
                                                    primaryBeam);
    if (merged) {
        const size_t warps = static_cast<size_t>(g.steps) * g.tilesX * g.tilesY;
        const int blocks = int(std::min<size_t>((warps + 7) / 8, 148 * 16));
        cudaError_t e = launch_pdl(work_merge_kernel, dim3(blocks), dim3(256), 0, s, g, layer0, nLayers, codes,
                                   static_cast<const LayerStateDev*>(ls), beam, work);
        if (e != cudaSuccess) return e;
    } else {
        const size_t total = static_cast<size_t>(g.steps) * g.tilesX * g.tilesY * nLayers;
        const int blocks = int(std::min<size_t>((total + 255) / 256, 148 * 8));
        work_scatter_kernel<<<blocks, 256, 0, s>>>(g, layer0, nLayers, codes, ls, beam, work, workCapacity);
    }
    return cudaGetLastError();
}

}  // namespace pbs
