// CT preparation, BEV ray tracing, per-step WEPL minimum and the device-side
// beam planner.
#include <float.h>

#include <algorithm>
#include <climits>

#include "device_util.cuh"
#include "kernels.h"
#include "launch_util.h"
#include "../../include/subsecondpbs.h"

namespace pbs {

namespace {

constexpr float kInf20 = 1.0e20f;  // the reference's INF stored in a float (Macro.cuh:7)
constexpr int kTraceSegments = 16;  // warps per tracing CTA; each marches one depth segment
constexpr int kNone = 0x7fffffff;
constexpr size_t kTraceCacheMaxBytes = 160 * 1024;  // CT samples kept on chip up to ~1280 steps
// Packed CT: entry (x, y, z) holds the corners (x, y), (x+1, y), (x, y+1), (x+1, y+1)
// of slice z, for x in [-2, dx + 1], y in [-2, dy + 1], z in [-2, dz + 2] (zero
// outside the CT): every floor index the clamped sample point can take.
constexpr int kQuadPad = 2;

struct CtCorners {
    float c[8];
    float tx, ty, tz;
};

// Trilinear sample of a [Z][Y][X] volume, texel centres at i + 0.5, zero outside
// (sample3DLinearBorder, src/core/bev_ray_tracing.cu:16-61), split into its eight
// corner loads (ct_fetch) and its arithmetic (ct_combine) so that the loads of the
// next sample can be issued first.
__device__ __forceinline__ void ct_fetch(const float* __restrict__ vol, int dx, int dy, int dz, float x, float y,
                                         float z, CtCorners& o) {
    float fx = x - 0.5f, fy = y - 0.5f, fz = z - 0.5f;
    fx = fminf(fmaxf(fx, -2.0f), float(dx) + 1.0f);
    fy = fminf(fmaxf(fy, -2.0f), float(dy) + 1.0f);
    fz = fminf(fmaxf(fz, -2.0f), float(dz) + 1.0f);
    const float flx = floorf(fx), fly = floorf(fy), flz = floorf(fz);
    const int x0 = int(flx), y0 = int(fly), z0 = int(flz);
    o.tx = fx - flx;
    o.ty = fy - fly;
    o.tz = fz - flz;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const int xi = x0 + (i & 1), yi = y0 + ((i >> 1) & 1), zi = z0 + (i >> 2);
        const bool in = xi >= 0 && yi >= 0 && zi >= 0 && xi < dx && yi < dy && zi < dz;
        o.c[i] = in ? __ldg(vol + (static_cast<size_t>(zi) * dy + yi) * dx + xi) : 0.0f;
    }
}

__device__ __forceinline__ float ct_combine(const CtCorners& o) {
    const float c00 = o.c[0] + (o.c[1] - o.c[0]) * o.tx;
    const float c10 = o.c[2] + (o.c[3] - o.c[2]) * o.tx;
    const float c01 = o.c[4] + (o.c[5] - o.c[4]) * o.tx;
    const float c11 = o.c[6] + (o.c[7] - o.c[6]) * o.tx;
    const float c0 = c00 + (c10 - c00) * o.ty;
    const float c1 = c01 + (c11 - c01) * o.ty;
    return c0 + (c1 - c0) * o.tz;
}

// The same eight corners from the packed CT (ct_quad_kernel): two aligned 16-byte
// loads, the border zeros stored in the padding.
__device__ __forceinline__ void ct_fetch_quad(const float4* __restrict__ quad, int dx, int dy, int dz, float x,
                                              float y, float z, CtCorners& o) {
    float fx = x - 0.5f, fy = y - 0.5f, fz = z - 0.5f;
    fx = fminf(fmaxf(fx, -2.0f), float(dx) + 1.0f);
    fy = fminf(fmaxf(fy, -2.0f), float(dy) + 1.0f);
    fz = fminf(fmaxf(fz, -2.0f), float(dz) + 1.0f);
    const float flx = floorf(fx), fly = floorf(fy), flz = floorf(fz);
    const int x0 = int(flx), y0 = int(fly), z0 = int(flz);
    o.tx = fx - flx;
    o.ty = fy - fly;
    o.tz = fz - flz;
    const size_t px = size_t(dx) + kQuadPad + 2, py = size_t(dy) + kQuadPad + 2;
    const size_t i = (size_t(z0 + kQuadPad) * py + size_t(y0 + kQuadPad)) * px + size_t(x0 + kQuadPad);
    const float4 a = __ldg(quad + i), b = __ldg(quad + i + px * py);
    o.c[0] = a.x;
    o.c[1] = a.y;
    o.c[2] = a.z;
    o.c[3] = a.w;
    o.c[4] = b.x;
    o.c[5] = b.y;
    o.c[6] = b.z;
    o.c[7] = b.w;
}

template <bool kQuad>
__device__ __forceinline__ void ct_fetch_any(const float* __restrict__ ct, const float4* __restrict__ quad, int dx,
                                             int dy, int dz, V3 p, CtCorners& o) {
    if (kQuad)
        ct_fetch_quad(quad, dx, dy, dz, p.x, p.y, p.z, o);
    else
        ct_fetch(ct, dx, dy, dz, p.x, p.y, p.z, o);
}

__device__ __forceinline__ void kahan_add(float& sum, float& comp, float v) {
    const float y = v - comp;
    const float t = sum + y;
    comp = (t - sum) - y;
    sum = t;
}

// One CTA traces 32 neighbouring rays of one ray row; warp w marches depth segment w
// (16 segments). In pass 1 the eight CT corners of the next step are loaded while
// the current step is combined, looked up and summed.
// Pass 1 sums each segment, the segment sums are prefix-scanned per ray, and pass 2
// re-marches the segment writing density and compensated cumulative WEPL.
//
// Pass 2 also folds each step's WEPL into the per-step minimum over rays
// (sliceMinVarIgnoreNeverEnter, wrapper.cu:1991-2023): one warp minimum and one
// atomic per warp and step on the bit patterns of the non-negative WEPL values. In
// this path every ray has firstStepOutside >= 1 (lastInside starts at 0,
// bev_ray_tracing.cu:157), so the reference's never-entered filter keeps every ray.
//
// With kCache the first pass keeps every CT sample of the segment in shared memory
// ([segment step][lane], 128 B per step and warp) and the second pass reads them
// back instead of sampling the CT again.
template <bool kCache, bool kQuad>
// Three CTAs per SM (at most 42 registers): the headline grid of 416 row CTAs then
// runs as one wave instead of 1.4.
__global__ void __launch_bounds__(32 * kTraceSegments, 3)
trace_kernel(BeamGeomDev g, LutsDev luts, const float* __restrict__ ct, const float4* __restrict__ ctQuad, int ctX,
             int ctY, int ctZ,
             float* __restrict__ density, float* __restrict__ wepl, int* __restrict__ firstInside,
             int* __restrict__ firstOutside, unsigned* __restrict__ weplMinBits, BeamStateDev* __restrict__ beam) {
    extern __shared__ float shCache[];  // [kTraceSegments][seg][32] with kCache
    const int lane = threadIdx.x, w = threadIdx.y;
    const int x = blockIdx.x * 32 + lane;
    const int y = blockIdx.y;
    const bool active = x < g.rayX;
    const int S = g.steps;
    const int seg = (S + kTraceSegments - 1) / kTraceSegments;
    const int s0 = min(S, w * seg), s1 = min(S, s0 + seg);

    __shared__ float shHu[kTraceSegments][32];
    __shared__ double shSp[kTraceSegments][32];
    __shared__ int shFirst[kTraceSegments][32];
    __shared__ int shLast[kTraceSegments][32];

    V3 pos0 = v3(0.f, 0.f, 0.f), inc = v3(0.f, 0.f, 0.f);
    float stepLen = 0.f;
    if (active) {
        const V3 start = tracer_start(g.tracer, x, y);
        inc = tracer_inc(g.tracer, x, y);
        stepLen = tracer_step_len(g.tracer, x, y);
        // The reference advances the sample point by repeated float additions.
        pos0 = v3(fadd(start.x, 0.5f), fadd(start.y, 0.5f), fadd(start.z, 0.5f));
        for (int k = 0; k < s0; ++k) pos0 = add(pos0, inc);
    }

    // Pass 1: segment sums of HU+1000 and of WEPL increments.
    float huSum = 0.f, spSum = 0.f, spComp = 0.f;
    float* myCache = shCache + static_cast<size_t>(w) * seg * 32 + lane;
    if (active && s0 < s1) {
        V3 pos = pos0;
        CtCorners cur, nxt;
        ct_fetch_any<kQuad>(ct, ctQuad, ctX, ctY, ctZ, pos, cur);
        for (int k = s0; k < s1; ++k) {
            const V3 posN = add(pos, inc);
            if (k + 1 < s1) ct_fetch_any<kQuad>(ct, ctQuad, ctX, ctY, ctZ, posN, nxt);
            const float hu = ct_combine(cur);
            if (kCache) myCache[(k - s0) * 32] = hu;
            huSum += hu;
            const float sp = lut_linear_clamp(luts.sp, luts.nSp, hu * luts.spScale + 0.5f);
            kahan_add(spSum, spComp, stepLen * sp);
            pos = posN;
            cur = nxt;
        }
    }
    shHu[w][lane] = huSum;
    shSp[w][lane] = double(spSum) - double(spComp);
    __syncthreads();

    float huPre = 0.f;
    double spPre = 0.0;
    for (int q = 0; q < w; ++q) {
        huPre += shHu[q][lane];
        spPre += shSp[q][lane];
    }

    // Pass 2: write the per-step samples (every lane runs the loop: it holds the
    // warp reductions of the step minimum).
    int firstK = kNone, lastK = -1;
    {
        V3 pos = pos0;
        float cumHu = huPre;
        float cum = float(spPre);
        float comp = float(double(cum) - spPre);
        const size_t plane = static_cast<size_t>(g.rayX) * g.rayY;
        size_t idx = static_cast<size_t>(s0) * plane + static_cast<size_t>(y) * g.rayX + x;
        for (int k = s0; k < s1; ++k) {
            unsigned bits = 0xffffffffu;
            if (active) {
                float hu;
                if (kCache) {
                    hu = myCache[(k - s0) * 32];
                } else {
                    CtCorners c;
                    ct_fetch_any<kQuad>(ct, ctQuad, ctX, ctY, ctZ, pos, c);
                    hu = ct_combine(c);
                }
                cumHu += hu;
                density[idx] = lut_linear_clamp(luts.density, luts.nDensity, hu * luts.densityScale + 0.5f);
                const float sp = lut_linear_clamp(luts.sp, luts.nSp, hu * luts.spScale + 0.5f);
                kahan_add(cum, comp, stepLen * sp);
                wepl[idx] = cum;
                if (firstK == kNone && !(cumHu < 150.0f)) firstK = k;
                if (hu > 150.0f) lastK = k;
                pos = add(pos, inc);
                idx += plane;
                // NaN stays out of the minimum, as with the reference's `v < min` test.
                bits = cum >= 0.0f ? (__float_as_uint(cum) & 0x7fffffffu) : (cum < 0.0f ? 0u : 0xffffffffu);
            }
            bits = __reduce_min_sync(0xffffffffu, bits);
            if (lane == 0 && bits != 0xffffffffu) atomicMin(weplMinBits + k, bits);
        }
    }
    shFirst[w][lane] = firstK;
    shLast[w][lane] = lastK;
    __syncthreads();

    if (w == 0) {
        int fk = kNone, lk = -1;
        for (int q = 0; q < kTraceSegments; ++q) {
            fk = min(fk, shFirst[q][lane]);
            lk = max(lk, shLast[q][lane]);
        }
        // beforeFirstInside + 1 and lastInside + 1 in the reference's convention.
        const int fi = (fk == kNone) ? S : max(fk, 1);
        const int fo = (lk < 0) ? 1 : lk + 1;
        int wmin = active ? fi : INT_MAX;
        int wmax = active ? fo : INT_MIN;
        if (active) {
            firstInside[y * g.rayX + x] = fi;
            firstOutside[y * g.rayX + x] = fo;
        }
        for (int o = 16; o > 0; o >>= 1) {
            wmin = min(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
            wmax = max(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
        }
        if (lane == 0) {
            atomicMin(&beam->firstInside, wmin);
            atomicMax(&beam->firstOutside, wmax);
        }
    }
}

// Packed CT (kQuadPad): one thread per entry.
__global__ void ct_quad_kernel(const float* __restrict__ ct, int dx, int dy, int dz, float4* __restrict__ quad) {
    const size_t px = size_t(dx) + kQuadPad + 2, py = size_t(dy) + kQuadPad + 2, pz = size_t(dz) + kQuadPad + 3;
    const size_t n = px * py * pz;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const int x = int(i % px) - kQuadPad;
        const size_t r = i / px;
        const int y = int(r % py) - kQuadPad;
        const int z = int(r / py) - kQuadPad;
        auto at = [&](int xi, int yi) -> float {
            if (xi < 0 || yi < 0 || z < 0 || xi >= dx || yi >= dy || z >= dz) return 0.0f;
            return ct[(size_t(z) * dy + yi) * dx + xi];
        };
        quad[i] = make_float4(at(x, y), at(x + 1, y), at(x, y + 1), at(x + 1, y + 1));
    }
}

// ---- water-equivalence import transport -------------------------------------
// fillBevFromWeqVolumeKernel (wrapper.cu:1923-1989): the exporter's per-ray water-
// equivalent depths replace the CT trace. Ray (x, y) at (origin + index * ray
// spacing) reads the WEQ texel nearest to it (body [nx][ny][steps], depth fastest);
// WEPL is that depth, density its per-step increase divided by the WEQ step, and
// the ray enters at its first step with density above 1e-4 (firstInside = that
// step + 1, else `steps`) and leaves after its last (firstOutside = last + 1, else 0).
// A ray outside the WEQ lattice keeps depth 0; steps beyond the active ones keep the
// last depth read.
//
// Layout: one CTA per 32 consecutive rays (ray index y * rayX + x). Depths are read
// depth-fastest (one warp per ray and 32-step chunk, coalesced) and written
// ray-fastest ([step][ray], coalesced) through a 32 x 33 shared tile.
struct WeqParams {
    const float* body;
    int nx, ny, storedSteps, activeSteps;
    float stepMm;
    float rayOriginX, rayOriginY, rayStepX, rayStepY;
    float x0, y0, dx, dy;
};

constexpr int kWeqRaysPerCta = 32;

__global__ void __launch_bounds__(256)
weq_fill_kernel(BeamGeomDev g, WeqParams q, float* __restrict__ density, float* __restrict__ wepl,
                int* __restrict__ firstInside, int* __restrict__ firstOutside, BeamStateDev* __restrict__ beam) {
    __shared__ float tile[32][33];
    __shared__ float carry[32];
    __shared__ long long base[kWeqRaysPerCta];
    __shared__ int sFirst[8][32], sLast[8][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int rays = g.rayX * g.rayY, S = g.steps;
    const int r0 = blockIdx.x * kWeqRaysPerCta;
    const float safeStep = q.stepMm > 0.0f ? q.stepMm : 1.0f;
    if (w == 0) {
        long long b = -1;
        const int r = r0 + lane;
        if (r < rays) {
            const int x = r % g.rayX, y = r / g.rayX;
            const float rx = fmaf(float(x), q.rayStepX, q.rayOriginX);
            const float ry = fmaf(float(y), q.rayStepY, q.rayOriginY);
            const int wx = fabsf(q.dx) > 0.0f ? int(lroundf((rx - q.x0) / q.dx)) : -1;
            const int wy = fabsf(q.dy) > 0.0f ? int(lroundf((ry - q.y0) / q.dy)) : -1;
            if (wx >= 0 && wx < q.nx && wy >= 0 && wy < q.ny)
                b = (static_cast<long long>(wx) * q.ny + wy) * q.storedSteps;
        }
        base[lane] = b;
        carry[lane] = 0.0f;
    }
    __syncthreads();
    int first = INT_MAX, last = -1;
    const size_t plane = static_cast<size_t>(rays);
    for (int k0 = 0; k0 < S; k0 += 32) {
#pragma unroll
        for (int j = 0; j < kWeqRaysPerCta / 8; ++j) {
            const int ray = w * (kWeqRaysPerCta / 8) + j;
            const long long b = base[ray];
            const int k = min(k0 + lane, q.activeSteps - 1);
            tile[lane][ray] = (b >= 0 && k >= 0) ? q.body[b + k] : 0.0f;
        }
        __syncthreads();
        const int r = r0 + lane;
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            const int kk = w + 8 * i, k = k0 + kk;
            if (k < S && r < rays) {
                const float v = tile[kk][lane];
                const float prev = kk > 0 ? tile[kk - 1][lane] : carry[lane];
                const float d = fmaxf(0.0f, v - prev) / safeStep;
                wepl[static_cast<size_t>(k) * plane + r] = v;
                density[static_cast<size_t>(k) * plane + r] = d;
                if (d > 1.0e-4f) {
                    first = min(first, k);
                    last = max(last, k);
                }
            }
        }
        __syncthreads();
        if (w == 0) carry[lane] = tile[31][lane];
        __syncthreads();
    }
    sFirst[w][lane] = first;
    sLast[w][lane] = last;
    __syncthreads();
    if (w == 0) {
        int fk = INT_MAX, lk = -1;
        for (int q8 = 0; q8 < 8; ++q8) {
            fk = min(fk, sFirst[q8][lane]);
            lk = max(lk, sLast[q8][lane]);
        }
        const int r = r0 + lane;
        const bool active = r < rays;
        const int fi = fk == INT_MAX ? S : fk + 1;
        const int fo = lk >= 0 ? lk + 1 : 0;
        if (active) {
            firstInside[r] = fi;
            firstOutside[r] = fo;
        }
        int wmin = active ? fi : INT_MAX, wmax = active ? fo : INT_MIN;
        for (int o = 16; o > 0; o >>= 1) {
            wmin = min(wmin, __shfl_xor_sync(0xffffffffu, wmin, o));
            wmax = max(wmax, __shfl_xor_sync(0xffffffffu, wmax, o));
        }
        if (lane == 0) {
            atomicMin(&beam->firstInside, wmin);
            atomicMax(&beam->firstOutside, wmax);
        }
    }
}

// sliceMinVarIgnoreNeverEnter (wrapper.cu:1991-2023): per step the minimum WEPL
// over the rays that enter (firstOutside > 0), 1e20 where none does. One CTA per
// step, reading the step's rays contiguously.
__global__ void __launch_bounds__(256)
weq_step_min_kernel(BeamGeomDev g, const float* __restrict__ wepl, const int* __restrict__ firstOutside,
                    float* __restrict__ weplMin) {
    __shared__ float red[8];
    const int rays = g.rayX * g.rayY;
    const float* row = wepl + static_cast<size_t>(blockIdx.x) * rays;
    float m = kInf20;
    for (int r = threadIdx.x; r < rays; r += blockDim.x)
        if (firstOutside[r] > 0) {
            const float v = row[r];
            if (v < m) m = v;
        }
    for (int o = 16; o > 0; o >>= 1) {
        const float other = __shfl_xor_sync(0xffffffffu, m, o);
        if (other < m) m = other;
    }
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < 8; ++i)
            if (red[i] < m) m = red[i];
        weplMin[blockIdx.x] = m;
    }
}

// include/utils/vector_find.h:61-82
__device__ int find_first_larger_ordered_dev(const float* v, int n, float value) {
    int upper = n - 1, lower = 0;
    if (v[n - 1] <= value) return upper;
    if (v[0] > value) return 0;
    while (upper - lower > 1) {
        const int pivot = (upper + lower) / 2;
        if (v[pivot] <= value) lower = pivot;
        else upper = pivot;
    }
    return lower + 1;
}

__global__ void beam_planner_kernel(BeamGeomDev g, float* __restrict__ weplMin,
                                    const LayerParamsDev* __restrict__ lp, LayerStateDev* __restrict__ ls,
                                    BeamStateDev* __restrict__ beam) {
    __shared__ int shPassive;
    __shared__ float shEntryZ;
    // Steps that no ray reached keep the cleared pattern: they hold the
    // reference's INF (Macro.cuh:7).
    for (int k = threadIdx.x; k < g.steps; k += blockDim.x)
        if (__float_as_uint(weplMin[k]) == 0xffffffffu) weplMin[k] = kInf20;
    __syncthreads();
    if (threadIdx.x == 0) {
        const int first = beam->firstInside;
        const float limitAll = fmul(kBpDepthCutoff, g.maxPeakDepthMm);
        const int g0 = find_first_larger_ordered_dev(weplMin, g.steps, limitAll);
        const int passive = min(g0, beam->firstOutside);
        beam->guaranteedPassive = passive;
        const float entryZ = fadd(fmul(float(first), g.fanDelta.z), g.fanCorner.z);
        beam->entryZ = entryZ;
        beam->pxSpMultX = fsub(1.0f, fdiv(entryZ, g.sourceDist.x));
        beam->pxSpMultY = fsub(1.0f, fdiv(entryZ, g.sourceDist.y));
        beam->maxCalcPassive = first;
        beam->liveTiles = 0;
        beam->superposeFma = 0;
        shPassive = passive;
        shEntryZ = entryZ;
    }
    __syncthreads();
    const float z = shEntryZ;
    for (int l = threadIdx.x; l < g.numLayers; l += blockDim.x) {
        const LayerParamsDev p = lp[l];
        LayerStateDev& st = ls[l];
        const float limit = fmul(kBpDepthCutoff, p.peakDepth);
        st.afterLast = min(find_first_larger_ordered_dev(weplMin, g.steps, limit), shPassive);
        // Entry sigma of the convolution (wrapper.cu:3776-3833).
        {
            const float a = fdiv(0.00270f, fsub(p.convPeakDepth, 4.50f));
            const float b = fdiv(-4.39f, fsub(p.convPeakDepth, 3.86f));
            const float base = fadd(fmul(fmul(a, z), z), fmul(b, z));
            st.entrySigmaX = fmul(fsqrt(fmaxf(0.0f, fadd(base, fmul(p.sigmaXmm, p.sigmaXmm)))), g.entrySigmaScale);
            st.entrySigmaY = fmul(fsqrt(fmaxf(0.0f, fadd(base, fmul(p.sigmaYmm, p.sigmaYmm)))), g.entrySigmaScale);
        }
        // IDD entry variance (wrapper.cu:4309-4313).
        {
            const float a = fdiv(0.00270f, fsub(p.peakDepth, 4.50f));
            const float b = fdiv(-4.39f, fsub(p.peakDepth, 3.86f));
            st.entrySigmaSq = fadd(fadd(fmul(fmul(a, z), z), fmul(b, z)), fmul(p.sigmaXmm, p.sigmaXmm));
        }
        st.maxFirstPassive = INT_MIN;
        st.calcPassive = 0;
        st.liveTiles = 0;
        st.maxIddBits = 0;
        for (int i = 0; i < kBuckets; ++i) {
            st.hist[i] = 0;
            st.batchedR[i] = 0;
            st.histAll[i] = 0;
            st.liveHist[i] = 0;
        }
        for (int i = 0; i < 33; ++i) st.batchedCounts[i] = 0;
        for (int i = 0; i < 3; ++i) {
            st.liveLo[i] = INT_MAX;
            st.liveHi[i] = INT_MIN;
        }
    }
}

// Type detection of the reference's CT adapter (wrapper.cu:2327-2337) on the sample
// minimum and maximum.
__device__ __forceinline__ int ct_type_from_range(float mn, float mx) {
    if (mn < -200.0f) return PBS_CT_HU;
    if (mx <= 20.0f && mn >= 0.0f) return PBS_CT_DENSITY;
    return PBS_CT_HU_PLUS_1000;
}

// With `rangeKeys` (order keys of the sample minimum and maximum, from
// ct_sample_range_kernel) the type is detected here; `lut` is then the density
// table, the only one detection can call for. The voxels converted are the box
// [lo, lo + ext) of the [dims.z][dims.y][dims.x] grid.
__global__ void ct_convert_kernel(float* ct, int3 dims, int3 lo, int3 ext, int type, const float* __restrict__ lut,
                                  int lutN, float lutScale, const unsigned* __restrict__ rangeKeys) {
    if (rangeKeys) {
        type = ct_type_from_range(float_from_order_key(rangeKeys[0]), float_from_order_key(rangeKeys[1]));
        if (type == PBS_CT_HU_PLUS_1000) return;
    }
    const size_t total = size_t(ext.x) * ext.y * ext.z;
    for (size_t b = blockIdx.x * size_t(blockDim.x) + threadIdx.x; b < total; b += size_t(gridDim.x) * blockDim.x) {
        const size_t r = b / size_t(ext.x);
        const size_t i = (size_t(int(r / size_t(ext.y)) + lo.z) * dims.y + (int(r % size_t(ext.y)) + lo.y)) *
                             size_t(dims.x) +
                         (int(b % size_t(ext.x)) + lo.x);
        const float v = ct[i];
        if (type == PBS_CT_HU) {
            ct[i] = v + 1000.0f;
        } else if (type == PBS_CT_DENSITY || type == PBS_CT_SPR) {
            // findFractionalIndexMonotonic (wrapper.cu:2339-2376), then / scale.
            float idx;
            const bool inc = lut[lutN - 1] >= lut[0];
            if (lutN <= 1) {
                idx = 0.0f;
            } else if (inc ? (v <= lut[0]) : (v >= lut[0])) {
                idx = 0.0f;
            } else if (inc ? (v >= lut[lutN - 1]) : (v <= lut[lutN - 1])) {
                idx = float(lutN - 1);
            } else {
                int lo = 0, hi = lutN - 1;
                while (hi - lo > 1) {
                    const int mid = (lo + hi) >> 1;
                    const float vm = lut[mid];
                    if (inc) {
                        if (vm <= v) lo = mid; else hi = mid;
                    } else {
                        if (vm >= v) lo = mid; else hi = mid;
                    }
                }
                const float v0 = lut[lo], den = __fsub_rn(lut[lo + 1], v0);
                float t = 0.0f;
                if (den != 0.0f) t = __fdiv_rn(__fsub_rn(v, v0), den);
                t = fminf(fmaxf(t, 0.0f), 1.0f);
                idx = __fadd_rn(float(lo), t);
            }
            ct[i] = __fdiv_rn(idx, lutScale);
        }
    }
}

// The reference's strided sample (every `stride`-th value, wrapper.cu:2307-2325), one
// thread per sample, reduced into order keys of its minimum and maximum (NaN is
// left out, as under std::min / std::max). Used on the caller's page-locked host CT
// through its device mapping, so that the CT type is known without a host pass.
// Range of the CT type samples (every `stride`-th voxel, wrapper.cu:2307-2337) in two
// passes. Pass 0 reads the samples inside the uploaded box from the device copy
// (raw values: the conversion runs after both passes). Pass 1 reads the samples
// outside the box from the caller's page-locked host CT through its device mapping
// (latency-bound reads over the host link), unless pass 0 already found a value
// below -200: the type is then HU whatever the other samples hold, since the
// detection tests the minimum against -200 first (ct_type_from_range).
__global__ void ct_sample_range_kernel(const float* __restrict__ hostCt, const float* __restrict__ devCt, int3 dims,
                                       int3 lo, int3 hi, size_t stride, size_t samples, unsigned* keys, int pass) {
    if (pass == 1 && float_from_order_key(*(volatile unsigned*)keys) < -200.0f) return;
    const size_t k = blockIdx.x * size_t(blockDim.x) + threadIdx.x;
    unsigned kl = 0xffffffffu, kh = 0u;
    if (k < samples) {
        const size_t idx = k * stride;
        const size_t plane = size_t(dims.x) * dims.y;
        const int z = int(idx / plane);
        const size_t r = idx - size_t(z) * plane;
        const int y = int(r / dims.x), x = int(r - size_t(y) * dims.x);
        const bool inBox = x >= lo.x && x <= hi.x && y >= lo.y && y <= hi.y && z >= lo.z && z <= hi.z;
        if (inBox == (pass == 0)) {
            const float v = inBox ? devCt[idx] : hostCt[idx];
            if (v == v) kl = kh = float_order_key(v);
        }
    }
    kl = __reduce_min_sync(0xffffffffu, kl);
    kh = __reduce_max_sync(0xffffffffu, kh);
    if ((threadIdx.x & 31) == 0) {
        if (kl != 0xffffffffu) atomicMin(keys, kl);
        if (kh != 0u) atomicMax(keys + 1, kh);
    }
}

__global__ void ct_stats_kernel(const float* __restrict__ ct, size_t n, size_t stride, float* minmax) {
    float mn = ct[0], mx = ct[0];
    for (size_t i = size_t(threadIdx.x) * stride; i < n; i += size_t(blockDim.x) * stride) {
        mn = fminf(mn, ct[i]);
        mx = fmaxf(mx, ct[i]);
    }
    for (int o = 16; o > 0; o >>= 1) {
        mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
        mx = fmaxf(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    }
    __shared__ float a[32], b[32];
    if ((threadIdx.x & 31) == 0) {
        a[threadIdx.x >> 5] = mn;
        b[threadIdx.x >> 5] = mx;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int i = 1; i < int(blockDim.x >> 5); ++i) {
            mn = fminf(mn, a[i]);
            mx = fmaxf(mx, b[i]);
        }
        minmax[0] = fminf(mn, a[0]);
        minmax[1] = fmaxf(mx, b[0]);
    }
}

}  // namespace

cudaError_t launch_ct_convert(float* ct, size_t n, int type, const float* lut, int lutN, float lutScale,
                              cudaStream_t s) {
    if (type == PBS_CT_HU_PLUS_1000 || n == 0) return cudaSuccess;
    // A flat buffer as one row of n voxels (n fits an int for every CT this takes).
    if (n > size_t(INT_MAX)) return cudaErrorInvalidValue;
    const int3 d = make_int3(int(n), 1, 1);
    const int blocks = int(std::min<size_t>((n + 255) / 256, 148 * 16));
    ct_convert_kernel<<<blocks, 256, 0, s>>>(ct, d, make_int3(0, 0, 0), d, type, lut, lutN, lutScale, nullptr);
    return cudaGetLastError();
}

cudaError_t launch_ct_convert_box(float* ct, const int dims[3], const int lo[3], const int hi[3], int type,
                                  const float* lut, int lutN, float lutScale, cudaStream_t s) {
    if (type == PBS_CT_HU_PLUS_1000) return cudaSuccess;
    for (int i = 0; i < 3; ++i)
        if (lo[i] < 0 || hi[i] >= dims[i] || hi[i] < lo[i]) return cudaErrorInvalidValue;
    const int3 d = make_int3(dims[0], dims[1], dims[2]);
    const int3 e = make_int3(hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1);
    const size_t total = size_t(e.x) * e.y * e.z;
    const int blocks = int(std::min<size_t>((total + 255) / 256, 148 * 16));
    ct_convert_kernel<<<blocks, 256, 0, s>>>(ct, d, make_int3(lo[0], lo[1], lo[2]), e, type, lut, lutN, lutScale,
                                             nullptr);
    return cudaGetLastError();
}

size_t ct_type_sample_count(size_t n) {
    const size_t maxSamples = 100000;
    const size_t stride = (n > maxSamples) ? (n / maxSamples) : 1;
    return n == 0 ? 0 : (n + stride - 1) / stride;
}

cudaError_t launch_ct_convert_detect(float* ct, size_t n, const float* hostCtMapped, const int dims[3],
                                     const int boxLo[3], const int boxHi[3], const float* densityLut, int lutN,
                                     float lutScale, unsigned* keys, cudaStream_t s) {
    if (n == 0) return cudaSuccess;
    const size_t maxSamples = 100000;
    const size_t stride = (n > maxSamples) ? (n / maxSamples) : 1;
    const size_t samples = ct_type_sample_count(n);
    cudaError_t e = cudaMemsetAsync(keys, 0xff, sizeof(unsigned), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(keys + 1, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return e;
    const int3 d = make_int3(dims[0], dims[1], dims[2]);
    const int3 lo = make_int3(boxLo[0], boxLo[1], boxLo[2]), hi = make_int3(boxHi[0], boxHi[1], boxHi[2]);
    for (int pass = 0; pass < 2; ++pass)
        ct_sample_range_kernel<<<unsigned((samples + 255) / 256), 256, 0, s>>>(hostCtMapped, ct, d, lo, hi, stride,
                                                                               samples, keys, pass);
    // Only the uploaded box is converted: the tracers sample nothing outside it.
    const int3 ext = make_int3(hi.x - lo.x + 1, hi.y - lo.y + 1, hi.z - lo.z + 1);
    if (ext.x <= 0 || ext.y <= 0 || ext.z <= 0) return cudaGetLastError();
    const size_t total = size_t(ext.x) * ext.y * ext.z;
    const int blocks = int(std::min<size_t>((total + 255) / 256, 148 * 16));
    ct_convert_kernel<<<blocks, 256, 0, s>>>(ct, d, lo, ext, PBS_CT_AUTO, densityLut, lutN, lutScale, keys);
    return cudaGetLastError();
}

cudaError_t launch_ct_stats(const float* ct, size_t n, float* minmax2, cudaStream_t s) {
    const size_t maxSamples = 100000;
    const size_t stride = (n > maxSamples) ? (n / maxSamples) : 1;
    ct_stats_kernel<<<1, 1024, 0, s>>>(ct, n, stride, minmax2);
    return cudaGetLastError();
}

size_t ct_quad_bytes(const int dims[3]) {
    return (size_t(dims[0]) + kQuadPad + 2) * (size_t(dims[1]) + kQuadPad + 2) * (size_t(dims[2]) + kQuadPad + 3) *
           sizeof(float4);
}

// Packed entries (x, y, z) for x, y, z in [lo, lo + ext) only; lo may reach into the
// padding (negative, or past the CT), where the entries hold the border zeros.
__global__ void ct_quad_box_kernel(const float* __restrict__ ct, int dx, int dy, int dz, int3 lo, int3 ext,
                                   float4* __restrict__ quad) {
    const size_t px = size_t(dx) + kQuadPad + 2, py = size_t(dy) + kQuadPad + 2;
    const size_t total = size_t(ext.x) * ext.y * ext.z;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const int x = lo.x + int(i % size_t(ext.x));
        const size_t r = i / size_t(ext.x);
        const int y = lo.y + int(r % size_t(ext.y));
        const int z = lo.z + int(r / size_t(ext.y));
        auto at = [&](int xi, int yi) -> float {
            if (xi < 0 || yi < 0 || z < 0 || xi >= dx || yi >= dy || z >= dz) return 0.0f;
            return ct[(size_t(z) * dy + yi) * dx + xi];
        };
        quad[(size_t(z + kQuadPad) * py + size_t(y + kQuadPad)) * px + size_t(x + kQuadPad)] =
            make_float4(at(x, y), at(x + 1, y), at(x, y + 1), at(x + 1, y + 1));
    }
}

cudaError_t launch_ct_quad_box(const float* ct, const int dims[3], const int lo[3], const int hi[3], float4* quad,
                               cudaStream_t s) {
    int a[3], b[3];
    for (int i = 0; i < 3; ++i) {
        if (lo[i] < 0 || hi[i] >= dims[i] || hi[i] < lo[i]) return cudaErrorInvalidValue;
        // A box on a face of the CT takes the padding beyond that face along: the
        // tracer clamps sample points outside the CT into it.
        a[i] = lo[i] == 0 ? -kQuadPad : lo[i];
        b[i] = hi[i] == dims[i] - 1 ? dims[i] - 1 + kQuadPad + (i == 2 ? 1 : 0) : hi[i];
    }
    const int3 l = make_int3(a[0], a[1], a[2]);
    const int3 e = make_int3(b[0] - a[0] + 1, b[1] - a[1] + 1, b[2] - a[2] + 1);
    const size_t total = size_t(e.x) * e.y * e.z;
    const int blocks = int(std::min<size_t>((total + 255) / 256, 148 * 16));
    ct_quad_box_kernel<<<blocks, 256, 0, s>>>(ct, dims[0], dims[1], dims[2], l, e, quad);
    return cudaGetLastError();
}

cudaError_t launch_ct_quad(const float* ct, const int dims[3], float4* quad, cudaStream_t s) {
    const size_t n = ct_quad_bytes(dims) / sizeof(float4);
    const int blocks = int(std::min<size_t>((n + 255) / 256, 148 * 16));
    ct_quad_kernel<<<blocks, 256, 0, s>>>(ct, dims[0], dims[1], dims[2], quad);
    return cudaGetLastError();
}

cudaError_t launch_trace(const BeamGeomDev& g, const LutsDev& luts, const float* ct, const float4* ctQuad, int ctX,
                         int ctY, int ctZ, float* density, float* wepl, int* firstInside, int* firstOutside,
                         float* weplMin, BeamStateDev* beam, cudaStream_t s) {
    // 0xff bytes: the largest unsigned pattern, the identity of the atomic minimum.
    cudaError_t e = cudaMemsetAsync(weplMin, 0xff, sizeof(float) * size_t(g.steps), s);
    if (e != cudaSuccess) return e;
    dim3 block(32, kTraceSegments);
    dim3 grid((g.rayX + 31) / 32, g.rayY);
    const int seg = (g.steps + kTraceSegments - 1) / kTraceSegments;
    const size_t cache = static_cast<size_t>(kTraceSegments) * seg * 32 * sizeof(float);
    unsigned* mins = reinterpret_cast<unsigned*>(weplMin);
    auto k = cache <= kTraceCacheMaxBytes ? (ctQuad ? trace_kernel<true, true> : trace_kernel<true, false>)
                                          : (ctQuad ? trace_kernel<false, true> : trace_kernel<false, false>);
    const size_t smem = cache <= kTraceCacheMaxBytes ? cache : 0;
    if (smem) {
        e = set_smem_limit(reinterpret_cast<const void*>(k), smem);
        if (e != cudaSuccess) return e;
    }
    k<<<grid, block, smem, s>>>(g, luts, ct, ctQuad, ctX, ctY, ctZ, density, wepl, firstInside, firstOutside, mins,
                                beam);
    return cudaGetLastError();
}

cudaError_t launch_weq_trace(const BeamGeomDev& g, const float* body, int nx, int ny, int storedSteps,
                             int activeSteps, float stepMm, float rayOriginX, float rayOriginY, float rayStepX,
                             float rayStepY, float x0, float y0, float dx, float dy, float* density, float* wepl,
                             int* firstInside, int* firstOutside, float* weplMin, BeamStateDev* beam, cudaStream_t s) {
    WeqParams q{body, nx, ny, storedSteps, activeSteps, stepMm, rayOriginX, rayOriginY, rayStepX, rayStepY,
                x0, y0, dx, dy};
    const int rays = g.rayX * g.rayY;
    weq_fill_kernel<<<(rays + kWeqRaysPerCta - 1) / kWeqRaysPerCta, 256, 0, s>>>(g, q, density, wepl, firstInside,
                                                                                  firstOutside, beam);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    weq_step_min_kernel<<<g.steps, 256, 0, s>>>(g, wepl, firstOutside, weplMin);
    return cudaGetLastError();
}

cudaError_t launch_beam_planner(const BeamGeomDev& g, float* weplMin, const LayerParamsDev* lp,
                                LayerStateDev* ls, BeamStateDev* beam, cudaStream_t s) {
    beam_planner_kernel<<<1, 64, 0, s>>>(g, weplMin, lp, ls, beam);
    return cudaGetLastError();
}

}  // namespace pbs
