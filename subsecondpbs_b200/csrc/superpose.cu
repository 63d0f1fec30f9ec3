// Tile-based Gaussian superposition of the per-ray IDD into the padded BEV dose.
//
// Each work item is one 32x8 tile of source rays at one step with its batched radius
// R (kernelSuperposition<R>, complete_superposition.cu:264-335), for one layer or,
// for R <= kSplitR, for up to kMergeLayers layers whose tile has the same radius at
// that step (their footprints land on the same BEV cells). Every source s spreads
// idd_s * e_s(dy) * e_s(dx) over a (2R+1)^2 footprint, where
// e_s(0) = erf(r/2) and e_s(k) = (erf((k+1/2) r) - erf((k-1/2) r)) / 2.
//
// Formulation on the FP32 FMA pipe (one CTA per item, persistent grid):
//   * table phase (per layer of the item): each thread builds its source's rows
//     e_s(0..R) (float4 chunks, chunk-major so that the stores and the broadcast
//     reads are conflict-free) and idd_s * e_s(0..R) (odd row stride); sources
//     without dose get zero rows;
//   * accumulation phase: a warp lane is one column distance |d| of one source
//     column (radii 0..15) or one signed offset (radii 16..32); a source column's
//     eight sources share the lane's output columns, so the lane keeps the whole
//     footprint height (8+2R rows) in registers and adds idd_s e_s(|d|) * e_s(k) to
//     rows sy+R+-k. Up to radius 15 the column at +d, equal to the one at -d, is
//     accumulated once and added to both: the FMAs and shared loads are
//     (R+1)/(2R+1) of the direct (2R+1)^2 formulation. Several source columns share
//     one warp instruction; for radii 16..32 the tile's (column, offset) pairs are
//     dealt out 32 at a time. A pair ends with one shared-memory add per footprint
//     row and output column; pairs whose source column has no depositing source are
//     skipped;
//   * the footprint accumulates in 32-bit fixed point: a float add to shared memory
//     has no native instruction on this part (it is a compare-and-swap loop, a
//     third of the throughput of an integer add), while the integer add is native
//     and order-independent. Every footprint value and every partial sum of it is at
//     most the item's total dose (each e_s(k) <= 1 and each source adds to a row of
//     a pair once), so the power-of-two scale 2^30 / total keeps every sum inside
//     int32 with a resolution of 2^-30 of the item's dose;
//   * the footprint of all the item's layers is then added to the BEV dose of its
//     step (all layers of the beam share one BEV volume) in 64-bit fixed point: a
//     BEV cell sums many items, and integer adds commute, so the dose does not depend
//     on the order in which the items land. The chunk's exponent
//     (layer_plan_kernel) bounds every cell below 2^62; a last pass adds the chunk
//     to the float BEV and clears it.
// Up to radius 7 a warp has at most one (column, distance) unit, so its column sums
// stay in registers over all the item's layers and are flushed once per item.
// Radii 16..32, 8..15 and 0..7 run as three persistent instances with 128, 48 and
// 40 registers: 2, 5 and 6 CTAs per SM.
#include <algorithm>

#include "device_util.cuh"
#include "work_blocks.cuh"
#include "kernels.h"
#include "launch_util.h"

namespace pbs {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;

// A footprint value q * 2^-sc as a BEV fixed-point value at 2^shift (truncated
// below the BEV's resolution). q >= 0; the chunk's shift leaves headroom for items
// of up to kMergeLayers tiles, so the result stays below 2^62.
__device__ __forceinline__ unsigned long long to_bev_fixed(int q, int sc, int shift) {
    const int e = shift - sc;
    if (e >= 0) return static_cast<unsigned long long>(q) << min(e, 62);
    return e > -63 ? static_cast<unsigned long long>(q) >> (-e) : 0ull;
}

// Fixed-point exponent of an item of total dose `total`: 2^(30 - ex) with
// total < 2^ex, so total * 2^sc < 2^30.
__device__ __forceinline__ int footprint_exponent(float total) {
    int ex;
    frexpf(total, &ex);
    return min(30 - ex, 126);
}

// Adds the item's fixed-point footprint [H][Wo] to the BEV.
template <int H, int Wo>
__device__ __forceinline__ void write_footprint(const int* __restrict__ out, unsigned long long* __restrict__ dst,
                                                int bevX, int sc, int shift) {
    for (int i = threadIdx.x; i < H * Wo; i += kThreads) {
        const int q = out[i];
        const int oy = i / Wo, ox = i - oy * Wo;
        if (q != 0) atomicAdd(dst + static_cast<size_t>(oy) * bevX + ox, to_bev_fixed(q, sc, shift));
    }
}

struct ItemArgs {
    const float* idd;
    const float* rsig;
    size_t layerStride;         // IDD elements per chunk layer
    size_t src;                 // this thread's source ray within a layer
    unsigned long long* dst;    // footprint origin in the fixed-point BEV dose
    unsigned layers;            // chunk layers of the item, one per byte (0xff: none)
    int bevX;
    int shift;                  // BEV fixed-point exponent
};

// ============================================================================
// Radii 0..15: lanes over (source column, |d|) pairs, layer by layer of a merged
// item into one fixed-point footprint.
// ============================================================================

template <int RMax>
struct PairShape {
    static constexpr int kQ = (RMax + 1 + 3) / 4;            // float4 chunks of e_s(k), k <= RMax
    static constexpr int kEWStride = (RMax + 1) | 1;          // odd: lanes of one row hit distinct banks
    static constexpr int kOutInts = (kTileY + 2 * RMax) * (kTileX + 2 * RMax);
    static constexpr size_t kSmemBytes =
        (size_t(kQ) * kThreads * 4 + size_t(kThreads) * kEWStride + kOutInts) * sizeof(float);
};

// Column part of the slot of source (sy, sx) in the chunk-major e_s table
// (slot = sy * 32 + e4_col(sx)): the low bits are XORed with bits 3..4 so that
// source columns 4, 8 or 16 apart (read together by the lane groups of one
// instruction) land in different banks.
__device__ __forceinline__ int e4_col(int sx) { return sx ^ ((sx >> 3) & 3); }

template <int R, int RMax>
__device__ __forceinline__ void pair_item(float4* __restrict__ E4, float* __restrict__ EW, int* __restrict__ out,
                                          unsigned* __restrict__ sCol, float* __restrict__ sSum,
                                          const ItemArgs& a) {
    constexpr int H = kTileY + 2 * R;
    constexpr int Wo = kTileX + 2 * R;
    constexpr int Q = (R + 1 + 3) / 4;
    constexpr int EWS = PairShape<RMax>::kEWStride;
    // A source column's footprint is the same column vector at offsets +d and -d (the
    // weights depend on |d| only): one lane per (source column, |d|) pair adds it to
    // both output columns. floor(32 / (R+1)) source columns, spaced so that their
    // pairs fill distinct lanes, share one warp instruction.
    constexpr int M = R + 1;
    constexpr int G = 32 / M;                   // source columns per instruction
    constexpr int S = (32 + G - 1) / G;         // column spacing
    constexpr int kUnits = S;
    const int t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31;

    // Up to radius 7 a warp holds at most one (column, |d|) unit, whose column sums stay
    // in registers over the item's layers and are flushed once.
    constexpr bool kOneFlush = kUnits <= kWarps;

    // H and Wo are even and `out` is 16-byte aligned.
    for (int i = t; i < H * Wo / 4; i += kThreads) reinterpret_cast<int4*>(out)[i] = make_int4(0, 0, 0, 0);
    // Fixed-point scale from the dose of every layer of the item: each thread sums its
    // source over the layers, then the warps and the CTA add up. With one flush per
    // item the sums run in the table phases and the scale is applied at the flush;
    // with a flush per layer they run first and the scale is folded into the weights.
    // Either way the total (the same additions in the same order) and the flushed
    // values are the same.
    float rowDose = 0.0f;
    int sc = 0;
    float scale = 1.0f;
    auto item_scale = [&]() {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rowDose += __shfl_xor_sync(0xffffffffu, rowDose, o);
        if (lane == 0) sSum[warp] = rowDose;
        __syncthreads();
        float total = 0.0f;
#pragma unroll
        for (int w = 0; w < kWarps; ++w) total += sSum[w];
        sc = footprint_exponent(total);
        scale = ldexpf(1.0f, sc);
    };
    if constexpr (!kOneFlush) {
#pragma unroll 1
        for (int j = 0; j < kMergeLayers; ++j) {
            const unsigned lc = (a.layers >> (8 * j)) & 0xffu;
            if (lc == 0xffu) break;
            rowDose += fmaxf(a.idd[lc * a.layerStride + a.src], 0.0f);
        }
        item_scale();
    }

    // Table phase of one layer (complete_superposition.cu:298-307): thread t is source
    // (sy, sx) = (warp, lane); its rows e_s(0..R) go in float4 chunks (chunk-major)
    // and idd_s e_s(0..R) 2^sc (the fixed-point scale is a power of two, so the column
    // sums come out scaled exactly as if each were scaled at the flush); sources
    // without dose get zero rows, and colMask[sx] collects the depositing sources of
    // every column.
    auto table = [&](unsigned lc, unsigned* colMask) {
        const size_t src = lc * a.layerStride + a.src;
        const float dose = a.idd[src];
        if constexpr (kOneFlush) rowDose += fmaxf(dose, 0.0f);
        const bool live = dose > 0.0f;
        if (live) atomicOr(&colMask[lane], 1u << warp);
        float e[4 * Q];
        if (live) {
            float row[R + 1];
            superposition_row<R>(a.rsig[src], row);
            const float doseScaled = kOneFlush ? dose : dose * scale;
#pragma unroll
            for (int k = 0; k <= R; ++k) {
                e[k] = row[k];
                EW[t * EWS + k] = doseScaled * row[k];
            }
        } else {
#pragma unroll
            for (int k = 0; k <= R; ++k) {
                e[k] = 0.0f;
                EW[t * EWS + k] = 0.0f;
            }
        }
#pragma unroll
        for (int k = R + 1; k < 4 * Q; ++k) e[k] = 0.0f;
        const int pt = warp * kTileX + e4_col(lane);
#pragma unroll
        for (int q = 0; q < Q; ++q)
            E4[q * kThreads + pt] = make_float4(e[4 * q], e[4 * q + 1], e[4 * q + 2], e[4 * q + 3]);
    };
    // Adds the eight sources of source column sx at distance d to the column sums.
    auto accumulate = [&](int sx, int d, float (&acc)[H]) {
        const float* ewCol = EW + sx * EWS + d;
        const float4* eCol = E4 + e4_col(sx);
#pragma unroll
        for (int sy = 0; sy < kTileY; ++sy) {
            const float w = ewCol[sy * kTileX * EWS];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const float4 v = eCol[q * kThreads + sy * kTileX];
                const float ev[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int k = 4 * q + c;
                    if (k <= R) {
                        acc[sy + R + k] = fmaf(w, ev[c], acc[sy + R + k]);
                        if (k > 0) acc[sy + R - k] = fmaf(w, ev[c], acc[sy + R - k]);
                    }
                }
            }
            // Lets the loads of the next source overlap this pair's FMAs but keeps
            // later sources' loads from being hoisted (which would hold every row
            // of the column in registers).
            if (sy & 1) asm volatile("" ::: "memory");
        }
    };
    // Adds a pair's column sums to both of its output columns.
    auto flush = [&](int sx, int d, const float (&acc)[H]) {
        int qv[H];
#pragma unroll
        for (int i = 0; i < H; ++i) qv[i] = __float2int_rn(kOneFlush ? acc[i] * scale : acc[i]);
        int* col = out + sx + R + d;
#pragma unroll
        for (int i = 0; i < H; ++i) atomicAdd(col + i * Wo, qv[i]);
        if (d > 0) {
            col = out + sx + R - d;
#pragma unroll
            for (int i = 0; i < H; ++i) atomicAdd(col + i * Wo, qv[i]);
        }
    };

    if constexpr (kOneFlush) {
        // One pair unit per warp: its column sums stay in registers over all the
        // item's layers and are flushed once. The column masks OR over the layers.
        const int g = lane / M;
        int d = lane - g * M;
        int sx = warp + g * S;
        const bool valid = warp < kUnits && g < G && sx < kTileX;
        if (!valid) {
            sx = 0;
            d = 0;
        }
        float acc[H];
#pragma unroll
        for (int i = 0; i < H; ++i) acc[i] = 0.0f;
#pragma unroll 1
        for (int j = 0; j < kMergeLayers; ++j) {
            const unsigned lc = (a.layers >> (8 * j)) & 0xffu;
            if (lc == 0xffu) break;
            table(lc, sCol);
            __syncthreads();
            // Lanes outside the footprint read source column 0 and are never flushed.
            // Every lane takes part in the shuffle.
            const unsigned colAll = __shfl_sync(0xffffffffu, sCol[lane], sx);
            const unsigned colLive = valid ? colAll : 0u;
            if (__any_sync(0xffffffffu, colLive != 0)) accumulate(sx, d, acc);
            // The next layer's tables overwrite these.
            __syncthreads();
        }
        item_scale();
        const unsigned colAll = __shfl_sync(0xffffffffu, sCol[lane], sx);
        const unsigned colLive = valid ? colAll : 0u;
        if (colLive) flush(sx, d, acc);
        __syncthreads();
        if (t < kTileX) sCol[t] = 0;
    } else {
#pragma unroll 1
        for (int j = 0; j < kMergeLayers; ++j) {
            const unsigned lc = (a.layers >> (8 * j)) & 0xffu;
            if (lc == 0xffu) break;
            // The layers alternate between two column-mask buffers: a buffer is
            // cleared after the barrier that ends its layer's accumulation, and
            // refilled two layers later.
            unsigned* colMask = sCol + (j & 1) * kTileX;
            table(lc, colMask);
            __syncthreads();
            // Lanes outside the footprint read source column 0 and are never flushed;
            // pairs whose source column has no depositing source are skipped.
            const unsigned colBits = colMask[lane];
#pragma unroll 1
            for (int u = warp; u < kUnits; u += kWarps) {
                const int g = lane / M;
                int d = lane - g * M;
                int sx = u + g * S;
                const bool valid = g < G && sx < kTileX;
                if (!valid) {
                    sx = 0;
                    d = 0;
                }
                const unsigned colAll = __shfl_sync(0xffffffffu, colBits, sx);
                const unsigned colLive = valid ? colAll : 0u;
                if (!__any_sync(0xffffffffu, colLive != 0)) continue;
                float acc[H];
#pragma unroll
                for (int i = 0; i < H; ++i) acc[i] = 0.0f;
                accumulate(sx, d, acc);
                if (colLive) flush(sx, d, acc);
            }
            // The next layer's tables overwrite these.
            __syncthreads();
            if (t < kTileX) colMask[t] = 0;
        }
    }
    __syncthreads();

    // ---- write-out -------------------------------------------------------------
    write_footprint<H, Wo>(out, a.dst, a.bevX, sc, a.shift);
}

template <int R, int RHi, int RMax>
__device__ __forceinline__ bool dispatch_pair(int r, float4* E4, float* EW, int* out, unsigned* sCol, float* sSum,
                                              const ItemArgs& a) {
    if (r == R) {
        pair_item<R, RMax>(E4, EW, out, sCol, sSum, a);
        return true;
    }
    if constexpr (R < RHi) return dispatch_pair<R + 1, RHi, RMax>(r, E4, EW, out, sCol, sSum, a);
    return false;
}

// ============================================================================
// Radii 16..32: one layer per item, lanes over (source column, signed offset).
// ============================================================================

template <int RMax>
struct WideShape {
    static constexpr int kQ = (RMax + 1 + 3) / 4;            // float4 chunks of e_s(k), k <= RMax
    static constexpr int kEWStride = (RMax + 1) | 1;          // odd: lanes of one row hit distinct banks
    static constexpr int kOutFloats = (kTileY + 2 * RMax) * (kTileX + 2 * RMax);
    static constexpr size_t kSmemBytes =
        (size_t(kQ) * kThreads * 4 + size_t(kThreads) * kEWStride + kOutFloats) * sizeof(float);
};

template <int R, int RMax>
__device__ __forceinline__ void wide_item(float4* __restrict__ E4, float* __restrict__ EW, int* __restrict__ out,
                                          unsigned* __restrict__ sCol, float* __restrict__ sSum,
                                          const ItemArgs& a) {
    constexpr int H = kTileY + 2 * R;
    constexpr int Wo = kTileX + 2 * R;
    constexpr int Q = (R + 1 + 3) / 4;
    constexpr int EWS = WideShape<RMax>::kEWStride;
    constexpr int M = 2 * R + 1;                 // signed offsets per source column
    constexpr int kPairs = kTileX * M;
    constexpr int kUnits = (kPairs + 31) / 32;
    const int t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31;
    const size_t src = (a.layers & 0xffu) * a.layerStride + a.src;

    // ---- table phase ----------------------------------------------------------
    {
        const float dose = a.idd[src];
        const bool live = dose > 0.0f;
        if (live) atomicOr(&sCol[lane], 1u << warp);
        float rowDose = live ? dose : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rowDose += __shfl_xor_sync(0xffffffffu, rowDose, o);
        if (lane == 0) sSum[warp] = rowDose;
        float e[4 * Q];
        if (live) {
            float row[R + 1];
            superposition_row<R>(a.rsig[src], row);
#pragma unroll
            for (int k = 0; k <= R; ++k) {
                e[k] = row[k];
                EW[t * EWS + k] = dose * row[k];
            }
        } else {
#pragma unroll
            for (int k = 0; k <= R; ++k) {
                e[k] = 0.0f;
                EW[t * EWS + k] = 0.0f;
            }
        }
#pragma unroll
        for (int k = R + 1; k < 4 * Q; ++k) e[k] = 0.0f;
        const int pt = warp * kTileX + e4_col(lane);
#pragma unroll
        for (int q = 0; q < Q; ++q) E4[q * kThreads + pt] = make_float4(e[4 * q], e[4 * q + 1], e[4 * q + 2], e[4 * q + 3]);
        for (int i = t; i < H * Wo / 4; i += kThreads) reinterpret_cast<int4*>(out)[i] = make_int4(0, 0, 0, 0);
    }
    __syncthreads();

    float total = 0.0f;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) total += sSum[w];
    const int sc = footprint_exponent(total);
    const float scale = ldexpf(1.0f, sc);

    // ---- accumulation phase -----------------------------------------------------
    const unsigned colBits = sCol[lane];
#pragma unroll 1
    for (int u = warp; u < kUnits; u += kWarps) {
        const int pr = u * 32 + lane;
        const bool valid = pr < kPairs;
        int sx = pr / M;
        int d = pr - sx * M - R;
        if (!valid) {
            sx = 0;
            d = 0;
        }
        const int ad = d < 0 ? -d : d;
        const unsigned colAll = __shfl_sync(0xffffffffu, colBits, sx);
        const unsigned colLive = valid ? colAll : 0u;
        if (!__any_sync(0xffffffffu, colLive != 0)) continue;
        // Lanes outside the footprint read source column 0 and are never flushed.
        const float* ewCol = EW + sx * EWS + ad;
        const float4* eCol = E4 + e4_col(sx);
        float acc[H];
#pragma unroll
        for (int i = 0; i < H; ++i) acc[i] = 0.0f;
#pragma unroll
        for (int sy = 0; sy < kTileY; ++sy) {
            const float w = ewCol[sy * kTileX * EWS];
#pragma unroll
            for (int q = 0; q < Q; ++q) {
                const float4 v = eCol[q * kThreads + sy * kTileX];
                const float ev[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    const int k = 4 * q + c;
                    if (k <= R) {
                        acc[sy + R + k] = fmaf(w, ev[c], acc[sy + R + k]);
                        if (k > 0) acc[sy + R - k] = fmaf(w, ev[c], acc[sy + R - k]);
                    }
                }
            }
            if (sy & 1) asm volatile("" ::: "memory");
        }
        if (colLive) {
            int* col = out + sx + R + d;
#pragma unroll
            for (int i = 0; i < H; ++i) atomicAdd(col + i * Wo, __float2int_rn(acc[i] * scale));
        }
    }
    __syncthreads();

    // ---- write-out ---------------------------------------------------------------
    if (t < kTileX) sCol[t] = 0;
    write_footprint<H, Wo>(out, a.dst, a.bevX, sc, a.shift);
}

template <int R, int RHi, int RMax>
__device__ __forceinline__ bool dispatch_wide(int r, float4* E4, float* EW, int* out, unsigned* sCol, float* sSum,
                                              const ItemArgs& a) {
    if (r == R) {
        wide_item<R, RMax>(E4, EW, out, sCol, sSum, a);
        return true;
    }
    if constexpr (R < RHi) return dispatch_wide<R + 1, RHi, RMax>(r, E4, EW, out, sCol, sSum, a);
    return false;
}

// ============================================================================
// The persistent kernel.
// ============================================================================

// Persistent CTA loop over the merged items of radii RLo..RHi, claimed one at a
// time through the range's counter (the next claim is issued before the current
// item runs so that its latency is hidden). Items are taken radius block by radius
// block, so the CTAs of the SM mostly run the code of one radius at a time.
//
// The three instances of a beam are launched back to back with programmatic
// dependent launch: every CTA lets the next instance start at once (its items are
// independent of this instance's: both only add to the fixed-point BEV), so the next
// instance's CTAs take the SMs this instance's CTAs leave at its tail. Before it
// exits a CTA waits for the previous instance to complete, so an instance is complete
// only once all earlier ones are, and the kernel after the last one (launched
// normally) sees every item's adds.
template <bool kWide, int RLo, int RHi, int MinBlocks>
__global__ void __launch_bounds__(kThreads, MinBlocks)
superpose_kernel(BeamGeomDev g, const float* __restrict__ idd, const float* __restrict__ rsig,
                 const int4* __restrict__ work, BeamStateDev* __restrict__ beam, unsigned long long* __restrict__ bev,
                 int shiftOffset, int range, size_t layerBevStride) {
    extern __shared__ __align__(16) float sm[];
    __shared__ int sItem[2];
    // Per source column, its depositing sources over sy (radii 0..15: two buffers).
    __shared__ unsigned sCol[2 * kTileX];
    __shared__ float sSum[kTileY];
    __shared__ RadiusBlocks<RLo, RHi> sBlocks;

    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const int t = threadIdx.x;
    // Range 0: R > kSplitR, 1: kSplitR2 < R <= kSplitR, 2: R <= kSplitR2.
    int* counter = range == 0 ? &beam->workNext : (range == 1 ? &beam->workNextSmall : &beam->workNextTiny);
    const size_t padPlane = static_cast<size_t>(g.pitchX) * g.pitchY;
    const size_t bevPlane = static_cast<size_t>(g.bevX) * g.bevY;

    load_blocks<RLo, RHi>(beam, sBlocks);
    if (t == 0) sItem[0] = atomicAdd(counter, 1);
    if (t < 2 * kTileX) sCol[t] = 0;
    if (t < kTileY) sSum[t] = 0.0f;
    __syncthreads();
    ItemArgs a;
    a.idd = idd;
    a.rsig = rsig;
    a.layerStride = static_cast<size_t>(g.steps) * padPlane;
    a.bevX = g.bevX;
    a.shift = beam->fixedShift + shiftOffset;
    int buf = 0;
    for (;;) {
        const int c = sItem[buf];
        if (c >= sBlocks.total) break;
        if (t == 0) sItem[buf ^ 1] = atomicAdd(counter, 1);
        const int4 it = work[block_slot<RLo, RHi>(sBlocks, c)];
        const int tile = it.y, zRel = it.z, R = it.w;
        const int tx = tile % g.tilesX, ty = tile / g.tilesX;
        a.layers = static_cast<unsigned>(it.x);
        a.src = zRel * padPlane + static_cast<size_t>(ty * kTileY + (t >> 5)) * g.pitchX + tx * kTileX + (t & 31);
        // One BEV volume per layer when layerBevStride is set (one-layer items: batched
        // influence columns), else one volume for all layers.
        a.dst = bev + (it.x & 0xff) * layerBevStride + static_cast<size_t>(zRel) * bevPlane +
                static_cast<size_t>(ty * kTileY - R + kMaxR) * g.bevX + (tx * kTileX - R + kMaxR);
        bool ok;
        if constexpr (kWide) {
            float4* E4 = reinterpret_cast<float4*>(sm);                                       // [Q][256] e_s(4q..4q+3)
            float* EW = sm + WideShape<RHi>::kQ * kThreads * 4;                               // [256][EWS] idd_s e_s(k)
            int* out = reinterpret_cast<int*>(EW + kThreads * WideShape<RHi>::kEWStride);   // [8+2R][32+2R]
            ok = dispatch_wide<RLo, RHi, RHi>(R, E4, EW, out, sCol, sSum, a);
        } else {
            float4* E4 = reinterpret_cast<float4*>(sm);                                       // [Q][256] e_s(4q..4q+3)
            float* EW = sm + PairShape<RHi>::kQ * kThreads * 4;                               // [256][EWS] idd_s e_s(k)
            int* out = reinterpret_cast<int*>(EW + kThreads * PairShape<RHi>::kEWStride);   // [8+2R][32+2R]
            ok = dispatch_pair<RLo, RHi, RHi>(R, E4, EW, out, sCol, sSum, a);
        }
        if (!ok && t == 0) atomicOr(&beam->errorFlags, 2);
        // Every thread is past the item (and has read sItem[buf]) before the next
        // claim lands in that slot.
        __syncthreads();
        buf ^= 1;
    }
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

// `overlap`: launch as a programmatic dependent of the previous kernel on `s` (the
// previous superposition instance).
template <bool kWide, int RLo, int RHi, int MinBlocks>
cudaError_t launch_range(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                         BeamStateDev* beam, unsigned long long* bev, int shiftOffset, int gridBlocks, int range,
                         bool overlap, size_t layerBevStride, cudaStream_t s) {
    auto k = superpose_kernel<kWide, RLo, RHi, MinBlocks>;
    const size_t smem = kWide ? WideShape<RHi>::kSmemBytes : PairShape<RHi>::kSmemBytes;
    cudaError_t e = set_smem_limit(reinterpret_cast<const void*>(k), smem);
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(gridBlocks);
    cfg.blockDim = dim3(kThreads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = overlap ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, k, g, idd, rsigma, work, beam, bev, shiftOffset, range, layerBevStride);
}

// Adds the fixed-point BEV of the chunk to the float BEV and clears it for the next
// superposition, over the cells the items can have written: the box of live cells
// (BeamStateDev::liveLo/liveHi, from work_merge_kernel) within the planes written so
// far, [0, maxCalcPassive - firstInside). Every cell is converted once, so the float BEV is
// the same on every run.
__global__ void __launch_bounds__(256) bev_fixed_to_float_kernel(BeamGeomDev g, const BeamStateDev* __restrict__ beam,
                                                                 unsigned long long* __restrict__ fixed,
                                                                 float* __restrict__ bev, int shiftOffset) {
    pdl_wait();
    const int planes = min(beam->maxCalcPassive - beam->firstInside, g.steps);
    if (planes <= 0 || beam->liveLo[0] > beam->liveHi[0]) return;
    // bevX is even (the padded ray pitch plus 2 kMaxR), so cells go in aligned pairs.
    const int x0 = max(beam->liveLo[0], 0) & ~1, x1 = min(beam->liveHi[0], g.bevX - 1) | 1;
    const int y0 = max(beam->liveLo[1], 0), y1 = min(beam->liveHi[1], g.bevY - 1);
    const int z0 = max(beam->liveLo[2], 0), z1 = min(beam->liveHi[2], planes - 1);
    if (x1 < x0 || y1 < y0 || z1 < z0) return;
    const int pw = (x1 - x0 + 1) / 2, rows = y1 - y0 + 1;
    const size_t n = static_cast<size_t>(pw) * rows * (z1 - z0 + 1);
    const double unit = ldexp(1.0, -(beam->fixedShift + shiftOffset));
    ulonglong2* f2 = reinterpret_cast<ulonglong2*>(fixed);
    float2* b2 = reinterpret_cast<float2*>(bev);
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const int xp = static_cast<int>(i % pw);
        const size_t r = i / pw;
        const int y = y0 + static_cast<int>(r % rows);
        const int z = z0 + static_cast<int>(r / rows);
        const size_t pr = ((static_cast<size_t>(z) * g.bevY + y) * g.bevX + x0) / 2 + xp;
        const ulonglong2 v = f2[pr];
        if (v.x | v.y) {
            float2 o = b2[pr];
            o.x += float(double(v.x) * unit);
            o.y += float(double(v.y) * unit);
            b2[pr] = o;
            f2[pr] = make_ulonglong2(0ull, 0ull);
        }
    }
}

// Resident CTAs per SM of the instances.
constexpr int kWideBlocks = 2;
constexpr int kMidBlocks = 5;
constexpr int kNarrowBlocks = 6;

}  // namespace

namespace {

// The three instances over `work` (items sorted by range: the wide radii first).
cudaError_t launch_instances(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                             BeamStateDev* beam, unsigned long long* bevFixed, int shiftOffset, int numSMs,
                             size_t layerBevStride, cudaStream_t s) {
    cudaError_t e = launch_range<true, kSplitR + 1, kMaxR, kWideBlocks>(
        g, idd, rsigma, work, beam, bevFixed, shiftOffset, numSMs * kWideBlocks, 0, false, layerBevStride, s);
    if (e != cudaSuccess) return e;
    e = launch_range<false, kSplitR2 + 1, kSplitR, kMidBlocks>(g, idd, rsigma, work, beam, bevFixed, shiftOffset,
                                                               numSMs * kMidBlocks, 1, true, layerBevStride, s);
    if (e != cudaSuccess) return e;
    return launch_range<false, 0, kSplitR2, kNarrowBlocks>(g, idd, rsigma, work, beam, bevFixed, shiftOffset,
                                                           numSMs * kNarrowBlocks, 2, true, layerBevStride, s);
}

// A superposition over the chunk's whole one-layer work list (work_scatter_kernel):
// radius block R is [rStart[R], rStart[R - 1]) (or up to workCount), and the claim
// counters restart.
__global__ void one_layer_list_view_kernel(BeamStateDev* __restrict__ beam) {
    const int t = threadIdx.x;
    if (t <= kMaxR) {
        const int end = t > 0 ? beam->rStart[t - 1] : beam->workCount;
        beam->mergedR[t] = max(end - beam->rStart[t], 0);
    }
    if (t == 0) {
        beam->workNext = 0;
        beam->workNextSmall = 0;
        beam->workNextTiny = 0;
    }
}

// Batched influence columns: bev_fixed_to_float_kernel for volume q (blockIdx.y) over
// its layer's live cells (LayerStateDev::liveLo/liveHi).
__global__ void __launch_bounds__(256) column_fixed_to_float_kernel(BeamGeomDev g, const BeamStateDev* __restrict__ beam,
                                                                    const LayerStateDev* __restrict__ ls,
                                                                    unsigned long long* __restrict__ fixed,
                                                                    float* __restrict__ bev, size_t stride) {
    const int q = blockIdx.y;
    const LayerStateDev& st = ls[q];
    if (st.liveLo[0] > st.liveHi[0]) return;
    const int x0 = max(st.liveLo[0], 0) & ~1, x1 = min(st.liveHi[0], g.bevX - 1) | 1;
    const int y0 = max(st.liveLo[1], 0), y1 = min(st.liveHi[1], g.bevY - 1);
    const int z0 = max(st.liveLo[2], 0), z1 = min(st.liveHi[2], g.steps - 1);
    if (x1 < x0 || y1 < y0 || z1 < z0) return;
    const int pw = (x1 - x0 + 1) / 2, rows = y1 - y0 + 1;
    const size_t n = static_cast<size_t>(pw) * rows * (z1 - z0 + 1);
    const double unit = ldexp(1.0, -beam->fixedShift);
    // stride is even (bevX is), so every volume starts on a cell pair.
    ulonglong2* f2 = reinterpret_cast<ulonglong2*>(fixed + static_cast<size_t>(q) * stride);
    float2* b2 = reinterpret_cast<float2*>(bev + static_cast<size_t>(q) * stride);
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const int xp = static_cast<int>(i % pw);
        const size_t r = i / pw;
        const int y = y0 + static_cast<int>(r % rows);
        const int z = z0 + static_cast<int>(r / rows);
        const size_t pr = ((static_cast<size_t>(z) * g.bevY + y) * g.bevX + x0) / 2 + xp;
        const ulonglong2 v = f2[pr];
        if (v.x | v.y) {
            float2 o = b2[pr];
            o.x += float(double(v.x) * unit);
            o.y += float(double(v.y) * unit);
            b2[pr] = o;
            f2[pr] = make_ulonglong2(0ull, 0ull);
        }
    }
}

}  // namespace

cudaError_t launch_superpose(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                             BeamStateDev* beam, float* bev, unsigned long long* bevFixed, int shiftOffset, int numSMs,
                             cudaStream_t s) {
    cudaError_t e = launch_instances(g, idd, rsigma, work, beam, bevFixed, shiftOffset, numSMs, 0, s);
    if (e != cudaSuccess) return e;
    e = launch_pdl(bev_fixed_to_float_kernel, dim3(numSMs * 8), dim3(256), 0, s, g,
                   static_cast<const BeamStateDev*>(beam), bevFixed, bev, shiftOffset);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t launch_one_layer_list_view(BeamStateDev* beam, cudaStream_t s) {
    one_layer_list_view_kernel<<<1, 64, 0, s>>>(beam);
    return cudaGetLastError();
}

cudaError_t launch_superpose_columns(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                                     BeamStateDev* beam, const LayerStateDev* ls, int nCols, float* bev,
                                     unsigned long long* bevFixed, size_t stride, int numSMs, cudaStream_t s) {
    if (nCols <= 0) return cudaSuccess;
    if (stride % 2) return cudaErrorInvalidValue;
    one_layer_list_view_kernel<<<1, 64, 0, s>>>(beam);
    cudaError_t e = launch_instances(g, idd, rsigma, work, beam, bevFixed, 0, numSMs, stride, s);
    if (e != cudaSuccess) return e;
    const int per = std::max(1, (numSMs * 8) / nCols);
    column_fixed_to_float_kernel<<<dim3(per, nCols), 256, 0, s>>>(g, beam, ls, bevFixed, bev, stride);
    return cudaGetLastError();
}

}  // namespace pbs
