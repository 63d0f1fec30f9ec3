// Tile-based Gaussian superposition of the per-ray IDD into the padded BEV dose.
//
// Work items come from the radius-sorted list built on the device; each item is one
// 32x8 tile of source rays at one step of one layer with its batched radius R
// (kernelSuperposition<R>, complete_superposition.cu:264-335). Every source s
// spreads idd_s * e_s(dy) * e_s(dx) over a (2R+1)^2 footprint, where
// e_s(0) = erf(r/2) and e_s(k) = (erf((k+1/2) r) - erf((k-1/2) r)) / 2.
//
// Formulation on the FP32 FMA pipe (one CTA per tile, persistent grid):
//   * table phase: each thread builds its source's rows e_s(0..R) (float4 chunks,
//     chunk-major so that the stores and the broadcast reads are conflict-free)
//     and idd_s * e_s(0..R) (odd row stride); sources without dose get zero rows;
//   * accumulation phase: a warp lane is one column distance |d| of one source
//     column; a source column's eight sources share the lane's output
//     columns, so the lane keeps the whole footprint height (8+2R rows) in
//     registers and adds idd_s e_s(|d|) * e_s(k) to rows sy+R+-k. The column at
//     +d equals the one at -d, so up to radius 15 it is accumulated once and added
//     to both: the FMAs and shared loads are (R+1)/(2R+1) of the direct (2R+1)^2
//     formulation. Several source columns share one warp instruction; for radii
//     16..32 a lane is one signed offset and the tile's (column, offset) pairs are
//     dealt out 32 at a time. A pair ends with one
//     shared-memory add per footprint row and output column; pairs whose source
//     column has no depositing source are skipped;
//   * the footprint accumulates in 32-bit fixed point: a float add to shared memory
//     has no native instruction on this part (it is a compare-and-swap loop, a
//     third of the throughput of an integer add), while the integer add is native
//     and order-independent. Every footprint value and every partial sum of it is at
//     most the tile's total dose (each e_s(k) <= 1 and each source adds to a row of
//     a pair once), so the power-of-two scale 2^30 / total keeps every sum inside
//     int32 with a resolution of 2^-30 of the tile's dose, finer than FP32 near the
//     footprint's peak;
//   * the tile footprint is then added to the BEV dose of its step (all layers of
//     the beam share one BEV volume).
// Radii 16..32, 8..15 and 0..7 run as three instances of the kernel with 128, 48
// and 32 registers and 96, 43 and 21 KB of shared memory: 2, 5 and 8 CTAs per SM
// (the narrower instances trade a few spilled registers for occupancy).
#include "device_util.cuh"
#include "kernels.h"
#include "launch_util.h"

namespace pbs {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
// Resident CTAs per SM of the paired instances (radii 12..15, 8..11, 0..7).
constexpr int kMidBlocks = 2;
constexpr int kMidNarrowBlocks = 3;
constexpr int kNarrowBlocks = 4;
constexpr int kPairs = kTileX / 2;                 // column pairs per tile row
constexpr int kPairSlots = kTileY * kPairs;        // (row, pair) slots per tile

template <int RMax>
struct Shape {
    static constexpr int kQ = (RMax + 1 + 3) / 4;            // float4 chunks of e_s(k), k <= RMax
    static constexpr int kEWStride = (RMax + 1) | 1;          // odd: lanes of one row hit distinct banks
    static constexpr int kOutFloats = (kTileY + 2 * RMax) * (kTileX + 2 * RMax);
    static constexpr size_t kSmemBytes =
        (size_t(kQ) * kThreads * 4 + size_t(kThreads) * kEWStride + kOutFloats) * sizeof(float);
};

// Paired layout (instances with radii up to kSplitR): the sources of source columns
// 2p and 2p+1 (a column pair p) are stored interleaved, so that one 16-byte load
// gives e(k) and e(k+1) of both columns as two register pairs and one 8-byte load
// gives idd * e(d) of both; the accumulation then runs on packed FP32x2 FMAs, one
// instruction per footprint row for the two columns.
template <int RMax>
struct PairShape {
    static constexpr int kQ2 = (RMax + 2) / 2;                // float4 = (e_a(k), e_b(k), e_a(k+1), e_b(k+1))
    static constexpr int kEW2 = (RMax + 1) | 1;               // float2 stride per (row, pair), odd
    static constexpr int kOutInts = (kTileY + 2 * RMax) * (kTileX + 2 * RMax);
    static constexpr size_t kSmemBytes =
        size_t(kQ2) * kPairSlots * 16 + size_t(kPairSlots) * kEW2 * 8 + size_t(kOutInts) * 4;
};

// Slot of column pair p (0..15) within a source row: pairs 8 apart, read together by
// the lane groups of one instruction, land in different banks.
__device__ __forceinline__ int pair_slot(int p) { return p ^ ((p >> 3) & 1); }

// Column part of the slot of source (sy, sx) in the chunk-major e_s table
// (slot = sy * 32 + e4_col(sx)): the low bits are XORed with bits 3..4 so that
// source columns 4, 8 or 16 apart (read together by the lane groups of one
// instruction) land in different banks.
__device__ __forceinline__ int e4_col(int sx) { return sx ^ ((sx >> 3) & 3); }

struct TileArgs {
    const float* idd;
    const float* rsig;
    float* bev;
    size_t src;        // this thread's source ray in the IDD / rSigma arrays
    float* dst;        // footprint origin in the BEV dose
    int bevX;
};

// Table phase, accumulation phase and write-out of one tile at radius R.
template <int R, int RMax>
__device__ __forceinline__ void superpose_tile(float4* __restrict__ E4, float* __restrict__ EW,
                                               int* __restrict__ out, unsigned* __restrict__ sCol,
                                               float* __restrict__ sSum, const TileArgs& a) {
    constexpr int H = kTileY + 2 * R;
    constexpr int Wo = kTileX + 2 * R;
    constexpr int Q = (R + 1 + 3) / 4;
    constexpr int EWS = Shape<RMax>::kEWStride;
    const int t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31;

    // ---- table phase (complete_superposition.cu:298-307) --------------------
    // Sources without dose get zero rows, so the accumulation needs no per-source
    // test; sCol[sx] collects the depositing sources of every source column (one
    // shared OR per depositing source) and sSum[sy] the dose of every source row.
    {
        const float dose = a.idd[a.src];
        const bool live = dose > 0.0f;
        if (live) atomicOr(&sCol[lane], 1u << warp);
        float rowDose = live ? dose : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rowDose += __shfl_xor_sync(0xffffffffu, rowDose, o);
        if (lane == 0) sSum[warp] = rowDose;
        float e[4 * Q];
        if (live) {
            float row[R + 1];
            superposition_row<R>(a.rsig[a.src], row);
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
        // H and Wo are even and `out` is 16-byte aligned.
        for (int i = t; i < H * Wo / 4; i += kThreads) reinterpret_cast<int4*>(out)[i] = make_int4(0, 0, 0, 0);
    }
    __syncthreads();

    // Fixed-point scale: 2^(30 - ex) with total < 2^ex, so total * scale < 2^30.
    float total = 0.0f;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) total += sSum[w];
    int ex;
    frexpf(total, &ex);
    const float scale = ldexpf(1.0f, min(30 - ex, 126));
    const float invScale = 1.0f / scale;

    // ---- accumulation phase --------------------------------------------------
    {
        // A source column's footprint is the same column vector at offsets +d and -d
        // (the weights depend on |d| only). Up to radius kSplitR one lane per (source
        // column, |d|) pair accumulates it once and adds it to both output columns;
        // wider footprints keep one lane per signed offset (their doubled flushes
        // cost more than the saved FMAs).
        constexpr bool kMirror = R <= kSplitR;
        constexpr int M = kMirror ? R + 1 : 2 * R + 1;             // pairs per source column
        constexpr bool kGrouped = M <= 32;
        constexpr int G = kGrouped ? 32 / M : 1;                   // source columns per instruction
        constexpr int S = kGrouped ? (32 + G - 1) / G : 1;         // column spacing
        // Otherwise the tile's 32 * M pairs are dealt out 32 per instruction.
        constexpr int kPairs = kTileX * M;
        constexpr int kUnits = kGrouped ? S : (kPairs + 31) / 32;
        // Depositing sources of source column `lane`, as an 8-bit mask over sy.
        const unsigned colBits = sCol[lane];
#pragma unroll 1
        for (int u = warp; u < kUnits; u += kWarps) {
            int sx, d;  // d: |d| when mirrored, else the signed offset
            bool valid;
            if (kGrouped) {
                const int g = lane / M;
                d = lane - g * M;
                sx = u + g * S;
                valid = g < G && sx < kTileX;
            } else {
                const int pr = u * 32 + lane;
                sx = pr / M;
                d = pr - sx * M;
                valid = pr < kPairs;
            }
            if (!kMirror) d -= R;
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
                // Lets the loads of the next source overlap this pair's FMAs but keeps
                // later sources' loads from being hoisted (which would hold every row
                // of the column in registers).
                if (sy & 1) asm volatile("" ::: "memory");
            }
            if (colLive) {
                int q[H];
#pragma unroll
                for (int i = 0; i < H; ++i) q[i] = __float2int_rn(acc[i] * scale);
                int* col = out + sx + R + d;
#pragma unroll
                for (int i = 0; i < H; ++i) atomicAdd(col + i * Wo, q[i]);
                if (kMirror && d > 0) {
                    col = out + sx + R - d;
#pragma unroll
                    for (int i = 0; i < H; ++i) atomicAdd(col + i * Wo, q[i]);
                }
            }
        }
    }
    __syncthreads();

    // ---- write-out -------------------------------------------------------------
    // The column masks were last read before the barrier: clear them for the next tile.
    if (t < kTileX) sCol[t] = 0;
    for (int i = t; i < H * Wo; i += kThreads) {
        const int q = out[i];
        const int oy = i / Wo, ox = i - oy * Wo;
        if (q != 0) atomicAdd(a.dst + static_cast<size_t>(oy) * a.bevX + ox, float(q) * invScale);
    }
}

// Paired variant of superpose_tile for radii up to kSplitR. A lane is one column
// distance |d| of one column pair (2p, 2p+1): it keeps both columns' footprint
// heights as register pairs and adds (idd_a e_a(d), idd_b e_b(d)) * (e_a(k), e_b(k))
// to rows sy+R+-k with one packed FP32x2 FMA per row. The table phase, fixed-point
// flush and write-out are those of superpose_tile.
template <int R, int RMax>
__device__ __forceinline__ void superpose_tile_paired(float4* __restrict__ E2, float2* __restrict__ EW2,
                                                      int* __restrict__ out, unsigned* __restrict__ sCol,
                                                      float* __restrict__ sSum, const TileArgs& a) {
    constexpr int H = kTileY + 2 * R;
    constexpr int Wo = kTileX + 2 * R;
    constexpr int Q2 = (R + 2) / 2;
    constexpr int EWS = PairShape<RMax>::kEW2;
    const int t = threadIdx.x;
    const int warp = t >> 5, lane = t & 31;

    // ---- table phase (complete_superposition.cu:298-307) --------------------
    {
        const float dose = a.idd[a.src];
        const bool live = dose > 0.0f;
        if (live) atomicOr(&sCol[lane], 1u << warp);
        float rowDose = live ? dose : 0.0f;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) rowDose += __shfl_xor_sync(0xffffffffu, rowDose, o);
        if (lane == 0) sSum[warp] = rowDose;
        float e[R + 1];
        if (live) {
            superposition_row<R>(a.rsig[a.src], e);
        } else {
#pragma unroll
            for (int k = 0; k <= R; ++k) e[k] = 0.0f;
        }
        // This source is half h of column pair p: its e(k) goes to component
        // (k & 1) * 2 + h of float4 k / 2 of its (row, pair) slot, its idd * e(k) to
        // component h of float2 k of its (row, pair) row.
        const int pr = lane >> 1, h = lane & 1;
        float* e2 = reinterpret_cast<float*>(E2 + warp * kPairs + pair_slot(pr)) + h;
        float* ew = reinterpret_cast<float*>(EW2 + (warp * kPairs + pr) * EWS) + h;
#pragma unroll
        for (int k = 0; k <= R; ++k) {
            e2[(k >> 1) * kPairSlots * 4 + (k & 1) * 2] = e[k];
            ew[2 * k] = dose * e[k];
        }
        if ((R & 1) == 0) e2[(R >> 1) * kPairSlots * 4 + 2] = 0.0f;  // k = R + 1 of the last float4
        // H and Wo are even and `out` is 16-byte aligned.
        for (int i = t; i < H * Wo / 4; i += kThreads) reinterpret_cast<int4*>(out)[i] = make_int4(0, 0, 0, 0);
    }
    __syncthreads();

    // Fixed-point scale: 2^(30 - ex) with total < 2^ex, so total * scale < 2^30.
    float total = 0.0f;
#pragma unroll
    for (int w = 0; w < kWarps; ++w) total += sSum[w];
    int ex;
    frexpf(total, &ex);
    const float scale = ldexpf(1.0f, min(30 - ex, 126));
    const float invScale = 1.0f / scale;

    // ---- accumulation phase --------------------------------------------------
    {
        constexpr int M = R + 1;                         // distances |d| per column pair
        constexpr int G = (32 / M) < kPairs ? (32 / M) : kPairs;  // column pairs per instruction
        constexpr int S = (kPairs + G - 1) / G;          // pair spacing = units per tile
        const unsigned colBits = sCol[lane];
#pragma unroll 1
        for (int u = warp; u < S; u += kWarps) {
            const int g = lane / M;
            int d = lane - g * M;
            int pr = u + g * S;
            const bool valid = g < G && pr < kPairs;
            if (!valid) {
                pr = 0;
                d = 0;
            }
            const unsigned colA = __shfl_sync(0xffffffffu, colBits, 2 * pr);
            const unsigned colB = __shfl_sync(0xffffffffu, colBits, 2 * pr + 1);
            const bool liveA = valid && colA != 0u, liveB = valid && colB != 0u;
            if (!__any_sync(0xffffffffu, liveA || liveB)) continue;
            // Lanes outside the footprint read pair 0 and are never flushed.
            const float2* ewCol = EW2 + pr * EWS + d;
            const float4* eCol = E2 + pair_slot(pr);
            float2 acc[H];
#pragma unroll
            for (int i = 0; i < H; ++i) acc[i] = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int sy = 0; sy < kTileY; ++sy) {
                const float2 w = ewCol[sy * kPairs * EWS];
#pragma unroll
                for (int q = 0; q < Q2; ++q) {
                    const float4 v = eCol[q * kPairSlots + sy * kPairs];
                    const float2 ev[2] = {make_float2(v.x, v.y), make_float2(v.z, v.w)};
#pragma unroll
                    for (int c = 0; c < 2; ++c) {
                        const int k = 2 * q + c;
                        if (k <= R) {
                            acc[sy + R + k] = __ffma2_rn(w, ev[c], acc[sy + R + k]);
                            if (k > 0) acc[sy + R - k] = __ffma2_rn(w, ev[c], acc[sy + R - k]);
                        }
                    }
                }
                if (sy & 1) asm volatile("" ::: "memory");
            }
            if (liveA) {
                int* col = out + 2 * pr + R + d;
#pragma unroll
                for (int i = 0; i < H; ++i) {
                    const int q = __float2int_rn(acc[i].x * scale);
                    atomicAdd(col + i * Wo, q);
                    if (d > 0) atomicAdd(col - 2 * d + i * Wo, q);
                }
            }
            if (liveB) {
                int* col = out + 2 * pr + 1 + R + d;
#pragma unroll
                for (int i = 0; i < H; ++i) {
                    const int q = __float2int_rn(acc[i].y * scale);
                    atomicAdd(col + i * Wo, q);
                    if (d > 0) atomicAdd(col - 2 * d + i * Wo, q);
                }
            }
        }
    }
    __syncthreads();

    // ---- write-out -------------------------------------------------------------
    if (t < kTileX) sCol[t] = 0;
    for (int i = t; i < H * Wo; i += kThreads) {
        const int q = out[i];
        const int oy = i / Wo, ox = i - oy * Wo;
        if (q != 0) atomicAdd(a.dst + static_cast<size_t>(oy) * a.bevX + ox, float(q) * invScale);
    }
}

// Chain of compile-time radii RLo..RHi; returns false if r is outside it.
template <int R, int RHi, int RMax>
__device__ __forceinline__ bool dispatch_radius(int r, float4* E4, float* EW, int* out, unsigned* sCol,
                                                float* sSum, const TileArgs& a) {
    if (r == R) {
        if constexpr (RMax <= kSplitR)
            superpose_tile_paired<R, RMax>(E4, reinterpret_cast<float2*>(EW), out, sCol, sSum, a);
        else
            superpose_tile<R, RMax>(E4, EW, out, sCol, sSum, a);
        return true;
    }
    if constexpr (R < RHi) return dispatch_radius<R + 1, RHi, RMax>(r, E4, EW, out, sCol, sSum, a);
    return false;
}

// Persistent CTA loop over the work items [begin, end) of radii RLo..RHi, claimed
// one at a time through `counter` (the next claim is issued before the current
// tile runs so that its latency is hidden).
template <int RLo, int RHi, int MinBlocks>
__global__ void __launch_bounds__(kThreads, MinBlocks)
superpose_kernel(BeamGeomDev g, const float* __restrict__ idd, const float* __restrict__ rsig,
                 const int4* __restrict__ work, BeamStateDev* __restrict__ beam, float* __restrict__ bev, int range) {
    extern __shared__ __align__(16) float sm[];
    constexpr bool kPaired = RHi <= kSplitR;
    // Wide radii: E4 = [Q][256] e_s(4q..4q+3) at slot sy*32+e4_col(sx), EW = [256][EWS]
    // idd_s e_s(k). Paired radii: E4 = [Q2][128] pair float4s at slot sy*16+pair_slot(p),
    // EW = [128][EW2] float2 (idd_a e_a(k), idd_b e_b(k)). Then the [8+2R][32+2R]
    // fixed-point footprint.
    constexpr size_t kE4Floats = kPaired ? size_t(PairShape<RHi>::kQ2) * kPairSlots * 4
                                         : size_t(Shape<RHi>::kQ) * kThreads * 4;
    constexpr size_t kEWFloats = kPaired ? size_t(kPairSlots) * PairShape<RHi>::kEW2 * 2
                                         : size_t(kThreads) * Shape<RHi>::kEWStride;
    float4* E4 = reinterpret_cast<float4*>(sm);
    float* EW = sm + kE4Floats;
    int* out = reinterpret_cast<int*>(EW + kEWFloats);
    __shared__ int sItem[2];
    __shared__ unsigned sCol[kTileX];     // per source column: depositing sources over sy
    __shared__ float sSum[kTileY];

    const int t = threadIdx.x;
    // Range 0: R > kSplitR, 1: kSplitR3 < R <= kSplitR, 3: kSplitR2 < R <= kSplitR3,
    // 2: R <= kSplitR2 (the work list holds them in the order 0, 1, 3, 2).
    int begin, end, *counter;
    if (range == 0) {
        begin = 0, end = beam->workSplit, counter = &beam->workNext;
    } else if (range == 1) {
        begin = beam->workSplit, end = beam->workSplit3, counter = &beam->workNextSmall;
    } else if (range == 3) {
        begin = beam->workSplit3, end = beam->workSplit2, counter = &beam->workNextMid;
    } else {
        begin = beam->workSplit2, end = beam->workCount, counter = &beam->workNextTiny;
    }
    const size_t padPlane = static_cast<size_t>(g.pitchX) * g.pitchY;
    const size_t layerStride = static_cast<size_t>(g.steps) * padPlane;
    const size_t bevPlane = static_cast<size_t>(g.bevX) * g.bevY;

    if (t == 0) sItem[0] = atomicAdd(counter, 1);
    if (t < kTileX) sCol[t] = 0;
    __syncthreads();
    int buf = 0;
    for (;;) {
        const int w = begin + sItem[buf];
        if (w >= end) break;
        if (t == 0) sItem[buf ^ 1] = atomicAdd(counter, 1);
        const int4 it = work[w];
        const int lc = it.x, tile = it.y, zRel = it.z, R = it.w;
        const int tx = tile % g.tilesX, ty = tile / g.tilesX;
        TileArgs a;
        a.idd = idd;
        a.rsig = rsig;
        a.bev = bev;
        a.src = lc * layerStride + zRel * padPlane + static_cast<size_t>(ty * kTileY + (t >> 5)) * g.pitchX +
                tx * kTileX + (t & 31);
        a.dst = bev + static_cast<size_t>(zRel) * bevPlane + static_cast<size_t>(ty * kTileY - R + kMaxR) * g.bevX +
                (tx * kTileX - R + kMaxR);
        a.bevX = g.bevX;
        if (!dispatch_radius<RLo, RHi, RHi>(R, E4, EW, out, sCol, sSum, a)) {
            if (t == 0) atomicOr(&beam->errorFlags, 2);
        }
        // Every thread is past the tile (and has read sItem[buf]) before the
        // next claim lands in that slot.
        __syncthreads();
        buf ^= 1;
    }
}

template <int RLo, int RHi, int MinBlocks>
cudaError_t launch_range(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                         BeamStateDev* beam, float* bev, int gridBlocks, int range, cudaStream_t s) {
    auto k = superpose_kernel<RLo, RHi, MinBlocks>;
    const size_t smem = RHi <= kSplitR ? PairShape<RHi>::kSmemBytes : Shape<RHi>::kSmemBytes;
    cudaError_t e = set_smem_limit(reinterpret_cast<const void*>(k), smem);
    if (e != cudaSuccess) return e;
    k<<<gridBlocks, kThreads, smem, s>>>(g, idd, rsigma, work, beam, bev, range);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_superpose(const BeamGeomDev& g, const float* idd, const float* rsigma, const int4* work,
                             BeamStateDev* beam, float* bev, int numSMs, cudaStream_t s) {
    // Items are sorted by descending radius: the wide radii come first.
    cudaError_t e = launch_range<kSplitR + 1, kMaxR, 2>(g, idd, rsigma, work, beam, bev, numSMs * 2, 0, s);
    if (e != cudaSuccess) return e;
    e = launch_range<kSplitR3 + 1, kSplitR, kMidBlocks>(g, idd, rsigma, work, beam, bev, numSMs * kMidBlocks, 1, s);
    if (e != cudaSuccess) return e;
    e = launch_range<kSplitR2 + 1, kSplitR3, kMidNarrowBlocks>(g, idd, rsigma, work, beam, bev,
                                                                numSMs * kMidNarrowBlocks, 3, s);
    if (e != cudaSuccess) return e;
    return launch_range<0, kSplitR2, kNarrowBlocks>(g, idd, rsigma, work, beam, bev, numSMs * kNarrowBlocks, 2, s);
}

}  // namespace pbs
