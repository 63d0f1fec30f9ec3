// Spot-preserving operator mode: the batch plan of the reference's operator-mode
// helper (include/core/rtd_operator_mode.h:43-111), and a dose-influence export
// in compressed sparse columns (one column per spot, one row per dose voxel) that
// the reference plans for but does not compute (cuCalDose3 only zeroes its CSC
// outputs, raytracedicom_pybind.cpp:1955-2053).
//
// Column j of the influence matrix is the dose of the beam with spot j at unit
// weight and every other spot at zero: the same plan, ray grid and lattice as the
// whole beam, so that A . w equals the forward dose of w up to the live-ray mask
// (ray weight < 1e-6, idd_sigma.cu:78) and rounding. Each column is compacted on
// the device from the FP64 grid's dirty box in ascending voxel order, with its
// offsets scanned on the device, so a batch of columns needs one synchronisation.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>
#include <cmath>
#include <string>
#include <vector>

#include "context.h"
#include "../../include/subsecondpbs.h"

namespace pbs {

namespace {

constexpr int kOpThreads = 256;
constexpr int kOpPasses = 8;
constexpr int kOpChunk = kOpThreads * kOpPasses;  // box voxels per chunk
constexpr int kOpGridBlocks = 148 * 4;              // blocks striding over a column's chunks

// The columns of one export share the beam's geometry and so its trace: the first
// column traces into this store's buffer and the others skip the tracer and wait
// on its event (the TraceStore contract of Context::run_beam).
struct ColumnTraces : TraceStore {
    DevBuf mem;
    cudaEvent_t ready = nullptr;
    TraceSlot slot{};
    bool have = false;

    ~ColumnTraces() override {
        if (ready) cudaEventDestroy(ready);
        mem.release();
    }
    int acquire(Context&, const BeamGeomDev& g, TraceSlot& ts) override {
        if (!have) {
            const size_t rays = size_t(g.rayX) * g.rayY, S = size_t(g.steps);
            if (int rc = mem.ensure(trace_bytes(S, rays))) return rc;
            if (!ready && cudaEventCreateWithFlags(&ready, cudaEventDisableTiming) != cudaSuccess)
                return PBS_ERR_CUDA;
            auto up = [](size_t n) { return (n + 255) / 256 * 256; };
            char* p = static_cast<char*>(mem.ptr);
            slot.dens = reinterpret_cast<float*>(p);
            p += up(S * rays * 4);
            slot.wepl = reinterpret_cast<float*>(p);
            p += up(S * rays * 4);
            slot.firstIn = reinterpret_cast<int*>(p);
            p += up(rays * 4);
            slot.firstOut = reinterpret_cast<int*>(p);
            p += up(rays * 4);
            slot.weplMin = reinterpret_cast<float*>(p);
            p += up(S * 4);
            slot.inOut = reinterpret_cast<int*>(p);
            slot.ready = ready;
        }
        ts = slot;
        ts.traced = have;
        return PBS_OK;
    }
    int traced(Context& c, TraceSlot&) override {
        if (cudaEventRecord(ready, c.stream) != cudaSuccess) return PBS_ERR_CUDA;
        have = true;
        return PBS_OK;
    }
};

// Installs a ColumnTraces on a context without a trace store of its own for the
// lifetime of the guard.
struct ColumnTraceGuard {
    Context& c;
    ColumnTraces traces;
    bool installed;
    explicit ColumnTraceGuard(Context& ctx) : c(ctx), installed(ctx.traceStore == nullptr) {
        if (installed) c.traceStore = &traces;
    }
    ~ColumnTraceGuard() {
        if (installed) c.traceStore = nullptr;
    }
};

// An inclusive voxel box of the dose grid walked in grid order (x fastest).
struct OpBox {
    int lo[3];
    int ext[3];
    int X, Y;
    long long n;  // voxels in the box
};

__device__ __forceinline__ long long box_to_grid(const OpBox& a, long long b) {
    const int bx = int(b % a.ext[0]);
    const long long r = b / a.ext[0];
    const int by = int(r % a.ext[1]);
    const int bz = int(r / a.ext[1]);
    return (static_cast<long long>(a.lo[2] + bz) * a.Y + (a.lo[1] + by)) * a.X + (a.lo[0] + bx);
}

// The voxels a beam's transfer can have written: its device-side transfer box with
// the launch's block rounding in x (32) and y (8), as transfer_kernel walks it.
__device__ __forceinline__ void written_box(const BeamStateDev* bs, int X, int Y, int lo[3], int hi[3]) {
    if (!bs || !bs->transferValid) {
        lo[0] = lo[1] = lo[2] = INT_MAX;
        hi[0] = hi[1] = hi[2] = INT_MIN;
        return;
    }
    for (int i = 0; i < 3; ++i) lo[i] = bs->transferStart[i];
    hi[0] = lo[0] + min(((bs->transferMax[0] - lo[0] + 1 + 31) / 32) * 32, X - lo[0]) - 1;
    hi[1] = lo[1] + min(((bs->transferMax[1] - lo[1] + 1 + 7) / 8) * 8, Y - lo[1]) - 1;
    hi[2] = bs->transferMax[2];
}

// The part of the column's host box `a` that the primary and halo transfers can
// have written; every other voxel of `a` is zero.
__device__ __forceinline__ OpBox column_box(const OpBox& a, const BeamStateDev* pb, const BeamStateDev* nb) {
    int l0[3], h0[3], l1[3], h1[3];
    written_box(pb, a.X, a.Y, l0, h0);
    written_box(nb, a.X, a.Y, l1, h1);
    OpBox e = a;
    e.n = 1;
    for (int i = 0; i < 3; ++i) {
        const int lo = max(min(l0[i], l1[i]), a.lo[i]);
        const int hi = min(max(h0[i], h1[i]), a.lo[i] + a.ext[i] - 1);
        e.lo[i] = lo;
        e.ext[i] = hi >= lo ? hi - lo + 1 : 0;
        e.n *= e.ext[i];
    }
    return e;
}

// Entries above the threshold in each kOpChunk-voxel chunk of the column's box
// (column_box: known on the device only), the blocks striding over the chunks; block
// 0 also stores the number of chunks for the scan.
__global__ void __launch_bounds__(kOpThreads) influence_count_kernel(const double* __restrict__ dose, OpBox host,
                                                                     const BeamStateDev* __restrict__ pb,
                                                                     const BeamStateDev* __restrict__ nb,
                                                                     double thr, long long* __restrict__ blockOff,
                                                                     long long* __restrict__ nChunksOut) {
    const OpBox a = column_box(host, pb, nb);
    const long long nChunks = (a.n + kOpChunk - 1) / kOpChunk;
    if (blockIdx.x == 0 && threadIdx.x == 0) *nChunksOut = nChunks;
    for (long long ch = blockIdx.x; ch < nChunks; ch += gridDim.x) {
        const long long base = ch * kOpChunk;
        int c = 0;
        for (int p = 0; p < kOpPasses; ++p) {
            const long long b = base + p * kOpThreads + threadIdx.x;
            const bool keep = b < a.n && fabs(dose[box_to_grid(a, b)]) > thr;
            c += __syncthreads_count(keep);
        }
        if (threadIdx.x == 0) blockOff[ch] = c;
    }
}

// One block: chunk counts -> absolute exclusive offsets (starting at colPtr[col]),
// and colPtr[col + 1] = colPtr[col] + entries of the column.
__global__ void __launch_bounds__(1024) influence_scan_kernel(long long* __restrict__ blockOff,
                                                              const long long* __restrict__ nChunksIn,
                                                              long long* __restrict__ colPtr, int col) {
    __shared__ long long carry;
    __shared__ long long warpSums[32];
    const int nBlocks = static_cast<int>(*nChunksIn);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) carry = colPtr[col];
    __syncthreads();
    for (int start = 0; start < nBlocks; start += 1024) {
        const int i = start + threadIdx.x;
        const long long v = i < nBlocks ? blockOff[i] : 0;
        long long x = v;
        for (int o = 1; o < 32; o <<= 1) {
            const long long y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warpSums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            long long s = warpSums[lane];
            for (int o = 1; o < 32; o <<= 1) {
                const long long y = __shfl_up_sync(0xffffffffu, s, o);
                if (lane >= o) s += y;
            }
            warpSums[lane] = s;
        }
        __syncthreads();
        const long long incl = x + (warp > 0 ? warpSums[warp - 1] : 0);
        const long long c0 = carry;
        if (i < nBlocks) blockOff[i] = c0 + incl - v;
        __syncthreads();
        if (threadIdx.x == 1023) carry = c0 + incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) colPtr[col + 1] = carry;
}

// Ordered compaction of each chunk, the blocks striding over the chunks as in the
// count: entries keep the box order, which is ascending voxel order. Entries past
// `cap` are counted but not written. Every voxel of the box is zeroed once read, so
// the grid is zero again for the next column.
__global__ void __launch_bounds__(kOpThreads) influence_write_kernel(double* __restrict__ dose, OpBox host,
                                                                     const BeamStateDev* __restrict__ pb,
                                                                     const BeamStateDev* __restrict__ nb,
                                                                     double thr, const long long* __restrict__ blockOff,
                                                                     int* __restrict__ rows, float* __restrict__ vals,
                                                                     long long cap) {
    __shared__ int warpCounts[kOpThreads / 32];
    const OpBox a = column_box(host, pb, nb);
    const long long nChunks = (a.n + kOpChunk - 1) / kOpChunk;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (long long ch = blockIdx.x; ch < nChunks; ch += gridDim.x) {
        long long pos = blockOff[ch];
        const long long base = ch * kOpChunk;
        for (int p = 0; p < kOpPasses; ++p) {
            const long long b = base + p * kOpThreads + threadIdx.x;
            long long g = 0;
            double v = 0.0;
            bool keep = false;
            if (b < a.n) {
                g = box_to_grid(a, b);
                v = dose[g];
                dose[g] = 0.0;
                keep = fabs(v) > thr;
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) warpCounts[warp] = __popc(m);
            __syncthreads();
            int before = 0, total = 0;
            for (int w = 0; w < kOpThreads / 32; ++w) {
                const int c = warpCounts[w];
                if (w < warp) before += c;
                total += c;
            }
            if (keep) {
                const long long at = pos + before + __popc(m & ((1u << lane) - 1u));
                if (at < cap) {
                    rows[at] = static_cast<int>(g);
                    vals[at] = static_cast<float>(v);
                }
            }
            pos += total;
            __syncthreads();
        }
    }
}

// ---- Batched columns: buffer q (blockIdx.y) of colDose, laid out over fb --------

// Voxel b of a column box [lo, hi] (x fastest): its linear grid index and its index
// in a column buffer over fb.
__device__ __forceinline__ void col_voxel(const int lo[3], const int ext[3], const ColBox& fb, int X, int Y,
                                          long long b, long long& g, size_t& at) {
    const int bx = int(b % ext[0]);
    const long long r = b / ext[0];
    const int by = int(r % ext[1]);
    const int bz = int(r / ext[1]);
    const int x = lo[0] + bx, y = lo[1] + by, z = lo[2] + bz;
    g = (static_cast<long long>(z) * Y + y) * X + x;
    at = (static_cast<size_t>(z - fb.lo[2]) * fb.ext[1] + (y - fb.lo[1])) * fb.ext[0] + (x - fb.lo[0]);
}

__device__ __forceinline__ long long col_box(const LayerStateDev& st, const ColBox& fb, int X, int Y, int lo[3],
                                             int ext[3]) {
    int hi[3];
    if (!column_written_box(st, X, Y, fb, lo, hi)) return 0;
    long long n = 1;
    for (int i = 0; i < 3; ++i) {
        ext[i] = hi[i] - lo[i] + 1;
        n *= ext[i];
    }
    return n;
}

// Entries above the threshold per kOpChunk-voxel chunk of each column's box; the
// column's chunk count goes to nChunks[q].
__global__ void __launch_bounds__(kOpThreads) col_count_kernel(const double* __restrict__ colDose, ColBox fb,
                                                               const LayerStateDev* __restrict__ ls, int X, int Y,
                                                               double thr, long long* __restrict__ blockOff,
                                                               int maxChunks, long long* __restrict__ nChunks) {
    const int q = blockIdx.y;
    int lo[3], ext[3];
    const long long n = col_box(ls[q], fb, X, Y, lo, ext);
    const long long nCh = (n + kOpChunk - 1) / kOpChunk;
    if (blockIdx.x == 0 && threadIdx.x == 0) nChunks[q] = nCh;
    const size_t fbN = static_cast<size_t>(fb.ext[0]) * fb.ext[1] * fb.ext[2];
    const double* d = colDose + static_cast<size_t>(q) * fbN;
    for (long long ch = blockIdx.x; ch < nCh; ch += gridDim.x) {
        int c = 0;
        for (int p = 0; p < kOpPasses; ++p) {
            const long long b = ch * kOpChunk + p * kOpThreads + threadIdx.x;
            bool keep = false;
            if (b < n) {
                long long g;
                size_t at;
                col_voxel(lo, ext, fb, X, Y, b, g, at);
                keep = fabs(d[at]) > thr;
            }
            c += __syncthreads_count(keep);
        }
        if (threadIdx.x == 0) blockOff[static_cast<size_t>(q) * maxChunks + ch] = c;
    }
}

// One block: the columns' chunk counts -> absolute offsets, column after column
// (colPtr[col0 + q + 1] = colPtr[col0 + q] + entries of column q).
__global__ void __launch_bounds__(1024) col_scan_kernel(long long* __restrict__ blockOff, int maxChunks,
                                                        const long long* __restrict__ nChunks, int nCols,
                                                        long long* __restrict__ colPtr, int col0) {
    __shared__ long long carry;
    __shared__ long long warpSums[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int q = 0; q < nCols; ++q) {
        long long* off = blockOff + static_cast<size_t>(q) * maxChunks;
        const int nBlocks = static_cast<int>(nChunks[q]);
        if (threadIdx.x == 0) carry = colPtr[col0 + q];
        __syncthreads();
        for (int start = 0; start < nBlocks; start += 1024) {
            const int i = start + threadIdx.x;
            const long long v = i < nBlocks ? off[i] : 0;
            long long x = v;
            for (int o = 1; o < 32; o <<= 1) {
                const long long y = __shfl_up_sync(0xffffffffu, x, o);
                if (lane >= o) x += y;
            }
            if (lane == 31) warpSums[warp] = x;
            __syncthreads();
            if (warp == 0) {
                long long t = warpSums[lane];
                for (int o = 1; o < 32; o <<= 1) {
                    const long long y = __shfl_up_sync(0xffffffffu, t, o);
                    if (lane >= o) t += y;
                }
                warpSums[lane] = t;
            }
            __syncthreads();
            const long long incl = x + (warp > 0 ? warpSums[warp - 1] : 0);
            const long long c0 = carry;
            if (i < nBlocks) off[i] = c0 + incl - v;
            __syncthreads();
            if (threadIdx.x == 1023) carry = c0 + incl;
            __syncthreads();
        }
        if (threadIdx.x == 0) colPtr[col0 + q + 1] = carry;
        __syncthreads();
    }
}

// Ordered compaction of each column's chunks (rows = linear grid indices, ascending);
// every voxel read is zeroed, so the buffers are zero for the next batch.
__global__ void __launch_bounds__(kOpThreads) col_write_kernel(double* __restrict__ colDose, ColBox fb,
                                                               const LayerStateDev* __restrict__ ls, int X, int Y,
                                                               double thr, const long long* __restrict__ blockOff,
                                                               int maxChunks, int* __restrict__ rows,
                                                               float* __restrict__ vals, long long cap) {
    __shared__ int warpCounts[kOpThreads / 32];
    const int q = blockIdx.y;
    int lo[3], ext[3];
    const long long n = col_box(ls[q], fb, X, Y, lo, ext);
    const long long nCh = (n + kOpChunk - 1) / kOpChunk;
    const size_t fbN = static_cast<size_t>(fb.ext[0]) * fb.ext[1] * fb.ext[2];
    double* d = colDose + static_cast<size_t>(q) * fbN;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (long long ch = blockIdx.x; ch < nCh; ch += gridDim.x) {
        long long pos = blockOff[static_cast<size_t>(q) * maxChunks + ch];
        for (int p = 0; p < kOpPasses; ++p) {
            const long long b = ch * kOpChunk + p * kOpThreads + threadIdx.x;
            long long g = 0;
            double v = 0.0;
            bool keep = false;
            if (b < n) {
                size_t at;
                col_voxel(lo, ext, fb, X, Y, b, g, at);
                v = d[at];
                d[at] = 0.0;
                keep = fabs(v) > thr;
            }
            const unsigned m = __ballot_sync(0xffffffffu, keep);
            if (lane == 0) warpCounts[warp] = __popc(m);
            __syncthreads();
            int before = 0, total = 0;
            for (int w = 0; w < kOpThreads / 32; ++w) {
                const int c = warpCounts[w];
                if (w < warp) before += c;
                total += c;
            }
            if (keep) {
                const long long at = pos + before + __popc(m & ((1u << lane) - 1u));
                if (at < cap) {
                    rows[at] = static_cast<int>(g);
                    vals[at] = static_cast<float>(v);
                }
            }
            pos += total;
            __syncthreads();
        }
    }
}

// Row norms of a batch of columns: every voxel of fb adds the squares of the columns
// whose box holds it, in column order (deterministic), and zeroes them.
constexpr int kMaxColumnsPerBatch = 64;
__global__ void __launch_bounds__(kOpThreads) col_norm_kernel(double* __restrict__ colDose, ColBox fb,
                                                              const LayerStateDev* __restrict__ ls, int nCols, int X,
                                                              int Y, double* __restrict__ norm) {
    __shared__ int sLo[kMaxColumnsPerBatch][3], sHi[kMaxColumnsPerBatch][3];
    __shared__ int sAny[kMaxColumnsPerBatch];
    for (int q = threadIdx.x; q < nCols; q += blockDim.x) {
        int lo[3], hi[3];
        sAny[q] = column_written_box(ls[q], X, Y, fb, lo, hi);
        for (int i = 0; i < 3; ++i) {
            sLo[q][i] = lo[i];
            sHi[q][i] = hi[i];
        }
    }
    __syncthreads();
    const size_t fbN = static_cast<size_t>(fb.ext[0]) * fb.ext[1] * fb.ext[2];
    for (size_t at = blockIdx.x * size_t(blockDim.x) + threadIdx.x; at < fbN; at += size_t(gridDim.x) * blockDim.x) {
        const int x = fb.lo[0] + static_cast<int>(at % fb.ext[0]);
        const size_t r = at / fb.ext[0];
        const int y = fb.lo[1] + static_cast<int>(r % fb.ext[1]);
        const int z = fb.lo[2] + static_cast<int>(r / fb.ext[1]);
        double acc = 0.0;
        bool any = false;
        for (int q = 0; q < nCols; ++q) {
            if (!sAny[q] || x < sLo[q][0] || x > sHi[q][0] || y < sLo[q][1] || y > sHi[q][1] || z < sLo[q][2] ||
                z > sHi[q][2])
                continue;
            double* d = colDose + static_cast<size_t>(q) * fbN + at;
            const double v = *d;
            *d = 0.0;
            acc += v * v;
            any = true;
        }
        if (any) norm[(static_cast<long long>(z) * Y + y) * X + x] += acc;
    }
}

// The voxels the column just transferred can have written: the grid's dirty box,
// or the whole grid when the context does not track one.
OpBox dirty_op_box(const Context& c) {
    OpBox a{};
    int lo[3], hi[3];
    const bool boxed = c.doseBoxed && !c.doseExposed;
    for (int i = 0; i < 3; ++i) {
        lo[i] = boxed ? c.dirtyLo[i] : 0;
        hi[i] = boxed ? c.dirtyHi[i] : c.doseGrid.dims[i] - 1;
    }
    const bool empty = hi[0] < lo[0] || hi[1] < lo[1] || hi[2] < lo[2];
    for (int i = 0; i < 3; ++i) {
        a.lo[i] = lo[i];
        a.ext[i] = empty ? 0 : hi[i] - lo[i] + 1;
    }
    a.X = c.doseGrid.dims[0];
    a.Y = c.doseGrid.dims[1];
    a.n = empty ? 0 : static_cast<long long>(a.ext[0]) * a.ext[1] * a.ext[2];
    return a;
}

// Spots per batched pass of an influence export (one plan layer and one BEV volume
// and dose buffer each): at most the layers of one chunk's layer plan, and as many
// as fit kColumnBudget bytes and a quarter of the device. A pass whose buffers do not
// fit the free memory is retried with half as many spots (run_column_batches).
constexpr long long kColumnBudget = 6LL << 30;

int column_batch_size(const Context& c, const BeamPlan& base, ColBox& fb, size_t& maxChunks) {
    size_t cells = 0, perColumn = 0;
    c.column_layout(base, fb, cells, perColumn);
    const size_t fbN = size_t(fb.ext[0]) * fb.ext[1] * fb.ext[2];
    maxChunks = std::max<size_t>((fbN + kOpChunk - 1) / kOpChunk, 1);
    if (c.compatBevZShift) return kMaxColumnsPerBatch;  // one layer at a time through the dose grid
    size_t freeB = 0, totalB = 0;
    long long budget = kColumnBudget;
    if (cudaMemGetInfo(&freeB, &totalB) == cudaSuccess) budget = std::min<long long>(budget, (long long)(totalB / 4));
    const long long k = budget / std::max<long long>((long long)perColumn, 1);
    return static_cast<int>(std::max<long long>(1, std::min<long long>(k, kMaxColumnsPerBatch)));
}

int op_cuda(cudaError_t e, const char* where) {
    if (e == cudaSuccess) return PBS_OK;
    set_error(std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? PBS_ERR_OUT_OF_MEMORY : PBS_ERR_CUDA;
}

// Row norms of the influence matrix: the squared dose of one column added to the
// Squares of the column's dose added into the FP64 norm grid, over the part of the
// column's host box its transfers can have written (column_box); every voxel read is
// zeroed, so the grid is zero again for the next column.
__global__ void __launch_bounds__(kOpThreads) row_norm_add_kernel(double* __restrict__ dose, OpBox host,
                                                                  const BeamStateDev* __restrict__ pb,
                                                                  const BeamStateDev* __restrict__ nb,
                                                                  double* __restrict__ norm) {
    const OpBox a = column_box(host, pb, nb);
    for (long long b = blockIdx.x * static_cast<long long>(kOpThreads) + threadIdx.x; b < a.n;
         b += static_cast<long long>(gridDim.x) * kOpThreads) {
        const long long g = box_to_grid(a, b);
        const double v = dose[g];
        dose[g] = 0.0;
        norm[g] += v * v;
    }
}

// Float copy of the norm grid at the requested voxels (all voxels when null).
__global__ void __launch_bounds__(kOpThreads) row_norm_gather_kernel(const double* __restrict__ norm,
                                                                     const long long* __restrict__ voxels,
                                                                     long long n, float* __restrict__ out) {
    for (long long i = blockIdx.x * static_cast<long long>(kOpThreads) + threadIdx.x; i < n;
         i += static_cast<long long>(gridDim.x) * kOpThreads)
        out[i] = float(norm[voxels ? voxels[i] : i]);
}

}  // namespace

// rtd_operator_mode.h:43-111: the same validation (an invalid beam returns the
// fields filled so far and valid = 0), spans in layer order, and batches of at most
// max(1, maxSpotsPerBatch) consecutive spots with the layers of their first and
// last spot (the first non-empty span holding the spot, -1 if none).
int operator_batch_plan(const PbsBeamDesc& beam, int maxSpotsPerBatch, OperatorPlan& plan) {
    plan = OperatorPlan{};
    plan.totalLayers = static_cast<int>(beam.layer_spot_counts ? beam.n_layer_spot_counts : 0);
    const size_t nEnergies = beam.energies ? beam.n_energies : 0;
    if (plan.totalLayers <= 0 || static_cast<int>(nEnergies) != plan.totalLayers) return PBS_OK;
    int totalSpots = 0;
    for (int l = 0; l < plan.totalLayers; ++l) {
        if (beam.layer_spot_counts[l] < 0) return PBS_OK;
        totalSpots += beam.layer_spot_counts[l];
    }
    plan.totalSpots = totalSpots;
    if (totalSpots <= 0) return PBS_OK;
    const size_t nWeights = beam.spot_weights ? beam.n_spot_weights : 0;
    const size_t nPositions = beam.spot_positions ? beam.n_spot_positions : 0;
    const size_t nDirections = beam.spot_beam_directions ? beam.n_spot_beam_directions : 0;
    if (nWeights != 0 && static_cast<int>(nWeights) != totalSpots) return PBS_OK;
    if (nPositions != 0 && static_cast<int>(nPositions / 2u) != totalSpots) return PBS_OK;
    if (nDirections != 0 && static_cast<int>(nDirections / 3u) != totalSpots) return PBS_OK;

    const size_t nCutoffs = beam.layer_longitudinal_cutoffs ? beam.n_layer_longitudinal_cutoffs : 0;
    int running = 0;
    for (int l = 0; l < plan.totalLayers; ++l) {
        PbsOperatorLayerSpan s{};
        s.layer_index = l;
        s.spot_begin = running;
        s.spot_count = beam.layer_spot_counts[l];
        s.energy = beam.energies[l];
        s.longitudinal_cutoff = static_cast<size_t>(l) < nCutoffs ? beam.layer_longitudinal_cutoffs[l] : 0.0f;
        plan.spans.push_back(s);
        running += s.spot_count;
    }
    plan.maxSpotsPerBatch = std::max(1, maxSpotsPerBatch);
    auto layerOf = [&](int spot) {
        for (const PbsOperatorLayerSpan& s : plan.spans) {
            if (s.spot_count <= 0) continue;
            if (spot >= s.spot_begin && spot < s.spot_begin + s.spot_count) return s.layer_index;
        }
        return -1;
    };
    for (int begin = 0, index = 0; begin < totalSpots; begin += plan.maxSpotsPerBatch, ++index) {
        PbsOperatorBatch b{};
        b.batch_index = index;
        b.spot_begin = begin;
        b.spot_count = std::min(plan.maxSpotsPerBatch, totalSpots - begin);
        b.first_layer_index = layerOf(b.spot_begin);
        b.last_layer_index = layerOf(b.spot_begin + b.spot_count - 1);
        plan.batches.push_back(b);
        // A batch size that reaches past INT_MAX ends the walk instead of wrapping.
        if (begin > INT_MAX - plan.maxSpotsPerBatch) break;
    }
    plan.valid = !plan.spans.empty() && !plan.batches.empty();
    return PBS_OK;
}

// Validation and the one plan shared by every column of an influence export.
int Context::plan_columns(const PbsBeamDesc& beam, long long spotBegin, long long spotCount, const char* what,
                          ColumnPlan& cp) {
    if (int rc = op_cuda(cudaSetDevice(device), "cudaSetDevice")) return rc;
    if (!hasDose) {
        set_error("dose grid not set");
        return PBS_ERR_NOT_READY;
    }
    const std::string tag = std::string(what) + ": ";
    if (!beam.layer_spot_counts || beam.n_layer_spot_counts == 0) {
        set_error(tag + "the beam has no layer spot counts");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    long long nSpots = 0;
    for (size_t l = 0; l < beam.n_layer_spot_counts; ++l) {
        if (beam.layer_spot_counts[l] < 0) {
            set_error(tag + "negative layer spot count");
            return PBS_ERR_INVALID_ARGUMENT;
        }
        nSpots += beam.layer_spot_counts[l];
    }
    if (spotBegin < 0 || spotCount < 0 || spotBegin > nSpots || spotCount > nSpots - spotBegin ||
        spotCount > INT_MAX - 1) {
        set_error(tag + "spot range of " + std::to_string(spotCount) + " spots from " + std::to_string(spotBegin) +
                  " lies outside the beam's " + std::to_string(nSpots) + " spots");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    // One plan for every column. The beam geometry, ray grid and spot lattice do not
    // depend on the weights, so the plan is made once with every spot at unit weight
    // and a column only replaces the lattice weights by its spot's shares. A beam
    // without a raw spot lattice would fall back to the legacy CPB fluence, which
    // reads the subspot table and ignores per-spot weights: it has no columns.
    cp.unit.assign(static_cast<size_t>(nSpots), 1.0f);
    cp.beam = beam;
    cp.beam.spot_weights = cp.unit.data();
    cp.beam.n_spot_weights = cp.unit.size();
    {
        std::string err;
        if (int rc = plan_beam(cp.beam, energy, ctGrid, doseGrid, cp.base, err)) {
            set_error(tag + err);
            return rc;
        }
    }
    if (!cp.base.hasLattice) {
        set_error(tag + "needs a beam with a raw spot lattice (spot positions, weights and layer counts on one "
                        "lattice phase); the legacy CPB fluence it would fall back to ignores per-spot weights" +
                  (cp.base.lattice.failure.empty() ? std::string() : " (" + cp.base.lattice.failure + ")"));
        return PBS_ERR_UNSUPPORTED;
    }
    if (!lattice_spot_cells(cp.beam, cp.base.lattice, cp.cells, cp.shares)) {
        set_error(tag + "failed to map the spots onto the beam's lattice");
        return PBS_ERR_GEOMETRY;
    }
    return PBS_OK;
}

// Dose of spot j alone at unit weight into the (zeroed) FP64 grid, with the box of
// voxels it can have written.
int Context::run_column(ColumnPlan& cp, size_t j, int nuclear, void* boxOut, bool gridZero) {
    // The column is the dose of spot j's layer alone: the other layers' weights are
    // zero, so they add nothing, and every per-layer decision (steps, radii, work
    // items) depends on the layer's own parameters and the beam's geometry only. The
    // plan is cut down to that layer unless the biological or CarbonPBS profile
    // models, which index the beam's layers, are on.
    const size_t plane = static_cast<size_t>(cp.base.lattice.nx) * cp.base.lattice.ny;
    int layer = -1;
    for (int slot = 0; slot < 4; ++slot)
        if (cp.cells[j * 4 + slot] >= 0) layer = static_cast<int>(cp.cells[j * 4 + slot] / plane);
    const bool oneLayer = layer >= 0 && !bioModel && !carbonProfile;
    BeamPlan P;
    if (oneLayer) {
        // Copy the plan without its per-layer vectors, then give it the one layer.
        std::vector<float> weights;
        std::vector<LayerHost> layers;
        std::swap(cp.base.lattice.weights, weights);
        std::swap(cp.base.layers, layers);
        P = cp.base;
        std::swap(cp.base.lattice.weights, weights);
        std::swap(cp.base.layers, layers);
        P.numLayers = 1;
        P.layers.assign(1, cp.base.layers[static_cast<size_t>(layer)]);
        P.lattice.nl = 1;
        P.lattice.weights.assign(plane, 0.0f);
    } else {
        P = cp.base;
        std::fill(P.lattice.weights.begin(), P.lattice.weights.end(), 0.0f);
    }
    const size_t cellBase = oneLayer ? static_cast<size_t>(layer) * plane : 0;
    for (int slot = 0; slot < 4; ++slot) {
        const int c = cp.cells[j * 4 + slot];
        if (c >= 0) P.lattice.weights[static_cast<size_t>(c) - cellBase] += cp.shares[j * 4 + slot];
    }
    // A grid known to be zero only needs its dirty box forgotten.
    if (gridZero && doseBoxed && !doseExposed && !pendingDoseInit && !bioModel) {
        for (int i = 0; i < 3; ++i) {
            dirtyLo[i] = INT_MAX;
            dirtyHi[i] = -1;
        }
    } else if (int rc = reset_dose(nullptr, 0)) {
        return rc;
    }
    if (int rc = add_planned_beam(cp.beam, nuclear, std::move(P))) return rc;
    if (int rc = join_side_work()) return rc;
    OpBox& a = *static_cast<OpBox*>(boxOut);
    int lo[3], hi[3];
    for (int i = 0; i < 3; ++i) {
        const bool boxed = doseBoxed && !doseExposed;
        lo[i] = boxed ? dirtyLo[i] : 0;
        hi[i] = boxed ? dirtyHi[i] : doseGrid.dims[i] - 1;
    }
    const bool empty = hi[0] < lo[0] || hi[1] < lo[1] || hi[2] < lo[2];
    for (int i = 0; i < 3; ++i) {
        a.lo[i] = lo[i];
        a.ext[i] = empty ? 0 : hi[i] - lo[i] + 1;
    }
    a.X = doseGrid.dims[0];
    a.Y = doseGrid.dims[1];
    a.n = empty ? 0 : static_cast<long long>(a.ext[0]) * a.ext[1] * a.ext[2];
    return PBS_OK;
}

// Spots [spotBegin, spotBegin + spotCount) in passes of `batch` spots; a pass whose
// device buffers do not fit is retried with half as many (after its buffers are
// released and the default memory pool's unused memory is handed back). `first` is
// set to each pass's first column before the pass.
int Context::run_column_batches(ColumnPlan& cp, long long spotBegin, long long spotCount, int batch, ColumnSink& sink,
                                long long& first) {
    bool gridZero = false;
    for (long long k0 = 0; k0 < spotCount;) {
        const int kb = static_cast<int>(std::min<long long>(batch, spotCount - k0));
        first = k0;
        const int rc = run_column_batch(cp, static_cast<size_t>(spotBegin + k0), kb, sink, gridZero);
        if (rc == PBS_ERR_OUT_OF_MEMORY && batch > 1) {
            cudaGetLastError();
            for (DevBuf* b : {&colBev, &colFixed, &colDose}) b->release();
            colClean = false;
            cudaMemPool_t pool;
            if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) cudaMemPoolTrimTo(pool, 0);
            batch /= 2;
            gridZero = false;
            continue;
        }
        if (rc) return rc;
        gridZero = true;
        k0 += kb;
    }
    return PBS_OK;
}

int Context::run_column_batch(ColumnPlan& cp, size_t firstSpot, int count, ColumnSink& sink, bool gridZero) {
    if (count <= 0) return PBS_OK;
    const size_t plane = static_cast<size_t>(cp.base.lattice.nx) * cp.base.lattice.ny;
    // The plan without its per-layer vectors, then one layer per spot: the spot's own
    // layer's parameters and, as that layer's lattice weights, the spot's shares.
    BeamPlan P;
    {
        std::vector<float> weights;
        std::vector<LayerHost> layers;
        std::swap(cp.base.lattice.weights, weights);
        std::swap(cp.base.layers, layers);
        P = cp.base;
        std::swap(cp.base.lattice.weights, weights);
        std::swap(cp.base.layers, layers);
    }
    P.numLayers = count;
    P.lattice.nl = count;
    P.layers.resize(static_cast<size_t>(count));
    P.lattice.weights.assign(plane * static_cast<size_t>(count), 0.0f);
    for (int q = 0; q < count; ++q) {
        const size_t j = firstSpot + static_cast<size_t>(q);
        int layer = -1;
        for (int slot = 0; slot < 4; ++slot)
            if (cp.cells[j * 4 + slot] >= 0) layer = static_cast<int>(cp.cells[j * 4 + slot] / plane);
        // A spot on no lattice cell keeps an all-zero layer: an empty column.
        P.layers[static_cast<size_t>(q)] = cp.base.layers[static_cast<size_t>(std::max(layer, 0))];
        for (int slot = 0; slot < 4; ++slot) {
            const int c = cp.cells[j * 4 + slot];
            if (c >= 0)
                P.lattice.weights[static_cast<size_t>(q) * plane + (static_cast<size_t>(c) - size_t(layer) * plane)] +=
                    cp.shares[j * 4 + slot];
        }
    }
    if (gridZero && doseBoxed && !doseExposed && !pendingDoseInit) {
        for (int i = 0; i < 3; ++i) {
            dirtyLo[i] = INT_MAX;
            dirtyHi[i] = -1;
        }
    } else if (int rc = reset_dose(nullptr, 0)) {
        return rc;
    }
    return run_beam(cp.beam, 0, nullptr, &P, &sink);
}

int Context::influence_row_norms(const PbsBeamDesc& beam, int nuclear, long long spotBegin, long long spotCount,
                                 const long long* voxelsHost, long long nVoxels, float* outHost) {
    const long long gridN = hasDose ? static_cast<long long>(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2]
                                    : 0;
    if (!outHost || nVoxels < 0 || (nVoxels > 0 && !voxelsHost)) {
        set_error("influence row norms: null output or negative voxel count");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    for (long long i = 0; i < nVoxels; ++i)
        if (voxelsHost[i] < 0 || voxelsHost[i] >= gridN) {
            set_error("influence row norms: voxel index " + std::to_string(voxelsHost[i]) + " outside the dose grid");
            return PBS_ERR_INVALID_ARGUMENT;
        }
    ColumnPlan cp;
    if (int rc = plan_columns(beam, spotBegin, spotCount, "influence row norms", cp)) return rc;
    ColumnTraceGuard sharedTrace(*this);
    auto fail = [&](int rc) {
        const std::string msg = last_error();
        reset_dose(nullptr, 0);
        set_error(msg);
        return rc;
    };
    const long long nOut = voxelsHost ? nVoxels : gridN;
    if (int rc = opNorm.ensure(static_cast<size_t>(gridN) * sizeof(double))) return fail(rc);
    if (int rc = opVals.ensure(static_cast<size_t>(std::max(nOut, 1LL)) * sizeof(float))) return fail(rc);
    if (voxelsHost && nVoxels > 0) {
        if (int rc = opVoxels.ensure(static_cast<size_t>(nVoxels) * sizeof(long long))) return fail(rc);
        if (int rc = upload(opVoxels.ptr, voxelsHost, static_cast<size_t>(nVoxels) * sizeof(long long)))
            return fail(rc);
    }
    double* norm = static_cast<double*>(opNorm.ptr);
    if (int rc = op_cuda(cudaMemsetAsync(norm, 0, static_cast<size_t>(gridN) * sizeof(double), stream),
                         "row norm clear"))
        return fail(rc);
    double* d = static_cast<double*>(dose64.ptr);
    auto add = [&](const OpBox& a, bool nuc) {
        if (a.n > 0) {
            const int blocks = static_cast<int>(std::min<long long>((a.n + kOpThreads - 1) / kOpThreads, 148 * 8));
            row_norm_add_kernel<<<blocks, kOpThreads, 0, stream>>>(
                d, a, static_cast<const BeamStateDev*>(bs.ptr),
                nuc ? static_cast<const BeamStateDev*>(nucBs.ptr) : nullptr, norm);
        }
        return op_cuda(cudaGetLastError(), "row norm kernel");
    };
    if (!nuclear && !bioModel && !carbonProfile) {
        // Batched: each batch's columns in their own dose buffers, their squares added
        // voxel by voxel in column order.
        struct Sink : ColumnSink {
            Context& c;
            decltype(add)& run;
            double* norm;
            Sink(Context& ctx, decltype(add)& f, double* nm) : c(ctx), run(f), norm(nm) {}
            int columns(int first, int count) override {
                if (c.compatBevZShift) return run(dirty_op_box(c), false);
                const ColBox fb = c.colBox;
                const size_t fbN = size_t(fb.ext[0]) * fb.ext[1] * fb.ext[2];
                if (fbN == 0 || count <= 0) return PBS_OK;
                const int blocks = static_cast<int>(std::min<size_t>((fbN + kOpThreads - 1) / kOpThreads, 148 * 8));
                col_norm_kernel<<<blocks, kOpThreads, 0, c.stream>>>(
                    static_cast<double*>(c.colDose.ptr), fb, static_cast<const LayerStateDev*>(c.ls.ptr) + first,
                    count, c.doseGrid.dims[0], c.doseGrid.dims[1], norm);
                return op_cuda(cudaGetLastError(), "column row norms");
            }
        } sink(*this, add, norm);
        ColBox fb;
        size_t maxChunks = 0;
        const int batch = column_batch_size(*this, cp.base, fb, maxChunks);
        long long first = 0;
        if (int rc = run_column_batches(cp, spotBegin, spotCount, batch, sink, first)) return fail(rc);
    } else {
        for (long long k = 0; k < spotCount; ++k) {
            OpBox a{};
            // The previous column's norm pass zeroed what its transfers wrote.
            if (int rc = run_column(cp, static_cast<size_t>(spotBegin + k), nuclear, &a, k > 0)) return fail(rc);
            if (int rc = add(a, lastNuclear)) return fail(rc);
        }
    }
    if (nOut > 0) {
        const int blocks = static_cast<int>(std::min<long long>((nOut + kOpThreads - 1) / kOpThreads, 148 * 8));
        row_norm_gather_kernel<<<blocks, kOpThreads, 0, stream>>>(
            norm, voxelsHost ? static_cast<const long long*>(opVoxels.ptr) : nullptr, nOut,
            static_cast<float*>(opVals.ptr));
        if (int rc = op_cuda(cudaGetLastError(), "row norm gather")) return fail(rc);
        if (int rc = op_cuda(cudaMemcpyAsync(outHost, opVals.ptr, static_cast<size_t>(nOut) * sizeof(float),
                                             cudaMemcpyDeviceToHost, stream),
                             "row norms D2H"))
            return fail(rc);
        copiedD2H += static_cast<unsigned long long>(nOut) * sizeof(float);
    }
    if (int rc = op_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize")) return fail(rc);
    if (int rc = take_device_errors()) return fail(rc);
    if (int rc = reset_dose(nullptr, 0)) return rc;
    return op_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
}

int Context::influence_csc(const PbsBeamDesc& beam, int nuclear, long long spotBegin, long long spotCount,
                           double threshold, long long* colPtrHost, int* rowsHost, float* valsHost,
                           long long capacity, long long* nnzOut) {
    if (!(threshold >= 0.0) || !std::isfinite(threshold)) {
        set_error("influence export: the threshold must be finite and >= 0");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    if (!colPtrHost || !nnzOut || capacity < 0 || (capacity > 0 && (!rowsHost || !valsHost))) {
        set_error("influence export: null output or negative capacity");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    const long long gridN =
        hasDose ? static_cast<long long>(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2] : 0;
    if (gridN > INT_MAX) {
        set_error("influence export: the dose grid has more voxels than an int32 row index holds");
        return PBS_ERR_UNSUPPORTED;
    }
    ColumnPlan cp;
    if (int rc = plan_columns(beam, spotBegin, spotCount, "influence export", cp)) return rc;
    ColumnTraceGuard sharedTrace(*this);

    // Any failure below leaves the dose grid zeroed, as a finished export does.
    auto fail = [&](int rc) {
        const std::string msg = last_error();
        reset_dose(nullptr, 0);
        set_error(msg);
        return rc;
    };
    const long long maxBlocks = (gridN + kOpChunk - 1) / kOpChunk;
    if (int rc = opColPtr.ensure(static_cast<size_t>(spotCount + 1) * sizeof(long long))) return fail(rc);
    // Chunk offsets, and after them the chunk count of the column being compacted.
    if (int rc = opBlockOff.ensure(static_cast<size_t>(maxBlocks + 1) * sizeof(long long))) return fail(rc);
    if (capacity > 0) {
        if (int rc = opRows.ensure(static_cast<size_t>(capacity) * sizeof(int))) return fail(rc);
        if (int rc = opVals.ensure(static_cast<size_t>(capacity) * sizeof(float))) return fail(rc);
    }
    long long* dColPtr = static_cast<long long*>(opColPtr.ptr);
    long long* dBlockOff = static_cast<long long*>(opBlockOff.ptr);
    int* dRows = capacity > 0 ? static_cast<int*>(opRows.ptr) : nullptr;
    float* dVals = capacity > 0 ? static_cast<float*>(opVals.ptr) : nullptr;
    if (int rc = op_cuda(cudaMemsetAsync(dColPtr, 0, sizeof(long long), stream), "influence colPtr clear"))
        return fail(rc);

    // Column k: its entries compacted from the FP64 grid (which the compaction zeroes
    // again) into the CSC arrays after column k - 1's.
    auto compact = [&](long long k, const OpBox& a, bool nuc) {
        // The host box bounds the device box (column_box) the kernels walk: at most
        // kOpGridBlocks blocks stride over its chunks.
        const int nBlocks = static_cast<int>(std::min<long long>((a.n + kOpChunk - 1) / kOpChunk, kOpGridBlocks));
        double* d = static_cast<double*>(dose64.ptr);
        const BeamStateDev* pb = static_cast<const BeamStateDev*>(bs.ptr);
        const BeamStateDev* nb = nuc ? static_cast<const BeamStateDev*>(nucBs.ptr) : nullptr;
        long long* dChunks = dBlockOff + maxBlocks;
        if (nBlocks > 0) {
            influence_count_kernel<<<nBlocks, kOpThreads, 0, stream>>>(d, a, pb, nb, threshold, dBlockOff, dChunks);
        } else if (int rc = op_cuda(cudaMemsetAsync(dChunks, 0, sizeof(long long), stream), "influence count clear")) {
            return rc;
        }
        influence_scan_kernel<<<1, 1024, 0, stream>>>(dBlockOff, dChunks, dColPtr, static_cast<int>(k));
        if (nBlocks > 0)
            influence_write_kernel<<<nBlocks, kOpThreads, 0, stream>>>(d, a, pb, nb, threshold, dBlockOff, dRows,
                                                                       dVals, capacity);
        return op_cuda(cudaGetLastError(), "influence kernels");
    };
    if (!nuclear && !bioModel && !carbonProfile) {
        // Batched: each batch's columns in their own dose buffers, compacted with one
        // count, one scan and one write launch per batch (column after column in the
        // CSC order).
        ColBox fb;
        size_t maxChunks = 0;
        const int batch = column_batch_size(*this, cp.base, fb, maxChunks);
        if (int rc = opBlockOff.ensure((std::max<size_t>(size_t(maxBlocks), size_t(batch) * maxChunks + batch) + 1) *
                                       sizeof(long long)))
            return fail(rc);
        dBlockOff = static_cast<long long*>(opBlockOff.ptr);
        struct Sink : ColumnSink {
            Context& c;
            decltype(compact)& run;
            long long first = 0;
            double thr;
            long long* off;
            int* rows;
            float* vals;
            long long cap, *colPtr;
            Sink(Context& ctx, decltype(compact)& f) : c(ctx), run(f) {}
            int columns(int l, int count) override {
                if (c.compatBevZShift) return run(first + l, dirty_op_box(c), false);
                const ColBox fb = c.colBox;
                const size_t fbN = size_t(fb.ext[0]) * fb.ext[1] * fb.ext[2];
                const int maxChunks = static_cast<int>(std::max<size_t>((fbN + kOpChunk - 1) / kOpChunk, 1));
                long long* nChunks = off + size_t(count) * maxChunks;
                const LayerStateDev* lsq = static_cast<const LayerStateDev*>(c.ls.ptr) + l;
                const int X = c.doseGrid.dims[0], Y = c.doseGrid.dims[1];
                // A few waves of blocks over all the batch's columns.
                const int per = std::max(1, std::min(maxChunks, (148 * 4) / std::max(count, 1) + 1));
                double* d = static_cast<double*>(c.colDose.ptr);
                col_count_kernel<<<dim3(per, count), kOpThreads, 0, c.stream>>>(d, fb, lsq, X, Y, thr, off, maxChunks,
                                                                                 nChunks);
                col_scan_kernel<<<1, 1024, 0, c.stream>>>(off, maxChunks, nChunks, count, colPtr,
                                                           static_cast<int>(first + l));
                col_write_kernel<<<dim3(per, count), kOpThreads, 0, c.stream>>>(d, fb, lsq, X, Y, thr, off, maxChunks,
                                                                                 rows, vals, cap);
                return op_cuda(cudaGetLastError(), "column compaction");
            }
        } sink(*this, compact);
        sink.thr = threshold;
        sink.off = dBlockOff;
        sink.rows = dRows;
        sink.vals = dVals;
        sink.cap = capacity;
        sink.colPtr = dColPtr;
        if (int rc = run_column_batches(cp, spotBegin, spotCount, batch, sink, sink.first)) return fail(rc);
    } else {
        for (long long k = 0; k < spotCount; ++k) {
            OpBox a{};
            // The previous column's compaction zeroed what its transfers wrote.
            if (int rc = run_column(cp, static_cast<size_t>(spotBegin + k), nuclear, &a, k > 0)) return fail(rc);
            if (int rc = compact(k, a, lastNuclear)) return fail(rc);
        }
    }
    if (int rc = op_cuda(cudaMemcpyAsync(colPtrHost, dColPtr, static_cast<size_t>(spotCount + 1) * sizeof(long long),
                                         cudaMemcpyDeviceToHost, stream),
                         "influence colPtr D2H"))
        return fail(rc);
    if (int rc = op_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize")) return fail(rc);
    if (int rc = take_device_errors()) return fail(rc);
    const long long nnz = colPtrHost[spotCount];
    *nnzOut = nnz;
    if (nnz > capacity) {
        reset_dose(nullptr, 0);
        set_error("influence export: " + std::to_string(nnz) + " entries do not fit the capacity of " +
                  std::to_string(capacity));
        return PBS_ERR_INVALID_ARGUMENT;
    }
    if (nnz > 0) {
        if (int rc = op_cuda(cudaMemcpyAsync(rowsHost, dRows, static_cast<size_t>(nnz) * sizeof(int),
                                             cudaMemcpyDeviceToHost, stream),
                             "influence rows D2H"))
            return fail(rc);
        if (int rc = op_cuda(cudaMemcpyAsync(valsHost, dVals, static_cast<size_t>(nnz) * sizeof(float),
                                             cudaMemcpyDeviceToHost, stream),
                             "influence values D2H"))
            return fail(rc);
    }
    if (int rc = reset_dose(nullptr, 0)) return rc;
    return op_cuda(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
}

}  // namespace pbs
