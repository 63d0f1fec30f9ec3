// BEV -> dose transfer and dose-grid helpers.
//
// The layer-summed BEV dose of a beam is sampled once at the divergent fan index
// of every dose voxel inside the transfer box and accumulated in FP64. The
// reference transfers every layer separately into an FP32 grid
// (wrapper.cu:5343-5505); the transfer is linear in the BEV dose, so one pass over
// the summed volume gives the same sum up to rounding.
#include <algorithm>

#include "device_util.cuh"
#include "kernels.h"
#include "launch_util.h"

namespace pbs {

namespace {

// Trilinear sample with texel centres at i + 0.5 and zero outside the volume,
// at texel-space coordinates (x, y, z) = texture coordinate - 0.5.
__device__ __forceinline__ float bev_sample(const float* __restrict__ v, int nx, int ny, int nz, float x, float y,
                                            float z) {
    x = fminf(fmaxf(x, -2.0f), float(nx) + 1.0f);
    y = fminf(fmaxf(y, -2.0f), float(ny) + 1.0f);
    z = fminf(fmaxf(z, -2.0f), float(nz) + 1.0f);
    const float fx = floorf(x), fy = floorf(y), fz = floorf(z);
    const int x0 = int(fx), y0 = int(fy), z0 = int(fz);
    const float tx = x - fx, ty = y - fy, tz = z - fz;
    float c000, c100, c010, c110, c001, c101, c011, c111;
    if (x0 >= 0 && y0 >= 0 && z0 >= 0 && x0 + 1 < nx && y0 + 1 < ny && z0 + 1 < nz) {
        // All eight texels inside: one base address.
        const size_t plane = static_cast<size_t>(nx) * ny;
        const float* p = v + (static_cast<size_t>(z0) * ny + y0) * nx + x0;
        c000 = __ldg(p);
        c100 = __ldg(p + 1);
        c010 = __ldg(p + nx);
        c110 = __ldg(p + nx + 1);
        c001 = __ldg(p + plane);
        c101 = __ldg(p + plane + 1);
        c011 = __ldg(p + plane + nx);
        c111 = __ldg(p + plane + nx + 1);
    } else {
        auto at = [&](int xi, int yi, int zi) -> float {
            if (xi < 0 || yi < 0 || zi < 0 || xi >= nx || yi >= ny || zi >= nz) return 0.0f;
            return __ldg(v + (static_cast<size_t>(zi) * ny + yi) * nx + xi);
        };
        c000 = at(x0, y0, z0);
        c100 = at(x0 + 1, y0, z0);
        c010 = at(x0, y0 + 1, z0);
        c110 = at(x0 + 1, y0 + 1, z0);
        c001 = at(x0, y0, z0 + 1);
        c101 = at(x0 + 1, y0, z0 + 1);
        c011 = at(x0, y0 + 1, z0 + 1);
        c111 = at(x0 + 1, y0 + 1, z0 + 1);
    }
    const float c00 = c000 + (c100 - c000) * tx;
    const float c10 = c010 + (c110 - c010) * tx;
    const float c01 = c001 + (c101 - c001) * tx;
    const float c11 = c011 + (c111 - c011) * tx;
    const float c0 = c00 + (c10 - c00) * ty;
    const float c1 = c01 + (c11 - c01) * ty;
    return c0 + (c1 - c0) * tz;
}

// Transfer box from the eight BEV corners (wrapper.cu:5343-5394) over the steps
// [first, passive). With `live` the corners are those of the cells the superposition
// items can have written (liveLo/liveHi, one cell of trilinear reach added): every
// voxel outside samples only zero cells, so the transfer and the box's readers skip
// it. Returns whether the box holds a voxel; no live cell gives an empty box.
__device__ bool plan_transfer_box(const BeamGeomDev& g, int first, int passive, bool live, const int* liveLo,
                                  const int* liveHi, int start[3], int maxi[3]) {
    start[0] = start[1] = start[2] = 0;
    maxi[0] = maxi[1] = maxi[2] = -1;
    float xs[2] = {-float(kMaxR), float(g.pitchX + kMaxR - 1)};
    float ys[2] = {-float(kMaxR), float(g.pitchY + kMaxR - 1)};
    float zs[2] = {float(first), float(passive - 1)};
    if (live) {
        if (liveLo[0] > liveHi[0]) return false;
        // Padded BEV cell c is ray coordinate c - kMaxR.
        xs[0] = fmaxf(xs[0], float(liveLo[0] - kMaxR - 1));
        xs[1] = fminf(xs[1], float(liveHi[0] - kMaxR + 1));
        ys[0] = fmaxf(ys[0], float(liveLo[1] - kMaxR - 1));
        ys[1] = fminf(ys[1], float(liveHi[1] - kMaxR + 1));
        zs[0] = fmaxf(zs[0], float(first + liveLo[2] - 1));
        zs[1] = fminf(zs[1], float(first + liveHi[2] + 1));
    }
    V3 mx = v3(-1.0f, -1.0f, -1.0f), mn = v3(100000.0f, 100000.0f, 100000.0f);
    for (int zi = 0; zi < 2; ++zi)
        for (int yi = 0; yi < 2; ++yi)
            for (int xi = 0; xi < 2; ++xi) {
                const V3 p = apply(g.rayIdxToDoseIdx, v3(xs[xi], ys[yi], zs[zi]));
                mx.x = fmaxf(mx.x, p.x);
                mx.y = fmaxf(mx.y, p.y);
                mx.z = fmaxf(mx.z, p.z);
                mn.x = fminf(mn.x, p.x);
                mn.y = fminf(mn.y, p.y);
                mn.z = fminf(mn.z, p.z);
            }
    start[0] = max((int(floorf(mn.x)) / 32) * 32, 0);
    start[1] = max(int(floorf(mn.y)), 0);
    start[2] = max(int(floorf(mn.z)), 0);
    maxi[0] = min(int(ceilf(mx.x)), g.doseX - 1);
    maxi[1] = min(int(ceilf(mx.y)), g.doseY - 1);
    maxi[2] = min(int(ceilf(mx.z)), g.doseZ - 1);
    return passive > first && start[0] <= maxi[0] && start[1] <= maxi[1] && start[2] <= maxi[2];
}

// The beam's transfer box: over the deepest superposed step of all layers, or of
// `layer` alone when it is given (plan_transfer_box), and the transfer parameters.
__global__ void transfer_planner_kernel(BeamGeomDev g, BeamStateDev* beam, const LayerStateDev* layer, int live) {
    pdl_trigger();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    // Last kernel of the beam's work list with one thread: hand the beam's error
    // flags to the context's error word, which outlives the beam state.
    if (g.errWord && beam->errorFlags) atomicOr(g.errWord, beam->errorFlags);
    const int first = beam->firstInside;
    const int passive = layer ? layer->calcPassive : beam->maxCalcPassive;
    // The live box is read before any field of the beam state is written.
    int lo[3], hi[3], start[3], maxi[3];
    for (int i = 0; i < 3; ++i) {
        lo[i] = beam->liveLo[i];
        hi[i] = beam->liveHi[i];
    }
    const int valid = plan_transfer_box(g, first, passive, live != 0, lo, hi, start, maxi);
    const ToFan t = invert_and_shift(g.rayIdxToDoseIdx, v3(float(kMaxR), float(kMaxR), -float(first)));
    beam->transfer = make_transfer_params(t);
    for (int i = 0; i < 3; ++i) {
        beam->transferStart[i] = start[i];
        beam->transferMax[i] = maxi[i];
    }
    beam->transferValid = valid;
}

// Batched influence columns: every layer of the chunk [layer0, layer0 + nCols) gets
// the transfer box of its own live cells (LayerStateDev::colStart/colMax/colValid);
// the beam gets the transfer parameters, which do not depend on the layer.
__global__ void column_transfer_planner_kernel(BeamGeomDev g, BeamStateDev* beam, LayerStateDev* ls, int nCols) {
    const int q = threadIdx.x;
    const int first = beam->firstInside;
    if (q == 0) {
        if (g.errWord && beam->errorFlags) atomicOr(g.errWord, beam->errorFlags);
        const ToFan t = invert_and_shift(g.rayIdxToDoseIdx, v3(float(kMaxR), float(kMaxR), -float(first)));
        beam->transfer = make_transfer_params(t);
    }
    if (q < nCols) {
        LayerStateDev& st = ls[q];
        st.colValid = plan_transfer_box(g, first, st.calcPassive, true, st.liveLo, st.liveHi, st.colStart, st.colMax);
    }
}

// primTransfDiv (src/algorithms/prim_transf_kernel.cu:11-44). The reference launches
// ceil(width/32) x ceil(height/8) blocks from the box start, so columns up to the
// next block boundary inside the dose grid are transferred too. Every voxel is
// independent: the box (known only on the device) is cut into items of one dose
// column (x, y) and kTransferZChunk consecutive z, x fastest so that a warp's FP64
// read-modify-writes are coalesced, and a persistent grid strides over the items.
// The chunk's voxels are sampled with independent loads (unrolled loop), so the
// latency of the BEV samples and of the dose reads overlaps.
constexpr int kTransferZChunk = 4;
constexpr int kTransferBlocksPerSM = 8;

__global__ void __launch_bounds__(256)
transfer_kernel(BeamGeomDev g, const float* __restrict__ bev, const BeamStateDev* __restrict__ beam,
                double* __restrict__ dose) {
    pdl_wait();
    if (!beam->transferValid) return;
    const int sx = beam->transferStart[0], sy = beam->transferStart[1], sz = beam->transferStart[2];
    const int mx = beam->transferMax[0], my = beam->transferMax[1], mz = beam->transferMax[2];
    // Columns of the launch box that lie inside the dose grid.
    const int nx = min(((mx - sx + 1 + 31) / 32) * 32, g.doseX - sx);
    const int ny = min(((my - sy + 1 + 7) / 8) * 8, g.doseY - sy);
    const int nzc = (mz - sz + kTransferZChunk) / kTransferZChunk;
    if (nx <= 0 || ny <= 0 || nzc <= 0) return;
    const long long items = static_cast<long long>(nx) * ny * nzc;
    const TransferParams T = beam->transfer;
    const float zShift = g.compatBevZShift ? float(beam->firstInside) : 0.0f;
    const size_t slice = static_cast<size_t>(g.doseX) * g.doseY;
    for (long long it = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; it < items;
         it += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = sx + static_cast<int>(it % nx);
        const long long r = it / nx;
        const int y = sy + static_cast<int>(r % ny);
        const int z0 = sz + static_cast<int>(r / ny) * kTransferZChunk;
        const V3 start = transfer_start(T, x, y);
        double* col = dose + static_cast<size_t>(y) * g.doseX + x;
        float v[kTransferZChunk];
#pragma unroll
        for (int k = 0; k < kTransferZChunk; ++k) {
            const int z = z0 + k;
            v[k] = 0.0f;
            if (z <= mz) {
                const V3 f = transfer_fan_idx(T, start, z);
                if (!(f.x + 0.5f < 0.0f || f.y + 0.5f < 0.0f || f.z + 0.5f < 0.0f))
                    v[k] = bev_sample(bev, g.bevX, g.bevY, g.steps, f.x, f.y, f.z - zShift);
            }
        }
#pragma unroll
        for (int k = 0; k < kTransferZChunk; ++k)
            if (v[k] > 0.0f) col[static_cast<size_t>(z0 + k) * slice] += double(v[k]);
    }
}

__global__ void dose_init_kernel(double* dose, const float* init, size_t n) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        dose[i] = init ? double(init[i]) : 0.0;
}

__global__ void dose_to_float_kernel(const double* dose, float* out, size_t n) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x)
        out[i] = float(dose[i]);
}

// Box [lo, lo + ext) of a [dims.z][dims.y][dims.x] grid: zeroes the FP64 dose there
// (out == nullptr) or converts it to float into the same voxels of `out`.
__global__ void dose_box_kernel(double* dose, float* out, int3 dims, int3 lo, int3 ext) {
    const size_t total = size_t(ext.x) * ext.y * ext.z;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const int x = int(i % size_t(ext.x));
        const size_t r = i / size_t(ext.x);
        const int y = int(r % size_t(ext.y));
        const int z = int(r / size_t(ext.y));
        const size_t v = (size_t(z + lo.z) * dims.y + (y + lo.y)) * size_t(dims.x) + (x + lo.x);
        if (out)
            out[v] = float(dose[v]);
        else
            dose[v] = 0.0;
    }
}

// Batched influence columns: column q (blockIdx.y) samples its own BEV volume
// (bev + q * bevStride) over its layer's transfer box (column_written_box) and adds
// into its own FP64 dose buffer laid out over `fb`. Items and sampling as in
// transfer_kernel; the blocks of a column stride over its items.
__global__ void __launch_bounds__(256)
column_transfer_kernel(BeamGeomDev g, const float* __restrict__ bev, size_t bevStride,
                       const BeamStateDev* __restrict__ beam, const LayerStateDev* __restrict__ ls, ColBox fb,
                       double* __restrict__ colDose) {
    const int q = blockIdx.y;
    int lo[3], hi[3];
    if (!column_written_box(ls[q], g.doseX, g.doseY, fb, lo, hi)) return;
    const int nx = hi[0] - lo[0] + 1, ny = hi[1] - lo[1] + 1;
    const int nzc = (hi[2] - lo[2] + kTransferZChunk) / kTransferZChunk;
    const long long items = static_cast<long long>(nx) * ny * nzc;
    const TransferParams T = beam->transfer;
    const float* v0 = bev + static_cast<size_t>(q) * bevStride;
    const size_t fbN = static_cast<size_t>(fb.ext[0]) * fb.ext[1] * fb.ext[2];
    double* out = colDose + static_cast<size_t>(q) * fbN;
    const size_t slice = static_cast<size_t>(fb.ext[0]) * fb.ext[1];
    for (long long it = blockIdx.x * static_cast<long long>(blockDim.x) + threadIdx.x; it < items;
         it += static_cast<long long>(gridDim.x) * blockDim.x) {
        const int x = lo[0] + static_cast<int>(it % nx);
        const long long r = it / nx;
        const int y = lo[1] + static_cast<int>(r % ny);
        const int z0 = lo[2] + static_cast<int>(r / ny) * kTransferZChunk;
        const V3 start = transfer_start(T, x, y);
        double* col = out + static_cast<size_t>(y - fb.lo[1]) * fb.ext[0] + (x - fb.lo[0]);
        float v[kTransferZChunk];
#pragma unroll
        for (int k = 0; k < kTransferZChunk; ++k) {
            const int z = z0 + k;
            v[k] = 0.0f;
            if (z <= hi[2]) {
                const V3 f = transfer_fan_idx(T, start, z);
                if (!(f.x + 0.5f < 0.0f || f.y + 0.5f < 0.0f || f.z + 0.5f < 0.0f))
                    v[k] = bev_sample(v0, g.bevX, g.bevY, g.steps, f.x, f.y, f.z);
            }
        }
#pragma unroll
        for (int k = 0; k < kTransferZChunk; ++k)
            if (v[k] > 0.0f) col[static_cast<size_t>(z0 + k - fb.lo[2]) * slice] += double(v[k]);
    }
}

// Batched influence columns: zeroes column q's float BEV volume over its layer's
// live cells (the only cells its superposition wrote), so every volume is zero for
// the next batch.
__global__ void __launch_bounds__(256) column_bev_clear_kernel(BeamGeomDev g, float* __restrict__ bev, size_t bevStride,
                                                               const LayerStateDev* __restrict__ ls) {
    const int q = blockIdx.y;
    const LayerStateDev& st = ls[q];
    if (st.liveLo[0] > st.liveHi[0]) return;
    const int x0 = max(st.liveLo[0], 0), x1 = min(st.liveHi[0], g.bevX - 1);
    const int y0 = max(st.liveLo[1], 0), y1 = min(st.liveHi[1], g.bevY - 1);
    const int z0 = max(st.liveLo[2], 0), z1 = min(st.liveHi[2], g.steps - 1);
    if (x1 < x0 || y1 < y0 || z1 < z0) return;
    const int w = x1 - x0 + 1, rows = y1 - y0 + 1;
    const size_t n = static_cast<size_t>(w) * rows * (z1 - z0 + 1);
    float* v0 = bev + static_cast<size_t>(q) * bevStride;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const int x = x0 + static_cast<int>(i % w);
        const size_t r = i / w;
        const int y = y0 + static_cast<int>(r % rows);
        const int z = z0 + static_cast<int>(r / rows);
        v0[(static_cast<size_t>(z) * g.bevY + y) * g.bevX + x] = 0.0f;
    }
}

// Box [lo, lo + ext) of the FP64 grid initialised from the same voxels of a float grid.
__global__ void dose_box_init_kernel(double* dose, const float* init, int3 dims, int3 lo, int3 ext) {
    const size_t total = size_t(ext.x) * ext.y * ext.z;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const int x = int(i % size_t(ext.x));
        const size_t r = i / size_t(ext.x);
        const int y = int(r % size_t(ext.y));
        const int z = int(r / size_t(ext.y));
        const size_t v = (size_t(z + lo.z) * dims.y + (y + lo.y)) * size_t(dims.x) + (x + lo.x);
        dose[v] = double(init[v]);
    }
}

}  // namespace

cudaError_t launch_dose_box_init(double* dose, const float* init, const int dims[3], const int lo[3], const int hi[3],
                                 cudaStream_t s) {
    for (int i = 0; i < 3; ++i)
        if (lo[i] < 0 || hi[i] >= dims[i] || hi[i] < lo[i]) return cudaErrorInvalidValue;
    const int3 d = make_int3(dims[0], dims[1], dims[2]);
    const int3 l = make_int3(lo[0], lo[1], lo[2]);
    const int3 e = make_int3(hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1);
    const size_t total = size_t(e.x) * e.y * e.z;
    const int blocks = int(std::min<size_t>((total + 255) / 256, 148 * 32));
    dose_box_init_kernel<<<blocks, 256, 0, s>>>(dose, init, d, l, e);
    return cudaGetLastError();
}

cudaError_t launch_column_transfer(const BeamGeomDev& g, const float* bev, size_t bevStride, BeamStateDev* beam,
                                   LayerStateDev* ls, int nCols, const ColBox& fb, double* colDose, cudaStream_t s) {
    if (nCols <= 0) return cudaSuccess;
    if (nCols > 1024) return cudaErrorInvalidValue;
    column_transfer_planner_kernel<<<1, ((nCols + 31) / 32) * 32, 0, s>>>(g, beam, ls, nCols);
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // Blocks per column: a few waves over all columns together.
    const int per = std::max(1, (sms * kTransferBlocksPerSM) / nCols);
    column_transfer_kernel<<<dim3(per, nCols), 256, 0, s>>>(g, bev, bevStride, beam, ls, fb, colDose);
    return cudaGetLastError();
}

cudaError_t launch_column_bev_clear(const BeamGeomDev& g, float* bev, size_t bevStride, const LayerStateDev* ls,
                                    int nCols, cudaStream_t s) {
    if (nCols <= 0) return cudaSuccess;
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int per = std::max(1, (sms * 8) / nCols);
    column_bev_clear_kernel<<<dim3(per, nCols), 256, 0, s>>>(g, bev, bevStride, ls);
    return cudaGetLastError();
}

cudaError_t launch_transfer_planner(const BeamGeomDev& g, BeamStateDev* beam, const LayerStateDev* layer, int live,
                                    cudaStream_t s) {
    transfer_planner_kernel<<<1, 32, 0, s>>>(g, beam, layer, live);
    return cudaGetLastError();
}

cudaError_t launch_transfer(const BeamGeomDev& g, const float* bev, const BeamStateDev* beam, double* dose,
                            cudaStream_t s) {
    int dev = 0, sms = 148;
    if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    // No more CTAs than the whole grid could need (small grids).
    const long long cap = ((static_cast<long long>(g.doseX) * g.doseY) * ((g.doseZ + kTransferZChunk - 1) / kTransferZChunk) +
                           255) / 256;
    const int blocks = static_cast<int>(std::max<long long>(1, std::min<long long>(cap, sms * kTransferBlocksPerSM)));
    cudaError_t e = launch_pdl(transfer_kernel, dim3(blocks), dim3(256), 0, s, g, bev, beam, dose);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t launch_dose_init(double* dose, const float* init, size_t n, cudaStream_t s) {
    const int blocks = int(std::min<size_t>((n + 255) / 256, 148 * 32));
    dose_init_kernel<<<blocks, 256, 0, s>>>(dose, init, n);
    return cudaGetLastError();
}

cudaError_t launch_dose_to_float(const double* dose, float* out, size_t n, cudaStream_t s) {
    const int blocks = int(std::min<size_t>((n + 255) / 256, 148 * 32));
    dose_to_float_kernel<<<blocks, 256, 0, s>>>(dose, out, n);
    return cudaGetLastError();
}

cudaError_t launch_dose_box(double* dose, float* out, const int dims[3], const int lo[3], const int hi[3],
                            cudaStream_t s) {
    for (int i = 0; i < 3; ++i)
        if (lo[i] < 0 || hi[i] >= dims[i] || hi[i] < lo[i]) return cudaErrorInvalidValue;
    const int3 d = make_int3(dims[0], dims[1], dims[2]);
    const int3 l = make_int3(lo[0], lo[1], lo[2]);
    const int3 e = make_int3(hi[0] - lo[0] + 1, hi[1] - lo[1] + 1, hi[2] - lo[2] + 1);
    const size_t total = size_t(e.x) * e.y * e.z;
    const int blocks = int(std::min<size_t>((total + 255) / 256, 148 * 32));
    dose_box_kernel<<<blocks, 256, 0, s>>>(dose, out, d, l, e);
    return cudaGetLastError();
}

}  // namespace pbs
