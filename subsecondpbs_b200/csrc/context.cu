// Resident dose context: device-resident lookup tables, CT and FP64 dose grid, and
// the per-beam launch sequence. A beam is planned on the host and then runs as one
// asynchronous sequence of kernels on the context stream with no host round trip:
// every trace-dependent decision (entry step, cut-off steps, passive steps, tile
// radii, batching, transfer box) is made on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <climits>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "context.h"
#include "kernels.h"
#include "plan.h"

namespace pbs {

namespace {
thread_local std::string g_lastError;
}

void set_error(const std::string& msg) { g_lastError = msg; }
const char* last_error() { return g_lastError.c_str(); }

static int cuda_fail(cudaError_t e, const char* where) {
    set_error(std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? PBS_ERR_OUT_OF_MEMORY : PBS_ERR_CUDA;
}

#define PBS_CUDA(call, where)                     \
    do {                                          \
        cudaError_t e_ = (call);                  \
        if (e_ != cudaSuccess) return cuda_fail(e_, where); \
    } while (0)

int DevBuf::ensure(size_t b) {
    if (b <= bytes) return PBS_OK;
    release();
    if (b == 0) return PBS_OK;
    cudaError_t e = allocStream ? cudaMallocAsync(&ptr, b, allocStream) : cudaMalloc(&ptr, b);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return cuda_fail(e, allocStream ? "cudaMallocAsync" : "cudaMalloc");
    }
    bytes = b;
    return PBS_OK;
}

void DevBuf::release() {
    if (ptr) {
        if (allocStream)
            cudaFreeAsync(ptr, allocStream);
        else
            cudaFree(ptr);
    }
    ptr = nullptr;
    bytes = 0;
}

int PinnedBuf::ensure(size_t b) {
    if (b <= bytes) return PBS_OK;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
    cudaError_t e = cudaMallocHost(&ptr, b);
    if (e != cudaSuccess) {
        ptr = nullptr;
        return cuda_fail(e, "cudaMallocHost");
    }
    bytes = b;
    return PBS_OK;
}

void PinnedBuf::release() {
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    bytes = 0;
}

Context::~Context() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (DevBuf* b : {&cidd, &density, &sp, &rrl, &ct, &ctQuad, &dose64, &dens, &wepl, &weplMin, &rayW, &interm, &lattice,
                      &iddBuf, &rsBuf, &bev, &cpb, &subspots, &floatOut, &firstIn, &firstOut, &firstPassive, &codes,
                      &work, &lp, &ls, &bs, &stats, &nucWeight, &nucSqSigma, &rayToNuc, &nucIddBuf, &nucRsBuf,
                      &nucCodes, &nucWork, &nucBev, &bevFixed, &nucLs, &nucBs, &errWord, &gradDoseBuf, &bevGrad, &rbarBuf,
                      &gradInterm, &gradLattice, &weqBody, &opColPtr, &opBlockOff, &opRows, &opVals})
        b->release();
    staging.release();
    errHost.release();
    if (copyStream) cudaStreamSynchronize(copyStream);
    if (stagingEvent) cudaEventDestroy(stagingEvent);
    if (copyStart) cudaEventDestroy(copyStart);
    if (doseCopied) cudaEventDestroy(doseCopied);
    if (doseZeroed) cudaEventDestroy(doseZeroed);
    if (bevCleared) cudaEventDestroy(bevCleared);
    if (copyStream) cudaStreamDestroy(copyStream);
    for (auto& e : ev)
        if (e) cudaEventDestroy(e);
    if (stream) cudaStreamDestroy(stream);
}

int Context::init(int gpu) {
    device = gpu;
    int n = 0;
    PBS_CUDA(cudaGetDeviceCount(&n), "cudaGetDeviceCount");
    if (gpu < 0 || gpu >= n) {
        set_error("gpu_id " + std::to_string(gpu) + " out of range (" + std::to_string(n) + " devices)");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    PBS_CUDA(cudaSetDevice(gpu), "cudaSetDevice");
    PBS_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate");
    PBS_CUDA(cudaStreamCreateWithFlags(&copyStream, cudaStreamNonBlocking), "cudaStreamCreate");
    PBS_CUDA(cudaEventCreateWithFlags(&copyStart, cudaEventDisableTiming), "cudaEventCreate");
    PBS_CUDA(cudaEventCreateWithFlags(&doseCopied, cudaEventDisableTiming), "cudaEventCreate");
    PBS_CUDA(cudaEventCreateWithFlags(&doseZeroed, cudaEventDisableTiming), "cudaEventCreate");
    PBS_CUDA(cudaEventCreateWithFlags(&bevCleared, cudaEventDisableTiming), "cudaEventCreate");
    PBS_CUDA(cudaEventCreateWithFlags(&stagingEvent, cudaEventDisableTiming), "cudaEventCreate");
    for (auto& e : ev) PBS_CUDA(cudaEventCreate(&e), "cudaEventCreate");
    // Callers of the reference-shaped entry points cannot pass options: the
    // environment selects the reference's BEV depth shift for them.
    if (const char* v = std::getenv("PBS_COMPAT_BEV_Z_SHIFT")) compatBevZShift = std::atoi(v) != 0;
    // The reference fixes its nuclear model at build time (NUCLEAR_CORR); here the
    // environment picks it for the wrapper entry points: 0 SOUKUP, 1 FLUKA, 2 GAUSS_FIT.
    if (const char* v = std::getenv("PBS_NUCLEAR_MODEL")) {
        const int m = std::atoi(v);
        if (m >= 0 && m <= 2) nuclearModel = m;
    }
    // The CarbonPBS lateral profile model is off in the reference; the environment
    // switches it on for the wrapper entry points (bits of PBS_OPT_CARBON_PROFILE).
    if (const char* v = std::getenv("PBS_CARBON_PROFILE")) {
        const int m = std::atoi(v);
        if (m >= 0 && m <= 3) carbonProfile = m;
    }
    int rc = errWord.ensure(sizeof(int));
    if (rc) return rc;
    PBS_CUDA(cudaMemset(errWord.ptr, 0, sizeof(int)), "cudaMemset");
    return PBS_OK;
}

int Context::take_device_errors() {
    int rc = errHost.ensure(sizeof(int));
    if (rc) return rc;
    volatile int* hostFlags = static_cast<volatile int*>(errHost.ptr);
    PBS_CUDA(cudaMemcpyAsync(errHost.ptr, errWord.ptr, sizeof(int), cudaMemcpyDeviceToHost, stream), "error flags D2H");
    copiedD2H += sizeof(int);
    PBS_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    const int flags = *hostFlags;
    if (!flags) return PBS_OK;
    PBS_CUDA(cudaMemsetAsync(errWord.ptr, 0, sizeof(int), stream), "cudaMemsetAsync");
    if (flags & 4) {
        // complete_superposition.cu:609-627 throws here.
        set_error("Nuclear superposition kernel radius exceeded kMaxSuperpR=32 (a halo sigma below the tile "
                  "radius threshold); the dose of that beam is incomplete");
        return PBS_ERR_UNSUPPORTED;
    }
    set_error("device reported an internal error flag " + std::to_string(flags) +
              " (1: work list overflow, 2: radius outside a superposition instance)");
    return PBS_ERR_CUDA;
}

// Copies `n` host bytes to the device through the pinned staging buffer so the
// copy is asynchronous with respect to earlier work on the stream.
int Context::upload(void* dst, const void* src, size_t n) {
    if (n == 0) return PBS_OK;
    PBS_CUDA(cudaEventSynchronize(stagingEvent), "cudaEventSynchronize");
    int rc = staging.ensure(n);
    if (rc) return rc;
    std::memcpy(staging.ptr, src, n);
    PBS_CUDA(cudaMemcpyAsync(dst, staging.ptr, n, cudaMemcpyHostToDevice, stream), "cudaMemcpyAsync H2D");
    copiedH2D += n;
    PBS_CUDA(cudaEventRecord(stagingEvent, stream), "cudaEventRecord");
    return PBS_OK;
}

int Context::set_energy(const PbsEnergyDesc& e) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!(e.n_energies > 0 && e.n_energy_samples > 0) || !e.energies_per_u || !e.peak_depths || !e.scale_facts ||
        !e.cidd_matrix || e.n_energies_per_u != size_t(e.n_energies) || e.n_peak_depths != size_t(e.n_energies) ||
        e.n_scale_facts != size_t(e.n_energies) ||
        e.n_cidd_matrix != size_t(e.n_energies) * size_t(e.n_energy_samples)) {
        set_error("[RTD_ENTRY_ASSERT] energy table dimensions are inconsistent");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    if (!e.density_vector || !e.sp_vector || !e.rrl_vector || e.n_density_samples <= 0 || e.n_sp_samples <= 0 ||
        e.n_rrl_samples <= 0 || size_t(e.n_density_samples) > e.n_density_vector ||
        size_t(e.n_sp_samples) > e.n_sp_vector || size_t(e.n_rrl_samples) > e.n_rrl_vector) {
        set_error("[RTD_ENTRY_ASSERT] density, stopping-power, and radiation-length LUTs are inconsistent");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    // The tables stay resident: a call with the same tables as the resident ones
    // (the common case of repeated wrapper calls) uploads nothing.
    auto same = [](const std::vector<float>& v, const float* p, size_t n) {
        return v.size() == n && (n == 0 || std::memcmp(v.data(), p, n * sizeof(float)) == 0);
    };
    {
        const size_t nTab = size_t(e.n_energies) * size_t(e.n_energy_samples);
        const bool nucGiven = e.nuc_weight_matrix && e.nuc_sq_sigma_matrix && e.n_nuc_weight_matrix == nTab &&
                              e.n_nuc_sq_sigma_matrix == nTab;
        if (hasEnergy && energy.n_energies == e.n_energies && energy.n_energy_samples == e.n_energy_samples &&
            energy.n_density_samples == e.n_density_samples && energy.n_sp_samples == e.n_sp_samples &&
            energy.n_rrl_samples == e.n_rrl_samples && energy.density_scale_fact == e.density_scale_fact &&
            energy.sp_scale_fact == e.sp_scale_fact && energy.rrl_scale_fact == e.rrl_scale_fact &&
            same(energiesPerU, e.energies_per_u, e.n_energies) && same(peakDepths, e.peak_depths, e.n_energies) &&
            same(scaleFacts, e.scale_facts, e.n_energies) && same(ciddHost, e.cidd_matrix, e.n_cidd_matrix) &&
            same(densityHost, e.density_vector, e.n_density_vector) && same(spHost, e.sp_vector, e.n_sp_vector) &&
            same(rrlHost, e.rrl_vector, e.n_rrl_vector) &&
            (nucGiven ? same(nucWeightHost, e.nuc_weight_matrix, nTab) &&
                            same(nucSqSigmaHost, e.nuc_sq_sigma_matrix, nTab) &&
                            nucTablesAligned == (e.nuclear_tables_aligned_to_primary_axis != 0)
                      : nucWeightHost.empty()))
            return PBS_OK;
    }
    energiesPerU.assign(e.energies_per_u, e.energies_per_u + e.n_energies);
    peakDepths.assign(e.peak_depths, e.peak_depths + e.n_energies);
    scaleFacts.assign(e.scale_facts, e.scale_facts + e.n_energies);
    ciddHost.assign(e.cidd_matrix, e.cidd_matrix + e.n_cidd_matrix);
    densityHost.assign(e.density_vector, e.density_vector + e.n_density_vector);
    spHost.assign(e.sp_vector, e.sp_vector + e.n_sp_vector);
    rrlHost.assign(e.rrl_vector, e.rrl_vector + e.n_rrl_vector);
    energy = e;
    energy.energies_per_u = energiesPerU.data();
    energy.peak_depths = peakDepths.data();
    energy.scale_facts = scaleFacts.data();
    energy.cidd_matrix = ciddHost.data();
    energy.density_vector = densityHost.data();
    energy.sp_vector = spHost.data();
    energy.rrl_vector = rrlHost.data();
    // Nuclear weight / sigma^2 tables on the CIDD axes (energy_reader.cpp:135-182),
    // kept only when both are complete.
    const size_t nTab = size_t(e.n_energies) * size_t(e.n_energy_samples);
    const bool hasNuc = e.nuc_weight_matrix && e.nuc_sq_sigma_matrix && e.n_nuc_weight_matrix == nTab &&
                        e.n_nuc_sq_sigma_matrix == nTab;
    nucWeightHost.assign(hasNuc ? e.nuc_weight_matrix : nullptr, hasNuc ? e.nuc_weight_matrix + nTab : nullptr);
    nucSqSigmaHost.assign(hasNuc ? e.nuc_sq_sigma_matrix : nullptr, hasNuc ? e.nuc_sq_sigma_matrix + nTab : nullptr);
    nucTablesAligned = hasNuc && e.nuclear_tables_aligned_to_primary_axis;
    energy.nuc_weight_matrix = hasNuc ? nucWeightHost.data() : nullptr;
    energy.n_nuc_weight_matrix = hasNuc ? nTab : 0;
    energy.nuc_sq_sigma_matrix = hasNuc ? nucSqSigmaHost.data() : nullptr;
    energy.n_nuc_sq_sigma_matrix = hasNuc ? nTab : 0;
    int rc;
    if ((rc = cidd.ensure(ciddHost.size() * 4)) || (rc = density.ensure(densityHost.size() * 4)) ||
        (rc = sp.ensure(spHost.size() * 4)) || (rc = rrl.ensure(rrlHost.size() * 4)))
        return rc;
    if (hasNuc) {
        if ((rc = nucWeight.ensure(nTab * 4)) || (rc = nucSqSigma.ensure(nTab * 4))) return rc;
        PBS_CUDA(cudaMemcpyAsync(nucWeight.ptr, nucWeightHost.data(), nTab * 4, cudaMemcpyHostToDevice, stream), "LUT");
        PBS_CUDA(cudaMemcpyAsync(nucSqSigma.ptr, nucSqSigmaHost.data(), nTab * 4, cudaMemcpyHostToDevice, stream),
                 "LUT");
    }
    PBS_CUDA(cudaMemcpyAsync(cidd.ptr, ciddHost.data(), ciddHost.size() * 4, cudaMemcpyHostToDevice, stream), "LUT");
    PBS_CUDA(cudaMemcpyAsync(density.ptr, densityHost.data(), densityHost.size() * 4, cudaMemcpyHostToDevice, stream),
             "LUT");
    PBS_CUDA(cudaMemcpyAsync(sp.ptr, spHost.data(), spHost.size() * 4, cudaMemcpyHostToDevice, stream), "LUT");
    // The tables are copied from pageable host vectors, which cudaMemcpyAsync
    // stages before it returns; no wait is needed before they are replaced.
    PBS_CUDA(cudaMemcpyAsync(rrl.ptr, rrlHost.data(), rrlHost.size() * 4, cudaMemcpyHostToDevice, stream), "LUT");
    copiedH2D += (ciddHost.size() + densityHost.size() + spHost.size() + rrlHost.size()) * 4 +
                 (hasNuc ? 2 * nTab * 4 : 0);
    luts.cidd = static_cast<const float*>(cidd.ptr);
    luts.nS = e.n_energy_samples;
    luts.nE = e.n_energies;
    luts.density = static_cast<const float*>(density.ptr);
    luts.nDensity = e.n_density_samples;
    luts.densityScale = e.density_scale_fact;
    luts.sp = static_cast<const float*>(sp.ptr);
    luts.nSp = e.n_sp_samples;
    luts.spScale = e.sp_scale_fact;
    luts.rrl = static_cast<const float*>(rrl.ptr);
    luts.nRrl = e.n_rrl_samples;
    luts.rrlScale = e.rrl_scale_fact;
    luts.nucWeight = hasNuc ? static_cast<const float*>(nucWeight.ptr) : nullptr;
    luts.nucSqSigma = hasNuc ? static_cast<const float*>(nucSqSigma.ptr) : nullptr;
    hasEnergy = true;
    return PBS_OK;
}

namespace {
// Copy of the voxel box [lo, hi] between two [Z][Y][X] float volumes of `dims`.
cudaError_t copy_box(void* dst, const void* src, const int dims[3], const int lo[3], const int hi[3],
                     cudaMemcpyKind kind, cudaStream_t s) {
    cudaMemcpy3DParms p = {};
    p.srcPtr = make_cudaPitchedPtr(const_cast<void*>(src), size_t(dims[0]) * 4, size_t(dims[0]), size_t(dims[1]));
    p.dstPtr = make_cudaPitchedPtr(dst, size_t(dims[0]) * 4, size_t(dims[0]), size_t(dims[1]));
    p.srcPos = make_cudaPos(size_t(lo[0]) * 4, size_t(lo[1]), size_t(lo[2]));
    p.dstPos = p.srcPos;
    p.extent = make_cudaExtent(size_t(hi[0] - lo[0] + 1) * 4, size_t(hi[1] - lo[1] + 1), size_t(hi[2] - lo[2] + 1));
    p.kind = kind;
    return cudaMemcpy3DAsync(&p, s);
}

bool box_empty(const int lo[3], const int hi[3]) { return hi[0] < lo[0] || hi[1] < lo[1] || hi[2] < lo[2]; }

unsigned long long box_bytes(const int lo[3], const int hi[3]) {
    if (box_empty(lo, hi)) return 0;
    return 4ull * (unsigned long long)(hi[0] - lo[0] + 1) * (hi[1] - lo[1] + 1) * (hi[2] - lo[2] + 1);
}

void merge_box(int lo[3], int hi[3], const int a[3], const int b[3]) {
    if (b[0] < a[0] || b[1] < a[1] || b[2] < a[2]) return;
    for (int i = 0; i < 3; ++i) {
        lo[i] = std::min(lo[i], a[i]);
        hi[i] = std::max(hi[i], b[i]);
    }
}

// Dose voxels a beam's transfer can write (transfer_planner_kernel and the block
// rounding of transfer_kernel), over all steps so that it bounds every layer.
void dose_transfer_box(const FromFan& f, int pitchX, int pitchY, int steps, const int dims[3], int lo[3],
                       int hi[3]) {
    const float xs[2] = {-float(kMaxR), float(pitchX + kMaxR - 1)};
    const float ys[2] = {-float(kMaxR), float(pitchY + kMaxR - 1)};
    const float zs[2] = {0.0f, float(steps - 1)};
    V3 mx = v3(-1.0f, -1.0f, -1.0f), mn = v3(100000.0f, 100000.0f, 100000.0f);
    for (int zi = 0; zi < 2; ++zi)
        for (int yi = 0; yi < 2; ++yi)
            for (int xi = 0; xi < 2; ++xi) {
                const V3 p = apply(f, v3(xs[xi], ys[yi], zs[zi]));
                mx.x = std::max(mx.x, p.x);
                mx.y = std::max(mx.y, p.y);
                mx.z = std::max(mx.z, p.z);
                mn.x = std::min(mn.x, p.x);
                mn.y = std::min(mn.y, p.y);
                mn.z = std::min(mn.z, p.z);
            }
    lo[0] = std::max((int(std::floor(mn.x)) / 32) * 32, 0);
    lo[1] = std::max(int(std::floor(mn.y)), 0);
    lo[2] = std::max(int(std::floor(mn.z)), 0);
    // The transfer rounds its x and y spans up to whole 32 x 8 blocks.
    hi[0] = std::min(int(std::ceil(mx.x)) + 32, dims[0] - 1);
    hi[1] = std::min(int(std::ceil(mx.y)) + 8, dims[1] - 1);
    hi[2] = std::min(int(std::ceil(mx.z)), dims[2] - 1);
}
}  // namespace

void Context::column_layout(const BeamPlan& P, ColBox& fb, size_t& bevCells, size_t& bytesPerColumn) const {
    int lo[3], hi[3];
    dose_transfer_box(P.rayIdxToDoseIdx, P.superpDims[0], P.superpDims[1], P.tracerSteps, doseGrid.dims, lo, hi);
    size_t voxels = 1;
    for (int i = 0; i < 3; ++i) {
        fb.lo[i] = lo[i];
        fb.ext[i] = std::max(hi[i] - lo[i] + 1, 0);
        voxels *= size_t(fb.ext[i]);
    }
    bevCells = size_t(P.tracerSteps) * size_t(P.superpDims[0] + 2 * kMaxR) * size_t(P.superpDims[1] + 2 * kMaxR);
    bytesPerColumn = bevCells * (sizeof(float) + sizeof(unsigned long long)) + voxels * sizeof(double);
}

int Context::set_ct_region(const float* data, const GridDesc& g, const int lo[3], const int hi[3]) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!data || g.dims[0] <= 0 || g.dims[1] <= 0 || g.dims[2] <= 0 ||
        !(g.res[0] > 0.0f && g.res[1] > 0.0f && g.res[2] > 0.0f)) {
        set_error("[RTD_ENTRY_ASSERT] CT grid must have positive dims and resolution");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    const size_t n = size_t(g.dims[0]) * g.dims[1] * g.dims[2];
    int rc = ct.ensure(n * 4);
    if (rc) return rc;
    ctView = nullptr;
    ctQuadValid = false;
    if (!box_empty(lo, hi)) {
        PBS_CUDA(copy_box(ct.ptr, data, g.dims, lo, hi, cudaMemcpyHostToDevice, stream), "CT H2D");
        copiedH2D += box_bytes(lo, hi);
    }
    // The CT type comes from the whole volume, as with a full upload.
    int type = ctInputType != PBS_CT_AUTO ? ctInputType : parse_ct_input_type_env();
    if (type == PBS_CT_AUTO) {
        // A page-locked host CT is visible to the device: the samples are read and the
        // type detected there, and the conversion follows without a host pass. The
        // caller's buffer outlives the call (the wrapper synchronises before returning).
        cudaPointerAttributes at{};
        const bool mapped = cudaPointerGetAttributes(&at, data) == cudaSuccess && at.type == cudaMemoryTypeHost &&
                            at.devicePointer != nullptr;
        cudaGetLastError();
        const int lutN = int(densityHost.size());
        if (mapped && hasEnergy && lutN > 0 && energy.density_scale_fact != 0.0f && stats.ensure(64) == PBS_OK) {
            PBS_CUDA(launch_ct_convert_detect(static_cast<float*>(ct.ptr), n, static_cast<const float*>(at.devicePointer),
                                              g.dims, lo, hi, static_cast<const float*>(density.ptr), lutN,
                                              energy.density_scale_fact, static_cast<unsigned*>(stats.ptr), stream),
                     "ct_convert_detect");
            // At most the samples outside the box cross the host link (none when the
            // box already holds a value below -200); counted as all samples.
            copiedH2D += ct_type_sample_count(n) * sizeof(float);
            ctType = PBS_CT_AUTO;
            ctGrid = g;
            hasCt = true;
            return build_ct_quad_box(lo, hi);
        }
        float mn, mx;
        sample_ct_stats(data, n, mn, mx);
        type = auto_detect_ct_type(mn, mx);
    }
    // Only the uploaded box is converted: the tracers sample nothing outside it.
    if (!box_empty(lo, hi) && (rc = convert_ct_buffer(static_cast<float*>(ct.ptr), n, type, g.dims, lo, hi)))
        return rc;
    ctType = type;
    ctGrid = g;
    hasCt = true;
    return build_ct_quad_box(lo, hi);
}

int Context::build_ct_quad_box(const int lo[3], const int hi[3]) {
    // The packed copy is an optimisation: without room for it the tracer samples
    // the CT directly.
    ctQuadValid = false;
    if (box_empty(lo, hi)) return PBS_OK;
    if (ctQuad.ensure(ct_quad_bytes(ctGrid.dims)) != PBS_OK) {
        cudaGetLastError();
        set_error("");
        return PBS_OK;
    }
    PBS_CUDA(launch_ct_quad_box(static_cast<const float*>(ct.ptr), ctGrid.dims, lo, hi,
                                static_cast<float4*>(ctQuad.ptr), stream),
             "ct_quad_box");
    ctQuadValid = true;
    return PBS_OK;
}

int Context::reset_dose_region(const float* init, const int lo[3], const int hi[3]) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!hasDose) {
        set_error("dose grid not set");
        return PBS_ERR_NOT_READY;
    }
    const size_t n = size_t(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2];
    int rc = floatOut.ensure(n * 4);
    if (rc) return rc;
    if (box_empty(lo, hi)) return reset_dose(nullptr, 0);
    // Voxels outside the box are initialised from stale values; no beam of the
    // call writes them and read_dose_region does not copy them back.
    doseBoxed = false;
    deferredInit = init;
    for (int i = 0; i < 3; ++i) {
        deferredLo[i] = lo[i];
        deferredHi[i] = hi[i];
    }
    pendingDoseInit = true;
    initBoxed = true;
    return PBS_OK;
}

int Context::issue_dose_copy() {
    if (!deferredInit) return PBS_OK;
    PBS_CUDA(cudaEventRecord(copyStart, stream), "cudaEventRecord");
    PBS_CUDA(cudaStreamWaitEvent(copyStream, copyStart, 0), "cudaStreamWaitEvent");
    PBS_CUDA(copy_box(floatOut.ptr, deferredInit, doseGrid.dims, deferredLo, deferredHi, cudaMemcpyHostToDevice,
                      copyStream),
             "dose H2D");
    copiedH2D += box_bytes(deferredLo, deferredHi);
    PBS_CUDA(cudaEventRecord(doseCopied, copyStream), "cudaEventRecord");
    deferredInit = nullptr;
    return PBS_OK;
}

int Context::read_dose_region(float* out, const int lo[3], const int hi[3]) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    const size_t n = size_t(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2];
    int rc = flush_dose_init();
    if (rc) return rc;
    if ((rc = floatOut.ensure(n * 4))) return rc;
    if (!box_empty(lo, hi)) {
        // Only the region is copied back, so only the region is converted.
        PBS_CUDA(launch_dose_box(static_cast<double*>(dose64.ptr), static_cast<float*>(floatOut.ptr), doseGrid.dims,
                                 lo, hi, stream),
                 "dose_to_float");
        PBS_CUDA(copy_box(out, floatOut.ptr, doseGrid.dims, lo, hi, cudaMemcpyDeviceToHost, stream), "dose D2H");
        copiedD2H += box_bytes(lo, hi);
    }
    PBS_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    return take_device_errors();
}

int Context::set_ct(const float* data, int onDevice, const GridDesc& g) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!data || g.dims[0] <= 0 || g.dims[1] <= 0 || g.dims[2] <= 0 ||
        !(g.res[0] > 0.0f && g.res[1] > 0.0f && g.res[2] > 0.0f)) {
        set_error("[RTD_ENTRY_ASSERT] CT grid must have positive dims and resolution");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    const size_t n = size_t(g.dims[0]) * g.dims[1] * g.dims[2];
    int rc = ct.ensure(n * 4);
    if (rc) return rc;
    ctView = nullptr;
    int type = ctInputType != PBS_CT_AUTO ? ctInputType : parse_ct_input_type_env();
    if (onDevice) {
        PBS_CUDA(cudaMemcpyAsync(ct.ptr, data, n * 4, cudaMemcpyDeviceToDevice, stream), "CT D2D");
        if (type == PBS_CT_AUTO) {
            rc = stats.ensure(64);
            if (rc) return rc;
            PBS_CUDA(launch_ct_stats(static_cast<float*>(ct.ptr), n, static_cast<float*>(stats.ptr), stream), "ct_stats");
            float mm[2];
            PBS_CUDA(cudaMemcpyAsync(mm, stats.ptr, 8, cudaMemcpyDeviceToHost, stream), "CT stats");
            PBS_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
            type = auto_detect_ct_type(mm[0], mm[1]);
        }
    } else {
        // The copy goes first: the CT type is sampled on the host while it runs.
        PBS_CUDA(cudaMemcpyAsync(ct.ptr, data, n * 4, cudaMemcpyHostToDevice, stream), "CT H2D");
        copiedH2D += n * 4;
        if (type == PBS_CT_AUTO) {
            float mn, mx;
            sample_ct_stats(data, n, mn, mx);
            type = auto_detect_ct_type(mn, mx);
        }
    }
    if ((rc = convert_ct(type, g))) return rc;
    // The packed copy is an optimisation: without room for it the tracer samples
    // the CT directly.
    ctQuadValid = false;
    if (ctQuad.ensure(ct_quad_bytes(g.dims)) == PBS_OK) {
        PBS_CUDA(launch_ct_quad(static_cast<const float*>(ct.ptr), g.dims, static_cast<float4*>(ctQuad.ptr), stream),
                 "ct_quad");
        ctQuadValid = true;
    } else {
        cudaGetLastError();
        set_error("");
    }
    return PBS_OK;
}

// CT adapter on the device (wrapper.cu:2290-2441): to HU+1000 in place.
int Context::convert_ct(int type, const GridDesc& g) {
    const size_t n = size_t(g.dims[0]) * g.dims[1] * g.dims[2];
    int rc = convert_ct_buffer(static_cast<float*>(ct.ptr), n, type);
    if (rc) return rc;
    ctType = type;
    ctGrid = g;
    hasCt = true;
    return PBS_OK;
}

int Context::convert_ct_buffer(float* data, size_t n, int type, const int* dims, const int* lo, const int* hi) {
    if (type == PBS_CT_DENSITY || type == PBS_CT_SPR) {
        if (!hasEnergy) {
            set_error("[CT_ADAPTER] density/SPR CT needs the lookup tables; call set_energy first");
            return PBS_ERR_NOT_READY;
        }
        const bool useDensity = type == PBS_CT_DENSITY;
        const float scale = useDensity ? energy.density_scale_fact : energy.sp_scale_fact;
        const int lutN = int(useDensity ? densityHost.size() : spHost.size());
        if (lutN == 0 || scale == 0.0f) {
            set_error("[CT_ADAPTER] LUT is empty or scale factor is 0; cannot convert");
            return PBS_ERR_INVALID_ARGUMENT;
        }
        const float* lut = static_cast<const float*>(useDensity ? density.ptr : sp.ptr);
        PBS_CUDA(dims ? launch_ct_convert_box(data, dims, lo, hi, type, lut, lutN, scale, stream)
                      : launch_ct_convert(data, n, type, lut, lutN, scale, stream),
                 "ct_convert");
    } else {
        PBS_CUDA(dims ? launch_ct_convert_box(data, dims, lo, hi, type, nullptr, 0, 1.0f, stream)
                      : launch_ct_convert(data, n, type, nullptr, 0, 1.0f, stream),
                 "ct_convert");
    }
    return PBS_OK;
}

int Context::set_dose_grid(const GridDesc& g) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (g.dims[0] <= 0 || g.dims[1] <= 0 || g.dims[2] <= 0 ||
        !(g.res[0] > 0.0f && g.res[1] > 0.0f && g.res[2] > 0.0f)) {
        set_error("[RTD_ENTRY_ASSERT] dose grid must have positive dims and resolution");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    const size_t n = size_t(g.dims[0]) * g.dims[1] * g.dims[2];
    int rc = join_side_work();
    if (rc) return rc;
    rc = dose64.ensure(n * 8);
    if (rc) return rc;
    doseGrid = g;
    hasDose = true;
    doseBoxed = false;
    deferredInit = nullptr;
    return reset_dose(nullptr, 0);
}

int Context::reset_dose(const float* init, int onDevice) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!hasDose) {
        set_error("dose grid not set");
        return PBS_ERR_NOT_READY;
    }
    const size_t n = size_t(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2];
    if (int rc = join_side_work()) return rc;
    deferredInit = nullptr;  // superseded
    initBoxed = false;
    if (init && !onDevice) {
        // The copy waits for the work already on the context stream (the CT upload
        // among it, which the next beam needs first) and then overlaps that beam.
        int rc = floatOut.ensure(n * 4);
        if (rc) return rc;
        PBS_CUDA(cudaEventRecord(copyStart, stream), "cudaEventRecord");
        PBS_CUDA(cudaStreamWaitEvent(copyStream, copyStart, 0), "cudaStreamWaitEvent");
        PBS_CUDA(cudaMemcpyAsync(floatOut.ptr, init, n * 4, cudaMemcpyHostToDevice, copyStream), "dose H2D");
        copiedH2D += n * 4;
        PBS_CUDA(cudaEventRecord(doseCopied, copyStream), "cudaEventRecord");
        pendingDoseInit = true;
        doseBoxed = false;
        return bioModel ? clear_bio() : PBS_OK;
    }
    pendingDoseInit = false;
    if (bioModel) {
        if (int rc = clear_bio()) return rc;
    }
    if (!init && doseBoxed && !doseExposed) {
        // Zero outside the dirty box already: clearing the box clears the grid. The
        // clear waits for the work on the context stream (the last readout) and
        // then runs beside the next beam's trace; flush_dose_init joins it.
        if (!box_empty(dirtyLo, dirtyHi)) {
            PBS_CUDA(cudaEventRecord(copyStart, stream), "cudaEventRecord");
            PBS_CUDA(cudaStreamWaitEvent(copyStream, copyStart, 0), "cudaStreamWaitEvent");
            PBS_CUDA(launch_dose_box(static_cast<double*>(dose64.ptr), nullptr, doseGrid.dims, dirtyLo, dirtyHi,
                                     copyStream),
                     "dose_box_zero");
            PBS_CUDA(cudaEventRecord(doseZeroed, copyStream), "cudaEventRecord");
            pendingDoseZero = true;
        }
    } else {
        PBS_CUDA(launch_dose_init(static_cast<double*>(dose64.ptr), init, n, stream), "dose_init");
    }
    doseBoxed = !init && !doseExposed;
    for (int i = 0; i < 3; ++i) {
        dirtyLo[i] = INT_MAX;
        dirtyHi[i] = -1;
    }
    return PBS_OK;
}

void Context::mark_dose_written(const int lo[3], const int hi[3]) {
    if (!doseBoxed || box_empty(lo, hi)) return;
    // One voxel of margin around the host bound of the transfer's writes.
    int a[3], b[3];
    for (int i = 0; i < 3; ++i) {
        a[i] = std::max(lo[i] - 1, 0);
        b[i] = std::min(hi[i] + 1, doseGrid.dims[i] - 1);
    }
    merge_box(dirtyLo, dirtyHi, a, b);
}

int Context::join_side_work() {
    if (pendingDoseZero) {
        PBS_CUDA(cudaStreamWaitEvent(stream, doseZeroed, 0), "cudaStreamWaitEvent");
        pendingDoseZero = false;
    }
    if (pendingBevClear) {
        PBS_CUDA(cudaStreamWaitEvent(stream, bevCleared, 0), "cudaStreamWaitEvent");
        pendingBevClear = false;
    }
    return PBS_OK;
}

int Context::flush_dose_init() {
    if (int rc = join_side_work()) return rc;
    if (!pendingDoseInit) return PBS_OK;
    if (int rc = issue_dose_copy()) return rc;
    const size_t n = size_t(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2];
    PBS_CUDA(cudaStreamWaitEvent(stream, doseCopied, 0), "cudaStreamWaitEvent");
    if (initBoxed) {
        // Only the uploaded box: the voxels outside it are neither written by the
        // call's beams nor copied back (reset_dose_region).
        PBS_CUDA(launch_dose_box_init(static_cast<double*>(dose64.ptr), static_cast<const float*>(floatOut.ptr),
                                      doseGrid.dims, deferredLo, deferredHi, stream),
                 "dose_init");
    } else {
        PBS_CUDA(launch_dose_init(static_cast<double*>(dose64.ptr), static_cast<const float*>(floatOut.ptr), n, stream),
                 "dose_init");
    }
    pendingDoseInit = false;
    initBoxed = false;
    return PBS_OK;
}

int Context::read_dose(float* out, int onDevice) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!hasDose) {
        set_error("dose grid not set");
        return PBS_ERR_NOT_READY;
    }
    const size_t n = size_t(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2];
    int frc = flush_dose_init();
    if (frc) return frc;
    if (!onDevice) {
        int rc = floatOut.ensure(n * 4);
        if (rc) return rc;
    }
    float* dst = onDevice ? out : static_cast<float*>(floatOut.ptr);
    if (doseBoxed && !doseExposed) {
        PBS_CUDA(cudaMemsetAsync(dst, 0, n * 4, stream), "dose memset");
        if (!box_empty(dirtyLo, dirtyHi))
            PBS_CUDA(launch_dose_box(static_cast<double*>(dose64.ptr), dst, doseGrid.dims, dirtyLo, dirtyHi, stream),
                     "dose_to_float");
    } else {
        PBS_CUDA(launch_dose_to_float(static_cast<const double*>(dose64.ptr), dst, n, stream), "dose_to_float");
    }
    if (onDevice) return PBS_OK;
    PBS_CUDA(cudaMemcpyAsync(out, floatOut.ptr, n * 4, cudaMemcpyDeviceToHost, stream), "dose D2H");
    copiedD2H += n * 4;
    PBS_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    return take_device_errors();
}

int Context::read_dose64(double* out, int onDevice) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!hasDose) {
        set_error("dose grid not set");
        return PBS_ERR_NOT_READY;
    }
    const size_t n = size_t(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2];
    int frc = flush_dose_init();
    if (frc) return frc;
    PBS_CUDA(cudaMemcpyAsync(out, dose64.ptr, n * 8, onDevice ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost,
                             stream),
             "dose64 copy");
    if (!onDevice) {
        PBS_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
        return take_device_errors();
    }
    return PBS_OK;
}

BeamBuffers beam_buffers(const BeamPlan& P, size_t nSubspotData, int nuclear, long long layerBudgetMiB) {
    BeamBuffers z;
    const size_t L = size_t(P.numLayers), S = size_t(P.tracerSteps);
    const size_t rays = size_t(P.rayDims[0]) * P.rayDims[1];
    const size_t pitchX = size_t(P.superpDims[0]), pitchY = size_t(P.superpDims[1]);
    const size_t padPlane = pitchX * pitchY;
    const size_t tiles = (pitchX / kTileX) * (pitchY / kTileY);
    const size_t perLayer = S * padPlane * 8 + S * tiles * (1 + sizeof(int4));
    const size_t budget = size_t(std::max<long long>(layerBudgetMiB, 1)) << 20;
    z.chunk = int(std::max<size_t>(1, std::min<size_t>(budget / std::max<size_t>(perLayer, 1), L)));
    z.chunk = std::min(z.chunk, 64);
    const size_t chunk = size_t(z.chunk);
    z.dens = z.wepl = S * rays * 4;
    z.weplMin = S * 4;
    z.firstIn = z.firstOut = rays * 4;
    z.rayW = L * rays * 4;
    z.bev = S * (pitchX + 2 * kMaxR) * (pitchY + 2 * kMaxR) * 4;
    z.codes = chunk * S * tiles;
    z.work = chunk * S * tiles * sizeof(int4);
    z.idd = z.rs = chunk * S * padPlane * 4;
    z.firstPassive = chunk * rays * 4;
    z.lp = L * sizeof(LayerParamsDev);
    z.ls = L * sizeof(LayerStateDev);
    z.bs = sizeof(BeamStateDev);
    if (P.hasLattice) {
        z.lattice = P.lattice.weights.size() * 4;
        z.interm = L * size_t(P.lattice.ny) * size_t(P.rayDims[0]) * 4;
    } else {
        z.subspots = nSubspotData * 4;
        z.cpb = L * rays * 4;
    }
    if (nuclear) {
        const size_t nucX = (size_t(P.lattice.nx) + kTileX - 1) / kTileX * kTileX;
        const size_t nucY = (size_t(P.lattice.ny) + kTileY - 1) / kTileY * kTileY;
        const size_t nucPlane = nucX * nucY, nucTiles = nucPlane / (kTileX * kTileY);
        z.rayToNuc = rays * 4;
        z.nucIdd = z.nucRs = chunk * S * nucPlane * 4;
        z.nucCodes = chunk * S * nucTiles;
        z.nucWork = chunk * S * nucTiles * sizeof(int4);
        z.nucBev = S * (nucX + 2 * kMaxR) * (nucY + 2 * kMaxR) * 4;
        z.nucLs = L * sizeof(LayerStateDev);
        z.nucBs = sizeof(BeamStateDev);
    }
    z.bevFixed = std::max(z.bev, z.nucBev) * 2;
    return z;
}

size_t BeamBuffers::total(bool withTrace) const {
    return (withTrace ? dens + wepl + weplMin + firstIn + firstOut : 0) + rayW + bev + codes + work + idd + rs +
           firstPassive + lp + ls + bs + lattice + interm + subspots + cpb + rayToNuc + nucIdd + nucRs + nucCodes +
           nucWork + nucBev + nucLs + nucBs + bevFixed;
}

size_t trace_bytes(size_t steps, size_t rays) {
    // dens, wepl | firstIn, firstOut | weplMin | inOut, each part 256-byte aligned
    auto up = [](size_t n) { return (n + 255) / 256 * 256; };
    return 2 * up(steps * rays * 4) + 2 * up(rays * 4) + up(steps * 4) + 256;
}

void Context::use_stream_ordered_allocation() {
    for (DevBuf* b : {&cidd, &density, &sp, &rrl, &ct, &ctQuad, &dose64, &dens, &wepl, &weplMin, &rayW, &interm, &lattice,
                      &iddBuf, &rsBuf, &bev, &cpb, &subspots, &floatOut, &firstIn, &firstOut, &firstPassive, &codes,
                      &work, &lp, &ls, &bs, &stats, &nucWeight, &nucSqSigma, &rayToNuc, &nucIddBuf, &nucRsBuf,
                      &nucCodes, &nucWork, &nucBev, &bevFixed, &nucLs, &nucBs, &gradDoseBuf, &bevGrad, &rbarBuf, &gradInterm,
                      &gradLattice, &weqBody, &opColPtr, &opBlockOff, &opRows, &opVals})
        if (!b->ptr) b->allocStream = stream;
}

size_t Context::device_bytes() const {
    size_t n = 0;
    for (const DevBuf* b : {&cidd, &density, &sp, &rrl, &ct, &ctQuad, &dose64, &dens, &wepl, &weplMin, &rayW, &interm, &lattice,
                            &iddBuf, &rsBuf, &bev, &cpb, &subspots, &floatOut, &firstIn, &firstOut, &firstPassive,
                            &codes, &work, &lp, &ls, &bs, &stats, &nucWeight, &nucSqSigma, &rayToNuc, &nucIddBuf,
                            &nucRsBuf, &nucCodes, &nucWork, &nucBev, &bevFixed, &nucLs, &nucBs, &errWord, &gradDoseBuf, &bevGrad,
                            &rbarBuf, &gradInterm, &gradLattice, &weqBody, &opColPtr, &opBlockOff, &opRows, &opVals,
                            &opNorm, &opVoxels, &colBev, &colFixed, &colDose})
        n += b->bytes;
    return n;
}

void Context::release_beam_buffers() {
    join_side_work();
    for (DevBuf* b : {&dens, &wepl, &weplMin, &rayW, &interm, &lattice, &iddBuf, &rsBuf, &bev, &cpb, &subspots,
                      &floatOut, &firstIn, &firstOut, &firstPassive, &codes, &work, &rayToNuc, &nucIddBuf, &nucRsBuf,
                      &nucCodes, &nucWork, &nucBev, &bevFixed, &gradDoseBuf, &bevGrad, &rbarBuf, &gradInterm, &gradLattice, &dose64,
                      &weqBody, &opColPtr, &opBlockOff, &opRows, &opVals, &opNorm, &opVoxels, &colBev, &colFixed,
                      &colDose})
        b->release();
    colClean = false;
    hasDose = false;
    doseBoxed = false;
    lastBeamValid = false;
}

int Context::attach_ct(const float* deviceCt, const GridDesc& g, int type) {
    if (!deviceCt) {
        set_error("attach_ct: null CT");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    ctView = deviceCt;
    ctQuadValid = false;
    ctGrid = g;
    ctType = type;
    hasCt = true;
    return PBS_OK;
}

int Context::add_beam(const PbsBeamDesc& b, int nuclear) { return run_beam(b, nuclear, nullptr); }

int Context::add_planned_beam(const PbsBeamDesc& b, int nuclear, BeamPlan&& planned) {
    return run_beam(b, nuclear, nullptr, &planned);
}

int Context::adjoint_beam(const PbsBeamDesc& b, const double* gradDose, int gradOnDevice, float* gradSpots,
                          size_t nSpots) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!hasDose) {
        set_error("dose grid not set");
        return PBS_ERR_NOT_READY;
    }
    size_t total = 0;
    for (size_t l = 0; l < b.n_layer_spot_counts && b.layer_spot_counts; ++l) total += size_t(b.layer_spot_counts[l]);
    if (!gradDose || !gradSpots || nSpots != total) {
        set_error("adjoint: the gradient output needs one float per spot of the beam");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    const size_t n = size_t(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2];
    const double* dGrad = gradDose;
    if (!gradOnDevice) {
        int rc = gradDoseBuf.ensure(n * 8);
        if (rc) return rc;
        PBS_CUDA(cudaMemcpyAsync(gradDoseBuf.ptr, gradDose, n * 8, cudaMemcpyHostToDevice, stream), "grad H2D");
        dGrad = static_cast<const double*>(gradDoseBuf.ptr);
    }
    AdjointArgs a{dGrad, gradSpots, nSpots};
    return run_beam(b, 0, &a);
}

int Context::run_beam(const PbsBeamDesc& b, int nuclear, const AdjointArgs* adj, BeamPlan* planned,
                      ColumnSink* cols) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (cols && (nuclear || adj || bioModel)) {
        set_error("batched influence columns: not available with the nuclear halo, the adjoint or biological maps");
        return PBS_ERR_UNSUPPORTED;
    }
    // Buffers may be resized below: nothing of an earlier beam may still be clearing them.
    if (int jrc = join_side_work()) return jrc;
    if (!hasEnergy || !hasCt || !hasDose) {
        set_error("context needs lookup tables, CT and dose grid before add_beam");
        return PBS_ERR_NOT_READY;
    }
    if (nuclear) {  // enforceNuclearCorrectionContract (wrapper.cu:1077-1097)
        if (!luts.nucWeight || !luts.nucSqSigma) {
            set_error("nuclear_correction=true requested, but RTDEnergyStruct does not carry nuclear_weight/sigma tables");
            return PBS_ERR_UNSUPPORTED;
        }
        if (!nucTablesAligned) {
            set_error("nuclear_correction=true requested, but nuclear LUTs are not aligned to the active primary "
                      "energy-depth axis");
            return PBS_ERR_UNSUPPORTED;
        }
    }
    std::string err;
    if (!validate_beam(b, 0, err)) {
        set_error(err);
        return PBS_ERR_INVALID_ARGUMENT;
    }
    lastBeamValid = false;
    int rc = PBS_OK;
    if (planned) {
        plan = std::move(*planned);
    } else if ((rc = plan_beam(b, energy, ctGrid, doseGrid, plan, err))) {
        set_error(err);
        return rc;
    }
    if (nuclear && !plan.hasLattice) {
        set_error("nuclear_correction=true requires raw spot lattice inputs; legacy CPB fallback cannot drive halo mode");
        return PBS_ERR_UNSUPPORTED;
    }
    if (bioModel && (nuclear || adj)) {
        set_error(nuclear ? "biological maps: beams with the nuclear halo are not supported while a model is set"
                          : "biological maps: clear the model (PBS_BIO_OFF) before the spot-weight adjoint");
        return PBS_ERR_UNSUPPORTED;
    }
    const BeamPlan& P = plan;
    BeamGeomDev& g = geom;
    std::memset(&g, 0, sizeof(g));
    g.tracer = P.tracer;
    g.rayIdxToDoseIdx = P.rayIdxToDoseIdx;
    g.rayX = P.rayDims[0];
    g.rayY = P.rayDims[1];
    g.pitchX = P.superpDims[0];
    g.pitchY = P.superpDims[1];
    g.tilesX = g.pitchX / kTileX;
    g.tilesY = g.pitchY / kTileY;
    g.steps = P.tracerSteps;
    g.numLayers = P.numLayers;
    g.maxPeakDepthMm = P.maxPeakDepthMm;
    g.fanCorner = P.fanCorner;
    g.fanDelta = P.fanDelta;
    g.sourceDist = P.sourceDist;
    g.volConst = P.volConst;
    g.volLin = P.volLin;
    g.volSq = P.volSq;
    g.latNx = P.lattice.nx;
    g.latNy = P.lattice.ny;
    g.latDx = P.lattice.dx;
    g.latDy = P.lattice.dy;
    g.latOx = P.lattice.ox;
    g.latOy = P.lattice.oy;
    g.cpbCornerX = P.cpbCorner.x;
    g.cpbCornerY = P.cpbCorner.y;
    g.cpbResX = P.cpbRes.x;
    g.cpbResY = P.cpbRes.y;
    g.bevX = g.pitchX + 2 * kMaxR;
    g.bevY = g.pitchY + 2 * kMaxR;
    g.doseX = doseGrid.dims[0];
    g.doseY = doseGrid.dims[1];
    g.doseZ = doseGrid.dims[2];
    g.compatBevZShift = compatBevZShift;
    g.errWord = static_cast<int*>(errWord.ptr);
    // Transport constants (idd_sigma.cu:102-121) and the nuclear halo grid.
    g.eRefSq = 198.81f;
    g.sigmaDelta = 0.21f;
    g.suppressDistalDip = 0;
    g.entrySigmaScale = 1.0f;
    if (nuclear) {
        if (nuclearModel == 0) {  // SOUKUP
            g.eRefSq = 190.44f;
            g.sigmaDelta = 0.0f;
        } else if (nuclearModel == 1) {  // FLUKA
            g.eRefSq = 216.09f;
            g.sigmaDelta = 0.08f;
        } else {  // GAUSS_FIT (wrapper.cu:3788-3795 narrows the entry sigma too)
            g.eRefSq = 169.00f;
            g.sigmaDelta = 0.06f;
            g.suppressDistalDip = 1;
            g.entrySigmaScale = 0.97f;
        }
        g.nucOn = 1;
        g.nucX = (P.lattice.nx + kTileX - 1) / kTileX * kTileX;
        g.nucY = (P.lattice.ny + kTileY - 1) / kTileY * kTileY;
    }
    // Halo lattice plan (buildHaloLatticePlan, wrapper.cu:804-929): the ray under
    // every lattice cell; the halo grid is the spot lattice padded to 32 x 8.
    std::vector<int> hRayToNuc;
    if (nuclear) {
        hRayToNuc.assign(size_t(g.rayX) * g.rayY, -1);
        for (int sy = 0; sy < P.lattice.ny; ++sy) {
            const float gy = P.lattice.oy + float(sy) * P.lattice.dy;
            const int ry = int(std::lround((gy - P.cpbCorner.y) / P.cpbRes.y));
            if (ry < 0 || ry >= g.rayY) {
                set_error("failed to build halo lattice plan: dense halo lattice row mapped outside active ray grid");
                return PBS_ERR_GEOMETRY;
            }
            for (int sx = 0; sx < P.lattice.nx; ++sx) {
                const float gx = P.lattice.ox + float(sx) * P.lattice.dx;
                const int rx = int(std::lround((gx - P.cpbCorner.x) / P.cpbRes.x));
                if (rx < 0 || rx >= g.rayX) {
                    set_error("failed to build halo lattice plan: dense halo lattice column mapped outside active ray "
                              "grid");
                    return PBS_ERR_GEOMETRY;
                }
                hRayToNuc[size_t(ry) * g.rayX + rx] = sy * g.nucX + sx;
            }
        }
        BeamGeomDev& gn = nucGeom;
        gn = g;
        gn.pitchX = g.nucX;
        gn.pitchY = g.nucY;
        gn.tilesX = g.nucX / kTileX;
        gn.tilesY = g.nucY / kTileY;
        gn.bevX = g.nucX + 2 * kMaxR;
        gn.bevY = g.nucY + 2 * kMaxR;
        // Halo BEV index -> dose index: the lattice spacing and offset (used as mm,
        // wrapper.cu:5522-5535) replace the ray grid in x and y.
        gn.rayIdxToDoseIdx.fanIdxToFan = idxxf(v3(P.lattice.dx, P.lattice.dy, P.fanDelta.z),
                                               v3(P.lattice.ox, P.lattice.oy, P.fanCorner.z));
    }
    lastNuclear = nuclear != 0;

    const int L = P.numLayers;
    const size_t S = size_t(P.tracerSteps);
    const size_t tiles = size_t(g.tilesX) * g.tilesY;
    const BeamBuffers z = beam_buffers(P, b.n_subspot_data, nuclear, layerBudgetMiB);
    // The reference transfers every layer on its own, with the box of that layer's
    // steps [first, calcPassive) (wrapper.cu:5343-5505). With its BEV depth indexing
    // (compat) a layer's dose lands deeper than its own steps and that box cuts it
    // off, so in that mode the layers are superposed and transferred one at a time.
    const bool perLayerTransfer = compatBevZShift && !adj;
    const int chunk = perLayerTransfer ? 1 : z.chunk;
    chunkLayers = chunk;
    // Batched influence columns (a sink): each layer of a chunk is superposed from its
    // own work list, selected from the chunk's one-layer list, and transferred alone.
    const bool columnLists = cols && !perLayerTransfer;
    size_t colCells = 0;
    if (columnLists) {
        size_t perColumn = 0;
        column_layout(P, colBox, colCells, perColumn);
        const size_t fbN = size_t(colBox.ext[0]) * colBox.ext[1] * colBox.ext[2];
        const size_t c = size_t(chunk);
        const bool had = colBev.bytes >= c * colCells * 4 && colFixed.bytes >= c * colCells * 8 &&
                         colDose.bytes >= c * fbN * 8;
        if ((rc = colBev.ensure(c * colCells * 4)) || (rc = colFixed.ensure(c * colCells * 8)) ||
            (rc = colDose.ensure(c * fbN * 8)))
            return rc;
        if (!had || !colClean) {
            PBS_CUDA(cudaMemsetAsync(colBev.ptr, 0, colBev.bytes, stream), "memset column BEV");
            PBS_CUDA(cudaMemsetAsync(colFixed.ptr, 0, colFixed.bytes, stream), "memset column BEV");
            PBS_CUDA(cudaMemsetAsync(colDose.ptr, 0, colDose.bytes, stream), "memset column dose");
        }
        // Clean again once every chunk's columns are compacted and cleared.
        colClean = false;
    }

    // The trace's home: the store's resident copy for this geometry, else the
    // context's own buffers.
    trace = TraceSlot{};
    // A WEQ beam's trace is its own input, not a function of the geometry: never shared.
    if (traceStore && !P.hasWeqVolume && (rc = traceStore->acquire(*this, g, trace))) return rc;
    if (!trace.dens) {
        if ((rc = dens.ensure(z.dens)) || (rc = wepl.ensure(z.wepl)) || (rc = weplMin.ensure(z.weplMin)) ||
            (rc = firstIn.ensure(z.firstIn)) || (rc = firstOut.ensure(z.firstOut)))
            return rc;
        trace.dens = static_cast<float*>(dens.ptr);
        trace.wepl = static_cast<float*>(wepl.ptr);
        trace.firstIn = static_cast<int*>(firstIn.ptr);
        trace.firstOut = static_cast<int*>(firstOut.ptr);
        trace.weplMin = static_cast<float*>(weplMin.ptr);
    }
    if ((rc = rayW.ensure(z.rayW)) || (rc = bev.ensure(z.bev)) || (rc = codes.ensure(z.codes)) ||
        (rc = work.ensure(z.work)) || (rc = iddBuf.ensure(z.idd)) || (rc = rsBuf.ensure(z.rs)) ||
        (rc = firstPassive.ensure(z.firstPassive)) || (rc = lp.ensure(z.lp)) || (rc = ls.ensure(z.ls)) ||
        (rc = bs.ensure(z.bs)))
        return rc;
    const size_t nucPlane = size_t(g.nucX) * g.nucY, nucTiles = nucPlane / (kTileX * kTileY);
    if (nuclear &&
        ((rc = rayToNuc.ensure(z.rayToNuc)) || (rc = nucIddBuf.ensure(z.nucIdd)) || (rc = nucRsBuf.ensure(z.nucRs)) ||
         (rc = nucCodes.ensure(z.nucCodes)) || (rc = nucWork.ensure(z.nucWork)) || (rc = nucBev.ensure(z.nucBev)) ||
         (rc = nucLs.ensure(z.nucLs)) || (rc = nucBs.ensure(z.nucBs))))
        return rc;
    if (!adj) {
        const size_t had = bevFixed.bytes;
        if ((rc = bevFixed.ensure(z.bevFixed))) return rc;
        if (bevFixed.bytes != had || !bevFixedClean) {
            PBS_CUDA(cudaMemsetAsync(bevFixed.ptr, 0, bevFixed.bytes, stream), "memset fixed BEV");
            bevFixedClean = true;
        }
    }
    if (idd_smem_bytes(g, luts) > size_t(200) * 1024) {
        set_error("beam needs " + std::to_string(P.tracerSteps) + " tracer steps; at most ~3000 are supported");
        return PBS_ERR_UNSUPPORTED;
    }
    if (adj && compatBevZShift) {
        // The forward of that mode transfers each layer with its own box.
        set_error("adjoint: not available with PBS_OPT_COMPAT_BEV_Z_SHIFT");
        return PBS_ERR_UNSUPPORTED;
    }
    if (adj && (chunk < L || nuclear || !P.hasLattice)) {
        set_error(chunk < L ? "adjoint: every layer of the beam must fit one chunk; raise PBS_OPT_LAYER_BUDGET_MIB"
                            : "adjoint: needs a beam with a raw spot lattice and no nuclear halo");
        return PBS_ERR_UNSUPPORTED;
    }
    if (keepDebug && chunk < L) {
        if (perLayerTransfer) {
            set_error("PBS_OPT_KEEP_DEBUG with PBS_OPT_COMPAT_BEV_Z_SHIFT needs a beam of one layer");
            return PBS_ERR_UNSUPPORTED;
        }
        set_error("PBS_OPT_KEEP_DEBUG needs every layer of the beam in one chunk; raise PBS_OPT_LAYER_BUDGET_MIB");
        return PBS_ERR_OUT_OF_MEMORY;
    }

    // Biological model: the layers' fractional rows on the LET table's energy axis.
    const bool bio = bioModel != 0;
    if (bio) {
        std::vector<float> rows(L);
        for (int l = 0; l < L; ++l)
            rows[l] = find_fractional_index_monotonic(bioLetEnergies.data(), int(bioLetEnergies.size()),
                                                      b.energies[l]);
        const size_t bevN = S * size_t(g.bevX) * g.bevY;
        const int nCh = bioModel == PBS_BIO_LQ ? 3 : 2;
        if ((rc = bioLayerRow.ensure(size_t(L) * 4)) || (rc = bioIdd.ensure(z.idd)) ||
            (rc = bioBev.ensure(size_t(nCh) * bevN * 4)))
            return rc;
        if ((rc = upload(bioLayerRow.ptr, rows.data(), size_t(L) * 4))) return rc;
        PBS_CUDA(cudaMemsetAsync(bioBev.ptr, 0, size_t(nCh) * bevN * 4, stream), "memset bio BEV");
    }

    // CarbonPBS lateral profile model: which of its two parts this beam runs.
    ProfilePlan prof;
    if (carbonProfile) {
        plan_carbon_profile(b, energy, P, prof);
        if ((carbonProfile & 1) && prof.sigmaOverride()) g.profileMode |= 1;
        if ((carbonProfile & 2) && prof.overallWeight()) g.profileMode |= 2;
    }
    const size_t profBytes = g.profileMode ? b.n_profile_data * 4 : 0;
    if (profBytes) {
        if ((rc = profileBuf.ensure(profBytes))) return rc;
        g.profile = static_cast<const float*>(profileBuf.ptr);
        g.profileRows = prof.rows;
        g.profileDepthN = prof.depthN;
        g.profileChannels = prof.channels;
        g.profileDepth0 = prof.depth0;
        g.profileDepthStep = prof.depthStep;
        g.beamParaPos = b.beam_para_pos;
    }

    // Host -> device inputs of the beam: layer parameters, initial beam state and
    // the fluence source (dense spot lattice or legacy subspot table).
    std::vector<LayerParamsDev> hlp(L);
    for (int l = 0; l < L; ++l) {
        const LayerHost& H = P.layers[l];
        LayerParamsDev& d = hlp[l];
        d.energyIdx = H.energyIdx;
        d.energyScaleFact = H.energyScaleFact;
        d.peakDepth = H.peakDepth;
        d.rangeStopDepth = H.rangeStopDepth;
        d.sigmaSqAirQuad = H.sigmaSqAirQuad;
        d.sigmaSqAirLin = H.sigmaSqAirLin;
        d.convPeakDepth = H.convPeakDepth;
        d.sigmaXmm = H.sigmaXmm;
        d.sigmaYmm = H.sigmaYmm;
        d.spotDist = H.spotDist;
        if (g.profileMode) {
            d.profileRow = prof.row[l];
            d.bp0 = prof.bp0[l];
            d.bp1 = prof.bp1[l];
            d.bp2 = prof.bp2[l];
        }
        // With the halo the lattice spacing is taken as mm when the beam gives no
        // explicit spot spacing (wrapper.cu:4333-4347).
        if (nuclear && std::fabs(P.fanDelta.x) > 1e-6f) {
            const float spacing = b.spot_delta[0] > b.ray_spacing[0] * 1.5f ? b.spot_delta[0] : P.lattice.dx;
            d.spotDist = std::fabs(spacing / P.fanDelta.x);
        }
    }
    layerSpotDist.resize(L);
    for (int l = 0; l < L; ++l) layerSpotDist[l] = hlp[l].spotDist;
    BeamStateDev hbs;
    std::memset(&hbs, 0, sizeof(hbs));
    hbs.firstInside = INT32_MAX;
    hbs.firstOutside = INT32_MIN;
    for (int i = 0; i < 3; ++i) {
        hbs.liveLo[i] = INT32_MAX;
        hbs.liveHi[i] = INT32_MIN;
    }
    const size_t latBytes = P.hasLattice ? P.lattice.weights.size() * 4 : 0;
    const size_t subBytes = P.hasLattice ? 0 : b.n_subspot_data * 4;
    const size_t nucMapBytes = nuclear ? hRayToNuc.size() * 4 : 0;
    const size_t upBytes = hlp.size() * sizeof(LayerParamsDev) + 2 * sizeof(BeamStateDev) + latBytes + subBytes +
                           nucMapBytes + profBytes;
    {
        PBS_CUDA(cudaEventSynchronize(stagingEvent), "cudaEventSynchronize");
        if ((rc = staging.ensure(upBytes + 256))) return rc;
        char* p = static_cast<char*>(staging.ptr);
        std::memcpy(p, hlp.data(), hlp.size() * sizeof(LayerParamsDev));
        PBS_CUDA(cudaMemcpyAsync(lp.ptr, p, hlp.size() * sizeof(LayerParamsDev), cudaMemcpyHostToDevice, stream), "H2D");
        p += hlp.size() * sizeof(LayerParamsDev);
        std::memcpy(p, &hbs, sizeof(hbs));
        PBS_CUDA(cudaMemcpyAsync(bs.ptr, p, sizeof(hbs), cudaMemcpyHostToDevice, stream), "H2D");
        p += sizeof(hbs);
        if (latBytes) {
            if ((rc = lattice.ensure(z.lattice)) || (rc = interm.ensure(z.interm))) return rc;
            std::memcpy(p, P.lattice.weights.data(), latBytes);
            PBS_CUDA(cudaMemcpyAsync(lattice.ptr, p, latBytes, cudaMemcpyHostToDevice, stream), "H2D");
            p += latBytes;
        }
        if (subBytes) {
            if ((rc = subspots.ensure(z.subspots)) || (rc = cpb.ensure(z.cpb))) return rc;
            std::memcpy(p, b.subspot_data, subBytes);
            PBS_CUDA(cudaMemcpyAsync(subspots.ptr, p, subBytes, cudaMemcpyHostToDevice, stream), "H2D");
            p += subBytes;
        }
        if (nuclear) {
            std::memcpy(p, hRayToNuc.data(), nucMapBytes);
            PBS_CUDA(cudaMemcpyAsync(rayToNuc.ptr, p, nucMapBytes, cudaMemcpyHostToDevice, stream), "H2D");
            p += nucMapBytes;
            std::memcpy(p, &hbs, sizeof(hbs));
            PBS_CUDA(cudaMemcpyAsync(nucBs.ptr, p, sizeof(hbs), cudaMemcpyHostToDevice, stream), "H2D");
            p += sizeof(hbs);
            PBS_CUDA(cudaMemsetAsync(nucLs.ptr, 0, size_t(L) * sizeof(LayerStateDev), stream), "memset");
            PBS_CUDA(cudaMemsetAsync(nucBev.ptr, 0, S * nucGeom.bevX * nucGeom.bevY * 4, stream), "memset");
        }
        if (profBytes) {
            std::memcpy(p, b.profile_data, profBytes);
            PBS_CUDA(cudaMemcpyAsync(profileBuf.ptr, p, profBytes, cudaMemcpyHostToDevice, stream), "H2D");
            p += profBytes;
        }
        PBS_CUDA(cudaEventRecord(stagingEvent, stream), "cudaEventRecord");
        copiedH2D += upBytes;
    }

    LayerParamsDev* dlp = static_cast<LayerParamsDev*>(lp.ptr);
    LayerStateDev* dls = static_cast<LayerStateDev*>(ls.ptr);
    BeamStateDev* dbs = static_cast<BeamStateDev*>(bs.ptr);
    float* dDens = trace.dens;
    float* dWepl = trace.wepl;
    int* dFi = trace.firstIn;
    int* dFo = trace.firstOut;
    float* dRayW = static_cast<float*>(rayW.ptr);
    float* dBev = static_cast<float*>(bev.ptr);
    auto mark = [&](int slot) -> int {
        if (stageTiming) PBS_CUDA(cudaEventRecord(ev[slot], stream), "cudaEventRecord");
        return PBS_OK;
    };

    // The BEV clear runs beside the trace, the planner and the fluence kernels;
    // the superposition waits for it.
    PBS_CUDA(cudaEventRecord(copyStart, stream), "cudaEventRecord");
    PBS_CUDA(cudaStreamWaitEvent(copyStream, copyStart, 0), "cudaStreamWaitEvent");
    PBS_CUDA(cudaMemsetAsync(dBev, 0, S * g.bevX * g.bevY * 4, copyStream), "memset BEV");
    PBS_CUDA(cudaEventRecord(bevCleared, copyStream), "cudaEventRecord");
    pendingBevClear = true;
    if ((rc = mark(0))) return rc;
    static_assert(offsetof(BeamStateDev, firstOutside) == offsetof(BeamStateDev, firstInside) + sizeof(int),
                  "the trace's beam steps are two adjacent ints");
    if (trace.traced) {
        // A resident trace of this geometry: its beam steps replace the tracer's.
        PBS_CUDA(cudaStreamWaitEvent(stream, trace.ready, 0), "cudaStreamWaitEvent");
        PBS_CUDA(cudaMemcpyAsync(&dbs->firstInside, trace.inOut, 2 * sizeof(int), cudaMemcpyDeviceToDevice, stream),
                 "trace steps D2D");
    } else if (P.hasWeqVolume) {
        // Water-equivalence import: the exporter's depths replace the CT trace.
        const size_t weqN = size_t(P.weqNx) * P.weqNy * P.weqSteps;
        if ((rc = weqBody.ensure(weqN * 4))) return rc;
        PBS_CUDA(cudaMemcpyAsync(weqBody.ptr, b.water_equivalence + 9, weqN * 4, cudaMemcpyHostToDevice, stream),
                 "WEQ H2D");
        copiedH2D += weqN * 4;
        PBS_CUDA(launch_weq_trace(g, static_cast<const float*>(weqBody.ptr), P.weqNx, P.weqNy, P.weqSteps,
                                  P.weqActiveSteps, P.weqStepMm, P.cpbCorner.x, P.cpbCorner.y, P.cpbRes.x, P.cpbRes.y,
                                  P.weqX0, P.weqY0, P.weqDx, P.weqDy, dDens, dWepl, dFi, dFo, trace.weplMin, dbs,
                                  stream),
                 "weq_trace");
    } else {
        const float4* quad = !ctView && ctQuadValid ? static_cast<const float4*>(ctQuad.ptr) : nullptr;
        PBS_CUDA(launch_trace(g, luts, ctView ? ctView : static_cast<const float*>(ct.ptr), quad, ctGrid.dims[0],
                              ctGrid.dims[1], ctGrid.dims[2], dDens, dWepl, dFi, dFo, trace.weplMin, dbs, stream),
                 "trace");
        if (trace.inOut) {
            PBS_CUDA(cudaMemcpyAsync(trace.inOut, &dbs->firstInside, 2 * sizeof(int), cudaMemcpyDeviceToDevice,
                                     stream),
                     "trace steps D2D");
            if ((rc = traceStore->traced(*this, trace))) return rc;
        }
    }
    if ((rc = mark(1))) return rc;
    if ((rc = issue_dose_copy())) return rc;
    PBS_CUDA(launch_beam_planner(g, trace.weplMin, dlp, dls, dbs, stream), "beam_planner");
    if ((rc = mark(2))) return rc;
    if (P.hasLattice) {
        PBS_CUDA(launch_conv_lattice(g, static_cast<const float*>(lattice.ptr), static_cast<float*>(interm.ptr), dRayW,
                                     dls, dbs, stream),
                 "conv_lattice");
    } else {
        PBS_CUDA(launch_conv_cpb(g, static_cast<const float*>(subspots.ptr), b.max_subspots_per_layer,
                                 static_cast<float*>(cpb.ptr), dRayW, stream),
                 "conv_cpb");
    }
    if ((rc = mark(3))) return rc;
    if (smCount <= 0) PBS_CUDA(cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, device), "SM count");
    const int workCap = int(size_t(chunk) * S * tiles);
    const int nucWorkCap = int(size_t(chunk) * S * nucTiles);
    float* dNucIdd = static_cast<float*>(nucIddBuf.ptr);
    float* dNucRs = static_cast<float*>(nucRsBuf.ptr);
    LayerStateDev* dNucLs = static_cast<LayerStateDev*>(nucLs.ptr);
    BeamStateDev* dNucBs = static_cast<BeamStateDev*>(nucBs.ptr);
    if ((rc = join_side_work())) return rc;
    // BEV -> dose: the box over the steps of every layer, or of `layer` (and of
    // `nucLayer` for the halo) alone; the dose grid's pending initialisation and
    // dirty box are settled before the first transfer.
    bool doseReady = false;
    auto transfer_layers = [&](const LayerStateDev* layer, const LayerStateDev* nucLayer) -> int {
        int trc;
        if (!doseReady) {
            if ((trc = flush_dose_init())) return trc;
            if (doseBoxed) {
                int lo[3], hi[3];
                dose_transfer_box(plan.rayIdxToDoseIdx, plan.superpDims[0], plan.superpDims[1], plan.tracerSteps,
                                  doseGrid.dims, lo, hi);
                mark_dose_written(lo, hi);
                if (nuclear) {
                    dose_transfer_box(nucGeom.rayIdxToDoseIdx, nucGeom.pitchX, nucGeom.pitchY, plan.tracerSteps,
                                      doseGrid.dims, lo, hi);
                    mark_dose_written(lo, hi);
                }
            }
            doseReady = true;
        }
        // The box over the cells the items wrote (work_merge_kernel) for the whole beam;
        // the per-layer transfers of the reference's depth convention take the box over
        // the layer's steps.
        PBS_CUDA(launch_transfer_planner(g, dbs, layer, layer == nullptr, stream), "transfer_planner");
        PBS_CUDA(launch_transfer(g, dBev, dbs, static_cast<double*>(dose64.ptr), stream), "transfer");
        if (bio) {
            // The beam's own dose and the channels into the biological accumulators.
            const size_t n = size_t(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2];
            const size_t bevN = S * size_t(g.bevX) * g.bevY;
            double* acc = static_cast<double*>(bioAcc.ptr);
            PBS_CUDA(launch_transfer(g, dBev, dbs, acc, stream), "bio transfer");
            const int nCh = bioModel == PBS_BIO_LQ ? 3 : 2;
            for (int slot = 0; slot < nCh; ++slot) {
                // Slots are channels 0, 1, 2 (LQ) or 0, 2 (MKM); accumulator c + 1.
                const int c = bioModel == PBS_BIO_LQ ? slot : (slot == 0 ? 0 : 2);
                PBS_CUDA(launch_transfer(g, static_cast<const float*>(bioBev.ptr) + size_t(slot) * bevN, dbs,
                                         acc + size_t(c + 1) * n, stream),
                         "bio transfer");
            }
        }
        if (nuclear) {
            PBS_CUDA(launch_transfer_planner(nucGeom, dNucBs, nucLayer, nucLayer == nullptr, stream),
                     "nuc_transfer_planner");
            PBS_CUDA(launch_transfer(nucGeom, static_cast<const float*>(nucBev.ptr), dNucBs,
                                     static_cast<double*>(dose64.ptr), stream),
                     "nuc_transfer");
        }
        return PBS_OK;
    };
    for (int l0 = 0; l0 < L; l0 += chunk) {
        const int nl = std::min(chunk, L - l0);
        if (nuclear) PBS_CUDA(launch_nuc_prepare(nucGeom, nl, dNucIdd, dNucRs, stream), "nuc_prepare");
        PBS_CUDA(launch_idd(g, luts, l0, nl, dDens, dWepl, dFi, dFo, dRayW, dlp, dls, dbs,
                            static_cast<float*>(iddBuf.ptr), static_cast<float*>(rsBuf.ptr),
                            static_cast<uint8_t*>(codes.ptr), static_cast<int*>(firstPassive.ptr),
                            static_cast<const int*>(rayToNuc.ptr), static_cast<const float*>(lattice.ptr), dNucIdd,
                            dNucRs, stream),
                 "idd");
        if (l0 == 0 && (rc = mark(4))) return rc;
        PBS_CUDA(launch_bin_plan(g, l0, nl, static_cast<const uint8_t*>(codes.ptr), dls, dbs,
                                 static_cast<int4*>(work.ptr), workCap, adj == nullptr && !columnLists, nullptr,
                                 nullptr, stream),
                 "bin_plan");
        if (nuclear) {
            PBS_CUDA(launch_nuc_codes(nucGeom, l0, nl, dNucIdd, dNucRs, dls, dbs, dNucLs,
                                      static_cast<uint8_t*>(nucCodes.ptr), stream),
                     "nuc_codes");
            PBS_CUDA(launch_bin_plan(nucGeom, l0, nl, static_cast<const uint8_t*>(nucCodes.ptr), dNucLs, dNucBs,
                                     static_cast<int4*>(nucWork.ptr), nucWorkCap, adj == nullptr, dls, dbs, stream),
                     "nuc_bin_plan");
        }
        if (l0 == 0 && (rc = mark(5))) return rc;
        if (adj) break;  // the adjoint's superposition runs after the transfer box is known
        unsigned long long* dFixed = static_cast<unsigned long long*>(bevFixed.ptr);
        if (columnLists) {
            // One column per layer of the chunk: the whole one-layer list superposed at
            // once, layer q into BEV volume q, transferred into dose buffer q; the sink
            // compacts the columns, then the volumes' live cells are cleared.
            float* cBev = static_cast<float*>(colBev.ptr);
            unsigned long long* cFixed = static_cast<unsigned long long*>(colFixed.ptr);
            PBS_CUDA(launch_superpose_columns(g, static_cast<const float*>(iddBuf.ptr),
                                              static_cast<const float*>(rsBuf.ptr), static_cast<const int4*>(work.ptr),
                                              dbs, dls + l0, nl, cBev, cFixed, colCells, smCount, stream),
                     "superpose_columns");
            PBS_CUDA(launch_column_transfer(g, cBev, colCells, dbs, dls + l0, nl, colBox,
                                            static_cast<double*>(colDose.ptr), stream),
                     "column_transfer");
            if ((rc = cols->columns(l0, nl))) return rc;
            PBS_CUDA(launch_column_bev_clear(g, cBev, colCells, dls + l0, nl, stream), "column_bev_clear");
            continue;
        }
        bevFixedClean = false;
        PBS_CUDA(launch_superpose(g, static_cast<const float*>(iddBuf.ptr), static_cast<const float*>(rsBuf.ptr),
                                  static_cast<const int4*>(work.ptr), dbs, dBev, dFixed, 0, smCount, stream),
                 "superpose");
        if (nuclear)
            PBS_CUDA(launch_superpose(nucGeom, dNucIdd, dNucRs, static_cast<const int4*>(nucWork.ptr), dNucBs,
                                      static_cast<float*>(nucBev.ptr), dFixed, 0, smCount, stream),
                     "nuc_superpose");
        if (bio) {
            // Every biological channel: the IDD scaled by the channel's factor,
            // superposed with the same radii and work list into its own BEV volume.
            const size_t bevN = S * size_t(g.bevX) * g.bevY;
            const int channels[3] = {0, 1, 2};
            int slot = 0;
            for (int c : channels) {
                if (c == 1 && bioModel != PBS_BIO_LQ) continue;
                PBS_CUDA(launch_bio_channel(g, bioDev, l0, nl, static_cast<const float*>(iddBuf.ptr), dWepl, dls, dbs,
                                            static_cast<const float*>(bioLayerRow.ptr), c,
                                            static_cast<float*>(bioIdd.ptr), stream),
                         "bio_channel");
                PBS_CUDA(launch_reset_work_claims(dbs, stream), "reset work claims");
                PBS_CUDA(launch_superpose(g, static_cast<const float*>(bioIdd.ptr),
                                          static_cast<const float*>(rsBuf.ptr), static_cast<const int4*>(work.ptr),
                                          dbs, static_cast<float*>(bioBev.ptr) + size_t(slot) * bevN, dFixed,
                                          bioShiftOffset[c], smCount, stream),
                         "bio_superpose");
                ++slot;
            }
        }
        bevFixedClean = true;
        if (perLayerTransfer) {
            // This layer alone, then empty BEV volumes for the next one (the last
            // layer's BEV stays for the debug readouts).
            if ((rc = transfer_layers(dls + l0, nuclear ? dNucLs + l0 : nullptr))) return rc;
            if (cols && (rc = cols->columns(l0, 1))) return rc;
        }
        if (perLayerTransfer && l0 + nl < L) {
            PBS_CUDA(cudaMemsetAsync(dBev, 0, S * size_t(g.bevX) * g.bevY * 4, stream), "memset BEV");
            if (nuclear)
                PBS_CUDA(cudaMemsetAsync(nucBev.ptr, 0, S * size_t(nucGeom.bevX) * nucGeom.bevY * 4, stream),
                         "memset BEV");
            if (bio)
                PBS_CUDA(cudaMemsetAsync(bioBev.ptr, 0,
                                         size_t(bioModel == PBS_BIO_LQ ? 3 : 2) * S * size_t(g.bevX) * g.bevY * 4,
                                         stream),
                         "memset BEV");
        }
    }
    if ((rc = mark(6))) return rc;
    if (adj) return finish_adjoint(*adj, b);
    if (columnLists) colClean = true;
    if (!perLayerTransfer && !cols && (rc = transfer_layers(nullptr, nullptr))) return rc;
    if ((rc = mark(7))) return rc;
    lastChunks = (L + chunk - 1) / chunk;
    // trace, planner, two fluence kernels, seven per chunk (IDD, layer plan, work
    // list, three superposition ranges, fixed-point write-out), and per transfer (one,
    // or one per layer in the per-layer mode) the transfer planner and transfer; the
    // halo adds eight per chunk (clear, codes, layer plan, work list, three
    // superposition ranges, write-out) and its own transfer planner and transfer.
    const int transfers = perLayerTransfer ? lastChunks : 1;
    lastLaunches = 4 + 7 * lastChunks + 2 * transfers + (nuclear ? 8 * lastChunks + 2 * transfers : 0);
    // The biological channels: per chunk and channel, the scaling, a claim reset,
    // three superposition ranges and the write-out; per transfer one transfer per
    // accumulator.
    if (bio) {
        const int nCh = bioModel == PBS_BIO_LQ ? 3 : 2;
        lastLaunches += nCh * 6 * lastChunks + (nCh + 1) * transfers;
    }
    lastBeamValid = true;
    lastStageTimed = stageTiming != 0;
    return PBS_OK;
}

// Dose gradient -> spot-weight gradient for the beam whose IDD, binning and work
// list run_beam just enqueued: T^T, S^T with the IDD scaling, the transposed
// convolution, then the lattice-cell shares of every spot on the host.
int Context::finish_adjoint(const AdjointArgs& a, const PbsBeamDesc& b) {
    const BeamGeomDev& g = geom;
    BeamStateDev* dbs = static_cast<BeamStateDev*>(bs.ptr);
    const size_t S = size_t(g.steps), rays = size_t(g.rayX) * g.rayY, L = size_t(g.numLayers);
    const size_t bevN = S * g.bevX * g.bevY, latN = L * g.latNy * g.latNx;
    int rc;
    if ((rc = bevGrad.ensure(bevN * 4)) || (rc = rbarBuf.ensure(L * rays * 4)) ||
        (rc = gradInterm.ensure(L * g.latNy * g.rayX * 4)) || (rc = gradLattice.ensure(latN * 4)))
        return rc;
    PBS_CUDA(launch_transfer_planner(g, dbs, nullptr, 0, stream), "transfer_planner");
    PBS_CUDA(cudaMemsetAsync(bevGrad.ptr, 0, bevN * 4, stream), "memset");
    PBS_CUDA(cudaMemsetAsync(rbarBuf.ptr, 0, L * rays * 4, stream), "memset");
    PBS_CUDA(launch_transfer_adjoint(g, a.gradDose, dbs, static_cast<float*>(bevGrad.ptr), stream), "transfer_adjoint");
    PBS_CUDA(launch_superpose_adjoint(g, static_cast<const float*>(iddBuf.ptr), static_cast<const float*>(rsBuf.ptr),
                                      static_cast<const int4*>(work.ptr), dbs, static_cast<const float*>(bevGrad.ptr),
                                      static_cast<float*>(rbarBuf.ptr), smCount, stream),
             "superpose_adjoint");
    PBS_CUDA(launch_conv_lattice_adjoint(g, static_cast<const float*>(rbarBuf.ptr), static_cast<const float*>(rayW.ptr),
                                         static_cast<float*>(gradInterm.ptr), static_cast<float*>(gradLattice.ptr),
                                         static_cast<const LayerStateDev*>(ls.ptr), dbs, stream),
             "conv_adjoint");
    std::vector<float> hLat(latN);
    PBS_CUDA(cudaMemcpyAsync(hLat.data(), gradLattice.ptr, latN * 4, cudaMemcpyDeviceToHost, stream), "grad D2H");
    PBS_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    std::vector<int> cells;
    std::vector<float> shares;
    if (!lattice_spot_cells(b, plan.lattice, cells, shares)) {
        set_error("adjoint: could not map the spots onto the lattice");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    for (size_t s = 0; s < a.nSpots; ++s) {
        double v = 0.0;
        for (int k = 0; k < 4; ++k) {
            const int c = cells[s * 4 + k];
            if (c >= 0) v += double(shares[s * 4 + k]) * double(hLat[size_t(c)]);
        }
        a.gradSpots[s] = float(v);
    }
    lastLaunches = 0;
    lastBeamValid = true;
    return take_device_errors();
}

int Context::beam_stats(PbsBeamStats* out) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!lastBeamValid) {
        set_error("no beam has been added");
        return PBS_ERR_NOT_READY;
    }
    BeamStateDev h;
    PBS_CUDA(cudaMemcpyAsync(&h, bs.ptr, sizeof(h), cudaMemcpyDeviceToHost, stream), "stats D2H");
    PBS_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    const BeamPlan& P = plan;
    std::memset(out, 0, sizeof(*out));
    out->num_layers = P.numLayers;
    out->conv_mode = P.convMode;
    out->ray_dims[0] = P.rayDims[0];
    out->ray_dims[1] = P.rayDims[1];
    out->superp_dims[0] = P.superpDims[0];
    out->superp_dims[1] = P.superpDims[1];
    out->tracer_steps = P.tracerSteps;
    out->lattice_dims[0] = P.lattice.nx;
    out->lattice_dims[1] = P.lattice.ny;
    out->lattice_delta[0] = P.lattice.dx;
    out->lattice_delta[1] = P.lattice.dy;
    out->lattice_offset[0] = P.lattice.ox;
    out->lattice_offset[1] = P.lattice.oy;
    out->cpb_corner[0] = P.cpbCorner.x;
    out->cpb_corner[1] = P.cpbCorner.y;
    out->cpb_resolution[0] = P.cpbRes.x;
    out->cpb_resolution[1] = P.cpbRes.y;
    out->fan_corner[0] = P.fanCorner.x;
    out->fan_corner[1] = P.fanCorner.y;
    out->fan_corner[2] = P.fanCorner.z;
    out->fan_delta[0] = P.fanDelta.x;
    out->fan_delta[1] = P.fanDelta.y;
    out->fan_delta[2] = P.fanDelta.z;
    out->source_dist[0] = P.sourceDist.x;
    out->source_dist[1] = P.sourceDist.y;
    out->len_to_mm = P.lenToMm;
    out->energy_depth_to_mm = P.energyDepthToMm;
    out->max_peak_depth_mm = P.maxPeakDepthMm;
    out->first_inside = h.firstInside;
    out->first_outside = h.firstOutside;
    out->guaranteed_passive = h.guaranteedPassive;
    for (int i = 0; i < 3; ++i) {
        out->transfer_start[i] = h.transferStart[i];
        out->transfer_max[i] = h.transferMax[i];
    }
    out->live_tiles = h.liveTiles;
    out->superpose_fma = h.superposeFma;
    out->kernel_launches = lastLaunches;
    out->layer_chunks = lastChunks;
    int flags = h.errorFlags;
    if (lastNuclear) {
        BeamStateDev hn;
        PBS_CUDA(cudaMemcpy(&hn, nucBs.ptr, sizeof(hn), cudaMemcpyDeviceToHost), "stats D2H");
        out->nuc_dims[0] = geom.nucX;
        out->nuc_dims[1] = geom.nucY;
        out->nuc_live_tiles = hn.liveTiles;
        out->nuc_superpose_fma = hn.superposeFma;
        flags |= hn.errorFlags;
    }
    if (flags & 4) {
        set_error("Nuclear superposition kernel radius exceeded kMaxSuperpR=32");
        return PBS_ERR_UNSUPPORTED;
    }
    if (flags) {
        set_error("device reported an internal error flag " + std::to_string(flags));
        return PBS_ERR_CUDA;
    }
    return PBS_OK;
}

int Context::layer_stats(int layer, PbsLayerStats* out) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!lastBeamValid || layer < 0 || layer >= plan.numLayers) {
        set_error("layer out of range or no beam");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    LayerStateDev h;
    PBS_CUDA(cudaMemcpyAsync(&h, static_cast<LayerStateDev*>(ls.ptr) + layer, sizeof(h), cudaMemcpyDeviceToHost, stream),
             "stats D2H");
    PBS_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    const LayerHost& H = plan.layers[layer];
    std::memset(out, 0, sizeof(*out));
    out->energy_idx = H.energyIdx;
    out->energy_scale_fact = H.energyScaleFact;
    out->peak_depth = H.peakDepth;
    out->entry_sigma[0] = h.entrySigmaX;
    out->entry_sigma[1] = h.entrySigmaY;
    out->after_last_step = h.afterLast;
    out->max_first_passive = h.maxFirstPassive;
    out->calc_passive = h.calcPassive;
    for (int i = 0; i < kBuckets; ++i) out->tile_rad_counts[i] = h.hist[i];
    for (int i = 0; i <= kMaxR; ++i) out->batched_counts[i] = h.batchedCounts[i];
    out->live_tiles = h.liveTiles;
    out->spot_dist = layer < int(layerSpotDist.size()) ? layerSpotDist[layer] : 0.0f;
    if (lastNuclear) {
        LayerStateDev hn;
        PBS_CUDA(cudaMemcpy(&hn, static_cast<LayerStateDev*>(nucLs.ptr) + layer, sizeof(hn), cudaMemcpyDeviceToHost),
                 "stats D2H");
        for (int i = 0; i < kBuckets; ++i) out->nuc_tile_rad_counts[i] = hn.hist[i];
        for (int i = 0; i <= kMaxR; ++i) out->nuc_batched_counts[i] = hn.batchedCounts[i];
    }
    return PBS_OK;
}

int Context::stage_times(float* ms, int n) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!lastStageTimed) {
        set_error("stage timing was not enabled for the last beam");
        return PBS_ERR_NOT_READY;
    }
    PBS_CUDA(cudaEventSynchronize(ev[7]), "cudaEventSynchronize");
    // Slots: 0 trace+wepl_min, 1 planner, 2 conv, 3 idd (first chunk), 4 bin (first chunk),
    // 5 superposition (+ later chunks), 6 transfer.
    const int map[PBS_STAGE_COUNT][2] = {{0, 1}, {1, 2}, {2, 3}, {3, 4}, {4, 5}, {5, 6}, {6, 7}};
    for (int i = 0; i < n && i < PBS_STAGE_COUNT; ++i) {
        float t = 0.f;
        PBS_CUDA(cudaEventElapsedTime(&t, ev[map[i][0]], ev[map[i][1]]), "cudaEventElapsedTime");
        ms[i] = t;
    }
    return PBS_OK;
}

int Context::debug_copy(int which, int layer, void* out, size_t bytes) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!lastBeamValid) {
        set_error("no beam has been added");
        return PBS_ERR_NOT_READY;
    }
    PBS_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    const size_t S = size_t(geom.steps), rays = size_t(geom.rayX) * geom.rayY;
    const size_t padPlane = size_t(geom.pitchX) * geom.pitchY;
    const size_t tiles = size_t(geom.tilesX) * geom.tilesY;
    auto copy = [&](const void* src, size_t n) -> int {
        if (bytes != n) {
            set_error("debug_copy: expected " + std::to_string(n) + " bytes, got " + std::to_string(bytes));
            return PBS_ERR_INVALID_ARGUMENT;
        }
        PBS_CUDA(cudaMemcpy(out, src, n, cudaMemcpyDeviceToHost), "debug D2H");
        return PBS_OK;
    };
    const bool perLayer = which == PBS_DBG_IDD || which == PBS_DBG_RSIGMA || which == PBS_DBG_TILE_BINS ||
                          which == PBS_DBG_FIRST_PASSIVE || which == PBS_DBG_NUC_IDD || which == PBS_DBG_NUC_RSIGMA ||
                          which == PBS_DBG_NUC_TILE_BINS;
    const bool nucBuf = which >= PBS_DBG_NUC_IDD && which <= PBS_DBG_RAY_TO_NUC;
    if (nucBuf && !lastNuclear) {
        set_error("the last beam has no nuclear halo");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    if (perLayer) {
        if (!keepDebug || layer < 0 || layer >= plan.numLayers || layer >= chunkLayers) {
            set_error("per-layer debug buffers need PBS_OPT_KEEP_DEBUG and a valid layer");
            return PBS_ERR_INVALID_ARGUMENT;
        }
    }
    BeamStateDev h;
    PBS_CUDA(cudaMemcpy(&h, bs.ptr, sizeof(h), cudaMemcpyDeviceToHost), "debug D2H");
    const int first = h.firstInside;
    switch (which) {
        case PBS_DBG_DENSITY: return copy(trace.dens, S * rays * 4);
        case PBS_DBG_WEPL: return copy(trace.wepl, S * rays * 4);
        case PBS_DBG_FIRST_INSIDE: return copy(trace.firstIn, rays * 4);
        case PBS_DBG_FIRST_OUTSIDE: return copy(trace.firstOut, rays * 4);
        case PBS_DBG_WEPL_MIN: return copy(trace.weplMin, S * 4);
        case PBS_DBG_RAY_WEIGHTS: return copy(rayW.ptr, size_t(plan.numLayers) * rays * 4);
        case PBS_DBG_FIRST_PASSIVE: return copy(static_cast<char*>(firstPassive.ptr) + size_t(layer) * rays * 4, rays * 4);
        case PBS_DBG_DOSE64: {
            const size_t n = size_t(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2];
            int frc = flush_dose_init();
            if (frc) return frc;
            PBS_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
            return copy(dose64.ptr, n * 8);
        }
        case PBS_DBG_BEV_DOSE: {
            // Layer-summed BEV at absolute step index: planes before `first` are zero.
            const size_t plane = size_t(geom.bevX) * geom.bevY;
            if (bytes != S * plane * 4) {
                set_error("debug_copy: BEV size mismatch");
                return PBS_ERR_INVALID_ARGUMENT;
            }
            std::memset(out, 0, bytes);
            const size_t nz = S - size_t(std::max(first, 0));
            PBS_CUDA(cudaMemcpy(static_cast<char*>(out) + size_t(first) * plane * 4, bev.ptr, nz * plane * 4,
                                cudaMemcpyDeviceToHost),
                     "debug D2H");
            return PBS_OK;
        }
        case PBS_DBG_IDD:
        case PBS_DBG_RSIGMA: {
            if (bytes != S * padPlane * 4) {
                set_error("debug_copy: IDD size mismatch");
                return PBS_ERR_INVALID_ARGUMENT;
            }
            LayerStateDev lh;
            PBS_CUDA(cudaMemcpy(&lh, static_cast<LayerStateDev*>(ls.ptr) + layer, sizeof(lh), cudaMemcpyDeviceToHost),
                     "debug D2H");
            float* o = static_cast<float*>(out);
            const float fill = which == PBS_DBG_IDD ? 0.0f : __builtin_inff();
            std::fill(o, o + S * padPlane, fill);
            const int nz = std::max(0, lh.afterLast - first);
            const char* src = static_cast<const char*>(which == PBS_DBG_IDD ? iddBuf.ptr : rsBuf.ptr) +
                              size_t(layer) * S * padPlane * 4;
            if (nz > 0)
                PBS_CUDA(cudaMemcpy(o + size_t(first) * padPlane, src, size_t(nz) * padPlane * 4, cudaMemcpyDeviceToHost),
                         "debug D2H");
            return PBS_OK;
        }
        case PBS_DBG_TILE_BINS: {
            if (bytes != S * tiles) {
                set_error("debug_copy: tile bins size mismatch");
                return PBS_ERR_INVALID_ARGUMENT;
            }
            LayerStateDev lh;
            PBS_CUDA(cudaMemcpy(&lh, static_cast<LayerStateDev*>(ls.ptr) + layer, sizeof(lh), cudaMemcpyDeviceToHost),
                     "debug D2H");
            uint8_t* o = static_cast<uint8_t*>(out);
            std::memset(o, 0xff, bytes);
            const int nz = std::max(0, lh.afterLast - first);
            if (nz > 0)
                PBS_CUDA(cudaMemcpy(o + size_t(first) * tiles, static_cast<const char*>(codes.ptr) + size_t(layer) * S * tiles,
                                    size_t(nz) * tiles, cudaMemcpyDeviceToHost),
                         "debug D2H");
            return PBS_OK;
        }
        case PBS_DBG_RAY_TO_NUC: return copy(rayToNuc.ptr, rays * 4);
        case PBS_DBG_NUC_BEV_DOSE: {
            const size_t plane = size_t(nucGeom.bevX) * nucGeom.bevY;
            if (bytes != S * plane * 4) {
                set_error("debug_copy: halo BEV size mismatch");
                return PBS_ERR_INVALID_ARGUMENT;
            }
            std::memset(out, 0, bytes);
            const size_t nz = S - size_t(std::max(first, 0));
            PBS_CUDA(cudaMemcpy(static_cast<char*>(out) + size_t(first) * plane * 4, nucBev.ptr, nz * plane * 4,
                                cudaMemcpyDeviceToHost),
                     "debug D2H");
            return PBS_OK;
        }
        case PBS_DBG_NUC_IDD:
        case PBS_DBG_NUC_RSIGMA:
        case PBS_DBG_NUC_TILE_BINS: {
            const size_t nucPlane = size_t(geom.nucX) * geom.nucY;
            const size_t nucTiles = nucPlane / (kTileX * kTileY);
            const bool bins = which == PBS_DBG_NUC_TILE_BINS;
            const size_t elem = bins ? 1 : 4, per = bins ? nucTiles : nucPlane;
            if (bytes != S * per * elem) {
                set_error("debug_copy: halo buffer size mismatch");
                return PBS_ERR_INVALID_ARGUMENT;
            }
            LayerStateDev lh;
            PBS_CUDA(cudaMemcpy(&lh, static_cast<LayerStateDev*>(ls.ptr) + layer, sizeof(lh), cudaMemcpyDeviceToHost),
                     "debug D2H");
            if (bins) {
                std::memset(out, 0xff, bytes);
            } else {
                float* o = static_cast<float*>(out);
                std::fill(o, o + S * per, which == PBS_DBG_NUC_IDD ? 0.0f : __builtin_inff());
            }
            // The halo is computed over [first, afterLast); its codes over [first, calcPassive).
            const int nz = std::max(0, (bins ? lh.calcPassive : lh.afterLast) - first);
            const void* srcBase = bins ? nucCodes.ptr : (which == PBS_DBG_NUC_IDD ? nucIddBuf.ptr : nucRsBuf.ptr);
            const char* src = static_cast<const char*>(srcBase) + size_t(layer) * S * per * elem;
            if (nz > 0)
                PBS_CUDA(cudaMemcpy(static_cast<char*>(out) + size_t(first) * per * elem, src, size_t(nz) * per * elem,
                                    cudaMemcpyDeviceToHost),
                         "debug D2H");
            return PBS_OK;
        }
        default:
            set_error("unknown debug buffer");
            return PBS_ERR_INVALID_ARGUMENT;
    }
}

// ---- one-shot wrapper -----------------------------------------------------------

namespace {
std::mutex g_cacheMutex;
std::map<int, Context*> g_cache;

// CT voxels the tracer of a beam can read: the sample points are multilinear in
// (ray x, ray y, step), so the corner rays at the first and last step bound them;
// two voxels of margin cover the trilinear footprint and the rounding of the
// repeated step additions (trace_kernel).
void ct_trace_box(const BeamPlan& P, const int dims[3], int lo[3], int hi[3]) {
    float mn[3] = {1e30f, 1e30f, 1e30f}, mx[3] = {-1e30f, -1e30f, -1e30f};
    const int xs[2] = {0, P.rayDims[0] - 1}, ys[2] = {0, P.rayDims[1] - 1};
    const float ks[2] = {0.0f, float(P.tracerSteps - 1)};
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b) {
            const V3 st = tracer_start(P.tracer, xs[a], ys[b]);
            const V3 inc = tracer_inc(P.tracer, xs[a], ys[b]);
            for (int c = 0; c < 2; ++c) {
                const float q[3] = {st.x + 0.5f + ks[c] * inc.x, st.y + 0.5f + ks[c] * inc.y,
                                    st.z + 0.5f + ks[c] * inc.z};
                for (int i = 0; i < 3; ++i) {
                    mn[i] = std::min(mn[i], q[i]);
                    mx[i] = std::max(mx[i], q[i]);
                }
            }
        }
    for (int i = 0; i < 3; ++i) {
        lo[i] = std::max(int(std::floor(std::max(mn[i], -1e9f))) - 2, 0);
        hi[i] = std::min(int(std::floor(std::min(mx[i], 1e9f))) + 2, dims[i] - 1);
    }
}

}  // namespace

namespace {
// Host<->device bytes of the calling thread's last completed wrapper call.
thread_local unsigned long long g_lastWrapperCopies[2] = {0, 0};
int wrapper_body(Context* ctx, const float* ctData, const GridDesc& cg, float* doseData, const GridDesc& dg,
                 const PbsBeamDesc* beams, size_t numBeams, const PbsEnergyDesc* energyData, int nuclear,
                 int verbose);
}  // namespace

int subsecond_wrapper(const float* ctData, const int ctDims[3], const float ctRes[3], const float ctCorner[3],
                      float* doseData, const int doseDims[3], const float doseRes[3], const float doseCorner[3],
                      const PbsBeamDesc* beams, size_t numBeams, const PbsEnergyDesc* energyData, int gpuId,
                      int nuclear, int verbose) {
    GridDesc cg, dg;
    for (int i = 0; i < 3; ++i) {
        cg.dims[i] = ctDims ? ctDims[i] : 0;
        cg.res[i] = ctRes ? ctRes[i] : 0.f;
        cg.corner[i] = ctCorner ? ctCorner[i] : 0.f;
        dg.dims[i] = doseDims ? doseDims[i] : 0;
        dg.res[i] = doseRes ? doseRes[i] : 0.f;
        dg.corner[i] = doseCorner ? doseCorner[i] : 0.f;
    }
    std::string err;
    if (!validate_global(ctData, cg, doseData, dg, beams, numBeams, energyData, err)) {
        set_error(err);
        return PBS_ERR_INVALID_ARGUMENT;
    }
    for (size_t i = 0; i < numBeams; ++i) {
        if (!validate_beam(beams[i], i, err)) {
            set_error(err);
            return PBS_ERR_INVALID_ARGUMENT;
        }
    }
    std::lock_guard<std::mutex> lock(g_cacheMutex);
    Context*& ctx = g_cache[gpuId];
    if (!ctx) {
        Context* c = new Context();
        int rc = c->init(gpuId);
        if (rc) {
            delete c;
            return rc;
        }
        ctx = c;
    }
    ctx->copiedH2D = ctx->copiedD2H = 0;
    int rc = wrapper_body(ctx, ctData, cg, doseData, dg, beams, numBeams, energyData, nuclear, verbose);
    g_lastWrapperCopies[0] = ctx->copiedH2D;
    g_lastWrapperCopies[1] = ctx->copiedD2H;
    return rc;
}

int wrapper_copy_bytes(unsigned long long out[2]) {
    out[0] = g_lastWrapperCopies[0];
    out[1] = g_lastWrapperCopies[1];
    return PBS_OK;
}

namespace {

int wrapper_body(Context* ctx, const float* ctData, const GridDesc& cg, float* doseData, const GridDesc& dg,
                 const PbsBeamDesc* beams, size_t numBeams, const PbsEnergyDesc* energyData, int nuclear,
                 int verbose) {
    int rc;
    if ((rc = ctx->set_energy(*energyData))) return rc;
    // Every beam is planned up front, and the plan is handed to add_planned_beam: the CT
    // voxels their tracers can sample and the dose voxels their transfers can write
    // bound the host copies of this call.
    int ctLo[3] = {INT_MAX, INT_MAX, INT_MAX}, ctHi[3] = {-1, -1, -1};
    int dLo[3] = {INT_MAX, INT_MAX, INT_MAX}, dHi[3] = {-1, -1, -1};
    std::vector<BeamPlan> plans(numBeams);
    for (size_t i = 0; i < numBeams; ++i) {
        BeamPlan& P = plans[i];
        std::string perr;
        if ((rc = plan_beam(beams[i], ctx->energy, cg, dg, P, perr))) {
            set_error(perr);
            return rc;
        }
        int lo[3], hi[3];
        ct_trace_box(P, cg.dims, lo, hi);
        merge_box(ctLo, ctHi, lo, hi);
        dose_transfer_box(P.rayIdxToDoseIdx, P.superpDims[0], P.superpDims[1], P.tracerSteps, dg.dims, lo, hi);
        merge_box(dLo, dHi, lo, hi);
        if (nuclear && P.hasLattice) {
            FromFan nf = P.rayIdxToDoseIdx;
            nf.fanIdxToFan = idxxf(v3(P.lattice.dx, P.lattice.dy, P.fanDelta.z),
                                   v3(P.lattice.ox, P.lattice.oy, P.fanCorner.z));
            const int nx = (P.lattice.nx + kTileX - 1) / kTileX * kTileX;
            const int ny = (P.lattice.ny + kTileY - 1) / kTileY * kTileY;
            dose_transfer_box(nf, nx, ny, P.tracerSteps, dg.dims, lo, hi);
            merge_box(dLo, dHi, lo, hi);
        }
    }
    if ((rc = ctx->set_ct_region(ctData, cg, ctLo, ctHi))) return rc;
    if ((rc = ctx->set_dose_grid(dg))) return rc;
    if ((rc = ctx->reset_dose_region(doseData, dLo, dHi))) return rc;
    for (size_t i = 0; i < numBeams; ++i) {
        // The plan made above used the same tables and grids as the context now holds.
        if ((rc = ctx->add_planned_beam(beams[i], nuclear, std::move(plans[i])))) return rc;
        if (verbose > 0) {
            PbsBeamStats st;
            if (ctx->beam_stats(&st) == PBS_OK)
                std::fprintf(stderr,
                             "[pbs] beam %zu: rays %dx%d steps %d layers %d first %d passive %d live tiles %lld\n", i,
                             st.ray_dims[0], st.ray_dims[1], st.tracer_steps, st.num_layers, st.first_inside,
                             st.guaranteed_passive, st.live_tiles);
        }
    }
    return ctx->read_dose_region(doseData, dLo, dHi);
}

}  // namespace

// ---- biological maps -----------------------------------------------------

int Context::clear_bio() {
    if (!hasDose) return PBS_OK;
    const size_t n = size_t(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2];
    if (int rc = bioAcc.ensure(4 * n * sizeof(double))) return rc;
    PBS_CUDA(cudaMemsetAsync(bioAcc.ptr, 0, 4 * n * sizeof(double), stream), "memset bio accumulators");
    return PBS_OK;
}

int Context::set_bio_model(const PbsBioModel* m) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!m || m->model == PBS_BIO_OFF) {
        bioModel = 0;
        return PBS_OK;
    }
    const bool lq = m->model == PBS_BIO_LQ, mkm = m->model == PBS_BIO_MKM;
    if (!lq && !mkm) {
        set_error("biological maps: unknown model");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    if (!m->let_table || !m->let_energies || m->let_rows <= 0 || m->let_depths <= 0 || !(m->let_depth_step > 0.0f) ||
        m->let_samples <= 0 || m->n_lq <= 0 || !(m->lq_log_step > 0.0f) ||
        (lq && (!m->lq_alpha || !m->lq_beta)) || (mkm && (!m->z1d || !(m->beta0 > 0.0f)))) {
        set_error("biological maps: missing or empty table, or a non-positive axis step");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    for (int r = 1; r < m->let_rows; ++r)
        if (!(m->let_energies[r] > m->let_energies[r - 1])) {
            set_error("biological maps: let_energies must ascend");
            return PBS_ERR_INVALID_ARGUMENT;
        }
    const size_t nLet = size_t(m->let_rows) * m->let_depths, nLq = size_t(m->n_lq);
    auto finite = [](const float* p, size_t n) {
        for (size_t i = 0; i < n; ++i)
            if (!std::isfinite(p[i])) return false;
        return true;
    };
    if (!finite(m->let_table, nLet) || (lq && (!finite(m->lq_alpha, nLq) || !finite(m->lq_beta, nLq))) ||
        (mkm && !finite(m->z1d, nLq))) {
        set_error("biological maps: a table holds a NaN or an infinity");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    std::vector<float> host(nLet + 2 * nLq);
    std::memcpy(host.data(), m->let_table, nLet * 4);
    if (lq) {
        std::memcpy(host.data() + nLet, m->lq_alpha, nLq * 4);
        std::memcpy(host.data() + nLet + nLq, m->lq_beta, nLq * 4);
    } else {
        std::memcpy(host.data() + nLet, m->z1d, nLq * 4);
    }
    if (int rc = bioTables.ensure(host.size() * 4)) return rc;
    if (int rc = upload(bioTables.ptr, host.data(), host.size() * 4)) return rc;
    const float* t = static_cast<const float*>(bioTables.ptr);
    BioDev& d = bioDev;
    d = BioDev{};
    d.model = m->model;
    d.letTable = t;
    d.letRows = m->let_rows;
    d.letDepths = m->let_depths;
    d.letDepth0 = m->let_depth0;
    d.letDepthStep = m->let_depth_step;
    d.letSamples = m->let_samples;
    d.estDimension = m->est_dimension;
    d.rangeShifter = m->range_shifter;
    d.alpha = lq ? t + nLet : nullptr;
    d.beta = lq ? t + nLet + nLq : nullptr;
    d.z1d = mkm ? t + nLet : nullptr;
    d.nLq = m->n_lq;
    d.lqLog0 = m->lq_log0;
    d.lqLogStep = m->lq_log_step;
    d.alpha0 = m->alpha0;
    d.beta0 = m->beta0;
    // A channel scales the IDD by at most its table's largest factor f < 2^e: its
    // fixed-point superposition runs e bits lower than the dose's.
    auto largest = [](const float* p, size_t n) {
        float v = 0.0f;
        for (size_t i = 0; i < n; ++i) v = std::max(v, p[i]);
        return v;
    };
    auto bits = [](float f) {
        int e = 0;
        std::frexp(f, &e);
        return f > 0.0f ? -std::max(e, 0) : 0;
    };
    const float* lqHost = host.data() + nLet;
    bioShiftOffset[0] = bits(largest(lqHost, nLq));
    bioShiftOffset[1] = lq ? bits(std::sqrt(largest(lqHost + nLq, nLq))) : 0;
    bioShiftOffset[2] = bits(largest(host.data(), nLet));
    bioLetEnergies.assign(m->let_energies, m->let_energies + m->let_rows);
    bioModel = m->model;
    return clear_bio();
}

int Context::read_bio_map(int map, float* out, int onDevice) {
    PBS_CUDA(cudaSetDevice(device), "cudaSetDevice");
    if (!bioModel) {
        set_error("biological maps: no model set");
        return PBS_ERR_NOT_READY;
    }
    if (!hasDose) {
        set_error("dose grid not set");
        return PBS_ERR_NOT_READY;
    }
    if (map < PBS_BIO_MAP_DOSE || map > PBS_BIO_MAP_Z1D ||
        ((map == PBS_BIO_MAP_ALPHA || map == PBS_BIO_MAP_BETA) && bioModel != PBS_BIO_LQ) ||
        (map == PBS_BIO_MAP_Z1D && bioModel != PBS_BIO_MKM)) {
        set_error("biological maps: unknown map, or a map of the other model");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    if (int rc = join_side_work()) return rc;
    const size_t n = size_t(doseGrid.dims[0]) * doseGrid.dims[1] * doseGrid.dims[2];
    if (int rc = floatOut.ensure(n * 4)) return rc;
    const double* acc = static_cast<const double*>(bioAcc.ptr);
    float* dst = onDevice ? out : static_cast<float*>(floatOut.ptr);
    PBS_CUDA(launch_bio_map(acc, acc + n, acc + 2 * n, acc + 3 * n, n, bioDev, map, dst, stream), "bio_map");
    if (onDevice) return PBS_OK;
    PBS_CUDA(cudaMemcpyAsync(out, floatOut.ptr, n * 4, cudaMemcpyDeviceToHost, stream), "bio map D2H");
    copiedD2H += n * 4;
    PBS_CUDA(cudaStreamSynchronize(stream), "cudaStreamSynchronize");
    return take_device_errors();
}

}  // namespace pbs
