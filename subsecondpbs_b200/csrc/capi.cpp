// extern "C" entry points: the plain C ABI of include/subsecondpbs.h and the C++
// drop-in face of include/raytracedicom_integration.h.
#include <cuda_runtime.h>

#include <cstdio>
#include <algorithm>
#include <stdexcept>
#include <string>

#include "../../include/raytracedicom_integration.h"
#include "../../include/subsecondpbs.h"
#include "context.h"

using pbs::Context;

struct PbsContext {
    Context impl;
};

namespace {

int guard(PbsContext* c) {
    if (!c) {
        pbs::set_error("null context");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    return PBS_OK;
}

pbs::GridDesc grid(const int d[3], const float r[3], const float c[3]) {
    pbs::GridDesc g;
    for (int i = 0; i < 3; ++i) {
        g.dims[i] = d ? d[i] : 0;
        g.res[i] = r ? r[i] : 0.f;
        g.corner[i] = c ? c[i] : 0.f;
    }
    return g;
}

}  // namespace

extern "C" {

const char* pbs_version(void) { return "subsecondpbs_b200 0.1.0 (sm_100a)"; }

const char* pbs_last_error(void) { return pbs::last_error(); }

int pbs_device_count(int* count) {
    if (!count) return PBS_ERR_INVALID_ARGUMENT;
    cudaError_t e = cudaGetDeviceCount(count);
    if (e != cudaSuccess) {
        *count = 0;
        pbs::set_error(std::string("cudaGetDeviceCount: ") + cudaGetErrorString(e));
        return PBS_ERR_CUDA;
    }
    return PBS_OK;
}

int pbs_subsecond_wrapper(const float* ct_data, const int ct_dims[3], const float ct_resolution[3],
                          const float ct_corner[3], float* dose_data, const int dose_dims[3],
                          const float dose_resolution[3], const float dose_corner[3], const PbsBeamDesc* beams,
                          size_t num_beams, const PbsEnergyDesc* energy, int gpu_id, int nuclear_correction,
                          int verbose) {
    return pbs::subsecond_wrapper(ct_data, ct_dims, ct_resolution, ct_corner, dose_data, dose_dims, dose_resolution,
                                  dose_corner, beams, num_beams, energy, gpu_id, nuclear_correction, verbose);
}

int pbs_wrapper_copy_bytes(unsigned long long out[2]) {
    if (!out) {
        pbs::set_error("null argument");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    return pbs::wrapper_copy_bytes(out);
}

int pbs_plan_beam(const PbsBeamDesc* beam, const PbsEnergyDesc* energy, const int ct_dims[3],
                  const float ct_resolution[3], const float ct_corner[3], const int dose_dims[3],
                  const float dose_resolution[3], const float dose_corner[3], PbsBeamStats* out, float* layer_params,
                  float* lattice, size_t lattice_len) {
    if (!beam || !energy || !out) {
        pbs::set_error("null argument");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    const pbs::GridDesc cg = grid(ct_dims, ct_resolution, ct_corner);
    const pbs::GridDesc dg = grid(dose_dims, dose_resolution, dose_corner);
    std::string err;
    float dummy = 0.f;
    if (!pbs::validate_global(&dummy, cg, &dummy, dg, beam, 1, energy, err) || !pbs::validate_beam(*beam, 0, err)) {
        pbs::set_error(err);
        return PBS_ERR_INVALID_ARGUMENT;
    }
    pbs::BeamPlan P;
    const int rc = pbs::plan_beam(*beam, *energy, cg, dg, P, err);
    if (rc) {
        pbs::set_error(err);
        return rc;
    }
    *out = PbsBeamStats{};
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
    if (layer_params) {
        for (int l = 0; l < P.numLayers; ++l) {
            const pbs::LayerHost& H = P.layers[l];
            float* o = layer_params + 8 * l;
            o[0] = H.energyIdx;
            o[1] = H.energyScaleFact;
            o[2] = H.peakDepth;
            o[3] = H.convPeakDepth;
            o[4] = H.sigmaSqAirQuad;
            o[5] = H.sigmaSqAirLin;
            o[6] = H.sigmaXmm;
            o[7] = H.sigmaYmm;
        }
    }
    if (lattice && P.hasLattice && lattice_len == P.lattice.weights.size())
        std::copy(P.lattice.weights.begin(), P.lattice.weights.end(), lattice);
    return PBS_OK;
}

int pbs_context_create(int gpu_id, PbsContext** out) {
    if (!out) return PBS_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    PbsContext* c = new PbsContext();
    int rc = c->impl.init(gpu_id);
    if (rc) {
        delete c;
        return rc;
    }
    *out = c;
    return PBS_OK;
}

int pbs_context_destroy(PbsContext* ctx) {
    delete ctx;
    return PBS_OK;
}

int pbs_context_set_option(PbsContext* ctx, int option, long long value) {
    if (int rc = guard(ctx)) return rc;
    switch (option) {
        case PBS_OPT_COMPAT_BEV_Z_SHIFT: ctx->impl.compatBevZShift = value != 0; return PBS_OK;
        case PBS_OPT_STAGE_TIMING: ctx->impl.stageTiming = value != 0; return PBS_OK;
        case PBS_OPT_LAYER_BUDGET_MIB: ctx->impl.layerBudgetMiB = value; return PBS_OK;
        case PBS_OPT_CT_INPUT_TYPE:
            if (value < PBS_CT_AUTO || value > PBS_CT_SPR) break;
            ctx->impl.ctInputType = int(value);
            return PBS_OK;
        case PBS_OPT_KEEP_DEBUG: ctx->impl.keepDebug = value != 0; return PBS_OK;
        case PBS_OPT_NUCLEAR_MODEL:
            if (value < 0 || value > 2) break;
            ctx->impl.nuclearModel = int(value);
            return PBS_OK;
        case PBS_OPT_CARBON_PROFILE:
            if (value < 0 || value > 3) break;
            ctx->impl.carbonProfile = int(value);
            return PBS_OK;
        default: break;
    }
    pbs::set_error("unknown option or value");
    return PBS_ERR_INVALID_ARGUMENT;
}

int pbs_context_set_energy(PbsContext* ctx, const PbsEnergyDesc* energy) {
    if (int rc = guard(ctx)) return rc;
    if (!energy) return PBS_ERR_INVALID_ARGUMENT;
    return ctx->impl.set_energy(*energy);
}

int pbs_context_set_ct(PbsContext* ctx, const float* ct, int ct_on_device, const int dims[3],
                       const float resolution[3], const float corner[3]) {
    if (int rc = guard(ctx)) return rc;
    return ctx->impl.set_ct(ct, ct_on_device, grid(dims, resolution, corner));
}

int pbs_context_set_dose_grid(PbsContext* ctx, const int dims[3], const float resolution[3], const float corner[3]) {
    if (int rc = guard(ctx)) return rc;
    return ctx->impl.set_dose_grid(grid(dims, resolution, corner));
}

int pbs_context_reset_dose(PbsContext* ctx, const float* initial, int initial_on_device) {
    if (int rc = guard(ctx)) return rc;
    return ctx->impl.reset_dose(initial, initial_on_device);
}

int pbs_context_add_beam(PbsContext* ctx, const PbsBeamDesc* beam, int nuclear_correction) {
    if (int rc = guard(ctx)) return rc;
    if (!beam) return PBS_ERR_INVALID_ARGUMENT;
    return ctx->impl.add_beam(*beam, nuclear_correction);
}

int pbs_context_adjoint_beam(PbsContext* ctx, const PbsBeamDesc* beam, const double* grad_dose, int grad_on_device,
                             float* grad_weights, size_t n_weights) {
    if (int rc = guard(ctx)) return rc;
    if (!beam) return PBS_ERR_INVALID_ARGUMENT;
    return ctx->impl.adjoint_beam(*beam, grad_dose, grad_on_device, grad_weights, n_weights);
}

int pbs_operator_batch_plan(const PbsBeamDesc* beam, int max_spots_per_batch, PbsOperatorLayerSpan* spans,
                            int span_capacity, PbsOperatorBatch* batches, int batch_capacity, int info[6]) {
    if (!beam || !info) {
        pbs::set_error("null beam or info");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    pbs::OperatorPlan plan;
    if (int rc = pbs::operator_batch_plan(*beam, max_spots_per_batch, plan)) return rc;
    const int nSpans = static_cast<int>(plan.spans.size()), nBatches = static_cast<int>(plan.batches.size());
    const int vals[6] = {plan.valid ? 1 : 0, plan.totalLayers, plan.totalSpots, plan.maxSpotsPerBatch, nSpans, nBatches};
    for (int i = 0; i < 6; ++i) info[i] = vals[i];
    if ((spans && span_capacity < nSpans) || (batches && batch_capacity < nBatches)) {
        pbs::set_error("operator batch plan: output capacity below " + std::to_string(nSpans) + " spans / " +
                       std::to_string(nBatches) + " batches");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    if (spans) std::copy(plan.spans.begin(), plan.spans.end(), spans);
    if (batches) std::copy(plan.batches.begin(), plan.batches.end(), batches);
    return PBS_OK;
}

int pbs_context_influence_csc(PbsContext* ctx, const PbsBeamDesc* beam, int nuclear_correction, long long spot_begin,
                              long long spot_count, double threshold, long long* col_ptr, int* rows, float* values,
                              long long capacity, long long* nnz) {
    if (int rc = guard(ctx)) return rc;
    if (!beam) return PBS_ERR_INVALID_ARGUMENT;
    return ctx->impl.influence_csc(*beam, nuclear_correction, spot_begin, spot_count, threshold, col_ptr, rows, values,
                                   capacity, nnz);
}

int pbs_context_influence_row_norms(PbsContext* ctx, const PbsBeamDesc* beam, int nuclear_correction,
                                    long long spot_begin, long long spot_count, const long long* voxels,
                                    long long n_voxels, float* out) {
    if (int rc = guard(ctx)) return rc;
    if (!beam) return PBS_ERR_INVALID_ARGUMENT;
    return ctx->impl.influence_row_norms(*beam, nuclear_correction, spot_begin, spot_count, voxels, n_voxels, out);
}

int pbs_context_set_bio_model(PbsContext* ctx, const PbsBioModel* model) {
    if (int rc = guard(ctx)) return rc;
    return ctx->impl.set_bio_model(model);
}

int pbs_context_read_bio_map(PbsContext* ctx, int map, float* out, int out_on_device) {
    if (int rc = guard(ctx)) return rc;
    if (!out) return PBS_ERR_INVALID_ARGUMENT;
    return ctx->impl.read_bio_map(map, out, out_on_device);
}

int pbs_context_read_dose(PbsContext* ctx, float* out, int out_on_device) {
    if (int rc = guard(ctx)) return rc;
    if (!out) return PBS_ERR_INVALID_ARGUMENT;
    return ctx->impl.read_dose(out, out_on_device);
}

int pbs_context_read_dose64(PbsContext* ctx, double* out, int out_on_device) {
    if (int rc = guard(ctx)) return rc;
    if (!out) return PBS_ERR_INVALID_ARGUMENT;
    return ctx->impl.read_dose64(out, out_on_device);
}

int pbs_measure_fp32_peak(int gpu_id, double* tflops) {
    if (!tflops) return PBS_ERR_INVALID_ARGUMENT;
    return pbs::measure_fp32_peak(gpu_id, tflops);
}

int pbs_context_synchronize(PbsContext* ctx) {
    if (int rc = guard(ctx)) return rc;
    cudaSetDevice(ctx->impl.device);
    if (int rc = ctx->impl.flush_dose_init()) return rc;
    cudaError_t e = cudaStreamSynchronize(ctx->impl.stream);
    if (e != cudaSuccess) {
        pbs::set_error(std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
        return PBS_ERR_CUDA;
    }
    return ctx->impl.take_device_errors();
}

void* pbs_context_stream(PbsContext* ctx) { return ctx ? static_cast<void*>(ctx->impl.stream) : nullptr; }

void* pbs_context_dose_device_ptr(PbsContext* ctx) {
    if (!ctx) return nullptr;
    // The caller may now write anywhere in the grid: resets and readouts cover all of it.
    ctx->impl.doseExposed = true;
    ctx->impl.doseBoxed = false;
    return ctx->impl.dose64.ptr;
}

int pbs_context_beam_stats(PbsContext* ctx, PbsBeamStats* out) {
    if (int rc = guard(ctx)) return rc;
    if (!out) return PBS_ERR_INVALID_ARGUMENT;
    return ctx->impl.beam_stats(out);
}

int pbs_context_layer_stats(PbsContext* ctx, int layer, PbsLayerStats* out) {
    if (int rc = guard(ctx)) return rc;
    if (!out) return PBS_ERR_INVALID_ARGUMENT;
    return ctx->impl.layer_stats(layer, out);
}

int pbs_context_stage_times(PbsContext* ctx, float* ms, int n) {
    if (int rc = guard(ctx)) return rc;
    if (!ms) return PBS_ERR_INVALID_ARGUMENT;
    return ctx->impl.stage_times(ms, n);
}

int pbs_context_debug_copy(PbsContext* ctx, int which, int layer, void* host_out, size_t bytes) {
    if (int rc = guard(ctx)) return rc;
    if (!host_out) return PBS_ERR_INVALID_ARGUMENT;
    return ctx->impl.debug_copy(which, layer, host_out, bytes);
}

// ---- C++ drop-in face ---------------------------------------------------------

void subsecondWrapper(const float* ctData, const int3& ctDims, const float3& ctResolution, const float3& ctCorner,
                      float* doseData, const int3& doseDims, const float3& doseResolution, const float3& doseCorner,
                      const RTDBeamSettings* beamSettings, size_t numBeams, const RTDEnergyStruct* energyData,
                      int gpuId, bool nuclearCorrection, int verbose) {
    std::vector<PbsBeamDesc> beams(beamSettings ? numBeams : 0);
    for (size_t i = 0; i < beams.size(); ++i) {
        const RTDBeamSettings& s = beamSettings[i];
        PbsBeamDesc& d = beams[i];
        d = PbsBeamDesc{};
        d.energies = s.energies.data();
        d.n_energies = s.energies.size();
        d.spot_sigmas = reinterpret_cast<const float*>(s.spotSigmas.data());
        d.n_spot_sigmas = 2 * s.spotSigmas.size();
        d.ray_spacing[0] = s.raySpacing.x;
        d.ray_spacing[1] = s.raySpacing.y;
        d.steps = s.steps;
        d.source_dist[0] = s.sourceDist.x;
        d.source_dist[1] = s.sourceDist.y;
        d.spot_offset[0] = s.spotOffset.x;
        d.spot_offset[1] = s.spotOffset.y;
        d.spot_offset[2] = s.spotOffset.z;
        d.spot_delta[0] = s.spotDelta.x;
        d.spot_delta[1] = s.spotDelta.y;
        d.spot_delta[2] = s.spotDelta.z;
        d.max_subspots_per_layer = s.maxSubspotsPerLayer;
        d.subspot_data = s.subspotData.data();
        d.n_subspot_data = s.subspotData.size();
        d.layer_spot_counts = s.layerSpotCounts.data();
        d.n_layer_spot_counts = s.layerSpotCounts.size();
        d.spot_positions = s.spotPositions.data();
        d.n_spot_positions = s.spotPositions.size();
        d.spot_positions_are_indices = s.spotPositionsAreIndices;
        d.spot_weights = s.spotWeights.data();
        d.n_spot_weights = s.spotWeights.size();
        d.spot_beam_directions = s.spotBeamDirections.data();
        d.n_spot_beam_directions = s.spotBeamDirections.size();
        d.layer_longitudinal_cutoffs = s.layerLongitudinalCutoffs.data();
        d.n_layer_longitudinal_cutoffs = s.layerLongitudinalCutoffs.size();
        d.water_equivalence = s.waterEquivalence.data();
        d.n_water_equivalence = s.waterEquivalence.size();
        d.ray_weq_header = s.rayWeqHeader.data();
        d.n_ray_weq_header = s.rayWeqHeader.size();
        d.profile_data = s.profileData.data();
        d.n_profile_data = s.profileData.size();
        d.profile_setting = s.profileSetting.data();
        d.n_profile_setting = s.profileSetting.size();
        d.beam_para_data = s.beamParaData.data();
        d.n_beam_para_data = s.beamParaData.size();
        const float3* v[4] = {&s.beamDirection, &s.bmXDirection, &s.bmYDirection, &s.sourcePosition};
        float* o[4] = {d.beam_direction, d.bm_x_direction, d.bm_y_direction, d.source_position};
        for (int k = 0; k < 4; ++k) {
            o[k][0] = v[k]->x;
            o[k][1] = v[k]->y;
            o[k][2] = v[k]->z;
        }
        d.sad = s.sad;
        d.ref_plane_z = s.refPlaneZ;
        d.roi_linear_indices = s.roiLinearIndices.data();
        d.n_roi_linear_indices = s.roiLinearIndices.size();
        d.profile_energies = s.profileEnergies.data();
        d.n_profile_energies = s.profileEnergies.size();
        d.beam_para_pos = s.beamParaPos;
    }
    PbsEnergyDesc e{};
    if (energyData) {
        const RTDEnergyStruct& s = *energyData;
        e.n_energy_samples = s.nEnergySamples;
        e.n_energies = s.nEnergies;
        e.energies_per_u = s.energiesPerU.data();
        e.n_energies_per_u = s.energiesPerU.size();
        e.peak_depths = s.peakDepths.data();
        e.n_peak_depths = s.peakDepths.size();
        e.scale_facts = s.scaleFacts.data();
        e.n_scale_facts = s.scaleFacts.size();
        e.cidd_matrix = s.ciddMatrix.data();
        e.n_cidd_matrix = s.ciddMatrix.size();
        e.n_density_samples = s.nDensitySamples;
        e.density_scale_fact = s.densityScaleFact;
        e.density_vector = s.densityVector.data();
        e.n_density_vector = s.densityVector.size();
        e.n_sp_samples = s.nSpSamples;
        e.sp_scale_fact = s.spScaleFact;
        e.sp_vector = s.spVector.data();
        e.n_sp_vector = s.spVector.size();
        e.n_rrl_samples = s.nRRlSamples;
        e.rrl_scale_fact = s.rRlScaleFact;
        e.rrl_vector = s.rRlVector.data();
        e.n_rrl_vector = s.rRlVector.size();
        e.nuc_weight_matrix = s.nucWeightMatrix.data();
        e.n_nuc_weight_matrix = s.nucWeightMatrix.size();
        e.nuc_sq_sigma_matrix = s.nucSqSigmaMatrix.data();
        e.n_nuc_sq_sigma_matrix = s.nucSqSigmaMatrix.size();
        e.nuclear_tables_aligned_to_primary_axis = s.nuclearTablesAlignedToPrimaryAxis;
    }
    const int cd[3] = {ctDims.x, ctDims.y, ctDims.z};
    const float cr[3] = {ctResolution.x, ctResolution.y, ctResolution.z};
    const float cc[3] = {ctCorner.x, ctCorner.y, ctCorner.z};
    const int dd[3] = {doseDims.x, doseDims.y, doseDims.z};
    const float dr[3] = {doseResolution.x, doseResolution.y, doseResolution.z};
    const float dc[3] = {doseCorner.x, doseCorner.y, doseCorner.z};
    const int rc = pbs::subsecond_wrapper(ctData, cd, cr, cc, doseData, dd, dr, dc,
                                          beamSettings ? beams.data() : nullptr, numBeams,
                                          energyData ? &e : nullptr, gpuId, nuclearCorrection, verbose);
    // The reference throws for geometry failures and for every nuclear-halo contract
    // failure (wrapper.cu:1077-1097, 3418-3450; complete_superposition.cu:609-627).
    if (rc == PBS_ERR_GEOMETRY || rc == PBS_ERR_UNSUPPORTED) throw std::runtime_error(pbs::last_error());
    if (rc != PBS_OK) std::fprintf(stderr, "%s\n", pbs::last_error());
}

RTDBeamSettings* createRTDBeamSettings() { return new RTDBeamSettings(); }
void destroyRTDBeamSettings(RTDBeamSettings* beam) { delete beam; }
RTDEnergyStruct* createRTDEnergyStruct() { return new RTDEnergyStruct(); }
void destroyRTDEnergyStruct(RTDEnergyStruct* energy) { delete energy; }

}  // extern "C"
