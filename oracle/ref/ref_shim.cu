// C shim over the reference's subsecondWrapper (test infrastructure only): fills the
// reference's RTDBeamSettings / RTDEnergyStruct from the flat descriptors of
// include/subsecondpbs.h so the reference can be driven from ctypes on identical
// inputs. Compiled together with the reference sources by build_ref.sh.
#include <cstdio>
#include <exception>
#include <vector>

#include "raytracedicom_integration.h"  // the reference's header (include/core)
#include "../../include/subsecondpbs.h"

namespace {

template <typename T>
std::vector<T> vec(const T* p, size_t n) {
    return p && n ? std::vector<T>(p, p + n) : std::vector<T>();
}

float3 f3(const float* v) { return make_float3(v[0], v[1], v[2]); }

}  // namespace

// RTDBeamSettings of the reference from the flat descriptor.
static RTDBeamSettings to_reference(const PbsBeamDesc& d) {
    RTDBeamSettings b;
    b.energies = vec(d.energies, d.n_energies);
    b.spotSigmas.clear();
    for (size_t k = 0; 2 * k + 1 < d.n_spot_sigmas; ++k)
        b.spotSigmas.push_back(make_float2(d.spot_sigmas[2 * k], d.spot_sigmas[2 * k + 1]));
    b.raySpacing = make_float2(d.ray_spacing[0], d.ray_spacing[1]);
    b.steps = d.steps;
    b.sourceDist = make_float2(d.source_dist[0], d.source_dist[1]);
    b.spotOffset = f3(d.spot_offset);
    b.spotDelta = f3(d.spot_delta);
    b.gantryToImOffset = make_float3(0, 0, 0);
    b.gantryToImMatrix = make_float3(0, 0, 0);
    b.gantryToDoseOffset = make_float3(0, 0, 0);
    b.gantryToDoseMatrix = make_float3(0, 0, 0);
    b.maxSubspotsPerLayer = d.max_subspots_per_layer;
    b.subspotData = vec(d.subspot_data, d.n_subspot_data);
    b.layerSpotCounts = vec(d.layer_spot_counts, d.n_layer_spot_counts);
    b.spotPositions = vec(d.spot_positions, d.n_spot_positions);
    b.spotPositionsAreIndices = d.spot_positions_are_indices != 0;
    b.spotWeights = vec(d.spot_weights, d.n_spot_weights);
    b.spotBeamDirections = vec(d.spot_beam_directions, d.n_spot_beam_directions);
    b.layerLongitudinalCutoffs = vec(d.layer_longitudinal_cutoffs, d.n_layer_longitudinal_cutoffs);
    b.waterEquivalence = vec(d.water_equivalence, d.n_water_equivalence);
    b.rayWeqHeader = vec(d.ray_weq_header, d.n_ray_weq_header);
    b.profileData = vec(d.profile_data, d.n_profile_data);
    b.profileSetting = vec(d.profile_setting, d.n_profile_setting);
    b.beamParaData = vec(d.beam_para_data, d.n_beam_para_data);
    b.profileEnergies = vec(d.profile_energies, d.n_profile_energies);
    b.beamParaPos = d.beam_para_pos;
    b.beamDirection = f3(d.beam_direction);
    b.bmXDirection = f3(d.bm_x_direction);
    b.bmYDirection = f3(d.bm_y_direction);
    b.sourcePosition = f3(d.source_position);
    b.sad = d.sad;
    b.refPlaneZ = d.ref_plane_z;
    b.roiLinearIndices = vec(d.roi_linear_indices, d.n_roi_linear_indices);
    return b;
}

extern "C" int ref_subsecond_wrapper(const float* ct, const int* ctDims, const float* ctRes, const float* ctCorner,
                                     float* dose, const int* doseDims, const float* doseRes, const float* doseCorner,
                                     const PbsBeamDesc* beams, size_t nBeams, const PbsEnergyDesc* e, int gpuId,
                                     int nuclear, int verbose) {
    std::vector<RTDBeamSettings> bs(nBeams);
    for (size_t i = 0; i < nBeams; ++i) bs[i] = to_reference(beams[i]);
    RTDEnergyStruct es;
    es.nEnergySamples = e->n_energy_samples;
    es.nEnergies = e->n_energies;
    es.energiesPerU = vec(e->energies_per_u, e->n_energies_per_u);
    es.peakDepths = vec(e->peak_depths, e->n_peak_depths);
    es.scaleFacts = vec(e->scale_facts, e->n_scale_facts);
    es.ciddMatrix = vec(e->cidd_matrix, e->n_cidd_matrix);
    es.nDensitySamples = e->n_density_samples;
    es.densityScaleFact = e->density_scale_fact;
    es.densityVector = vec(e->density_vector, e->n_density_vector);
    es.nSpSamples = e->n_sp_samples;
    es.spScaleFact = e->sp_scale_fact;
    es.spVector = vec(e->sp_vector, e->n_sp_vector);
    es.nRRlSamples = e->n_rrl_samples;
    es.rRlScaleFact = e->rrl_scale_fact;
    es.rRlVector = vec(e->rrl_vector, e->n_rrl_vector);
    if (e->nuc_weight_matrix && e->n_nuc_weight_matrix) {
        es.nNucEnergySamples = e->n_energy_samples;
        es.nNucEnergies = e->n_energies;
        es.nucEnergiesPerU = es.energiesPerU;
        es.nucPeakDepths = es.peakDepths;
        es.nucScaleFacts = es.scaleFacts;
        es.nucWeightMatrix = vec(e->nuc_weight_matrix, e->n_nuc_weight_matrix);
        es.nucSqSigmaMatrix = vec(e->nuc_sq_sigma_matrix, e->n_nuc_sq_sigma_matrix);
        es.nuclearTablesAlignedToPrimaryAxis = e->nuclear_tables_aligned_to_primary_axis != 0;
    }
    const int3 cd = make_int3(ctDims[0], ctDims[1], ctDims[2]);
    const int3 dd = make_int3(doseDims[0], doseDims[1], doseDims[2]);
    try {
        subsecondWrapper(ct, cd, make_float3(ctRes[0], ctRes[1], ctRes[2]),
                         make_float3(ctCorner[0], ctCorner[1], ctCorner[2]), dose, dd,
                         make_float3(doseRes[0], doseRes[1], doseRes[2]),
                         make_float3(doseCorner[0], doseCorner[1], doseCorner[2]), bs.data(), bs.size(), &es, gpuId,
                         nuclear != 0, verbose);
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "reference threw: %s\n", ex.what());
        return 2;
    }
    return 0;
}

// The reference's own table parser (src/utils/energy_reader.cpp:21-185) on `dir`.
// Call once with null outputs to get the sizes: sizes[0..4] = nEnergySamples,
// nEnergies, nDensitySamples, nSpSamples, nRRlSamples; sizes[5] = 1 when nuclear
// tables were read (a NUCLEAR_CORR build). scales[0..2] = density, sp, rRl scale
// factors. Then call again with buffers of those sizes: `energy` takes energiesPerU,
// peakDepths and scaleFacts (3 x nEnergies), `cidd` nEnergies x nEnergySamples,
// `luts` density | sp | rRl, `nuc` weights | sqSigmas (2 x nEnergies x nEnergySamples).
#include "energy_reader.h"
#include "energy_struct.h"
#include <cstring>
#include <string>

extern "C" int ref_energy_reader(const char* dir, int* sizes, float* scales, float* energy, float* cidd, float* luts,
                                 float* nuc) {
    EnergyStruct es;
    try {
        es = energyReader(std::string(dir));
    } catch (const std::exception& ex) {
        std::fprintf(stderr, "reference energyReader threw: %s\n", ex.what());
        return 2;
    }
    sizes[0] = es.nEnergySamples;
    sizes[1] = es.nEnergies;
    sizes[2] = es.nDensitySamples;
    sizes[3] = es.nSpSamples;
    sizes[4] = es.nRRlSamples;
    sizes[5] = es.nucWeightMatrix.empty() ? 0 : 1;
    scales[0] = es.densityScaleFact;
    scales[1] = es.spScaleFact;
    scales[2] = es.rRlScaleFact;
    auto put = [](float* dst, const std::vector<float>& v) {
        if (!v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(float));
        return dst + v.size();
    };
    if (energy) put(put(put(energy, es.energiesPerU), es.peakDepths), es.scaleFacts);
    if (cidd) put(cidd, es.ciddMatrix);
    if (luts) put(put(put(luts, es.densityVector), es.spVector), es.rRlVector);
    if (nuc && sizes[5]) put(put(nuc, es.nucWeightMatrix), es.nucSqSigmaMatrix);
    return 0;
}

// The reference's spot batch plan (include/core/rtd_operator_mode.h:43-111) for
// the beam, in the output form of pbs_operator_batch_plan: info = {valid,
// total_layers, total_spots, max_spots_per_batch, n_spans, n_batches}; spans and
// batches receive up to the given capacities.
#include "rtd_operator_mode.h"

extern "C" int ref_operator_batch_plan(const PbsBeamDesc* beam, int maxSpotsPerBatch, PbsOperatorLayerSpan* spans,
                                       int spanCapacity, PbsOperatorBatch* batches, int batchCapacity, int* info) {
    const RTDOperatorBatchPlan p = buildRTDOperatorBatchPlan(to_reference(*beam), maxSpotsPerBatch);
    info[0] = p.valid ? 1 : 0;
    info[1] = p.totalLayers;
    info[2] = p.totalSpots;
    info[3] = p.maxSpotsPerBatch;
    info[4] = static_cast<int>(p.layerSpans.size());
    info[5] = static_cast<int>(p.batches.size());
    for (int i = 0; i < info[4] && i < spanCapacity; ++i) {
        const RTDOperatorLayerSpan& a = p.layerSpans[static_cast<size_t>(i)];
        spans[i].layer_index = a.layerIndex;
        spans[i].spot_begin = a.spotBegin;
        spans[i].spot_count = a.spotCount;
        spans[i].energy = a.energy;
        spans[i].longitudinal_cutoff = a.longitudinalCutoff;
    }
    for (int i = 0; i < info[5] && i < batchCapacity; ++i) {
        const RTDOperatorBatch& a = p.batches[static_cast<size_t>(i)];
        batches[i].batch_index = a.batchIndex;
        batches[i].spot_begin = a.spotBegin;
        batches[i].spot_count = a.spotCount;
        batches[i].first_layer_index = a.firstLayerIndex;
        batches[i].last_layer_index = a.lastLayerIndex;
    }
    return 0;
}
