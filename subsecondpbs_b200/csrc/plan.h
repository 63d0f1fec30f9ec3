// Host-side planning of one beam: validation, gantry frame, spot lattice, ray grid,
// tracer geometry and the per-layer energy parameters that do not depend on the
// traced CT. Everything that depends on the trace (entry step, cut-off steps,
// passive steps, tile radii) is computed on the device by the beam planner kernel.
#pragma once

#include <string>
#include <vector>

#include "pbs_geom.h"
#include "../../include/subsecondpbs.h"

namespace pbs {

struct GridDesc {
    int dims[3];
    float res[3];
    float corner[3];
};

// Dense spot-weight lattice (wrapper.cu:755-764, built at 1259-1473).
struct RawLattice {
    bool valid = false;
    int nx = 0, ny = 0, nl = 0;
    float dx = 0.f, dy = 0.f, ox = 0.f, oy = 0.f;
    int skippedZeroWeightSpots = 0;
    std::string failure;
    std::vector<float> weights;  // [nl][ny][nx]
};

// Per-layer parameters fixed before tracing.
struct LayerHost {
    float energy = 0.f;
    // Spot->ray convolution stage (wrapper.cu:3774-3833).
    float convPeakDepth = 0.f;  // mm, findDecimalOrdered-based peak depth
    float sigmaXmm = 0.f, sigmaYmm = 0.f;
    // IDD stage (wrapper.cu:3926-4053, 4140-4292).
    float energyIdx = 0.f;
    float energyScaleFact = 1.f;
    float peakDepth = 0.f;
    float rangeStopDepth = 0.f;
    float sigmaSqAirQuad = 0.f;
    float sigmaSqAirLin = 0.f;
    float spotDist = 1.f;
    float sigmaXidd = 0.f;  // spot sigma x in mm used for the IDD entry variance
};

struct BeamPlan {
    int numLayers = 0;
    int maxSubspots = 0;
    float lenToMm = 1.f;
    float energyDepthToMm = 1.f;
    V3 bmX{}, bmY{}, bmZ{};
    Affine gantryToWorld{}, worldToGantry{}, gantryToImIdx{}, gantryToDoseIdx{};
    bool hasLattice = false;
    RawLattice lattice;
    int convMode = 0;  // 0 raw lattice, 1 legacy CPB
    V3 cpbCorner{}, cpbRes{};
    int cpbDims[3] = {0, 0, 0};
    int rayDims[2] = {0, 0};
    int superpDims[2] = {0, 0};
    V2 sourceDist{};
    float minGZ = 0.f, maxGZ = 0.f;
    float stepLengthMm = 0.f;
    float startZ = 0.f;
    int tracerSteps = 0;
    V3 fanCorner{}, fanDelta{};
    FromFan fanIdxToImIdx{};
    FromFan rayIdxToDoseIdx{};
    TracerParams tracer{};
    float volConst = 0.f, volLin = 0.f, volSq = 0.f;
    float maxPeakDepthMm = 0.f;
    std::vector<LayerHost> layers;
    // Water-equivalence import transport (wrapper.cu:3316-3395, 3566-3640): the
    // exporter's per-ray water-equivalent depths [weqNx][weqNy][weqSteps] replace
    // the CT trace. Lattice origin and spacing are in beam length units.
    bool hasWeqVolume = false;
    bool startAlignedToWeq = false;
    int weqNx = 0, weqNy = 0, weqSteps = 0, weqActiveSteps = 0;
    float weqStepMm = 1.f;
    float weqX0 = 0.f, weqY0 = 0.f, weqDx = 0.f, weqDy = 0.f;
};

// CarbonPBS lateral profile model of one beam: the table shape the reference infers
// from profile_setting / profile_data / beam_para_data (wrapper.cu:2816-2862) and,
// per layer, the fractional table row and the interpolated beam parameters
// (wrapper.cu:4577-4606).
struct ProfilePlan {
    bool table = false;          // profile_data has the inferred [rows][depthN][channels] shape
    bool beamPara = false;       // beam_para_data holds at least 3 values per layer
    int rows = 0, depthN = 0, channels = 0;
    float depth0 = 0.f, depthStep = 0.f;
    std::vector<float> row, bp0, bp1, bp2;  // per layer
    // What the reference's two switches would run on this beam (wrapper.cu:4656-4660,
    // 4814-4818) and their kernels' own early returns (wrapper.cu:2103-2104, 2171).
    bool sigmaOverride() const {
        return table && beamPara && depthN > 0 && channels >= 3 && (channels - 1) / 2 > 0 && depthStep > 0.0f;
    }
    bool overallWeight() const { return table && depthN > 0 && channels > 0 && depthStep > 0.0f; }
};
void plan_carbon_profile(const PbsBeamDesc& b, const PbsEnergyDesc& e, const BeamPlan& P, ProfilePlan& out);

// wrapper.cu:1025-1075 (+ the LUT sample counts the textures are built with).
bool validate_global(const float* ct, const GridDesc& ctGrid, const void* dose, const GridDesc& doseGrid,
                     const PbsBeamDesc* beams, size_t numBeams, const PbsEnergyDesc* e, std::string& err);
// wrapper.cu:1099-1157
bool validate_beam(const PbsBeamDesc& b, size_t beamIdx, std::string& err);

// Plans one beam. Returns PBS_OK or a PBS_ERR_* code with `err` set.
int plan_beam(const PbsBeamDesc& b, const PbsEnergyDesc& e, const GridDesc& ctGrid, const GridDesc& doseGrid,
              BeamPlan& out, std::string& err);

// Reference host helpers (include/utils/vector_find.h, vector_interpolate.h).
// Lattice cells (four slots per spot, cell -1 unused) and shares each spot of the
// beam feeds in the lattice that plan_beam builds for it.
bool lattice_spot_cells(const PbsBeamDesc& b, const RawLattice& lat, std::vector<int>& cells,
                        std::vector<float>& shares);

int find_first_larger_ordered(const float* v, int n, float value);
float find_decimal_ordered(const float* v, int n, float value);
float vector_interpolate(const float* v, int n, float idx);

// CT interpretation (wrapper.cu:2290-2337).
int parse_ct_input_type_env();
void sample_ct_stats(const float* data, size_t n, float& mn, float& mx);
int auto_detect_ct_type(float mn, float mx);
float find_fractional_index_monotonic(const float* v, int n, float value);

}  // namespace pbs
