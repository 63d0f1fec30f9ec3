/*
 * raytracedicom_integration.h - C++ drop-in face of libsubsecondpbs_b200.so.
 *
 * Declares the same structs (member order and types) and the same entry points as
 * the reference's include/core/raytracedicom_integration.h:31-144, so code written
 * against the reference (for example its pybind module,
 * src/bindings/raytracedicom_pybind.cpp:1612,1850, or its integration test,
 * src/tests/wrapper_integration_test.cu:4136) compiles and links against this
 * library unchanged. The structs carry std::vector members, so this face is a C++17
 * ABI; plain-C and FFI callers use subsecondpbs.h instead.
 *
 * Behaviour of subsecondWrapper follows the reference: invalid input prints a
 * message to stderr and returns without touching doseData; beam-geometry failures
 * throw std::runtime_error. CUDA failures print and return (the reference exits
 * the process). The dose of every beam is accumulated into doseData.
 */
#ifndef SUBSECONDPBS_RAYTRACEDICOM_INTEGRATION_H
#define SUBSECONDPBS_RAYTRACEDICOM_INTEGRATION_H

#include <cuda_runtime.h>
#include <vector>

#if defined(__GNUC__)
#define RTD_API __attribute__((visibility("default")))
#else
#define RTD_API
#endif

/* Physics constants of the reference header (raytracedicom_integration.h:22-28). */
#ifndef P_INV
#define P_INV 0.5649718f
#endif
#ifndef E_COEF
#define E_COEF 8.639415f
#endif
#ifndef SQRT2
#define SQRT2 1.41421356f
#endif
#ifndef E_REF_SQ
#define E_REF_SQ 198.81f
#endif
#ifndef SIGMA_DELTA
#define SIGMA_DELTA 0.21f
#endif
#ifndef RAY_WEIGHT_CUTOFF
#define RAY_WEIGHT_CUTOFF 1e-6f
#endif

/* Replaces RTDBeamSettings, raytracedicom_integration.h:31-97 (same members). */
struct RTDBeamSettings {
    std::vector<float> energies;
    std::vector<float2> spotSigmas;
    float2 raySpacing;
    unsigned int steps;
    float2 sourceDist;
    float3 spotOffset;
    float3 spotDelta;
    float3 gantryToImOffset;
    float3 gantryToImMatrix;
    float3 gantryToDoseOffset;
    float3 gantryToDoseMatrix;
    int maxSubspotsPerLayer = 0;
    std::vector<float> subspotData;
    std::vector<int> layerSpotCounts;
    std::vector<float> spotPositions;
    bool spotPositionsAreIndices = false;
    std::vector<float> spotWeights;
    std::vector<float> spotBeamDirections;
    std::vector<float> layerLongitudinalCutoffs;
    std::vector<float> waterEquivalence;
    std::vector<float> rayWeqHeader;
    std::vector<float> profileEnergies;
    std::vector<float> profileData;
    std::vector<float> profileSetting;
    std::vector<float> beamParaData;
    float beamParaPos = 0.0f;
    float3 beamDirection = {0.0f, 0.0f, 1.0f};
    float3 bmXDirection = {1.0f, 0.0f, 0.0f};
    float3 bmYDirection = {0.0f, 1.0f, 0.0f};
    float3 sourcePosition = {0.0f, 0.0f, 0.0f};
    float sad = 0.0f;
    float refPlaneZ = 0.0f;
    std::vector<int> roiLinearIndices;
};

/* Replaces RTDEnergyStruct, raytracedicom_integration.h:99-128 (same members). */
struct RTDEnergyStruct {
    int nEnergySamples = 0;
    int nEnergies = 0;
    std::vector<float> energiesPerU;
    std::vector<float> peakDepths;
    std::vector<float> scaleFacts;
    std::vector<float> ciddMatrix;
    int nDensitySamples = 0;
    float densityScaleFact = 0.0f;
    std::vector<float> densityVector;
    int nSpSamples = 0;
    float spScaleFact = 0.0f;
    std::vector<float> spVector;
    int nRRlSamples = 0;
    float rRlScaleFact = 0.0f;
    std::vector<float> rRlVector;
    int nNucEnergySamples = 0;
    int nNucEnergies = 0;
    std::vector<float> nucEnergiesPerU;
    std::vector<float> nucPeakDepths;
    std::vector<float> nucScaleFacts;
    std::vector<float> nucWeightMatrix;
    std::vector<float> nucSqSigmaMatrix;
    bool nuclearTablesAlignedToPrimaryAxis = false;
    bool nuclearTablesResampledFromReference = false;
};

/* Replaces subsecondWrapper, raytracedicom_integration.h:132-139
 * (implementation src/core/raytracedicom_wrapper.cu:2446-5661). */
extern "C" RTD_API void subsecondWrapper(const float* ctData, const int3& ctDims, const float3& ctResolution,
                                 const float3& ctCorner, float* doseData, const int3& doseDims,
                                 const float3& doseResolution, const float3& doseCorner,
                                 const RTDBeamSettings* beamSettings, size_t numBeams,
                                 const RTDEnergyStruct* energyData, int gpuId = 0, bool nuclearCorrection = false,
                                 int verbose = 0);

/* Replace raytracedicom_integration.h:141-144 (raytracedicom_wrapper.cu:5664-5678). */
extern "C" RTD_API RTDBeamSettings* createRTDBeamSettings();
extern "C" RTD_API void destroyRTDBeamSettings(RTDBeamSettings* beam);
extern "C" RTD_API RTDEnergyStruct* createRTDEnergyStruct();
extern "C" RTD_API void destroyRTDEnergyStruct(RTDEnergyStruct* energy);

#endif /* SUBSECONDPBS_RAYTRACEDICOM_INTEGRATION_H */
