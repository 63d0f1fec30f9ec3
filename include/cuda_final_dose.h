/*
 * cuda_final_dose.h - the legacy cudaFinalDose symbol of the reference
 * (include/algorithms/cuda_final_dose.h:42-56, src/algorithms/cuda_final_dose.cu:230),
 * exported by libsubsecondpbs_b200.so with the reference's observable behaviour.
 *
 * The reference's implementation is a stub: it reduces the ROI to a bounding box,
 * tests whether the beam points at the box centre, computes CPB weights and sigma
 * maps that it then discards, and finally zeroes finalDose (a device array of
 * doseGridDims.x * .y * .z floats). When the beam does not point at the ROI it
 * returns without touching finalDose. This library does the same observable work:
 * the same ROI box and intersection test (cuda_final_dose.cu:58-151), then the
 * zeroing. Dose computation goes through subsecondWrapper / pbs_subsecond_wrapper.
 */
#ifndef SUBSECONDPBS_CUDA_FINAL_DOSE_H
#define SUBSECONDPBS_CUDA_FINAL_DOSE_H

#include <cuda_runtime.h>

#if defined(__GNUC__)
#define CFD_API __attribute__((visibility("default")))
#else
#define CFD_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* The reference's vec3f / vec3i (include/core/common.cuh:39-78): 12 bytes, no padding. */
typedef struct { float x, y, z; } pbs_vec3f;
typedef struct { int x, y, z; } pbs_vec3i;

/* Replaces cudaFinalDose (include/algorithms/cuda_final_dose.h:42-56). `roiIndices`
 * is device (or host) memory of numROIIndices voxel indices; `finalDose` is device
 * memory. `subspotData`, `sad`, `refPlaneZ`, `numLayers` and `maxSubspotsPerLayer`
 * only fed the reference's discarded intermediate results. */
CFD_API void cudaFinalDose(cudaTextureObject_t subspotData, const pbs_vec3i* roiIndices, int numROIIndices,
                           pbs_vec3f doseGridResolution, pbs_vec3f doseGridCorner, pbs_vec3f beamDirection,
                           pbs_vec3f sourcePosition, float sad, float refPlaneZ, int numLayers,
                           int maxSubspotsPerLayer, float* finalDose, pbs_vec3i doseGridDims);

#ifdef __cplusplus
}
#endif

#endif /* SUBSECONDPBS_CUDA_FINAL_DOSE_H */
