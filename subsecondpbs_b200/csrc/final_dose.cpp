// cudaFinalDose with the observable behaviour of the reference's stub
// (src/algorithms/cuda_final_dose.cu:58-151, 230-390): ROI bounding box, the
// beam-points-at-the-ROI test, then finalDose is zeroed.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <vector>

#include "../../include/cuda_final_dose.h"

namespace {
constexpr float kRoiMarginX = 5.0f, kRoiMarginY = 5.0f, kRoiMarginZ = 2.0f;  // Macro.cuh:53-55
}  // namespace

extern "C" void cudaFinalDose(cudaTextureObject_t subspotData, const pbs_vec3i* roiIndices, int numROIIndices,
                              pbs_vec3f doseGridResolution, pbs_vec3f doseGridCorner, pbs_vec3f beamDirection,
                              pbs_vec3f sourcePosition, float sad, float refPlaneZ, int numLayers,
                              int maxSubspotsPerLayer, float* finalDose, pbs_vec3i doseGridDims) {
    (void)subspotData;
    (void)sad;
    (void)refPlaneZ;
    (void)numLayers;
    (void)maxSubspotsPerLayer;
    // calculateROIRangeKernel (cuda_final_dose.cu:58-129): index bounding box,
    // corners in grid units plus the margins; an empty ROI gives the origin.
    float mn[3] = {0.f, 0.f, 0.f}, mx[3] = {0.f, 0.f, 0.f};
    if (numROIIndices > 0 && roiIndices) {
        std::vector<pbs_vec3i> idx(static_cast<size_t>(numROIIndices));
        if (cudaMemcpy(idx.data(), roiIndices, idx.size() * sizeof(pbs_vec3i), cudaMemcpyDefault) != cudaSuccess) {
            std::fprintf(stderr, "[CUDA_FINAL_DOSE] cannot read the ROI indices\n");
            return;
        }
        pbs_vec3i lo = idx[0], hi = idx[0];
        for (const pbs_vec3i& v : idx) {
            lo.x = std::min(lo.x, v.x);
            lo.y = std::min(lo.y, v.y);
            lo.z = std::min(lo.z, v.z);
            hi.x = std::max(hi.x, v.x);
            hi.y = std::max(hi.y, v.y);
            hi.z = std::max(hi.z, v.z);
        }
        mn[0] = doseGridCorner.x + float(lo.x) * doseGridResolution.x - kRoiMarginX;
        mn[1] = doseGridCorner.y + float(lo.y) * doseGridResolution.y - kRoiMarginY;
        mn[2] = doseGridCorner.z + float(lo.z) * doseGridResolution.z - kRoiMarginZ;
        mx[0] = doseGridCorner.x + float(hi.x + 1) * doseGridResolution.x + kRoiMarginX;
        mx[1] = doseGridCorner.y + float(hi.y + 1) * doseGridResolution.y + kRoiMarginY;
        mx[2] = doseGridCorner.z + float(hi.z + 1) * doseGridResolution.z + kRoiMarginZ;
    }
    // checkBeamROIIntersectionKernel (cuda_final_dose.cu:132-151).
    const float cx = (mn[0] + mx[0]) * 0.5f, cy = (mn[1] + mx[1]) * 0.5f, cz = (mn[2] + mx[2]) * 0.5f;
    const float dot = beamDirection.x * (cx - sourcePosition.x) + beamDirection.y * (cy - sourcePosition.y) +
                      beamDirection.z * (cz - sourcePosition.z);
    if (!(dot > 0.0f)) {
        std::fprintf(stderr, "[CUDA_FINAL_DOSE] ERROR: Beam does not intersect with ROI!\n");
        return;
    }
    const size_t n = size_t(std::max(doseGridDims.x, 0)) * size_t(std::max(doseGridDims.y, 0)) *
                     size_t(std::max(doseGridDims.z, 0));
    if (finalDose && n) cudaMemset(finalDose, 0, n * sizeof(float));
}
