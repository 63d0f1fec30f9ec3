// Legacy CPB fluence (subspots -> CPB cells -> ray weights) for callers that must
// not allocate device memory: the CPB grid lives in a fixed static device array of
// this module instead of a context buffer. Same kernels as the context path
// (convolution.cu:95-152 and 269-339 of the reference, via launch_conv_cpb).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "context.h"
#include "kernels.h"
#include "../../include/subsecondpbs.h"

// 2^20 float CPB cells (4 MiB) per device: ray grid cells x layers of one call.
static constexpr size_t kScratchCells = size_t(1) << 20;
static __device__ __align__(256) float g_cpbScratch[kScratchCells];

namespace pbs {

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratchMutex;
float* g_scratchPtr[kMaxDevices] = {};

// Device address of the scratch array on the current device, looked up once per
// device (the first call on a device does it) and kept for the life of the process.
// A cudaDeviceReset of that device unloads the module the address belongs to, so
// the entry point must not be used on that device after such a reset.
int scratch_for_current_device(int device, float** out) {
    std::lock_guard<std::mutex> lock(g_scratchMutex);
    if (!g_scratchPtr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_cpbScratch);
        if (e != cudaSuccess) {
            set_error(std::string("cudaGetSymbolAddress of the static CPB scratch failed: ") + cudaGetErrorString(e));
            return PBS_ERR_CUDA;
        }
        g_scratchPtr[device] = static_cast<float*>(p);
    }
    *out = g_scratchPtr[device];
    return PBS_OK;
}

}  // namespace

}  // namespace pbs

extern "C" PBS_API int pbs_cpb_fluence_no_alloc(const float* d_subspots, int max_subspots, int n_layers,
                                                const int ray_dims[2], const float cpb_corner[2],
                                                const float cpb_resolution[2], float* d_ray_weights, void* stream) {
    using namespace pbs;
    if (!d_subspots || !d_ray_weights || !ray_dims || !cpb_corner || !cpb_resolution || max_subspots <= 0 ||
        n_layers <= 0 || ray_dims[0] <= 0 || ray_dims[1] <= 0 || !(cpb_resolution[0] > 0.0f) ||
        !(cpb_resolution[1] > 0.0f)) {
        set_error("pbs_cpb_fluence_no_alloc: null pointer or non-positive size");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    // Launch limits of the two kernels: layers run on grid y / z (at most 65535) and
    // ray rows in groups of 8 on grid y.
    if (n_layers > 65535 || (ray_dims[1] + 7) / 8 > 65535) {
        set_error("pbs_cpb_fluence_no_alloc: n_layers = " + std::to_string(n_layers) + " and ray_dims[1] = " +
                  std::to_string(ray_dims[1]) + " exceed the launch limits (n_layers <= 65535, ray_dims[1] <= 524280)");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    const size_t cells = size_t(ray_dims[0]) * size_t(ray_dims[1]) * size_t(n_layers);
    if (cells > kScratchCells) {
        set_error("pbs_cpb_fluence_no_alloc: ray_dims[0]*ray_dims[1]*n_layers = " + std::to_string(cells) +
                  " CPB cells exceeds the static scratch of " + std::to_string(kScratchCells) +
                  " cells; split the layers over several calls");
        return PBS_ERR_INVALID_ARGUMENT;
    }
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) {
        set_error(std::string("pbs_cpb_fluence_no_alloc: no usable current device: ") + cudaGetErrorString(e));
        return PBS_ERR_CUDA;
    }
    if (device < 0 || device >= kMaxDevices) {
        set_error("pbs_cpb_fluence_no_alloc: current device " + std::to_string(device) +
                  " is beyond the " + std::to_string(kMaxDevices) + " devices this entry point keeps scratch for");
        return PBS_ERR_UNSUPPORTED;
    }
    float* scratch = nullptr;
    int rc = scratch_for_current_device(device, &scratch);
    if (rc) return rc;
    BeamGeomDev g{};
    g.rayX = ray_dims[0];
    g.rayY = ray_dims[1];
    g.numLayers = n_layers;
    g.cpbCornerX = cpb_corner[0];
    g.cpbCornerY = cpb_corner[1];
    g.cpbResX = cpb_resolution[0];
    g.cpbResY = cpb_resolution[1];
    // launch_conv_cpb clears the scratch cells it accumulates into before its kernels run.
    e = launch_conv_cpb(g, d_subspots, max_subspots, scratch, d_ray_weights, static_cast<cudaStream_t>(stream));
    if (e != cudaSuccess) {
        set_error(std::string("pbs_cpb_fluence_no_alloc: launch failed: ") + cudaGetErrorString(e));
        return PBS_ERR_CUDA;
    }
    return PBS_OK;
}
