// Biological maps on top of the physical dose. CarbonPBS accumulates, per voxel,
// the dose-weighted linear-quadratic parameters of its point-kernel dose
// (cuCalFinalDoseAndRBEKernel, carbonPBS/deviceCalDose.cu:587-736, alpha and
// sqrt(beta) weighted by dose, LET by dose) and turns them into RBE maps
// (LQRBEKernel :738-772, mkmRBEMapKernel :1060-1126). Here the factors ride on the
// pencil-beam pipeline: bio_channel_kernel scales every step's IDD by the step's
// factor (alpha, sqrt(beta), z1D or LET at the step's water-equivalent depth),
// the scaled IDD is superposed with the dose's own radii and work list and
// transferred like the dose, and bio_map_kernel evaluates the maps per voxel.
#include <cuda_runtime.h>

#include <algorithm>

#include "kernels.h"
#include "../../include/subsecondpbs.h"

namespace pbs {

namespace {

// Value of a [n] table at fractional index x, clamped to the table.
__device__ __forceinline__ float table_at(const float* __restrict__ t, int n, float x) {
    x = fminf(fmaxf(x, 0.0f), float(n - 1));
    const float f = floorf(x);
    const int i0 = int(f), i1 = min(i0 + 1, n - 1);
    const float a = __ldg(t + i0), b = __ldg(t + i1);
    return a + (b - a) * (x - f);
}

// LET of a step: dose-averaged over the depth samples of the layer's row.
__device__ __forceinline__ float step_let(const BioDev& m, float row, float weq) {
    row = fminf(fmaxf(row, 0.0f), float(m.letRows - 1));
    const float fr = floorf(row);
    const int r0 = int(fr), r1 = min(r0 + 1, m.letRows - 1);
    const float ar = row - fr;
    float s1 = 0.0f, s2 = 0.0f;
    for (int j = 0; j < m.letSamples; ++j) {
        const float depth =
            weq + m.rangeShifter + (float(j) - 0.5f * float(m.letSamples - 1)) * m.estDimension / float(m.letSamples);
        const float x = (depth - m.letDepth0) / m.letDepthStep;
        const float a = table_at(m.letTable + static_cast<size_t>(r0) * m.letDepths, m.letDepths, x);
        const float b = table_at(m.letTable + static_cast<size_t>(r1) * m.letDepths, m.letDepths, x);
        const float t = a + (b - a) * ar;
        s1 += t;
        s2 += t * t;
    }
    return s1 > 0.0f ? s2 / s1 : 0.0f;
}

// One chunk of layers: out = idd * factor of `channel` at every computed step
// (channel 0: alpha (LQ) or z1D (MKM), 1: sqrt(beta) (LQ), 2: LET).
__global__ void __launch_bounds__(256)
bio_channel_kernel(BeamGeomDev g, BioDev m, int layer0, int nLayers, const float* __restrict__ idd,
                   const float* __restrict__ wepl, const LayerStateDev* __restrict__ ls,
                   const BeamStateDev* __restrict__ beam, const float* __restrict__ layerRow, int channel,
                   float* __restrict__ out) {
    const size_t padPlane = static_cast<size_t>(g.pitchX) * g.pitchY;
    const size_t layerStride = static_cast<size_t>(g.steps) * padPlane;
    const size_t rayPlane = static_cast<size_t>(g.rayX) * g.rayY;
    const int first = beam->firstInside;
    const size_t total = static_cast<size_t>(nLayers) * layerStride;
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < total; i += size_t(gridDim.x) * blockDim.x) {
        const int lc = int(i / layerStride);
        const size_t r = i - size_t(lc) * layerStride;
        const int zr = int(r / padPlane);
        const size_t p = r - size_t(zr) * padPlane;
        const int y = int(p / g.pitchX), x = int(p - size_t(y) * g.pitchX);
        const int l = layer0 + lc;
        const int k = first + zr;
        float v = 0.0f;
        if (k < ls[l].afterLast && x < g.rayX && y < g.rayY) {
            const float d = idd[i];
            if (d > 0.0f) {
                const float weq = wepl[static_cast<size_t>(k) * rayPlane + static_cast<size_t>(y) * g.rayX + x];
                const float let = step_let(m, layerRow[l], weq);
                float f = let;
                if (channel < 2) {
                    const float li = let > 0.0f ? (log10f(let) - m.lqLog0) / m.lqLogStep : 0.0f;
                    if (m.model == PBS_BIO_MKM)
                        f = table_at(m.z1d, m.nLq, li);
                    else
                        f = channel == 0 ? table_at(m.alpha, m.nLq, li) : sqrtf(fmaxf(table_at(m.beta, m.nLq, li), 0.0f));
                }
                v = d * f;
            }
        }
        out[i] = v;
    }
}

// Maps from the FP64 accumulators (dose, dose * channel 0, 1, 2).
__global__ void bio_map_kernel(const double* __restrict__ dose, const double* __restrict__ c0,
                               const double* __restrict__ c1, const double* __restrict__ c2, size_t n, BioDev m,
                               int map, float* __restrict__ out) {
    for (size_t i = blockIdx.x * size_t(blockDim.x) + threadIdx.x; i < n; i += size_t(gridDim.x) * blockDim.x) {
        const double d = dose[i];
        double v = 0.0;
        if (map == PBS_BIO_MAP_DOSE) {
            v = d;
        } else if (map == PBS_BIO_MAP_LETD) {
            v = d > 0.0 ? c2[i] / d : 0.0;
        } else if (map == PBS_BIO_MAP_ALPHA) {
            v = d > 0.0 ? c0[i] / d : 0.0;
        } else if (map == PBS_BIO_MAP_BETA) {
            const double sb = d > 0.0 ? c1[i] / d : 0.0;
            v = sb * sb;
        } else if (map == PBS_BIO_MAP_Z1D) {
            const double z = d > 0.0 ? c0[i] / d : 0.0;
            v = 0.172 + double(m.beta0) * z;
        } else {  // RBE or RBE x dose
            double rbe = 1.0;
            if (m.model == PBS_BIO_MKM) {
                // mkmRBEMapKernel (deviceCalDose.cu:1060-1126): the photon dose of equal
                // effect over the ion dose, 1 at or below 1e-3 Gy.
                const double z = d > 0.0 ? c0[i] / d : 0.0;
                const double a = 0.172 + double(m.beta0) * z;
                const double b0 = double(m.beta0), t2 = double(m.alpha0) / 2.0 / b0;
                const double dx = -t2 + sqrt(t2 * t2 + (a * d + b0 * d * d) / b0);
                rbe = d > 1e-3 ? dx / d : 1.0;
            } else {
                // LQRBEKernel (deviceCalDose.cu:738-772): 3.988565 Gy over the ion dose of
                // 10 % survival, 1 where the dose, alpha or beta vanishes.
                if (d != 0.0 && c0[i] != 0.0 && c1[i] != 0.0) {
                    const double a = c0[i] / d;
                    const double sb = c1[i] / d, b = sb * sb;
                    const double d10 = (-a + sqrt(a * a - 4.0 * -2.302585 * b)) / b * 0.5;
                    rbe = 3.988565 / d10;
                }
            }
            v = map == PBS_BIO_MAP_RBE ? rbe : rbe * d;
        }
        out[i] = float(v);
    }
}

}  // namespace

cudaError_t launch_bio_channel(const BeamGeomDev& g, const BioDev& m, int layer0, int nLayers, const float* idd,
                               const float* wepl, const LayerStateDev* ls, const BeamStateDev* beam,
                               const float* layerRow, int channel, float* out, cudaStream_t s) {
    const size_t total = static_cast<size_t>(nLayers) * g.steps * g.pitchX * g.pitchY;
    const int blocks = int(std::min<size_t>((total + 255) / 256, 148 * 16));
    bio_channel_kernel<<<blocks, 256, 0, s>>>(g, m, layer0, nLayers, idd, wepl, ls, beam, layerRow, channel, out);
    return cudaGetLastError();
}

cudaError_t launch_bio_map(const double* dose, const double* c0, const double* c1, const double* c2, size_t n,
                           const BioDev& m, int map, float* out, cudaStream_t s) {
    const int blocks = int(std::min<size_t>((n + 255) / 256, 148 * 16));
    bio_map_kernel<<<blocks, 256, 0, s>>>(dose, c0, c1, c2, n, m, map, out);
    return cudaGetLastError();
}

__global__ void reset_work_claims_kernel(BeamStateDev* beam) {
    beam->workNext = 0;
    beam->workNextSmall = 0;
    beam->workNextTiny = 0;
}

cudaError_t launch_reset_work_claims(BeamStateDev* beam, cudaStream_t s) {
    reset_work_claims_kernel<<<1, 1, 0, s>>>(beam);
    return cudaGetLastError();
}

}  // namespace pbs
