// Spot -> ray fluence.
//   Mode A (raw spot lattice): separable erf-integrated Gaussian gather-resample,
//     x pass then y pass, all layers in one launch each.
//   Mode B (legacy CPB): subspot Gaussians integrated over CPB cells, then the
//     CPB -> ray area-overlap map.
#include "device_util.cuh"
#include "kernels.h"
#include "launch_util.h"

namespace pbs {

namespace {

constexpr float kConvSigmaCutoff = 3.0f;  // convolution.cu:194
constexpr int kMaxGatherTaps = 1 << 16;   // bound on the gather loop

// xConvGathResampGpu (src/algorithms/convolution.cu:198-228): interm[l][iy][x].
__global__ void conv_x_kernel(BeamGeomDev g, const float* __restrict__ lattice, float* __restrict__ interm,
                              const LayerStateDev* __restrict__ ls, const BeamStateDev* __restrict__ beam) {
    pdl_trigger();
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = blockIdx.z;
    if (iy >= g.latNy || x >= g.rayX) return;
    const float pixelSp = g.cpbResX * beam->pxSpMultX;
    const float inOutDelta = g.latDx / g.cpbResX;
    const float inOutOffset = (g.latOx - g.cpbCornerX) / g.cpbResX;
    const float sigmaEff = ls[l].entrySigmaX / pixelSp;
    const float rSigma = 0.70710678f / sigmaEff;
    const float reach = kConvSigmaCutoff * sigmaEff + 0.5f;
    float res = 0.0f;
    if (inOutDelta > 0.0f && sigmaEff > 0.0f) {
        int i = int(ceilf((float(x) - reach - inOutOffset) / inOutDelta));
        float dist = float(i) * inOutDelta + inOutOffset - float(x);
        const float* row = lattice + (static_cast<size_t>(l) * g.latNy + iy) * g.latNx;
        for (int taps = 0; dist < reach && taps < kMaxGatherTaps; ++taps) {
            if (i >= 0 && i < g.latNx)
                res += 0.5f * (erff((dist + 0.5f) * rSigma) - erff((dist - 0.5f) * rSigma)) * row[i];
            ++i;
            dist = float(i) * inOutDelta + inOutOffset - float(x);
        }
    }
    interm[(static_cast<size_t>(l) * g.latNy + iy) * g.rayX + x] = res;
}

// yConvGathResampGpu (src/algorithms/convolution.cu:231-262): rayW[l][y][x].
__global__ void conv_y_kernel(BeamGeomDev g, const float* __restrict__ interm, float* __restrict__ rayW,
                              const LayerStateDev* __restrict__ ls, const BeamStateDev* __restrict__ beam) {
    pdl_wait();
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int l = blockIdx.z;
    if (x >= g.rayX || y >= g.rayY) return;
    const float pixelSp = g.cpbResY * beam->pxSpMultY;
    const float inOutDelta = g.latDy / g.cpbResY;
    const float inOutOffset = (g.latOy - g.cpbCornerY) / g.cpbResY;
    const float sigmaEff = ls[l].entrySigmaY / pixelSp;
    const float rSigma = 0.70710678f / sigmaEff;
    const float reach = kConvSigmaCutoff * sigmaEff + 0.5f;
    float res = 0.0f;
    if (inOutDelta > 0.0f && sigmaEff > 0.0f) {
        int i = int(ceilf((float(y) - reach - inOutOffset) / inOutDelta));
        float dist = float(i) * inOutDelta + inOutOffset - float(y);
        const float* col = interm + static_cast<size_t>(l) * g.latNy * g.rayX + x;
        for (int taps = 0; dist < reach && taps < kMaxGatherTaps; ++taps) {
            if (i >= 0 && i < g.latNy)
                res += 0.5f * (erff((dist + 0.5f) * rSigma) - erff((dist - 0.5f) * rSigma)) *
                       col[static_cast<size_t>(i) * g.rayX];
            ++i;
            dist = float(i) * inOutDelta + inOutOffset - float(y);
        }
    }
    rayW[(static_cast<size_t>(l) * g.rayY + y) * g.rayX + x] = res;
}

// SubspotInfo (include/core/common.cuh:163-217) read with the legacy gantry frame of
// wrapper.cu:3486-3493: the subspot sits at (dx, -dy) on the reference plane.
// subspotToCPBConvolutionOptimizedKernel (src/algorithms/convolution.cu:95-152)
// with the ranges of calculateSubspotRangeKernel (convolution.cu:45-92).
__global__ void subspot_to_cpb_kernel(BeamGeomDev g, const float* __restrict__ subspots, int maxSubspots,
                                      float* __restrict__ cpb) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    const int l = blockIdx.y;
    if (m >= maxSubspots) return;
    const float* d = subspots + (static_cast<size_t>(l) * maxSubspots + m) * 5;
    const float posX = d[0], posY = -d[1], w = d[2], sx = d[3], sy = d[4];
    if (!(w > 1e-6f) || !(sx > 1e-6f) || !(sy > 1e-6f)) return;
    const int nx = g.rayX, ny = g.rayY;
    const float cx0 = g.cpbCornerX, cy0 = g.cpbCornerY, rx = g.cpbResX, ry = g.cpbResY;
    const int minX = max(0, int(floorf((posX - 3.0f * sx - cx0) / rx)));
    const int maxX = min(nx - 1, int(ceilf((posX + 3.0f * sx - cx0) / rx)));
    const int minY = max(0, int(floorf((posY - 3.0f * sy - cy0) / ry)));
    const int maxY = min(ny - 1, int(ceilf((posY + 3.0f * sy - cy0) / ry)));
    const float dsx = 1.41421356f * sx, dsy = 1.41421356f * sy;
    for (int cy = minY; cy <= maxY; ++cy) {
        const float dy = (cy0 + (float(cy) + 0.5f) * ry) - posY;
        const float ey = erff((dy + 0.5f * ry) / dsy) - erff((dy - 0.5f * ry) / dsy);
        for (int cx = minX; cx <= maxX; ++cx) {
            const float dx = (cx0 + (float(cx) + 0.5f) * rx) - posX;
            const float ex = erff((dx + 0.5f * rx) / dsx) - erff((dx - 0.5f * rx) / dsx);
            atomicAdd(cpb + (static_cast<size_t>(l) * ny + cy) * nx + cx, 0.25f * ex * ey * w);
        }
    }
}

// mapCPBWeightsToRayWeightsKernel (src/algorithms/convolution.cu:269-339); the CPB
// and ray grids coincide in the legacy path (wrapper.cu:3495-3505).
__global__ void cpb_to_ray_kernel(BeamGeomDev g, const float* __restrict__ cpb, float* __restrict__ rayW) {
    const int rx = blockIdx.x * blockDim.x + threadIdx.x;
    const int ry = blockIdx.y * blockDim.y + threadIdx.y;
    const int l = blockIdx.z;
    if (rx >= g.rayX || ry >= g.rayY) return;
    const float resX = g.cpbResX, resY = g.cpbResY, cX = g.cpbCornerX, cY = g.cpbCornerY;
    const float x0 = cX + rx * resX, x1 = x0 + resX;
    const float y0 = cY + ry * resY, y1 = y0 + resY;
    int minX = int(floorf((x0 - cX) / resX)), maxX = int(ceilf((x1 - cX) / resX)) - 1;
    int minY = int(floorf((y0 - cY) / resY)), maxY = int(ceilf((y1 - cY) / resY)) - 1;
    minX = max(minX, 0);
    minY = max(minY, 0);
    maxX = min(maxX, g.rayX - 1);
    maxY = min(maxY, g.rayY - 1);
    const float area = resX * resY;
    float acc = 0.0f;
    if (area > 0.0f && minX <= maxX && minY <= maxY) {
        for (int cy = minY; cy <= maxY; ++cy) {
            const float cy0 = cY + cy * resY, cy1 = cy0 + resY;
            const float oy = fmaxf(0.0f, fminf(y1, cy1) - fmaxf(y0, cy0));
            if (oy <= 0.0f) continue;
            for (int cx = minX; cx <= maxX; ++cx) {
                const float cx0 = cX + cx * resX, cx1 = cx0 + resX;
                const float ox = fmaxf(0.0f, fminf(x1, cx1) - fmaxf(x0, cx0));
                if (ox <= 0.0f) continue;
                acc += cpb[(static_cast<size_t>(l) * g.rayY + cy) * g.rayX + cx] * ((ox * oy) / area);
            }
        }
    }
    rayW[(static_cast<size_t>(l) * g.rayY + ry) * g.rayX + rx] = acc;
}

// Transposes of the two gather passes for the spot-weight adjoint. A forward
// output o takes tap i when i >= ceil((o - reach - off) / delta) and
// dist = i * delta + off - o < reach; the transpose visits, for tap i, the
// outputs o near i * delta + off and applies that same test and weight.
__device__ __forceinline__ float conv_tap(int o, int i, float delta, float off, float reach, float rSigma,
                                          bool& taken) {
    const int i0 = int(ceilf((float(o) - reach - off) / delta));
    const float dist = float(i) * delta + off - float(o);
    taken = i >= i0 && dist < reach;
    return taken ? 0.5f * (erff((dist + 0.5f) * rSigma) - erff((dist - 0.5f) * rSigma)) : 0.0f;
}

// y pass transposed: gradInterm[l][iy][x] = sum_y w(y, iy) * gradRay[l][y][x], where
// gradRay is the ray-weight gradient (rbar / rayW on rays with weight).
__global__ void conv_y_adjoint_kernel(BeamGeomDev g, const float* __restrict__ rbar, const float* __restrict__ rayW,
                                      float* __restrict__ gradInterm, const LayerStateDev* __restrict__ ls,
                                      const BeamStateDev* __restrict__ beam) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    const int l = blockIdx.z;
    if (x >= g.rayX || iy >= g.latNy) return;
    const float pixelSp = g.cpbResY * beam->pxSpMultY;
    const float delta = g.latDy / g.cpbResY;
    const float off = (g.latOy - g.cpbCornerY) / g.cpbResY;
    const float sigmaEff = ls[l].entrySigmaY / pixelSp;
    const float rSigma = 0.70710678f / sigmaEff;
    const float reach = kConvSigmaCutoff * sigmaEff + 0.5f;
    float acc = 0.0f;
    if (delta > 0.0f && sigmaEff > 0.0f) {
        const float c = float(iy) * delta + off;
        const int y0 = max(int(floorf(c - reach)) - 2, 0), y1 = min(int(ceilf(c + reach)) + 2, g.rayY - 1);
        for (int y = y0; y <= y1; ++y) {
            bool taken;
            const float w = conv_tap(y, iy, delta, off, reach, rSigma, taken);
            if (!taken) continue;
            const size_t r = (static_cast<size_t>(l) * g.rayY + y) * g.rayX + x;
            const float rw = rayW[r];
            if (rw > 0.0f) acc += w * (rbar[r] / rw);
        }
    }
    gradInterm[(static_cast<size_t>(l) * g.latNy + iy) * g.rayX + x] = acc;
}

// x pass transposed: gradLattice[l][iy][ix] = sum_x w(x, ix) * gradInterm[l][iy][x].
__global__ void conv_x_adjoint_kernel(BeamGeomDev g, const float* __restrict__ gradInterm,
                                      float* __restrict__ gradLattice, const LayerStateDev* __restrict__ ls,
                                      const BeamStateDev* __restrict__ beam) {
    const int ix = blockIdx.x * blockDim.x + threadIdx.x;
    const int iy = blockIdx.y * blockDim.y + threadIdx.y;
    const int l = blockIdx.z;
    if (ix >= g.latNx || iy >= g.latNy) return;
    const float pixelSp = g.cpbResX * beam->pxSpMultX;
    const float delta = g.latDx / g.cpbResX;
    const float off = (g.latOx - g.cpbCornerX) / g.cpbResX;
    const float sigmaEff = ls[l].entrySigmaX / pixelSp;
    const float rSigma = 0.70710678f / sigmaEff;
    const float reach = kConvSigmaCutoff * sigmaEff + 0.5f;
    float acc = 0.0f;
    if (delta > 0.0f && sigmaEff > 0.0f) {
        const float c = float(ix) * delta + off;
        const int x0 = max(int(floorf(c - reach)) - 2, 0), x1 = min(int(ceilf(c + reach)) + 2, g.rayX - 1);
        const float* row = gradInterm + (static_cast<size_t>(l) * g.latNy + iy) * g.rayX;
        for (int x = x0; x <= x1; ++x) {
            bool taken;
            const float w = conv_tap(x, ix, delta, off, reach, rSigma, taken);
            if (taken) acc += w * row[x];
        }
    }
    gradLattice[(static_cast<size_t>(l) * g.latNy + iy) * g.latNx + ix] = acc;
}

}  // namespace

cudaError_t launch_conv_lattice_adjoint(const BeamGeomDev& g, const float* rbar, const float* rayW, float* gradInterm,
                                        float* gradLattice, const LayerStateDev* ls, const BeamStateDev* beam,
                                        cudaStream_t s) {
    dim3 block(32, 8);
    dim3 gy((g.rayX + 31) / 32, (g.latNy + 7) / 8, g.numLayers);
    conv_y_adjoint_kernel<<<gy, block, 0, s>>>(g, rbar, rayW, gradInterm, ls, beam);
    dim3 gx((g.latNx + 31) / 32, (g.latNy + 7) / 8, g.numLayers);
    conv_x_adjoint_kernel<<<gx, block, 0, s>>>(g, gradInterm, gradLattice, ls, beam);
    return cudaGetLastError();
}

cudaError_t launch_conv_lattice(const BeamGeomDev& g, const float* lattice, float* interm, float* rayW,
                                const LayerStateDev* ls, const BeamStateDev* beam, cudaStream_t s) {
    dim3 block(32, 8);
    dim3 gx((g.rayX + 31) / 32, (g.latNy + 7) / 8, g.numLayers);
    conv_x_kernel<<<gx, block, 0, s>>>(g, lattice, interm, ls, beam);
    dim3 gy((g.rayX + 31) / 32, (g.rayY + 7) / 8, g.numLayers);
    cudaError_t e = launch_pdl(conv_y_kernel, gy, block, 0, s, g, static_cast<const float*>(interm), rayW, ls, beam);
    if (e != cudaSuccess) return e;
    return cudaGetLastError();
}

cudaError_t launch_conv_cpb(const BeamGeomDev& g, const float* subspots, int maxSubspots, float* cpb, float* rayW,
                            cudaStream_t s) {
    const size_t n = static_cast<size_t>(g.rayX) * g.rayY * g.numLayers;
    cudaError_t e = cudaMemsetAsync(cpb, 0, n * sizeof(float), s);
    if (e != cudaSuccess) return e;
    dim3 gs((maxSubspots + 127) / 128, g.numLayers);
    subspot_to_cpb_kernel<<<gs, 128, 0, s>>>(g, subspots, maxSubspots, cpb);
    dim3 block(32, 8);
    dim3 gr((g.rayX + 31) / 32, (g.rayY + 7) / 8, g.numLayers);
    cpb_to_ray_kernel<<<gr, block, 0, s>>>(g, cpb, rayW);
    return cudaGetLastError();
}

}  // namespace pbs
