// Small device helpers shared by several kernels.
#pragma once

#include <cuda_runtime.h>

namespace pbs {

// tex1D with linear filtering, clamp addressing and unnormalised coordinates
// (texel i centred at i + 0.5), evaluated with full-precision weights.
__device__ __forceinline__ float lut_linear_clamp(const float* __restrict__ t, int n, float x) {
    float xb = x - 0.5f;
    xb = fminf(fmaxf(xb, -1.0f), float(n));
    const float fl = floorf(xb);
    const int i = int(fl);
    const float a = xb - fl;
    const int i0 = min(max(i, 0), n - 1);
    const int i1 = min(max(i + 1, 0), n - 1);
    const float v0 = __ldg(t + i0), v1 = __ldg(t + i1);
    return v0 + (v1 - v0) * a;
}

// Unsigned key with the order of the float values (negative floats reversed).
__device__ __forceinline__ unsigned float_order_key(float v) {
    const unsigned b = __float_as_uint(v);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float float_from_order_key(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// Same lookup on a table staged in shared memory.
__device__ __forceinline__ float lut_linear_clamp_smem(const float* t, int n, float x) {
    float xb = x - 0.5f;
    xb = fminf(fmaxf(xb, -1.0f), float(n));
    const float fl = floorf(xb);
    const int i = int(fl);
    const float a = xb - fl;
    const int i0 = min(max(i, 0), n - 1);
    const int i1 = min(max(i + 1, 0), n - 1);
    const float v0 = t[i0], v1 = t[i1];
    return v0 + (v1 - v0) * a;
}

// Radius bucket of a tile from its minimum rSigmaEff (complete_superposition.cu:242):
// min(int(3 / (sqrt(2) * min) + 0.5), 33), with IEEE division.
__device__ __forceinline__ int tile_radius_bucket(float minRSigma) {
    const float q = __fadd_rn(__fdiv_rn(3.0f, __fmul_rn(1.41421354f, minRSigma)), 0.5f);
    if (!(q < 34.0f)) return (q != q) ? 0 : 33;
    return min(int(q), 33);
}

}  // namespace pbs
