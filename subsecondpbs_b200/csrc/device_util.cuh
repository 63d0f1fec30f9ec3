// Small device helpers shared by several kernels.
#pragma once

#include <cuda_runtime.h>

namespace pbs {

// Programmatic dependent launch: a kernel launched with launch_pdl calls pdl_wait()
// first (its predecessor on the stream has completed and its writes are visible); a
// kernel that may precede one calls pdl_trigger() to let it be scheduled early.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_trigger() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }

// tex1D with linear filtering, clamp addressing and unnormalised coordinates
// (texel i centred at i + 0.5), evaluated with full-precision weights. The texel
// coordinate is clamped to [0, n - 1] before the split into index and weight: below
// the table and past its end the filter returns the edge texel either way (the two
// taps coincide or the weight is 0), and a NaN coordinate gives texel 0.
__device__ __forceinline__ float lut_linear_clamp(const float* __restrict__ t, int n, float x) {
    const float xb = fminf(fmaxf(x - 0.5f, 0.0f), float(n - 1));
    const float fl = floorf(xb);
    const int i0 = int(fl);
    const int i1 = min(i0 + 1, n - 1);
    const float a = xb - fl;
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
    const float xb = fminf(fmaxf(x - 0.5f, 0.0f), float(n - 1));
    const float fl = floorf(xb);
    const int i0 = int(fl);
    const int i1 = min(i0 + 1, n - 1);
    const float a = xb - fl;
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

// erf(x), x >= 0, from Abramowitz & Stegun 7.1.26 (Hastings' rational
// approximation, |error| <= 1.5e-7): 1 - t (a1 + t (a2 + t (a3 + t (a4 + t a5)))) e^{-x^2}
// with t = 1 / (1 + p x). The caller supplies e^{-x^2}.
__device__ __forceinline__ float erf_hastings(float x, float expNegX2) {
    constexpr float p = 0.3275911f;
    constexpr float a1 = 0.254829592f, a2 = -0.284496736f, a3 = 1.421413741f, a4 = -1.453152027f,
                    a5 = 1.061405429f;
    const float t = __fdividef(1.0f, fmaf(p, x, 1.0f));
    const float poly = t * fmaf(t, fmaf(t, fmaf(t, fmaf(t, a5, a4), a3), a2), a1);
    return fmaf(-poly, expNegX2, 1.0f);
}

// Superposition weights of one source (complete_superposition.cu:298-307):
// e[0] = erf(r/2), e[k] = (erf((k+1/2) r) - erf((k-1/2) r)) / 2 for k = 1..R. The
// factor e^{-((k+1/2) r)^2} follows E_{k+1} = E_k G_k, G_k = e^{-2 (k+1) r^2}.
template <int R>
__device__ __forceinline__ void superposition_row(float rs, float (&e)[R + 1]) {
    const float r2 = rs * rs;
    const float step2 = __expf(-2.0f * r2);
    float E = __expf(-0.25f * r2);
    float G = step2;
    float fPrev = erf_hastings(rs * 0.5f, E);
    e[0] = fPrev;
#pragma unroll
    for (int k = 1; k <= R; ++k) {
        E *= G;
        G *= step2;
        const float f = erf_hastings(rs * (float(k) + 0.5f), E);
        e[k] = 0.5f * (f - fPrev);
        fPrev = f;
    }
}

}  // namespace pbs
