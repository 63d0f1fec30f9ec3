// Beam geometry shared by the host planner and the device kernels.
//
// Every operation is written with explicit round-to-nearest float helpers so the
// host planner, the on-device beam planner and the reference's host code (which
// runs on x86 without FMA contraction) produce bit-identical coordinates. The
// integer decisions downstream (ray-grid sizes, tracer step counts, transfer
// bounding boxes) depend on these values.
//
// Semantics follow the reference:
//   Matrix3x3              include/algorithms/matrix_3x3.h:17-103
//   Float3AffineTransform  include/algorithms/float3_affine_transform.h:20-62
//   Float3IdxTransform     include/algorithms/float3_idx_transform.h:16-51
//   Float3FromFanTransform include/algorithms/fan_transforms.h:24-57
//   Float3ToFanTransform   include/algorithms/fan_transforms.h:62-95
//   DensityAndSpTracerParams include/core/ray_tracing.h:27-92
//   TransferParamStructDiv3  include/algorithms/transfer_param_struct_div3.cuh:19-46
//                            src/algorithms/transfer_param_struct_div3_impl.cu:13-34
#pragma once

#include <math.h>

#if defined(__CUDACC__)
#define PBS_HD __host__ __device__ __forceinline__
#else
#define PBS_HD inline
#endif

namespace pbs {

constexpr int kTileX = 32;               // SUPERP_TILE_X, include/core/Macro.cuh:65
constexpr int kTileY = 8;                // SUPERP_TILE_Y, include/core/Macro.cuh:66
constexpr int kMaxR = 32;                // MAX_SUPERP_RADIUS, include/core/Macro.cuh:64
constexpr int kSplitR = 15;              // radii <= kSplitR run in the medium and narrow superposition instances
constexpr int kSplitR2 = 7;              // radii <= kSplitR2 run in the narrow instance
// Up to kMergeLayers layers of one tile at one step with the same radius (<= kSplitR)
// share one superposition item: their footprints land on the same BEV cells.
constexpr int kMergeLayers = 4;
constexpr int kMinTilesInBatch = 16;     // MIN_TILES_IN_BATCH, include/core/Macro.cuh:67
constexpr float kBpDepthCutoff = 1.05f;  // BP_DEPTH_CUTOFF, include/core/Macro.cuh:46

// Round-to-nearest float arithmetic without contraction into FMA.
PBS_HD float fadd(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fadd_rn(a, b);
#else
    return a + b;
#endif
}
PBS_HD float fsub(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fsub_rn(a, b);
#else
    return a - b;
#endif
}
PBS_HD float fmul(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fmul_rn(a, b);
#else
    return a * b;
#endif
}
PBS_HD float fdiv(float a, float b) {
#if defined(__CUDA_ARCH__)
    return __fdiv_rn(a, b);
#else
    return a / b;
#endif
}
PBS_HD float fsqrt(float a) {
#if defined(__CUDA_ARCH__)
    return __fsqrt_rn(a);
#else
    return sqrtf(a);
#endif
}

struct V2 {
    float x, y;
};
struct V3 {
    float x, y, z;
};
struct I3 {
    int x, y, z;
};

PBS_HD V2 v2(float x, float y) { V2 r; r.x = x; r.y = y; return r; }
PBS_HD V3 v3(float x, float y, float z) { V3 r; r.x = x; r.y = y; r.z = z; return r; }
PBS_HD V3 v3s(float s) { return v3(s, s, s); }
PBS_HD I3 i3(int x, int y, int z) { I3 r; r.x = x; r.y = y; r.z = z; return r; }

PBS_HD V3 add(V3 a, V3 b) { return v3(fadd(a.x, b.x), fadd(a.y, b.y), fadd(a.z, b.z)); }
PBS_HD V3 sub(V3 a, V3 b) { return v3(fsub(a.x, b.x), fsub(a.y, b.y), fsub(a.z, b.z)); }
PBS_HD V3 scale(V3 a, float s) { return v3(fmul(a.x, s), fmul(a.y, s), fmul(a.z, s)); }
PBS_HD V3 hadamard(V3 a, V3 b) { return v3(fmul(a.x, b.x), fmul(a.y, b.y), fmul(a.z, b.z)); }
PBS_HD V3 divs(V3 a, float s) { return v3(fdiv(a.x, s), fdiv(a.y, s), fdiv(a.z, s)); }
// Left-to-right sum of products, as the reference's dot() evaluates it.
PBS_HD float dot(V3 a, V3 b) { return fadd(fadd(fmul(a.x, b.x), fmul(a.y, b.y)), fmul(a.z, b.z)); }
PBS_HD V3 cross(V3 a, V3 b) {
    return v3(fsub(fmul(a.y, b.z), fmul(a.z, b.y)),
              fsub(fmul(a.z, b.x), fmul(a.x, b.z)),
              fsub(fmul(a.x, b.y), fmul(a.y, b.x)));
}

// Row-major 3x3 matrix.
struct M3 {
    V3 r0, r1, r2;
};

PBS_HD M3 m3(V3 a, V3 b, V3 c) { M3 m; m.r0 = a; m.r1 = b; m.r2 = c; return m; }
PBS_HD M3 m3diag(float a, float b, float c) { return m3(v3(a, 0.f, 0.f), v3(0.f, b, 0.f), v3(0.f, 0.f, c)); }
PBS_HD M3 transpose(M3 m) {
    return m3(v3(m.r0.x, m.r1.x, m.r2.x), v3(m.r0.y, m.r1.y, m.r2.y), v3(m.r0.z, m.r1.z, m.r2.z));
}
PBS_HD V3 mulv(M3 m, V3 a) { return v3(dot(m.r0, a), dot(m.r1, a), dot(m.r2, a)); }
// Matrix product evaluated as row . column with the right factor transposed.
PBS_HD M3 mulm(M3 a, M3 b) {
    M3 t = transpose(b);
    return m3(v3(dot(a.r0, t.r0), dot(a.r0, t.r1), dot(a.r0, t.r2)),
              v3(dot(a.r1, t.r0), dot(a.r1, t.r1), dot(a.r1, t.r2)),
              v3(dot(a.r2, t.r0), dot(a.r2, t.r1), dot(a.r2, t.r2)));
}
PBS_HD float det(M3 m) {
    const V3 a = m.r0, b = m.r1, c = m.r2;
    return fadd(fsub(fmul(a.x, fsub(fmul(b.y, c.z), fmul(b.z, c.y))),
                     fmul(a.y, fsub(fmul(b.x, c.z), fmul(b.z, c.x)))),
                fmul(a.z, fsub(fmul(b.x, c.y), fmul(b.y, c.x))));
}
// Adjugate times (1/det), the product taken as a matrix product with s*I.
PBS_HD M3 inverse(M3 m) {
    const float s = fdiv(1.0f, det(m));
    const V3 a = m.r0, b = m.r1, c = m.r2;
    M3 adj = m3(v3(fsub(fmul(b.y, c.z), fmul(b.z, c.y)), fsub(fmul(a.z, c.y), fmul(a.y, c.z)),
                   fsub(fmul(a.y, b.z), fmul(a.z, b.y))),
                v3(fsub(fmul(b.z, c.x), fmul(b.x, c.z)), fsub(fmul(a.x, c.z), fmul(a.z, c.x)),
                   fsub(fmul(a.z, b.x), fmul(a.x, b.z))),
                v3(fsub(fmul(b.x, c.y), fmul(b.y, c.x)), fsub(fmul(a.y, c.x), fmul(a.x, c.y)),
                   fsub(fmul(a.x, b.y), fmul(a.y, b.x))));
    return mulm(adj, m3diag(s, s, s));
}

// out = M * in + v
struct Affine {
    M3 m;
    V3 v;
};
PBS_HD Affine affine(M3 m, V3 v) { Affine a; a.m = m; a.v = v; return a; }
PBS_HD V3 apply(Affine a, V3 p) { return add(mulv(a.m, p), a.v); }
PBS_HD Affine inverse(Affine a) {
    const M3 mi = inverse(a.m);
    return affine(mi, mulv(mi, scale(a.v, -1.0f)));
}
// Apply `first`, then `second`.
PBS_HD Affine concat(Affine first, Affine second) {
    return affine(mulm(second.m, first.m), add(mulv(second.m, first.v), second.v));
}

// out = in (*) delta + offset, element-wise.
struct IdxXf {
    V3 delta;
    V3 offset;
};
PBS_HD IdxXf idxxf(V3 d, V3 o) { IdxXf t; t.delta = d; t.offset = o; return t; }
PBS_HD V3 apply(IdxXf t, V3 p) { return add(hadamard(p, t.delta), t.offset); }
PBS_HD IdxXf inverse(IdxXf t) {
    const V3 inv = v3(fdiv(1.0f, t.delta.x), fdiv(1.0f, t.delta.y), fdiv(1.0f, t.delta.z));
    return idxxf(inv, v3(fmul(-t.offset.x, inv.x), fmul(-t.offset.y, inv.y), fmul(-t.offset.z, inv.z)));
}

// Fan index -> image (or dose) index: idx -> fan coords, divergence, gantry -> index.
struct FromFan {
    IdxXf fanIdxToFan;
    Affine gantryToIdx;
    V2 dist;
};
PBS_HD V3 apply(FromFan f, V3 fanIdx) {
    V3 g = apply(f.fanIdxToFan, fanIdx);
    g.x = fmul(g.x, fsub(1.0f, fdiv(g.z, f.dist.x)));
    g.y = fmul(g.y, fsub(1.0f, fdiv(g.z, f.dist.y)));
    return apply(f.gantryToIdx, g);
}

// Image (or dose) index -> fan index.
struct ToFan {
    Affine idxToGantry;
    V2 dist;
    IdxXf fanToFanIdx;
};
PBS_HD V3 apply(ToFan f, V3 idx) {
    V3 g = apply(f.idxToGantry, idx);
    g.x = fdiv(g.x, fsub(1.0f, fdiv(g.z, f.dist.x)));
    g.y = fdiv(g.y, fsub(1.0f, fdiv(g.z, f.dist.y)));
    return apply(f.fanToFanIdx, g);
}
PBS_HD ToFan invert_and_shift(FromFan f, V3 shift) {
    ToFan t;
    t.idxToGantry = inverse(f.gantryToIdx);
    t.dist = f.dist;
    IdxXf inv = inverse(f.fanIdxToFan);
    inv.offset = add(inv.offset, shift);
    t.fanToFanIdx = inv;
    return t;
}

// Per-ray start point, step increment and step length of the divergent tracer.
struct TracerParams {
    float densityScale;
    float spScale;
    int steps;
    V3 coefOffset, coefIdxI, coefIdxJ, transl;
    V3 corner, delta;
    V2 dist;
};
PBS_HD TracerParams make_tracer_params(float densityScale, float spScale, int steps, FromFan f) {
    TracerParams p;
    p.densityScale = densityScale;
    p.spScale = spScale;
    p.steps = steps;
    p.dist = f.dist;
    p.corner = f.fanIdxToFan.offset;
    p.delta = f.fanIdxToFan.delta;
    const M3 t = transpose(f.gantryToIdx.m);
    p.coefOffset = sub(sub(t.r2, scale(t.r0, fdiv(p.corner.x, p.dist.x))), scale(t.r1, fdiv(p.corner.y, p.dist.y)));
    p.coefIdxI = scale(t.r0, p.delta.x);
    p.coefIdxJ = scale(t.r1, p.delta.y);
    p.transl = add(add(add(f.gantryToIdx.v, scale(t.r2, p.corner.z)),
                       scale(t.r0, fmul(p.corner.x, fsub(1.0f, fdiv(p.corner.z, p.dist.x))))),
                   scale(t.r1, fmul(p.corner.y, fsub(1.0f, fdiv(p.corner.z, p.dist.y)))));
    return p;
}
PBS_HD V3 tracer_start(const TracerParams& p, int i, int j) {
    return add(add(scale(p.coefIdxI, fmul(float(i), fsub(1.0f, fdiv(p.corner.z, p.dist.x)))),
                   scale(p.coefIdxJ, fmul(float(j), fsub(1.0f, fdiv(p.corner.z, p.dist.y))))),
               p.transl);
}
PBS_HD V3 tracer_inc(const TracerParams& p, int i, int j) {
    return scale(sub(sub(p.coefOffset, scale(p.coefIdxI, fdiv(float(i), p.dist.x))),
                     scale(p.coefIdxJ, fdiv(float(j), p.dist.y))),
                 p.delta.z);
}
PBS_HD float tracer_step_len(const TracerParams& p, int i, int j) {
    const float dx = fdiv(fadd(p.corner.x, fmul(float(i), p.delta.x)), p.dist.x);
    const float dy = fdiv(fadd(p.corner.y, fmul(float(j), p.delta.y)), p.dist.y);
    return fmul(fabsf(p.delta.z), fsqrt(fadd(fadd(1.0f, fmul(dx, dx)), fmul(dy, dy))));
}

// Dose index -> BEV (fan) index used by the transfer.
struct TransferParams {
    V3 globalOffset, coefOffset, coefIdxI, coefIdxJ, inc;
    V2 normDist;
};
PBS_HD TransferParams make_transfer_params(ToFan t) {
    TransferParams p;
    const M3 tt = transpose(t.idxToGantry.m);
    const V3 delta = t.fanToFanIdx.delta;
    p.coefIdxI = hadamard(tt.r0, delta);
    p.coefIdxJ = hadamard(tt.r1, delta);
    p.coefOffset = hadamard(t.idxToGantry.v, delta);
    p.globalOffset = t.fanToFanIdx.offset;
    p.inc = hadamard(tt.r2, delta);
    p.normDist = v2(fmul(delta.z, t.dist.x), fmul(delta.z, t.dist.y));
    return p;
}
PBS_HD V3 transfer_start(const TransferParams& p, int i, int j) {
    return add(add(hadamard(v3s(float(i)), p.coefIdxI), hadamard(v3s(float(j)), p.coefIdxJ)), p.coefOffset);
}
PBS_HD V3 transfer_fan_idx(const TransferParams& p, V3 start, int k) {
    V3 r = add(start, hadamard(v3s(float(k)), p.inc));
    r.x = fmul(r.x, fadd(1.0f, fdiv(r.z, fsub(p.normDist.x, r.z))));
    r.y = fmul(r.y, fadd(1.0f, fdiv(r.z, fsub(p.normDist.y, r.z))));
    return add(r, p.globalOffset);
}

}  // namespace pbs
