/*
 * CPU oracle of the pencil-beam dose path - test infrastructure only.
 * See oracle.h for scope. Compiled with -ffp-contract=off so single-precision
 * geometry is evaluated exactly as written. Reference citations are paths within
 * Nelgcis/subsecondPBS.
 */
#include "oracle.h"

#include <float.h>
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static char g_err[512];
const char* oracle_last_error(void) { return g_err; }
static int fail(int code, const char* msg) {
    snprintf(g_err, sizeof g_err, "%s", msg);
    return code;
}

#define INF20F ((float)1.0e20) /* Macro.cuh:7 INF stored in a float */
#define TILE_X 32
#define TILE_Y 8
#define MAX_R 32
#define MIN_TILES_IN_BATCH 16
#define BP_CUT 1.05f

/* ---- single-precision geometry (headers under include/algorithms) ---------- */
typedef struct { float x, y, z; } V3;
typedef struct { float x, y; } V2;
typedef struct { V3 r0, r1, r2; } M3;
typedef struct { M3 m; V3 v; } Aff;
typedef struct { V3 delta, offset; } IdxT;
typedef struct { IdxT fan; Aff g; V2 dist; } FromFan;
typedef struct { Aff g; V2 dist; IdxT fan; } ToFan;

static V3 v3(float x, float y, float z) { V3 r = {x, y, z}; return r; }
static V3 vadd(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
static V3 vsub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
static V3 vmul(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
static V3 vhad(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
static V3 vdiv(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
static float vdot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static V3 vcross(V3 a, V3 b) { return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static V3 vnorm_safe(V3 v) { /* raytracedicom_wrapper.cu:2862-2866 */
    float len = sqrtf(vdot(v, v));
    if (len > 1e-8f) v = vdiv(v, len);
    return v;
}
static M3 m3(V3 a, V3 b, V3 c) { M3 m = {a, b, c}; return m; }
static M3 mT(M3 m) { return m3(v3(m.r0.x, m.r1.x, m.r2.x), v3(m.r0.y, m.r1.y, m.r2.y), v3(m.r0.z, m.r1.z, m.r2.z)); }
static V3 mv(M3 m, V3 a) { return v3(vdot(m.r0, a), vdot(m.r1, a), vdot(m.r2, a)); }
static M3 mm(M3 a, M3 b) { /* matrix_3x3.h:64-73 */
    M3 t = mT(b);
    return m3(v3(vdot(a.r0, t.r0), vdot(a.r0, t.r1), vdot(a.r0, t.r2)),
              v3(vdot(a.r1, t.r0), vdot(a.r1, t.r1), vdot(a.r1, t.r2)),
              v3(vdot(a.r2, t.r0), vdot(a.r2, t.r1), vdot(a.r2, t.r2)));
}
static M3 mdiag(float a, float b, float c) { return m3(v3(a, 0, 0), v3(0, b, 0), v3(0, 0, c)); }
static M3 minv(M3 m) { /* matrix_3x3.h:78-93 */
    V3 a = m.r0, b = m.r1, c = m.r2;
    float det = a.x * (b.y * c.z - b.z * c.y) - a.y * (b.x * c.z - b.z * c.x) + a.z * (b.x * c.y - b.y * c.x);
    float s = 1.0f / det;
    M3 adj = m3(v3(b.y * c.z - b.z * c.y, a.z * c.y - a.y * c.z, a.y * b.z - a.z * b.y),
                v3(b.z * c.x - b.x * c.z, a.x * c.z - a.z * c.x, a.z * b.x - a.x * b.z),
                v3(b.x * c.y - b.y * c.x, a.y * c.x - a.x * c.y, a.x * b.y - a.y * b.x));
    return mm(adj, mdiag(s, s, s));
}
static Aff aff(M3 m, V3 v) { Aff a = {m, v}; return a; }
static V3 aapply(Aff a, V3 p) { return vadd(mv(a.m, p), a.v); }
static Aff ainv(Aff a) { /* float3_affine_transform.h:37-40 */
    M3 mi = minv(a.m);
    return aff(mi, mv(mi, vmul(a.v, -1.0f)));
}
static Aff aconcat(Aff first, Aff second) { /* float3_affine_transform.h:57-62 */
    return aff(mm(second.m, first.m), vadd(mv(second.m, first.v), second.v));
}
static IdxT idxt(V3 d, V3 o) { IdxT t = {d, o}; return t; }
static V3 iapply(IdxT t, V3 p) { return vadd(vhad(p, t.delta), t.offset); }
static IdxT iinv(IdxT t) { /* float3_idx_transform.h:34-38 */
    V3 inv = v3(1.0f / t.delta.x, 1.0f / t.delta.y, 1.0f / t.delta.z);
    return idxt(inv, v3(-t.offset.x * inv.x, -t.offset.y * inv.y, -t.offset.z * inv.z));
}
static V3 ffapply(FromFan f, V3 p) { /* fan_transforms.h:39-50 */
    V3 g = iapply(f.fan, p);
    g.x *= (1.0f - g.z / f.dist.x);
    g.y *= (1.0f - g.z / f.dist.y);
    return aapply(f.g, g);
}
static ToFan ff_invert_shift(FromFan f, V3 shift) { /* fan_transforms.h:103-106 */
    ToFan t;
    t.g = ainv(f.g);
    t.dist = f.dist;
    t.fan = iinv(f.fan);
    t.fan.offset = vadd(t.fan.offset, shift);
    return t;
}

/* DensityAndSpTracerParams (include/core/ray_tracing.h:48-87). */
typedef struct { V3 coefOffset, coefIdxI, coefIdxJ, transl, corner, delta; V2 dist; } TracerP;
static TracerP tracer_params(FromFan f) {
    TracerP p;
    p.dist = f.dist;
    p.corner = f.fan.offset;
    p.delta = f.fan.delta;
    M3 t = mT(f.g.m);
    p.coefOffset = vsub(vsub(t.r2, vmul(t.r0, p.corner.x / p.dist.x)), vmul(t.r1, p.corner.y / p.dist.y));
    p.coefIdxI = vmul(t.r0, p.delta.x);
    p.coefIdxJ = vmul(t.r1, p.delta.y);
    p.transl = vadd(vadd(vadd(f.g.v, vmul(t.r2, p.corner.z)),
                         vmul(t.r0, p.corner.x * (1.0f - p.corner.z / p.dist.x))),
                    vmul(t.r1, p.corner.y * (1.0f - p.corner.z / p.dist.y)));
    return p;
}
static V3 tr_start(const TracerP* p, int i, int j) {
    return vadd(vadd(vmul(p->coefIdxI, (float)i * (1.0f - p->corner.z / p->dist.x)),
                     vmul(p->coefIdxJ, (float)j * (1.0f - p->corner.z / p->dist.y))),
                p->transl);
}
static V3 tr_inc(const TracerP* p, int i, int j) {
    return vmul(vsub(vsub(p->coefOffset, vmul(p->coefIdxI, (float)i / p->dist.x)), vmul(p->coefIdxJ, (float)j / p->dist.y)),
                p->delta.z);
}
static float tr_steplen(const TracerP* p, int i, int j) {
    float dx = (p->corner.x + (float)i * p->delta.x) / p->dist.x;
    float dy = (p->corner.y + (float)j * p->delta.y) / p->dist.y;
    return fabsf(p->delta.z) * sqrtf(1.0f + dx * dx + dy * dy);
}

/* TransferParamStructDiv3 (transfer_param_struct_div3.cuh:19-46, _impl.cu:13-34). */
typedef struct { V3 globalOffset, coefOffset, coefIdxI, coefIdxJ, inc; V2 normDist; } TransferP;
static TransferP transfer_params(ToFan t) {
    TransferP p;
    M3 tt = mT(t.g.m);
    V3 d = t.fan.delta;
    p.coefIdxI = vhad(tt.r0, d);
    p.coefIdxJ = vhad(tt.r1, d);
    p.coefOffset = vhad(t.g.v, d);
    p.globalOffset = t.fan.offset;
    p.inc = vhad(tt.r2, d);
    p.normDist.x = d.z * t.dist.x;
    p.normDist.y = d.z * t.dist.y;
    return p;
}
static V3 tp_fan(const TransferP* p, int i, int j, int k) {
    V3 s = vadd(vadd(vhad(v3((float)i, (float)i, (float)i), p->coefIdxI), vhad(v3((float)j, (float)j, (float)j), p->coefIdxJ)),
                p->coefOffset);
    V3 r = vadd(s, vhad(v3((float)k, (float)k, (float)k), p->inc));
    r.x *= 1 + r.z / (p->normDist.x - r.z);
    r.y *= 1 + r.z / (p->normDist.y - r.z);
    return vadd(r, p->globalOffset);
}

/* ---- reference host helpers ------------------------------------------------ */
/* include/utils/vector_find.h:61-82 (float values). */
static int ffl_f(const float* v, int n, float value) {
    int upper = n - 1, lower = 0;
    if (v[n - 1] <= value) return upper;
    if (v[0] > value) return 0;
    while (upper - lower > 1) {
        int pivot = (upper + lower) / 2;
        if (v[pivot] <= value) lower = pivot; else upper = pivot;
    }
    return lower + 1;
}
/* Same search over double values compared against a float threshold. */
static int ffl_d(const double* v, int n, float value) {
    int upper = n - 1, lower = 0;
    if (v[n - 1] <= (double)value) return upper;
    if (v[0] > (double)value) return 0;
    while (upper - lower > 1) {
        int pivot = (upper + lower) / 2;
        if (v[pivot] <= (double)value) lower = pivot; else upper = pivot;
    }
    return lower + 1;
}
/* vector_find.h:94-110, 129-144 */
static float find_decimal(const float* v, int n, float value) {
    if (value >= v[n - 1]) return (float)(n - 1);
    if (value < v[0]) return 0.0f;
    int upper = n - 1, lower = 0;
    if (v[n - 1] <= value) lower = upper;
    else {
        while (upper - lower > 1) {
            int pivot = (upper + lower) / 2;
            if (v[pivot] <= value) lower = pivot; else upper = pivot;
        }
    }
    unsigned f = (unsigned)lower;
    float corr = (value - v[f]) / (v[f + 1] - v[f]);
    return (float)f + corr;
}
/* vector_interpolate.h:19-31 */
static float vinterp(const float* v, int n, float idx) {
    if (idx <= 0.0f) return v[0];
    if (idx >= (float)(n - 1)) return v[n - 1];
    float ip;
    float dec = modff(idx, &ip);
    unsigned f = (unsigned)ip;
    return v[f] + (v[f + 1] - v[f]) * dec;
}

/* Optional emulation of the texture unit's interpolation weights, which hardware
 * stores as 9-bit fixed point with 8 fractional bits (CUDA programming guide,
 * texture fetching appendix). 0 = exact weights (default). */
static int g_texq = 0;
static double texw(double a) { return g_texq == 1 ? rint(a * 256.0) / 256.0 : (g_texq == 2 ? floor(a * 256.0) / 256.0 : a); }
void oracle_set_texture_quantization(int on) { g_texq = on; }

static float frac_index_monotonic(const float* v, int n, float value);

/* CarbonPBS lateral profile model (off by default, as in the reference): bit 1
 * overrideRSigmaFromCarbonProfileKernel (raytracedicom_wrapper.cu:2080-2152), bit 2
 * applyCarbonProfileOverallWeightKernel (raytracedicom_wrapper.cu:2154-2187). */
static int g_profile = 0;
void oracle_set_carbon_profile(int mode) { g_profile = mode; }

typedef struct ProfileC {
    int table, beamPara, rows, depthN, channels;
    float depth0, depthStep;
} ProfileC;

/* Table shape the reference infers (raytracedicom_wrapper.cu:2816-2862). */
static void profile_shape(const PbsBeamDesc* b, int L, ProfileC* o) {
    memset(o, 0, sizeof(*o));
    const size_t nData = b->profile_data ? b->n_profile_data : 0;
    const size_t nPara = b->beam_para_data ? b->n_beam_para_data : 0;
    const size_t nProfE = b->profile_energies ? b->n_profile_energies : 0;
    o->beamPara = nPara >= (size_t)L * 3u;
    if (!(b->profile_setting && b->n_profile_setting >= 3 && lroundf(b->profile_setting[2]) > 0 && nData > 0)) return;
    o->depth0 = b->profile_setting[0];
    o->depthStep = b->profile_setting[1];
    o->depthN = (int)lroundf(b->profile_setting[2]);
    if (o->depthN < 1) o->depthN = 1;
    const size_t plane = (size_t)o->depthN;
    const int paraRows = (int)(nPara / 3u);
    if (paraRows > 0 && nPara == (size_t)paraRows * 3u && nData % ((size_t)paraRows * plane) == 0)
        o->rows = paraRows;
    else if (nProfE > 0 && nData % (nProfE * plane) == 0)
        o->rows = (int)nProfE;
    else if (L > 0 && nData % ((size_t)L * plane) == 0)
        o->rows = L;
    else if (nData % plane == 0 && (nData / plane) % 11u == 0)
        o->rows = (int)((nData / plane) / 11u);
    const size_t perRow = o->rows > 0 ? nData / (size_t)o->rows : 0;
    if (o->rows > 0 && perRow >= plane) {
        o->channels = (int)(perRow / plane);
        o->table = o->channels > 0 && (size_t)o->rows * plane * (size_t)o->channels == nData;
    }
}

/* Fractional table row of layer l (raytracedicom_wrapper.cu:4577-4590). */
static float profile_row(const PbsBeamDesc* b, const PbsEnergyDesc* e, const ProfileC* pc, int L, int l, float eIdx) {
    const int lastRow = pc->rows - 1 > 0 ? pc->rows - 1 : 0;
    const size_t nProfE = b->profile_energies ? b->n_profile_energies : 0;
    float r;
    if (pc->rows == L)
        r = (float)l;
    else if (nProfE > 0 && pc->rows == (int)nProfE)
        r = frac_index_monotonic(b->profile_energies, (int)nProfE, b->energies[l]);
    else if (pc->rows == e->n_energies && e->energies_per_u && e->n_energies_per_u > 0)
        r = fminf(fmaxf(eIdx, 0.0f), (float)(pc->rows - 1));
    else
        r = fminf(fmaxf((float)l, 0.0f), (float)lastRow);
    return fminf(fmaxf(r, 0.0f), (float)lastRow);
}

/* Linear filter of the profile texture at channel c, depth index d, row index r
 * (both clamped to the table), in double. */
static double profile_at(const float* t, const ProfileC* pc, int c, double d, double r) {
    double fd = floor(d), fr = floor(r);
    int d0 = (int)fd, r0 = (int)fr;
    int d1 = d0 + 1 < pc->depthN ? d0 + 1 : pc->depthN - 1, r1 = r0 + 1 < pc->rows ? r0 + 1 : pc->rows - 1;
    double ad = texw(d - fd), ar = texw(r - fr);
    double a0 = t[((size_t)r0 * pc->depthN + d0) * pc->channels + c], a1 = t[((size_t)r0 * pc->depthN + d1) * pc->channels + c];
    double b0 = t[((size_t)r1 * pc->depthN + d0) * pc->channels + c], b1 = t[((size_t)r1 * pc->depthN + d1) * pc->channels + c];
    double lo = a0 + (a1 - a0) * ad, hi = b0 + (b1 - b0) * ad;
    return lo + (hi - lo) * ar;
}

/* Biological model (pbs_context_set_bio_model): when set, every layer's IDD is
 * also scaled by the steps' biological factors, superposed and transferred into
 * the accumulators [4][Z][Y][X]: dose, dose x alpha (LQ) or z1D (MKM), dose x
 * sqrt(beta) (LQ), dose x LET. */
static const PbsBioModel* g_bio = NULL;
static double* g_bioAcc = NULL;
void oracle_set_bio(const PbsBioModel* m, double* acc) {
    g_bio = (m && m->model != PBS_BIO_OFF) ? m : NULL;
    g_bioAcc = acc;
}

static double table_at_d(const float* t, int n, double x) {
    if (x < 0.0) x = 0.0;
    if (x > n - 1) x = n - 1;
    double f = floor(x);
    int i0 = (int)f, i1 = i0 + 1 < n ? i0 + 1 : n - 1;
    return t[i0] + ((double)t[i1] - t[i0]) * (x - f);
}

/* Dose-averaged LET of a step over the model's depth samples (deviceCalDose.cu:686-692). */
static double bio_let(const PbsBioModel* m, double row, double weq) {
    if (row < 0.0) row = 0.0;
    if (row > m->let_rows - 1) row = m->let_rows - 1;
    double fr = floor(row);
    int r0 = (int)fr, r1 = r0 + 1 < m->let_rows ? r0 + 1 : m->let_rows - 1;
    double ar = row - fr, s1 = 0.0, s2 = 0.0;
    for (int j = 0; j < m->let_samples; ++j) {
        double depth = weq + m->range_shifter + (j - 0.5 * (m->let_samples - 1)) * m->est_dimension / m->let_samples;
        double x = (depth - m->let_depth0) / m->let_depth_step;
        double a = table_at_d(m->let_table + (size_t)r0 * m->let_depths, m->let_depths, x);
        double b = table_at_d(m->let_table + (size_t)r1 * m->let_depths, m->let_depths, x);
        double t = a + (b - a) * ar;
        s1 += t;
        s2 += t * t;
    }
    return s1 > 0.0 ? s2 / s1 : 0.0;
}

/* Factor of channel c (0: alpha or z1D, 1: sqrt(beta), 2: LET) at LET `let`. */
static double bio_factor(const PbsBioModel* m, int c, double let) {
    if (c == 2) return let;
    double li = let > 0.0 ? (log10(let) - m->lq_log0) / m->lq_log_step : 0.0;
    if (m->model == PBS_BIO_MKM) return table_at_d(m->z1d, m->n_lq, li);
    if (c == 0) return table_at_d(m->lq_alpha, m->n_lq, li);
    double b = table_at_d(m->lq_beta, m->n_lq, li);
    return sqrt(b > 0.0 ? b : 0.0);
}

/* The maps of pbs_context_read_bio_map from the accumulators (LQRBEKernel,
 * deviceCalDose.cu:738-772; mkmRBEMapKernel, :1060-1126). */
void oracle_bio_map(const PbsBioModel* m, const double* acc, size_t n, int map, double* out) {
    const double *D = acc, *c0 = acc + n, *c1 = acc + 2 * n, *c2 = acc + 3 * n;
    for (size_t i = 0; i < n; ++i) {
        double d = D[i], v = 0.0;
        if (map == PBS_BIO_MAP_DOSE) v = d;
        else if (map == PBS_BIO_MAP_LETD) v = d > 0.0 ? c2[i] / d : 0.0;
        else if (map == PBS_BIO_MAP_ALPHA) v = d > 0.0 ? c0[i] / d : 0.0;
        else if (map == PBS_BIO_MAP_BETA) { double sb = d > 0.0 ? c1[i] / d : 0.0; v = sb * sb; }
        else if (map == PBS_BIO_MAP_Z1D) v = 0.172 + (double)m->beta0 * (d > 0.0 ? c0[i] / d : 0.0);
        else {
            double rbe = 1.0;
            if (m->model == PBS_BIO_MKM) {
                double a = 0.172 + (double)m->beta0 * (d > 0.0 ? c0[i] / d : 0.0);
                double b0 = m->beta0, t2 = (double)m->alpha0 / 2.0 / b0;
                double dx = -t2 + sqrt(t2 * t2 + (a * d + b0 * d * d) / b0);
                rbe = d > 1e-3 ? dx / d : 1.0;
            } else if (d != 0.0 && c0[i] != 0.0 && c1[i] != 0.0) {
                double a = c0[i] / d, sb = c1[i] / d, b = sb * sb;
                double d10 = (-a + sqrt(a * a - 4.0 * -2.302585 * b)) / b * 0.5;
                rbe = 3.988565 / d10;
            }
            v = map == PBS_BIO_MAP_RBE ? rbe : rbe * d;
        }
        out[i] = v;
    }
}

/* tex1D linear/clamp/unnormalised evaluated in double. */
static double lut1(const float* t, int n, double x) {
    double xb = x - 0.5;
    if (xb < -1.0) xb = -1.0;
    if (xb > (double)n) xb = (double)n;
    double fl = floor(xb);
    int i = (int)fl;
    double a = texw(xb - fl);
    int i0 = i < 0 ? 0 : (i > n - 1 ? n - 1 : i);
    int i1 = i + 1 < 0 ? 0 : (i + 1 > n - 1 ? n - 1 : i + 1);
    return (1.0 - a) * t[i0] + a * t[i1];
}
/* Trilinear, texel centres at +0.5, zero outside (bev_ray_tracing.cu:16-61). */
static double tri_border(const float* vol, int dx, int dy, int dz, double x, double y, double z) {
    double fx = x - 0.5, fy = y - 0.5, fz = z - 0.5;
    if (fx < -2.0) fx = -2.0;
    if (fy < -2.0) fy = -2.0;
    if (fz < -2.0) fz = -2.0;
    if (fx > dx + 1.0) fx = dx + 1.0;
    if (fy > dy + 1.0) fy = dy + 1.0;
    if (fz > dz + 1.0) fz = dz + 1.0;
    double flx = floor(fx), fly = floor(fy), flz = floor(fz);
    int x0 = (int)flx, y0 = (int)fly, z0 = (int)flz;
    double tx = texw(fx - flx), ty = texw(fy - fly), tz = texw(fz - flz);
    double c[2][2][2];
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int cc = 0; cc < 2; ++cc) {
                int xi = x0 + cc, yi = y0 + b, zi = z0 + a;
                c[a][b][cc] = (xi < 0 || yi < 0 || zi < 0 || xi >= dx || yi >= dy || zi >= dz)
                                  ? 0.0 : vol[((size_t)zi * dy + yi) * dx + xi];
            }
    double c00 = c[0][0][0] + (c[0][0][1] - c[0][0][0]) * tx, c10 = c[0][1][0] + (c[0][1][1] - c[0][1][0]) * tx;
    double c01 = c[1][0][0] + (c[1][0][1] - c[1][0][0]) * tx, c11 = c[1][1][0] + (c[1][1][1] - c[1][1][0]) * tx;
    double c0 = c00 + (c10 - c00) * ty, c1 = c01 + (c11 - c01) * ty;
    return c0 + (c1 - c0) * tz;
}
static double tri_border_d(const double* vol, int dx, int dy, int dz, double x, double y, double z) {
    if (x < -2.0) x = -2.0;
    if (y < -2.0) y = -2.0;
    if (z < -2.0) z = -2.0;
    if (x > dx + 1.0) x = dx + 1.0;
    if (y > dy + 1.0) y = dy + 1.0;
    if (z > dz + 1.0) z = dz + 1.0;
    double flx = floor(x), fly = floor(y), flz = floor(z);
    int x0 = (int)flx, y0 = (int)fly, z0 = (int)flz;
    double tx = texw(x - flx), ty = texw(y - fly), tz = texw(z - flz);
    double acc = 0.0;
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int cc = 0; cc < 2; ++cc) {
                int xi = x0 + cc, yi = y0 + b, zi = z0 + a;
                if (xi < 0 || yi < 0 || zi < 0 || xi >= dx || yi >= dy || zi >= dz) continue;
                double w = (cc ? tx : 1.0 - tx) * (b ? ty : 1.0 - ty) * (a ? tz : 1.0 - tz);
                acc += w * vol[((size_t)zi * dy + yi) * dx + xi];
            }
    return acc;
}

/* ---- CT adapter (raytracedicom_wrapper.cu:2290-2441) ---------------------------- */
static int detect_ct_type(const float* d, size_t n) {
    size_t stride = n > 100000 ? n / 100000 : 1;
    float mn = d[0], mx = d[0];
    for (size_t i = 0; i < n; i += stride) {
        if (d[i] < mn) mn = d[i];
        if (d[i] > mx) mx = d[i];
    }
    if (mn < -200.0f) return PBS_CT_HU;
    if (mx <= 20.0f && mn >= 0.0f) return PBS_CT_DENSITY;
    return PBS_CT_HU_PLUS_1000;
}
static float frac_index_monotonic(const float* v, int n, float value) {
    if (n <= 1) return 0.0f;
    int inc = v[n - 1] >= v[0];
    if (inc) {
        if (value <= v[0]) return 0.0f;
        if (value >= v[n - 1]) return (float)(n - 1);
    } else {
        if (value >= v[0]) return 0.0f;
        if (value <= v[n - 1]) return (float)(n - 1);
    }
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (inc) { if (v[mid] <= value) lo = mid; else hi = mid; }
        else { if (v[mid] >= value) lo = mid; else hi = mid; }
    }
    float den = v[lo + 1] - v[lo], t = 0.0f;
    if (den != 0.0f) t = (value - v[lo]) / den;
    if (t < 0.0f) t = 0.0f;
    if (t > 1.0f) t = 1.0f;
    return (float)lo + t;
}

/* ---- spot lattice (raytracedicom_wrapper.cu:1259-1473) ----------------------- */
typedef struct {
    int valid, nx, ny, nl;
    float dx, dy, ox, oy;
    float* w; /* [nl][ny][nx] */
} Lattice;

static const float* weq_header(const PbsBeamDesc* b, size_t* n) {
    if (b->water_equivalence && b->n_water_equivalence >= 9) { *n = b->n_water_equivalence; return b->water_equivalence; }
    *n = b->ray_weq_header ? b->n_ray_weq_header : 0;
    return b->ray_weq_header;
}

static int cmp_float(const void* a, const void* b) {
    float x = *(const float*)a, y = *(const float*)b;
    return (x > y) - (x < y);
}

static int build_lattice(const PbsBeamDesc* b, Lattice* L) {
    memset(L, 0, sizeof *L);
    int nl = (int)b->n_energies;
    if (!b->layer_spot_counts || !b->n_layer_spot_counts || !b->spot_positions || !b->n_spot_positions ||
        !b->spot_weights || !b->n_spot_weights)
        return 0;
    if ((int)b->n_layer_spot_counts != nl || b->n_spot_positions % 2) return 0;
    int total = 0;
    for (int l = 0; l < nl; ++l) total += b->layer_spot_counts[l];
    if (total <= 0 || (int)(b->n_spot_positions / 2) != total || (int)b->n_spot_weights != total) return 0;
    size_t nh;
    const float* hdr = weq_header(b, &nh);
    if (b->spot_positions_are_indices) {
        if (nh < 9) return 0;
        int nx = (int)lroundf(hdr[8]); if (nx < 1) nx = 1;
        int ny = (int)lroundf(hdr[5]); if (ny < 1) ny = 1;
        float* w = (float*)calloc((size_t)nx * ny * nl, sizeof(float));
        int off = 0;
        for (int l = 0; l < nl; ++l) {
            int cnt = b->layer_spot_counts[l];
            if (cnt <= 0) { free(w); return 0; }
            for (int i = 0; i < cnt; ++i) {
                int s = off + i;
                float wt = b->spot_weights[s];
                if (!isfinite(wt) || wt < 0.0f) { free(w); return 0; }
                if (wt == 0.0f) continue;
                float lx = b->spot_positions[2 * s] - 0.5f, ly = b->spot_positions[2 * s + 1] - 0.5f;
                int ix0 = (int)floorf(lx), iy0 = (int)floorf(ly);
                float tx = lx - (float)ix0, ty = ly - (float)iy0;
                float fr[4] = {(1.0f - tx) * (1.0f - ty), tx * (1.0f - ty), (1.0f - tx) * ty, tx * ty};
                int ixs[4] = {ix0, ix0 + 1, ix0, ix0 + 1}, iys[4] = {iy0, iy0, iy0 + 1, iy0 + 1};
                double written = 0.0;
                for (int q = 0; q < 4; ++q) {
                    if (!(fr[q] > 0.0f) || ixs[q] < 0 || ixs[q] >= nx || iys[q] < 0 || iys[q] >= ny) continue;
                    w[((size_t)l * ny + iys[q]) * nx + ixs[q]] += wt * fr[q];
                    written += (double)wt * fr[q];
                }
                if (!(written > 0.0)) { free(w); return 0; }
            }
            off += cnt;
        }
        L->valid = 1; L->nx = nx; L->ny = ny; L->nl = nl;
        L->dx = hdr[7]; L->dy = hdr[4]; L->ox = hdr[6]; L->oy = hdr[3]; L->w = w;
        return 1;
    }
    float* xs = (float*)malloc(sizeof(float) * total);
    float* ys = (float*)malloc(sizeof(float) * total);
    for (int i = 0; i < total; ++i) { xs[i] = b->spot_positions[2 * i]; ys[i] = b->spot_positions[2 * i + 1]; }
    float* ux = (float*)malloc(sizeof(float) * total);
    float* uy = (float*)malloc(sizeof(float) * total);
    memcpy(ux, xs, sizeof(float) * total);
    memcpy(uy, ys, sizeof(float) * total);
    qsort(ux, total, sizeof(float), cmp_float);
    qsort(uy, total, sizeof(float), cmp_float);
    int nux = 0, nuy = 0;
    for (int i = 0; i < total; ++i) {
        if (nux == 0 || !(fabsf(ux[nux - 1] - ux[i]) <= 1e-4f)) ux[nux++] = ux[i];
        if (nuy == 0 || !(fabsf(uy[nuy - 1] - uy[i]) <= 1e-4f)) uy[nuy++] = uy[i];
    }
    float dx = INF20F, dy = INF20F;
    for (int i = 1; i < nux; ++i) { float d = ux[i] - ux[i - 1]; if (d > 1.0e-4f && d < dx) dx = d; }
    for (int i = 1; i < nuy; ++i) { float d = uy[i] - uy[i - 1]; if (d > 1.0e-4f && d < dy) dy = d; }
    float ox = ux[0], oy = uy[0];
    int nx = (int)lroundf((ux[nux - 1] - ox) / dx) + 1; if (nx < 1) nx = 1;
    int ny = (int)lroundf((uy[nuy - 1] - oy) / dy) + 1; if (ny < 1) ny = 1;
    float* w = (float*)calloc((size_t)nx * ny * nl, sizeof(float));
    int off = 0, ok = 1;
    for (int l = 0; l < nl && ok; ++l) {
        int cnt = b->layer_spot_counts[l];
        if (cnt <= 0) { ok = 0; break; }
        for (int i = 0; i < cnt; ++i) {
            int s = off + i;
            float wt = b->spot_weights[s];
            if (!isfinite(wt) || wt < 0.0f) { ok = 0; break; }
            if (wt == 0.0f) continue;
            float fx = dx != 0.0f ? (xs[s] - ox) / dx : 0.0f;
            float fy = dy != 0.0f ? (ys[s] - oy) / dy : 0.0f;
            int ix = (int)lroundf(fx), iy = (int)lroundf(fy);
            if (ix < 0 || ix >= nx || iy < 0 || iy >= ny) { ok = 0; break; }
            if (!(fabsf(ox + ix * dx - xs[s]) <= 2e-2f) || !(fabsf(oy + iy * dy - ys[s]) <= 2e-2f)) { ok = 0; break; }
            w[((size_t)l * ny + iy) * nx + ix] += wt;
        }
        off += cnt;
    }
    free(xs); free(ys); free(ux); free(uy);
    if (!ok) { free(w); return 0; }
    L->valid = 1; L->nx = nx; L->ny = ny; L->nl = nl; L->dx = dx; L->dy = dy; L->ox = ox; L->oy = oy; L->w = w;
    return 1;
}

/* raytracedicom_wrapper.cu:970-997 */
static int align_grid(float mn, float mx, float ref, float step, int mult, float* origin, int* count) {
    if (!(step > 0.0f) || !isfinite(mn) || !isfinite(mx) || !isfinite(ref)) return 0;
    if (mx < mn) { float t = mn; mn = mx; mx = t; }
    const float eps = 1.0e-4f;
    int first = (int)ceilf((mn - ref) / step - eps);
    int last = (int)floorf((mx - ref) / step + eps);
    if (last < first) return 0;
    *origin = ref + (float)first * step;
    int c = last - first + 1;
    if (c < 1) c = 1;
    if (mult > 1) c = ((c + mult - 1) / mult) * mult;
    *count = c;
    return 1;
}

static int decoded_bounds(const PbsBeamDesc* b, float* mnx, float* mxx, float* mny, float* mxy) {
    if (!b->layer_spot_counts || !b->n_layer_spot_counts || !b->spot_positions || !b->n_spot_positions) return 0;
    size_t nh;
    const float* hdr = weq_header(b, &nh);
    if (b->spot_positions_are_indices && nh < 9) return 0;
    *mnx = INF20F; *mxx = -INF20F; *mny = INF20F; *mxy = -INF20F;
    for (size_t i = 0; i < b->n_spot_positions / 2; ++i) {
        float x = b->spot_positions[2 * i], y = b->spot_positions[2 * i + 1];
        if (b->spot_positions_are_indices) {
            x = hdr[6] + (x - 0.5f) * hdr[7];
            y = hdr[3] + (y - 0.5f) * hdr[4];
        }
        if (x < *mnx) *mnx = x;
        if (x > *mxx) *mxx = x;
        if (y < *mny) *mny = y;
        if (y > *mxy) *mxy = y;
    }
    return *mnx <= *mxx && *mny <= *mxy;
}

/* raytracedicom_wrapper.cu:1847-1921 */
static int est_source_dist(const PbsBeamDesc* b, V3 bmX, V3 bmY, V3 bmZ, float sad, float* sx, float* sy) {
    if (!(sad > 1.0e-6f) || !b->spot_beam_directions || !b->n_spot_beam_directions || !b->spot_positions ||
        !b->n_spot_positions)
        return 0;
    if (b->n_spot_beam_directions % 3 || b->n_spot_positions % 2) return 0;
    size_t n = b->n_spot_beam_directions / 3 < b->n_spot_positions / 2 ? b->n_spot_beam_directions / 3 : b->n_spot_positions / 2;
    size_t nh;
    const float* hdr = weq_header(b, &nh);
    int hh = nh >= 9;
    float* ax = (float*)malloc(sizeof(float) * (n + 1));
    float* ay = (float*)malloc(sizeof(float) * (n + 1));
    size_t na = 0, nb = 0;
    for (size_t i = 0; i < n; ++i) {
        float px = b->spot_positions[2 * i], py = b->spot_positions[2 * i + 1];
        if (b->spot_positions_are_indices) {
            if (!hh) { free(ax); free(ay); return 0; }
            px = hdr[6] + (px - 0.5f) * hdr[7];
            py = hdr[3] + (py - 0.5f) * hdr[4];
        }
        V3 d = v3(b->spot_beam_directions[3 * i], b->spot_beam_directions[3 * i + 1], b->spot_beam_directions[3 * i + 2]);
        float len = sqrtf(vdot(d, d));
        if (!(len > 1.0e-6f)) continue;
        d = vdiv(d, len);
        float a = vdot(d, bmZ);
        if (!(fabsf(a) > 1.0e-6f)) continue;
        float bx = vdot(d, bmX), by = vdot(d, bmY);
        if (fabsf(px) > 1.0e-3f && fabsf(bx) > 1.0e-6f) { float c = fabsf(px * a / bx); if (c > 1.0f && isfinite(c)) ax[na++] = c; }
        if (fabsf(py) > 1.0e-3f && fabsf(by) > 1.0e-6f) { float c = fabsf(py * a / by); if (c > 1.0f && isfinite(c)) ay[nb++] = c; }
    }
    qsort(ax, na, sizeof(float), cmp_float);
    qsort(ay, nb, sizeof(float), cmp_float);
    *sx = na ? ax[na / 2] : 0.0f;
    *sy = nb ? ay[nb / 2] : 0.0f;
    free(ax); free(ay);
    return *sx > 0.0f || *sy > 0.0f;
}

/* ---- beam plan ------------------------------------------------------------------- */
typedef struct {
    OraclePlan p;
    Lattice lat;
    FromFan fanToIm, fanToDose;
    TracerP tracer;
    float volConst, volLin, volSq;
    float* lp; /* [L][8] */
    /* Water-equivalence import (wrapper.cu:3316-3395, 3566-3640). */
    int weq, weqNx, weqNy, weqSteps, weqActive;
    float weqStepMm, weqX0, weqY0, weqDx, weqDy;
    const float* weqBody;
} Plan;

static void free_plan(Plan* P) {
    free(P->lat.w);
    free(P->lp);
    memset(P, 0, sizeof *P);
}

static int plan_beam(const PbsBeamDesc* b, const PbsEnergyDesc* e, const int* cd, const float* cr, const float* cc,
                     const int* dd, const float* dr, const float* dc, Plan* P) {
    memset(P, 0, sizeof *P);
    int L = (int)b->n_energies;
    P->p.num_layers = L;
    /* Units (wrapper.cu:2729-2797). */
    float lenToMm = (cr[2] > 0.0f && cr[2] < 0.3f) ? 10.0f : 1.0f;
    float e2mm = lenToMm;
    {
        float peakMax = 0.0f;
        for (int i = 0; i < e->n_energies; ++i) if (e->peak_depths[i] > peakMax) peakMax = e->peak_depths[i];
        const char* es = getenv("RTD_ENERGY_DEPTH_SCALE");
        const char* eu = getenv("RTD_ENERGY_DEPTH_UNIT");
        if (es && es[0]) {
            e2mm = (float)atof(es);
            if (e2mm < 0.0f) e2mm = 0.0f;
            if (e2mm == 0.0f) e2mm = lenToMm;
        } else if (eu && eu[0]) {
            if (!strcasecmp(eu, "cm")) e2mm = 10.0f;
            else if (!strcasecmp(eu, "mm")) e2mm = 1.0f;
        } else if (lenToMm == 10.0f && peakMax > 200.0f) {
            e2mm = 1.0f;
        }
    }
    P->p.len_to_mm = lenToMm;
    P->p.energy_depth_to_mm = e2mm;
    /* Gantry frame (wrapper.cu:2880-2933). */
    V3 bdir = vnorm_safe(v3(b->beam_direction[0], b->beam_direction[1], b->beam_direction[2]));
    V3 bxd = vnorm_safe(v3(b->bm_x_direction[0], b->bm_x_direction[1], b->bm_x_direction[2]));
    V3 byd = vnorm_safe(v3(b->bm_y_direction[0], b->bm_y_direction[1], b->bm_y_direction[2]));
    V3 src = v3(b->source_position[0], b->source_position[1], b->source_position[2]);
    float sad = b->sad > 0.0f ? b->sad : b->source_dist[0];
    V3 bc = vnorm_safe(vcross(bxd, byd));
    int haveCross = vdot(bc, bc) > 1.0e-8f, haveDir = vdot(bdir, bdir) > 1.0e-8f;
    V3 bmZ = haveCross ? bc : bdir;
    if (haveCross && haveDir && vdot(bmZ, bdir) < 0.0f) bmZ = vmul(bmZ, -1.0f);
    if (!(vdot(bmZ, bmZ) > 1.0e-8f)) bmZ = v3(0, 0, 1);
    V3 bmX = vnorm_safe(vsub(bxd, vmul(bmZ, vdot(bxd, bmZ))));
    if (!(vdot(bmX, bmX) > 1.0e-8f)) bmX = vnorm_safe(vcross(byd, bmZ));
    if (!(vdot(bmX, bmX) > 1.0e-8f)) bmX = v3(1, 0, 0);
    V3 bmY = vnorm_safe(vcross(bmZ, bmX));
    if (vdot(bmY, byd) < 0.0f) bmY = vmul(bmY, -1.0f);
    bmX = vnorm_safe(vcross(bmY, bmZ));
    V3 gX = bmX, gY = vmul(bmY, -1.0f), gZ = vmul(bmZ, -1.0f);
    V3 iso = vadd(vmul(src, lenToMm), vmul(bmZ, sad * lenToMm));
    Aff g2w = aff(m3(v3(gX.x, gY.x, gZ.x), v3(gX.y, gY.y, gZ.y), v3(gX.z, gY.z, gZ.z)), iso);
    Aff w2g = ainv(g2w);
    int hasLat = build_lattice(b, &P->lat);
    /* Dose projection + subspot bounds for the legacy grid (wrapper.cu:2981-3031). */
    V3 doseRes = v3(dr[0] * lenToMm, dr[1] * lenToMm, dr[2] * lenToMm);
    V3 doseCorner = v3(dc[0] * lenToMm, dc[1] * lenToMm, dc[2] * lenToMm);
    float minGX = 1e30f, maxGX = -1e30f, minGY = 1e30f, maxGY = -1e30f;
    {
        V3 sz = v3((float)(dd[0] - 1 > 0 ? dd[0] - 1 : 0) * doseRes.x, (float)(dd[1] - 1 > 0 ? dd[1] - 1 : 0) * doseRes.y,
                   (float)(dd[2] - 1 > 0 ? dd[2] - 1 : 0) * doseRes.z);
        for (int x = 0; x <= 1; ++x)
            for (int y = 0; y <= 1; ++y)
                for (int z = 0; z <= 1; ++z) {
                    V3 g = aapply(w2g, vadd(doseCorner, v3((float)x * sz.x, (float)y * sz.y, (float)z * sz.z)));
                    minGX = fminf(minGX, g.x); maxGX = fmaxf(maxGX, g.x);
                    minGY = fminf(minGY, g.y); maxGY = fmaxf(maxGY, g.y);
                }
        int M = b->max_subspots_per_layer;
        for (int li = 0; li < L; ++li)
            for (int si = 0; si < M; ++si) {
                size_t base = ((size_t)li * M + si) * 5;
                if (b->n_subspot_data <= base + 4) break;
                if (b->subspot_data[base + 2] > 0.0f) {
                    float sx = b->subspot_data[base] / lenToMm, sy = b->subspot_data[base + 1] / lenToMm;
                    minGX = fminf(minGX, sx); maxGX = fmaxf(maxGX, sx);
                    minGY = fminf(minGY, sy); maxGY = fmaxf(maxGY, sy);
                }
            }
    }
    /* Ray grid (wrapper.cu:3039-3212). */
    size_t nh;
    const float* hdr = weq_header(b, &nh);
    float msx = 0.0f, msy = 0.0f;
    for (size_t i = 0; 2 * i + 1 < b->n_spot_sigmas; ++i) {
        if (b->spot_sigmas[2 * i] > msx) msx = b->spot_sigmas[2 * i];
        if (b->spot_sigmas[2 * i + 1] > msy) msy = b->spot_sigmas[2 * i + 1];
    }
    float rsx = b->ray_spacing[0], rsy = b->ray_spacing[1];
    V3 cpbCorner, cpbRes;
    int nX = 0, nY = 0;
    if (hasLat && rsx > 0.0f && rsy > 0.0f) {
        float mX = 3.0f * msx + 0.5f * rsx, mY = 3.0f * msy + 0.5f * rsy, oX, oY;
        const Lattice* R = &P->lat;
        if (!align_grid(R->ox - mX, R->ox + (float)(R->nx - 1) * R->dx + mX, R->ox, rsx, TILE_X, &oX, &nX) ||
            !align_grid(R->oy - mY, R->oy + (float)(R->ny - 1) * R->dy + mY, R->oy, rsy, TILE_Y, &oY, &nY))
            return fail(PBS_ERR_GEOMETRY, "Failed to align CPB grid to raw spot lattice phase");
        cpbCorner = v3(oX, oY, 0.0f);
        cpbRes = v3(rsx, rsy, dr[2]);
    } else if (nh >= 9) {
        int cropped = 0;
        float a, bb, c, d;
        if (rsx > 0.0f && rsy > 0.0f && decoded_bounds(b, &a, &bb, &c, &d)) {
            float mX = 3.0f * msx + 0.5f * rsx, mY = 3.0f * msy + 0.5f * rsy, oX, oY;
            if (align_grid(a - mX, bb + mX, hdr[6] / lenToMm, rsx, TILE_X, &oX, &nX) &&
                align_grid(c - mY, d + mY, hdr[3] / lenToMm, rsy, TILE_Y, &oY, &nY)) {
                cpbCorner = v3(oX, oY, 0.0f);
                cpbRes = v3(rsx, rsy, dr[2]);
                cropped = 1;
            }
        }
        if (!cropped) {
            cpbCorner = v3(hdr[6] / lenToMm, hdr[3] / lenToMm, 0.0f);
            cpbRes = v3(hdr[7] / lenToMm, hdr[4] / lenToMm, dr[2]);
            int ax = (int)lroundf(hdr[8]), ay = (int)lroundf(hdr[5]);
            nX = (((ax < 1 ? 1 : ax) + TILE_X - 1) / TILE_X) * TILE_X;
            nY = (((ay < 1 ? 1 : ay) + TILE_Y - 1) / TILE_Y) * TILE_Y;
        }
    } else {
        if (!(rsx > 0.0f) || !(rsy > 0.0f))
            return fail(PBS_ERR_GEOMETRY, "Legacy CPB path requires explicit beam.raySpacing");
        float covX = (maxGX - minGX) / lenToMm, covY = (maxGY - minGY) / lenToMm;
        if (!(covX > 0.0f) || !(covY > 0.0f))
            return fail(PBS_ERR_GEOMETRY, "Legacy CPB path produced non-positive projected coverage");
        const char* env = getenv("RTD_CPB_COVERAGE_CM");
        if (env) { float v = (float)atof(env); if (v > 0.0f && isfinite(v)) covX = covY = v; }
        cpbCorner = v3(minGX / lenToMm, minGY / lenToMm, 0.0f);
        cpbRes = v3(rsx, rsy, dr[2]);
        nX = (int)ceilf(covX / cpbRes.x); if (nX < 1) nX = 1;
        nY = (int)ceilf(covY / cpbRes.y); if (nY < 1) nY = 1;
    }
    P->p.conv_mode = hasLat ? 0 : 1;
    P->p.ray_x = nX;
    P->p.ray_y = nY;
    P->p.pitch_x = ((nX + TILE_X - 1) / TILE_X) * TILE_X;
    P->p.pitch_y = ((nY + TILE_Y - 1) / TILE_Y) * TILE_Y;
    P->p.tiles_x = P->p.pitch_x / TILE_X;
    P->p.tiles_y = P->p.pitch_y / TILE_Y;
    P->p.cpb_corner[0] = cpbCorner.x; P->p.cpb_corner[1] = cpbCorner.y;
    P->p.cpb_res[0] = cpbRes.x; P->p.cpb_res[1] = cpbRes.y;
    P->p.lat_nx = P->lat.nx; P->p.lat_ny = P->lat.ny;
    P->p.lat_dx = P->lat.dx; P->p.lat_dy = P->lat.dy; P->p.lat_ox = P->lat.ox; P->p.lat_oy = P->lat.oy;
    /* Index transforms (wrapper.cu:3219-3248). */
    V3 ctRes = v3(cr[0] * lenToMm, cr[1] * lenToMm, cr[2] * lenToMm);
    V3 ctCorner = v3(cc[0] * lenToMm, cc[1] * lenToMm, cc[2] * lenToMm);
    Aff w2i = aff(mdiag(1.0f / ctRes.x, 1.0f / ctRes.y, 1.0f / ctRes.z),
                  v3(-ctCorner.x / ctRes.x, -ctCorner.y / ctRes.y, -ctCorner.z / ctRes.z));
    Aff g2i = aconcat(g2w, w2i);
    Aff w2d = aff(mdiag(1.0f / doseRes.x, 1.0f / doseRes.y, 1.0f / doseRes.z),
                  v3(-doseCorner.x / doseRes.x, -doseCorner.y / doseRes.y, -doseCorner.z / doseRes.z));
    Aff g2d = aconcat(g2w, w2d);
    /* Source distances (wrapper.cu:3250-3271). */
    float ix = 0, iy = 0;
    int inferred = est_source_dist(b, bmX, bmY, bmZ, sad, &ix, &iy);
    float distX = b->source_dist[0] * lenToMm, distY = b->source_dist[1] * lenToMm;
    int legacy = fabsf(b->source_dist[0] - b->sad) < 1.0e-3f && fabsf(b->source_dist[1] - b->sad) < 1.0e-3f;
    if (inferred && (!(distX > 1e-6f) || legacy)) distX = ix * lenToMm;
    if (inferred && (!(distY > 1e-6f) || legacy)) distY = iy * lenToMm;
    if (!(distX > 1e-6f)) distX = sad * lenToMm;
    if (!(distY > 1e-6f)) distY = sad * lenToMm;
    P->p.source_dist[0] = distX;
    P->p.source_dist[1] = distY;
    /* Tracer extent (wrapper.cu:3286-3364). */
    float minGZ = 1e30f, maxGZ = -1e30f;
    {
        V3 sz = v3((float)(cd[0] - 1 > 0 ? cd[0] - 1 : 0) * ctRes.x, (float)(cd[1] - 1 > 0 ? cd[1] - 1 : 0) * ctRes.y,
                   (float)(cd[2] - 1 > 0 ? cd[2] - 1 : 0) * ctRes.z);
        for (int x = 0; x <= 1; ++x)
            for (int y = 0; y <= 1; ++y)
                for (int z = 0; z <= 1; ++z) {
                    V3 g = aapply(w2g, vadd(ctCorner, v3((float)x * sz.x, (float)y * sz.y, (float)z * sz.z)));
                    minGZ = fminf(minGZ, g.z);
                    maxGZ = fmaxf(maxGZ, g.z);
                }
    }
    const int hasWeq = nh >= 9 && b->water_equivalence && b->n_water_equivalence > 9;
    float stepMm = hasWeq ? hdr[1] * lenToMm : cr[2] * lenToMm;
    if (!(stepMm > 0.0f)) stepMm = cr[2] * lenToMm;
    float startZ = maxGZ;
    int steps;
    P->weq = hasWeq;
    if (hasWeq) {
        /* BEV start plane at the exporter's projected WEQ origin when it is positive,
         * finite and within max(WEQ depth span, 50 mm) of the CT start
         * (wrapper.cu:3316-3364); steps from the header (wrapper.cu:3365-3367). */
        float weqStart = hdr[0] * lenToMm;
        float aligned = 0.5f * (distX + distY) - weqStart;
        long hs = lroundf(hdr[2]);
        float span = fabsf(hdr[1] * lenToMm) * (float)(hs > 0 ? hs : 0);
        float maxDelta = span > 50.0f ? span : 50.0f;
        if (isfinite(aligned) && isfinite(weqStart) && weqStart > 0.0f && fabsf(aligned - maxGZ) <= maxDelta)
            startZ = aligned;
        steps = (int)lroundf(hdr[2]);
        if (steps < 1) steps = 1;
        P->weqSteps = steps;
        P->weqNy = (int)lroundf(hdr[5]); if (P->weqNy < 1) P->weqNy = 1;
        P->weqNx = (int)lroundf(hdr[8]); if (P->weqNx < 1) P->weqNx = 1;
        /* Only nx*ny*nStep samples are depths (wrapper.cu:3566-3590). */
        if (b->n_water_equivalence - 9 < (size_t)P->weqNx * P->weqNy * P->weqSteps)
            return fail(PBS_ERR_GEOMETRY, "water_equivalence payload is smaller than header-declared nx*ny*nStep");
        P->weqActive = steps < P->weqSteps ? steps : P->weqSteps;
        P->weqStepMm = fabsf(hdr[1] * lenToMm);
        P->weqX0 = hdr[6] / lenToMm;
        P->weqY0 = hdr[3] / lenToMm;
        P->weqDx = hdr[7] / lenToMm;
        P->weqDy = hdr[4] / lenToMm;
        P->weqBody = b->water_equivalence + 9;
    } else {
        steps = (int)ceilf((maxGZ - minGZ) / fabsf(stepMm)) + 1;
        if (steps < 1) steps = 1;
    }
    P->p.steps = steps;
    V3 fanCorner = v3(cpbCorner.x * lenToMm, cpbCorner.y * lenToMm, startZ);
    V3 fanDelta = v3(cpbRes.x * lenToMm, cpbRes.y * lenToMm, -fabsf(stepMm));
    P->p.fan_corner[0] = fanCorner.x; P->p.fan_corner[1] = fanCorner.y; P->p.fan_corner[2] = fanCorner.z;
    P->p.fan_delta[0] = fanDelta.x; P->p.fan_delta[1] = fanDelta.y; P->p.fan_delta[2] = fanDelta.z;
    P->fanToIm.fan = idxt(fanDelta, fanCorner);
    P->fanToIm.g = g2i;
    P->fanToIm.dist.x = distX;
    P->fanToIm.dist.y = distY;
    P->fanToDose = P->fanToIm;
    P->fanToDose.g = g2d;
    P->tracer = tracer_params(P->fanToIm);
    {
        float dX = fanDelta.x, dY = fanDelta.y, dZ = fanDelta.z, cZ = fanCorner.z;
        float dXYZ = fabsf(dX * dY * dZ);
        P->volConst = dXYZ * (1.0f - cZ / distX - cZ / distY + (cZ * cZ + dZ * dZ / 12.0f) / (distX * distY));
        P->volLin = dXYZ * dZ * (-1.0f / distX - 1.0f / distY + 2.0f * cZ / (distX * distY));
        P->volSq = dXYZ * dZ * dZ / (distX * distY);
    }
    {
        float maxE = b->energies[0];
        for (int l = 1; l < L; ++l) if (b->energies[l] > maxE) maxE = b->energies[l];
        float idx = find_decimal(e->energies_per_u, e->n_energies, maxE);
        P->p.max_peak_depth_mm = vinterp(e->peak_depths, e->n_energies, idx) * e2mm;
    }
    P->p.bev_x = P->p.pitch_x + 2 * MAX_R;
    P->p.bev_y = P->p.pitch_y + 2 * MAX_R;
    if (hasLat) { /* halo lattice padded to the tile size (wrapper.cu:862-864) */
        P->p.nuc_x = ((P->lat.nx + TILE_X - 1) / TILE_X) * TILE_X;
        P->p.nuc_y = ((P->lat.ny + TILE_Y - 1) / TILE_Y) * TILE_Y;
        P->p.nuc_bev_x = P->p.nuc_x + 2 * MAX_R;
        P->p.nuc_bev_y = P->p.nuc_y + 2 * MAX_R;
    }
    /* Per-layer energy parameters (wrapper.cu:3926-4053, fill_idd_and_sigma_params.cuh:66-78). */
    P->lp = (float*)calloc((size_t)L * 8, sizeof(float));
    int nE = e->n_energies;
    const float* E = e->energies_per_u;
    for (int l = 0; l < L; ++l) {
        float en = b->energies[l];
        float sxx = 1.0f, syy = 1.0f;
        if (2 * (size_t)l + 1 < b->n_spot_sigmas) { sxx = b->spot_sigmas[2 * l]; syy = b->spot_sigmas[2 * l + 1]; }
        if (lenToMm > 1.0f && sxx > 0.0f && sxx < 1.0f) sxx *= 10.0f;
        if (lenToMm > 1.0f && syy > 0.0f && syy < 1.0f) syy *= 10.0f;
        float convPeak = vinterp(e->peak_depths, nE, find_decimal(E, nE, en)) * e2mm;
        float eIdx;
        int asc = nE > 1 ? E[0] < E[nE - 1] : 1;
        int iLow = asc ? 0 : nE - 1, iHigh = asc ? nE - 1 : 0;
        if (nE <= 1) eIdx = 0.0f;
        else if (en <= E[iLow]) eIdx = (float)iLow;
        else if (en >= E[iHigh]) eIdx = (float)iHigh;
        else {
            int fi = 0;
            float e0 = E[0], e1 = E[0];
            for (int i = 0; i < nE - 1; ++i) {
                float a = E[i], c = E[i + 1];
                float lo = a < c ? a : c, hi = a < c ? c : a;
                if (en >= lo && en <= hi) { fi = i; e0 = a; e1 = c; break; }
            }
            float den = e1 - e0;
            float corr = den != 0.0f ? (en - e0) / den : 0.0f;
            if (!isfinite(corr)) corr = 0.0f;
            if (corr < 0.0f) corr = 0.0f;
            if (corr > 1.0f) corr = 1.0f;
            eIdx = (float)fi + corr;
        }
        float scaleT, peakT;
        if (eIdx <= 0.0f) { scaleT = e->scale_facts[0]; peakT = e->peak_depths[0]; }
        else if (eIdx >= (float)(nE - 1)) { scaleT = e->scale_facts[nE - 1]; peakT = e->peak_depths[nE - 1]; }
        else {
            float ip, dec = modff(eIdx, &ip);
            int f = (int)ip;
            scaleT = e->scale_facts[f] + (e->scale_facts[f + 1] - e->scale_facts[f]) * dec;
            peakT = e->peak_depths[f] + (e->peak_depths[f + 1] - e->peak_depths[f]) * dec;
        }
        float peak = peakT * e2mm;
        float a = 0.00270f / (peak - 4.50f), bq = -4.39f / (peak - 3.86f);
        float* o = P->lp + 8 * l;
        o[0] = eIdx;
        o[1] = scaleT / e2mm;
        o[2] = peak;
        o[3] = convPeak;
        o[4] = a * 1.0f * fanDelta.z * fanDelta.z;
        o[5] = 2.0f * a * 1.0f * fanDelta.z * fanCorner.z + bq * fanDelta.z;
        o[6] = sxx;
        o[7] = syy;
    }
    return PBS_OK;
}

int oracle_plan(const PbsBeamDesc* beam, const PbsEnergyDesc* energy, const int cd[3], const float cr[3],
                const float cc[3], const int dd[3], const float dr[3], const float dc[3], OraclePlan* out,
                float* layer_params, float* lattice, size_t lattice_len) {
    Plan P;
    int rc = plan_beam(beam, energy, cd, cr, cc, dd, dr, dc, &P);
    if (rc) { free_plan(&P); return rc; }
    *out = P.p;
    if (layer_params) memcpy(layer_params, P.lp, sizeof(float) * 8 * P.p.num_layers);
    if (lattice && P.lat.valid && lattice_len == (size_t)P.lat.nx * P.lat.ny * P.lat.nl)
        memcpy(lattice, P.lat.w, sizeof(float) * lattice_len);
    free_plan(&P);
    return PBS_OK;
}

/* ---- radius buckets and batching -------------------------------------------- */
int oracle_radius_bucket(float m) { /* complete_superposition.cu:242 with IEEE float division */
    float q = 3.0f / (1.41421354f * m) + 0.5f;
    if (!(q < 34.0f)) return (q != q) ? 0 : 33;
    int r = (int)q;
    return r > 33 ? 33 : r;
}

void oracle_batch(const int hist_in[34], int batched[33], int map[34]) {
    int h[34];
    memcpy(h, hist_in, sizeof h);
    if (h[MAX_R + 1] > 0) { h[MAX_R] += h[MAX_R + 1]; h[MAX_R + 1] = 0; } /* primary overflow merge */
    int layerMax = 0;
    for (int i = 0; i < 34; ++i) if (h[i] > 0) layerMax = i;
    for (int i = 0; i <= MAX_R; ++i) batched[i] = 0;
    for (int i = 0; i < 34; ++i) map[i] = i;
    batched[0] = h[0];
    map[0] = 0;
    int rec = layerMax;
    for (int rad = layerMax; rad > 0; --rad) {
        map[rad] = rec;
        batched[rec] += h[rad];
        if (batched[rec] >= MIN_TILES_IN_BATCH) rec = rad - 1;
    }
    map[MAX_R + 1] = map[MAX_R];
}

/* ---- pipeline ----------------------------------------------------------------- */
static double erfd(double x) { return erf(x); }

/* Tile radius codes of one step on a grid of TXg x TYg tiles (tileRadCalc,
 * complete_superposition.cu:198-255): minimum rSigmaEff and any(idd > 0). */
static void tile_codes(const double* iddK, const double* rsgK, int PXg, int TXg, int TYg, unsigned char* out) {
    for (int ty = 0; ty < TYg; ++ty)
        for (int tx = 0; tx < TXg; ++tx) {
            double mn = INFINITY;
            int anyLive = 0;
            for (int sy = 0; sy < TILE_Y; ++sy)
                for (int sx = 0; sx < TILE_X; ++sx) {
                    size_t o = (size_t)(ty * TILE_Y + sy) * PXg + tx * TILE_X + sx;
                    if (rsgK[o] < mn) mn = rsgK[o];
                    if (iddK[o] > 0.0) anyLive = 1;
                }
            int R = oracle_radius_bucket((float)mn);
            out[ty * TXg + tx] = (unsigned char)(R | (anyLive ? 0x80 : 0));
        }
}

/* kernelSuperposition<R> (complete_superposition.cu:264-335) of the live tiles of
 * one step into one BEV plane padded by MAX_R on every side. */
static double superpose_step(const double* iddK, const double* rsgK, const unsigned char* codesK, const int* map,
                             int PXg, int TXg, int TYg, double* plane, int BXg) {
    double fma = 0.0, ed[MAX_R + 1];
    for (int t = 0; t < TXg * TYg; ++t) {
        unsigned char c = codesK[t];
        if (!(c & 0x80)) continue;
        int R = map[c & 0x3f];
        fma += 256.0 * (2 * R + 1) * (2 * R + 1);
        int tx = t % TXg, ty = t / TXg;
        for (int sy = 0; sy < TILE_Y; ++sy)
            for (int sx = 0; sx < TILE_X; ++sx) {
                size_t o = (size_t)(ty * TILE_Y + sy) * PXg + tx * TILE_X + sx;
                double dose_ = iddK[o];
                if (!(dose_ > 0.0)) continue;
                double rs = rsgK[o];
                double en = erf(rs * 0.5), eo = -en;
                for (int i = 0; i <= R; ++i) {
                    ed[i] = 0.5 * (en - eo);
                    eo = en;
                    en = erf(rs * ((double)i + 1.5));
                }
                int oy0 = ty * TILE_Y + sy - R + MAX_R, ox0 = tx * TILE_X + sx - R + MAX_R;
                for (int i = 0; i < 2 * R + 1; ++i) {
                    double wy = dose_ * ed[abs(R - i)];
                    double* rowp = plane + (size_t)(oy0 + i) * BXg + ox0;
                    for (int j = 0; j < 2 * R + 1; ++j) rowp[j] += wy * ed[abs(R - j)];
                }
            }
    }
    return fma;
}

/* Divergent transfer of one layer's BEV dose (wrapper.cu:5343-5505 primary,
 * 5510-5600 nuclear; prim_transf_kernel.cu:11-78): bounding box of the padded BEV
 * grid in dose indices, then a trilinear sample per voxel added where positive. */
static void transfer_layer(const FromFan* fanToDose, int gridX, int gridY, int first, int calc, int passive,
                           int compat, const double* bev, int BXg, int BYg, double* dose, const int* dd, int box[6]) {
    box[0] = box[1] = box[2] = 0;
    box[3] = box[4] = box[5] = -1;
    const float xs[2] = {-(float)MAX_R, (float)(gridX + MAX_R - 1)};
    const float ys[2] = {-(float)MAX_R, (float)(gridY + MAX_R - 1)};
    const float zs[2] = {(float)first, (float)(calc - 1)};
    V3 mx = v3(-1.0f, -1.0f, -1.0f), mn = v3(100000.0f, 100000.0f, 100000.0f);
    for (int zi = 0; zi < 2; ++zi)
        for (int yi = 0; yi < 2; ++yi)
            for (int xi = 0; xi < 2; ++xi) {
                V3 p = ffapply(*fanToDose, v3(xs[xi], ys[yi], zs[zi]));
                mx.x = fmaxf(mx.x, p.x); mx.y = fmaxf(mx.y, p.y); mx.z = fmaxf(mx.z, p.z);
                mn.x = fminf(mn.x, p.x); mn.y = fminf(mn.y, p.y); mn.z = fminf(mn.z, p.z);
            }
    int sx0 = ((int)floorf(mn.x) / 32) * 32;
    box[0] = sx0 > 0 ? sx0 : 0;
    box[1] = (int)floorf(mn.y) > 0 ? (int)floorf(mn.y) : 0;
    box[2] = (int)floorf(mn.z) > 0 ? (int)floorf(mn.z) : 0;
    box[3] = (int)ceilf(mx.x) < dd[0] - 1 ? (int)ceilf(mx.x) : dd[0] - 1;
    box[4] = (int)ceilf(mx.y) < dd[1] - 1 ? (int)ceilf(mx.y) : dd[1] - 1;
    box[5] = (int)ceilf(mx.z) < dd[2] - 1 ? (int)ceilf(mx.z) : dd[2] - 1;
    if (!(box[0] <= box[3] && box[1] <= box[4] && box[2] <= box[5])) return;
    ToFan tf = ff_invert_shift(*fanToDose, v3((float)MAX_R, (float)MAX_R, -(float)first));
    TransferP T = transfer_params(tf);
    int spanX = ((box[3] - box[0] + 1 + 31) / 32) * 32, spanY = ((box[4] - box[1] + 1 + 7) / 8) * 8;
    int xEnd = box[0] + spanX < dd[0] ? box[0] + spanX : dd[0];
    int yEnd = box[1] + spanY < dd[1] ? box[1] + spanY : dd[1];
    /* The reference's BEV texture spans planes [0, guaranteedPassive). */
    const int nz = passive;
    const double zshift = compat ? 0.0 : (double)first;
    const int b1 = box[1], b0 = box[0], b2 = box[2], b5 = box[5];
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = b1; y < yEnd; ++y)
        for (int x = b0; x < xEnd; ++x)
            for (int z = b2; z <= b5; ++z) {
                V3 f = tp_fan(&T, x, y, z);
                if (f.x + 0.5f < 0.0f || f.y + 0.5f < 0.0f || f.z + 0.5f < 0.0f) continue;
                double v = tri_border_d(bev, BXg, BYg, nz, f.x, f.y, (double)f.z + zshift);
                if (v > 0.0) dose[((size_t)z * dd[1] + y) * dd[0] + x] += v;
            }
}

/* Energy-interpolated row of a [nE][nS] table at a fixed energy coordinate: the
 * bilinear texture lookup of the reference is a depth lerp of this row. */
static void table_row(const float* tab, int nE, int nS, float eIdx, double* row) {
    double eb = eIdx;
    if (eb < -1.0) eb = -1.0;
    if (eb > nE) eb = nE;
    double fl = floor(eb), bb = texw(eb - fl);
    int e0 = (int)fl < 0 ? 0 : ((int)fl > nE - 1 ? nE - 1 : (int)fl);
    int e1 = (int)fl + 1 < 0 ? 0 : ((int)fl + 1 > nE - 1 ? nE - 1 : (int)fl + 1);
    for (int d = 0; d < nS; ++d)
        row[d] = (1.0 - bb) * tab[(size_t)e0 * nS + d] + bb * tab[(size_t)e1 * nS + d];
}

static double row_lookup(const double* row, int nS, double xi) {
    double xb = xi - 0.5;
    if (xb < -1.0) xb = -1.0;
    if (xb > nS) xb = nS;
    double fl = floor(xb), aa = texw(xb - fl);
    int i0 = (int)fl < 0 ? 0 : ((int)fl > nS - 1 ? nS - 1 : (int)fl);
    int i1 = (int)fl + 1 < 0 ? 0 : ((int)fl + 1 > nS - 1 ? nS - 1 : (int)fl + 1);
    return (1.0 - aa) * row[i0] + aa * row[i1];
}

static int run_beam(const float* ct, const int* cd, double* dose, const int* dd, const PbsBeamDesc* b,
                    const PbsEnergyDesc* e, const Plan* P, int compat, int nucModel, OracleCapture* cap) {
    const int L = P->p.num_layers, S = P->p.steps, RX = P->p.ray_x, RY = P->p.ray_y;
    const int PX = P->p.pitch_x, PY = P->p.pitch_y, TX = P->p.tiles_x, TY = P->p.tiles_y;
    const size_t rays = (size_t)RX * RY, pad = (size_t)PX * PY, tiles = (size_t)TX * TY;
    const int BX = P->p.bev_x, BY = P->p.bev_y;
    const size_t bevPlane = (size_t)BX * BY;
    /* Nuclear halo plan (buildHaloLatticePlan, wrapper.cu:804-929, driven from
     * wrapper.cu:3412-3452): the dense spot lattice padded to 32 x 8, and the ray
     * under every lattice cell. */
    const int nuc = nucModel >= 0;
    const int NXn = P->p.nuc_x, NYn = P->p.nuc_y, NTX = NXn / TILE_X, NTY = NYn / TILE_Y;
    const size_t nucPad = (size_t)NXn * NYn, nucTiles = (size_t)NTX * NTY;
    const int NBX = P->p.nuc_bev_x, NBY = P->p.nuc_bev_y;
    const size_t nucBevPlane = (size_t)NBX * NBY;
    int* rayToNuc = NULL;
    if (nuc) {
        if (P->p.conv_mode != 0)
            return fail(PBS_ERR_INVALID_ARGUMENT,
                        "nuclear_correction=true requires raw spot lattice inputs; legacy CPB fallback cannot drive halo mode");
        rayToNuc = (int*)malloc(sizeof(int) * rays);
        for (size_t r = 0; r < rays; ++r) rayToNuc[r] = -1;
        for (int sy = 0; sy < P->lat.ny; ++sy) {
            const float gy = P->lat.oy + (float)sy * P->lat.dy;
            const int ry = (int)lroundf((gy - P->p.cpb_corner[1]) / P->p.cpb_res[1]);
            if (ry < 0 || ry >= RY) {
                free(rayToNuc);
                return fail(PBS_ERR_GEOMETRY, "dense halo lattice row mapped outside active ray grid");
            }
            for (int sx = 0; sx < P->lat.nx; ++sx) {
                const float gx = P->lat.ox + (float)sx * P->lat.dx;
                const int rx = (int)lroundf((gx - P->p.cpb_corner[0]) / P->p.cpb_res[0]);
                if (rx < 0 || rx >= RX) {
                    free(rayToNuc);
                    return fail(PBS_ERR_GEOMETRY, "dense halo lattice column mapped outside active ray grid");
                }
                rayToNuc[(size_t)ry * RX + rx] = sy * NXn + sx;
            }
        }
    }
    /* Model constants (idd_sigma.cu:102-121) and the GAUSS_FIT entry-sigma scale
     * (wrapper.cu:3788-3795, 3834-3841). */
    double eRefSq = 198.81, sigDelta = 0.21;
    int suppressDip = 0;
    float entryScale = 1.0f;
    if (nuc) {
        if (nucModel == 0) { eRefSq = 190.44; sigDelta = 0.0; }
        else if (nucModel == 1) { eRefSq = 216.09; sigDelta = 0.08; }
        else { eRefSq = 169.00; sigDelta = 0.06; suppressDip = 1; entryScale = 0.97f; }
    }
    double* dens = (double*)malloc(sizeof(double) * S * rays);
    double* wepl = (double*)malloc(sizeof(double) * S * rays);
    int* fin = (int*)malloc(sizeof(int) * rays);
    int* fout = (int*)malloc(sizeof(int) * rays);
    if (P->weq) {
        /* fillBevFromWeqVolumeKernel (wrapper.cu:1923-1989): the ray at
         * origin + index * spacing reads its nearest WEQ texel ([nx][ny][steps],
         * depth fastest); density is the per-step depth increase over the WEQ step;
         * entry/exit from the first/last step with density above 1e-4. */
        const float safeStep = P->weqStepMm > 0.0f ? P->weqStepMm : 1.0f;
        for (int y = 0; y < RY; ++y)
            for (int x = 0; x < RX; ++x) {
                const float rx = P->p.cpb_corner[0] + (float)x * P->p.cpb_res[0];
                const float ry = P->p.cpb_corner[1] + (float)y * P->p.cpb_res[1];
                const int wx = fabsf(P->weqDx) > 0.0f ? (int)lroundf((rx - P->weqX0) / P->weqDx) : -1;
                const int wy = fabsf(P->weqDy) > 0.0f ? (int)lroundf((ry - P->weqY0) / P->weqDy) : -1;
                const int inside = wx >= 0 && wx < P->weqNx && wy >= 0 && wy < P->weqNy;
                float prev = 0.0f, last = 0.0f;
                int firstMat = -1, lastMat = -1;
                size_t idx = (size_t)y * RX + x;
                for (int k = 0; k < S; ++k) {
                    float w = last;
                    if (inside && k < P->weqActive) {
                        w = P->weqBody[((size_t)wx * P->weqNy + wy) * P->weqSteps + k];
                        last = w;
                    }
                    const float d = fmaxf(0.0f, w - prev) / safeStep;
                    wepl[idx] = w;
                    dens[idx] = d;
                    if (d > 1.0e-4f) {
                        if (firstMat < 0) firstMat = k;
                        lastMat = k;
                    }
                    prev = w;
                    idx += rays;
                }
                fin[(size_t)y * RX + x] = firstMat >= 0 ? firstMat + 1 : S;
                fout[(size_t)y * RX + x] = lastMat >= 0 ? lastMat + 1 : 0;
            }
    } else
    /* Trace (bev_ray_tracing.cu:65-159) with double sums; sample points advance by
     * repeated single-precision additions as in the reference. */
#pragma omp parallel for schedule(dynamic, 4)
    for (int y = 0; y < RY; ++y)
        for (int x = 0; x < RX; ++x) {
            V3 st = tr_start(&P->tracer, x, y), inc = tr_inc(&P->tracer, x, y);
            double sl = tr_steplen(&P->tracer, x, y);
            V3 pos = v3(st.x + 0.5f, st.y + 0.5f, st.z + 0.5f);
            double cumSp = 0.0, cumHu = 0.0;
            int before = 0, lastIn = 0, flag = 1;
            size_t idx = (size_t)y * RX + x;
            for (int k = 0; k < S; ++k) {
                double hu = tri_border(ct, cd[0], cd[1], cd[2], pos.x, pos.y, pos.z);
                cumHu += hu;
                dens[idx] = lut1(e->density_vector, e->n_density_samples, hu * e->density_scale_fact + 0.5);
                cumSp += sl * lut1(e->sp_vector, e->n_sp_samples, hu * e->sp_scale_fact + 0.5);
                if (flag && cumHu < 150.0) before = k; else flag = 0;
                if (hu > 150.0) lastIn = k;
                wepl[idx] = cumSp;
                idx += rays;
                pos = vadd(pos, inc);
            }
            fin[(size_t)y * RX + x] = before + 1;
            fout[(size_t)y * RX + x] = lastIn + 1;
        }
    int first = INT_MAX, outMax = INT_MIN;
    for (size_t r = 0; r < rays; ++r) {
        if (fin[r] < first) first = fin[r];
        if (fout[r] > outMax) outMax = fout[r];
    }
    double* wmin = (double*)malloc(sizeof(double) * S);
    for (int k = 0; k < S; ++k) { /* sliceMinVarIgnoreNeverEnter (wrapper.cu:1991-2023) */
        double m = (double)INF20F;
        for (size_t r = 0; r < rays; ++r)
            if (fout[r] > 0 && wepl[(size_t)k * rays + r] < m) m = wepl[(size_t)k * rays + r];
        wmin[k] = m;
    }
    int g0 = ffl_d(wmin, S, BP_CUT * P->p.max_peak_depth_mm);
    int passive = g0 < outMax ? g0 : outMax; /* wrapper.cu:3683-3700 */
    float entryZ = (float)first * P->p.fan_delta[2] + P->p.fan_corner[2];
    float pxX = 1.0f - entryZ / P->p.source_dist[0], pxY = 1.0f - entryZ / P->p.source_dist[1];
    /* Fluence (ray weights per layer). */
    double* rayW = (double*)calloc((size_t)L * rays, sizeof(double));
    float* eSig = (float*)calloc((size_t)L * 2, sizeof(float));
    if (P->p.conv_mode == 0) {
        /* performExactRTDConvolution2D (convolution.cu:198-262, 477-513). */
        const int NX = P->p.lat_nx, NY = P->p.lat_ny;
        for (int l = 0; l < L; ++l) {
            const float* lp = P->lp + 8 * l;
            float a = 0.00270f / (lp[3] - 4.50f), bq = -4.39f / (lp[3] - 3.86f);
            float base = a * entryZ * entryZ + bq * entryZ;
            float sgx = base + lp[6] * lp[6], sgy = base + lp[7] * lp[7];
            eSig[2 * l] = sqrtf(sgx > 0.0f ? sgx : 0.0f);
            eSig[2 * l + 1] = sqrtf(sgy > 0.0f ? sgy : 0.0f);
            if (entryScale != 1.0f) {
                eSig[2 * l] *= entryScale;
                eSig[2 * l + 1] *= entryScale;
            }
        }
#pragma omp parallel for schedule(dynamic, 1)
        for (int l = 0; l < L; ++l) {
            double* interm = (double*)calloc((size_t)NY * RX, sizeof(double));
            const float* lw = P->lat.w + (size_t)l * NX * NY;
            float pixX = P->p.cpb_res[0] * pxX, pixY = P->p.cpb_res[1] * pxY;
            float dX = P->p.lat_dx / P->p.cpb_res[0], oX = (P->p.lat_ox - P->p.cpb_corner[0]) / P->p.cpb_res[0];
            float dY = P->p.lat_dy / P->p.cpb_res[1], oY = (P->p.lat_oy - P->p.cpb_corner[1]) / P->p.cpb_res[1];
            float sX = eSig[2 * l] / pixX, sY = eSig[2 * l + 1] / pixY;
            double rX = 1.0 / (sqrt(2.0) * sX), rY = 1.0 / (sqrt(2.0) * sY);
            float reachX = 3.0f * sX + 0.5f, reachY = 3.0f * sY + 0.5f;
            for (int iy = 0; iy < NY; ++iy)
                for (int x = 0; x < RX; ++x) {
                    double res = 0.0;
                    if (dX > 0.0f && sX > 0.0f) {
                        int i = (int)ceilf(((float)x - reachX - oX) / dX);
                        float dist = (float)i * dX + oX - (float)x;
                        for (int taps = 0; dist < reachX && taps < 65536; ++taps) {
                            if (i >= 0 && i < NX)
                                res += 0.5 * (erfd(((double)dist + 0.5) * rX) - erfd(((double)dist - 0.5) * rX)) *
                                       lw[(size_t)iy * NX + i];
                            ++i;
                            dist = (float)i * dX + oX - (float)x;
                        }
                    }
                    interm[(size_t)iy * RX + x] = res;
                }
            for (int y = 0; y < RY; ++y)
                for (int x = 0; x < RX; ++x) {
                    double res = 0.0;
                    if (dY > 0.0f && sY > 0.0f) {
                        int i = (int)ceilf(((float)y - reachY - oY) / dY);
                        float dist = (float)i * dY + oY - (float)y;
                        for (int taps = 0; dist < reachY && taps < 65536; ++taps) {
                            if (i >= 0 && i < NY)
                                res += 0.5 * (erfd(((double)dist + 0.5) * rY) - erfd(((double)dist - 0.5) * rY)) *
                                       interm[(size_t)i * RX + x];
                            ++i;
                            dist = (float)i * dY + oY - (float)y;
                        }
                    }
                    rayW[(size_t)l * rays + (size_t)y * RX + x] = res;
                }
            free(interm);
        }
    } else {
        /* Legacy CPB fluence (convolution.cu:95-152, 269-339; wrapper.cu:3454-3507). */
        const int M = b->max_subspots_per_layer;
        double* cpb = (double*)calloc((size_t)L * rays, sizeof(double));
        float cX = P->p.cpb_corner[0], cY = P->p.cpb_corner[1], resX = P->p.cpb_res[0], resY = P->p.cpb_res[1];
        for (int l = 0; l < L; ++l)
            for (int m = 0; m < M; ++m) {
                const float* d = b->subspot_data + ((size_t)l * M + m) * 5;
                float px = d[0], py = -d[1], w = d[2], sx = d[3], sy = d[4];
                if (!(w > 1e-6f) || !(sx > 1e-6f) || !(sy > 1e-6f)) continue;
                int x0 = (int)floorf((px - 3.0f * sx - cX) / resX), x1 = (int)ceilf((px + 3.0f * sx - cX) / resX);
                int y0 = (int)floorf((py - 3.0f * sy - cY) / resY), y1 = (int)ceilf((py + 3.0f * sy - cY) / resY);
                if (x0 < 0) x0 = 0;
                if (y0 < 0) y0 = 0;
                if (x1 > RX - 1) x1 = RX - 1;
                if (y1 > RY - 1) y1 = RY - 1;
                for (int cy = y0; cy <= y1; ++cy) {
                    double dy = (double)(cY + ((float)cy + 0.5f) * resY) - py;
                    double ey = erfd((dy + 0.5 * resY) / (sqrt(2.0) * sy)) - erfd((dy - 0.5 * resY) / (sqrt(2.0) * sy));
                    for (int cx = x0; cx <= x1; ++cx) {
                        double dx = (double)(cX + ((float)cx + 0.5f) * resX) - px;
                        double ex = erfd((dx + 0.5 * resX) / (sqrt(2.0) * sx)) - erfd((dx - 0.5 * resX) / (sqrt(2.0) * sx));
                        cpb[((size_t)l * RY + cy) * RX + cx] += 0.25 * ex * ey * w;
                    }
                }
            }
        /* The CPB and ray grids coincide: the area-overlap map is the identity. */
        memcpy(rayW, cpb, sizeof(double) * L * rays);
        free(cpb);
    }
    /* Layers. */
    double* idd = (double*)malloc(sizeof(double) * S * pad);
    double* rsg = (double*)malloc(sizeof(double) * S * pad);
    unsigned char* codes = (unsigned char*)malloc((size_t)S * tiles);
    double* bevL = (double*)malloc(sizeof(double) * S * bevPlane);
    double* bevSum = cap && cap->bev ? cap->bev : NULL;
    if (bevSum) memset(bevSum, 0, sizeof(double) * S * bevPlane);
    double *nIdd = NULL, *nRsg = NULL, *nBevL = NULL, *nBevSum = NULL;
    unsigned char* nCodes = NULL;
    if (nuc) {
        nIdd = (double*)malloc(sizeof(double) * S * nucPad);
        nRsg = (double*)malloc(sizeof(double) * S * nucPad);
        nCodes = (unsigned char*)malloc((size_t)S * nucTiles);
        nBevL = (double*)malloc(sizeof(double) * S * nucBevPlane);
        nBevSum = cap && cap->nuc_bev ? cap->nuc_bev : NULL;
        if (nBevSum) memset(nBevSum, 0, sizeof(double) * S * nucBevPlane);
    }
    int maxCalc = first;
    double fmaTotal = 0.0, nucFmaTotal = 0.0;
    int rc = PBS_OK;
    const double NaNinf = INFINITY;
    const int nS = e->n_energy_samples, nE = e->n_energies;
    double* row = (double*)malloc(sizeof(double) * nS);
    double* nwRow = (double*)malloc(sizeof(double) * nS);
    double* nsRow = (double*)malloc(sizeof(double) * nS);
    for (int l = 0; l < L && rc == PBS_OK; ++l) {
        const float* lp = P->lp + 8 * l;
        const float eIdx = lp[0], escale = lp[1], peak = lp[2];
        const float rangeStop = BP_CUT * peak;
        int afterLastL = ffl_d(wmin, S, BP_CUT * peak);
        if (afterLastL > passive) afterLastL = passive;
        /* CIDD (and nuclear) rows at this energy. */
        table_row(e->cidd_matrix, nE, nS, eIdx, row);
        /* Halo inputs of the layer (wrapper.cu:4111-4135, 4140-4386). */
        float spotDist = 0.0f, entrySigmaSq = 0.0f;
        const float* haloW = NULL;
        if (nuc) {
            table_row(e->nuc_weight_matrix, nE, nS, eIdx, nwRow);
            table_row(e->nuc_sq_sigma_matrix, nE, nS, eIdx, nsRow);
            haloW = P->lat.w + (size_t)l * P->lat.nx * P->lat.ny;
            const float spacing = b->spot_delta[0] > b->ray_spacing[0] * 1.5f ? b->spot_delta[0] : P->lat.dx;
            if (fabsf(P->p.fan_delta[0]) > 1e-6f) spotDist = fabsf(spacing / P->p.fan_delta[0]);
            const float a = 0.00270f / (peak - 4.50f), bq = -4.39f / (peak - 3.86f);
            entrySigmaSq = a * entryZ * entryZ + bq * entryZ + lp[6] * lp[6];
        }
        const int nucOn = nuc && spotDist > 0.0f;
        const double rEref = nucOn ? eRefSq : 198.81, rDelta = nucOn ? sigDelta : 0.21;
        const int rSuppress = nucOn ? suppressDip : 0;
        /* CarbonPBS profile model of the layer: what each switch runs on this beam
         * (raytracedicom_wrapper.cu:4656-4660, 4814-4818, and the kernels' own early
         * returns), the table row and the interpolated beam parameters (4592-4606). */
        ProfileC pc;
        profile_shape(b, L, &pc);
        const int pOverride = (g_profile & 1) && pc.table && pc.beamPara && pc.channels >= 3 &&
                              (pc.channels - 1) / 2 > 0 && pc.depthStep > 0.0f;
        const int pWeight = (g_profile & 2) && pc.table && pc.channels > 0 && pc.depthStep > 0.0f;
        const float pRow = profile_row(b, e, &pc, L, l, eIdx);
        double bp[3] = {0.0, 0.0, 0.0};
        if (pc.rows > 0 && b->beam_para_data && b->n_beam_para_data >= (size_t)pc.rows * 3u) {
            const float cr = fminf(fmaxf(pRow, 0.0f), (float)(pc.rows - 1));
            int i0 = (int)floorf(cr);
            if (i0 < 0) i0 = 0;
            if (i0 > pc.rows - 1) i0 = pc.rows - 1;
            const int i1 = i0 + 1 < pc.rows ? i0 + 1 : pc.rows - 1;
            const float t = cr - (float)i0;
            for (int k = 0; k < 3; ++k) {
                const float v0 = b->beam_para_data[(size_t)i0 * 3 + k], v1 = b->beam_para_data[(size_t)i1 * 3 + k];
                bp[k] = v0 + (v1 - v0) * t;
            }
        }
        for (size_t i = 0; i < (size_t)S * pad; ++i) { idd[i] = 0.0; rsg[i] = NaNinf; }
        if (nucOn)
            for (size_t i = 0; i < (size_t)S * nucPad; ++i) { nIdd[i] = 0.0; nRsg[i] = NaNinf; }
        int maxFP = INT_MIN;
        const double quad = lp[4], lin = lp[5];
        const double stepLen = fabs((double)P->p.fan_delta[2]);
        /* fillIddAndSigmaKernel (idd_sigma.cu:46-259). A ray without a halo cell
         * writes no halo value (the reference offsets its -1 index by the first
         * step before testing it, idd_sigma.cu:131-137, and so races on the last
         * halo cell of the previous plane). */
#pragma omp parallel for schedule(dynamic, 8) reduction(max : maxFP)
        for (int y = 0; y < RY; ++y)
            for (int x = 0; x < RX; ++x) {
                size_t r = (size_t)y * RX + x;
                int firstIn = fin[r];
                int al0 = fout[r] < afterLastL ? fout[r] : afterLastL;
                unsigned afterLast = (unsigned)al0;
                double w = rayW[(size_t)l * rays + r];
                const int nIdx = nucOn ? rayToNuc[r] : -1;
                const double nW = nIdx >= 0 ? (double)haloW[(nIdx / NXn) * P->lat.nx + nIdx % NXn] : 0.0;
                int live = 1;
                if (w < 1e-6 || afterLast < (unsigned)first) { live = 0; afterLast = 0; }
                double spOld = 0.0, cdOld = 0.0, incScat = 0.0, incinc = 0.0;
                double incDiv = lin + (2.0 * first - 1.0) * quad;
                double sig2 = -incDiv;
                for (int k = first; k < afterLastL; ++k) {
                    double res = 0.0, rs = NaNinf, nRes = 0.0, nRs = NaNinf;
                    if (live) {
                        size_t idx = (size_t)k * rays + r;
                        double sp = wepl[idx];
                        double cd_ = row_lookup(row, nS, sp * escale + 0.5);
                        double rho = dens[idx];
                        if (sp < peak) {
                            double resE = 8.639415 * pow((double)peak - 0.5 * (sp + spOld), 0.5649718);
                            double betaP = resE + 938.3 - 938.3 * 938.3 / (resE + 938.3);
                            double rRl = rho * lut1(e->rrl_vector, e->n_rrl_samples, rho * e->rrl_scale_fact + 0.5);
                            double th2 = rEref / (betaP * betaP) * stepLen * rRl;
                            sig2 += incScat + incDiv;
                            incinc += 2.0 * th2 * stepLen * stepLen;
                            incScat += incinc;
                            incDiv += 2.0 * quad;
                        } else if (!rSuppress) {
                            sig2 -= 1.5 * (incScat + incDiv) * rho;
                        }
                        double zk = (double)P->p.fan_corner[2] + (double)k * P->p.fan_delta[2];
                        double vwx = P->p.fan_delta[0] * (1.0 - zk / P->p.source_dist[0]);
                        double vwy = P->p.fan_delta[1] * (1.0 - zk / P->p.source_dist[1]);
                        rs = 0.5 * (vwx + vwy) / (sqrt(2.0) * (sqrt(sig2) + rDelta));
                        double kk = (double)k;
                        double vol = (double)P->volConst + kk * P->volLin + kk * kk * P->volSq;
                        double mass = rho * vol;
                        double depthMid = 0.5 * (sp + spOld) * escale + 0.5;
                        if (mass > 1e-2) {
                            if (nucOn) {
                                double nw = row_lookup(nwRow, nS, depthMid);
                                res = (1.0 - nw) * w * (cd_ - cdOld) / mass;
                                if (nIdx >= 0) nRes = nw * nW * (cd_ - cdOld) / (mass * (double)spotDist * spotDist);
                            } else {
                                res = w * (cd_ - cdOld) / mass;
                            }
                        }
                        if (nucOn && nIdx >= 0) {
                            double ns2 = row_lookup(nsRow, nS, depthMid);
                            nRs = 0.5 * spotDist * (vwx + vwy) / (sqrt(2.0) * sqrt(sig2 + ns2 + (double)entrySigmaSq));
                        }
                        spOld = sp;
                        cdOld = cd_;
                        if (sp > (double)rangeStop || (unsigned)k == afterLast) { live = 0; afterLast = (unsigned)k; }
                    }
                    if (!live || k < firstIn - 1) { res = 0.0; rs = NaNinf; nRes = 0.0; nRs = NaNinf; }
                    if (pOverride || pWeight) {
                        const double sp = wepl[(size_t)k * rays + r];
                        double dI = (sp - pc.depth0) / pc.depthStep;
                        if (dI < 0.0) dI = 0.0;
                        if (dI > pc.depthN - 1) dI = pc.depthN - 1;
                        if (pOverride) {
                            if (!(res > 0.0)) {
                                rs = NaNinf;
                            } else {
                                const int nG = (pc.channels - 1) / 2;
                                double sumW = 0.0, sumS2 = 0.0;
                                for (int gi = 0; gi < nG; ++gi) {
                                    const double wv = profile_at(b->profile_data, &pc, gi, dI, pRow);
                                    const double sv = profile_at(b->profile_data, &pc, gi + nG, dI, pRow);
                                    sumW += wv;
                                    sumS2 += wv * sv * sv;
                                }
                                if (!(sumW > 1.0e-8)) {
                                    rs = NaNinf;
                                } else {
                                    const double sad = 0.5 * ((double)P->p.source_dist[0] + P->p.source_dist[1]);
                                    const double fx = (double)P->p.fan_corner[0] + x * (double)P->p.fan_delta[0];
                                    const double fy = (double)P->p.fan_corner[1] + y * (double)P->p.fan_delta[1];
                                    const double fz = (double)P->p.fan_corner[2] + k * (double)P->p.fan_delta[2];
                                    const double sdx = P->p.source_dist[0], sdy = P->p.source_dist[1];
                                    const double proj = (sad - fz) * sqrt(1.0 + fx * fx / (sdx * sdx) + fy * fy / (sdy * sdy));
                                    const double phy = proj - (sad - (double)b->beam_para_pos);
                                    const double r2 = bp[0] + 2.0 * bp[1] * phy + bp[2] * phy * phy;
                                    double ax2 = r2 + sumS2 / sumW;
                                    ax2 = 0.5 * (ax2 > 0.0 ? ax2 : 0.0);
                                    const double zk = (double)P->p.fan_corner[2] + (double)k * P->p.fan_delta[2];
                                    const double vx = P->p.fan_delta[0] * (1.0 - zk / P->p.source_dist[0]);
                                    const double vy = P->p.fan_delta[1] * (1.0 - zk / P->p.source_dist[1]);
                                    rs = 0.5 * (0.5 * (vx + vy)) / (sqrt(2.0) * (sqrt(ax2) + 0.21));
                                }
                            }
                        }
                        if (pWeight && res > 0.0) {
                            const double ow = profile_at(b->profile_data, &pc, pc.channels - 1, dI, pRow);
                            res *= ow > 0.0 ? ow : 0.0;
                        }
                    }
                    idd[(size_t)k * pad + (size_t)y * PX + x] = res;
                    rsg[(size_t)k * pad + (size_t)y * PX + x] = rs;
                    if (nIdx >= 0) {
                        nIdd[(size_t)k * nucPad + nIdx] = nRes;
                        nRsg[(size_t)k * nucPad + nIdx] = nRs;
                    }
                }
                if ((int)afterLast > maxFP) maxFP = (int)afterLast;
            }
        /* beamFirstCalculatedPassive (wrapper.cu:4975-4990). */
        int calc = maxFP;
        if (calc < first + 1) calc = first + 1;
        if (calc < 0) calc = first + 1;
        if (calc > afterLastL) calc = afterLastL;
        if (calc > S) calc = S;
        if (calc > maxCalc) maxCalc = calc;
        /* Tile radius buckets (tileRadCalc, complete_superposition.cu:198-255). */
        memset(codes, 0xff, (size_t)S * tiles);
        int hist[34] = {0}, live = 0;
        for (int k = first; k < afterLastL; ++k) {
            tile_codes(idd + (size_t)k * pad, rsg + (size_t)k * pad, PX, TX, TY, codes + (size_t)k * tiles);
            if (k < calc)
                for (size_t t = 0; t < tiles; ++t) {
                    unsigned char c = codes[(size_t)k * tiles + t];
                    hist[c & 0x3f]++;
                    live += (c & 0x80) ? 1 : 0;
                }
        }
        int batched[33], map[34];
        oracle_batch(hist, batched, map);
        /* Superposition at the batched radius into the layer BEV at absolute steps. */
        memset(bevL, 0, sizeof(double) * S * bevPlane);
        double fmaL = 0.0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : fmaL)
        for (int k = first; k < calc; ++k)
            fmaL += superpose_step(idd + (size_t)k * pad, rsg + (size_t)k * pad, codes + (size_t)k * tiles, map, PX,
                                   TX, TY, bevL + (size_t)k * bevPlane, BX);
        fmaTotal += fmaL;
        if (bevSum)
            for (size_t i = 0; i < (size_t)S * bevPlane; ++i) bevSum[i] += bevL[i];
        int box[6];
        transfer_layer(&P->fanToDose, PX, PY, first, calc, passive, compat, bevL, BX, BY, dose, dd, box);
        if (g_bio && g_bioAcc) {
            /* Biological channels with the layer's radii: IDD x factor, superposed
             * and transferred like the dose; the layer's dose into accumulator 0. */
            const size_t nGrid = (size_t)dd[0] * dd[1] * dd[2];
            int bbox[6];
            transfer_layer(&P->fanToDose, PX, PY, first, calc, passive, compat, bevL, BX, BY, g_bioAcc, dd, bbox);
            const double bioRow = frac_index_monotonic(g_bio->let_energies, g_bio->let_rows, b->energies[l]);
            double* cIdd = (double*)malloc(sizeof(double) * S * pad);
            double* cBev = (double*)malloc(sizeof(double) * S * bevPlane);
            for (int c = 0; c < 3; ++c) {
                if (c == 1 && g_bio->model != PBS_BIO_LQ) continue;
                for (size_t i = 0; i < (size_t)S * pad; ++i) cIdd[i] = 0.0;
#pragma omp parallel for schedule(static)
                for (int k = first; k < afterLastL; ++k)
                    for (int y = 0; y < RY; ++y)
                        for (int x = 0; x < RX; ++x) {
                            const size_t o = (size_t)k * pad + (size_t)y * PX + x;
                            if (!(idd[o] > 0.0)) continue;
                            const double let = bio_let(g_bio, bioRow, wepl[(size_t)k * rays + (size_t)y * RX + x]);
                            cIdd[o] = idd[o] * bio_factor(g_bio, c, let);
                        }
                memset(cBev, 0, sizeof(double) * S * bevPlane);
#pragma omp parallel for schedule(dynamic, 1)
                for (int k = first; k < calc; ++k)
                    superpose_step(cIdd + (size_t)k * pad, rsg + (size_t)k * pad, codes + (size_t)k * tiles, map, PX,
                                   TX, TY, cBev + (size_t)k * bevPlane, BX);
                transfer_layer(&P->fanToDose, PX, PY, first, calc, passive, compat, cBev, BX, BY,
                               g_bioAcc + (size_t)(c + 1) * nGrid, dd, bbox);
            }
            free(cIdd);
            free(cBev);
        }
        /* Nuclear halo: tile radii over [first, calc) with no overflow merge
         * (complete_superposition.cu:558-708), superposition on the halo grid and
         * its own transfer (wrapper.cu:5510-5600, prim_transf_kernel.cu:46-78). */
        int nHist[34] = {0}, nBatched[33] = {0}, nMap[34];
        if (nucOn) {
            memset(nCodes, 0xff, (size_t)S * nucTiles);
            for (int k = first; k < calc; ++k) {
                tile_codes(nIdd + (size_t)k * nucPad, nRsg + (size_t)k * nucPad, NXn, NTX, NTY,
                           nCodes + (size_t)k * nucTiles);
                for (size_t t = 0; t < nucTiles; ++t) nHist[nCodes[(size_t)k * nucTiles + t] & 0x3f]++;
            }
            if (nHist[MAX_R + 1] > 0) {
                rc = fail(PBS_ERR_UNSUPPORTED, "nuclear superposition radius exceeds 32 (the reference throws, "
                                               "complete_superposition.cu:609-627)");
            } else {
                oracle_batch(nHist, nBatched, nMap);
                memset(nBevL, 0, sizeof(double) * S * nucBevPlane);
                double nf = 0.0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : nf)
                for (int k = first; k < calc; ++k)
                    nf += superpose_step(nIdd + (size_t)k * nucPad, nRsg + (size_t)k * nucPad,
                                         nCodes + (size_t)k * nucTiles, nMap, NXn, NTX, NTY,
                                         nBevL + (size_t)k * nucBevPlane, NBX);
                nucFmaTotal += nf;
                if (nBevSum)
                    for (size_t i = 0; i < (size_t)S * nucBevPlane; ++i) nBevSum[i] += nBevL[i];
                FromFan nf2d = P->fanToDose;
                nf2d.fan = idxt(v3(P->lat.dx, P->lat.dy, P->p.fan_delta[2]), v3(P->lat.ox, P->lat.oy, P->p.fan_corner[2]));
                int nbox[6];
                transfer_layer(&nf2d, NXn, NYn, first, calc, passive, compat, nBevL, NBX, NBY, dose, dd, nbox);
            }
        }
        if (cap) {
            if (cap->idd) memcpy(cap->idd + (size_t)l * S * pad, idd, sizeof(double) * S * pad);
            if (cap->rsigma) memcpy(cap->rsigma + (size_t)l * S * pad, rsg, sizeof(double) * S * pad);
            if (cap->codes) memcpy(cap->codes + (size_t)l * S * tiles, codes, (size_t)S * tiles);
            if (cap->layer_ints) {
                int* li = cap->layer_ints + 8 * l;
                li[0] = afterLastL; li[1] = maxFP; li[2] = calc; li[3] = live;
            }
            if (cap->layer_box) memcpy(cap->layer_box + 6 * l, box, sizeof box);
            if (cap->hist) memcpy(cap->hist + 34 * l, hist, sizeof hist);
            if (cap->batched) memcpy(cap->batched + 33 * l, batched, sizeof batched);
            if (nucOn) {
                if (cap->nuc_idd) memcpy(cap->nuc_idd + (size_t)l * S * nucPad, nIdd, sizeof(double) * S * nucPad);
                if (cap->nuc_rsigma) memcpy(cap->nuc_rsigma + (size_t)l * S * nucPad, nRsg, sizeof(double) * S * nucPad);
                if (cap->nuc_codes) memcpy(cap->nuc_codes + (size_t)l * S * nucTiles, nCodes, (size_t)S * nucTiles);
                if (cap->nuc_hist) memcpy(cap->nuc_hist + 34 * l, nHist, sizeof nHist);
                if (cap->nuc_batched) memcpy(cap->nuc_batched + 33 * l, nBatched, sizeof nBatched);
            }
        }
    }
    free(row); free(nwRow); free(nsRow);
    if (cap) {
        if (cap->density) memcpy(cap->density, dens, sizeof(double) * S * rays);
        if (cap->wepl) memcpy(cap->wepl, wepl, sizeof(double) * S * rays);
        if (cap->first_inside) memcpy(cap->first_inside, fin, sizeof(int) * rays);
        if (cap->first_outside) memcpy(cap->first_outside, fout, sizeof(int) * rays);
        if (cap->wepl_min) memcpy(cap->wepl_min, wmin, sizeof(double) * S);
        if (cap->ray_weights) memcpy(cap->ray_weights, rayW, sizeof(double) * L * rays);
        if (cap->entry_sigma) memcpy(cap->entry_sigma, eSig, sizeof(float) * L * 2);
        if (cap->beam_ints) {
            cap->beam_ints[0] = first;
            cap->beam_ints[1] = outMax;
            cap->beam_ints[2] = passive;
            cap->beam_ints[3] = maxCalc;
        }
        cap->superpose_fma = fmaTotal;
        cap->nuc_superpose_fma = nucFmaTotal;
        if (cap->ray_to_nuc && rayToNuc) memcpy(cap->ray_to_nuc, rayToNuc, sizeof(int) * rays);
    }
    free(dens); free(wepl); free(fin); free(fout); free(wmin); free(rayW); free(eSig);
    free(idd); free(rsg); free(codes); free(bevL);
    free(nIdd); free(nRsg); free(nCodes); free(nBevL); free(rayToNuc);
    return rc;
}

int oracle_dose(const float* ct, const int cd[3], const float cr[3], const float cc[3], double* dose,
                const int dd[3], const float dr[3], const float dc[3], const PbsBeamDesc* beams, size_t nb,
                const PbsEnergyDesc* e, int ct_type, int compat, int threads, OracleCapture* cap) {
    return oracle_dose_nuclear(ct, cd, cr, cc, dose, dd, dr, dc, beams, nb, e, ct_type, compat, -1, threads, cap);
}

int oracle_dose_nuclear(const float* ct, const int cd[3], const float cr[3], const float cc[3], double* dose,
                        const int dd[3], const float dr[3], const float dc[3], const PbsBeamDesc* beams, size_t nb,
                        const PbsEnergyDesc* e, int ct_type, int compat, int nucModel, int threads,
                        OracleCapture* cap) {
    if (!ct || !dose || !beams || !e || nb == 0) return fail(PBS_ERR_INVALID_ARGUMENT, "null input");
    if (nucModel > 2) return fail(PBS_ERR_INVALID_ARGUMENT, "unknown nuclear model");
    if (nucModel >= 0) { /* enforceNuclearCorrectionContract (wrapper.cu:1077-1097) */
        const size_t n = (size_t)e->n_energies * e->n_energy_samples;
        if (!e->nuc_weight_matrix || !e->nuc_sq_sigma_matrix || e->n_nuc_weight_matrix != n ||
            e->n_nuc_sq_sigma_matrix != n)
            return fail(PBS_ERR_INVALID_ARGUMENT, "nuclear_correction=true requested, but the energy tables do not "
                                                  "carry nuclear_weight/sigma tables");
        if (!e->nuclear_tables_aligned_to_primary_axis)
            return fail(PBS_ERR_INVALID_ARGUMENT, "nuclear_correction=true requested, but nuclear LUTs are not "
                                                  "aligned to the active primary energy-depth axis");
    }
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#else
    (void)threads;
#endif
    size_t n = (size_t)cd[0] * cd[1] * cd[2];
    int type = ct_type == PBS_CT_AUTO ? detect_ct_type(ct, n) : ct_type;
    float* hu = (float*)malloc(sizeof(float) * n);
    if (type == PBS_CT_HU) {
        for (size_t i = 0; i < n; ++i) hu[i] = ct[i] + 1000.0f;
    } else if (type == PBS_CT_DENSITY || type == PBS_CT_SPR) {
        const float* lut = type == PBS_CT_DENSITY ? e->density_vector : e->sp_vector;
        int ln = (int)(type == PBS_CT_DENSITY ? e->n_density_vector : e->n_sp_vector);
        float sc = type == PBS_CT_DENSITY ? e->density_scale_fact : e->sp_scale_fact;
        for (size_t i = 0; i < n; ++i) hu[i] = frac_index_monotonic(lut, ln, ct[i]) / sc;
    } else {
        memcpy(hu, ct, sizeof(float) * n);
    }
    int rc = PBS_OK;
    for (size_t bi = 0; bi < nb && !rc; ++bi) {
        Plan P;
        rc = plan_beam(&beams[bi], e, cd, cr, cc, dd, dr, dc, &P);
        if (!rc) rc = run_beam(hu, cd, dose, dd, &beams[bi], e, &P, compat, nucModel, bi + 1 == nb ? cap : NULL);
        free_plan(&P);
    }
    free(hu);
    return rc;
}
