// Host-side beam planning. Float arithmetic is plain IEEE single precision,
// evaluated in the reference's operand order and compiled without FMA
// contraction, so the integer decisions match the reference's host code.
#include "plan.h"

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <cctype>
#include <cmath>
#include <cstdlib>
#include <string>
#include <thread>
#include <vector>

namespace pbs {

namespace {

// The reference's INF macro is the double 1.0e20 (include/core/Macro.cuh:7) and is
// stored into floats.
const float kInfF = static_cast<float>(1.0e20);

bool host_finite(float v) { return std::isfinite(v); }

int round_up(int v, int m) { return m <= 1 ? v : ((v + m - 1) / m) * m; }

V3 normalize_safe(V3 v) {
    const float len = std::sqrt(dot(v, v));
    if (len > 1e-8f) v = divs(v, len);
    return v;
}

std::string str_lower(const char* s) {
    std::string r(s);
    for (char& c : r) c = static_cast<char>(std::tolower(static_cast<unsigned char>(c)));
    return r;
}

// wrapper.cu:970-997
bool align_grid_to_reference_phase(float minCoord, float maxCoord, float refOrigin, float step, int multiple,
                                   float& origin, int& count) {
    if (!(step > 0.0f) || !host_finite(minCoord) || !host_finite(maxCoord) || !host_finite(refOrigin)) return false;
    if (maxCoord < minCoord) std::swap(minCoord, maxCoord);
    const float eps = 1.0e-4f;
    const int firstStep = static_cast<int>(std::ceil((minCoord - refOrigin) / step - eps));
    const int lastStep = static_cast<int>(std::floor((maxCoord - refOrigin) / step + eps));
    if (lastStep < firstStep) return false;
    origin = refOrigin + static_cast<float>(firstStep) * step;
    count = std::max(1, lastStep - firstStep + 1);
    if (multiple > 1) count = ((count + multiple - 1) / multiple) * multiple;
    return true;
}

const float* active_weq_header(const PbsBeamDesc& b, size_t& n) {
    if (b.water_equivalence && b.n_water_equivalence >= 9) {
        n = b.n_water_equivalence;
        return b.water_equivalence;
    }
    n = b.ray_weq_header ? b.n_ray_weq_header : 0;
    return b.ray_weq_header;
}

// wrapper.cu:1004-1023
bool decode_spot_position(const PbsBeamDesc& b, const float* hdr, size_t nh, float rawX, float rawY, float& x,
                          float& y) {
    if (!b.spot_positions_are_indices) {
        x = rawX;
        y = rawY;
        return true;
    }
    if (nh < 9) return false;
    x = hdr[6] + (rawX - 0.5f) * hdr[7];
    y = hdr[3] + (rawY - 0.5f) * hdr[4];
    return true;
}

// wrapper.cu:931-968
bool rasterize_continuous(std::vector<float>& dense, int nx, int ny, int layer, float lx, float ly, float w) {
    if (nx <= 0 || ny <= 0 || layer < 0 || dense.empty()) return false;
    const int ix0 = static_cast<int>(std::floor(lx));
    const int iy0 = static_cast<int>(std::floor(ly));
    const float tx = lx - static_cast<float>(ix0);
    const float ty = ly - static_cast<float>(iy0);
    double written = 0.0;
    auto acc = [&](int ix, int iy, float frac) {
        if (!(frac > 0.0f)) return;
        if (ix < 0 || ix >= nx || iy < 0 || iy >= ny) return;
        dense[(static_cast<size_t>(layer) * ny + iy) * nx + ix] += w * frac;
        written += static_cast<double>(w) * static_cast<double>(frac);
    };
    acc(ix0, iy0, (1.0f - tx) * (1.0f - ty));
    acc(ix0 + 1, iy0, tx * (1.0f - ty));
    acc(ix0, iy0 + 1, (1.0f - tx) * ty);
    acc(ix0 + 1, iy0 + 1, tx * ty);
    return written > 0.0;
}

// wrapper.cu:1259-1473
bool build_raw_lattice(const PbsBeamDesc& b, RawLattice& out) {
    out = RawLattice{};
    auto fail = [&](const std::string& m) {
        out.failure = m;
        return false;
    };
    const int L = static_cast<int>(b.n_energies);
    if (!b.layer_spot_counts || b.n_layer_spot_counts == 0 || !b.spot_positions || b.n_spot_positions == 0 ||
        !b.spot_weights || b.n_spot_weights == 0)
        return fail("missing layerSpotCounts/spotPositions/spotWeights input");
    if (static_cast<int>(b.n_layer_spot_counts) != L) return fail("layerSpotCounts size does not match energies");
    if (b.n_spot_positions % 2 != 0) return fail("spotPositions does not contain [N][2] rows");
    int total = 0;
    for (int l = 0; l < L; ++l) total += b.layer_spot_counts[l];
    if (total <= 0) return fail("beam contains no spots");
    if (static_cast<int>(b.n_spot_positions / 2) != total) return fail("spotPositions rows != summed layerSpotCounts");
    if (static_cast<int>(b.n_spot_weights) != total) return fail("spotWeights size != summed layerSpotCounts");
    size_t nh = 0;
    const float* hdr = active_weq_header(b, nh);
    if (b.spot_positions_are_indices && nh < 9) return fail("spotPositionsAreIndices requires a 9-value WEQ header");

    if (b.spot_positions_are_indices) {
        const int nx = std::max(1, static_cast<int>(std::lround(hdr[8])));
        const int ny = std::max(1, static_cast<int>(std::lround(hdr[5])));
        std::vector<float> dense(static_cast<size_t>(nx) * ny * L, 0.0f);
        int off = 0;
        for (int l = 0; l < L; ++l) {
            const int cnt = b.layer_spot_counts[l];
            if (cnt <= 0) return false;
            for (int i = 0; i < cnt; ++i) {
                const int s = off + i;
                const float w = b.spot_weights[s];
                if (!host_finite(w)) return fail("non-finite spot weight");
                if (w < 0.0f) return fail("negative spot weight");
                if (w == 0.0f) {
                    out.skippedZeroWeightSpots++;
                    continue;
                }
                const float lx = b.spot_positions[2 * s] - 0.5f;
                const float ly = b.spot_positions[2 * s + 1] - 0.5f;
                if (!rasterize_continuous(dense, nx, ny, l, lx, ly, w))
                    return fail("positive-weight spot could not be rasterized onto rayweq lattice");
            }
            off += cnt;
        }
        out.valid = true;
        out.nx = nx;
        out.ny = ny;
        out.nl = L;
        out.dx = hdr[7];
        out.dy = hdr[4];
        out.ox = hdr[6];
        out.oy = hdr[3];
        out.weights = std::move(dense);
        return true;
    }

    std::vector<float> xs(total), ys(total);
    for (int i = 0; i < total; ++i) {
        if (!decode_spot_position(b, hdr, nh, b.spot_positions[2 * i], b.spot_positions[2 * i + 1], xs[i], ys[i]))
            return fail("failed to decode spot position");
    }
    auto unique_axis = [](std::vector<float> v) {
        // Exact duplicates (every layer repeats the spot grid) cannot change the
        // tolerance merge below, so they are dropped before the sort (open
        // addressing on the bit patterns; 0xffffffff, a NaN, marks a free slot).
        size_t cap = 16;
        while (cap < 2 * v.size()) cap <<= 1;
        std::vector<uint32_t> table(cap, 0xffffffffu);
        size_t n = 0;
        for (float x : v) {
            uint32_t bits;
            std::memcpy(&bits, &x, sizeof(bits));
            if (bits == 0xffffffffu) {
                v[n++] = x;
                continue;
            }
            size_t h = (bits * 2654435761u) & (cap - 1);
            while (table[h] != 0xffffffffu && table[h] != bits) h = (h + 1) & (cap - 1);
            if (table[h] == 0xffffffffu) {
                table[h] = bits;
                v[n++] = x;
            }
        }
        v.resize(n);
        std::sort(v.begin(), v.end());
        std::vector<float> u;
        for (float x : v)
            if (u.empty() || !(std::fabs(u.back() - x) <= 1e-4f)) u.push_back(x);
        return u;
    };
    auto grid_step = [](const std::vector<float>& u) {
        float step = kInfF;
        for (size_t i = 1; i < u.size(); ++i) {
            const float d = u[i] - u[i - 1];
            if (d > 1.0e-4f && d < step) step = d;
        }
        // The reference compares this float against the double 1e20, which never
        // holds, so a single-column axis keeps the 1e20 step.
        return step;
    };
    // A layer that repeats the previous layer's positions bit for bit adds no new
    // axis values: only the first of such a run enters the merge.
    std::vector<float> axX, axY;
    axX.reserve(xs.size());
    axY.reserve(ys.size());
    for (int l = 0, o = 0, po = -1, pc = -1; l < L; o += b.layer_spot_counts[l], ++l) {
        const int c = b.layer_spot_counts[l];
        if (c <= 0) return false;  // as the weight pass below refuses it
        const bool rep = c == pc && std::memcmp(xs.data() + o, xs.data() + po, sizeof(float) * size_t(c)) == 0 &&
                         std::memcmp(ys.data() + o, ys.data() + po, sizeof(float) * size_t(c)) == 0;
        if (!rep) {
            axX.insert(axX.end(), xs.begin() + o, xs.begin() + o + c);
            axY.insert(axY.end(), ys.begin() + o, ys.begin() + o + c);
        }
        po = o;
        pc = c;
    }
    const std::vector<float> ux = unique_axis(std::move(axX)), uy = unique_axis(std::move(axY));
    if (ux.empty() || uy.empty()) return fail("empty lattice axes");
    const float dx = grid_step(ux), dy = grid_step(uy);
    const float ox = ux.front(), oy = uy.front();
    const int nx = std::max(1, static_cast<int>(std::lround((ux.back() - ox) / dx)) + 1);
    const int ny = std::max(1, static_cast<int>(std::lround((uy.back() - oy) / dy)) + 1);
    std::vector<float> dense(static_cast<size_t>(nx) * ny * L, 0.0f);
    // Lattice cell of every spot (-1: outside, -2: off the lattice phase). A layer
    // whose positions repeat the previous layer's bit for bit reuses its cells.
    std::vector<int> cell(static_cast<size_t>(total));
    int off = 0, prevOff = -1, prevCnt = -1;
    for (int l = 0; l < L; ++l) {
        const int cnt = b.layer_spot_counts[l];
        if (cnt <= 0) return false;
        const bool same = cnt == prevCnt &&
                          std::memcmp(xs.data() + off, xs.data() + prevOff, sizeof(float) * size_t(cnt)) == 0 &&
                          std::memcmp(ys.data() + off, ys.data() + prevOff, sizeof(float) * size_t(cnt)) == 0;
        for (int i = 0; i < cnt; ++i) {
            const int s = off + i;
            if (same) {
                cell[s] = cell[prevOff + i];
                continue;
            }
            const float x = xs[s], y = ys[s];
            const float fx = (dx != 0.0f) ? ((x - ox) / dx) : 0.0f;
            const float fy = (dy != 0.0f) ? ((y - oy) / dy) : 0.0f;
            const int ix = static_cast<int>(std::lround(fx));
            const int iy = static_cast<int>(std::lround(fy));
            if (ix < 0 || ix >= nx || iy < 0 || iy >= ny)
                cell[s] = -1;
            else if (!(std::fabs(ox + ix * dx - x) <= 2e-2f) || !(std::fabs(oy + iy * dy - y) <= 2e-2f))
                cell[s] = -2;
            else
                cell[s] = iy * nx + ix;
        }
        for (int i = 0; i < cnt; ++i) {
            const int s = off + i;
            const float w = b.spot_weights[s];
            if (!host_finite(w)) return fail("non-finite spot weight");
            if (w < 0.0f) return fail("negative spot weight");
            if (w == 0.0f) {
                out.skippedZeroWeightSpots++;
                continue;
            }
            if (cell[s] == -1) return fail("spot outside inferred lattice bounds");
            if (cell[s] == -2) return fail("spot does not align with inferred lattice phase");
            dense[static_cast<size_t>(l) * ny * nx + cell[s]] += w;
        }
        prevOff = off;
        prevCnt = cnt;
        off += cnt;
    }
    out.valid = true;
    out.nx = nx;
    out.ny = ny;
    out.nl = L;
    out.dx = dx;
    out.dy = dy;
    out.ox = ox;
    out.oy = oy;
    out.weights = std::move(dense);
    return true;
}

// wrapper.cu:1822-1845
bool decoded_spot_bounds(const PbsBeamDesc& b, float& minX, float& maxX, float& minY, float& maxY) {
    if (!b.layer_spot_counts || b.n_layer_spot_counts == 0 || !b.spot_positions || b.n_spot_positions == 0)
        return false;
    size_t nh = 0;
    const float* hdr = active_weq_header(b, nh);
    if (b.spot_positions_are_indices && nh < 9) return false;
    minX = kInfF;
    maxX = -kInfF;
    minY = kInfF;
    maxY = -kInfF;
    const int total = static_cast<int>(b.n_spot_positions / 2);
    for (int i = 0; i < total; ++i) {
        float x = 0.f, y = 0.f;
        if (!decode_spot_position(b, hdr, nh, b.spot_positions[2 * i], b.spot_positions[2 * i + 1], x, y))
            return false;
        minX = std::min(minX, x);
        maxX = std::max(maxX, x);
        minY = std::min(minY, y);
        maxY = std::max(maxY, y);
    }
    return minX <= maxX && minY <= maxY;
}

// wrapper.cu:1847-1921
bool estimate_virtual_source_distances(const PbsBeamDesc& b, V3 bmX, V3 bmY, V3 bmZ, float sad, float& sadX,
                                       float& sadY) {
    if (!(sad > 1.0e-6f)) return false;
    if (!b.spot_beam_directions || b.n_spot_beam_directions == 0 || !b.spot_positions || b.n_spot_positions == 0)
        return false;
    if (b.n_spot_beam_directions % 3 != 0 || b.n_spot_positions % 2 != 0) return false;
    const size_t n = std::min(b.n_spot_beam_directions / 3, b.n_spot_positions / 2);
    if (n == 0) return false;
    size_t nh = 0;
    const float* hdr = active_weq_header(b, nh);
    const bool haveHdr = nh >= 9;
    const float x0 = haveHdr ? hdr[6] : 0.0f, y0 = haveHdr ? hdr[3] : 0.0f;
    const float dx = haveHdr ? hdr[7] : 1.0f, dy = haveHdr ? hdr[4] : 1.0f;
    std::vector<float> sx, sy;
    for (size_t i = 0; i < n; ++i) {
        float spotX = b.spot_positions[2 * i], spotY = b.spot_positions[2 * i + 1];
        if (b.spot_positions_are_indices) {
            if (!haveHdr) return false;
            spotX = x0 + (spotX - 0.5f) * dx;
            spotY = y0 + (spotY - 0.5f) * dy;
        }
        V3 dir = v3(b.spot_beam_directions[3 * i], b.spot_beam_directions[3 * i + 1], b.spot_beam_directions[3 * i + 2]);
        const float len = std::sqrt(dot(dir, dir));
        if (!(len > 1.0e-6f)) continue;
        dir = divs(dir, len);
        const float a = dot(dir, bmZ);
        if (!(std::fabs(a) > 1.0e-6f)) continue;
        const float bx = dot(dir, bmX), by = dot(dir, bmY);
        if (std::fabs(spotX) > 1.0e-3f && std::fabs(bx) > 1.0e-6f) {
            const float c = std::fabs(spotX * a / bx);
            if (c > 1.0f && host_finite(c)) sx.push_back(c);
        }
        if (std::fabs(spotY) > 1.0e-3f && std::fabs(by) > 1.0e-6f) {
            const float c = std::fabs(spotY * a / by);
            if (c > 1.0f && host_finite(c)) sy.push_back(c);
        }
    }
    auto median = [](std::vector<float>& v) -> float {
        if (v.empty()) return 0.0f;
        std::sort(v.begin(), v.end());
        return v[v.size() / 2];
    };
    sadX = median(sx);
    sadY = median(sy);
    return sadX > 0.0f || sadY > 0.0f;
}

}  // namespace

// Lattice cells each spot feeds, with its share (the linear map spot weights ->
// lattice of build_raw_lattice): one cell for spot positions in mm, the bilinear
// splat for positions given as rayweq indices. Four (cell, share) slots per spot;
// unused slots have cell -1.
bool lattice_spot_cells(const PbsBeamDesc& b, const RawLattice& lat, std::vector<int>& cells,
                        std::vector<float>& shares) {
    const int L = static_cast<int>(b.n_energies);
    int total = 0;
    for (int l = 0; l < L; ++l) total += b.layer_spot_counts[l];
    cells.assign(static_cast<size_t>(total) * 4, -1);
    shares.assign(static_cast<size_t>(total) * 4, 0.0f);
    size_t nh = 0;
    const float* hdr = active_weq_header(b, nh);
    int off = 0;
    for (int l = 0; l < L; ++l) {
        for (int i = 0; i < b.layer_spot_counts[l]; ++i) {
            const int s = off + i;
            auto put = [&](int slot, int ix, int iy, float share) {
                if (!(share > 0.0f) || ix < 0 || ix >= lat.nx || iy < 0 || iy >= lat.ny) return;
                cells[size_t(s) * 4 + slot] = (l * lat.ny + iy) * lat.nx + ix;
                shares[size_t(s) * 4 + slot] = share;
            };
            if (b.spot_positions_are_indices) {
                const float lx = b.spot_positions[2 * s] - 0.5f, ly = b.spot_positions[2 * s + 1] - 0.5f;
                const int ix0 = static_cast<int>(std::floor(lx)), iy0 = static_cast<int>(std::floor(ly));
                const float tx = lx - static_cast<float>(ix0), ty = ly - static_cast<float>(iy0);
                put(0, ix0, iy0, (1.0f - tx) * (1.0f - ty));
                put(1, ix0 + 1, iy0, tx * (1.0f - ty));
                put(2, ix0, iy0 + 1, (1.0f - tx) * ty);
                put(3, ix0 + 1, iy0 + 1, tx * ty);
            } else {
                float x, y;
                if (!decode_spot_position(b, hdr, nh, b.spot_positions[2 * s], b.spot_positions[2 * s + 1], x, y))
                    return false;
                const float fx = (lat.dx != 0.0f) ? ((x - lat.ox) / lat.dx) : 0.0f;
                const float fy = (lat.dy != 0.0f) ? ((y - lat.oy) / lat.dy) : 0.0f;
                put(0, static_cast<int>(std::lround(fx)), static_cast<int>(std::lround(fy)), 1.0f);
            }
        }
        off += b.layer_spot_counts[l];
    }
    return true;
}


// ---- reference host helpers ---------------------------------------------

// include/utils/vector_find.h:61-82
int find_first_larger_ordered(const float* v, int n, float value) {
    int upper = n - 1, lower = 0;
    if (v[n - 1] <= value) return upper;
    if (v[0] > value) return 0;
    while (upper - lower > 1) {
        const int pivot = (upper + lower) / 2;
        if (v[pivot] <= value)
            lower = pivot;
        else
            upper = pivot;
    }
    return lower + 1;
}

// include/utils/vector_find.h:94-110
static int find_last_smaller_or_eq_ordered(const float* v, int n, float value) {
    int upper = n - 1, lower = 0;
    if (v[n - 1] <= value) return upper;
    if (v[0] > value) return -1;
    while (upper - lower > 1) {
        const int pivot = (upper + lower) / 2;
        if (v[pivot] <= value)
            lower = pivot;
        else
            upper = pivot;
    }
    return lower;
}

// include/utils/vector_find.h:129-144
float find_decimal_ordered(const float* v, int n, float value) {
    if (value >= v[n - 1]) return static_cast<float>(n - 1);
    if (value < v[0]) return 0.0f;
    const unsigned int f = static_cast<unsigned int>(find_last_smaller_or_eq_ordered(v, n, value));
    const float corr = (value - v[f]) / (v[f + 1] - v[f]);
    return static_cast<float>(f) + corr;
}

// include/utils/vector_interpolate.h:19-31
float vector_interpolate(const float* v, int n, float idx) {
    if (idx <= 0.0f) return v[0];
    if (idx >= static_cast<float>(n - 1)) return v[n - 1];
    float ip;
    const float dec = std::modf(idx, &ip);
    const unsigned int f = static_cast<unsigned int>(ip);
    const float corr = (v[f + 1] - v[f]) * dec;
    return v[f] + corr;
}

int parse_ct_input_type_env() {
    const char* v = std::getenv("RTD_CT_INPUT_TYPE");
    if (!v) return PBS_CT_AUTO;
    const std::string s = str_lower(v);
    if (s == "hu") return PBS_CT_HU;
    if (s == "hu+1000" || s == "huplus1000" || s == "hup1000") return PBS_CT_HU_PLUS_1000;
    if (s == "density" || s == "rho") return PBS_CT_DENSITY;
    if (s == "spr" || s == "stoppingpower" || s == "stopping_power") return PBS_CT_SPR;
    return PBS_CT_AUTO;
}

// wrapper.cu:2307-2325: strided sample of at most ~100k values.
void sample_ct_stats(const float* data, size_t n, float& mn, float& mx) {
    mn = mx = 0.0f;
    if (!data || n == 0) return;
    const size_t maxSamples = 100000;
    const size_t stride = (n > maxSamples) ? (n / maxSamples) : 1;
    const size_t samples = (n + stride - 1) / stride;
    // The samples are cache lines apart and memory bound: four threads split them
    // (minimum and maximum do not depend on the order).
    const int threads = samples < 4096 ? 1 : 4;
    float lo[4], hi[4];
    auto part = [&](int t) {
        const size_t a = samples * t / threads, b = samples * (t + 1) / threads;
        float l = data[0], h = data[0];
        for (size_t k = a; k < b; ++k) {
            const float v = data[k * stride];
            l = std::min(l, v);
            h = std::max(h, v);
        }
        lo[t] = l;
        hi[t] = h;
    };
    std::vector<std::thread> pool;
    for (int t = 1; t < threads; ++t) pool.emplace_back(part, t);
    part(0);
    for (auto& th : pool) th.join();
    mn = lo[0];
    mx = hi[0];
    for (int t = 1; t < threads; ++t) {
        mn = std::min(mn, lo[t]);
        mx = std::max(mx, hi[t]);
    }
}

// wrapper.cu:2327-2337
int auto_detect_ct_type(float mn, float mx) {
    if (mn < -200.0f) return PBS_CT_HU;
    if (mx <= 20.0f && mn >= 0.0f) return PBS_CT_DENSITY;
    return PBS_CT_HU_PLUS_1000;
}

// wrapper.cu:2339-2376
float find_fractional_index_monotonic(const float* v, int n, float value) {
    if (n <= 1) return 0.0f;
    const bool inc = v[n - 1] >= v[0];
    if (inc) {
        if (value <= v[0]) return 0.0f;
        if (value >= v[n - 1]) return static_cast<float>(n - 1);
    } else {
        if (value >= v[0]) return 0.0f;
        if (value <= v[n - 1]) return static_cast<float>(n - 1);
    }
    int lo = 0, hi = n - 1;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        const float vm = v[mid];
        if (inc) {
            if (vm <= value) lo = mid; else hi = mid;
        } else {
            if (vm >= value) lo = mid; else hi = mid;
        }
    }
    const float v0 = v[lo], v1 = v[lo + 1], den = v1 - v0;
    float t = 0.0f;
    if (den != 0.0f) t = (value - v0) / den;
    if (t < 0.0f) t = 0.0f;
    if (t > 1.0f) t = 1.0f;
    return static_cast<float>(lo) + t;
}

// ---- CarbonPBS lateral profile model ----------------------------------------

void plan_carbon_profile(const PbsBeamDesc& b, const PbsEnergyDesc& e, const BeamPlan& P, ProfilePlan& out) {
    out = ProfilePlan{};
    const int L = P.numLayers;
    const size_t nData = b.profile_data ? b.n_profile_data : 0;
    const size_t nPara = b.beam_para_data ? b.n_beam_para_data : 0;
    const size_t nProfE = b.profile_energies ? b.n_profile_energies : 0;
    out.beamPara = nPara >= size_t(L) * 3u;
    const bool model = b.profile_setting && b.n_profile_setting >= 3 &&
                       std::lround(b.profile_setting[2]) > 0 && nData > 0;
    if (model) {
        out.depth0 = b.profile_setting[0];
        out.depthStep = b.profile_setting[1];
        out.depthN = std::max(1, static_cast<int>(std::lround(b.profile_setting[2])));
        const size_t plane = size_t(out.depthN);
        const int paraRows = static_cast<int>(nPara / 3u);
        // The row count: beam-parameter rows, else the profile energy axis, else the
        // layers, else a 11-channel export (wrapper.cu:2830-2849).
        if (paraRows > 0 && nPara == size_t(paraRows) * 3u && nData % (size_t(paraRows) * plane) == 0)
            out.rows = paraRows;
        else if (nProfE > 0 && nData % (nProfE * plane) == 0)
            out.rows = static_cast<int>(nProfE);
        else if (L > 0 && nData % (size_t(L) * plane) == 0)
            out.rows = L;
        else if (nData % plane == 0 && (nData / plane) % 11u == 0)
            out.rows = static_cast<int>((nData / plane) / 11u);
        const size_t perRow = out.rows > 0 ? nData / size_t(out.rows) : 0;
        if (out.rows > 0 && perRow >= plane) {
            out.channels = static_cast<int>(perRow / plane);
            out.table = out.channels > 0 && size_t(out.rows) * plane * size_t(out.channels) == nData;
        }
    }
    out.row.assign(L, 0.0f);
    out.bp0.assign(L, 0.0f);
    out.bp1.assign(L, 0.0f);
    out.bp2.assign(L, 0.0f);
    const int lastRow = std::max(0, out.rows - 1);
    for (int l = 0; l < L; ++l) {
        const float energy = b.energies[l];
        float r;
        if (out.rows == L)
            r = float(l);
        else if (nProfE > 0 && out.rows == static_cast<int>(nProfE))
            r = find_fractional_index_monotonic(b.profile_energies, static_cast<int>(nProfE), energy);
        else if (out.rows == e.n_energies && e.energies_per_u && e.n_energies_per_u > 0)
            r = std::fmin(std::fmax(P.layers[l].energyIdx, 0.0f), float(out.rows - 1));
        else
            r = std::fmin(std::fmax(float(l), 0.0f), float(lastRow));
        r = std::fmin(std::fmax(r, 0.0f), float(lastRow));
        out.row[l] = r;
        // interpBeamParaCoeff (wrapper.cu:4592-4603).
        if (out.rows > 0 && nPara >= size_t(out.rows) * 3u) {
            const float c = std::fmin(std::fmax(r, 0.0f), float(out.rows - 1));
            const int i0 = std::max(0, std::min(out.rows - 1, static_cast<int>(std::floor(c))));
            const int i1 = std::max(0, std::min(out.rows - 1, i0 + 1));
            const float t = c - float(i0);
            float* dst[3] = {&out.bp0[l], &out.bp1[l], &out.bp2[l]};
            for (int k = 0; k < 3; ++k) {
                const float v0 = b.beam_para_data[size_t(i0) * 3u + k], v1 = b.beam_para_data[size_t(i1) * 3u + k];
                *dst[k] = v0 + (v1 - v0) * t;
            }
        }
    }
}

// ---- validation -------------------------------------------------------------

bool validate_global(const float* ct, const GridDesc& ctGrid, const void* dose, const GridDesc& doseGrid,
                     const PbsBeamDesc* beams, size_t numBeams, const PbsEnergyDesc* e, std::string& err) {
    auto fail = [&](const char* m) {
        err = std::string("[RTD_ENTRY_ASSERT] ") + m;
        return false;
    };
    if (!ct) return fail("ctData must not be null");
    if (!dose) return fail("doseData must not be null");
    if (!beams) return fail("beamSettings must not be null");
    if (!e) return fail("energyData must not be null");
    if (numBeams == 0) return fail("numBeams must be positive");
    if (ctGrid.dims[0] <= 0 || ctGrid.dims[1] <= 0 || ctGrid.dims[2] <= 0) return fail("ctDims must be positive");
    if (doseGrid.dims[0] <= 0 || doseGrid.dims[1] <= 0 || doseGrid.dims[2] <= 0) return fail("doseDims must be positive");
    if (!(ctGrid.res[0] > 0.0f && ctGrid.res[1] > 0.0f && ctGrid.res[2] > 0.0f)) return fail("ctResolution must be positive");
    if (!(doseGrid.res[0] > 0.0f && doseGrid.res[1] > 0.0f && doseGrid.res[2] > 0.0f))
        return fail("doseResolution must be positive");
    if (!(e->n_energies > 0 && e->n_energy_samples > 0)) return fail("energyData dimensions must be positive");
    if (e->n_energies_per_u != static_cast<size_t>(e->n_energies) || !e->energies_per_u)
        return fail("energiesPerU size must match energyData->nEnergies");
    if (e->n_peak_depths != static_cast<size_t>(e->n_energies) || !e->peak_depths)
        return fail("peakDepths size must match energyData->nEnergies");
    if (e->n_scale_facts != static_cast<size_t>(e->n_energies) || !e->scale_facts)
        return fail("scaleFacts size must match energyData->nEnergies");
    if (e->n_cidd_matrix != static_cast<size_t>(e->n_energies) * static_cast<size_t>(e->n_energy_samples) ||
        !e->cidd_matrix)
        return fail("ciddMatrix size must equal nEnergies*nEnergySamples");
    if (!e->density_vector || e->n_density_vector == 0 || !e->sp_vector || e->n_sp_vector == 0 || !e->rrl_vector ||
        e->n_rrl_vector == 0)
        return fail("density, stopping-power, and radiation-length LUTs must not be empty");
    // The reference builds its 1-D textures with n*Samples texels read from the vectors.
    if (e->n_density_samples <= 0 || static_cast<size_t>(e->n_density_samples) > e->n_density_vector)
        return fail("nDensitySamples must be in [1, densityVector size]");
    if (e->n_sp_samples <= 0 || static_cast<size_t>(e->n_sp_samples) > e->n_sp_vector)
        return fail("nSpSamples must be in [1, spVector size]");
    if (e->n_rrl_samples <= 0 || static_cast<size_t>(e->n_rrl_samples) > e->n_rrl_vector)
        return fail("nRRlSamples must be in [1, rRlVector size]");
    return true;
}

bool validate_beam(const PbsBeamDesc& b, size_t beamIdx, std::string& err) {
    auto fail = [&](const std::string& m) {
        err = "[RTD_ENTRY_ASSERT] beamIdx=" + std::to_string(beamIdx) + " " + m;
        return false;
    };
    if (!b.energies || b.n_energies == 0) return fail("beam.energies must not be empty");
    if (b.max_subspots_per_layer <= 0) return fail("beam.maxSubspotsPerLayer must be positive");
    const size_t expSub = b.n_energies * static_cast<size_t>(b.max_subspots_per_layer) * 5u;
    if (b.n_subspot_data != expSub || !b.subspot_data)
        return fail("beam.subspotData size must equal numLayers*maxSubspotsPerLayer*5");
    if (b.layer_spot_counts && b.n_layer_spot_counts > 0) {
        if (b.n_layer_spot_counts != b.n_energies) return fail("layerSpotCounts size must match beam.energies size");
        int total = 0;
        for (size_t i = 0; i < b.n_layer_spot_counts; ++i) total += b.layer_spot_counts[i];
        if (b.spot_weights && b.n_spot_weights > 0 && total != static_cast<int>(b.n_spot_weights))
            return fail("sum(layerSpotCounts) must match spotWeights size");
        if (b.spot_positions && b.n_spot_positions > 0) {
            if (b.n_spot_positions % 2 != 0) return fail("spotPositions must be shaped as [N][2]");
            if (total != static_cast<int>(b.n_spot_positions / 2))
                return fail("sum(layerSpotCounts) must match spotPositions row count");
        }
    }
    if (b.spot_beam_directions && b.n_spot_beam_directions > 0) {
        if (b.n_spot_beam_directions % 3 != 0) return fail("spotBeamDirections must be shaped as [N][3]");
        if (b.spot_positions && b.n_spot_positions > 0 && b.n_spot_beam_directions / 3 != b.n_spot_positions / 2)
            return fail("spotBeamDirections row count must match spotPositions row count");
    }
    if (b.layer_longitudinal_cutoffs && b.n_layer_longitudinal_cutoffs > 0 &&
        b.n_layer_longitudinal_cutoffs != b.n_energies)
        return fail("layerLongitudinalCutoffs size must match beam.energies size");
    if (b.profile_data && b.n_profile_data > 0 && b.n_profile_setting < 3)
        return fail("profileData requires profileSetting[depth0,step,n]");
    if (b.beam_para_data && b.n_beam_para_data > 0 && b.n_beam_para_data % 3 != 0)
        return fail("beamParaData must be shaped as [rows][3]");
    size_t nh = 0;
    active_weq_header(b, nh);
    if (b.spot_positions_are_indices && nh < 9) return fail("spotPositionsAreIndices=true requires a 9-value WEQ header");
    if (b.n_spot_sigmas < 2 * b.n_energies) {
        // The reference reads spotSigmas[layer] where present and defaults to (1,1)
        // otherwise (wrapper.cu:3823-3825); odd lengths are rejected.
        if (b.n_spot_sigmas % 2 != 0) return fail("spotSigmas must be shaped as [L][2]");
    }
    return true;
}

// ---- beam planning (wrapper.cu:2664-3406, 3926-4386) ----------------------------

int plan_beam(const PbsBeamDesc& b, const PbsEnergyDesc& e, const GridDesc& ctGrid, const GridDesc& doseGrid,
              BeamPlan& P, std::string& err) {
    P = BeamPlan{};
    const int L = static_cast<int>(b.n_energies);
    P.numLayers = L;
    P.maxSubspots = b.max_subspots_per_layer;

    // Units (wrapper.cu:2729-2797).
    const float stepLengthInput = ctGrid.res[2];
    const float lenToMm = (stepLengthInput > 0.0f && stepLengthInput < 0.3f) ? 10.0f : 1.0f;
    P.lenToMm = lenToMm;
    float energyDepthToMm = lenToMm;
    {
        float peakMax = 0.0f;
        for (int i = 0; i < e.n_energies; ++i) peakMax = std::max(peakMax, e.peak_depths[i]);
        const char* envScale = std::getenv("RTD_ENERGY_DEPTH_SCALE");
        const char* envUnit = std::getenv("RTD_ENERGY_DEPTH_UNIT");
        if (envScale && envScale[0] != '\0') {
            energyDepthToMm = std::max(0.0f, static_cast<float>(std::atof(envScale)));
            if (energyDepthToMm == 0.0f) energyDepthToMm = lenToMm;
        } else if (envUnit && envUnit[0] != '\0') {
            const std::string u = str_lower(envUnit);
            if (u == "cm") energyDepthToMm = 10.0f;
            else if (u == "mm") energyDepthToMm = 1.0f;
        } else if (lenToMm == 10.0f && peakMax > 200.0f) {
            energyDepthToMm = 1.0f;
        }
    }
    P.energyDepthToMm = energyDepthToMm;

    // Gantry frame (wrapper.cu:2880-2933).
    const V3 beamDirW = normalize_safe(v3(b.beam_direction[0], b.beam_direction[1], b.beam_direction[2]));
    const V3 bmXDirW = normalize_safe(v3(b.bm_x_direction[0], b.bm_x_direction[1], b.bm_x_direction[2]));
    const V3 bmYDirW = normalize_safe(v3(b.bm_y_direction[0], b.bm_y_direction[1], b.bm_y_direction[2]));
    const V3 sourceW = v3(b.source_position[0], b.source_position[1], b.source_position[2]);
    const float sad = (b.sad > 0.0f) ? b.sad : b.source_dist[0];
    const V3 basisCross = normalize_safe(cross(bmXDirW, bmYDirW));
    const bool haveCross = dot(basisCross, basisCross) > 1.0e-8f;
    const bool haveBeamDir = dot(beamDirW, beamDirW) > 1.0e-8f;
    V3 bmZ = haveCross ? basisCross : beamDirW;
    if (haveCross && haveBeamDir && dot(bmZ, beamDirW) < 0.0f) bmZ = scale(bmZ, -1.0f);
    if (!(dot(bmZ, bmZ) > 1.0e-8f)) bmZ = v3(0.f, 0.f, 1.f);
    V3 bmX = normalize_safe(sub(bmXDirW, scale(bmZ, dot(bmXDirW, bmZ))));
    if (!(dot(bmX, bmX) > 1.0e-8f)) bmX = normalize_safe(cross(bmYDirW, bmZ));
    if (!(dot(bmX, bmX) > 1.0e-8f)) bmX = v3(1.f, 0.f, 0.f);
    V3 bmY = normalize_safe(cross(bmZ, bmX));
    if (dot(bmY, bmYDirW) < 0.0f) bmY = scale(bmY, -1.0f);
    bmX = normalize_safe(cross(bmY, bmZ));
    P.bmX = bmX;
    P.bmY = bmY;
    P.bmZ = bmZ;
    const V3 gX = bmX, gY = scale(bmY, -1.0f), gZ = scale(bmZ, -1.0f);
    const V3 sourceMm = scale(sourceW, lenToMm);
    const float sadMm = sad * lenToMm;
    const V3 isoMm = add(sourceMm, scale(bmZ, sadMm));

    P.hasLattice = build_raw_lattice(b, P.lattice);

    const M3 g2wM = m3(v3(gX.x, gY.x, gZ.x), v3(gX.y, gY.y, gZ.y), v3(gX.z, gY.z, gZ.z));
    P.gantryToWorld = affine(g2wM, isoMm);
    P.worldToGantry = inverse(P.gantryToWorld);

    // Dose-box projection and subspot bounds, used by the legacy CPB grid (wrapper.cu:2981-3031).
    const V3 doseRes = v3(doseGrid.res[0] * lenToMm, doseGrid.res[1] * lenToMm, doseGrid.res[2] * lenToMm);
    const V3 doseCorner = v3(doseGrid.corner[0] * lenToMm, doseGrid.corner[1] * lenToMm, doseGrid.corner[2] * lenToMm);
    float minGX = 1e30f, maxGX = -1e30f, minGY = 1e30f, maxGY = -1e30f;
    {
        const V3 sz = v3(static_cast<float>(std::max(doseGrid.dims[0] - 1, 0)) * doseRes.x,
                         static_cast<float>(std::max(doseGrid.dims[1] - 1, 0)) * doseRes.y,
                         static_cast<float>(std::max(doseGrid.dims[2] - 1, 0)) * doseRes.z);
        for (int cx = 0; cx <= 1; ++cx)
            for (int cy = 0; cy <= 1; ++cy)
                for (int cz = 0; cz <= 1; ++cz) {
                    const V3 w = add(doseCorner, v3(float(cx) * sz.x, float(cy) * sz.y, float(cz) * sz.z));
                    const V3 g = apply(P.worldToGantry, w);
                    minGX = fminf(minGX, g.x);
                    maxGX = fmaxf(maxGX, g.x);
                    minGY = fminf(minGY, g.y);
                    maxGY = fmaxf(maxGY, g.y);
                }
        const int M = b.max_subspots_per_layer;
        for (int li = 0; li < L; ++li)
            for (int si = 0; si < M; ++si) {
                const size_t base = (static_cast<size_t>(li) * M + si) * 5;
                if (b.n_subspot_data <= base + 4) break;
                if (b.subspot_data[base + 2] > 0.0f) {
                    const float sx = b.subspot_data[base + 0] / lenToMm;
                    const float sy = b.subspot_data[base + 1] / lenToMm;
                    minGX = fminf(minGX, sx);
                    maxGX = fmaxf(maxGX, sx);
                    minGY = fminf(minGY, sy);
                    maxGY = fmaxf(maxGY, sy);
                }
            }
    }

    // Ray grid (wrapper.cu:3039-3212).
    size_t nh = 0;
    const float* hdr = active_weq_header(b, nh);
    const bool hasHdr = nh >= 9;
    float maxSigmaX = 0.0f, maxSigmaY = 0.0f;
    for (size_t i = 0; 2 * i + 1 < b.n_spot_sigmas; ++i) {
        maxSigmaX = std::max(maxSigmaX, b.spot_sigmas[2 * i]);
        maxSigmaY = std::max(maxSigmaY, b.spot_sigmas[2 * i + 1]);
    }
    const float rsx = b.ray_spacing[0], rsy = b.ray_spacing[1];
    if (P.hasLattice && rsx > 0.0f && rsy > 0.0f) {
        const float mX = 3.0f * maxSigmaX + 0.5f * rsx;
        const float mY = 3.0f * maxSigmaY + 0.5f * rsy;
        float oX = 0.f, oY = 0.f;
        int nX = 0, nY = 0;
        const RawLattice& R = P.lattice;
        const bool ax = align_grid_to_reference_phase(R.ox - mX, R.ox + float(R.nx - 1) * R.dx + mX, R.ox, rsx, kTileX, oX, nX);
        const bool ay = align_grid_to_reference_phase(R.oy - mY, R.oy + float(R.ny - 1) * R.dy + mY, R.oy, rsy, kTileY, oY, nY);
        if (!ax || !ay) {
            err = "Failed to align CPB grid to raw spot lattice phase";
            return PBS_ERR_GEOMETRY;
        }
        P.cpbCorner = v3(oX, oY, 0.0f);
        P.cpbRes = v3(rsx, rsy, doseGrid.res[2]);
        P.cpbDims[0] = nX;
        P.cpbDims[1] = nY;
    } else if (hasHdr) {
        bool cropped = false;
        float sMinX = 0, sMaxX = 0, sMinY = 0, sMaxY = 0;
        if (rsx > 0.0f && rsy > 0.0f && decoded_spot_bounds(b, sMinX, sMaxX, sMinY, sMaxY)) {
            const float mX = 3.0f * maxSigmaX + 0.5f * rsx;
            const float mY = 3.0f * maxSigmaY + 0.5f * rsy;
            float oX = 0.f, oY = 0.f;
            int nX = 0, nY = 0;
            const bool ax = align_grid_to_reference_phase(sMinX - mX, sMaxX + mX, hdr[6] / lenToMm, rsx, kTileX, oX, nX);
            const bool ay = align_grid_to_reference_phase(sMinY - mY, sMaxY + mY, hdr[3] / lenToMm, rsy, kTileY, oY, nY);
            if (ax && ay) {
                P.cpbCorner = v3(oX, oY, 0.0f);
                P.cpbRes = v3(rsx, rsy, doseGrid.res[2]);
                P.cpbDims[0] = nX;
                P.cpbDims[1] = nY;
                cropped = true;
            }
        }
        if (!cropped) {
            P.cpbCorner = v3(hdr[6] / lenToMm, hdr[3] / lenToMm, 0.0f);
            P.cpbRes = v3(hdr[7] / lenToMm, hdr[4] / lenToMm, doseGrid.res[2]);
            P.cpbDims[0] = round_up(std::max(1, static_cast<int>(std::lround(hdr[8]))), kTileX);
            P.cpbDims[1] = round_up(std::max(1, static_cast<int>(std::lround(hdr[5]))), kTileY);
        }
    } else {
        if (!(rsx > 0.0f) || !(rsy > 0.0f)) {
            err = "Legacy CPB path requires explicit beam.raySpacing";
            return PBS_ERR_GEOMETRY;
        }
        float covX = (maxGX - minGX) / lenToMm;
        float covY = (maxGY - minGY) / lenToMm;
        if (!(covX > 0.0f) || !(covY > 0.0f)) {
            err = "Legacy CPB path produced non-positive projected coverage";
            return PBS_ERR_GEOMETRY;
        }
        if (const char* env = std::getenv("RTD_CPB_COVERAGE_CM")) {
            const float v = static_cast<float>(std::atof(env));
            if (v > 0.0f && std::isfinite(v)) covX = covY = v;
        }
        P.cpbCorner = v3(minGX / lenToMm, minGY / lenToMm, 0.0f);
        P.cpbRes = v3(rsx, rsy, doseGrid.res[2]);
        P.cpbDims[0] = std::max(1, static_cast<int>(std::ceil(covX / P.cpbRes.x)));
        P.cpbDims[1] = std::max(1, static_cast<int>(std::ceil(covY / P.cpbRes.y)));
    }
    P.cpbDims[2] = L;
    P.rayDims[0] = P.cpbDims[0];
    P.rayDims[1] = P.cpbDims[1];
    P.superpDims[0] = round_up(P.rayDims[0], kTileX);
    P.superpDims[1] = round_up(P.rayDims[1], kTileY);
    P.convMode = P.hasLattice ? 0 : 1;

    // Gantry -> image / dose index (wrapper.cu:3219-3248).
    const V3 ctRes = v3(ctGrid.res[0] * lenToMm, ctGrid.res[1] * lenToMm, ctGrid.res[2] * lenToMm);
    const V3 ctCorner = v3(ctGrid.corner[0] * lenToMm, ctGrid.corner[1] * lenToMm, ctGrid.corner[2] * lenToMm);
    const Affine worldToIm = affine(m3diag(1.0f / ctRes.x, 1.0f / ctRes.y, 1.0f / ctRes.z),
                                    v3(-ctCorner.x / ctRes.x, -ctCorner.y / ctRes.y, -ctCorner.z / ctRes.z));
    P.gantryToImIdx = concat(P.gantryToWorld, worldToIm);
    const Affine worldToDose = affine(m3diag(1.0f / doseRes.x, 1.0f / doseRes.y, 1.0f / doseRes.z),
                                      v3(-doseCorner.x / doseRes.x, -doseCorner.y / doseRes.y, -doseCorner.z / doseRes.z));
    P.gantryToDoseIdx = concat(P.gantryToWorld, worldToDose);

    // Source distances (wrapper.cu:3250-3271).
    float infX = 0.f, infY = 0.f;
    const bool inferred = estimate_virtual_source_distances(b, bmX, bmY, bmZ, sad, infX, infY);
    float distX = b.source_dist[0] * lenToMm, distY = b.source_dist[1] * lenToMm;
    const bool legacySad = std::fabs(b.source_dist[0] - b.sad) < 1.0e-3f && std::fabs(b.source_dist[1] - b.sad) < 1.0e-3f;
    if (inferred && (!(distX > 1e-6f) || legacySad)) distX = infX * lenToMm;
    if (inferred && (!(distY > 1e-6f) || legacySad)) distY = infY * lenToMm;
    if (!(distX > 1e-6f)) distX = sadMm;
    if (!(distY > 1e-6f)) distY = sadMm;
    P.sourceDist = v2(distX, distY);

    // Tracer extent along the beam (wrapper.cu:3286-3364).
    float minGZ = 1e30f, maxGZ = -1e30f;
    {
        const V3 sz = v3(static_cast<float>(std::max(ctGrid.dims[0] - 1, 0)) * ctRes.x,
                         static_cast<float>(std::max(ctGrid.dims[1] - 1, 0)) * ctRes.y,
                         static_cast<float>(std::max(ctGrid.dims[2] - 1, 0)) * ctRes.z);
        for (int cx = 0; cx <= 1; ++cx)
            for (int cy = 0; cy <= 1; ++cy)
                for (int cz = 0; cz <= 1; ++cz) {
                    const V3 w = add(ctCorner, v3(float(cx) * sz.x, float(cy) * sz.y, float(cz) * sz.z));
                    const V3 g = apply(P.worldToGantry, w);
                    minGZ = fminf(minGZ, g.z);
                    maxGZ = fmaxf(maxGZ, g.z);
                }
    }
    P.minGZ = minGZ;
    P.maxGZ = maxGZ;
    const bool hasWeqVolume = hasHdr && b.water_equivalence && b.n_water_equivalence > 9;
    float stepMm = hasWeqVolume ? hdr[1] * lenToMm : ctGrid.res[2] * lenToMm;
    if (!(stepMm > 0.0f)) stepMm = ctGrid.res[2] * lenToMm;
    P.stepLengthMm = stepMm;
    P.startZ = maxGZ;
    P.hasWeqVolume = hasWeqVolume;
    if (hasWeqVolume) {
        // The BEV start plane follows the exporter's projected WEQ origin when that
        // origin is positive, finite and within the WEQ depth span (at least 5 cm)
        // of the CT-derived start (wrapper.cu:3316-3364).
        const float weqStartMm = hdr[0] * lenToMm;
        const float aligned = 0.5f * (distX + distY) - weqStartMm;
        const float span = std::fabs(hdr[1] * lenToMm) * static_cast<float>(std::max(0L, std::lround(hdr[2])));
        if (std::isfinite(aligned) && std::isfinite(weqStartMm) && weqStartMm > 0.0f &&
            std::fabs(aligned - maxGZ) <= std::max(span, 50.0f)) {
            P.startZ = aligned;
            P.startAlignedToWeq = true;
        }
        P.tracerSteps = std::max(1, static_cast<int>(std::lround(hdr[2])));
        P.weqSteps = P.tracerSteps;
        P.weqNy = std::max(1, static_cast<int>(std::lround(hdr[5])));
        P.weqNx = std::max(1, static_cast<int>(std::lround(hdr[8])));
        // Only the header's nx*ny*nStep samples are depths; a longer payload is
        // preallocated capacity (wrapper.cu:3566-3590).
        const size_t need = size_t(P.weqNx) * size_t(P.weqNy) * size_t(P.weqSteps);
        if (b.n_water_equivalence - 9 < need) {
            err = "water_equivalence payload is smaller than header-declared nx*ny*nStep";
            return PBS_ERR_GEOMETRY;
        }
        P.weqActiveSteps = std::min(P.tracerSteps, P.weqSteps);
        P.weqStepMm = std::fabs(hdr[1] * lenToMm);
        P.weqX0 = hdr[6] / lenToMm;
        P.weqY0 = hdr[3] / lenToMm;
        P.weqDx = hdr[7] / lenToMm;
        P.weqDy = hdr[4] / lenToMm;
    } else {
        P.tracerSteps = std::max(1, static_cast<int>(std::ceil((maxGZ - minGZ) / std::fabs(stepMm))) + 1);
    }

    P.fanCorner = v3(P.cpbCorner.x * lenToMm, P.cpbCorner.y * lenToMm, P.startZ);
    P.fanDelta = v3(P.cpbRes.x * lenToMm, P.cpbRes.y * lenToMm, -std::fabs(stepMm));
    P.fanIdxToImIdx.fanIdxToFan = idxxf(P.fanDelta, P.fanCorner);
    P.fanIdxToImIdx.gantryToIdx = P.gantryToImIdx;
    P.fanIdxToImIdx.dist = P.sourceDist;
    P.rayIdxToDoseIdx = P.fanIdxToImIdx;
    P.rayIdxToDoseIdx.gantryToIdx = P.gantryToDoseIdx;
    P.tracer = make_tracer_params(e.density_scale_fact, e.sp_scale_fact, P.tracerSteps, P.fanIdxToImIdx);

    // Step volume polynomial (wrapper.cu:4281-4292).
    {
        const float dX = P.fanDelta.x, dY = P.fanDelta.y, dZ = P.fanDelta.z, cZ = P.fanCorner.z;
        const float dsX = P.sourceDist.x, dsY = P.sourceDist.y;
        const float dXYZ = std::fabs(dX * dY * dZ);
        P.volConst = dXYZ * (1.0f - cZ / dsX - cZ / dsY + (cZ * cZ + dZ * dZ / 12.0f) / (dsX * dsY));
        P.volLin = dXYZ * dZ * (-1.0f / dsX - 1.0f / dsY + 2.0f * cZ / (dsX * dsY));
        P.volSq = dXYZ * dZ * dZ / (dsX * dsY);
    }

    // Beam-level peak depth for the guaranteed-passive step (wrapper.cu:3683-3700).
    {
        const float maxE = *std::max_element(b.energies, b.energies + L);
        const float maxIdx = find_decimal_ordered(e.energies_per_u, e.n_energies, maxE);
        P.maxPeakDepthMm = vector_interpolate(e.peak_depths, e.n_energies, maxIdx) * energyDepthToMm;
    }

    // Per-layer parameters.
    P.layers.resize(L);
    const int nE = e.n_energies;
    const float* E = e.energies_per_u;
    for (int l = 0; l < L; ++l) {
        LayerHost& H = P.layers[l];
        const float energy = b.energies[l];
        H.energy = energy;
        // Spot sigma in mm (wrapper.cu:3753-3757, 3823-3827).
        float sx = 1.0f, sy = 1.0f;
        if (2 * static_cast<size_t>(l) + 1 < b.n_spot_sigmas) {
            sx = b.spot_sigmas[2 * l];
            sy = b.spot_sigmas[2 * l + 1];
        }
        auto toMm = [&](float s) { return (lenToMm > 1.0f && s > 0.0f && s < 1.0f) ? s * 10.0f : s; };
        H.sigmaXmm = toMm(sx);
        H.sigmaYmm = toMm(sy);
        {
            const float convIdx = find_decimal_ordered(E, nE, energy);
            H.convPeakDepth = vector_interpolate(e.peak_depths, nE, convIdx) * energyDepthToMm;
        }
        // Energy index with ascending/descending tables (wrapper.cu:3926-3997).
        float energyIdx = 0.0f;
        const bool asc = (nE > 1) ? (E[0] < E[nE - 1]) : true;
        const int iLow = asc ? 0 : nE - 1, iHigh = asc ? nE - 1 : 0;
        if (nE <= 1) {
            energyIdx = 0.0f;
        } else if (energy <= E[iLow]) {
            energyIdx = static_cast<float>(iLow);
        } else if (energy >= E[iHigh]) {
            energyIdx = static_cast<float>(iHigh);
        } else {
            int fIdx = 0;
            float e0 = E[0], e1 = E[0];
            for (int i = 0; i < nE - 1; ++i) {
                const float a = E[i], bb = E[i + 1];
                const float lo = (a < bb) ? a : bb, hi = (a < bb) ? bb : a;
                if (energy >= lo && energy <= hi) {
                    fIdx = i;
                    e0 = a;
                    e1 = bb;
                    break;
                }
            }
            const float den = e1 - e0;
            float corr = (den != 0.0f) ? ((energy - e0) / den) : 0.0f;
            if (!std::isfinite(corr)) corr = 0.0f;
            corr = std::min(1.0f, std::max(0.0f, corr));
            energyIdx = static_cast<float>(fIdx) + corr;
        }
        auto interp = [&](const float* v) {
            if (energyIdx <= 0.0f) return v[0];
            if (energyIdx >= static_cast<float>(nE - 1)) return v[nE - 1];
            float ip;
            const float dec = std::modf(energyIdx, &ip);
            const int f = static_cast<int>(ip);
            return v[f] + (v[f + 1] - v[f]) * dec;
        };
        const float scaleTable = interp(e.scale_facts);
        const float peakTable = interp(e.peak_depths);
        H.energyIdx = energyIdx;
        H.energyScaleFact = scaleTable / energyDepthToMm;
        H.peakDepth = peakTable * energyDepthToMm;
        H.rangeStopDepth = kBpDepthCutoff * H.peakDepth;
        // initStepAndAirDiv (include/algorithms/fill_idd_and_sigma_params.cuh:66-73).
        const float a = 0.00270f / (H.peakDepth - 4.50f);
        const float bq = -4.39f / (H.peakDepth - 3.86f);
        const float relStepLenSq = 1.0f;
        H.sigmaSqAirQuad = a * relStepLenSq * P.fanDelta.z * P.fanDelta.z;
        H.sigmaSqAirLin = 2.0f * a * relStepLenSq * P.fanDelta.z * P.fanCorner.z + bq * P.fanDelta.z;
        H.sigmaXidd = H.sigmaXmm;
        // Spot spacing in rays (wrapper.cu:4315-4331); consumed by the nuclear branch.
        if (std::fabs(P.fanDelta.x) > 1e-6f) {
            float spacingMm;
            if (b.spot_delta[0] > b.ray_spacing[0] * 1.5f)
                spacingMm = b.spot_delta[0];
            else
                spacingMm = (P.hasLattice ? P.lattice.dx : b.spot_delta[0]) * lenToMm;
            H.spotDist = std::fabs(spacingMm / P.fanDelta.x);
        }
    }
    return PBS_OK;
}

}  // namespace pbs
