// Test infrastructure: a CPU restatement of the reference's mesh rasteriser
// (crates/sims-field/src/raster.rs and bvh.rs), the checker of the CUDA rasteriser. A ray's
// nearest crossing is found by testing every triangle (no hierarchy): Bvh::ray returns the
// nearest crossing past `least` over all triangles its boxes do not rule out, so the brute-force
// search is the same function without the pruning. f64 throughout, in the reference's operation
// order (built with -ffp-contract=off).
#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <map>
#include <vector>

namespace {

using P3 = std::array<double, 3>;

P3 sub(const P3& a, const P3& b) { return {a[0] - b[0], a[1] - b[1], a[2] - b[2]}; }
double dot(const P3& a, const P3& b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
P3 cross(const P3& a, const P3& b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}

struct Tri {
    P3 p[3];
};

// bvh.rs:156-177
bool hit(const Tri& t, const P3& origin, const P3& dir, double* out) {
    const P3 e1 = sub(t.p[1], t.p[0]), e2 = sub(t.p[2], t.p[0]);
    const P3 p = cross(dir, e2);
    const double det = dot(e1, p);
    if (std::fabs(det) < 1.0e-18) return false;
    const double inv = 1.0 / det;
    const P3 s = sub(origin, t.p[0]);
    const double u = dot(s, p) * inv;
    if (!(u >= -1.0e-9 && u <= 1.0 + 1.0e-9)) return false;
    const P3 q = cross(s, e1);
    const double v = dot(dir, q) * inv;
    if (v < -1.0e-9 || u + v > 1.0 + 1.0e-9) return false;
    *out = dot(e2, q) * inv;
    return true;
}

double ray(const std::vector<Tri>& tris, const P3& o, const P3& dir, double least) {
    double best = INFINITY;
    for (const Tri& t : tris) {
        double x;
        if (hit(t, o, dir, &x) && x > least && x < best) best = x;
    }
    return best;
}

size_t partition_point(const std::vector<double>& l, double v, bool or_equal) {
    size_t i = 0;
    while (i < l.size() && (or_equal ? l[i] <= v : l[i] < v)) ++i;   // sorted lines: a linear scan
    return i;
}

size_t nearest(const std::vector<double>& line, double v) {   // grid.rs:48-55
    const size_t i = partition_point(line, v, false);
    if (i >= 1 && i < line.size()) {
        if (std::fabs(v - line[i - 1]) <= std::fabs(line[i] - v)) return i - 1;
        return i;
    }
    if (i >= 1) return i - 1;
    return std::min(i, line.empty() ? 0 : line.size() - 1);
}

size_t cell_of(const std::vector<double>& line, double v) {   // grid.rs:57-59
    const size_t c = partition_point(line, v, true);
    const size_t i = c >= 1 ? c - 1 : 0;
    return std::min(i, line.size() >= 2 ? line.size() - 2 : 0);
}

std::vector<Tri> tris_of(const double* t, uint64_t n) {
    std::vector<Tri> out(n);
    for (uint64_t q = 0; q < n; ++q)
        for (int v = 0; v < 3; ++v)
            for (int a = 0; a < 3; ++a) out[q].p[v][a] = t[q * 9 + v * 3 + a];
    return out;
}

// fill (raster.rs:24-104); index(c) as order 0 / 1 over the index dimensions m.
void fill(const std::vector<Tri>& tris, const std::vector<double>* samples, const uint64_t* m, int order,
          uint8_t* inside, uint8_t* thin) {
    const size_t total = size_t(m[0] * m[1] * m[2]);
    std::memset(inside, 0, total);
    std::memset(thin, 0, total);
    if (tris.empty()) return;
    P3 low = {INFINITY, INFINITY, INFINITY}, high = {-INFINITY, -INFINITY, -INFINITY};
    for (const Tri& t : tris)
        for (const P3& p : t.p)
            for (int a = 0; a < 3; ++a) { low[a] = std::fmin(low[a], p[a]); high[a] = std::fmax(high[a], p[a]); }
    double step[3];
    for (int a = 0; a < 3; ++a) {
        double s = INFINITY;
        for (size_t i = 0; i + 1 < samples[a].size(); ++i) {
            const double d = samples[a][i + 1] - samples[a][i];
            if (d > 0.0) s = std::fmin(s, d);
        }
        step[a] = std::isfinite(s) ? s : std::fmax(std::fmax(high[0] - low[0], high[1] - low[1]), 1.0);
    }
    size_t sp0[3], sp1[3];
    for (int a = 0; a < 3; ++a) {   // span (raster.rs:17-22)
        const auto& line = samples[a];
        if (line.empty()) return;
        size_t first = partition_point(line, low[a], true);
        first = first >= 1 ? first - 1 : 0;
        first = first >= 2 ? first - 2 : 0;
        const size_t last = std::min(partition_point(line, high[a], false) + 2, line.size() - 1);
        if (first > last) return;
        sp0[a] = first;
        sp1[a] = last;
    }
    auto index = [&](const size_t* c) -> size_t {
        if (order == 0) return (c[0] * m[1] + c[1]) * m[2] + c[2];
        return c[0] + (c[1] + c[2] * m[1]) * m[0];
    };
    std::vector<uint8_t> skins(total, 0);
    for (int axis = 0; axis < 3; ++axis) {
        const int u = (axis + 1) % 3, v = (axis + 2) % 3;
        const auto& line = samples[axis];
        const size_t n = line.size();
        const size_t wide = sp1[u] - sp0[u] + 1, tall = sp1[v] - sp0[v] + 1;
        const double start = std::fmin(line[0], low[axis]) - 2.0 * step[axis];
        P3 dir = {0.0, 0.0, 0.0};
        dir[axis] = 1.0;
        const double reach0 = line[0] - step[axis] * 0.5, reach1 = line[n - 1] + step[axis] * 0.5;
#pragma omp parallel for schedule(dynamic, 16)
        for (long long column = 0; column < (long long)(wide * tall); ++column) {
            size_t cell[3] = {0, 0, 0};
            cell[u] = sp0[u] + size_t(column) % wide;
            cell[v] = sp0[v] + size_t(column) / wide;
            P3 from;
            from[u] = samples[u][cell[u]] + step[u] * 1.234567e-6;
            from[v] = samples[v][cell[v]] + step[v] * 2.345678e-6;
            from[axis] = start;
            std::vector<double> crossings;
            double last = 0.0;
            for (;;) {
                const double t = ray(tris, from, dir, last + step[axis] * 1.0e-9);
                if (!std::isfinite(t)) break;
                crossings.push_back(start + t);
                last = t;
            }
            for (size_t q = 0; q < crossings.size(); q += 2) {
                const double a = crossings[q], b = q + 1 < crossings.size() ? crossings[q + 1] : INFINITY;
                const size_t first = partition_point(line, a, false);
                const size_t pl = partition_point(line, b, true);
                if (pl >= 1 && first <= pl - 1) {
                    if (axis == 0)
                        for (size_t k = first; k <= pl - 1; ++k) {
                            size_t c[3] = {cell[0], cell[1], cell[2]};
                            c[axis] = k;
                            inside[index(c)] = 1;
                        }
                } else if (std::isfinite(b)) {
                    const double middle = 0.5 * (a + b);
                    if (middle >= reach0 && middle < reach1) {
                        size_t c[3] = {cell[0], cell[1], cell[2]};
                        c[axis] = nearest(line, middle);
                        skins[index(c)] = 1;
                    }
                }
            }
        }
    }
    for (size_t q = 0; q < total; ++q) thin[q] = (skins[q] && !inside[q]) ? 1 : 0;
}

double local(const std::vector<double>& line, size_t i, bool centre) {   // raster.rs:175-184
    const size_t n = line.size();
    if (centre) return line[std::min(i + 1, n - 1)] - line[std::min(i, n - 2)];
    const double before = i > 0 ? line[i] - line[i - 1] : line[1] - line[0];
    const double after = i + 1 < n ? line[i + 1] - line[i] : line[n - 1] - line[n - 2];
    return 0.5 * (before + after);
}

}  // namespace

extern "C" {

int fgo_raster_fill(const double* tris, uint64_t ntri, const double* s0, uint64_t n0, const double* s1, uint64_t n1,
                    const double* s2, uint64_t n2, const uint64_t* dims, int order, uint8_t* inside, uint8_t* thin) {
    const std::vector<double> s[3] = {std::vector<double>(s0, s0 + n0), std::vector<double>(s1, s1 + n1),
                                      std::vector<double>(s2, s2 + n2)};
    fill(tris_of(tris, ntri), s, dims, order, inside, thin);
    return 0;
}

// sheet_edges (raster.rs:186-264); mask is 3 x nx ny nz.
int fgo_raster_sheet_edges(const double* tp, uint64_t ntri, const double* x, uint64_t nx, const double* y,
                           uint64_t ny, const double* z, uint64_t nz, uint8_t* mask) {
    const std::vector<double> lines[3] = {std::vector<double>(x, x + nx), std::vector<double>(y, y + ny),
                                          std::vector<double>(z, z + nz)};
    const size_t n[3] = {size_t(nx), size_t(ny), size_t(nz)};
    const size_t total = n[0] * n[1] * n[2];
    std::memset(mask, 0, 3 * total);
    for (const Tri& t : tris_of(tp, ntri)) {
        const P3 normal = cross(sub(t.p[1], t.p[0]), sub(t.p[2], t.p[0]));
        const double area2 = std::sqrt(dot(normal, normal));
        if (area2 <= 1e-30) continue;
        const P3 nrm = {normal[0] / area2, normal[1] / area2, normal[2] / area2};
        P3 lo, hi;
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::fmin(std::fmin(std::fmin(INFINITY, t.p[0][a]), t.p[1][a]), t.p[2][a]);
            hi[a] = std::fmax(std::fmax(std::fmax(-INFINITY, t.p[0][a]), t.p[1][a]), t.p[2][a]);
        }
        auto range = [&](int a, bool centre, size_t* first, size_t* last) {
            const auto& line = lines[a];
            auto cell = [&](double v) {
                const size_t i = cell_of(line, v);
                return line[i + 1] - line[i];
            };
            const double reach = std::fmax(cell(lo[a]), cell(hi[a]));
            *first = partition_point(line, lo[a] - reach, false);
            size_t l = partition_point(line, hi[a] + reach, true);
            if (centre) l = std::min(l, line.size() - 1);
            *last = l;
        };
        const P3 e0 = sub(t.p[1], t.p[0]), e1 = sub(t.p[2], t.p[0]);
        const double d00 = dot(e0, e0), d01 = dot(e0, e1), d11 = dot(e1, e1);
        const double det = d00 * d11 - d01 * d01;
        for (int c = 0; c < 3; ++c) {
            if (std::fabs(nrm[c]) >= 0.75) continue;
            size_t f[3], l[3];
            for (int a = 0; a < 3; ++a) range(a, a == c, &f[a], &l[a]);
            for (size_t i = f[0]; i < l[0]; ++i)
                for (size_t j = f[1]; j < l[1]; ++j)
                    for (size_t k = f[2]; k < l[2]; ++k) {
                        const size_t p[3] = {i, j, k};
                        if (p[c] + 1 >= n[c]) continue;
                        P3 mid, h;
                        for (int a = 0; a < 3; ++a) {
                            mid[a] = a == c ? 0.5 * (lines[a][p[a]] + lines[a][p[a] + 1]) : lines[a][p[a]];
                            h[a] = local(lines[a], p[a], a == c);
                        }
                        double sum = 0.0;
                        for (int a = 0; a < 3; ++a) sum = sum + std::fabs(nrm[a]) * h[a];
                        const double tol = 0.5 * sum;
                        const double d = dot(sub(mid, t.p[0]), nrm);
                        const double eps = 1e-9 * tol;
                        if (d <= eps - tol || d > tol + eps) continue;
                        const P3 q = sub(sub(mid, {nrm[0] * d, nrm[1] * d, nrm[2] * d}), t.p[0]);
                        const double q0 = dot(q, e0), q1 = dot(q, e1);
                        const double v = (d11 * q0 - d01 * q1) / det;
                        const double w = (d00 * q1 - d01 * q0) / det;
                        if (v >= -1e-9 && w >= -1e-9 && v + w <= 1.0 + 1e-9) mask[c * total + (i * n[1] + j) * n[2] + k] = 1;
                    }
        }
    }
    return 0;
}

// closed (raster.rs:127-143)
int fgo_raster_closed(const double* tp, uint64_t ntri) {
    if (ntri == 0) return 0;
    const std::vector<Tri> tris = tris_of(tp, ntri);
    P3 lo = {INFINITY, INFINITY, INFINITY}, hi = {-INFINITY, -INFINITY, -INFINITY};
    for (const Tri& t : tris)
        for (const P3& p : t.p)
            for (int a = 0; a < 3; ++a) { lo[a] = std::fmin(lo[a], p[a]); hi[a] = std::fmax(hi[a], p[a]); }
    double size = 0.0;
    for (int a = 0; a < 3; ++a) size = std::fmax(size, hi[a] - lo[a]);
    size = std::fmax(size, 1e-30);
    const double base = std::fmin(std::fmin(lo[0], lo[1]), lo[2]);
    using K = std::array<int64_t, 3>;
    auto key = [&](const P3& p) {
        K k;
        for (int a = 0; a < 3; ++a) k[a] = int64_t(std::round((p[a] - base) / size * 1e9));
        return k;
    };
    std::map<std::pair<K, K>, unsigned> edges;
    for (const Tri& t : tris) {
        const K k[3] = {key(t.p[0]), key(t.p[1]), key(t.p[2])};
        if (k[0] == k[1] || k[1] == k[2] || k[0] == k[2]) continue;
        const int pr[3][2] = {{0, 1}, {1, 2}, {2, 0}};
        for (auto& e : pr) {
            const K& a = k[e[0]];
            const K& b = k[e[1]];
            edges[a < b ? std::make_pair(a, b) : std::make_pair(b, a)] += 1;
        }
    }
    if (edges.empty()) return 0;
    for (auto& kv : edges)
        if (kv.second % 2 != 0) return 0;
    return 1;
}

}  // extern "C"
