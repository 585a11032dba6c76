// TEST INFRASTRUCTURE — the oracle. Nothing in the product links, imports or calls this file;
// only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it, as the checker.
//
// A C++ restatement of the CPU FDTD of v0l/fieldgrid's `sims-field` crate:
//   crates/sims-field/src/fdtd/sim.rs   (axis, time_step, Sim::try_new, thin_wire, pulse, psi_idx)
//   crates/sims-field/src/fdtd/run.rs   (pack, CoefSets, port_loop)
//   crates/sims-field/src/fdtd/cpu.rs   (State::step and its parts, run_cpu)
//   crates/sims-field/src/fdtd/ntff.rs  (patches, Far)
// Templated on the field type T: T = float follows the reference's f32 semantics statement for
// statement (every `as f32` is a cast to T, f32 products are formed before widening, indices
// that pack() stores as f32 are stored as T and read back through a cast); T = double runs the
// same update in FP64 as the truth run the errors are stated against.
//
// The reference is Rust and cannot be built here (no cargo/rustc, no crate registry), so there is
// no run of the reference itself to pin against. The oracle is pinned instead on the reference's
// own known-answer tests, re-expressed in tests/test_oracle.py: the port-loop superposition and
// coefficient-set round trip (run.rs:775-858), analytic cavity modes within 0.4 %
// (tests/fdtd.rs:189-236), thin-wire stability (tests/fdtd.rs:238-269), the refusal texts
// (tests/fdtd.rs:176-187, :271-286).
//
// Memory: Sim::try_new keeps per-edge f64 averages of eps/sigma/inf/debye in twelve nn-long
// arrays (sim.rs:371-374). This restatement recomputes the same 4-cell average on demand with the
// same operations in the same order (bit-identical values) and keeps only the capacitor-adjusted
// eps of the few lumped edges, so a 513^3 grid fits the host's RAM.
#pragma once

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <map>
#include <set>
#include <stdexcept>
#include <string>
#include <unordered_map>
#include <unordered_set>
#include <vector>

namespace oracle {

constexpr double C0 = 299792458.0;          // sim.rs:1
constexpr double EPS0 = 8.8541878128e-12;   // sim.rs:2
constexpr double MU0 = 1.25663706212e-6;    // sim.rs:3
constexpr double ETA0 = 376.730313668;      // sim.rs:4
constexpr double PI = 3.14159265358979323846;

using N3 = std::array<size_t, 3>;

inline size_t idx(const N3& n, size_t i, size_t j, size_t k) { return (i * n[1] + j) * n[2] + k; }  // sim.rs:8-10
inline N3 unidx(const N3& n, size_t id) { return {id / (n[1] * n[2]), (id / n[2]) % n[1], id % n[2]}; }  // sim.rs:642-644

struct Error : std::runtime_error {
    using std::runtime_error::runtime_error;
};

struct Grid {  // grid.rs:2-7
    std::vector<double> x, y, z;
    size_t pml = 0;
    N3 dims() const { return {x.size(), y.size(), z.size()}; }
    size_t cells() const { return (x.size() - 1) * (y.size() - 1) * (z.size() - 1); }
    const std::vector<double>& axis(size_t a) const { return a == 0 ? x : (a == 1 ? y : z); }
};

template <class T>
struct Axis {  // sim.rs:12-27
    size_t n = 0;
    std::vector<double> d, dd;
    std::vector<T> inv_d, inv_dd, raw_inv_d, raw_inv_dd, be, ce, bh, ch;
    std::vector<int32_t> slot_e, slot_h;
};

// sim.rs:29-131
template <class T>
Axis<T> make_axis(const std::vector<double>& line, size_t pml, double dt) {
    const size_t n = line.size();
    Axis<T> a;
    a.n = n;
    a.d.resize(n);
    for (size_t i = 0; i < n; ++i) a.d[i] = (i + 1 < n) ? line[i + 1] - line[i] : line[i] - line[i - 1];
    a.dd.resize(n);
    for (size_t i = 0; i < n; ++i) {
        if (i == 0) a.dd[i] = a.d[0];
        else if (i + 1 >= n) a.dd[i] = a.d[n - 2];
        else a.dd[i] = 0.5 * (line[i + 1] - line[i - 1]);
    }
    const double m = 3.0, kappa_max = 1.0, alpha_max = 0.05;
    std::vector<double> ke(n, 1.0), kh(n, 1.0);
    a.be.assign(n, T(0)); a.ce.assign(n, T(0)); a.bh.assign(n, T(0)); a.ch.assign(n, T(0));
    a.slot_e.assign(n, -1); a.slot_h.assign(n, -1);
    if (pml > 0 && n > 2 * pml + 2) {
        const double left = line[pml], right = line[n - 1 - pml];
        const double depth_l = left - line[0], depth_r = line[n - 1] - right;
        auto coef = [&](double rho, double depth, double cell, double& kappa, double& b, double& c) {
            double r = std::clamp(rho / depth, 0.0, 1.0);
            double sigma_max = 0.8 * (m + 1.0) / (ETA0 * cell);
            double sigma = sigma_max * std::pow(r, m);
            kappa = 1.0 + (kappa_max - 1.0) * std::pow(r, m);
            double alpha = alpha_max * (1.0 - r) * 2.0 * PI * EPS0 * 1e9;
            b = std::exp(-(sigma / kappa + alpha) * dt / EPS0);
            c = sigma > 0.0 ? sigma * (b - 1.0) / (sigma * kappa + kappa * kappa * alpha) : 0.0;
        };
        auto zone = [&](double x, double& rho, double& depth, double& cell) {
            if (x < left) { rho = left - x; depth = depth_l; cell = a.d[0]; }
            else if (x > right) { rho = x - right; depth = depth_r; cell = a.d[n - 2]; }
            else { rho = 0.0; depth = 1.0; cell = 1.0; }
        };
        for (size_t i = 0; i < n; ++i) {
            double rho, depth, cell, k, b, c;
            zone(line[i], rho, depth, cell);
            if (rho > 0.0) {
                coef(rho, depth, cell, k, b, c);
                ke[i] = k; a.be[i] = T(b); a.ce[i] = T(c);
            }
            if (i < pml) a.slot_e[i] = int32_t(i);
            else if (i > n - 1 - pml) a.slot_e[i] = int32_t(i + 2 * pml - n);
            if (i + 1 < n) {
                double xc = 0.5 * (line[i] + line[i + 1]);
                zone(xc, rho, depth, cell);
                if (rho > 0.0) {
                    coef(rho, depth, cell, k, b, c);
                    kh[i] = k; a.bh[i] = T(b); a.ch[i] = T(c);
                }
                if (i < pml) a.slot_h[i] = int32_t(i);
                else if (i >= n - 1 - pml) a.slot_h[i] = int32_t(pml + i - (n - 1 - pml));
            }
        }
    }
    a.inv_d.resize(n); a.inv_dd.resize(n); a.raw_inv_d.resize(n); a.raw_inv_dd.resize(n);
    for (size_t i = 0; i < n; ++i) {
        a.inv_d[i] = T(1.0 / (kh[i] * a.d[i]));
        a.inv_dd[i] = T(1.0 / (ke[i] * a.dd[i]));
        a.raw_inv_d[i] = T(1.0 / a.d[i]);
        a.raw_inv_dd[i] = T(1.0 / a.dd[i]);
    }
    return a;
}

// sim.rs:133-137
inline double time_step(const Grid& g) {
    auto mn = [](const std::vector<double>& v) {
        double m = INFINITY;
        for (size_t i = 0; i + 1 < v.size(); ++i) m = std::fmin(m, v[i + 1] - v[i]);
        return m;
    };
    // powi(2) is a single product
    double mx = mn(g.x), my = mn(g.y), mz = mn(g.z);
    double s = 1.0 / (mx * mx) + 1.0 / (my * my) + 1.0 / (mz * mz);
    return 0.99 / (C0 * std::sqrt(s));
}

// sim.rs:139-143
inline size_t psi_len(const N3& n, size_t axis, size_t pml) {
    N3 m = n;
    m[axis] = 2 * pml;
    return pml == 0 ? 0 : m[0] * m[1] * m[2];
}

// sim.rs:659-665
inline size_t psi_idx(const N3& n, size_t axis, size_t pml, const N3& p, size_t slot) {
    if (axis == 0) return (slot * n[1] + p[1]) * n[2] + p[2];
    if (axis == 1) return (p[0] * 2 * pml + slot) * n[2] + p[2];
    return (p[0] * n[1] + p[1]) * 2 * pml + slot;
}

struct Edge {  // sim.rs:145-149
    size_t comp;
    N3 at;
};
enum Kind { RESISTOR = 0, CAPACITOR = 1, INDUCTOR = 2 };
struct Lumped { std::vector<Edge> edges; int kind; double value; };          // sim.rs:158-163
struct PortDef { std::vector<std::vector<Edge>> columns; double r; bool reference_above; };  // sim.rs:165-171
struct Resistive { size_t comp, id; double r; bool adaptive; size_t faces[2]; };  // sim.rs:208-215
struct Materials { std::vector<float> eps, sigma, inf, debye; };              // sim.rs:217-222
struct Media {                                                                // sim.rs:236-241
    std::vector<float> sheet_table{0.f, 0.f, 0.f, 0.f};
    size_t sheet_states = 0;
    std::vector<std::pair<double, double>> poles;
    std::vector<std::pair<Edge, double>> wires;
};

template <class T>
struct WireH { size_t h; std::array<std::pair<size_t, T>, 4> terms; };  // sim.rs:191-195
struct SheetEdge { size_t comp, id; double r; bool adaptive; size_t faces[2]; double len, c; };  // sim.rs:197-206

template <class T>
struct Sim {  // sim.rs:173-189
    Grid grid;
    std::array<Axis<T>, 3> ax;
    double dt = 0;
    std::array<std::vector<T>, 3> ca, cb;
    size_t pml = 0;
    std::vector<PortDef> ports;
    std::vector<std::vector<std::tuple<size_t, size_t, T>>> port_src;
    std::vector<std::tuple<size_t, size_t, T, T>> inductors;
    std::vector<SheetEdge> sheets;
    std::vector<float> sheet_table;
    size_t sheet_states = 0;
    std::vector<std::pair<double, double>> poles;
    std::vector<std::tuple<size_t, size_t, double>> debye_edges;
    std::vector<WireH<T>> wires;
    N3 dims() const { return grid.dims(); }
};

// sim.rs:303-313
inline double wire_factor(double d, double radius) {
    double lo = d * std::exp(-4.0), hi = 0.5 * d;
    if (radius >= lo && radius < hi) return 2.0 / std::log(d / radius);
    char buf[256];
    std::snprintf(buf, sizeof buf,
                  "a thin wire's radius must be from a 55th to half of its cell (%.3e to %.3e m), not %.3e m",
                  lo, hi, radius);
    throw Error(buf);
}

// sim.rs:315-336
inline std::vector<double> wire_cells(const Grid& g, const std::vector<std::pair<Edge, double>>& wires) {
    N3 n = g.dims();
    std::vector<double> out;
    for (auto& [e, radius] : wires) {
        size_t w = e.comp;
        N3 p = e.at, end = p;
        end[w] += 1;
        auto clear = [&](const N3& q) {
            for (int a = 0; a < 3; ++a)
                if (!(q[a] > g.pml && q[a] + 1 + g.pml < n[a])) return false;
            return true;
        };
        if (!clear(p) || !clear(end)) throw Error("a thin wire must stay clear of the grid's absorbing layer");
        for (size_t axis : {(w + 1) % 3, (w + 2) % 3}) {
            const auto& line = g.axis(axis);
            for (const N3& node : {p, end})
                for (size_t cell : {node[axis], node[axis] - 1}) out.push_back(wire_factor(line[cell + 1] - line[cell], radius));
        }
    }
    return out;
}

// Materials::at (sim.rs:296-300): the material tuple of a (clamped) cell, widened to f64.
inline std::array<double, 4> mat_at(const Materials& m, const N3& dims, const std::array<long, 3>& c) {
    size_t cc[3];
    for (int a = 0; a < 3; ++a) cc[a] = size_t(std::clamp<long>(c[a], 0, long(dims[a]) - 2));
    size_t id = (cc[0] * (dims[1] - 1) + cc[1]) * (dims[2] - 1) + cc[2];
    return {double(m.eps[id]), double(m.sigma[id]), double(m.inf[id]), double(m.debye[id])};
}

// The area-weighted 4-cell average of sim.rs:375-410 for one edge: {eps (times EPS0), sigma, inf,
// debye weight}. Edges the reference leaves at zero (on or beyond the boundary) return zeros.
template <class T>
std::array<double, 4> edge_average(const Sim<T>& s, const Materials& mats, size_t c, const N3& p) {
    const N3 n = s.dims();
    size_t u = (c + 1) % 3, v = (c + 2) % 3;
    if (p[c] + 1 >= n[c] || p[u] == 0 || p[u] + 1 >= n[u] || p[v] == 0 || p[v] + 1 >= n[v]) return {0, 0, 0, 0};
    double sum[4] = {0, 0, 0, 0};
    double w_sum = 0.0;
    const int offs[4][2] = {{-1, -1}, {0, -1}, {-1, 0}, {0, 0}};
    for (auto& o : offs) {
        std::array<long, 3> cell = {long(p[0]), long(p[1]), long(p[2])};
        cell[u] += o[0];
        cell[v] += o[1];
        double w = s.ax[u].d[size_t(cell[u])] * s.ax[v].d[size_t(cell[v])];
        auto m = mat_at(mats, n, cell);
        for (int q = 0; q < 4; ++q) sum[q] += m[q] * w;
        w_sum += w;
    }
    return {EPS0 * sum[0] / w_sum, sum[1] / w_sum, sum[2] / w_sum, sum[3] / w_sum};
}

// Sim::try_new (sim.rs:352-554) and thin_wire (sim.rs:556-635).
template <class T>
Sim<T> try_new(Grid grid, const Materials& mats, const std::function<bool(size_t, const N3&)>& pec,
               const std::vector<Lumped>& lumped, std::vector<PortDef> ports,
               const std::vector<Resistive>& resistive, const Media& media) {
    Sim<T> s;
    double speedup = 1.0;
    for (double f : wire_cells(grid, media.wires)) speedup = std::fmax(speedup, std::fmax(f, 1.0 / f));
    const double dt = time_step(grid) / std::sqrt(speedup);
    s.pml = grid.pml;
    s.ax = {make_axis<T>(grid.x, s.pml, dt), make_axis<T>(grid.y, s.pml, dt), make_axis<T>(grid.z, s.pml, dt)};
    s.grid = std::move(grid);
    s.dt = dt;
    const N3 n = s.dims();
    const size_t total = n[0] * n[1] * n[2];
    for (int c = 0; c < 3; ++c) { s.ca[c].assign(total, T(0)); s.cb[c].assign(total, T(0)); }

    auto area = [&](const Edge& e) {
        size_t u = (e.comp + 1) % 3, v = (e.comp + 2) % 3;
        return s.ax[u].dd[e.at[u]] * s.ax[v].dd[e.at[v]];
    };
    auto length = [&](const Edge& e) { return s.ax[e.comp].d[e.at[e.comp]]; };
    auto key = [&](size_t c, size_t id) { return uint64_t(c) * total + id; };

    // Capacitors add to the edge permittivity (sim.rs:418-430); kept as overrides of eps.
    std::unordered_map<uint64_t, double> eps_over;
    std::vector<std::tuple<size_t, size_t, double>> series_r;
    for (auto& l : lumped) {
        double count = double(std::max<size_t>(l.edges.size(), 1));
        for (auto& e : l.edges) {
            size_t id = idx(n, e.at[0], e.at[1], e.at[2]);
            if (l.kind == CAPACITOR) {
                auto it = eps_over.find(key(e.comp, id));
                double cur = it != eps_over.end() ? it->second : edge_average(s, mats, e.comp, e.at)[0];
                eps_over[key(e.comp, id)] = cur + l.value * count * length(e) / area(e);
            } else if (l.kind == RESISTOR) {
                series_r.emplace_back(e.comp, id, l.value / count);
            }
        }
    }
    auto eps_of = [&](size_t c, size_t id, const std::array<double, 4>& avg) {
        auto it = eps_over.find(key(c, id));
        return it != eps_over.end() ? it->second : avg[0];
    };
    // ca/cb (sim.rs:431-441)
    for (size_t c = 0; c < 3; ++c) {
#pragma omp parallel for schedule(static)
        for (long i = 0; i < long(n[0]); ++i)
            for (size_t j = 0; j < n[1]; ++j)
                for (size_t k = 0; k < n[2]; ++k) {
                    N3 p = {size_t(i), j, k};
                    size_t id = idx(n, p[0], j, k);
                    auto avg = edge_average(s, mats, c, p);
                    double eps = eps_of(c, id, avg);
                    if (eps == 0.0) continue;
                    double x = avg[1] * dt / (2.0 * eps);
                    s.ca[c][id] = T((1.0 - x) / (1.0 + x));
                    s.cb[c][id] = T(dt / eps / (1.0 + x));
                }
    }
    // PEC (sim.rs:442-454)
    for (size_t c = 0; c < 3; ++c)
        for (size_t i = 0; i < n[0]; ++i)
            for (size_t j = 0; j < n[1]; ++j)
                for (size_t k = 0; k < n[2]; ++k)
                    if (pec(c, N3{i, j, k})) {
                        size_t id = idx(n, i, j, k);
                        s.ca[c][id] = T(0);
                        s.cb[c][id] = T(0);
                    }
    // excluded edges (sim.rs:455-468)
    std::unordered_set<uint64_t> excluded;
    for (auto& l : lumped)
        for (auto& e : l.edges) excluded.insert(key(e.comp, idx(n, e.at[0], e.at[1], e.at[2])));
    for (auto& p : ports)
        for (auto& col : p.columns)
            for (auto& e : col) excluded.insert(key(e.comp, idx(n, e.at[0], e.at[1], e.at[2])));
    for (auto& r : resistive) excluded.insert(key(r.comp, r.id));
    // Debye edges (sim.rs:469-483)
    double half_g = 0.0;
    for (auto& [x, a] : media.poles) half_g += a * x * dt / (1.0 + 0.5 * x * dt);
    half_g *= 0.5;
    for (size_t c = 0; c < 3; ++c) {
        std::vector<std::vector<std::tuple<size_t, size_t, double>>> found(n[0]);
#pragma omp parallel for schedule(static)
        for (long i = 0; i < long(n[0]); ++i)
            for (size_t j = 0; j < n[1]; ++j)
                for (size_t k = 0; k < n[2]; ++k) {
                    size_t id = idx(n, size_t(i), j, k);
                    // dd_edge is zero wherever the average is not formed, so only those edges count
                    N3 p = {size_t(i), j, k};
                    auto avg = edge_average(s, mats, c, p);
                    double dd = avg[3];
                    if (dd <= 0.0 || s.cb[c][id] == T(0) || excluded.count(key(c, id))) continue;
                    double eps = EPS0 * (avg[2] + dd * half_g);
                    s.ca[c][id] = T(1.0);
                    s.cb[c][id] = T(dt / eps);
                    found[size_t(i)].emplace_back(c, id, dd);
                }
        for (auto& f : found) s.debye_edges.insert(s.debye_edges.end(), f.begin(), f.end());
    }
    // resistor closure (sim.rs:484-492)
    auto resistor = [&](const Edge& e, double r) {
        size_t id = idx(n, e.at[0], e.at[1], e.at[2]);
        auto avg = edge_average(s, mats, e.comp, e.at);
        double eps = eps_of(e.comp, id, avg);
        double x_sig = avg[1] * dt / (2.0 * eps);
        double beta = dt * length(e) / (2.0 * r * eps * area(e)) + x_sig;
        s.ca[e.comp][id] = T((1.0 - beta) / (1.0 + beta));
        s.cb[e.comp][id] = T(dt / (eps * (1.0 + beta)));
        return dt / (eps * (1.0 + beta) * r * area(e));
    };
    for (auto& [comp, id, r] : series_r) resistor(Edge{comp, unidx(n, id)}, r);
    // sheets (sim.rs:497-509)
    for (auto& r : resistive) {
        Edge e{r.comp, unidx(n, r.id)};
        s.sheets.push_back(SheetEdge{r.comp, r.id, r.r, r.adaptive, {r.faces[0], r.faces[1]}, length(e),
                                     double(s.cb[r.comp][r.id]) / area(e)});
    }
    // port sources (sim.rs:510-523)
    for (auto& p : ports) {
        double cols = double(std::max<size_t>(p.columns.size(), 1));
        std::vector<std::tuple<size_t, size_t, T>> v;
        for (auto& col : p.columns) {
            double m = double(std::max<size_t>(col.size(), 1));
            double re = p.r * cols / m;
            for (auto& e : col) {
                double src = resistor(e, re);
                v.emplace_back(e.comp, idx(n, e.at[0], e.at[1], e.at[2]), T(src / m));
            }
        }
        s.port_src.push_back(std::move(v));
    }
    // inductors (sim.rs:524-534)
    for (auto& l : lumped) {
        if (l.kind != INDUCTOR) continue;
        double count = double(std::max<size_t>(l.edges.size(), 1));
        for (auto& e : l.edges) {
            size_t id = idx(n, e.at[0], e.at[1], e.at[2]);
            double k_e = double(s.cb[e.comp][id]) / area(e);
            double k_i = dt * length(e) / (l.value / count);
            s.inductors.emplace_back(e.comp, id, T(k_e), T(k_i));
        }
    }
    s.ports = std::move(ports);
    s.sheet_table = media.sheet_table;
    s.sheet_states = media.sheet_states;
    s.poles = media.poles;

    // thin_wire (sim.rs:556-635)
    {
        const size_t nn = total;
        const double k_mu = dt / MU0;
        auto wkey = [&](size_t c, const N3& p) { return c * nn + idx(n, p[0], p[1], p[2]); };
        std::set<size_t> on_wire;
        for (auto& [e, r] : media.wires) on_wire.insert(wkey(e.comp, e.at));
        std::map<size_t, std::tuple<N3, size_t, double>> scaled_h;
        std::map<size_t, double> scaled_e;
        for (auto& [e, radius] : media.wires) {
            size_t w = e.comp;
            N3 p = e.at, end = p;
            end[w] += 1;
            for (size_t axis : {(w + 1) % 3, (w + 2) % 3}) {
                size_t c = 3 - w - axis;
                N3 qm = p;
                qm[axis] -= 1;
                std::pair<size_t, N3> hs[2] = {{p[axis], p}, {p[axis] - 1, qm}};
                for (auto& [cell, q] : hs) {
                    double f = wire_factor(s.ax[axis].d[cell], radius);
                    scaled_h.emplace(wkey(c, q), std::make_tuple(q, c, f));
                }
                for (const N3& node : {p, end}) {
                    N3 nm = node;
                    nm[axis] -= 1;
                    std::pair<size_t, N3> es[2] = {{node[axis], node}, {node[axis] - 1, nm}};
                    for (auto& [cell, at] : es) {
                        size_t id = wkey(axis, at);
                        if (!on_wire.count(id)) {
                            double f = wire_factor(s.ax[axis].d[cell], radius);
                            scaled_e.emplace(id, f);
                        }
                    }
                }
            }
        }
        for (auto& [id, f] : scaled_e) {
            size_t c = id / nn, at = id % nn;
            double ca = double(s.ca[c][at]), cb = double(s.cb[c][at]);
            if (cb == 0.0) continue;
            double a = (1.0 - ca) / (1.0 + ca);
            double scaled = a / f;
            s.ca[c][at] = T((1.0 - scaled) / (1.0 + scaled));
            s.cb[c][at] = T(cb * (1.0 + a) / (f * (1.0 + scaled)));
        }
        for (auto& [h, t] : scaled_h) {
            auto& [q, c, f] = t;
            size_t u = (c + 1) % 3, v = (c + 2) % 3;
            double sc = (f - 1.0) * k_mu;
            double du = double(s.ax[u].inv_d[q[u]]), dv = double(s.ax[v].inv_d[q[v]]);
            N3 qu = q, qv = q;
            qu[u] += 1;
            qv[v] += 1;
            std::pair<size_t, double> all[4] = {
                {wkey(v, qu), -sc * du}, {wkey(v, q), sc * du}, {wkey(u, qv), sc * dv}, {wkey(u, q), -sc * dv}};
            WireH<T> wh;
            wh.h = h;
            for (auto& tm : wh.terms) tm = {h, T(0)};
            size_t slot = 0;
            for (auto& [ei, cc] : all)
                if (!on_wire.count(ei)) wh.terms[slot++] = {ei, T(cc)};
            s.wires.push_back(wh);
        }
    }
    return s;
}

// pulse_shape (sim.rs:646-649)
inline void pulse_shape(double fc, double& t0, double& tau) {
    tau = std::sqrt(std::log(10.0)) / (PI * fc);
    t0 = 4.0 * tau;
}

// port_loop (run.rs:102-127): (id, comp, weight) sorted by (id, comp).
template <class T>
std::vector<std::tuple<size_t, size_t, double>> port_loop(const Sim<T>& s, const PortDef& p, size_t axis, size_t k) {
    N3 n = s.dims();
    size_t u = (axis + 1) % 3, v = (axis + 2) % 3;
    auto at = [&](size_t a, size_t b) {
        N3 q{0, 0, 0};
        q[u] = a;
        q[v] = b;
        q[axis] = k;
        return idx(n, q[0], q[1], q[2]);
    };
    std::map<std::pair<size_t, size_t>, int> turns;
    std::set<std::pair<size_t, size_t>> nodes;
    for (auto& c : p.columns) nodes.insert({c[0].at[u], c[0].at[v]});
    for (auto [a, b] : nodes) {
        turns[{at(a, b), v}] += 1;
        turns[{at(a - 1, b), v}] -= 1;
        turns[{at(a, b), u}] -= 1;
        turns[{at(a, b - 1), u}] += 1;
    }
    std::vector<std::tuple<size_t, size_t, double>> out;
    for (auto& [kc, t] : turns)
        if (t != 0) out.emplace_back(kc.first, kc.second, double(t) * s.ax[kc.second].dd[unidx(n, kc.first)[kc.second]]);
    return out;
}

// CoefSets (run.rs:61-100), kept for its unit test.
struct CoefSets {
    std::vector<uint32_t> index;
    std::vector<std::array<float, 2>> sets;
    bool wide = false;
};
inline CoefSets coef_sets(const Sim<float>& s, size_t narrow) {
    size_t nn = s.ca[0].size();
    std::unordered_map<uint64_t, uint32_t> lookup;
    CoefSets out;
    out.sets.push_back({0.f, 0.f});
    lookup[0] = 0;
    std::vector<uint32_t> flat;
    flat.reserve(3 * nn);
    uint64_t last_key = 0;
    uint32_t last_id = 0;
    for (int c = 0; c < 3; ++c)
        for (size_t id = 0; id < nn; ++id) {
            float a = s.ca[c][id], b = s.cb[c][id];
            uint32_t ab, bb;
            std::memcpy(&ab, &a, 4);
            std::memcpy(&bb, &b, 4);
            uint64_t key = (b == 0.f) ? 0 : (uint64_t(ab) << 32 | bb);
            if (key != last_key) {
                auto it = lookup.find(key);
                uint32_t v;
                if (it == lookup.end()) {
                    out.sets.push_back({a, b});
                    v = uint32_t(out.sets.size() - 1);
                    lookup[key] = v;
                } else v = it->second;
                last_key = key;
                last_id = v;
            }
            flat.push_back(last_id);
        }
    out.wide = out.sets.size() > narrow;
    if (out.wide) out.index = std::move(flat);
    else {
        for (size_t q = 0; q < flat.size(); q += 2)
            out.index.push_back(flat[q] | (q + 1 < flat.size() ? flat[q + 1] << 16 : 0));
    }
    return out;
}

struct Pulse { double f0, fc; };          // run.rs:47-50
struct Extras {                           // run.rs:34-45
    size_t min_steps = 0, max_steps = 0;
    double decay_db = 0;
    std::vector<double> freqs;
    bool has_plane_k = false;
    size_t plane_k = 0;
    bool has_ntff = false;
    std::vector<uint32_t> ntff;
    size_t check_every = 0;
};
template <class T>
struct Record {                           // run.rs:52-59, plus the final fields
    size_t steps = 0, ports = 0;
    std::vector<T> series;
    double decay_db = 0;
    std::vector<T> plane, ntff;
    std::vector<T> e, h;
};

// One sheet edge as pack() lays it out in 16 f32 slots (run.rs:259-289), named.
template <class T>
struct PackedSheet {
    size_t f, ha, hb;   // slots 0-2: field index, two H indices
    T len, c, r, adaptive;  // 3-6
    T aa, bb, ab, ma, mb, old, i_old;  // 7-13
    size_t face_a, face_b;  // 14-15
};

// pack (run.rs:205-376) and the CPU stepper State (cpu.rs:17-422).
template <class T>
struct State {
    const Sim<T>& sim;
    N3 n;
    size_t nn;
    uint32_t offsets[20] = {};
    size_t psi_total = 0;
    std::vector<T> source;     // [id, src, comp] (indices as T, run.rs:243-246)
    std::vector<T> inductor;   // [comp, id, ke, ki, I]
    std::vector<PackedSheet<T>> sheets;
    size_t states = 0;
    std::vector<size_t> debye_f;
    std::vector<T> debye_dd, debye_old;
    std::vector<T> debye_table;
    std::vector<T> probe_def, port_edges, loops;
    double t0 = 0, tau = 0;
    size_t cap = 0, ports = 0, nf = 0, plane_len = 0, patches = 0;
    std::vector<T> sheet_branch;
    // state
    std::vector<T> e, h, psi, current, debye_state, series, plane, ntff;
    std::vector<uint32_t> patch_idx;
    std::vector<T> omega;
    size_t plane_k = 0;
    T w0 = 0;

    State(const Sim<T>& s, size_t driven, const Pulse& pulse, const Extras& ex) : sim(s) {
        n = s.dims();
        nn = n[0] * n[1] * n[2];
        for (size_t ee = 0; ee < 2; ++ee)
            for (size_t c = 0; c < 3; ++c)
                for (size_t a = 0; a < 3; ++a) {
                    offsets[ee * 9 + c * 3 + a] = uint32_t(psi_total);
                    if (a != c) psi_total += psi_len(n, a, s.pml);
                }
        if (driven >= s.port_src.size()) throw Error("driven port out of range");
        for (auto& [comp, id, v] : s.port_src[driven]) {
            source.push_back(T(id));
            source.push_back(v);
            source.push_back(T(comp));
        }
        for (auto& [comp, id, ke, ki] : s.inductors) {
            T vals[5] = {T(comp), T(id), ke, ki, T(0)};
            inductor.insert(inductor.end(), vals, vals + 5);
        }
        states = s.sheet_states;
        for (auto& sh : s.sheets) {
            size_t hc;
            bool ok;
            if (sh.comp == 0) { hc = 1; ok = true; }
            else if (sh.comp == 1) { hc = 0; ok = true; }
            else { hc = 0; ok = false; }
            if (!ok || sh.id % n[2] == 0) continue;
            PackedSheet<T> p{sh.comp * nn + sh.id, hc * nn + sh.id, hc * nn + sh.id - 1,
                             T(sh.len), T(sh.c), T(sh.r), sh.adaptive ? T(1) : T(0),
                             T(0), T(0), T(0), T(0.5), T(0.5), T(0), T(0), sh.faces[0], sh.faces[1]};
            sheets.push_back(p);
        }
        for (auto& [c, id, dd] : s.debye_edges) {
            debye_f.push_back(c * nn + id);
            debye_dd.push_back(T(dd));
            debye_old.push_back(T(0));
        }
        debye_table.push_back(T(s.poles.size()));
        for (auto& [x, a] : s.poles) {
            double d = 1.0 + 0.5 * x * s.dt;
            debye_table.push_back(T((1.0 - 0.5 * x * s.dt) / d));
            debye_table.push_back(T(EPS0 * a * x / d));
        }
        for (auto& p : s.ports) {
            size_t axis = p.columns[0][0].comp;
            size_t u = (axis + 1) % 3, v = (axis + 2) % 3;
            const auto& mid = p.columns[p.columns.size() / 2];
            size_t first = port_edges.size() / 2;
            double polarity = p.reference_above ? -1.0 : 1.0;
            double weight = polarity / double(p.columns.size());
            for (auto& col : p.columns)
                for (auto& e : col) {
                    port_edges.push_back(T(idx(n, e.at[0], e.at[1], e.at[2])));
                    port_edges.push_back(T(s.ax[axis].d[e.at[axis]] * weight));
                }
            size_t probed = port_edges.size() / 2 - first;
            size_t loop_first = loops.size() / 3;
            double height = 0.0;
            for (auto& e : mid) height += s.ax[axis].d[e.at[axis]];
            for (auto& e : mid) {
                size_t k = e.at[axis];
                double share = polarity * s.ax[axis].d[k] / height;
                for (auto& [id, comp, w] : port_loop(s, p, axis, k)) {
                    loops.push_back(T(id));
                    loops.push_back(T(3 + comp));
                    loops.push_back(T(w * share));
                }
            }
            T defs[8] = {T(axis), T(first), T(probed), T(loop_first), T(loops.size() / 3 - loop_first), T(u), T(v), T(0)};
            probe_def.insert(probe_def.end(), defs, defs + 8);
        }
        for (size_t q = 0; q < port_edges.size(); q += 2)
            if (float(port_edges[q]) >= float(1u << 24)) throw Error("grid too large for f32 port indices");
        pulse_shape(pulse.fc, t0, tau);
        cap = ex.max_steps;
        ports = s.ports.size();
        nf = std::min<size_t>(ex.freqs.size(), 4);
        plane_len = ex.has_plane_k ? n[0] * n[1] * nf * 10 : 0;
        patches = ex.has_ntff ? ex.ntff.size() / 13 : 0;
        for (float v : s.sheet_table) sheet_branch.push_back(T(v));

        e.assign(3 * nn, T(0));
        h.assign(3 * nn, T(0));
        psi.assign(psi_total, T(0));
        current.assign(sheets.size() * states, T(0));
        debye_state.assign(debye_f.size() * s.poles.size(), T(0));
        series.assign(cap * ports * 2, T(0));
        plane.assign(plane_len, T(0));
        ntff.assign(patches * nf * 12, T(0));
        if (ex.has_ntff) patch_idx = ex.ntff;
        for (size_t q = 0; q < nf; ++q) omega.push_back(T(2.0 * PI * ex.freqs[q]));
        plane_k = ex.has_plane_k ? ex.plane_k : 0;
        w0 = T(2.0 * PI * pulse.f0);
    }

    size_t psi_base(size_t ee, size_t c, size_t a) const { return offsets[ee * 9 + c * 3 + a]; }

    // cpu.rs:48-107
    void update_h() {
        const size_t pml = sim.pml;
        const T k_mu = T(sim.dt / MU0);
        const auto& ax = sim.ax;
#pragma omp parallel for schedule(static)
        for (long ii = 0; ii < long(n[0]); ++ii) {
            size_t i = size_t(ii);
            for (size_t j = 0; j < n[1]; ++j)
                for (size_t k = 0; k < n[2]; ++k) {
                    N3 p = {i, j, k};
                    size_t id = (i * n[1] + j) * n[2] + k;
                    for (size_t c = 0; c < 3; ++c) {
                        size_t u = (c + 1) % 3, v = (c + 2) % 3;
                        if (p[u] + 1 >= n[u] || p[v] + 1 >= n[v]) continue;
                        N3 up = p, vp = p;
                        up[u] += 1;
                        vp[v] += 1;
                        T ev = e[v * nn + idx(n, up[0], up[1], up[2])] - e[v * nn + id];
                        T eu = e[u * nn + idx(n, vp[0], vp[1], vp[2])] - e[u * nn + id];
                        size_t pu = p[u], pv = p[v];
                        T t1 = ev * ax[u].inv_d[pu];
                        T t2 = eu * ax[v].inv_d[pv];
                        if (pml > 0) {
                            int su = ax[u].slot_h[pu];
                            if (su >= 0) {
                                T& r = psi[psi_base(1, c, u) + psi_idx(n, u, pml, p, size_t(su))];
                                r = ax[u].bh[pu] * r + ax[u].ch[pu] * ev * ax[u].raw_inv_d[pu];
                                t1 += r;
                            }
                            int sv = ax[v].slot_h[pv];
                            if (sv >= 0) {
                                T& r = psi[psi_base(1, c, v) + psi_idx(n, v, pml, p, size_t(sv))];
                                r = ax[v].bh[pv] * r + ax[v].ch[pv] * eu * ax[v].raw_inv_d[pv];
                                t2 += r;
                            }
                        }
                        h[c * nn + id] -= k_mu * (t1 - t2);
                    }
                }
        }
    }

    // cpu.rs:109-167
    void update_e() {
        const size_t pml = sim.pml;
        const auto& ax = sim.ax;
#pragma omp parallel for schedule(static)
        for (long ii = 0; ii < long(n[0]); ++ii) {
            size_t i = size_t(ii);
            for (size_t j = 0; j < n[1]; ++j)
                for (size_t k = 0; k < n[2]; ++k) {
                    N3 p = {i, j, k};
                    size_t id = (i * n[1] + j) * n[2] + k;
                    for (size_t c = 0; c < 3; ++c) {
                        T cb = sim.cb[c][id];
                        if (cb == T(0)) continue;
                        size_t u = (c + 1) % 3, v = (c + 2) % 3;
                        N3 um = p, vm = p;
                        um[u] -= 1;
                        vm[v] -= 1;
                        T hv = h[v * nn + id] - h[v * nn + idx(n, um[0], um[1], um[2])];
                        T hu = h[u * nn + id] - h[u * nn + idx(n, vm[0], vm[1], vm[2])];
                        size_t pu = p[u], pv = p[v];
                        T t1 = hv * ax[u].inv_dd[pu];
                        T t2 = hu * ax[v].inv_dd[pv];
                        if (pml > 0) {
                            int su = ax[u].slot_e[pu];
                            if (su >= 0) {
                                T& r = psi[psi_base(0, c, u) + psi_idx(n, u, pml, p, size_t(su))];
                                r = ax[u].be[pu] * r + ax[u].ce[pu] * hv * ax[u].raw_inv_dd[pu];
                                t1 += r;
                            }
                            int sv = ax[v].slot_e[pv];
                            if (sv >= 0) {
                                T& r = psi[psi_base(0, c, v) + psi_idx(n, v, pml, p, size_t(sv))];
                                r = ax[v].be[pv] * r + ax[v].ce[pv] * hu * ax[v].raw_inv_dd[pv];
                                t2 += r;
                            }
                        }
                        T& f = e[c * nn + id];
                        f = sim.ca[c][id] * f + cb * (t1 - t2);
                    }
                }
        }
    }

    // cpu.rs:169-193
    void sheet_before(size_t si, T old, T ha, T hb) {
        auto& sh = sheets[si];
        sh.old = old;
        T aa = sh.aa + ha * ha;
        T bb = sh.bb + hb * hb;
        T ab = sh.ab + ha * hb;
        sh.aa = aa;
        sh.bb = bb;
        sh.ab = ab;
        T sum = aa + bb;
        if (sum <= T(1e-30)) return;
        T scale = T(1);
        if (sh.adaptive != T(0)) {
            scale = sh.ma + sh.mb;
            T tot = aa + bb - T(2) * ab;
            if (tot > T(1e-30)) scale = std::clamp(sum / tot, T(0.5), T(4.0));
        }
        sh.ma = scale * aa / sum;
        sh.mb = scale * bb / sum;
    }

    // cpu.rs:195-237
    void sheet_after(size_t si) {
        auto& sh = sheets[si];
        const auto& br = sheet_branch;
        size_t f = sh.f;
        T len = sh.len, c = sh.c, r = sh.r;
        T ma = sh.ma, mb = sh.mb, old = sh.old, i_old = sh.i_old;
        size_t nr = size_t(br[0]), nc = size_t(br[1]);
        size_t stride = 2 + nr + 2 * nc;
        size_t faces = 4 + 2 * nr + 4 * nc;
        size_t fa = faces + sh.face_a * stride;
        size_t fb = faces + sh.face_b * stride;
        size_t base = si * (nr + 2 * nc);
        auto& cur = current;
        T hist = (ma * br[fa + 1] + mb * br[fb + 1]) * i_old;
        for (size_t k = 0; k < nr; ++k) hist -= (ma * br[fa + 2 + k] + mb * br[fb + 2 + k]) * cur[base + k];
        for (size_t k = 0; k < nc; ++k) {
            size_t o = 2 + nr + 2 * k;
            T cr = ma * br[fa + o] + mb * br[fb + o];
            T ci = ma * br[fa + o + 1] + mb * br[fb + o + 1];
            size_t u = base + nr + 2 * k;
            hist -= cr * cur[u] - ci * cur[u + 1];
        }
        T a = r * (ma * br[fa] + mb * br[fb]);
        T ibar = (T(0.5) * len * (e[f] + old) + r * hist) / (a + T(0.5) * len * c);
        e[f] -= c * ibar;
        sh.i_old = T(2) * ibar - i_old;
        for (size_t k = 0; k < nr; ++k) {
            size_t p = 4 + 2 * k;
            cur[base + k] = br[p] * cur[base + k] + br[p + 1] * ibar;
        }
        for (size_t k = 0; k < nc; ++k) {
            size_t p = 4 + 2 * nr + 4 * k;
            size_t u = base + nr + 2 * k;
            T ur = cur[u], ui = cur[u + 1];
            cur[u] = br[p] * ur - br[p + 1] * ui + br[p + 2] * ibar;
            cur[u + 1] = br[p] * ui + br[p + 1] * ur + br[p + 3] * ibar;
        }
    }

    // cpu.rs:239-260
    void debye_after(size_t si) {
        size_t f = debye_f[si];
        T dd = debye_dd[si], old = debye_old[si];
        T cb = sim.cb[f / nn][f % nn];
        size_t np = size_t(debye_table[0]);
        size_t count = debye_f.size();
        T s0 = T(0);
        for (size_t k = 0; k < np; ++k) s0 += T(0.5) * (T(1) + debye_table[1 + 2 * k]) * debye_state[k * count + si];
        T next = e[f] - cb * s0;
        e[f] = next;
        T de = next - old;
        for (size_t k = 0; k < np; ++k) {
            size_t q = k * count + si;
            debye_state[q] = debye_table[1 + 2 * k] * debye_state[q] + dd * debye_table[2 + 2 * k] * de;
        }
    }

    // cpu.rs:262-265
    T pulse_at(T t) const {
        T x = (t - T(t0)) / T(tau);
        return std::exp(-x * x) * std::cos(w0 * (t - T(t0)));
    }

    // cpu.rs:267-307
    void step(size_t ns) {
        update_h();
        for (size_t w = 0; w < sim.wires.size(); ++w) {
            const auto& wh = sim.wires[w];
            // h += e(1) + e(3) + e(5) + e(7), summed left to right (cpu.rs:270-273)
            T terms[4];
            for (int q = 0; q < 4; ++q) terms[q] = wh.terms[q].second * e[wh.terms[q].first];
            T acc = terms[0] + terms[1] + terms[2] + terms[3];
            h[wh.h] += acc;
        }
        for (size_t si = 0; si < sheets.size(); ++si)
            sheet_before(si, e[sheets[si].f], h[sheets[si].ha], h[sheets[si].hb]);
        for (size_t si = 0; si < debye_f.size(); ++si) debye_old[si] = e[debye_f[si]];
        update_e();
        for (size_t si = 0; si < sheets.size(); ++si) sheet_after(si);
        for (size_t si = 0; si < debye_f.size(); ++si) debye_after(si);
        T dt = T(sim.dt);
        T t = (T(ns) + T(0.5)) * dt;
        T pl = pulse_at(t);
        for (size_t q = 0; q + 2 < source.size(); q += 3) {
            size_t id = size_t(source[q]);
            T src = source[q + 1];
            size_t comp = size_t(source[q + 2]);
            e[comp * nn + id] -= src * pl;
        }
        for (size_t q = 0; q < inductor.size(); q += 5) {
            size_t f = size_t(inductor[q]) * nn + size_t(inductor[q + 1]);
            T x = e[f] - inductor[q + 2] * inductor[q + 4];
            e[f] = x;
            inductor[q + 4] += inductor[q + 3] * x;
        }
        probe(ns);
        field_dft(ns);
        far(ns);
    }

    // cpu.rs:309-334
    void probe(size_t ns) {
        for (size_t k = 0; k < ports; ++k) {
            const T* d = &probe_def[k * 8];
            size_t comp = size_t(d[0]);
            size_t first = size_t(d[1]), count = size_t(d[2]);
            size_t lf = size_t(d[3]), lc = size_t(d[4]);
            double v = 0.0;
            for (size_t q = first; q < first + count; ++q)
                v -= double(e[comp * nn + size_t(port_edges[2 * q])] * port_edges[2 * q + 1]);
            double cur = 0.0;
            for (size_t c = lf; c < lf + lc; ++c) {
                size_t hc = size_t(loops[3 * c + 1]) - 3;
                cur += double(h[hc * nn + size_t(loops[3 * c])] * loops[3 * c + 2]);
            }
            if (ns < cap) {
                series[(ns * ports + k) * 2] = T(v);
                series[(ns * ports + k) * 2 + 1] = T(cur);
            }
        }
    }

    // cpu.rs:336-361
    void field_dft(size_t ns) {
        if (plane_len == 0) return;
        const T dt = T(sim.dt);
        const T te = (T(ns) + T(1)) * dt;
        const T th = (T(ns) + T(0.5)) * dt;
        const size_t n1 = n[1], n2 = n[2];
#pragma omp parallel for schedule(static)
        for (long qq = 0; qq < long(n[0] * n[1]); ++qq) {
            size_t q = size_t(qq);
            size_t i = q / n1, j = q % n1;
            size_t id = (i * n1 + j) * n2 + plane_k;
            T f[5] = {e[id], e[nn + id], e[2 * nn + id], h[id], h[nn + id]};
            T* out = &plane[q * nf * 10];
            for (size_t k = 0; k < nf; ++k) {
                T w = omega[k];
                T ce0 = std::cos(w * te) * dt, ce1 = -std::sin(w * te) * dt;
                T ch0 = std::cos(w * th) * dt, ch1 = -std::sin(w * th) * dt;
                for (size_t c = 0; c < 5; ++c) {
                    T p0 = c >= 3 ? ch0 : ce0, p1 = c >= 3 ? ch1 : ce1;
                    out[k * 10 + 2 * c] += f[c] * p0;
                    out[k * 10 + 2 * c + 1] += f[c] * p1;
                }
            }
        }
    }

    // cpu.rs:363-415
    void far(size_t ns) {
        if (patches == 0 || nf == 0) return;
        const T dt = T(sim.dt);
        const T te = (T(ns) + T(1)) * dt;
        const T th = (T(ns) + T(0.5)) * dt;
#pragma omp parallel for schedule(static)
        for (long gg = 0; gg < long(patches); ++gg) {
            size_t g = size_t(gg);
            const uint32_t* b = &patch_idx[g * 13];
            uint32_t meta = b[0];
            size_t axis = meta & 3;
            T side = (meta & 4) ? T(1) : T(-1);
            size_t u = (axis + 1) % 3, v = (axis + 2) % 3;
            T ef[3] = {0, 0, 0}, hf[3] = {0, 0, 0};
            ef[u] = T(0.5) * (e[u * nn + b[1]] + e[u * nn + b[2]]);
            ef[v] = T(0.5) * (e[v * nn + b[3]] + e[v * nn + b[4]]);
            hf[u] = T(0.25) * (h[u * nn + b[5]] + h[u * nn + b[6]] + h[u * nn + b[7]] + h[u * nn + b[8]]);
            hf[v] = T(0.25) * (h[v * nn + b[9]] + h[v * nn + b[10]] + h[v * nn + b[11]] + h[v * nn + b[12]]);
            T nrm[3] = {0, 0, 0};
            nrm[axis] = side;
            T jv[3] = {nrm[1] * hf[2] - nrm[2] * hf[1], nrm[2] * hf[0] - nrm[0] * hf[2], nrm[0] * hf[1] - nrm[1] * hf[0]};
            T mv[3] = {ef[1] * nrm[2] - ef[2] * nrm[1], ef[2] * nrm[0] - ef[0] * nrm[2], ef[0] * nrm[1] - ef[1] * nrm[0]};
            T* out = &ntff[g * nf * 12];
            for (size_t k = 0; k < nf; ++k) {
                T wf = omega[k];
                T pe0 = std::cos(-wf * te) * dt, pe1 = std::sin(-wf * te) * dt;
                T ph0 = std::cos(-wf * th) * dt, ph1 = std::sin(-wf * th) * dt;
                size_t o = k * 12;
                for (size_t c = 0; c < 3; ++c) {
                    out[o + 2 * c] += ph0 * jv[c];
                    out[o + 2 * c + 1] += ph1 * jv[c];
                    out[o + 6 + 2 * c] += pe0 * mv[c];
                    out[o + 6 + 2 * c + 1] += pe1 * mv[c];
                }
            }
        }
    }

    // cpu.rs:417-421
    double energy() const {
        double se = 0.0, sh = 0.0;
#pragma omp parallel for reduction(+ : se, sh) schedule(static)
        for (long q = 0; q < long(e.size()); ++q) {
            double x = double(e[size_t(q)]);
            se += x * x;
            double y = double(h[size_t(q)]) * 376.73;
            sh += y * y;
        }
        return se + sh;
    }
};

// run_cpu (cpu.rs:424-482). progress(steps, decay) returns false to cancel.
template <class T>
Record<T> run_cpu(const Sim<T>& sim, size_t driven, const Pulse& pulse, const Extras& ex,
                  const std::function<bool(size_t, double)>& progress, bool keep_fields) {
    State<T> st(sim, driven, pulse, ex);
    size_t chunk = ex.check_every == 0 ? 1000 : ex.check_every;
    size_t pulse_end = size_t(2.0 * st.t0 / sim.dt);
    size_t steps = 0;
    double peak = 0.0, decay = 0.0;
    while (steps < ex.max_steps) {
        size_t k = std::min(chunk, ex.max_steps - steps);
        for (size_t s = 0; s < k; ++s) st.step(steps + s);
        steps += k;
        double e = st.energy();
        if (!std::isfinite(e)) throw Error("the FDTD run went unstable");
        peak = std::fmax(peak, e);
        decay = (e > 0.0 && peak > 0.0) ? 10.0 * std::log10(peak / e) : 0.0;
        if (!progress(steps, decay)) throw Error("cancelled");
        if (steps > std::max(pulse_end, ex.min_steps) && decay >= ex.decay_db) break;
    }
    Record<T> r;
    r.steps = steps;
    r.ports = st.ports;
    st.series.resize(steps * st.ports * 2);
    r.series = std::move(st.series);
    r.decay_db = decay;
    r.plane = std::move(st.plane);
    r.ntff = std::move(st.ntff);
    if (keep_fields) {
        r.e = std::move(st.e);
        r.h = std::move(st.h);
    }
    return r;
}

// patches (ntff.rs:11-59)
struct Patches {
    std::vector<std::array<double, 3>> pos;
    std::vector<double> area;
    std::vector<uint32_t> gpu;
};
template <class T>
Patches patches(const Sim<T>& sim, size_t inset) {
    N3 n = sim.dims();
    size_t p = sim.pml + inset;
    N3 lo = {p, p, p};
    N3 hi = {n[0] - 1 - p, n[1] - 1 - p, n[2] - 1 - p};
    const Grid& g = sim.grid;
    Patches out;
    for (size_t axis = 0; axis < 3; ++axis) {
        size_t u = (axis + 1) % 3, v = (axis + 2) % 3;
        std::pair<int, size_t> sides[2] = {{-1, lo[axis]}, {1, hi[axis]}};
        for (auto [side, plane] : sides)
            for (size_t a = lo[u]; a < hi[u]; ++a)
                for (size_t b = lo[v]; b < hi[v]; ++b) {
                    std::array<double, 3> pos{};
                    pos[axis] = g.axis(axis)[plane];
                    pos[u] = 0.5 * (g.axis(u)[a] + g.axis(u)[a + 1]);
                    pos[v] = 0.5 * (g.axis(v)[b] + g.axis(v)[b + 1]);
                    out.pos.push_back(pos);
                    out.area.push_back(sim.ax[u].d[a] * sim.ax[v].d[b]);
                    N3 q{0, 0, 0};
                    q[axis] = plane;
                    q[u] = a;
                    q[v] = b;
                    auto at = [&](std::initializer_list<std::pair<size_t, long>> moves) {
                        long r[3] = {long(q[0]), long(q[1]), long(q[2])};
                        for (auto [ax, d] : moves) r[ax] += d;
                        return uint32_t(idx(n, size_t(r[0]), size_t(r[1]), size_t(r[2])));
                    };
                    out.gpu.push_back(uint32_t(axis) | (side > 0 ? 4u : 0u));
                    for (uint32_t x : {at({}), at({{v, 1}}), at({}), at({{u, 1}})}) out.gpu.push_back(x);
                    for (uint32_t x : {at({}), at({{axis, -1}}), at({{u, 1}}), at({{axis, -1}, {u, 1}})}) out.gpu.push_back(x);
                    for (uint32_t x : {at({}), at({{axis, -1}}), at({{v, 1}}), at({{axis, -1}, {v, 1}})}) out.gpu.push_back(x);
                }
    }
    return out;
}

// Far (ntff.rs:61-137)
using Cx = std::array<double, 2>;
inline Cx cmul(Cx a, Cx b) { return {a[0] * b[0] - a[1] * b[1], a[0] * b[1] + a[1] * b[0]}; }
struct Far {
    std::vector<std::array<double, 3>> pos;
    std::vector<double> area;
    std::vector<std::array<Cx, 3>> j, m;
    double freq = 0;

    static Far load(const std::vector<std::array<double, 3>>& pos, const std::vector<double>& area,
                    const float* acc, size_t nf, size_t k, double freq, Cx scale) {
        Far f;
        size_t count = pos.size();
        for (size_t q = 0; q < count; ++q) {
            size_t o = (q * nf + k) * 12;
            auto c = [&](size_t x) { return cmul({double(acc[o + x]), double(acc[o + x + 1])}, scale); };
            f.j.push_back({c(0), c(2), c(4)});
            f.m.push_back({c(6), c(8), c(10)});
        }
        f.pos = pos;
        f.area = area;
        f.freq = freq;
        return f;
    }

    std::array<Cx, 3> field(const std::array<double, 3>& dir) const {
        double k = 2.0 * PI * freq / C0;
        Cx nn[3] = {{0, 0}, {0, 0}, {0, 0}}, ll[3] = {{0, 0}, {0, 0}, {0, 0}};
        for (size_t i = 0; i < pos.size(); ++i) {
            const auto& p = pos[i];
            double arg = k * (dir[0] * p[0] + dir[1] * p[1] + dir[2] * p[2]);
            Cx ph = {area[i] * std::cos(arg), area[i] * std::sin(arg)};
            for (int c = 0; c < 3; ++c) {
                Cx a = cmul(j[i][c], ph), b = cmul(m[i][c], ph);
                nn[c] = {nn[c][0] + a[0], nn[c][1] + a[1]};
                ll[c] = {ll[c][0] + b[0], ll[c][1] + b[1]};
            }
        }
        Cx rn = {0, 0};
        for (int c = 0; c < 3; ++c) rn = {rn[0] + nn[c][0] * dir[c], rn[1] + nn[c][1] * dir[c]};
        Cx perp[3];
        for (int c = 0; c < 3; ++c) perp[c] = {nn[c][0] - rn[0] * dir[c], nn[c][1] - rn[1] * dir[c]};
        Cx rl[3] = {{dir[1] * ll[2][0] - dir[2] * ll[1][0], dir[1] * ll[2][1] - dir[2] * ll[1][1]},
                    {dir[2] * ll[0][0] - dir[0] * ll[2][0], dir[2] * ll[0][1] - dir[0] * ll[2][1]},
                    {dir[0] * ll[1][0] - dir[1] * ll[0][0], dir[0] * ll[1][1] - dir[1] * ll[0][1]}};
        double scale = k / (4.0 * PI);
        std::array<Cx, 3> out;
        for (int c = 0; c < 3; ++c) out[c] = {(rl[c][0] - perp[c][0] * ETA0) * scale, (rl[c][1] - perp[c][1] * ETA0) * scale};
        return out;
    }

    double intensity(const std::array<double, 3>& dir) const {
        auto f = field(dir);
        double s = 0;
        for (auto& c : f) s += c[0] * c[0] + c[1] * c[1];
        return s / (2.0 * ETA0);
    }

    std::pair<double, double> radiated(size_t steps) const {
        double total = 0.0, peak = 0.0;
        for (size_t a = 0; a < steps; ++a) {
            double th = PI * (double(a) + 0.5) / double(steps);
            for (size_t b = 0; b < 2 * steps; ++b) {
                double ph = PI * double(b) / double(steps);
                std::array<double, 3> dir = {std::sin(th) * std::cos(ph), std::sin(th) * std::sin(ph), std::cos(th)};
                double u = intensity(dir);
                peak = std::fmax(peak, u);
                total += u * std::sin(th) * (PI / double(steps)) * (PI / double(steps));
            }
        }
        return {total, peak};
    }
};

}  // namespace oracle
