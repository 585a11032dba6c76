// Grid setup of the B200 engine: the product's Sim::try_new (sims-field/src/fdtd/sim.rs:352-635).
//
// The per-edge arithmetic is the reference's (same f64 operations in the same order, then the
// same casts to f32), so every edge gets bit-identical (ca, cb). The organisation is this
// engine's own:
//   * no nn-long f64 temporaries: an edge's 4-cell material average is formed where it is used;
//   * the few edges that lumped elements, ports, sheets and thin wires rewrite are resolved first,
//     in the reference's order, in a small map;
//   * one OpenMP pass over x-planes then settles every node's three edges, collects the Debye
//     edges and interns the node's (ca, cb) triple into the class table (per-thread tables merged
//     in plane order, so the result does not depend on scheduling).
// Compile with -ffp-contract=off: a fused multiply-add would change the f64 roundings.
#include <omp.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <map>
#include <memory>
#include <set>
#include <unordered_map>
#include <unordered_set>

#include "../../include/fieldgrid.h"
#include "host.hpp"

namespace fg {

double time_step(const std::vector<double>* line) {  // sim.rs:133-137
    double s = 0.0;
    for (int a = 0; a < 3; ++a) {
        double m = INFINITY;
        for (size_t i = 0; i + 1 < line[a].size(); ++i) m = std::fmin(m, line[a][i + 1] - line[a][i]);
        s += 1.0 / (m * m);
    }
    return 0.99 / (C0 * std::sqrt(s));
}

void pulse_shape(double fc, double& t0, double& tau) {  // sim.rs:646-649
    tau = std::sqrt(std::log(10.0)) / (PI * fc);
    t0 = 4.0 * tau;
}

namespace {

// sim.rs:29-131: spacings, CPML grading (m = 3, kappa_max = 1, alpha_max = 0.05) and psi slots.
Axis make_axis(const std::vector<double>& line, size_t pml, double dt) {
    const size_t n = line.size();
    Axis a;
    a.n = n;
    a.d.resize(n);
    a.dd.resize(n);
    for (size_t i = 0; i < n; ++i) a.d[i] = (i + 1 < n) ? line[i + 1] - line[i] : line[i] - line[i - 1];
    for (size_t i = 0; i < n; ++i)
        a.dd[i] = (i == 0) ? a.d[0] : (i + 1 >= n ? a.d[n - 2] : 0.5 * (line[i + 1] - line[i - 1]));
    std::vector<double> ke(n, 1.0), kh(n, 1.0);
    a.node.assign(n, AxisNode{0, 0, 0, 0, 0, 0, 0, 0, -1, -1});
    a.node64.assign(n, AxisNode64{0, 0, 0, 0, 0, 0, 0, 0, -1, -1});
    if (pml > 0 && n > 2 * pml + 2) {
        const double m = 3.0, kappa_max = 1.0, alpha_max = 0.05;
        const double left = line[pml], right = line[n - 1 - pml];
        const double depth_l = left - line[0], depth_r = line[n - 1] - right;
        // graded conductivity at distance rho into a layer of the given depth
        auto grade = [&](double x, double& kappa, double& b, double& c) -> bool {
            double rho, depth, cell;
            if (x < left) { rho = left - x; depth = depth_l; cell = a.d[0]; }
            else if (x > right) { rho = x - right; depth = depth_r; cell = a.d[n - 2]; }
            else return false;
            if (!(rho > 0.0)) return false;
            double r = std::clamp(rho / depth, 0.0, 1.0);
            double sigma = 0.8 * (m + 1.0) / (ETA0 * cell) * std::pow(r, m);
            kappa = 1.0 + (kappa_max - 1.0) * std::pow(r, m);
            double alpha = alpha_max * (1.0 - r) * 2.0 * PI * EPS0 * 1e9;
            b = std::exp(-(sigma / kappa + alpha) * dt / EPS0);
            c = sigma > 0.0 ? sigma * (b - 1.0) / (sigma * kappa + kappa * kappa * alpha) : 0.0;
            return true;
        };
        for (size_t i = 0; i < n; ++i) {
            double k, b, c;
            if (grade(line[i], k, b, c)) {
                ke[i] = k;
                a.node[i].be = float(b); a.node[i].ce = float(c);
                a.node64[i].be = b; a.node64[i].ce = c;
            }
            if (i < pml) a.node[i].slot_e = int32_t(i);
            else if (i > n - 1 - pml) a.node[i].slot_e = int32_t(i + 2 * pml - n);
            if (i + 1 < n) {
                if (grade(0.5 * (line[i] + line[i + 1]), k, b, c)) {
                    kh[i] = k;
                    a.node[i].bh = float(b); a.node[i].ch = float(c);
                    a.node64[i].bh = b; a.node64[i].ch = c;
                }
                if (i < pml) a.node[i].slot_h = int32_t(i);
                else if (i >= n - 1 - pml) a.node[i].slot_h = int32_t(pml + i - (n - 1 - pml));
            }
        }
    }
    for (size_t i = 0; i < n; ++i) {
        a.node[i].inv_d = float(1.0 / (kh[i] * a.d[i]));
        a.node[i].inv_dd = float(1.0 / (ke[i] * a.dd[i]));
        a.node[i].raw_inv_d = float(1.0 / a.d[i]);
        a.node[i].raw_inv_dd = float(1.0 / a.dd[i]);
        AxisNode64& w = a.node64[i];
        w.inv_d = 1.0 / (kh[i] * a.d[i]);
        w.inv_dd = 1.0 / (ke[i] * a.dd[i]);
        w.raw_inv_d = 1.0 / a.d[i];
        w.raw_inv_dd = 1.0 / a.dd[i];
        w.slot_e = a.node[i].slot_e;
        w.slot_h = a.node[i].slot_h;
    }
    return a;
}

// sim.rs:303-313
bool wire_factor(double d, double radius, double& f, std::string& err) {
    double lo = d * std::exp(-4.0), hi = 0.5 * d;
    if (radius >= lo && radius < hi) {
        f = 2.0 / std::log(d / radius);
        return true;
    }
    char buf[256];
    std::snprintf(buf, sizeof buf,
                  "a thin wire's radius must be from a 55th to half of its cell (%.3e to %.3e m), not %.3e m", lo,
                  hi, radius);
    err = buf;
    return false;
}

struct CoefKey {
    uint32_t w[6];
    bool operator==(const CoefKey& o) const { return std::memcmp(w, o.w, sizeof w) == 0; }
};
struct CoefHash {
    size_t operator()(const CoefKey& k) const {
        uint64_t h = 1469598103934665603ull;
        for (uint32_t v : k.w) { h ^= v; h *= 1099511628211ull; h ^= h >> 29; }
        return size_t(h);
    }
};
CoefKey key_of(const Coef& c) {
    CoefKey k;
    std::memcpy(k.w, &c, sizeof k.w);
    return k;
}

}  // namespace

// Builds the host model. Returns FG_OK or an error with the reference's message.
int sim_try_new(const fg_sim_spec* spec, HostSim** out, std::string& err) {
    *out = nullptr;
    if (!spec || !spec->x || !spec->y || !spec->z || spec->nx < 2 || spec->ny < 2 || spec->nz < 2) {
        err = "a grid needs at least two node lines per axis";
        return FG_ERR_INVALID;
    }
    auto s = std::make_unique<HostSim>();
    HostSim& S = *s;
    S.line[0].assign(spec->x, spec->x + spec->nx);
    S.line[1].assign(spec->y, spec->y + spec->ny);
    S.line[2].assign(spec->z, spec->z + spec->nz);
    S.pml = spec->pml;
    for (int a = 0; a < 3; ++a) S.n[a] = S.line[a].size();
    const size_t* n = S.n;
    const size_t nn = n[0] * n[1] * n[2];
    S.nn = nn;
    const size_t cells = S.cells();

    // wire_cells (sim.rs:315-336) and the time step (sim.rs:362-364)
    double speedup = 1.0;
    for (uint64_t q = 0; q < spec->n_wires; ++q) {
        const fg_edge& e = spec->wires[q].edge;
        double radius = spec->wires[q].radius;
        if (e.comp > 2) { err = "a wire edge has a component above 2"; return FG_ERR_INVALID; }
        size_t p[3] = {size_t(e.at[0]), size_t(e.at[1]), size_t(e.at[2])};
        size_t end[3] = {p[0], p[1], p[2]};
        end[e.comp] += 1;
        auto clear = [&](const size_t* q) {
            for (int a = 0; a < 3; ++a)
                if (!(q[a] > S.pml && q[a] + 1 + S.pml < n[a])) return false;
            return true;
        };
        if (!clear(p) || !clear(end)) { err = "a thin wire must stay clear of the grid's absorbing layer"; return FG_ERR_SETUP; }
        for (uint32_t axis : {(e.comp + 1) % 3, (e.comp + 2) % 3})
            for (const size_t* node : std::initializer_list<const size_t*>{p, end})
                for (size_t cell : {node[axis], node[axis] - 1}) {
                    double f;
                    if (!wire_factor(S.line[axis][cell + 1] - S.line[axis][cell], radius, f, err)) return FG_ERR_SETUP;
                    speedup = std::fmax(speedup, std::fmax(f, 1.0 / f));
                }
    }
    const double dt = time_step(S.line) / std::sqrt(speedup);
    S.dt = dt;
    for (int a = 0; a < 3; ++a) S.ax[a] = make_axis(S.line[a], S.pml, dt);

    // materials (sim.rs:285-301); NULL arrays are Materials::new's defaults
    const float* m_eps = spec->eps;
    const float* m_sig = spec->sigma;
    const float* m_inf = spec->inf;
    const float* m_dd = spec->debye;
    if (m_eps) S.cell_eps.assign(m_eps, m_eps + cells);
    if (m_sig) S.cell_sig.assign(m_sig, m_sig + cells);
    auto mat = [&](size_t ci, size_t cj, size_t ck, double out4[4]) {
        size_t id = (ci * (n[1] - 1) + cj) * (n[2] - 1) + ck;
        out4[0] = m_eps ? double(m_eps[id]) : 1.0;
        out4[1] = m_sig ? double(m_sig[id]) : 0.0;
        out4[2] = m_inf ? double(m_inf[id]) : 1.0;
        out4[3] = m_dd ? double(m_dd[id]) : 0.0;
    };
    (void)cells;
    // sim.rs:375-410 for one edge: {EPS0 * eps, sigma, inf, debye} or zeros off the interior
    auto average = [&](uint32_t c, size_t i, size_t j, size_t k, double r[4]) -> bool {
        const size_t p[3] = {i, j, k};
        const uint32_t u = (c + 1) % 3, v = (c + 2) % 3;
        if (p[c] + 1 >= n[c] || p[u] == 0 || p[u] + 1 >= n[u] || p[v] == 0 || p[v] + 1 >= n[v]) {
            r[0] = r[1] = r[2] = r[3] = 0.0;
            return false;
        }
        double sum[4] = {0, 0, 0, 0}, w_sum = 0.0;
        static const int offs[4][2] = {{-1, -1}, {0, -1}, {-1, 0}, {0, 0}};
        for (auto& o : offs) {
            long cell[3] = {long(i), long(j), long(k)};
            cell[u] += o[0];
            cell[v] += o[1];
            double w = S.ax[u].d[size_t(cell[u])] * S.ax[v].d[size_t(cell[v])];
            size_t cc[3];
            for (int a = 0; a < 3; ++a) cc[a] = size_t(std::clamp<long>(cell[a], 0, long(n[a]) - 2));
            double m4[4];
            mat(cc[0], cc[1], cc[2], m4);
            for (int q = 0; q < 4; ++q) sum[q] += m4[q] * w;
            w_sum += w;
        }
        r[0] = EPS0 * sum[0] / w_sum;
        r[1] = sum[1] / w_sum;
        r[2] = sum[2] / w_sum;
        r[3] = sum[3] / w_sum;
        return true;
    };
    auto key = [&](uint32_t c, size_t id) { return uint64_t(c) * nn + id; };
    auto nid = [&](const fg_edge& e) { return S.idx(size_t(e.at[0]), size_t(e.at[1]), size_t(e.at[2])); };
    auto area = [&](const fg_edge& e) {
        uint32_t u = (e.comp + 1) % 3, v = (e.comp + 2) % 3;
        return S.ax[u].dd[e.at[u]] * S.ax[v].dd[e.at[v]];
    };
    auto length = [&](const fg_edge& e) { return S.ax[e.comp].d[e.at[e.comp]]; };
    auto check_edge = [&](const fg_edge& e) {
        return e.comp <= 2 && e.at[0] < n[0] && e.at[1] < n[1] && e.at[2] < n[2];
    };

    // PEC predicate (sim.rs:442-454)
    std::function<bool(uint32_t, size_t, size_t, size_t)> pec;
    if (spec->pec_mask) {
        const uint8_t* mask = spec->pec_mask;
        pec = [mask, &S, nn](uint32_t c, size_t i, size_t j, size_t k) { return mask[c * nn + S.idx(i, j, k)] != 0; };
    } else if (spec->pec_fn) {
        fg_pec_fn fn = spec->pec_fn;
        void* user = spec->pec_user;
        pec = [fn, user](uint32_t c, size_t i, size_t j, size_t k) {
            uint64_t at[3] = {i, j, k};
            return fn(user, c, at) != 0;
        };
    }

    // capacitors and resistors (sim.rs:416-430)
    std::unordered_map<uint64_t, double> eps_over;
    std::vector<std::pair<fg_edge, double>> series_r;
    std::unordered_set<uint64_t> excluded;
    for (uint64_t q = 0; q < spec->n_lumped; ++q) {
        const fg_lumped& l = spec->lumped[q];
        double count = double(std::max<uint64_t>(l.n_edges, 1));
        for (uint64_t t = 0; t < l.n_edges; ++t) {
            const fg_edge& e = l.edges[t];
            if (!check_edge(e)) { err = "a lumped element's edge is outside the grid"; return FG_ERR_INVALID; }
            size_t id = nid(e);
            if (l.element == FG_CAPACITOR) {
                auto it = eps_over.find(key(e.comp, id));
                double cur;
                if (it != eps_over.end()) cur = it->second;
                else { double r[4]; average(e.comp, e.at[0], e.at[1], e.at[2], r); cur = r[0]; }
                eps_over[key(e.comp, id)] = cur + l.value * count * length(e) / area(e);
            } else if (l.element == FG_RESISTOR) {
                series_r.emplace_back(e, l.value / count);
            }
            excluded.insert(key(e.comp, id));
        }
    }
    for (uint64_t q = 0; q < spec->n_ports; ++q) {
        const fg_port& p = spec->ports[q];
        PortDef d;
        uint64_t at = 0;
        if (p.n_columns == 0) { err = "a port needs at least one column"; return FG_ERR_INVALID; }
        for (uint64_t c = 0; c < p.n_columns; ++c) {
            std::vector<Edge> col;
            if (p.column_len[c] == 0) { err = "a port column needs at least one edge"; return FG_ERR_INVALID; }
            for (uint64_t t = 0; t < p.column_len[c]; ++t) {
                const fg_edge& e = p.edges[at++];
                if (!check_edge(e)) { err = "a port edge is outside the grid"; return FG_ERR_INVALID; }
                col.push_back(Edge{e.comp, {size_t(e.at[0]), size_t(e.at[1]), size_t(e.at[2])}});
                excluded.insert(key(e.comp, nid(e)));
            }
            d.columns.push_back(std::move(col));
        }
        d.r = p.r;
        d.reference_above = p.reference_above != 0;
        S.ports.push_back(std::move(d));
    }
    for (uint64_t q = 0; q < spec->n_resistive; ++q) {
        const fg_resistive& r = spec->resistive[q];
        if (r.comp > 2 || r.id >= nn) { err = "a resistive edge is outside the grid"; return FG_ERR_INVALID; }
        excluded.insert(key(r.comp, r.id));
    }
    double half_g = 0.0;  // sim.rs:469-470
    for (uint64_t q = 0; q < spec->n_debye_poles; ++q) {
        double x = spec->debye_poles[2 * q], a = spec->debye_poles[2 * q + 1];
        half_g += a * x * dt / (1.0 + 0.5 * x * dt);
        S.poles.emplace_back(x, a);
    }
    half_g *= 0.5;

    // The value an edge has after ca/cb (sim.rs:431-441), PEC (:442-454) and Debye (:469-483).
    // Returns whether the edge is a Debye edge and its weight.
    auto base = [&](uint32_t c, size_t i, size_t j, size_t k, float& ca, float& cb, double& dd_out) -> bool {
        double r[4];
        average(c, i, j, k, r);
        size_t id = S.idx(i, j, k);
        double eps = r[0];
        if (!eps_over.empty()) {
            auto it = eps_over.find(key(c, id));
            if (it != eps_over.end()) eps = it->second;
        }
        ca = 0.f;
        cb = 0.f;
        if (eps != 0.0) {
            double x = r[1] * dt / (2.0 * eps);
            ca = float((1.0 - x) / (1.0 + x));
            cb = float(dt / eps / (1.0 + x));
        }
        if (pec && pec(c, i, j, k)) { ca = 0.f; cb = 0.f; }
        double dd = r[3];
        if (dd <= 0.0 || cb == 0.f || (!excluded.empty() && excluded.count(key(c, id)))) return false;
        double eps_d = EPS0 * (r[2] + dd * half_g);
        ca = 1.f;
        cb = float(dt / eps_d);
        dd_out = dd;
        return true;
    };

    // Edges rewritten after the base pass, resolved in the reference's order.
    std::unordered_map<uint64_t, std::pair<float, float>> over;
    auto current = [&](uint32_t c, size_t id) -> std::pair<float, float> {
        auto it = over.find(key(c, id));
        if (it != over.end()) return it->second;
        size_t i = id / (n[1] * n[2]), j = (id / n[2]) % n[1], k = id % n[2];
        float ca, cb;
        double dd;
        base(c, i, j, k, ca, cb, dd);
        return {ca, cb};
    };
    auto resistor = [&](const fg_edge& e, double r) -> double {  // sim.rs:484-492
        size_t id = nid(e);
        double avg[4];
        average(e.comp, e.at[0], e.at[1], e.at[2], avg);
        double eps = avg[0];
        auto it = eps_over.find(key(e.comp, id));
        if (it != eps_over.end()) eps = it->second;
        double x_sig = avg[1] * dt / (2.0 * eps);
        double beta = dt * length(e) / (2.0 * r * eps * area(e)) + x_sig;
        over[key(e.comp, id)] = {float((1.0 - beta) / (1.0 + beta)), float(dt / (eps * (1.0 + beta)))};
        return dt / (eps * (1.0 + beta) * r * area(e));
    };
    for (auto& [e, r] : series_r) resistor(e, r);  // sim.rs:493-496
    for (uint64_t q = 0; q < spec->n_resistive; ++q) {  // sim.rs:497-509
        const fg_resistive& r = spec->resistive[q];
        size_t i = r.id / (n[1] * n[2]), j = (r.id / n[2]) % n[1], k = r.id % n[2];
        fg_edge e{r.comp, 0, {i, j, k}};
        S.sheets.push_back(SheetEdge{r.comp, r.id, r.r, r.adaptive != 0, {r.faces[0], r.faces[1]}, length(e),
                                     double(current(r.comp, r.id).second) / area(e)});
    }
    for (uint64_t q = 0; q < spec->n_ports; ++q) {  // sim.rs:510-523
        const fg_port& p = spec->ports[q];
        double cols = double(std::max<uint64_t>(p.n_columns, 1));
        std::vector<SrcEdge> v;
        uint64_t at = 0;
        for (uint64_t c = 0; c < p.n_columns; ++c) {
            double m = double(std::max<uint64_t>(p.column_len[c], 1));
            double re = p.r * cols / m;
            for (uint64_t t = 0; t < p.column_len[c]; ++t) {
                const fg_edge& e = p.edges[at++];
                double src = resistor(e, re);
                v.push_back(SrcEdge{e.comp, nid(e), float(src / m)});
            }
        }
        S.port_src.push_back(std::move(v));
    }
    for (uint64_t q = 0; q < spec->n_lumped; ++q) {  // sim.rs:524-534
        const fg_lumped& l = spec->lumped[q];
        if (l.element != FG_INDUCTOR) continue;
        double count = double(std::max<uint64_t>(l.n_edges, 1));
        for (uint64_t t = 0; t < l.n_edges; ++t) {
            const fg_edge& e = l.edges[t];
            size_t id = nid(e);
            double k_e = double(current(e.comp, id).second) / area(e);
            double k_i = dt * length(e) / (l.value / count);
            S.inductors.push_back(Inductor{e.comp, id, float(k_e), float(k_i)});
        }
    }
    if (spec->sheet_table) {
        S.sheet_table.assign(spec->sheet_table, spec->sheet_table + spec->sheet_table_len);
        S.sheet_states = spec->sheet_states;
    } else {
        S.sheet_table.assign(4, 0.f);
        S.sheet_states = 0;
    }

    // thin_wire (sim.rs:556-635)
    {
        const double k_mu = dt / MU0;
        auto wkey = [&](uint32_t c, const size_t* p) { return uint64_t(c) * nn + S.idx(p[0], p[1], p[2]); };
        std::set<uint64_t> on_wire;
        for (uint64_t q = 0; q < spec->n_wires; ++q) {
            const fg_edge& e = spec->wires[q].edge;
            size_t p[3] = {size_t(e.at[0]), size_t(e.at[1]), size_t(e.at[2])};
            on_wire.insert(wkey(e.comp, p));
        }
        struct HEntry { size_t q[3]; uint32_t c; double f; };
        std::map<uint64_t, HEntry> scaled_h;
        std::map<uint64_t, double> scaled_e;
        for (uint64_t q = 0; q < spec->n_wires; ++q) {
            const fg_edge& e = spec->wires[q].edge;
            double radius = spec->wires[q].radius;
            uint32_t w = e.comp;
            size_t p[3] = {size_t(e.at[0]), size_t(e.at[1]), size_t(e.at[2])};
            size_t end[3] = {p[0], p[1], p[2]};
            end[w] += 1;
            for (uint32_t axis : {(w + 1) % 3, (w + 2) % 3}) {
                uint32_t c = 3 - w - axis;
                size_t qm[3] = {p[0], p[1], p[2]};
                qm[axis] -= 1;
                const size_t* hq[2] = {p, qm};
                size_t hcell[2] = {p[axis], p[axis] - 1};
                for (int t = 0; t < 2; ++t) {
                    double f;
                    if (!wire_factor(S.ax[axis].d[hcell[t]], radius, f, err)) return FG_ERR_SETUP;
                    HEntry he{{hq[t][0], hq[t][1], hq[t][2]}, c, f};
                    scaled_h.emplace(wkey(c, hq[t]), he);
                }
                const size_t* nodes2[2] = {p, end};
                for (const size_t* node : nodes2) {
                    size_t nm[3] = {node[0], node[1], node[2]};
                    nm[axis] -= 1;
                    const size_t* eq[2] = {node, nm};
                    size_t ecell[2] = {node[axis], node[axis] - 1};
                    for (int t = 0; t < 2; ++t) {
                        uint64_t id = wkey(axis, eq[t]);
                        if (!on_wire.count(id)) {
                            double f;
                            if (!wire_factor(S.ax[axis].d[ecell[t]], radius, f, err)) return FG_ERR_SETUP;
                            scaled_e.emplace(id, f);
                        }
                    }
                }
            }
        }
        for (auto& [id, f] : scaled_e) {
            uint32_t c = uint32_t(id / nn);
            size_t at = id % nn;
            auto [caf, cbf] = current(c, at);
            double ca = double(caf), cb = double(cbf);
            if (cb == 0.0) continue;
            double a = (1.0 - ca) / (1.0 + ca);
            double scaled = a / f;
            over[key(c, at)] = {float((1.0 - scaled) / (1.0 + scaled)), float(cb * (1.0 + a) / (f * (1.0 + scaled)))};
        }
        for (auto& [h, he] : scaled_h) {
            uint32_t c = he.c, u = (c + 1) % 3, v = (c + 2) % 3;
            double sc = (he.f - 1.0) * k_mu;
            double du = double(S.ax[u].node[he.q[u]].inv_d), dv = double(S.ax[v].node[he.q[v]].inv_d);
            size_t qu[3] = {he.q[0], he.q[1], he.q[2]}, qv[3] = {he.q[0], he.q[1], he.q[2]};
            qu[u] += 1;
            qv[v] += 1;
            std::pair<uint64_t, double> all[4] = {
                {wkey(v, qu), -sc * du}, {wkey(v, he.q), sc * du}, {wkey(u, qv), sc * dv}, {wkey(u, he.q), -sc * dv}};
            WireH wh;
            wh.h = h;
            for (int t = 0; t < 4; ++t) { wh.e[t] = h; wh.c[t] = 0.f; }
            int slot = 0;
            for (auto& [ei, cc] : all)
                if (!on_wire.count(ei)) { wh.e[slot] = ei; wh.c[slot] = float(cc); ++slot; }
            S.wires.push_back(wh);
        }
    }

    // One pass over x-planes: settle every node's triple, collect Debye edges, intern classes.
    S.node_class.assign(nn, 0);
    const int threads = std::max(1, std::min<int>(omp_get_max_threads(), int(n[0])));
    struct Local {
        std::unordered_map<CoefKey, uint32_t, CoefHash> lookup;
        std::vector<Coef> table;
        std::vector<DebyeEdge> debye[3];
        size_t i0 = 0, i1 = 0;
    };
    std::vector<Local> loc(threads);
#pragma omp parallel num_threads(threads)
    {
        int t = omp_get_thread_num();
        Local& L = loc[t];
        L.i0 = n[0] * size_t(t) / size_t(threads);
        L.i1 = n[0] * size_t(t + 1) / size_t(threads);
        uint32_t last_id = 0;
        CoefKey last_key;
        bool have_last = false;
        for (size_t i = L.i0; i < L.i1; ++i)
            for (size_t j = 0; j < n[1]; ++j)
                for (size_t k = 0; k < n[2]; ++k) {
                    size_t id = S.idx(i, j, k);
                    Coef cf;
                    for (uint32_t c = 0; c < 3; ++c) {
                        float ca, cb;
                        double dd = 0;
                        bool deb = base(c, i, j, k, ca, cb, dd);
                        if (deb) L.debye[c].push_back(DebyeEdge{c, id, dd});
                        if (!over.empty()) {
                            auto it = over.find(key(c, id));
                            if (it != over.end()) { ca = it->second.first; cb = it->second.second; }
                        }
                        if (cb == 0.f) ca = 0.f;  // an edge with cb == 0 is never updated
                        cf.ca[c] = ca;
                        cf.cb[c] = cb;
                    }
                    CoefKey kk = key_of(cf);
                    if (!(have_last && kk == last_key)) {
                        auto it = L.lookup.find(kk);
                        if (it == L.lookup.end()) {
                            last_id = uint32_t(L.table.size());
                            L.lookup.emplace(kk, last_id);
                            L.table.push_back(cf);
                        } else last_id = it->second;
                        last_key = kk;
                        have_last = true;
                    }
                    S.node_class[id] = last_id;
                }
    }
    std::unordered_map<CoefKey, uint32_t, CoefHash> global;
    std::vector<std::vector<uint32_t>> remap(threads);
    for (int t = 0; t < threads; ++t) {
        for (auto& cf : loc[t].table) {
            auto kk = key_of(cf);
            auto it = global.find(kk);
            uint32_t g;
            if (it == global.end()) {
                g = uint32_t(S.classes.size());
                global.emplace(kk, g);
                S.classes.push_back(cf);
            } else g = it->second;
            remap[t].push_back(g);
        }
    }
    // the global ids, in 16 bits when the classes allow (half the host memory, and half the bytes the
    // upload reads)
    const bool narrow = S.classes.size() <= size_t(65536);
    if (narrow) S.node_class16.resize(nn);
#pragma omp parallel num_threads(threads)
    {
        int t = omp_get_thread_num();
        const auto& rm = remap[t];
        size_t a = loc[t].i0 * n[1] * n[2], b = loc[t].i1 * n[1] * n[2];
        if (narrow)
            for (size_t id = a; id < b; ++id) S.node_class16[id] = uint16_t(rm[S.node_class[id]]);
        else
            for (size_t id = a; id < b; ++id) S.node_class[id] = rm[S.node_class[id]];
    }
    if (narrow) std::vector<uint32_t>().swap(S.node_class);
    for (uint32_t c = 0; c < 3; ++c)
        for (int t = 0; t < threads; ++t)
            S.debye_edges.insert(S.debye_edges.end(), loc[t].debye[c].begin(), loc[t].debye[c].end());
    *out = s.release();
    return FG_OK;
}

}  // namespace fg
