// TEST INFRASTRUCTURE — C exports of the oracle (fdtd_oracle.hpp) for tests/, smoke() and the
// cpu_baseline leg of bench.py. It takes the same fg_sim_spec / fg_extras structs as the product's
// C ABI (include/fieldgrid.h) so that both are driven from one description; it links nothing of
// the product. Prefix fgo_ = "fieldgrid oracle".
#include "fdtd_oracle.hpp"

#include <chrono>
#include <cstdio>
#include <memory>
#include <omp.h>

#include "../include/fieldgrid.h"

using namespace oracle;

namespace {

struct AnySim {
    int bits = 32;
    std::unique_ptr<Sim<float>> f;
    std::unique_ptr<Sim<double>> d;
};

struct AnyRecord {
    int bits = 32;
    Record<float> f;
    Record<double> d;
};

void set_err(char* err, size_t len, const char* msg) {
    if (err && len) {
        std::snprintf(err, len, "%s", msg);
    }
}

Grid grid_of(const fg_sim_spec* s) {
    Grid g;
    g.x.assign(s->x, s->x + s->nx);
    g.y.assign(s->y, s->y + s->ny);
    g.z.assign(s->z, s->z + s->nz);
    g.pml = s->pml;
    return g;
}

Edge edge_of(const fg_edge& e) { return Edge{e.comp, {size_t(e.at[0]), size_t(e.at[1]), size_t(e.at[2])}}; }

template <class T>
std::unique_ptr<Sim<T>> build(const fg_sim_spec* s) {
    Grid g = grid_of(s);
    size_t cells = g.cells();
    Materials m;
    m.eps = s->eps ? std::vector<float>(s->eps, s->eps + cells) : std::vector<float>(cells, 1.0f);
    m.sigma = s->sigma ? std::vector<float>(s->sigma, s->sigma + cells) : std::vector<float>(cells, 0.0f);
    m.inf = s->inf ? std::vector<float>(s->inf, s->inf + cells) : std::vector<float>(cells, 1.0f);
    m.debye = s->debye ? std::vector<float>(s->debye, s->debye + cells) : std::vector<float>(cells, 0.0f);
    N3 n = g.dims();
    size_t nn = n[0] * n[1] * n[2];
    std::function<bool(size_t, const N3&)> pec;
    if (s->pec_mask) {
        const uint8_t* mask = s->pec_mask;
        pec = [mask, n, nn](size_t c, const N3& p) { return mask[c * nn + idx(n, p[0], p[1], p[2])] != 0; };
    } else if (s->pec_fn) {
        fg_pec_fn fn = s->pec_fn;
        void* user = s->pec_user;
        pec = [fn, user](size_t c, const N3& p) {
            uint64_t at[3] = {p[0], p[1], p[2]};
            return fn(user, uint32_t(c), at) != 0;
        };
    } else {
        pec = [](size_t, const N3&) { return false; };
    }
    std::vector<Lumped> lumped;
    for (uint64_t q = 0; q < s->n_lumped; ++q) {
        Lumped l;
        for (uint64_t e = 0; e < s->lumped[q].n_edges; ++e) l.edges.push_back(edge_of(s->lumped[q].edges[e]));
        l.kind = s->lumped[q].element;
        l.value = s->lumped[q].value;
        lumped.push_back(l);
    }
    std::vector<PortDef> ports;
    for (uint64_t q = 0; q < s->n_ports; ++q) {
        const fg_port& p = s->ports[q];
        PortDef d;
        size_t at = 0;
        for (uint64_t c = 0; c < p.n_columns; ++c) {
            std::vector<Edge> col;
            for (uint64_t e = 0; e < p.column_len[c]; ++e) col.push_back(edge_of(p.edges[at++]));
            d.columns.push_back(col);
        }
        d.r = p.r;
        d.reference_above = p.reference_above != 0;
        ports.push_back(d);
    }
    std::vector<Resistive> res;
    for (uint64_t q = 0; q < s->n_resistive; ++q) {
        const fg_resistive& r = s->resistive[q];
        res.push_back(Resistive{r.comp, size_t(r.id), r.r, r.adaptive != 0, {size_t(r.faces[0]), size_t(r.faces[1])}});
    }
    Media media;
    if (s->sheet_table) {
        media.sheet_table.assign(s->sheet_table, s->sheet_table + s->sheet_table_len);
        media.sheet_states = s->sheet_states;
    }
    for (uint64_t q = 0; q < s->n_debye_poles; ++q) media.poles.emplace_back(s->debye_poles[2 * q], s->debye_poles[2 * q + 1]);
    for (uint64_t q = 0; q < s->n_wires; ++q) media.wires.emplace_back(edge_of(s->wires[q].edge), s->wires[q].radius);
    return std::make_unique<Sim<T>>(try_new<T>(std::move(g), m, pec, lumped, std::move(ports), res, media));
}

Extras extras_of(const fg_extras* x) {
    Extras e;
    e.min_steps = x->min_steps;
    e.max_steps = x->max_steps;
    e.decay_db = x->decay_db;
    if (x->freqs) e.freqs.assign(x->freqs, x->freqs + x->n_freqs);
    e.has_plane_k = x->has_plane_k != 0;
    e.plane_k = x->plane_k;
    e.has_ntff = x->ntff != nullptr;
    if (x->ntff) e.ntff.assign(x->ntff, x->ntff + x->ntff_len);
    e.check_every = x->check_every;
    return e;
}

template <class T>
uint64_t count_of(const Sim<T>& s, const char* what) {
    std::string w(what);
    if (w == "ports") return s.ports.size();
    if (w == "inductors") return s.inductors.size();
    if (w == "sheets") return s.sheets.size();
    if (w == "debye_edges") return s.debye_edges.size();
    if (w == "wires") return s.wires.size();
    if (w.rfind("port_src", 0) == 0) {
        size_t p = std::stoul(w.substr(8));
        return p < s.port_src.size() ? s.port_src[p].size() : 0;
    }
    return 0;
}

template <class T>
const std::vector<T>* pick(const Record<T>& r, const char* which) {
    std::string w(which);
    if (w == "series") return &r.series;
    if (w == "plane") return &r.plane;
    if (w == "ntff") return &r.ntff;
    if (w == "e") return &r.e;
    if (w == "h") return &r.h;
    return nullptr;
}

}  // namespace

extern "C" {

int fgo_threads(void) { return omp_get_max_threads(); }

int fgo_sim_try_new(const fg_sim_spec* spec, int bits, void** out, char* err, size_t errlen) {
    *out = nullptr;
    try {
        auto a = std::make_unique<AnySim>();
        a->bits = bits;
        if (bits == 64) a->d = build<double>(spec);
        else a->f = build<float>(spec);
        *out = a.release();
        return FG_OK;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return FG_ERR_SETUP;
    }
}

void fgo_sim_free(void* p) { delete static_cast<AnySim*>(p); }

double fgo_sim_dt(void* p) {
    auto* a = static_cast<AnySim*>(p);
    return a->bits == 64 ? a->d->dt : a->f->dt;
}

uint64_t fgo_sim_count(void* p, const char* what) {
    auto* a = static_cast<AnySim*>(p);
    return a->bits == 64 ? count_of(*a->d, what) : count_of(*a->f, what);
}

int fgo_sim_coefs(void* p, uint32_t comp, double* ca, double* cb) {
    auto* a = static_cast<AnySim*>(p);
    if (comp > 2) return FG_ERR_INVALID;
    if (a->bits == 64) {
        for (size_t q = 0; q < a->d->ca[comp].size(); ++q) { ca[q] = a->d->ca[comp][q]; cb[q] = a->d->cb[comp][q]; }
    } else {
        for (size_t q = 0; q < a->f->ca[comp].size(); ++q) { ca[q] = a->f->ca[comp][q]; cb[q] = a->f->cb[comp][q]; }
    }
    return FG_OK;
}

// Sim.wires: h, then 4 x (e index, coefficient) per wire.
int fgo_sim_wires(void* p, uint64_t* h, uint64_t* e, double* c) {
    auto* a = static_cast<AnySim*>(p);
    auto fill = [&](auto& s) {
        for (size_t w = 0; w < s.wires.size(); ++w) {
            h[w] = s.wires[w].h;
            for (int q = 0; q < 4; ++q) {
                e[4 * w + q] = s.wires[w].terms[q].first;
                c[4 * w + q] = double(s.wires[w].terms[q].second);
            }
        }
    };
    if (a->bits == 64) fill(*a->d);
    else fill(*a->f);
    return FG_OK;
}

// Sim.ax[axis] (sim.rs:12-27): per node inv_d, inv_dd, raw_inv_d, raw_inv_dd, be, ce, bh, ch,
// slot_e, slot_h (10 values, the order of the packed axis table, run.rs:205-212).
int fgo_sim_axis(void* p, uint32_t axis, double* out) {
    auto* a = static_cast<AnySim*>(p);
    if (axis > 2) return FG_ERR_INVALID;
    auto fill = [&](auto& s) {
        const auto& x = s.ax[axis];
        for (size_t q = 0; q < x.inv_d.size(); ++q) {
            const double v[10] = {double(x.inv_d[q]), double(x.inv_dd[q]), double(x.raw_inv_d[q]),
                                  double(x.raw_inv_dd[q]), double(x.be[q]), double(x.ce[q]), double(x.bh[q]),
                                  double(x.ch[q]), double(x.slot_e[q]), double(x.slot_h[q])};
            for (int f = 0; f < 10; ++f) out[10 * q + f] = v[f];
        }
    };
    if (a->bits == 64) fill(*a->d);
    else fill(*a->f);
    return FG_OK;
}

// The Sim's sparse lists: "debye" (comp, id; dd), "sources<p>" of port p (comp, id; src),
// "inductors" (comp, id; ke, ki), "poles" (-; x, a). idx gets 2 entries, val 2 per item.
int fgo_sim_list(void* p, const char* what, uint64_t* idx, double* val, uint64_t* count) {
    auto* a = static_cast<AnySim*>(p);
    const std::string w(what);
    auto fill = [&](auto& s) -> int {
        size_t n = 0;
        if (w == "debye") {
            for (auto& [c, id, dd] : s.debye_edges) { idx[2 * n] = c; idx[2 * n + 1] = id; val[2 * n] = dd; val[2 * n + 1] = 0; ++n; }
        } else if (w.rfind("sources", 0) == 0) {
            const size_t port = std::stoul(w.substr(7));
            if (port >= s.port_src.size()) return FG_ERR_INVALID;
            for (auto& [c, id, v] : s.port_src[port]) { idx[2 * n] = c; idx[2 * n + 1] = id; val[2 * n] = double(v); val[2 * n + 1] = 0; ++n; }
        } else if (w == "inductors") {
            for (auto& [c, id, ke, ki] : s.inductors) { idx[2 * n] = c; idx[2 * n + 1] = id; val[2 * n] = double(ke); val[2 * n + 1] = double(ki); ++n; }
        } else if (w == "poles") {
            for (auto& [x, am] : s.poles) { idx[2 * n] = 0; idx[2 * n + 1] = 0; val[2 * n] = x; val[2 * n + 1] = am; ++n; }
        } else {
            return FG_ERR_INVALID;
        }
        *count = n;
        return FG_OK;
    };
    return a->bits == 64 ? fill(*a->d) : fill(*a->f);
}

// Sim.sheets (sim.rs:197-206): idx gets comp, id, faces[0], faces[1]; val gets r, adaptive, len,
// c; table (NULL: count only) gets Sim.sheet_table.
int fgo_sim_sheets(void* p, uint64_t* idx, double* val, uint64_t* count, float* table, uint64_t* table_len) {
    auto* a = static_cast<AnySim*>(p);
    auto fill = [&](auto& s) {
        *count = s.sheets.size();
        *table_len = s.sheet_table.size();
        if (!idx) return;
        for (size_t q = 0; q < s.sheets.size(); ++q) {
            const auto& e = s.sheets[q];
            idx[4 * q] = e.comp; idx[4 * q + 1] = e.id; idx[4 * q + 2] = e.faces[0]; idx[4 * q + 3] = e.faces[1];
            val[4 * q] = e.r; val[4 * q + 1] = e.adaptive ? 1.0 : 0.0; val[4 * q + 2] = e.len; val[4 * q + 3] = e.c;
        }
        std::copy(s.sheet_table.begin(), s.sheet_table.end(), table);
    };
    if (a->bits == 64) fill(*a->d);
    else fill(*a->f);
    return FG_OK;
}

// port_loop (run.rs:102-127) for port `port`, around axis `axis` at height k.
int fgo_port_loop(void* p, uint64_t port, uint64_t axis, uint64_t k, uint64_t* ids, uint32_t* comps, double* w,
                  uint64_t cap, uint64_t* count) {
    auto* a = static_cast<AnySim*>(p);
    if (a->bits != 32 || port >= a->f->ports.size()) return FG_ERR_INVALID;
    auto lp = port_loop(*a->f, a->f->ports[port], axis, k);
    *count = lp.size();
    for (size_t q = 0; q < lp.size() && q < cap; ++q) {
        ids[q] = std::get<0>(lp[q]);
        comps[q] = uint32_t(std::get<1>(lp[q]));
        w[q] = std::get<2>(lp[q]);
    }
    return FG_OK;
}

// CoefSets::build (run.rs:72-99).
int fgo_coef_sets(void* p, uint64_t narrow, uint32_t* index, uint64_t index_cap, float* sets, uint64_t sets_cap,
                  uint64_t* n_index, uint64_t* n_sets, int* wide) {
    auto* a = static_cast<AnySim*>(p);
    if (a->bits != 32) return FG_ERR_INVALID;
    CoefSets cs = coef_sets(*a->f, narrow);
    *n_index = cs.index.size();
    *n_sets = cs.sets.size();
    *wide = cs.wide ? 1 : 0;
    if (index)
        for (size_t q = 0; q < cs.index.size() && q < index_cap; ++q) index[q] = cs.index[q];
    if (sets)
        for (size_t q = 0; q < cs.sets.size() && q < sets_cap; ++q) { sets[2 * q] = cs.sets[q][0]; sets[2 * q + 1] = cs.sets[q][1]; }
    return FG_OK;
}

// run_cpu (cpu.rs:424-482); keep_fields in extras also returns the final E/H.
int fgo_run_cpu(void* p, uint64_t driven, const fg_pulse* pulse, const fg_extras* extras, fg_progress_fn progress,
                void* user, void** out, char* err, size_t errlen) {
    *out = nullptr;
    auto* a = static_cast<AnySim*>(p);
    try {
        Extras ex = extras_of(extras);
        Pulse pl{pulse->f0, pulse->fc};
        std::function<bool(size_t, double)> prog = [&](size_t steps, double decay) {
            return progress ? progress(user, steps, decay) != 0 : true;
        };
        auto r = std::make_unique<AnyRecord>();
        r->bits = a->bits;
        if (a->bits == 64) r->d = run_cpu(*a->d, driven, pl, ex, prog, extras->keep_fields != 0);
        else r->f = run_cpu(*a->f, driven, pl, ex, prog, extras->keep_fields != 0);
        *out = r.release();
        return FG_OK;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        std::string m(e.what());
        if (m == "cancelled") return FG_ERR_CANCELLED;
        if (m == "the FDTD run went unstable") return FG_ERR_UNSTABLE;
        if (m == "grid too large for f32 port indices") return FG_ERR_PORT_INDEX;
        return FG_ERR_INVALID;
    }
}

uint64_t fgo_record_steps(void* p) {
    auto* r = static_cast<AnyRecord*>(p);
    return r->bits == 64 ? r->d.steps : r->f.steps;
}
double fgo_record_decay_db(void* p) {
    auto* r = static_cast<AnyRecord*>(p);
    return r->bits == 64 ? r->d.decay_db : r->f.decay_db;
}

uint64_t fgo_record_len(void* p, const char* which) {
    auto* r = static_cast<AnyRecord*>(p);
    if (r->bits == 64) { auto* v = pick(r->d, which); return v ? v->size() : 0; }
    auto* v = pick(r->f, which);
    return v ? v->size() : 0;
}

// Copies a record array widened to f64 (f32 values widen exactly).
int fgo_record_get(void* p, const char* which, double* dst) {
    auto* r = static_cast<AnyRecord*>(p);
    if (r->bits == 64) {
        auto* v = pick(r->d, which);
        if (!v) return FG_ERR_INVALID;
        std::copy(v->begin(), v->end(), dst);
    } else {
        auto* v = pick(r->f, which);
        if (!v) return FG_ERR_INVALID;
        for (size_t q = 0; q < v->size(); ++q) dst[q] = (*v)[q];
    }
    return FG_OK;
}

void fgo_record_free(void* p) { delete static_cast<AnyRecord*>(p); }

// patches (ntff.rs:11-59): dst == NULL asks for the count only.
int fgo_patches(void* p, uint64_t inset, uint32_t* gpu, double* pos, double* area, uint64_t* count) {
    auto* a = static_cast<AnySim*>(p);
    Patches ps = a->bits == 64 ? patches(*a->d, inset) : patches(*a->f, inset);
    *count = ps.area.size();
    if (gpu) std::copy(ps.gpu.begin(), ps.gpu.end(), gpu);
    if (pos)
        for (size_t q = 0; q < ps.pos.size(); ++q)
            for (int c = 0; c < 3; ++c) pos[3 * q + c] = ps.pos[q][c];
    if (area) std::copy(ps.area.begin(), ps.area.end(), area);
    return FG_OK;
}

// Far::load + Far::field / intensity (ntff.rs:77-120) for n directions.
int fgo_far_eval(const double* pos, const double* area, uint64_t count, const float* acc, uint64_t nf, uint64_t k,
                 double freq, double scale_re, double scale_im, const double* dirs, uint64_t n, double* field,
                 double* intensity) {
    std::vector<std::array<double, 3>> ps(count);
    for (size_t q = 0; q < count; ++q) ps[q] = {pos[3 * q], pos[3 * q + 1], pos[3 * q + 2]};
    std::vector<double> ar(area, area + count);
    Far f = Far::load(ps, ar, acc, nf, k, freq, {scale_re, scale_im});
#pragma omp parallel for schedule(dynamic, 4)
    for (long q = 0; q < long(n); ++q) {
        std::array<double, 3> d = {dirs[3 * q], dirs[3 * q + 1], dirs[3 * q + 2]};
        auto fl = f.field(d);
        if (field)
            for (int c = 0; c < 3; ++c) { field[6 * q + 2 * c] = fl[c][0]; field[6 * q + 2 * c + 1] = fl[c][1]; }
        if (intensity) {
            double s = 0;
            for (auto& c : fl) s += c[0] * c[0] + c[1] * c[1];
            intensity[q] = s / (2.0 * ETA0);
        }
    }
    return FG_OK;
}

// Far::radiated (ntff.rs:122-136).
int fgo_far_radiated(const double* pos, const double* area, uint64_t count, const float* acc, uint64_t nf, uint64_t k,
                     double freq, double scale_re, double scale_im, uint64_t steps, double* total, double* peak) {
    std::vector<std::array<double, 3>> ps(count);
    for (size_t q = 0; q < count; ++q) ps[q] = {pos[3 * q], pos[3 * q + 1], pos[3 * q + 2]};
    std::vector<double> ar(area, area + count);
    Far f = Far::load(ps, ar, acc, nf, k, freq, {scale_re, scale_im});
    auto [t, pk] = f.radiated(steps);
    *total = t;
    *peak = pk;
    return FG_OK;
}

// The CPU baseline: builds the stepper State of run_cpu (cpu.rs:431-453) and times `steps` calls
// of State::step (cpu.rs:267-307) with all OpenMP threads, excluding the state set-up.
int fgo_time_steps(void* p, uint64_t driven, const fg_pulse* pulse, const fg_extras* extras, uint64_t warmup,
                   uint64_t steps, double* seconds, char* err, size_t errlen) {
    auto* a = static_cast<AnySim*>(p);
    if (a->bits != 32) return FG_ERR_INVALID;
    try {
        State<float> st(*a->f, driven, Pulse{pulse->f0, pulse->fc}, extras_of(extras));
        for (uint64_t s = 0; s < warmup; ++s) st.step(s);
        auto t0 = std::chrono::steady_clock::now();
        for (uint64_t s = 0; s < steps; ++s) st.step(warmup + s);
        auto t1 = std::chrono::steady_clock::now();
        *seconds = std::chrono::duration<double>(t1 - t0).count();
        return FG_OK;
    } catch (const std::exception& e) {
        set_err(err, errlen, e.what());
        return FG_ERR_INVALID;
    }
}

}  // extern "C"
