// The C ABI of include/fieldgrid.h. Thin: argument checks, error texts, and the run loop of
// run.rs:681-757 (chunks of check_every steps, energy check, decay, progress, early stop) on top of
// the device session.
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/fieldgrid.h"
#include "engine.hpp"

using namespace fg;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string& msg, char* err, size_t errlen) {
    g_last_error = msg;
    if (err && errlen) std::snprintf(err, errlen, "%s", msg.c_str());
    return code;
}

RunSpec run_spec(uint64_t driven, const fg_pulse* pulse, const fg_extras* x) {
    RunSpec rs;
    rs.driven = driven;
    rs.f0 = pulse->f0;
    rs.fc = pulse->fc;
    rs.max_steps = x->max_steps;
    if (x->freqs) rs.freqs.assign(x->freqs, x->freqs + x->n_freqs);
    rs.has_plane_k = x->has_plane_k != 0;
    rs.plane_k = x->plane_k;
    rs.has_ntff = x->ntff != nullptr;
    if (x->ntff) rs.ntff.assign(x->ntff, x->ntff + x->ntff_len);
    // Extras.fused_e picks the pipeline as in the reference (run.rs:430, :616-657): the fused
    // E+H march, or the separate H and E kernels.
    rs.fused = x->fused_e != 0;
    rs.profile = x->profile != 0;
    return rs;
}

struct Far {
    std::vector<double> pos, area, jm;  // jm: 12 doubles per patch (J then M, re/im, x y z)
    double freq = 0;
};

// FIELDGRID_SETUP_TIMES=1: fg_run prints the wall time of its phases to stderr
struct RunClock {
    bool on = false;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now(), last = t0;
    std::string text;
    RunClock() { const char* v = std::getenv("FIELDGRID_SETUP_TIMES"); on = v && v[0] == '1'; }
    void mark(const char* what) {
        if (!on) return;
        const auto now = std::chrono::steady_clock::now();
        char buf[64];
        std::snprintf(buf, sizeof buf, " %s %.2f ms;", what, std::chrono::duration<double, std::milli>(now - last).count());
        text += buf;
        last = now;
    }
    ~RunClock() {
        if (on) std::fprintf(stderr, "fg_run:%s total %.1f ms\n", text.c_str(),
                             std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
};

}  // namespace

namespace fg {
// lets other translation units of the library report through fg_last_error
void set_last_error(const std::string& msg) { g_last_error = msg; }
}  // namespace fg

struct fg_gpu { Gpu* g; };
struct fg_sim { HostSim* s; };
struct fg_session { Session* s; };
struct fg_far { Far f; };
struct fg_record {
    uint64_t steps = 0, ports = 0;
    double decay_db = 0;
    std::vector<float> series, plane, ntff, e, h;
    bool has_fields = false;
    uint64_t h2d = 0, d2h = 0;
};

extern "C" {

const char* fg_version(void) { return "fieldgrid-b200 0.1 (sm_100a)"; }
const char* fg_last_error(void) { return g_last_error.c_str(); }

int fg_gpu_open(int device, fg_gpu** out, char* err, size_t errlen) {
    if (!out) return fail(FG_ERR_INVALID, "null output handle", err, errlen);
    *out = nullptr;
    Gpu* g = nullptr;
    std::string e;
    int rc = gpu_open(device, &g, e);
    if (rc) return fail(rc, e, err, errlen);
    *out = new fg_gpu{g};
    return FG_OK;
}

void fg_gpu_close(fg_gpu* g) {
    if (!g) return;
    gpu_close(g->g);
    delete g;
}

int fg_gpu_name(const fg_gpu* g, char* dst, size_t len) {
    if (!g || !dst || !len) return FG_ERR_INVALID;
    std::snprintf(dst, len, "%s", g->g->name.c_str());
    return FG_OK;
}

int fg_sim_try_new(const fg_sim_spec* spec, fg_sim** out, char* err, size_t errlen) {
    if (!out) return fail(FG_ERR_INVALID, "null output handle", err, errlen);
    *out = nullptr;
    HostSim* s = nullptr;
    std::string e;
    int rc;
    try {
        rc = sim_try_new(spec, &s, e);
    } catch (const std::bad_alloc&) {
        return fail(FG_ERR_TOO_LARGE, "out of host memory building the grid", err, errlen);
    }
    if (rc) return fail(rc, e, err, errlen);
    *out = new fg_sim{s};
    return FG_OK;
}

void fg_sim_free(fg_sim* s) {
    if (!s) return;
    delete s->s;
    delete s;
}

double fg_sim_dt(const fg_sim* s) { return s ? s->s->dt : 0.0; }

void fg_sim_dims(const fg_sim* s, uint64_t n[3]) {
    for (int a = 0; a < 3; ++a) n[a] = s ? s->s->n[a] : 0;
}

uint64_t fg_sim_count(const fg_sim* sim, const char* what) {
    if (!sim || !what) return 0;
    const HostSim& s = *sim->s;
    std::string w(what);
    if (w == "ports") return s.ports.size();
    if (w == "inductors") return s.inductors.size();
    if (w == "sheets") return s.sheets.size();
    if (w == "debye_edges") return s.debye_edges.size();
    if (w == "wires") return s.wires.size();
    if (w.rfind("port_src", 0) == 0) {
        size_t p = std::strtoul(w.c_str() + 8, nullptr, 10);
        return p < s.port_src.size() ? s.port_src[p].size() : 0;
    }
    return 0;
}

int fg_sim_coefs(const fg_sim* sim, uint32_t comp, float* ca, float* cb) {
    if (!sim || comp > 2 || !ca || !cb) return FG_ERR_INVALID;
    const HostSim& s = *sim->s;
    for (size_t id = 0; id < s.nn; ++id) {
        const Coef& c = s.classes[s.cls(id)];
        ca[id] = c.ca[comp];
        cb[id] = c.cb[comp];
    }
    return FG_OK;
}

int fg_sim_wires(const fg_sim* sim, uint32_t* dst, uint64_t len) {
    if (!sim || !dst) return FG_ERR_INVALID;
    const HostSim& s = *sim->s;
    if (len < 9 * s.wires.size()) return FG_ERR_INVALID;
    for (size_t w = 0; w < s.wires.size(); ++w) {
        dst[9 * w] = uint32_t(s.wires[w].h);
        for (int t = 0; t < 4; ++t) {
            dst[9 * w + 1 + 2 * t] = uint32_t(s.wires[w].e[t]);
            std::memcpy(&dst[9 * w + 2 + 2 * t], &s.wires[w].c[t], 4);
        }
    }
    return FG_OK;
}

uint64_t fg_sim_coef_classes(const fg_sim* sim) { return sim ? sim->s->classes.size() : 0; }

double fg_time_step(const double* x, uint64_t nx, const double* y, uint64_t ny, const double* z, uint64_t nz) {
    std::vector<double> l[3] = {std::vector<double>(x, x + nx), std::vector<double>(y, y + ny),
                                std::vector<double>(z, z + nz)};
    return time_step(l);
}

int fg_session_new(fg_gpu* g, const fg_sim* sim, uint64_t driven, const fg_pulse* pulse, const fg_extras* extras,
                   fg_session** out, char* err, size_t errlen) {
    if (!out) return fail(FG_ERR_INVALID, "null output handle", err, errlen);
    *out = nullptr;
    if (!g) return fail(FG_ERR_NO_DEVICE, "no GPU: this engine has no CPU path", err, errlen);
    if (!sim || !pulse || !extras) return fail(FG_ERR_INVALID, "null argument", err, errlen);
    Session* s = nullptr;
    std::string e;
    int rc = session_new(g->g, *sim->s, run_spec(driven, pulse, extras), &s, e);
    if (rc) return fail(rc, e, err, errlen);
    *out = new fg_session{s};
    return FG_OK;
}

int fg_session_step(fg_session* s, uint64_t k) {
    if (!s) return FG_ERR_INVALID;
    std::string e;
    int rc = session_step(s->s, k, e);
    if (rc) g_last_error = e;
    return rc;
}

int fg_session_sync(fg_session* s) {
    if (!s) return FG_ERR_INVALID;
    std::string e;
    int rc = session_sync(s->s, e);
    if (rc) g_last_error = e;
    return rc;
}

int fg_session_energy(fg_session* s, double* out) {
    if (!s || !out) return FG_ERR_INVALID;
    std::string e;
    int rc = session_energy(s->s, out, e);
    if (rc) g_last_error = e;
    return rc;
}

uint64_t fg_session_steps(const fg_session* s) { return s ? session_steps(s->s) : 0; }

int fg_session_read(fg_session* s, const char* which, float* dst, uint64_t len) {
    if (!s || !which || (!dst && len)) return FG_ERR_INVALID;
    std::string e;
    int rc = session_read(s->s, which, dst, len, e);
    if (rc) g_last_error = e;
    return rc;
}

void* fg_session_stream(fg_session* s) { return s ? session_stream(s->s) : nullptr; }
uint64_t fg_session_launches_per_step(const fg_session* s) { return s ? session_launches_per_step(s->s) : 0; }
uint64_t fg_session_device_bytes(const fg_session* s) { return s ? session_device_bytes(s->s) : 0; }
const char* fg_session_variant(const fg_session* s) { return s ? session_variant(s->s) : ""; }

void fg_session_free(fg_session* s) {
    if (!s) return;
    session_free(s->s);
    delete s;
}

int fg_run(fg_gpu* g, const fg_sim* sim, uint64_t driven, const fg_pulse* pulse, const fg_extras* extras,
           fg_progress_fn progress, void* user, fg_record** out, char* err, size_t errlen) {
    if (!out) return fail(FG_ERR_INVALID, "null output handle", err, errlen);
    *out = nullptr;
    if (!g) return fail(FG_ERR_NO_DEVICE, "no GPU: this engine has no CPU path", err, errlen);
    if (!sim || !pulse || !extras) return fail(FG_ERR_INVALID, "null argument", err, errlen);
    RunClock clk;
    Session* s = nullptr;
    std::string e;
    RunSpec rs = run_spec(driven, pulse, extras);
    int rc = session_new(g->g, *sim->s, rs, &s, e);
    if (rc) return fail(rc, e, err, errlen);
    clk.mark("session_new");
    struct Free {   // the session goes back before the clock reports
        RunClock& c;
        void operator()(Session* x) const { session_free(x); c.mark("free"); }
    };
    std::unique_ptr<Session, Free> guard(s, Free{clk});
    // run.rs:681-748
    const uint64_t chunk = extras->check_every == 0 ? 1000 : extras->check_every;
    const uint64_t pulse_end = uint64_t(2.0 * session_t0(s) / sim->s->dt);
    uint64_t steps = 0;
    double peak = 0.0, decay = 0.0;
    while (steps < extras->max_steps) {
        const uint64_t k = std::min(chunk, extras->max_steps - steps);
        rc = session_step(s, k, e);
        if (rc) return fail(rc, e, err, errlen);
        steps += k;
        double en = 0.0;
        rc = session_energy(s, &en, e);
        if (rc) return fail(rc, e, err, errlen);
        if (!std::isfinite(en)) return fail(FG_ERR_UNSTABLE, "the FDTD run went unstable", err, errlen);
        peak = std::fmax(peak, en);
        decay = (en > 0.0 && peak > 0.0) ? 10.0 * std::log10(peak / en) : 0.0;
        if (progress && !progress(user, steps, decay)) return fail(FG_ERR_CANCELLED, "cancelled", err, errlen);
        if (steps > std::max(pulse_end, extras->min_steps) && decay >= extras->decay_db) break;
    }
    clk.mark("steps");
    auto rec = std::make_unique<fg_record>();
    rec->steps = steps;
    rec->ports = session_ports(s);
    rec->decay_db = decay;
    rec->series.resize(std::min<uint64_t>(steps, extras->max_steps) * rec->ports * 2);
    rc = session_read(s, "series", rec->series.data(), rec->series.size(), e);
    if (!rc) {
        rec->plane.resize(session_plane_len(s));
        rc = session_read(s, "plane", rec->plane.data(), rec->plane.size(), e);
    }
    if (!rc) {
        rec->ntff.resize(session_ntff_len(s));
        rc = session_read(s, "ntff", rec->ntff.data(), rec->ntff.size(), e);
    }
    if (!rc && extras->keep_fields) {
        rec->e.resize(3 * sim->s->nn);
        rec->h.resize(3 * sim->s->nn);
        rc = session_read(s, "e", rec->e.data(), rec->e.size(), e);
        if (!rc) rc = session_read(s, "h", rec->h.data(), rec->h.size(), e);
        rec->has_fields = true;
    }
    if (rc) return fail(rc, e, err, errlen);
    clk.mark("read");
    rec->h2d = session_h2d_bytes(s);
    rec->d2h = session_d2h_bytes(s);
    // the kernel report steps the session further, so it comes after the record is read
    if (rs.profile) session_profile(s);
    *out = rec.release();
    return FG_OK;
}

uint64_t fg_record_steps(const fg_record* r) { return r ? r->steps : 0; }
uint64_t fg_record_ports(const fg_record* r) { return r ? r->ports : 0; }
double fg_record_decay_db(const fg_record* r) { return r ? r->decay_db : 0.0; }

static const float* view(const std::vector<float>& v, uint64_t* len) {
    if (len) *len = v.size();
    return v.empty() ? nullptr : v.data();
}
const float* fg_record_series(const fg_record* r, uint64_t* len) { return r ? view(r->series, len) : nullptr; }
const float* fg_record_plane(const fg_record* r, uint64_t* len) { return r ? view(r->plane, len) : nullptr; }
const float* fg_record_ntff(const fg_record* r, uint64_t* len) { return r ? view(r->ntff, len) : nullptr; }
const float* fg_record_e(const fg_record* r, uint64_t* len) {
    if (!r || !r->has_fields) { if (len) *len = 0; return nullptr; }
    return view(r->e, len);
}
const float* fg_record_h(const fg_record* r, uint64_t* len) {
    if (!r || !r->has_fields) { if (len) *len = 0; return nullptr; }
    return view(r->h, len);
}
void fg_record_transfer(const fg_record* r, uint64_t* h2d, uint64_t* d2h) {
    if (h2d) *h2d = r ? r->h2d : 0;
    if (d2h) *d2h = r ? r->d2h : 0;
}
void fg_record_free(fg_record* r) { delete r; }

int fg_session_kernel_times(fg_session* s, uint64_t steps, char* names, double* ms, uint64_t cap, uint64_t* count) {
    if (!s || !count) return FG_ERR_INVALID;
    std::vector<std::pair<std::string, double>> t;
    std::string e;
    int rc = session_kernel_times(s->s, steps, t, e);
    if (rc) { g_last_error = e; return rc; }
    *count = t.size();
    for (uint64_t q = 0; q < t.size() && q < cap; ++q) {
        if (names) std::snprintf(names + 64 * q, 64, "%s", t[q].first.c_str());
        if (ms) ms[q] = t[q].second;
    }
    return FG_OK;
}

// ntff.rs:11-59
int fg_patches(const fg_sim* sim, uint64_t inset, uint32_t* dst, double* pos, double* area, uint64_t* count) {
    if (!sim || !count) return FG_ERR_INVALID;
    const HostSim& s = *sim->s;
    const size_t* n = s.n;
    const size_t p = s.pml + inset;
    for (int a = 0; a < 3; ++a)
        if (n[a] < 2 * p + 2) { *count = 0; return FG_OK; }
    const size_t lo[3] = {p, p, p};
    const size_t hi[3] = {n[0] - 1 - p, n[1] - 1 - p, n[2] - 1 - p};
    uint64_t q = 0;
    for (int axis = 0; axis < 3; ++axis) {
        const int u = (axis + 1) % 3, v = (axis + 2) % 3;
        const std::pair<int, size_t> sides[2] = {{-1, lo[axis]}, {1, hi[axis]}};
        for (auto [side, plane] : sides)
            for (size_t a = lo[u]; a < hi[u]; ++a)
                for (size_t b = lo[v]; b < hi[v]; ++b, ++q) {
                    if (pos) {
                        double* ps = pos + 3 * q;
                        ps[axis] = s.line[axis][plane];
                        ps[u] = 0.5 * (s.line[u][a] + s.line[u][a + 1]);
                        ps[v] = 0.5 * (s.line[v][b] + s.line[v][b + 1]);
                    }
                    if (area) area[q] = s.ax[u].d[a] * s.ax[v].d[b];
                    if (dst) {
                        size_t c0[3];
                        c0[axis] = plane;
                        c0[u] = a;
                        c0[v] = b;
                        auto at = [&](int d_axis, int d_u, int d_v) {
                            long r[3] = {long(c0[0]), long(c0[1]), long(c0[2])};
                            r[axis] += d_axis;
                            r[u] += d_u;
                            r[v] += d_v;
                            return uint32_t(s.idx(size_t(r[0]), size_t(r[1]), size_t(r[2])));
                        };
                        uint32_t* o = dst + 13 * q;
                        o[0] = uint32_t(axis) | (side > 0 ? 4u : 0u);
                        o[1] = at(0, 0, 0); o[2] = at(0, 0, 1); o[3] = at(0, 0, 0); o[4] = at(0, 1, 0);
                        o[5] = at(0, 0, 0); o[6] = at(-1, 0, 0); o[7] = at(0, 1, 0); o[8] = at(-1, 1, 0);
                        o[9] = at(0, 0, 0); o[10] = at(-1, 0, 0); o[11] = at(0, 0, 1); o[12] = at(-1, 0, 1);
                    }
                }
    }
    *count = q;
    return FG_OK;
}

// Far::load (ntff.rs:77-88)
int fg_far_load(const double* pos, const double* area, uint64_t count, const float* acc, uint64_t nf, uint64_t k,
                double freq, double scale_re, double scale_im, fg_far** out) {
    if (!out || (count && (!pos || !area || !acc)) || k >= nf) return FG_ERR_INVALID;
    auto f = std::make_unique<fg_far>();
    f->f.pos.assign(pos, pos + 3 * count);
    f->f.area.assign(area, area + count);
    f->f.freq = freq;
    f->f.jm.resize(12 * count);
    for (uint64_t q = 0; q < count; ++q) {
        const uint64_t o = (q * nf + k) * 12;
        for (int x = 0; x < 12; x += 2) {
            const double re = double(acc[o + x]), im = double(acc[o + x + 1]);
            f->f.jm[12 * q + x] = re * scale_re - im * scale_im;
            f->f.jm[12 * q + x + 1] = re * scale_im + im * scale_re;
        }
    }
    *out = f.release();
    return FG_OK;
}

void fg_far_free(fg_far* f) { delete f; }

// Far::field (ntff.rs:90-116) on the host, for callers without a GPU handle.
static void far_field_host(const Far& f, const double* dir, double* out) {
    const double k = 2.0 * PI * f.freq / C0;
    double nn[3][2] = {{0, 0}, {0, 0}, {0, 0}}, ll[3][2] = {{0, 0}, {0, 0}, {0, 0}};
    const size_t count = f.area.size();
    for (size_t i = 0; i < count; ++i) {
        const double* p = &f.pos[3 * i];
        const double arg = k * (dir[0] * p[0] + dir[1] * p[1] + dir[2] * p[2]);
        const double ph0 = f.area[i] * std::cos(arg), ph1 = f.area[i] * std::sin(arg);
        const double* jm = &f.jm[12 * i];
        for (int c = 0; c < 3; ++c) {
            const double jr = jm[2 * c], ji = jm[2 * c + 1], mr = jm[6 + 2 * c], mi = jm[6 + 2 * c + 1];
            nn[c][0] += jr * ph0 - ji * ph1;
            nn[c][1] += jr * ph1 + ji * ph0;
            ll[c][0] += mr * ph0 - mi * ph1;
            ll[c][1] += mr * ph1 + mi * ph0;
        }
    }
    double rn[2] = {0, 0};
    for (int c = 0; c < 3; ++c) { rn[0] += nn[c][0] * dir[c]; rn[1] += nn[c][1] * dir[c]; }
    double perp[3][2];
    for (int c = 0; c < 3; ++c) { perp[c][0] = nn[c][0] - rn[0] * dir[c]; perp[c][1] = nn[c][1] - rn[1] * dir[c]; }
    const double rl[3][2] = {{dir[1] * ll[2][0] - dir[2] * ll[1][0], dir[1] * ll[2][1] - dir[2] * ll[1][1]},
                             {dir[2] * ll[0][0] - dir[0] * ll[2][0], dir[2] * ll[0][1] - dir[0] * ll[2][1]},
                             {dir[0] * ll[1][0] - dir[1] * ll[0][0], dir[0] * ll[1][1] - dir[1] * ll[0][1]}};
    const double scale = k / (4.0 * PI);
    for (int c = 0; c < 3; ++c) {
        out[2 * c] = (rl[c][0] - perp[c][0] * ETA0) * scale;
        out[2 * c + 1] = (rl[c][1] - perp[c][1] * ETA0) * scale;
    }
}

int fg_far_field(fg_gpu* g, const fg_far* f, const double* dirs, uint64_t n, double* out) {
    if (!f || (n && (!dirs || !out))) return FG_ERR_INVALID;
    if (g) {
        std::string e;
        int rc = far_field_gpu(g->g, f->f.pos.data(), f->f.area.data(), f->f.jm.data(), f->f.area.size(), f->f.freq,
                               dirs, n, out, e);
        if (rc) g_last_error = e;
        return rc;
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (long long q = 0; q < (long long)n; ++q) far_field_host(f->f, dirs + 3 * q, out + 6 * q);
    return FG_OK;
}

int fg_far_intensity(fg_gpu* g, const fg_far* f, const double* dirs, uint64_t n, double* out) {
    if (!f || (n && (!dirs || !out))) return FG_ERR_INVALID;
    std::vector<double> fl(6 * n);
    int rc = fg_far_field(g, f, dirs, n, fl.data());
    if (rc) return rc;
    for (uint64_t q = 0; q < n; ++q) {
        double s = 0;
        for (int c = 0; c < 6; ++c) s += fl[6 * q + c] * fl[6 * q + c];
        out[q] = s / (2.0 * ETA0);
    }
    return FG_OK;
}

// The port's voltage and current spectra of sims-antenna's finish (sims-antenna/src/fdtd/mod.rs:
// 229-266): per frequency f, V = sum_n V_n dt e^{-j w (n+1) dt} and I = sum_n I_n dt e^{-j w (n+1/2) dt}
// (E is sampled at (n+1) dt, H at (n+1/2) dt), w = 2 pi f, with each phase factor advanced by one
// complex multiplication per step in f64 as the reference does (not re-evaluated per step).
int fg_port_spectra(const float* series, uint64_t steps, uint64_t ports, uint64_t port, double dt,
                    const double* freqs, uint64_t nf, double* v, double* i) {
    if ((steps && !series) || (nf && (!freqs || !v || !i)) || port >= ports || !(dt > 0.0)) {
        g_last_error = "fg_port_spectra: invalid arguments";
        return FG_ERR_INVALID;
    }
#pragma omp parallel for schedule(static)
    for (long long q = 0; q < (long long)nf; ++q) {
        const double w = 2.0 * PI * freqs[q];
        // C64::from_polar(r, t) = (r cos t, r sin t)
        const double re_rot = std::cos(-w * dt), im_rot = std::sin(-w * dt);
        double pe_re = dt * std::cos(-w * dt), pe_im = dt * std::sin(-w * dt);
        double ph_re = dt * std::cos(-w * 0.5 * dt), ph_im = dt * std::sin(-w * 0.5 * dt);
        double vr = 0.0, vi = 0.0, ir = 0.0, ii = 0.0;
        for (uint64_t n = 0; n < steps; ++n) {
            const double vn = double(series[(n * ports + port) * 2]), in = double(series[(n * ports + port) * 2 + 1]);
            vr += pe_re * vn;
            vi += pe_im * vn;
            ir += ph_re * in;
            ii += ph_im * in;
            // (a + bj)(c + dj) = (ac - bd) + (ad + bc)j
            const double per = pe_re * re_rot - pe_im * im_rot, pei = pe_re * im_rot + pe_im * re_rot;
            const double phr = ph_re * re_rot - ph_im * im_rot, phi = ph_re * im_rot + ph_im * re_rot;
            pe_re = per; pe_im = pei;
            ph_re = phr; ph_im = phi;
        }
        v[2 * q] = vr; v[2 * q + 1] = vi;
        i[2 * q] = ir; i[2 * q + 1] = ii;
    }
    return FG_OK;
}

// Far::radiated (ntff.rs:122-136)
int fg_far_radiated(fg_gpu* g, const fg_far* f, uint64_t steps, double* total, double* peak) {
    if (!f || !total || !peak || steps == 0) return FG_ERR_INVALID;
    std::vector<double> dirs;
    std::vector<double> th_of;
    for (uint64_t a = 0; a < steps; ++a) {
        const double th = PI * (double(a) + 0.5) / double(steps);
        for (uint64_t b = 0; b < 2 * steps; ++b) {
            const double ph = PI * double(b) / double(steps);
            dirs.insert(dirs.end(), {std::sin(th) * std::cos(ph), std::sin(th) * std::sin(ph), std::cos(th)});
            th_of.push_back(th);
        }
    }
    std::vector<double> u(th_of.size());
    int rc = fg_far_intensity(g, f, dirs.data(), th_of.size(), u.data());
    if (rc) return rc;
    double t = 0.0, pk = 0.0;
    const double w = (PI / double(steps)) * (PI / double(steps));
    for (size_t q = 0; q < u.size(); ++q) {
        pk = std::fmax(pk, u[q]);
        t += u[q] * std::sin(th_of[q]) * w;
    }
    *total = t;
    *peak = pk;
    return FG_OK;
}

// fg_flux_spec -> FluxSpec (the default window: the nodes inside the CPML)
static int flux_spec(const HostSim& hs, const fg_flux_spec* spec, FluxSpec& sp, std::string& e) {
    for (int a = 0; a < 3; ++a) { sp.lo[a] = spec->design_lo[a]; sp.hi[a] = spec->design_hi[a]; }
    sp.plane_k = spec->plane_k;
    for (int a = 0; a < 2; ++a) {
        sp.win_lo[a] = spec->window_lo[a];
        sp.win_hi[a] = spec->window_hi[a];
    }
    if (sp.win_hi[0] == 0 && sp.win_hi[1] == 0)
        for (int a = 0; a < 2; ++a) {
            sp.win_lo[a] = hs.pml;
            sp.win_hi[a] = hs.n[a] > hs.pml ? hs.n[a] - hs.pml : 0;
        }
    sp.freq = spec->freq;
    sp.steps = spec->steps;
    sp.checkpoints = spec->checkpoints;
    if (spec->transposes != 0 && spec->transposes != 1) { e = "transposes must be 0 or 1"; return FG_ERR_INVALID; }
    sp.transposes = spec->transposes;
    return FG_OK;
}

static void flux_out(const FluxResult& r, fg_flux_result* out) {
    out->objective = r.J;
    out->flux_re = r.f_re;
    out->flux_im = r.f_im;
    out->forward_ms = r.forward_ms;
    out->recompute_ms = r.recompute_ms;
    out->adjoint_ms = r.adjoint_ms;
    out->backward_ms = r.backward_ms;
    out->setup_ms = r.setup_ms;
    out->segments = r.segments;
    out->segment_len = r.segment_len;
    out->design_edges = r.design_edges;
}

int fg_flux_gradient(fg_gpu* g, const fg_sim* sim, uint64_t driven, const fg_pulse* pulse, const fg_flux_spec* spec,
                     fg_flux_result* out, double* grad_eps, double* grad_sigma, char* err, size_t errlen) {
    if (!g) return fail(FG_ERR_NO_DEVICE, "no GPU: this engine has no CPU path", err, errlen);
    if (!sim || !pulse || !spec || !out) return fail(FG_ERR_INVALID, "null argument", err, errlen);
    if ((grad_eps == nullptr) != (grad_sigma == nullptr))
        return fail(FG_ERR_INVALID, "grad_eps and grad_sigma are both given or both NULL", err, errlen);
    const HostSim& hs = *sim->s;
    FluxSpec sp;
    std::string e;
    if (int rc = flux_spec(hs, spec, sp, e)) return fail(rc, e, err, errlen);
    FluxResult r;
    const bool want = grad_eps != nullptr;
    if (spec->precision == 64 && want) return fail(FG_ERR_INVALID, "the FP64 forward computes the objective alone", err, errlen);
    int rc = spec->precision == 64 ? flux_objective64(g->g, hs, driven, pulse->f0, pulse->fc, sp, r, e)
                                   : flux_gradient(g->g, hs, driven, pulse->f0, pulse->fc, sp, want, r, e);
    if (rc) return fail(rc, e, err, errlen);
    flux_out(r, out);
    if (want) {
        std::copy(r.g_eps.begin(), r.g_eps.end(), grad_eps);
        std::copy(r.g_sig.begin(), r.g_sig.end(), grad_sigma);
    }
    return FG_OK;
}

int fg_flux_gradient_batch(fg_gpu* g, const fg_sim* const* sims, const uint64_t* driven, const fg_pulse* pulses,
                           const fg_flux_spec* specs, uint64_t count, int group, fg_flux_result* out,
                           double* const* grad_eps, double* const* grad_sigma, char* err, size_t errlen) {
    if (!g) return fail(FG_ERR_NO_DEVICE, "no GPU: this engine has no CPU path", err, errlen);
    if (count == 0) return fail(FG_ERR_INVALID, "an empty batch", err, errlen);
    if (!sims || !driven || !pulses || !specs || !out || !grad_eps || !grad_sigma)
        return fail(FG_ERR_INVALID, "null argument", err, errlen);
    std::vector<const HostSim*> hs(count);
    std::vector<uint64_t> dv(driven, driven + count);
    std::vector<std::pair<double, double>> pv(count);
    std::vector<FluxSpec> sv(count);
    std::string e;
    for (uint64_t q = 0; q < count; ++q) {
        if (!sims[q] || !grad_eps[q] || !grad_sigma[q]) return fail(FG_ERR_INVALID, "null argument", err, errlen);
        if (specs[q].precision == 64) return fail(FG_ERR_INVALID, "the FP64 forward computes the objective alone", err, errlen);
        hs[q] = sims[q]->s;
        pv[q] = {pulses[q].f0, pulses[q].fc};
        if (int rc = flux_spec(*hs[q], &specs[q], sv[q], e)) return fail(rc, "job " + std::to_string(q) + ": " + e, err, errlen);
    }
    std::vector<FluxResult> rs;
    int rc = flux_gradient_batch(g->g, hs, dv, pv, sv, group, rs, e);
    if (rc) return fail(rc, e, err, errlen);
    for (uint64_t q = 0; q < count; ++q) {
        flux_out(rs[q], &out[q]);
        std::copy(rs[q].g_eps.begin(), rs[q].g_eps.end(), grad_eps[q]);
        std::copy(rs[q].g_sig.begin(), rs[q].g_sig.end(), grad_sigma[q]);
    }
    return FG_OK;
}

struct fg_batch { Batch* b; };

int fg_batch_new(fg_gpu* g, const fg_sim* const* sims, const uint64_t* driven, const fg_pulse* pulses, uint64_t count,
                 uint64_t max_steps, const fg_batch_options* opt, fg_batch** out, char* err, size_t errlen) {
    if (!out) return fail(FG_ERR_INVALID, "null output handle", err, errlen);
    *out = nullptr;
    if (!g) return fail(FG_ERR_NO_DEVICE, "no GPU: this engine has no CPU path", err, errlen);
    if (!sims || !pulses || count == 0) return fail(FG_ERR_INVALID, "a batch needs grids and pulses", err, errlen);
    std::vector<const HostSim*> hs;
    std::vector<RunSpec> specs;
    for (uint64_t b = 0; b < count; ++b) {
        if (!sims[b]) return fail(FG_ERR_INVALID, "null grid in the batch", err, errlen);
        hs.push_back(sims[b]->s);
        RunSpec rs;
        rs.driven = driven ? driven[b] : 0;
        rs.f0 = pulses[b].f0;
        rs.fc = pulses[b].fc;
        rs.max_steps = max_steps;
        specs.push_back(rs);
    }
    fg_batch_options o{1, 0, 0, 32, 10};
    if (opt) o = *opt;
    Batch* B = nullptr;
    std::string e;
    int rc = batch_new_c(g->g, hs, specs, o.tune != 0, o.tile, o.blocks_per_sm, o.seg, o.graph_steps, &B, e);
    if (rc) return fail(rc, e, err, errlen);
    *out = new fg_batch{B};
    return FG_OK;
}

int fg_batch_step(fg_batch* b, uint64_t steps, char* err, size_t errlen) {
    if (!b) return fail(FG_ERR_INVALID, "null batch", err, errlen);
    std::string e;
    int rc = batch_step(*b->b, steps, e);
    return rc ? fail(rc, e, err, errlen) : FG_OK;
}

int fg_batch_sync(fg_batch* b) {
    if (!b) return FG_ERR_INVALID;
    std::string e;
    int rc = batch_sync(*b->b, e);
    if (rc) fg::set_last_error(e);
    return rc;
}

int fg_batch_read(fg_batch* b, uint64_t index, const char* which, float* dst, uint64_t len, char* err, size_t errlen) {
    if (!b || !which || !dst) return fail(FG_ERR_INVALID, "null argument", err, errlen);
    std::string e;
    int rc = batch_read(*b->b, index, which, dst, len, e);
    return rc ? fail(rc, e, err, errlen) : FG_OK;
}

int fg_batch_info(const fg_batch* b, fg_batch_options* opt, int* persistent_blocks, double* tuned_ms, uint64_t* steps) {
    if (!b) return FG_ERR_INVALID;
    int tile = 0, bps = 0, seg = 0;
    batch_info(*b->b, &tile, &bps, &seg, persistent_blocks, tuned_ms, steps);
    if (opt) *opt = fg_batch_options{0, tile, bps, seg, 0};
    return FG_OK;
}

void fg_batch_free(fg_batch* b) {
    if (!b) return;
    batch_free(b->b);
    delete b;
}


// ---- rasterisation (raster.rs) ----------------------------------------------------------------

static std::vector<double> line_of(const double* v, uint64_t n) { return std::vector<double>(v, v + n); }

static std::vector<double> centres_of(const std::vector<double>& l) {   // grid::centres (grid.rs:61-63)
    std::vector<double> c;
    for (size_t i = 0; i + 1 < l.size(); ++i) c.push_back(0.5 * (l[i] + l[i + 1]));
    return c;
}

int fg_raster_fill(fg_gpu* g, const double* tris, uint64_t ntri, const double* s0, uint64_t n0, const double* s1,
                   uint64_t n1, const double* s2, uint64_t n2, int order, uint8_t* inside, uint8_t* thin,
                   char* err, size_t errlen) {
    if (!g) return fail(FG_ERR_NO_DEVICE, "no GPU: this engine has no CPU path", err, errlen);
    if ((ntri && !tris) || !inside || !thin || (order != 0 && order != 1)) return fail(FG_ERR_INVALID, "invalid argument", err, errlen);
    const std::vector<double> s[3] = {line_of(s0, n0), line_of(s1, n1), line_of(s2, n2)};
    const size_t dims[3] = {size_t(n0), size_t(n1), size_t(n2)};
    std::string e;
    const int rc = raster_fill(g->g, tris, ntri, s, dims, order, inside, thin, e);
    return rc ? fail(rc, e, err, errlen) : FG_OK;
}

int fg_raster_solid_edges(fg_gpu* g, const double* tris, uint64_t ntri, const double* x, uint64_t nx,
                          const double* y, uint64_t ny, const double* z, uint64_t nz, uint8_t* mask,
                          char* err, size_t errlen) {
    if (!g) return fail(FG_ERR_NO_DEVICE, "no GPU: this engine has no CPU path", err, errlen);
    if ((ntri && !tris) || !mask || nx < 2 || ny < 2 || nz < 2) return fail(FG_ERR_INVALID, "invalid argument", err, errlen);
    const std::vector<double> lines[3] = {line_of(x, nx), line_of(y, ny), line_of(z, nz)};
    const size_t dims[3] = {size_t(nx), size_t(ny), size_t(nz)};
    const size_t nn = dims[0] * dims[1] * dims[2];
    std::vector<uint8_t> inside(nn), thin(nn);
    for (int c = 0; c < 3; ++c) {
        // raster.rs:148-151: centres along c, the grid lines along the other axes
        std::vector<double> s[3] = {lines[0], lines[1], lines[2]};
        s[c] = centres_of(lines[c]);
        std::string e;
        const int rc = raster_fill(g->g, tris, ntri, s, dims, 0, inside.data(), thin.data(), e);
        if (rc) return fail(rc, e, err, errlen);
        uint8_t* m = mask + size_t(c) * nn;
        for (size_t q = 0; q < nn; ++q) m[q] = uint8_t(inside[q] | thin[q]);
    }
    return FG_OK;
}

int fg_raster_solid_cells(fg_gpu* g, const double* tris, uint64_t ntri, const double* x, uint64_t nx,
                          const double* y, uint64_t ny, const double* z, uint64_t nz, uint8_t* mask,
                          char* err, size_t errlen) {
    if (!g) return fail(FG_ERR_NO_DEVICE, "no GPU: this engine has no CPU path", err, errlen);
    if ((ntri && !tris) || !mask || nx < 2 || ny < 2 || nz < 2) return fail(FG_ERR_INVALID, "invalid argument", err, errlen);
    const std::vector<double> s[3] = {centres_of(line_of(x, nx)), centres_of(line_of(y, ny)), centres_of(line_of(z, nz))};
    const size_t dims[3] = {s[0].size(), s[1].size(), s[2].size()};
    const size_t n = dims[0] * dims[1] * dims[2];
    std::vector<uint8_t> thin(n);
    std::string e;
    const int rc = raster_fill(g->g, tris, ntri, s, dims, 0, mask, thin.data(), e);
    if (rc) return fail(rc, e, err, errlen);
    for (size_t q = 0; q < n; ++q) mask[q] = uint8_t(mask[q] | thin[q]);
    return FG_OK;
}

int fg_raster_sheet_edges(fg_gpu* g, const double* tris, uint64_t ntri, const double* x, uint64_t nx,
                          const double* y, uint64_t ny, const double* z, uint64_t nz, uint8_t* mask,
                          char* err, size_t errlen) {
    if (!g) return fail(FG_ERR_NO_DEVICE, "no GPU: this engine has no CPU path", err, errlen);
    if ((ntri && !tris) || !mask || nx < 2 || ny < 2 || nz < 2) return fail(FG_ERR_INVALID, "invalid argument", err, errlen);
    const std::vector<double> lines[3] = {line_of(x, nx), line_of(y, ny), line_of(z, nz)};
    std::string e;
    const int rc = raster_sheet_edges(g->g, tris, ntri, lines, mask, e);
    return rc ? fail(rc, e, err, errlen) : FG_OK;
}

int fg_raster_closed(const double* tris, uint64_t ntri) { return (tris && raster_closed(tris, ntri)) ? 1 : 0; }

}  // extern "C"
