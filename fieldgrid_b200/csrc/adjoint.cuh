// Host side of the adjoint: the flux objective's value and its gradient with respect to the
// permittivity and conductivity of every voxel of a design box, from one forward run on the
// fused march and one backward sweep of the adjoint kernels (adjoint_kernels.cuh).
//
// Objective: F = sum over the plane window of dA (Ex^ conj(Hy^) - Ey^ conj(Hx^)) at one frequency,
// with Ex^ .. Hy^ the running DFT of the z-plane plane_k the forward already accumulates
// (cpu.rs:336-361) and dA = dd_x(i) dd_y(j); J = |F|^2.
//
// Memory: with checkpoints = 0 the forward keeps every step's E^n and S^n of the design edges;
// otherwise it keeps the full state at the start of about `checkpoints` segments of an even number
// of steps, and the backward sweep re-runs each segment from its checkpoint (recording that
// segment's history) before sweeping it: segment recomputation with O(sqrt(N)) field checkpoints
// when checkpoints ~ sqrt(N). A re-run marches only the shrinking box of nodes that can still
// reach the design edges within the segment (FluxJob::rerun_cone), on a second stream while the
// sweep of the following segment runs.
//
// Included at the end of engine.cu (it uses the Session internals).
#pragma once

#include <chrono>
#include <complex>
#include <functional>
#include <memory>
#include <unordered_set>

namespace fg {

namespace {

// One design edge: its averaging cells and the derivatives of its (ca, cb) with respect to the
// edge's permittivity (F/m) and conductivity, from sim.rs:375-441 (x = sigma dt / 2 eps,
// ca = (1 - x)/(1 + x), cb = dt / eps / (1 + x), eps and sigma the area-weighted averages of the
// four cells around the edge).
struct DesignEdgeInfo {
    int4 at;                    // (comp, i, j, k)
    size_t cell[4];             // cell indices into the design box, or SIZE_MAX outside it
    double w[4];                // averaging weights / their sum
    double dca_de, dca_ds, dcb_de, dcb_ds;
};

bool design_edges(const HostSim& sim, const FluxSpec& sp, std::vector<DesignEdgeInfo>& out, std::string& err) {
    const size_t* n = sim.n;
    const double dt = sim.dt;
    const size_t bw[3] = {sp.hi[0] - sp.lo[0], sp.hi[1] - sp.lo[1], sp.hi[2] - sp.lo[2]};
    auto cell_eps = [&](size_t ci, size_t cj, size_t ck) {
        const size_t id = (ci * (n[1] - 1) + cj) * (n[2] - 1) + ck;
        return sim.cell_eps.empty() ? 1.0 : double(sim.cell_eps[id]);
    };
    auto cell_sig = [&](size_t ci, size_t cj, size_t ck) {
        const size_t id = (ci * (n[1] - 1) + cj) * (n[2] - 1) + ck;
        return sim.cell_sig.empty() ? 0.0 : double(sim.cell_sig[id]);
    };
    std::unordered_set<uint64_t> debye;   // (comp, node) of every Debye edge
    for (const auto& q : sim.debye_edges) debye.insert(uint64_t(q.comp) * sim.nn + q.id);
    for (uint32_t c = 0; c < 3; ++c) {
        const uint32_t u = (c + 1) % 3, v = (c + 2) % 3;
        size_t lo[3], hi[3];   // edges whose averaging cells meet the box
        lo[c] = sp.lo[c];
        hi[c] = sp.hi[c];
        lo[u] = sp.lo[u];
        hi[u] = sp.hi[u] + 1;
        lo[v] = sp.lo[v];
        hi[v] = sp.hi[v] + 1;
        for (size_t i = lo[0]; i < hi[0]; ++i)
            for (size_t j = lo[1]; j < hi[1]; ++j)
                for (size_t k = lo[2]; k < hi[2]; ++k) {
                    const size_t p[3] = {i, j, k};
                    if (p[c] + 1 >= n[c] || p[u] == 0 || p[u] + 1 >= n[u] || p[v] == 0 || p[v] + 1 >= n[v]) {
                        err = "the design box touches the grid boundary";
                        return false;
                    }
                    DesignEdgeInfo e{};
                    e.at = make_int4(int(c), int(i), int(j), int(k));
                    static const int offs[4][2] = {{-1, -1}, {0, -1}, {-1, 0}, {0, 0}};
                    double se = 0, ss = 0, wsum = 0, wq[4];
                    for (int q = 0; q < 4; ++q) {
                        size_t cc[3] = {i, j, k};
                        cc[u] = size_t(long(p[u]) + offs[q][0]);
                        cc[v] = size_t(long(p[v]) + offs[q][1]);
                        wq[q] = sim.ax[u].d[cc[u]] * sim.ax[v].d[cc[v]];
                        se += cell_eps(cc[0], cc[1], cc[2]) * wq[q];
                        ss += cell_sig(cc[0], cc[1], cc[2]) * wq[q];
                        wsum += wq[q];
                        bool in = true;
                        for (int a = 0; a < 3; ++a) in = in && cc[a] >= sp.lo[a] && cc[a] < sp.hi[a];
                        e.cell[q] = in ? ((cc[0] - sp.lo[0]) * bw[1] + (cc[1] - sp.lo[1])) * bw[2] + (cc[2] - sp.lo[2])
                                       : SIZE_MAX;
                    }
                    for (int q = 0; q < 4; ++q) e.w[q] = wq[q] / wsum;
                    const double eps = EPS0 * se / wsum, sig = ss / wsum;
                    const double x = sig * dt / (2.0 * eps);
                    // the edge must carry exactly the plain coefficients (no PEC, lumped element,
                    // port or Debye override)
                    const size_t id = sim.idx(i, j, k);
                    if (debye.count(uint64_t(c) * sim.nn + id) || sim.ca(c, id) != float((1.0 - x) / (1.0 + x)) ||
                        sim.cb(c, id) != float(dt / eps / (1.0 + x))) {
                        err = "the design box overlaps an edge with a PEC, lumped, port or Debye override";
                        return false;
                    }
                    const double den = eps + 0.5 * sig * dt;
                    e.dca_de = 2.0 * x / (eps * (1.0 + x) * (1.0 + x));
                    e.dca_ds = -dt / (eps * (1.0 + x) * (1.0 + x));
                    e.dcb_de = -dt / (den * den);
                    e.dcb_ds = -0.5 * dt * dt / (den * den);
                    out.push_back(e);
                }
    }
    return true;
}

}  // namespace

// Sets a session's history base and step counter in stream order (a launch carries the values,
// so no host buffer has to outlive the call).
__global__ void k_adj_set(long long* base, long long b, unsigned* counter, unsigned cnt, int set_counter) {
    if (base) *base = b;
    if (set_counter) *counter = cnt;
}

// One flux-gradient run in phases, so that many of them can be in flight on one GPU (each on its
// own streams): prepare (checks and every allocation), forward (enqueued), objective (waits for
// its forward, forms J and the adjoint weights), backward (enqueued), finish (waits, chain rule).
struct FluxJob {
    Gpu* gpu = nullptr;
    const HostSim* sim = nullptr;
    uint64_t driven = 0;
    double f0 = 0, fc = 0;
    FluxSpec sp;
    bool want_grad = true;
    FluxResult res;
    std::string err;

    std::vector<DesignEdgeInfo> info;
    std::vector<int4> edges;
    uint64_t N = 0, L = 0, S = 0;
    bool ckpt = false, sep = false;
    Session* s = nullptr;
    size_t fbytes = 0, pbytes = 0, nd_s = 0, dbytes = 0;
    struct Ck { float *e = nullptr, *h = nullptr, *psi = nullptr, *deb = nullptr; };
    std::vector<Ck> cks;
    char* ck_mem = nullptr;   // all checkpoints in one allocation
    float *lE[2] = {nullptr, nullptr}, *lH[2] = {nullptr, nullptr}, *lpsi[2] = {nullptr, nullptr}, *dw = nullptr;
    float *cam = nullptr, *cbm = nullptr;   // the separate transposes' masked coefficients
    float *lds = nullptr, *lold = nullptr;  // adjoint Debye state; each step's E_old term
    double *ga = nullptr, *gb = nullptr;
    double scale = 1.0;
    size_t wi = 0, wj = 0;
    cudaStream_t sw = nullptr;
    std::vector<cudaEvent_t> evs;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> t_rec, t_sw;   // per segment, for the parts' times
    std::chrono::steady_clock::time_point t0, b0;

    static double ms_since(std::chrono::steady_clock::time_point a) {
        return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - a).count();
    }

    ~FluxJob() {
        if (gpu) cudaSetDevice(gpu->device);
        if (sw) cudaStreamSynchronize(sw);
        if (s) cudaStreamSynchronize(s->stream);
        for (cudaEvent_t e : evs) cudaEventDestroy(e);
        if (sw) cudaStreamDestroy(sw);
        for (float* p : {lE[0], lE[1], lH[0], lH[1], lpsi[0], lpsi[1], dw, cam, cbm, lds, lold}) cudaFree(p);
        cudaFree(ga);
        cudaFree(gb);
        cudaFree(ck_mem);
        session_free(s);
    }

    int event(cudaEvent_t* e, bool timing) {
        FG_CUDA(cudaEventCreateWithFlags(e, timing ? cudaEventDefault : cudaEventDisableTiming));
        evs.push_back(*e);
        return FG_OK;
    }

    int set_base(long long b, bool counter = false, unsigned cnt = 0) {
        if (!s->hist_base && !counter) return FG_OK;
        k_adj_set<<<1, 1, 0, s->stream>>>(s->hist_base, b, s->counter, cnt, counter ? 1 : 0);
        FG_CUDA(cudaGetLastError());
        return FG_OK;
    }

    // checks, the session, the checkpoints and the adjoint buffers
    int prepare() {
        const auto p0 = std::chrono::steady_clock::now();
        const int rc = prepare_();
        res.setup_ms = ms_since(p0);
        return rc;
    }

    int prepare_() {
        if (!gpu) { err = "no GPU: this engine has no CPU path"; return FG_ERR_NO_DEVICE; }
        if (!sim->inductors.empty() || !sim->wires.empty() || !sim->sheets.empty()) {
            err = "the adjoint supports dielectric, conducting, Debye, PEC and port media only (no inductor, wire or sheet)";
            return FG_ERR_INVALID;
        }
        if (sp.steps == 0 || sp.freq <= 0.0) { err = "the adjoint needs steps > 0 and a frequency > 0"; return FG_ERR_INVALID; }
        for (int a = 0; a < 3; ++a)
            if (sp.lo[a] >= sp.hi[a] || sp.hi[a] > sim->n[a] - 1) { err = "empty or out-of-grid design box"; return FG_ERR_INVALID; }
        if (sp.plane_k >= sim->n[2]) { err = "plane_k is outside the grid"; return FG_ERR_INVALID; }
        for (int a = 0; a < 2; ++a)
            if (sp.win_lo[a] >= sp.win_hi[a] || sp.win_hi[a] > sim->n[a]) { err = "empty or out-of-grid flux window"; return FG_ERR_INVALID; }
        if (want_grad && !design_edges(*sim, sp, info, err)) return FG_ERR_INVALID;
        N = sp.steps;
        // segments of an even number of steps (the fused march alternates buffer sets)
        L = N;
        if (want_grad && sp.checkpoints > 0) {
            L = (N + sp.checkpoints - 1) / sp.checkpoints;
            L += L & 1;
        }
        S = (N + L - 1) / L;
        res.segments = S;
        res.segment_len = L;
        res.design_edges = info.size();
        sep = sp.transposes == 1;

        RunSpec rs;
        rs.driven = driven;
        rs.f0 = f0;
        rs.fc = fc;
        rs.max_steps = N;
        rs.freqs = {sp.freq};
        rs.has_plane_k = true;
        rs.plane_k = sp.plane_k;
        rs.fused = true;
        for (const auto& e : info) edges.push_back(e.at);
        rs.design = want_grad ? &edges : nullptr;
        rs.hist_cap = want_grad ? int(std::min<uint64_t>(S > 1 ? 2 * L : L, N)) : 0;   // checkpoints: a ring of two segments
        rs.design_in_steps = !(want_grad && S > 1);   // with checkpoints only the re-runs record
        int rc = session_new(gpu, *sim, rs, &s, err);
        if (rc) return rc;
        const Geom& g = s->geom;
        // checkpoints: E, H (buffer set 0 at even steps), every psi slab and the Debye state
        fbytes = size_t(3 * g.cs) * 4;
        pbytes = size_t(std::max<long long>(s->psi_total, 1)) * 4;
        nd_s = size_t(s->n_debye) * size_t(s->n_poles);
        dbytes = std::max<size_t>(nd_s, 1) * 4;
        ckpt = want_grad && S > 1;
        if (ckpt) {
            const size_t per = carve_size(fbytes) * 2 + carve_size(pbytes) + carve_size(dbytes);
            FG_CUDA(cudaMalloc(&ck_mem, per * S));
            for (uint64_t q = 0; q < S; ++q) {
                char* c = ck_mem + per * q;
                cks.push_back(Ck{reinterpret_cast<float*>(c), reinterpret_cast<float*>(c + carve_size(fbytes)),
                                 reinterpret_cast<float*>(c + 2 * carve_size(fbytes)),
                                 reinterpret_cast<float*>(c + 2 * carve_size(fbytes) + carve_size(pbytes))});
            }
        }
        if (!want_grad) return FG_OK;
        wi = sp.win_hi[0] - sp.win_lo[0];
        wj = sp.win_hi[1] - sp.win_lo[1];
        const int nd = int(edges.size());
        for (auto** p : {&lE[0], &lE[1], &lH[0]}) FG_CUDA(cudaMalloc(p, fbytes));
        if (sep) {
            for (auto** p : {&cam, &cbm}) FG_CUDA(cudaMalloc(p, fbytes));
        } else {
            FG_CUDA(cudaMalloc(&lH[1], fbytes));
        }
        for (auto** p : {&lpsi[0], &lpsi[1]}) FG_CUDA(cudaMalloc(p, pbytes));
        FG_CUDA(cudaMalloc(&lds, dbytes));
        FG_CUDA(cudaMalloc(&lold, std::max<size_t>(size_t(s->n_debye), 1) * 4));
        FG_CUDA(cudaMalloc(&dw, std::max<size_t>(wi * wj * 8, 1) * 4));
        FG_CUDA(cudaMalloc(&ga, size_t(std::max(nd, 1)) * 8));
        FG_CUDA(cudaMalloc(&gb, size_t(std::max(nd, 1)) * 8));
        // the sweep is the backward's critical path: its stream gets the highest priority, and the
        // re-runs fill the SMs it leaves idle
        int prio_lo = 0, prio_hi = 0;
        FG_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
        FG_CUDA(cudaStreamCreateWithPriority(&sw, cudaStreamNonBlocking, prio_hi));
        return FG_OK;
    }

    // The re-run of steps [a, b) for the design history, inside its dependency cone: one step moves
    // information one node along each axis (E^n+1 at p reads E^n and H^n-1/2 no further than one
    // node away), so of T steps the t-th marches only the nodes within T - 1 - t + 2 of the design
    // edges' nodes (the direct-load march over that box, no shell, no outputs) and the rest of the
    // grid is left stale. The recorded history equals that of the full step, bit for bit.
    int rerun_cone(uint64_t a, uint64_t b) {
        const uint64_t T = b - a;
        const int n[3] = {int(sim->n[0]), int(sim->n[1]), int(sim->n[2])};
        int base_lo[3], base_hi[3];   // nodes of the design edges and of the H they read, + 1
        for (int ax = 0; ax < 3; ++ax) {
            base_lo[ax] = std::max(0, int(sp.lo[ax]) - 2);
            base_hi[ax] = std::min(n[ax], int(sp.hi[ax]) + 3);
        }
        s->quiet = s->direct = s->boxed = true;
        int rc = FG_OK;
        for (uint64_t t = 0; t < T && !rc; ++t) {
            const int r = int(T - 1 - t);
            for (int ax = 0; ax < 3; ++ax) {
                s->box_lo[ax] = std::max(0, base_lo[ax] - r);
                s->box_hi[ax] = std::min(n[ax], base_hi[ax] + r);
            }
            rc = enqueue_step(*s, int((a + t) & 1), err);
            s->steps += 1;
        }
        s->quiet = s->direct = s->boxed = false;
        FG_CUDA(cudaGetLastError());
        return rc;
    }

    // the forward run, enqueued (checkpoints at the start of every segment)
    int forward() {
        FG_CUDA(cudaSetDevice(gpu->device));
        cudaStream_t st = s->stream;
        t0 = std::chrono::steady_clock::now();
        int rc = set_base(ckpt ? (1LL << 62) : 0);
        if (rc) return rc;
        if (!ckpt) return session_step(s, N, err);
        for (uint64_t q = 0; q < S; ++q) {
            const Ck& c = cks[q];
            FG_CUDA(cudaMemcpyAsync(c.e, s->e, fbytes, cudaMemcpyDeviceToDevice, st));
            FG_CUDA(cudaMemcpyAsync(c.h, s->h, fbytes, cudaMemcpyDeviceToDevice, st));
            FG_CUDA(cudaMemcpyAsync(c.psi, s->psi, pbytes, cudaMemcpyDeviceToDevice, st));
            if (nd_s) FG_CUDA(cudaMemcpyAsync(c.deb, s->debye_state, nd_s * 4, cudaMemcpyDeviceToDevice, st));
            if ((rc = session_step(s, std::min<uint64_t>(L, N - q * L), err))) return rc;
        }
        return FG_OK;
    }

    // waits for the forward; J from the plane DFT and, for the gradient, the adjoint sources
    int objective() {
        FG_CUDA(cudaSetDevice(gpu->device));
        int rc = session_sync(s, err);
        if (rc) return rc;
        res.forward_ms = ms_since(t0);
        std::vector<float> plane(s->plane_len);
        if ((rc = session_read(s, "plane", plane.data(), plane.size(), err))) return rc;
        using cd = std::complex<double>;
        const size_t n1 = sim->n[1];
        auto at = [&](size_t i, size_t j, int comp) {
            const size_t q = i * n1 + j;
            return cd(plane[q * 10 + 2 * comp], plane[q * 10 + 2 * comp + 1]);
        };
        cd F(0, 0);
        for (size_t i = sp.win_lo[0]; i < sp.win_hi[0]; ++i)
            for (size_t j = sp.win_lo[1]; j < sp.win_hi[1]; ++j) {
                const double dA = sim->ax[0].dd[i] * sim->ax[1].dd[j];
                F += dA * (at(i, j, 0) * std::conj(at(i, j, 4)) - at(i, j, 1) * std::conj(at(i, j, 3)));
            }
        res.J = std::norm(F);
        res.f_re = F.real();
        res.f_im = F.imag();
        if (!want_grad) return FG_OK;

        // adjoint sources: per window node the complex weights of dJ/dEx, dEy, dHx, dHy. The sweep
        // is linear: the weights are scaled so the injected values are O(1) in f32 (J is often far
        // below f32's range), and the gradient sums are divided back in f64.
        std::vector<double> wd(wi * wj * 8);
        std::vector<float> wts(wi * wj * 8);
        for (size_t a = 0; a < wi; ++a)
            for (size_t b = 0; b < wj; ++b) {
                const size_t i = sp.win_lo[0] + a, j = sp.win_lo[1] + b;
                const double dA = sim->ax[0].dd[i] * sim->ax[1].dd[j];
                const cd Fc = std::conj(F);
                const cd px = Fc * dA * std::conj(at(i, j, 4)), py = -Fc * dA * std::conj(at(i, j, 3));
                const cd qx = -Fc * dA * at(i, j, 1), qy = Fc * dA * at(i, j, 0);
                double* w = wd.data() + (a * wj + b) * 8;
                w[0] = px.real(); w[1] = px.imag();
                w[2] = py.real(); w[3] = py.imag();
                w[4] = qx.real(); w[5] = qx.imag();
                w[6] = qy.real(); w[7] = qy.imag();
            }
        double wmax = 0.0;
        for (double v : wd) wmax = std::max(wmax, std::fabs(v));
        scale = wmax > 0.0 ? 1.0 / (wmax * sim->dt) : 1.0;
        for (size_t q = 0; q < wd.size(); ++q) wts[q] = float(wd[q] * scale);
        // the weights go up before the call returns (wts is a host vector of this frame)
        FG_CUDA(cudaMemcpy(dw, wts.data(), wts.size() * 4, cudaMemcpyHostToDevice));
        return FG_OK;
    }

    // the backward sweep, enqueued segment by segment from the last. With checkpoints the history
    // is a ring of two segments: the re-run of segment q-1 (session stream) overlaps the sweep of
    // segment q (stream sw); it waits only for the sweep of q+1, whose half of the ring it overwrites.
    int backward() {
        FG_CUDA(cudaSetDevice(gpu->device));
        const Geom& g = s->geom;
        cudaStream_t st = s->stream;
        const int nd = int(edges.size());
        b0 = std::chrono::steady_clock::now();
        for (float* p : {lE[0], lE[1], lH[0], lH[1]})
            if (p) FG_CUDA(cudaMemsetAsync(p, 0, fbytes, st));
        for (float* p : {lpsi[0], lpsi[1]}) FG_CUDA(cudaMemsetAsync(p, 0, pbytes, st));
        FG_CUDA(cudaMemsetAsync(lds, 0, dbytes, st));
        FG_CUDA(cudaMemsetAsync(ga, 0, size_t(std::max(nd, 1)) * 8, st));
        FG_CUDA(cudaMemsetAsync(gb, 0, size_t(std::max(nd, 1)) * 8, st));
        if (sep) {
            const dim3 blk(64, 4, 1), grd((g.n2 + 63) / 64, (g.n1 + 3) / 4, g.n0);
            switch (s->cid_bytes) {
                case 1: k_adj_coefs<uint8_t><<<grd, blk, 0, st>>>(g, (const uint8_t*)s->node_class, s->classes, cam, cbm); break;
                case 2: k_adj_coefs<uint16_t><<<grd, blk, 0, st>>>(g, (const uint16_t*)s->node_class, s->classes, cam, cbm); break;
                default: k_adj_coefs<uint32_t><<<grd, blk, 0, st>>>(g, (const uint32_t*)s->node_class, s->classes, cam, cbm); break;
            }
        }
        const dim3 blk(64, 4, 1), grd((g.n2 + 63) / 64, (g.n1 + 3) / 4, g.n0);
        // the fused step: x-segments for about four waves of (32, 16) blocks on 148 SMs, 8 to 64 planes
        const long long adj_tiles = (long long)((g.n2 + ADJ_KOWN - 1) / ADJ_KOWN) * ((g.n1 + ADJ_TJ - 1) / ADJ_TJ);
        int adj_seg = 64;
        while (adj_seg > 8 && adj_tiles * ((g.n0 + adj_seg - 1) / adj_seg) < 148 * 4) adj_seg /= 2;
        const dim3 ablk(32, ADJ_ROWS, 1),
            agrd((g.n2 + ADJ_KOWN - 1) / ADJ_KOWN, (g.n1 + ADJ_TJ - 1) / ADJ_TJ, (g.n0 + adj_seg - 1) / adj_seg);
        const unsigned wblocks = unsigned((wi * wj + 127) / 128), dblocks = unsigned((nd + 127) / 128);
        // the source and the gradient share a launch unless a design edge is a window node
        bool apart = sep;
        for (const int4& e : edges)
            apart = apart || (e.x < 2 && uint64_t(e.w) == sp.plane_k && uint64_t(e.y) >= sp.win_lo[0] &&
                              uint64_t(e.y) < sp.win_hi[0] && uint64_t(e.z) >= sp.win_lo[1] && uint64_t(e.z) < sp.win_hi[1]);
        int rc;
        cudaEvent_t rec_done, swept[2];
        if ((rc = event(&rec_done, false)) || (rc = event(&swept[0], false)) || (rc = event(&swept[1], false))) return rc;
        auto recompute = [&](uint64_t q) -> int {
            const uint64_t a = q * L, b = std::min<uint64_t>(N, a + L);
            cudaEvent_t e0, e1;
            int r = event(&e0, true);
            if (!r) r = event(&e1, true);
            if (r) return r;
            FG_CUDA(cudaEventRecord(e0, st));
            FG_CUDA(cudaMemcpyAsync(s->e, cks[q].e, fbytes, cudaMemcpyDeviceToDevice, st));
            FG_CUDA(cudaMemcpyAsync(s->h, cks[q].h, fbytes, cudaMemcpyDeviceToDevice, st));
            FG_CUDA(cudaMemcpyAsync(s->psi, cks[q].psi, pbytes, cudaMemcpyDeviceToDevice, st));
            if (nd_s) FG_CUDA(cudaMemcpyAsync(s->debye_state, cks[q].deb, nd_s * 4, cudaMemcpyDeviceToDevice, st));
            s->steps = a;
            // the step counter at a, the history slots of ring half q & 1
            if ((r = set_base((long long)(a - (q & 1) * L), true, unsigned(a)))) return r;
            if ((r = rerun_cone(a, b))) return r;
            FG_CUDA(cudaEventRecord(e1, st));
            FG_CUDA(cudaEventRecord(rec_done, st));
            t_rec.push_back({e0, e1});
            return FG_OK;
        };
        // the sweep stream starts after the adjoint buffers are cleared (on st)
        cudaEvent_t ready;
        if ((rc = event(&ready, false))) return rc;
        FG_CUDA(cudaEventRecord(ready, st));
        FG_CUDA(cudaStreamWaitEvent(sw, ready, 0));
        int set = 0;
        if (ckpt && (rc = recompute(S - 1))) return rc;
        for (uint64_t q = S; q-- > 0;) {
            const uint64_t a = q * L, b = std::min<uint64_t>(N, a + L);
            const long long half = ckpt ? (long long)((q & 1) * L) : 0;
            cudaEvent_t e0, e1;
            if ((rc = event(&e0, true)) || (rc = event(&e1, true))) return rc;
            if (ckpt) FG_CUDA(cudaStreamWaitEvent(sw, rec_done, 0));
            FG_CUDA(cudaEventRecord(e0, sw));
            for (uint64_t n = b; n-- > a;) {
                float* lh = sep ? lH[0] : lH[set];
                if (apart) {
                    k_adj_inject<<<wblocks, 128, 0, sw>>>(g, int(sp.plane_k), int(sp.win_lo[0]), int(wi), int(sp.win_lo[1]),
                                                          int(wj), dw, s->sc.dft, 1, (long long)n, lE[set], lh);
                    if (nd) k_adj_grad<<<dblocks, 128, 0, sw>>>(g, s->design, nd, lE[set], s->hist_e, s->hist_s,
                                                                 (long long)(n - a) + half, ga, gb);
                } else {
                    k_adj_source_grad<<<wblocks + dblocks, 128, 0, sw>>>(
                        g, int(sp.plane_k), int(sp.win_lo[0]), int(wi), int(sp.win_lo[1]), int(wj), dw, s->sc.dft, 1,
                        (long long)n, lE[set], lh, wblocks, s->design, nd, s->hist_e, s->hist_s,
                        (long long)(n - a) + half, ga, gb);
                }
                if (s->n_debye) {
                    const unsigned qb = unsigned((s->n_debye + 255) / 256);
                    switch (s->cid_bytes) {
                        case 1: k_adj_debye_pre<uint8_t><<<qb, 256, 0, sw>>>(s->debye_f, s->debye_dd, s->n_debye, (const uint8_t*)s->node_class, s->classes, g.cs, s->debye_table, lds, lE[set], lold); break;
                        case 2: k_adj_debye_pre<uint16_t><<<qb, 256, 0, sw>>>(s->debye_f, s->debye_dd, s->n_debye, (const uint16_t*)s->node_class, s->classes, g.cs, s->debye_table, lds, lE[set], lold); break;
                        default: k_adj_debye_pre<uint32_t><<<qb, 256, 0, sw>>>(s->debye_f, s->debye_dd, s->n_debye, (const uint32_t*)s->node_class, s->classes, g.cs, s->debye_table, lds, lE[set], lold); break;
                    }
                }
                if (sep) {
                    k_adj_e<<<grd, blk, 0, sw>>>(g, cam, cbm, lE[set], lE[1 - set], lpsi[set], lpsi[1 - set], lh);
                    k_adj_h<<<grd, blk, 0, sw>>>(g, lh, lpsi[set], lpsi[1 - set], lE[1 - set], s->sc.k_mu);
                } else {
                    const AdjArgs aa{g, s->node_class, s->classes, lE[set], lE[1 - set], lH[set], lH[1 - set],
                                     lpsi[set], lpsi[1 - set], s->sc.k_mu};
                    switch (s->cid_bytes) {
                        case 1: k_adj_step<uint8_t><<<agrd, ablk, 0, sw>>>(aa, adj_seg); break;
                        case 2: k_adj_step<uint16_t><<<agrd, ablk, 0, sw>>>(aa, adj_seg); break;
                        default: k_adj_step<uint32_t><<<agrd, ablk, 0, sw>>>(aa, adj_seg); break;
                    }
                }
                if (s->n_debye)
                    k_adj_debye_post<<<unsigned((s->n_debye + 255) / 256), 256, 0, sw>>>(s->debye_f, s->n_debye, lold,
                                                                                         lE[1 - set]);
                set = 1 - set;
            }
            FG_CUDA(cudaGetLastError());
            FG_CUDA(cudaEventRecord(e1, sw));
            FG_CUDA(cudaEventRecord(swept[q & 1], sw));
            t_sw.push_back({e0, e1});
            if (ckpt && q > 0) {
                // segment q-1 goes to ring half (q-1) & 1, which the sweep of q+1 read
                if (q + 1 < S) FG_CUDA(cudaStreamWaitEvent(st, swept[(q + 1) & 1], 0));
                if ((rc = recompute(q - 1))) return rc;
            }
        }
        return FG_OK;
    }

    // waits for the backward; the parts' times and the chain rule to the design voxels
    int finish() {
        FG_CUDA(cudaSetDevice(gpu->device));
        FG_CUDA(cudaStreamSynchronize(sw));
        FG_CUDA(cudaStreamSynchronize(s->stream));
        res.backward_ms = ms_since(b0);
        for (auto& pr : t_rec) { float x = 0; FG_CUDA(cudaEventElapsedTime(&x, pr.first, pr.second)); res.recompute_ms += x; }
        for (auto& pr : t_sw) { float x = 0; FG_CUDA(cudaEventElapsedTime(&x, pr.first, pr.second)); res.adjoint_ms += x; }
        const int nd = int(edges.size());
        std::vector<double> hga, hgb;
        hga.resize(size_t(nd));
        hgb.resize(size_t(nd));
        if (nd) {
            FG_CUDA(cudaMemcpy(hga.data(), ga, size_t(nd) * 8, cudaMemcpyDeviceToHost));
            FG_CUDA(cudaMemcpy(hgb.data(), gb, size_t(nd) * 8, cudaMemcpyDeviceToHost));
        }
        const size_t ncell = (sp.hi[0] - sp.lo[0]) * (sp.hi[1] - sp.lo[1]) * (sp.hi[2] - sp.lo[2]);
        res.g_eps.assign(ncell, 0.0);
        res.g_sig.assign(ncell, 0.0);
        for (int t = 0; t < nd; ++t) {
            const DesignEdgeInfo& e = info[size_t(t)];
            const double ga_t = hga[size_t(t)] / scale, gb_t = hgb[size_t(t)] / scale;   // dJ/dca, dJ/dcb
            const double de = ga_t * e.dca_de + gb_t * e.dcb_de;   // dJ / d eps_edge (F/m)
            const double ds = ga_t * e.dca_ds + gb_t * e.dcb_ds;   // dJ / d sigma_edge
            for (int q = 0; q < 4; ++q) {
                if (e.cell[q] == SIZE_MAX) continue;
                res.g_eps[e.cell[q]] += de * EPS0 * e.w[q];
                res.g_sig[e.cell[q]] += ds * e.w[q];
            }
        }
        return FG_OK;
    }
};

int flux_gradient(Gpu* gpu, const HostSim& sim, uint64_t driven, double f0, double fc, const FluxSpec& sp,
                  bool want_grad, FluxResult& res, std::string& err) {
    FluxJob j;
    j.gpu = gpu;
    j.sim = &sim;
    j.driven = driven;
    j.f0 = f0;
    j.fc = fc;
    j.sp = sp;
    j.want_grad = want_grad;
    int rc = j.prepare();
    if (!rc) rc = j.forward();
    if (!rc) rc = j.objective();
    if (!rc && want_grad) rc = j.backward();
    if (!rc && want_grad) rc = j.finish();
    if (rc) { err = j.err; return rc; }
    res = std::move(j.res);
    return FG_OK;
}

// Many flux gradients on one GPU, in groups of up to `group` jobs: a group's jobs are prepared
// and their forwards enqueued together; each objective is formed as its forward ends; the
// backwards are enqueued together, and while they run the next group is prepared and its
// forwards enqueued, before the group is finished in turn. A group also stops growing when the
// device's free memory would not hold the next job (estimated from the bytes per node the jobs
// prepared so far took, with half again to spare) or when preparing a job runs out of device
// memory beside jobs in flight (a job's checkpoints and design history grow with its steps and
// design, not with its nodes): its jobs then wait for a later group, and a group that cannot open
// beside the running one opens after it. Each job's results are those of
// running it alone. The first error stops the batch (its message names the job).
int flux_gradient_batch(Gpu* gpu, const std::vector<const HostSim*>& sims, const std::vector<uint64_t>& driven,
                        const std::vector<std::pair<double, double>>& pulses, const std::vector<FluxSpec>& specs,
                        int group, std::vector<FluxResult>& out, std::string& err) {
    const size_t count = sims.size();
    out.assign(count, FluxResult{});
    if (group <= 0) group = 16;
    FG_CUDA(cudaSetDevice(gpu->device));
    using Group = std::vector<std::unique_ptr<FluxJob>>;
    int rc = FG_OK;
    size_t bad = 0;
    std::string bad_err;
    double per_node = 0.0;   // device bytes per node a prepared job took, at most
    auto fail = [&](size_t q, const FluxJob& j) {
        bad = q;
        bad_err = j.err;
    };
    auto free_bytes = [] {
        size_t f = 0, t = 0;
        return cudaMemGetInfo(&f, &t) == cudaSuccess ? double(f) : 0.0;
    };
    // prepare jobs from g0 while they fit (and, with `holding`, the first one only if it fits
    // beside the running group) and enqueue their forwards; returns the first job left out
    auto open = [&](size_t g0, Group& G, bool holding) -> size_t {
        size_t q = g0;
        for (; q < count && q < g0 + size_t(group) && !rc; ++q) {
            const double need = 1.5 * per_node * double(sims[q]->nn);
            const double before = free_bytes();
            if ((!G.empty() || holding) && per_node > 0.0 && before < need) break;
            auto j = std::make_unique<FluxJob>();
            j->gpu = gpu;
            j->sim = sims[q];
            j->driven = driven[q];
            j->f0 = pulses[q].first;
            j->fc = pulses[q].second;
            j->sp = specs[q];
            j->want_grad = true;
            if ((rc = j->prepare())) {
                // out of device memory beside jobs already in flight: this job waits for a later
                // group (its partial buffers go with it); alone, the error stands
                const bool oom = rc == FG_ERR_TOO_LARGE ||
                                 (rc == FG_ERR_CUDA && j->err.find("out of memory") != std::string::npos);
                if (oom && (!G.empty() || holding)) {
                    j.reset();
                    cudaGetLastError();
                    rc = FG_OK;
                    break;
                }
                fail(q, *j);
            }
            const double after = free_bytes();
            if (before > after) per_node = std::max(per_node, (before - after) / double(sims[q]->nn));
            G.push_back(std::move(j));
        }
        for (size_t t = 0; t < G.size() && !rc; ++t)
            if ((rc = G[t]->forward())) fail(g0 + t, *G[t]);
        return q;
    };
    Group cur, next;
    size_t g0 = 0, g1 = open(0, cur, false);
    while (!rc && g0 < count) {
        for (size_t q = 0; q < cur.size() && !rc; ++q)
            if ((rc = cur[q]->objective())) fail(g0 + q, *cur[q]);
        for (size_t q = 0; q < cur.size() && !rc; ++q)
            if ((rc = cur[q]->backward())) fail(g0 + q, *cur[q]);
        size_t g2 = g1;
        if (!rc && g1 < count) g2 = open(g1, next, true);
        for (size_t q = 0; q < cur.size() && !rc; ++q)
            if ((rc = cur[q]->finish())) fail(g0 + q, *cur[q]);
        if (rc) break;
        for (size_t q = 0; q < cur.size(); ++q) out[g0 + q] = std::move(cur[q]->res);
        cur.clear();   // the group's memory goes back before a deferred group opens
        if (next.empty() && g1 < count) g2 = open(g1, next, false);
        cur = std::move(next);
        next.clear();
        g0 = g1;
        g1 = g2;
    }
    if (rc) {
        err = "job " + std::to_string(bad) + ": " + bad_err;
        return rc;
    }
    return FG_OK;
}

}  // namespace fg
