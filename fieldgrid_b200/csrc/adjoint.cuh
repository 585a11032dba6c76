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
// when checkpoints ~ sqrt(N).
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

int flux_gradient(Gpu* gpu, const HostSim& sim, uint64_t driven, double f0, double fc, const FluxSpec& sp,
                  bool want_grad, FluxResult& res, std::string& err) {
    if (!gpu) { err = "no GPU: this engine has no CPU path"; return FG_ERR_NO_DEVICE; }
    if (!sim.inductors.empty() || !sim.wires.empty() || !sim.sheets.empty()) {
        err = "the adjoint supports dielectric, conducting, Debye, PEC and port media only (no inductor, wire or sheet)";
        return FG_ERR_INVALID;
    }
    if (sp.steps == 0 || sp.freq <= 0.0) { err = "the adjoint needs steps > 0 and a frequency > 0"; return FG_ERR_INVALID; }
    for (int a = 0; a < 3; ++a)
        if (sp.lo[a] >= sp.hi[a] || sp.hi[a] > sim.n[a] - 1) { err = "empty or out-of-grid design box"; return FG_ERR_INVALID; }
    if (sp.plane_k >= sim.n[2]) { err = "plane_k is outside the grid"; return FG_ERR_INVALID; }
    for (int a = 0; a < 2; ++a)
        if (sp.win_lo[a] >= sp.win_hi[a] || sp.win_hi[a] > sim.n[a]) { err = "empty or out-of-grid flux window"; return FG_ERR_INVALID; }
    std::vector<DesignEdgeInfo> info;
    if (want_grad && !design_edges(sim, sp, info, err)) return FG_ERR_INVALID;
    const uint64_t N = sp.steps;
    // segments of an even number of steps (the fused march alternates buffer sets)
    uint64_t L = N;
    if (want_grad && sp.checkpoints > 0) {
        L = (N + sp.checkpoints - 1) / sp.checkpoints;
        L += L & 1;
    }
    const uint64_t S = (N + L - 1) / L;
    res.segments = S;
    res.segment_len = L;
    res.design_edges = info.size();

    RunSpec rs;
    rs.driven = driven;
    rs.f0 = f0;
    rs.fc = fc;
    rs.max_steps = N;
    rs.freqs = {sp.freq};
    rs.has_plane_k = true;
    rs.plane_k = sp.plane_k;
    rs.fused = true;
    std::vector<int4> edges;
    for (const auto& e : info) edges.push_back(e.at);
    rs.design = want_grad ? &edges : nullptr;
    rs.hist_cap = want_grad ? int(std::min<uint64_t>(S > 1 ? 2 * L : L, N)) : 0;   // checkpoints: a ring of two segments
    Session* s = nullptr;
    int rc = session_new(gpu, sim, rs, &s, err);
    if (rc) return rc;
    std::unique_ptr<Session, void (*)(Session*)> guard(s, session_free);
    const Geom& g = s->geom;
    cudaStream_t st = s->stream;
    auto set_base = [&](long long b) -> int {
        if (!s->hist_base) return FG_OK;
        FG_CUDA(cudaMemcpyAsync(s->hist_base, &b, sizeof(b), cudaMemcpyHostToDevice, st));
        return FG_OK;
    };
    auto now = [] { return std::chrono::steady_clock::now(); };
    auto ms = [](auto a, auto b) { return std::chrono::duration<double, std::milli>(b - a).count(); };

    // checkpoints: E, H (buffer set 0 at even steps), every psi slab and the Debye state
    const size_t fbytes = size_t(3 * g.cs) * 4, pbytes = size_t(std::max<long long>(s->psi_total, 1)) * 4;
    const size_t nd_s = size_t(s->n_debye) * size_t(s->n_poles);   // Debye state entries
    const size_t dbytes = std::max<size_t>(nd_s, 1) * 4;
    struct Ck { float *e = nullptr, *h = nullptr, *psi = nullptr, *deb = nullptr; };
    std::vector<Ck> cks;
    char* ck_mem = nullptr;   // all checkpoints in one allocation
    std::unique_ptr<void, std::function<void(void*)>> ck_guard((void*)1, [&](void*) { cudaFree(ck_mem); });
    const bool ckpt = want_grad && S > 1;
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

    // 1. forward
    auto t0 = now();
    if (rc = set_base(ckpt ? (1LL << 62) : 0); rc) return rc;
    if (!ckpt) {
        if ((rc = session_step(s, N, err))) return rc;
    } else {
        for (uint64_t q = 0; q < S; ++q) {
            const Ck& c = cks[q];
            FG_CUDA(cudaMemcpyAsync(c.e, s->e, fbytes, cudaMemcpyDeviceToDevice, st));
            FG_CUDA(cudaMemcpyAsync(c.h, s->h, fbytes, cudaMemcpyDeviceToDevice, st));
            FG_CUDA(cudaMemcpyAsync(c.psi, s->psi, pbytes, cudaMemcpyDeviceToDevice, st));
            if (nd_s) FG_CUDA(cudaMemcpyAsync(c.deb, s->debye_state, nd_s * 4, cudaMemcpyDeviceToDevice, st));
            if ((rc = session_step(s, std::min<uint64_t>(L, N - q * L), err))) return rc;
        }
    }
    if ((rc = session_sync(s, err))) return rc;
    res.forward_ms = ms(t0, now());

    // 2. the objective from the plane DFT
    std::vector<float> plane(s->plane_len);
    if ((rc = session_read(s, "plane", plane.data(), plane.size(), err))) return rc;
    using cd = std::complex<double>;
    const size_t n1 = sim.n[1];
    auto at = [&](size_t i, size_t j, int comp) {
        const size_t q = i * n1 + j;
        return cd(plane[q * 10 + 2 * comp], plane[q * 10 + 2 * comp + 1]);
    };
    const size_t wi = sp.win_hi[0] - sp.win_lo[0], wj = sp.win_hi[1] - sp.win_lo[1];
    cd F(0, 0);
    for (size_t i = sp.win_lo[0]; i < sp.win_hi[0]; ++i)
        for (size_t j = sp.win_lo[1]; j < sp.win_hi[1]; ++j) {
            const double dA = sim.ax[0].dd[i] * sim.ax[1].dd[j];
            F += dA * (at(i, j, 0) * std::conj(at(i, j, 4)) - at(i, j, 1) * std::conj(at(i, j, 3)));
        }
    res.J = std::norm(F);
    res.f_re = F.real();
    res.f_im = F.imag();
    if (!want_grad) return FG_OK;

    // 3. adjoint sources: per window node the complex weights of dJ/dEx, dEy, dHx, dHy
    // The sweep is linear: the weights are scaled so the injected values are O(1) in f32 (J is
    // often far below f32's range), and the gradient sums are divided back in f64.
    std::vector<double> wd(wi * wj * 8);
    std::vector<float> wts(wi * wj * 8);
    for (size_t a = 0; a < wi; ++a)
        for (size_t b = 0; b < wj; ++b) {
            const size_t i = sp.win_lo[0] + a, j = sp.win_lo[1] + b;
            const double dA = sim.ax[0].dd[i] * sim.ax[1].dd[j];
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
    const double scale = wmax > 0.0 ? 1.0 / (wmax * sim.dt) : 1.0;
    for (size_t q = 0; q < wd.size(); ++q) wts[q] = float(wd[q] * scale);
    // adjoint state and gradient accumulators
    const int nd = int(edges.size());
    float *lE[2] = {nullptr, nullptr}, *lH[2] = {nullptr, nullptr}, *lpsi[2] = {nullptr, nullptr}, *dw = nullptr;
    float *cam = nullptr, *cbm = nullptr;   // the separate transposes' masked coefficients
    float *lds = nullptr, *lold = nullptr;  // adjoint Debye state; each step's E_old term
    double *ga = nullptr, *gb = nullptr;
    auto free_adj = [&] {
        cudaFree(lE[0]); cudaFree(lE[1]); cudaFree(lH[0]); cudaFree(lH[1]); cudaFree(lpsi[0]); cudaFree(lpsi[1]);
        cudaFree(dw); cudaFree(ga); cudaFree(gb); cudaFree(cam); cudaFree(cbm); cudaFree(lds); cudaFree(lold);
    };
    std::unique_ptr<void, std::function<void(void*)>> adj_guard((void*)1, [&](void*) { free_adj(); });
    const bool sep = sp.transposes == 1;
    for (auto** p : {&lE[0], &lE[1], &lH[0]}) FG_CUDA(cudaMalloc(p, fbytes));
    if (sep) {
        for (auto** p : {&cam, &cbm}) FG_CUDA(cudaMalloc(p, fbytes));
    } else {
        FG_CUDA(cudaMalloc(&lH[1], fbytes));
    }
    for (auto** p : {&lpsi[0], &lpsi[1]}) FG_CUDA(cudaMalloc(p, pbytes));
    FG_CUDA(cudaMalloc(&lds, dbytes));
    FG_CUDA(cudaMalloc(&lold, std::max<size_t>(size_t(s->n_debye), 1) * 4));
    FG_CUDA(cudaMemsetAsync(lds, 0, dbytes, st));
    FG_CUDA(cudaMalloc(&dw, wts.size() * 4));
    FG_CUDA(cudaMalloc(&ga, size_t(std::max(nd, 1)) * 8));
    FG_CUDA(cudaMalloc(&gb, size_t(std::max(nd, 1)) * 8));
    for (float* p : {lE[0], lE[1], lH[0], lH[1]})
        if (p) FG_CUDA(cudaMemsetAsync(p, 0, fbytes, st));
    for (float* p : {lpsi[0], lpsi[1]}) FG_CUDA(cudaMemsetAsync(p, 0, pbytes, st));
    FG_CUDA(cudaMemsetAsync(ga, 0, size_t(std::max(nd, 1)) * 8, st));
    FG_CUDA(cudaMemsetAsync(gb, 0, size_t(std::max(nd, 1)) * 8, st));
    FG_CUDA(cudaMemcpyAsync(dw, wts.data(), wts.size() * 4, cudaMemcpyHostToDevice, st));
    if (sep) {
        const dim3 blk(64, 4, 1), grd((g.n2 + 63) / 64, (g.n1 + 3) / 4, g.n0);
        switch (s->cid_bytes) {
            case 1: k_adj_coefs<uint8_t><<<grd, blk, 0, st>>>(g, (const uint8_t*)s->node_class, s->classes, cam, cbm); break;
            case 2: k_adj_coefs<uint16_t><<<grd, blk, 0, st>>>(g, (const uint16_t*)s->node_class, s->classes, cam, cbm); break;
            default: k_adj_coefs<uint32_t><<<grd, blk, 0, st>>>(g, (const uint32_t*)s->node_class, s->classes, cam, cbm); break;
        }
    }

    // 4. backward sweep, segment by segment from the last. With checkpoints the history is a ring of
    // two segments: the re-run of segment q-1 (session stream) overlaps the sweep of segment q (a
    // second stream); it waits only for the sweep of q+1, whose half of the ring it overwrites.
    const dim3 blk(64, 4, 1), grd((g.n2 + 63) / 64, (g.n1 + 3) / 4, g.n0);
    // the fused step: x-segments for about four waves of (32, 16) blocks on 148 SMs, 8 to 64 planes
    const long long adj_tiles = (long long)((g.n2 + ADJ_KOWN - 1) / ADJ_KOWN) * ((g.n1 + ADJ_TJ - 1) / ADJ_TJ);
    int adj_seg = 64;
    while (adj_seg > 8 && adj_tiles * ((g.n0 + adj_seg - 1) / adj_seg) < 148 * 4) adj_seg /= 2;
    const dim3 ablk(32, ADJ_ROWS, 1),
        agrd((g.n2 + ADJ_KOWN - 1) / ADJ_KOWN, (g.n1 + ADJ_TJ - 1) / ADJ_TJ, (g.n0 + adj_seg - 1) / adj_seg);
    const unsigned wblocks = unsigned((wi * wj + 127) / 128), dblocks = unsigned((nd + 127) / 128);
    cudaStream_t sw = nullptr;
    std::vector<cudaEvent_t> evs;
    std::unique_ptr<void, std::function<void(void*)>> sw_guard((void*)1, [&](void*) {
        for (cudaEvent_t e : evs) cudaEventDestroy(e);
        if (sw) cudaStreamDestroy(sw);
    });
    // the sweep is the backward's critical path: its stream gets the highest priority, and the
    // re-runs fill the SMs it leaves idle
    int prio_lo = 0, prio_hi = 0;
    FG_CUDA(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    FG_CUDA(cudaStreamCreateWithPriority(&sw, cudaStreamNonBlocking, prio_hi));
    auto event = [&](cudaEvent_t* e, bool timing) -> int {
        FG_CUDA(cudaEventCreateWithFlags(e, timing ? cudaEventDefault : cudaEventDisableTiming));
        evs.push_back(*e);
        return FG_OK;
    };
    cudaEvent_t rec_done, swept[2];
    if ((rc = event(&rec_done, false)) || (rc = event(&swept[0], false)) || (rc = event(&swept[1], false))) return rc;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> t_rec, t_sw;   // per segment, for the parts' times
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
        const unsigned cnt = unsigned(a);
        FG_CUDA(cudaMemcpyAsync(s->counter, &cnt, sizeof(cnt), cudaMemcpyHostToDevice, st));
        s->steps = a;
        if ((r = set_base((long long)(a - (q & 1) * L)))) return r;   // slots of ring half q & 1
        if ((r = session_rerun(s, b - a, err))) return r;
        FG_CUDA(cudaEventRecord(e1, st));
        FG_CUDA(cudaEventRecord(rec_done, st));
        t_rec.push_back({e0, e1});
        return FG_OK;
    };
    // the sweep stream starts after the adjoint buffers are cleared and the weights uploaded (on st)
    cudaEvent_t ready;
    if ((rc = event(&ready, false))) return rc;
    FG_CUDA(cudaEventRecord(ready, st));
    FG_CUDA(cudaStreamWaitEvent(sw, ready, 0));
    auto b0 = now();
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
            k_adj_inject<<<wblocks, 128, 0, sw>>>(g, int(sp.plane_k), int(sp.win_lo[0]), int(wi), int(sp.win_lo[1]),
                                                  int(wj), dw, s->sc.dft, 1, (long long)n, lE[set], lh);
            if (nd) k_adj_grad<<<dblocks, 128, 0, sw>>>(g, s->design, nd, lE[set], s->hist_e, s->hist_s,
                                                         (long long)(n - a) + half, ga, gb);
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
    FG_CUDA(cudaStreamSynchronize(sw));
    FG_CUDA(cudaStreamSynchronize(st));
    res.backward_ms = ms(b0, now());
    for (auto& pr : t_rec) { float x = 0; FG_CUDA(cudaEventElapsedTime(&x, pr.first, pr.second)); res.recompute_ms += x; }
    for (auto& pr : t_sw) { float x = 0; FG_CUDA(cudaEventElapsedTime(&x, pr.first, pr.second)); res.adjoint_ms += x; }

    // 5. chain rule to the design voxels
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

}  // namespace fg
