// The flux objective from an FP64 forward on the device: the reference's update (sims-field
// cpu.rs:48-167) with fields, psi, coefficients, the source pulse and the DFT phases in double,
// for checking gradients against central differences at full size. Dielectric and conducting
// edges take their (ca, cb) from the cell materials in f64 (sim.rs:375-441, before the rounding
// to f32); edges whose coefficients setup overrode (PEC, lumped elements, ports) keep their f32
// values, widened, as do the port's source coefficients. The layout is the reference's own
// (node (i*n1 + j)*n2 + k, component-major; psi_idx of sim.rs:659-665), the step the separate one
// (H in place, E in place, the driven port's source, the plane DFT). Debye media, inductors, thin
// wires and resistive sheets are refused, as in the adjoint.
//
// Included at the end of engine.cu.
#pragma once

namespace fg {

struct Geom64 {
    int n0, n1, n2, pml;
    long long nn;
    const AxisNode64* ax[3];
    long long psi_off[18];
};

__device__ __forceinline__ long long psi_at64(const Geom64& g, int a, int i, int j, int k, int s) {
    const long long w = 2 * g.pml;
    if (a == 0) return ((long long)s * g.n1 + j) * g.n2 + k;
    if (a == 1) return ((long long)i * w + s) * g.n2 + k;
    return ((long long)i * g.n1 + j) * w + s;
}

__global__ void __launch_bounds__(256) k_h64(Geom64 g, const double* __restrict__ e, double* __restrict__ h,
                                             double* __restrict__ psi, double k_mu) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, i = blockIdx.z;
    if (k >= g.n2 || j >= g.n1) return;
    const int p[3] = {i, j, k}, n[3] = {g.n0, g.n1, g.n2};
    const long long st[3] = {(long long)g.n1 * g.n2, g.n2, 1};
    const long long id = ((long long)i * g.n1 + j) * g.n2 + k;
#pragma unroll
    for (int C = 0; C < 3; ++C) {
        const int U = (C + 1) % 3, V = (C + 2) % 3;
        if (p[U] + 1 >= n[U] || p[V] + 1 >= n[V]) continue;
        const double ev = e[V * g.nn + id + st[U]] - e[V * g.nn + id];
        const double eu = e[U * g.nn + id + st[V]] - e[U * g.nn + id];
        const AxisNode64& au = g.ax[U][p[U]];
        const AxisNode64& av = g.ax[V][p[V]];
        double t1 = ev * au.inv_d, t2 = eu * av.inv_d;
        if (au.slot_h >= 0) {
            const long long q = g.psi_off[9 + C * 3 + U] + psi_at64(g, U, i, j, k, au.slot_h);
            const double r = au.bh * psi[q] + au.ch * ev * au.raw_inv_d;
            psi[q] = r;
            t1 += r;
        }
        if (av.slot_h >= 0) {
            const long long q = g.psi_off[9 + C * 3 + V] + psi_at64(g, V, i, j, k, av.slot_h);
            const double r = av.bh * psi[q] + av.ch * eu * av.raw_inv_d;
            psi[q] = r;
            t2 += r;
        }
        h[C * g.nn + id] -= k_mu * (t1 - t2);
    }
}

__global__ void __launch_bounds__(256) k_e64(Geom64 g, const double* __restrict__ ca, const double* __restrict__ cb,
                                             const double* __restrict__ h, double* __restrict__ e,
                                             double* __restrict__ psi) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y, i = blockIdx.z;
    if (k >= g.n2 || j >= g.n1) return;
    const int p[3] = {i, j, k};
    const long long st[3] = {(long long)g.n1 * g.n2, g.n2, 1};
    const long long id = ((long long)i * g.n1 + j) * g.n2 + k;
#pragma unroll
    for (int C = 0; C < 3; ++C) {
        const int U = (C + 1) % 3, V = (C + 2) % 3;
        const double b = cb[C * g.nn + id];
        if (b == 0.0 || p[U] == 0 || p[V] == 0) continue;
        const double hv = h[V * g.nn + id] - h[V * g.nn + id - st[U]];
        const double hu = h[U * g.nn + id] - h[U * g.nn + id - st[V]];
        const AxisNode64& au = g.ax[U][p[U]];
        const AxisNode64& av = g.ax[V][p[V]];
        double t1 = hv * au.inv_dd, t2 = hu * av.inv_dd;
        if (au.slot_e >= 0) {
            const long long q = g.psi_off[C * 3 + U] + psi_at64(g, U, i, j, k, au.slot_e);
            const double r = au.be * psi[q] + au.ce * hv * au.raw_inv_dd;
            psi[q] = r;
            t1 += r;
        }
        if (av.slot_e >= 0) {
            const long long q = g.psi_off[C * 3 + V] + psi_at64(g, V, i, j, k, av.slot_e);
            const double r = av.be * psi[q] + av.ce * hu * av.raw_inv_dd;
            psi[q] = r;
            t2 += r;
        }
        double& f = e[C * g.nn + id];
        f = ca[C * g.nn + id] * f + b * (t1 - t2);
    }
}

// the driven port's source at t = (n + 1/2) dt (cpu.rs:291-297)
__global__ void k_src64(const long long* __restrict__ f, const double* __restrict__ src, int ns, double pulse,
                        double* __restrict__ e) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < ns) e[f[q]] -= src[q] * pulse;
}

// the running DFT of Ex, Ey, Ez (with ce = dt (cos, -sin) of w te) and Hx, Hy (ch, of w th) on plane k
__global__ void k_dft64(Geom64 g, int plane_k, double ce0, double ce1, double ch0, double ch1,
                        const double* __restrict__ e, const double* __restrict__ h, double* __restrict__ acc) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)g.n0 * g.n1) return;
    const long long id = q * g.n2 + plane_k;
    const double f[5] = {e[id], e[g.nn + id], e[2 * g.nn + id], h[id], h[g.nn + id]};
    double* o = acc + q * 10;
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        const double a = c < 3 ? ce0 : ch0, b = c < 3 ? ce1 : ch1;
        o[2 * c] += f[c] * a;
        o[2 * c + 1] += f[c] * b;
    }
}

// (ca, cb) of edge c at node (i, j, k) from the cell materials in f64; false off the interior
bool plain_coef64(const HostSim& sim, uint32_t c, size_t i, size_t j, size_t k, double& ca, double& cb) {
    const size_t* n = sim.n;
    const size_t p[3] = {i, j, k};
    const uint32_t u = (c + 1) % 3, v = (c + 2) % 3;
    if (p[c] + 1 >= n[c] || p[u] == 0 || p[u] + 1 >= n[u] || p[v] == 0 || p[v] + 1 >= n[v]) return false;
    static const int offs[4][2] = {{-1, -1}, {0, -1}, {-1, 0}, {0, 0}};
    double se = 0, ss = 0, ws = 0;
    for (const auto& o : offs) {
        size_t cc[3] = {i, j, k};
        cc[u] = size_t(long(p[u]) + o[0]);
        cc[v] = size_t(long(p[v]) + o[1]);
        const double w = sim.ax[u].d[cc[u]] * sim.ax[v].d[cc[v]];
        const size_t id = (cc[0] * (n[1] - 1) + cc[1]) * (n[2] - 1) + cc[2];
        se += (sim.cell_eps.empty() ? 1.0 : double(sim.cell_eps[id])) * w;
        ss += (sim.cell_sig.empty() ? 0.0 : double(sim.cell_sig[id])) * w;
        ws += w;
    }
    const double eps = EPS0 * se / ws, x = (ss / ws) * sim.dt / (2.0 * eps);
    ca = (1.0 - x) / (1.0 + x);
    cb = sim.dt / eps / (1.0 + x);
    return true;
}

int flux_objective64(Gpu* gpu, const HostSim& sim, uint64_t driven, double f0, double fc, const FluxSpec& sp,
                     FluxResult& res, std::string& err) {
    if (!gpu) { err = "no GPU: this engine has no CPU path"; return FG_ERR_NO_DEVICE; }
    if (!sim.debye_edges.empty() || !sim.inductors.empty() || !sim.wires.empty() || !sim.sheets.empty()) {
        err = "the FP64 forward supports dielectric, conducting, PEC and port media only (no Debye, inductor, wire or sheet)";
        return FG_ERR_INVALID;
    }
    if (driven >= sim.port_src.size()) { err = "the driven port does not exist"; return FG_ERR_INVALID; }
    if (sp.plane_k >= sim.n[2]) { err = "plane_k is outside the grid"; return FG_ERR_INVALID; }
    FG_CUDA(cudaSetDevice(gpu->device));
    const size_t n0 = sim.n[0], n1 = sim.n[1], n2 = sim.n[2], nn = sim.nn;
    Geom64 g{};
    g.n0 = int(n0); g.n1 = int(n1); g.n2 = int(n2); g.pml = int(sim.pml); g.nn = (long long)nn;
    long long psi_total = 0;
    for (int f = 0; f < 2; ++f)
        for (int c = 0; c < 3; ++c)
            for (int a = 0; a < 3; ++a) {
                g.psi_off[f * 9 + c * 3 + a] = psi_total;
                if (a != c && sim.pml > 0) {
                    size_t m[3] = {n0, n1, n2};
                    m[a] = 2 * sim.pml;
                    psi_total += (long long)(m[0] * m[1] * m[2]);
                }
            }
    // per-edge coefficients in f64
    std::vector<double> ca(3 * nn), cb(3 * nn);
#pragma omp parallel for schedule(static)
    for (long long id = 0; id < (long long)nn; ++id) {
        const size_t i = size_t(id) / (n1 * n2), j = (size_t(id) / n2) % n1, k = size_t(id) % n2;
        for (uint32_t c = 0; c < 3; ++c) {
            double a64 = 0, b64 = 0;
            const float a32 = sim.ca(c, size_t(id)), b32 = sim.cb(c, size_t(id));
            const bool plain = plain_coef64(sim, c, i, j, k, a64, b64) && float(a64) == a32 && float(b64) == b32;
            ca[c * nn + size_t(id)] = plain ? a64 : double(a32);
            cb[c * nn + size_t(id)] = plain ? b64 : double(b32);
        }
    }
    std::vector<AxisNode64> axes;
    for (int a = 0; a < 3; ++a) axes.insert(axes.end(), sim.ax[a].node64.begin(), sim.ax[a].node64.end());
    std::vector<long long> sf;
    std::vector<double> sv;
    for (const SrcEdge& e : sim.port_src[driven]) {
        sf.push_back((long long)e.comp * (long long)nn + (long long)e.id);
        sv.push_back(double(e.src));
    }
    double *d_e = nullptr, *d_h = nullptr, *d_psi = nullptr, *d_ca = nullptr, *d_cb = nullptr, *d_sv = nullptr, *d_acc = nullptr;
    long long* d_sf = nullptr;
    AxisNode64* d_ax = nullptr;
    auto release = [&] {
        for (void* p : {(void*)d_e, (void*)d_h, (void*)d_psi, (void*)d_ca, (void*)d_cb, (void*)d_sv, (void*)d_acc,
                        (void*)d_sf, (void*)d_ax})
            cudaFree(p);
    };
    std::unique_ptr<void, std::function<void(void*)>> guard((void*)1, [&](void*) { release(); });
    const size_t fb = 3 * nn * 8;
    FG_CUDA(cudaMalloc(&d_e, fb));
    FG_CUDA(cudaMalloc(&d_h, fb));
    FG_CUDA(cudaMalloc(&d_psi, size_t(std::max<long long>(psi_total, 1)) * 8));
    FG_CUDA(cudaMalloc(&d_ca, fb));
    FG_CUDA(cudaMalloc(&d_cb, fb));
    FG_CUDA(cudaMalloc(&d_ax, axes.size() * sizeof(AxisNode64)));
    FG_CUDA(cudaMalloc(&d_sf, std::max<size_t>(sf.size(), 1) * 8));
    FG_CUDA(cudaMalloc(&d_sv, std::max<size_t>(sv.size(), 1) * 8));
    FG_CUDA(cudaMalloc(&d_acc, n0 * n1 * 10 * 8));
    FG_CUDA(cudaMemset(d_e, 0, fb));
    FG_CUDA(cudaMemset(d_h, 0, fb));
    FG_CUDA(cudaMemset(d_psi, 0, size_t(std::max<long long>(psi_total, 1)) * 8));
    FG_CUDA(cudaMemset(d_acc, 0, n0 * n1 * 10 * 8));
    FG_CUDA(cudaMemcpy(d_ca, ca.data(), fb, cudaMemcpyHostToDevice));
    FG_CUDA(cudaMemcpy(d_cb, cb.data(), fb, cudaMemcpyHostToDevice));
    FG_CUDA(cudaMemcpy(d_ax, axes.data(), axes.size() * sizeof(AxisNode64), cudaMemcpyHostToDevice));
    if (!sf.empty()) {
        FG_CUDA(cudaMemcpy(d_sf, sf.data(), sf.size() * 8, cudaMemcpyHostToDevice));
        FG_CUDA(cudaMemcpy(d_sv, sv.data(), sv.size() * 8, cudaMemcpyHostToDevice));
    }
    g.ax[0] = d_ax;
    g.ax[1] = d_ax + n0;
    g.ax[2] = d_ax + n0 + n1;
    double t0 = 0, tau = 0;
    pulse_shape(fc, t0, tau);
    const double w0 = 2.0 * PI * f0, w = 2.0 * PI * sp.freq, dt = sim.dt, k_mu = dt / MU0;
    const dim3 blk(64, 4, 1), grd(unsigned((n2 + 63) / 64), unsigned((n1 + 3) / 4), unsigned(n0));
    const unsigned pb = unsigned((n0 * n1 + 127) / 128);
    auto t_start = std::chrono::steady_clock::now();
    for (uint64_t n = 0; n < sp.steps; ++n) {
        const double tp = (double(n) + 0.5) * dt, x = (tp - t0) / tau;
        const double pulse = std::exp(-x * x) * std::cos(w0 * (tp - t0));
        const double te = (double(n) + 1.0) * dt, th = (double(n) + 0.5) * dt;
        k_h64<<<grd, blk>>>(g, d_e, d_h, d_psi, k_mu);
        k_e64<<<grd, blk>>>(g, d_ca, d_cb, d_h, d_e, d_psi);
        if (!sf.empty()) k_src64<<<unsigned((sf.size() + 127) / 128), 128>>>(d_sf, d_sv, int(sf.size()), pulse, d_e);
        k_dft64<<<pb, 128>>>(g, int(sp.plane_k), std::cos(w * te) * dt, -std::sin(w * te) * dt, std::cos(w * th) * dt,
                             -std::sin(w * th) * dt, d_e, d_h, d_acc);
    }
    FG_CUDA(cudaGetLastError());
    std::vector<double> acc(n0 * n1 * 10);
    FG_CUDA(cudaMemcpy(acc.data(), d_acc, acc.size() * 8, cudaMemcpyDeviceToHost));
    res.forward_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    using cdd = std::complex<double>;
    auto at = [&](size_t i, size_t j, int comp) {
        const size_t q = (i * n1 + j) * 10;
        return cdd(acc[q + 2 * comp], acc[q + 2 * comp + 1]);
    };
    cdd F(0, 0);
    for (size_t i = sp.win_lo[0]; i < sp.win_hi[0]; ++i)
        for (size_t j = sp.win_lo[1]; j < sp.win_hi[1]; ++j)
            F += sim.ax[0].dd[i] * sim.ax[1].dd[j] * (at(i, j, 0) * std::conj(at(i, j, 4)) - at(i, j, 1) * std::conj(at(i, j, 3)));
    res.J = std::norm(F);
    res.f_re = F.real();
    res.f_im = F.imag();
    return FG_OK;
}

}  // namespace fg
