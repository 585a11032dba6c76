// Kernels of the discrete adjoint of the FDTD step, for gradients of a flux objective with
// respect to per-voxel permittivity and conductivity. The step (sims-field cpu.rs:48-167) is linear
// in its state (E, H and the CPML psi), and only the E update's ca, cb depend on the materials, so
// the gradient needs, per design edge and step n, E^n and the curl term S^n that multiplied cb
// (E^n+1 = ca E^n + cb S^n), and the adjoint state swept backward in time:
//   lambda(before step n) = M_H^T M_E^T lambda(after step n) + dJ/d(state after step n - 1/2 ...)
// with M_E the E half of the step and M_H the H half. Each half's transpose is one kernel:
//   k_adj_e: lambda_E <- ca lambda_E; lambda_psiE <- be (+-cb lambda_E + lambda_psiE); lambda_H gathers
//            the E edges' adjoint differences (a curl of cb lambda_E, with the CPML terms);
//   k_adj_h: lambda_psiH <- bh (-+k_mu lambda_H + lambda_psiH); lambda_E gathers the H edges'
//            adjoint differences.
// Adjoint E and psi arrays ping-pong between two sets (a kernel reads its neighbours' old values).
#pragma once

#include "kernels.cuh"

namespace fg {

// After step n of the fused march: E^n (the step's input set) and the curl term S^n its E update
// used, for every design edge. The arithmetic is the E update's own (cpu.rs:125-162): the E psi
// slabs already hold the new psi, which is the term the update added.
__global__ void k_design_record(Geom g, const int4* __restrict__ edges, int n, const float* __restrict__ e_in,
                                const float* __restrict__ h_new, const float* __restrict__ psi,
                                const unsigned* __restrict__ counter, const long long* __restrict__ base, int cap,
                                float* __restrict__ hist_e, float* __restrict__ hist_s) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const long long slot = (long long)step_index(counter) - *base;
    if (slot < 0 || slot >= cap) return;
    const int4 d = edges[t];
    const int c = d.x;
    const int p[3] = {d.y, d.z, d.w};
    const int U = (c + 1) % 3, V = (c + 2) % 3;
    const long long st[3] = {(long long)g.n1 * g.p2, g.p2, 1};
    const long long id = ((long long)p[0] * g.n1 + p[1]) * g.p2 + p[2];
    const float a = h_new[V * g.cs + id] - h_new[V * g.cs + id - st[U]];
    const float b = h_new[U * g.cs + id] - h_new[U * g.cs + id - st[V]];
    const AxisNode& au = g.ax[U][p[U]];
    const AxisNode& av = g.ax[V][p[V]];
    float t1 = a * au.inv_dd, t2 = b * av.inv_dd;
    if (au.slot_e >= 0) t1 += psi[g.psi_off[c * 3 + U] + psi_at(g, U, p[0], p[1], p[2], au.slot_e)];
    if (av.slot_e >= 0) t2 += psi[g.psi_off[c * 3 + V] + psi_at(g, V, p[0], p[1], p[2], av.slot_e)];
    hist_e[slot * n + t] = e_in[c * g.cs + id];
    hist_s[slot * n + t] = t1 - t2;
}

// Each E edge's (ca, cb) where its update runs (cb != 0, off the low faces), else (1, 0): the
// adjoint's per-step reads of the coefficients, formed once (k_adj_coefs) as flat arrays.
template <typename CID>
__global__ void k_adj_coefs(Geom g, const CID* __restrict__ node_class, const DevCoef* __restrict__ classes,
                            float* __restrict__ cam, float* __restrict__ cbm) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= g.n2 || j >= g.n1) return;
    const int p[3] = {i, j, k};
    const long long id = ((long long)i * g.n1 + j) * g.p2 + k;
    const DevCoef cf = classes[node_class[id]];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const bool m = cf.cb[c] != 0.0f && p[(c + 1) % 3] > 0 && p[(c + 2) % 3] > 0;
        cam[c * g.cs + id] = m ? cf.ca[c] : 1.0f;
        cbm[c * g.cs + id] = m ? cf.cb[c] : 0.0f;
    }
}

// The adjoints of the two H differences a, b that E edge c at p reads (cb lambda_E through the
// inv_dd factors and the CPML terms); zero where the edge does not update or lies off the grid.
__device__ __forceinline__ void e_edge_lab(const Geom& g, const float* __restrict__ cbm, const float* __restrict__ lE,
                                           const float* __restrict__ lpsi, int c, int i, int j, int k, float& la,
                                           float& lb) {
    la = 0.f;
    lb = 0.f;
    if (i >= g.n0 || j >= g.n1 || k >= g.n2) return;
    const long long id = ((long long)i * g.n1 + j) * g.p2 + k;
    const float cb = cbm[c * g.cs + id];
    if (cb == 0.0f) return;
    const int p[3] = {i, j, k};
    const int U = (c + 1) % 3, V = (c + 2) % 3;
    const float gg = cb * lE[c * g.cs + id];
    const AxisNode& au = g.ax[U][p[U]];
    const AxisNode& av = g.ax[V][p[V]];
    la = gg * au.inv_dd;
    lb = -gg * av.inv_dd;
    if (au.slot_e >= 0)
        la += (au.ce * au.raw_inv_dd) * (gg + lpsi[g.psi_off[c * 3 + U] + psi_at(g, U, i, j, k, au.slot_e)]);
    if (av.slot_e >= 0)
        lb += (av.ce * av.raw_inv_dd) * (-gg + lpsi[g.psi_off[c * 3 + V] + psi_at(g, V, i, j, k, av.slot_e)]);
}

// The adjoints of the two E differences a, b that H edge c at p reads; zero where the H update
// does not run (a neighbour past the grid) or p lies off the grid.
__device__ __forceinline__ void h_edge_lab(const Geom& g, const float* __restrict__ lH,
                                           const float* __restrict__ lpsi, float k_mu, int c, int i, int j, int k,
                                           float& la, float& lb) {
    la = 0.f;
    lb = 0.f;
    if (i < 0 || j < 0 || k < 0) return;
    const int p[3] = {i, j, k};
    const int n[3] = {g.n0, g.n1, g.n2};
    const int U = (c + 1) % 3, V = (c + 2) % 3;
    if (p[U] + 1 >= n[U] || p[V] + 1 >= n[V]) return;
    const long long id = ((long long)i * g.n1 + j) * g.p2 + k;
    const float gh = -k_mu * lH[c * g.cs + id];
    const AxisNode& au = g.ax[U][p[U]];
    const AxisNode& av = g.ax[V][p[V]];
    la = gh * au.inv_d;
    lb = -gh * av.inv_d;
    if (au.slot_h >= 0)
        la += (au.ch * au.raw_inv_d) * (gh + lpsi[g.psi_off[9 + c * 3 + U] + psi_at(g, U, i, j, k, au.slot_h)]);
    if (av.slot_h >= 0)
        lb += (av.ch * av.raw_inv_d) * (-gh + lpsi[g.psi_off[9 + c * 3 + V] + psi_at(g, V, i, j, k, av.slot_h)]);
}

// Transpose of the E half of a step. Grid (ceil(n2/64), ceil(n1/4), n0), block (64, 4).
__global__ void __launch_bounds__(256) k_adj_e(Geom g, const float* __restrict__ cam, const float* __restrict__ cbm,
                                               const float* __restrict__ lE_in, float* __restrict__ lE_out,
                                               const float* __restrict__ lpsi_in, float* __restrict__ lpsi_out,
                                               float* __restrict__ lH) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= g.n2 || j >= g.n1) return;
    const int p[3] = {i, j, k};
    const long long id = ((long long)i * g.n1 + j) * g.p2 + k;
    float la[3], lb[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int U = (c + 1) % 3, V = (c + 2) % 3;
        const float l = lE_in[c * g.cs + id];
        const float cb = cbm[c * g.cs + id];
        const bool m = cb != 0.0f;
        lE_out[c * g.cs + id] = cam[c * g.cs + id] * l;
        const float gg = cb * l;
        const AxisNode& au = g.ax[U][p[U]];
        const AxisNode& av = g.ax[V][p[V]];
        la[c] = gg * au.inv_dd;
        lb[c] = -gg * av.inv_dd;
        if (au.slot_e >= 0) {
            const long long q = g.psi_off[c * 3 + U] + psi_at(g, U, i, j, k, au.slot_e);
            const float lp = lpsi_in[q];
            lpsi_out[q] = m ? au.be * (gg + lp) : lp;
            if (m) la[c] += (au.ce * au.raw_inv_dd) * (gg + lp);
        }
        if (av.slot_e >= 0) {
            const long long q = g.psi_off[c * 3 + V] + psi_at(g, V, i, j, k, av.slot_e);
            const float lp = lpsi_in[q];
            lpsi_out[q] = m ? av.be * (-gg + lp) : lp;
            if (m) lb[c] += (av.ce * av.raw_inv_dd) * (-gg + lp);
        }
    }
    // lambda_H_C += la(C+1, q) - la(C+1, q + e_(C+2)) + lb(C+2, q) - lb(C+2, q + e_(C+1))
    float na, nb, dummy;
    e_edge_lab(g, cbm, lE_in, lpsi_in, 1, i, j, k + 1, na, dummy);
    e_edge_lab(g, cbm, lE_in, lpsi_in, 2, i, j + 1, k, dummy, nb);
    lH[id] += (la[1] - na) + (lb[2] - nb);
    e_edge_lab(g, cbm, lE_in, lpsi_in, 2, i + 1, j, k, na, dummy);
    e_edge_lab(g, cbm, lE_in, lpsi_in, 0, i, j, k + 1, dummy, nb);
    lH[g.cs + id] += (la[2] - na) + (lb[0] - nb);
    e_edge_lab(g, cbm, lE_in, lpsi_in, 0, i, j + 1, k, na, dummy);
    e_edge_lab(g, cbm, lE_in, lpsi_in, 1, i + 1, j, k, dummy, nb);
    lH[2 * g.cs + id] += (la[0] - na) + (lb[1] - nb);
}

// Transpose of the H half of a step (lambda_H itself passes through unchanged).
__global__ void __launch_bounds__(256) k_adj_h(Geom g, const float* __restrict__ lH, const float* __restrict__ lpsi_in,
                                               float* __restrict__ lpsi_out, float* __restrict__ lE, float k_mu) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= g.n2 || j >= g.n1) return;
    const int p[3] = {i, j, k};
    const int n[3] = {g.n0, g.n1, g.n2};
    const long long id = ((long long)i * g.n1 + j) * g.p2 + k;
    float la[3], lb[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const int U = (c + 1) % 3, V = (c + 2) % 3;
        const bool r = p[U] + 1 < n[U] && p[V] + 1 < n[V];
        const float gh = r ? -k_mu * lH[c * g.cs + id] : 0.f;
        const AxisNode& au = g.ax[U][p[U]];
        const AxisNode& av = g.ax[V][p[V]];
        la[c] = gh * au.inv_d;
        lb[c] = -gh * av.inv_d;
        if (au.slot_h >= 0) {
            const long long q = g.psi_off[9 + c * 3 + U] + psi_at(g, U, i, j, k, au.slot_h);
            const float lp = lpsi_in[q];
            lpsi_out[q] = r ? au.bh * (gh + lp) : lp;
            if (r) la[c] += (au.ch * au.raw_inv_d) * (gh + lp);
        }
        if (av.slot_h >= 0) {
            const long long q = g.psi_off[9 + c * 3 + V] + psi_at(g, V, i, j, k, av.slot_h);
            const float lp = lpsi_in[q];
            lpsi_out[q] = r ? av.bh * (-gh + lp) : lp;
            if (r) lb[c] += (av.ch * av.raw_inv_d) * (-gh + lp);
        }
    }
    // lambda_E_C += la(C+1, q - e_(C+2)) - la(C+1, q) + lb(C+2, q - e_(C+1)) - lb(C+2, q)
    float na, nb, dummy;
    h_edge_lab(g, lH, lpsi_in, k_mu, 1, i, j, k - 1, na, dummy);
    h_edge_lab(g, lH, lpsi_in, k_mu, 2, i, j - 1, k, dummy, nb);
    lE[id] += (na - la[1]) + (nb - lb[2]);
    h_edge_lab(g, lH, lpsi_in, k_mu, 2, i - 1, j, k, na, dummy);
    h_edge_lab(g, lH, lpsi_in, k_mu, 0, i, j, k - 1, dummy, nb);
    lE[g.cs + id] += (na - la[2]) + (nb - lb[0]);
    h_edge_lab(g, lH, lpsi_in, k_mu, 0, i, j - 1, k, na, dummy);
    h_edge_lab(g, lH, lpsi_in, k_mu, 1, i - 1, j, k, dummy, nb);
    lE[2 * g.cs + id] += (na - la[0]) + (nb - lb[1]);
}

// dJ/d(state after step n) of the flux objective on the plane window: per window node four
// complex weights (Px, Py for Ex, Ey; Qx, Qy for Hx, Hy) times the step's DFT phase factors
// (the same per-step table the forward DFT used, frequency 0).
__global__ void k_adj_inject(Geom g, int plane_k, int i0, int wi, int j0, int wj, const float* __restrict__ w,
                             const float* __restrict__ dft, int nf, long long n, float* __restrict__ lE,
                             float* __restrict__ lH) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= wi * wj) return;
    const int i = i0 + t / wj, j = j0 + t % wj;
    const float* d = dft + (n * nf) * 4;
    const float* c = w + (long long)t * 8;   // Px, Py, Qx, Qy as (re, im)
    const long long id = ((long long)i * g.n1 + j) * g.p2 + plane_k;
    lE[id] += 2.0f * (c[0] * d[0] - c[1] * d[1]);
    lE[g.cs + id] += 2.0f * (c[2] * d[0] - c[3] * d[1]);
    lH[id] += 2.0f * (c[4] * d[2] + c[5] * d[3]);
    lH[g.cs + id] += 2.0f * (c[6] * d[2] + c[7] * d[3]);
}

// dJ/dca and dJ/dcb of every design edge: the adjoint of E^n+1 times E^n and S^n, summed in f64.
__global__ void k_adj_grad(Geom g, const int4* __restrict__ edges, int n, const float* __restrict__ lE,
                           const float* __restrict__ hist_e, const float* __restrict__ hist_s, long long slot,
                           double* __restrict__ ga, double* __restrict__ gb) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int4 d = edges[t];
    const long long id = ((long long)d.y * g.n1 + d.z) * g.p2 + d.w;
    const double l = lE[d.x * g.cs + id];
    ga[t] += l * double(hist_e[slot * n + t]);
    gb[t] += l * double(hist_s[slot * n + t]);
}

}  // namespace fg
