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

// ---- the fused adjoint step: both transposes in one march ----
//
// The E transpose gives, per E edge c at p, the adjoints (la_E, lb_E) of the two H differences it
// read; lambda_H'_C(p) = lambda_H_C(p) + la_E[C+1](p) - la_E[C+1](p + e_(C+2)) + lb_E[C+2](p)
// - lb_E[C+2](p + e_(C+1)). The H transpose then gives, per H edge, (la_H, lb_H) from lambda_H',
// and lambda_E_C(p) = ca lambda_E_C(p) + la_H[C+1](p - e_(C+2)) - la_H[C+1](p) + lb_H[C+2](p -
// e_(C+1)) - lb_H[C+2](p). So lambda_H' of plane i needs E-edge terms of planes i and i + 1, and
// lambda_E of plane i needs H-edge terms of planes i and i - 1: the forward's own data flow.
//
// A block marches along x over a tile of (j, k) nodes one node wider than it owns on every side:
// warp w serves row j0 - 1 + w and lane l column k0 - 1 + l, and owns rows 1..ADJ_TJ and lanes
// 1..30. Every thread forms the E-edge terms of its node (those of plane i + 1 one plane ahead,
// carried in registers); all but the last row and lane form lambda_H' and the H-edge terms; the
// owners form lambda_E. The k neighbours come by warp shuffles, the j neighbours through shared
// memory, and x neighbours stay in registers, so no thread recomputes another's terms and the
// warps do equal work. Every sum is formed in the order of k_adj_e and k_adj_h, so the fused step
// equals that pair of launches bit for bit. lambda_E, lambda_H and lambda_psi all ping-pong.
struct AdjArgs {
    Geom g;
    const void* node_class;
    const DevCoef* classes;
    const float* __restrict__ lE_in;
    float* __restrict__ lE_out;
    const float* __restrict__ lH_in;
    float* __restrict__ lH_out;
    const float* __restrict__ lpsi_in;
    float* __restrict__ lpsi_out;
    float k_mu;
};

// One axis node's factors as the adjoint reads them.
struct AdjAx {
    float inv_dd, be, cer;   // E side; cer = ce raw_inv_dd
    float inv_d, bh, chr;    // H side; chr = ch raw_inv_d
    int slot_e, slot_h;
};

__device__ __forceinline__ AdjAx adj_ax(const AxisNode* n) {
    AdjAx r;
    r.inv_dd = __ldg(&n->inv_dd);
    r.be = __ldg(&n->be);
    r.cer = __ldg(&n->ce) * __ldg(&n->raw_inv_dd);
    r.inv_d = __ldg(&n->inv_d);
    r.bh = __ldg(&n->bh);
    r.chr = __ldg(&n->ch) * __ldg(&n->raw_inv_d);
    r.slot_e = __ldg(&n->slot_e);
    r.slot_h = __ldg(&n->slot_h);
    return r;
}

constexpr int ADJ_TJ = 14;              // rows a block owns
constexpr int ADJ_ROWS = ADJ_TJ + 2;    // warps: the owned rows and the j - 1 and j + ADJ_TJ rows
constexpr int ADJ_KOWN = 30;            // columns a block owns (lanes 1..30)

// A block's y and z axis factors in shared memory (field-major, slots as int bits): a thread's j
// and k stay fixed along the march; the x factors are the plane's, one address for the block.
struct AdjSm {
    float y[8][ADJ_ROWS];
    float z[8][32];
};

template <int N>
__device__ __forceinline__ void adj_sm_fill(float (&t)[8][N], int at, const AxisNode* n) {
    const AdjAx r = adj_ax(n);
    t[0][at] = r.inv_dd;
    t[1][at] = r.be;
    t[2][at] = r.cer;
    t[3][at] = r.inv_d;
    t[4][at] = r.bh;
    t[5][at] = r.chr;
    t[6][at] = __int_as_float(r.slot_e);
    t[7][at] = __int_as_float(r.slot_h);
}

template <int N>
__device__ __forceinline__ AdjAx adj_sm_get(const float (&t)[8][N], int at) {
    AdjAx r;
    r.inv_dd = t[0][at];
    r.be = t[1][at];
    r.cer = t[2][at];
    r.inv_d = t[3][at];
    r.bh = t[4][at];
    r.chr = t[5][at];
    r.slot_e = __float_as_int(t[6][at]);
    r.slot_h = __float_as_int(t[7][at]);
    return r;
}

// Where a thread's axis factors are: the block's table and the thread's row (w) and lane.
struct AdjAt {
    const AdjSm* sm;
    int w, lane;
};

__device__ __forceinline__ AdjAx adj_axis(const Geom& g, int u, int i, const AdjAt& at) {
    if (u == 0) return adj_ax(g.ax[0] + i);
    return u == 1 ? adj_sm_get(at.sm->y, at.w) : adj_sm_get(at.sm->z, at.lane);
}

// E-edge c's terms at p given its coefficients: (la_E, lb_E) and ca lambda_E (le). `own` writes
// the edge's lambda_psi.
__device__ __forceinline__ void adj_e_terms(const AdjArgs& a, const AdjAt& at, int c, int i, int j, int k, float l,
                                            float ca, float cb, bool own, float& la, float& lb, float& le) {
    const Geom& g = a.g;
    const int p[3] = {i, j, k};
    const int U = (c + 1) % 3, V = (c + 2) % 3;
    const bool m = cb != 0.0f && p[U] > 0 && p[V] > 0;
    le = m ? ca * l : l;
    const float gg = m ? cb * l : 0.f;
    const AdjAx au = adj_axis(g, U, i, at);
    const AdjAx av = adj_axis(g, V, i, at);
    la = gg * au.inv_dd;
    lb = -gg * av.inv_dd;
    if (au.slot_e >= 0) {
        const long long q = g.psi_off[c * 3 + U] + psi_at(g, U, i, j, k, au.slot_e);
        const float lp = a.lpsi_in[q];
        if (own) a.lpsi_out[q] = m ? au.be * (gg + lp) : lp;
        if (m) la += au.cer * (gg + lp);
    }
    if (av.slot_e >= 0) {
        const long long q = g.psi_off[c * 3 + V] + psi_at(g, V, i, j, k, av.slot_e);
        const float lp = a.lpsi_in[q];
        if (own) a.lpsi_out[q] = m ? av.be * (-gg + lp) : lp;
        if (m) lb += av.cer * (-gg + lp);
    }
}

// All three E edges of node p from its lambda_E (l) and class id (cid); zero unless `ok`.
__device__ __forceinline__ void adj_e_from(const AdjArgs& a, const AdjAt& at, int i, int j, int k, bool ok, bool own,
                                           const float (&l)[3], unsigned cid, float (&la)[3], float (&lb)[3],
                                           float (&le)[3]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) la[c] = lb[c] = le[c] = 0.f;
    if (!ok) return;
    const DevCoef cf = a.classes[cid];
#pragma unroll
    for (int c = 0; c < 3; ++c) adj_e_terms(a, at, c, i, j, k, l[c], cf.ca[c], cf.cb[c], own, la[c], lb[c], le[c]);
}

// lambda_E and the class id of node p (zeros unless `ok`).
template <typename CID>
__device__ __forceinline__ void adj_e_load(const AdjArgs& a, long long id, bool ok, float (&l)[3], unsigned& cid) {
    const Geom& g = a.g;
    l[0] = l[1] = l[2] = 0.f;
    cid = 0;
    if (!ok) return;
    l[0] = a.lE_in[id];
    l[1] = a.lE_in[g.cs + id];
    l[2] = a.lE_in[2 * g.cs + id];
    cid = static_cast<const CID*>(a.node_class)[id];
}

// All three E edges of node p; zero where `in` is false (p off the grid) or past the last plane.
template <typename CID>
__device__ __forceinline__ void adj_e_all(const AdjArgs& a, const AdjAt& at, int i, int j, int k, bool in, bool own,
                                          float (&la)[3], float (&lb)[3], float (&le)[3]) {
    const Geom& g = a.g;
    const bool ok = in && i < g.n0;
    float l[3];
    unsigned cid;
    adj_e_load<CID>(a, ((long long)i * g.n1 + j) * g.p2 + k, ok, l, cid);
    adj_e_from(a, at, i, j, k, ok, own, l, cid, la, lb, le);
}

// H edge c's terms at p from its lambda_H' (lh): (la_H, lb_H); `own` writes its lambda_psi.
__device__ __forceinline__ float2 adj_h_terms(const AdjArgs& a, const AdjAt& at, int c, int i, int j, int k, float lh,
                                              bool own) {
    const Geom& g = a.g;
    const int p[3] = {i, j, k};
    const int n[3] = {g.n0, g.n1, g.n2};
    const int U = (c + 1) % 3, V = (c + 2) % 3;
    const bool r = p[U] + 1 < n[U] && p[V] + 1 < n[V];
    const float gh = r ? -a.k_mu * lh : 0.f;
    const AdjAx au = adj_axis(g, U, i, at);
    const AdjAx av = adj_axis(g, V, i, at);
    float la = gh * au.inv_d;
    float lb = -gh * av.inv_d;
    if (au.slot_h >= 0) {
        const long long q = g.psi_off[9 + c * 3 + U] + psi_at(g, U, i, j, k, au.slot_h);
        const float lp = a.lpsi_in[q];
        if (own) a.lpsi_out[q] = r ? au.bh * (gh + lp) : lp;
        if (r) la += au.chr * (gh + lp);
    }
    if (av.slot_h >= 0) {
        const long long q = g.psi_off[9 + c * 3 + V] + psi_at(g, V, i, j, k, av.slot_h);
        const float lp = a.lpsi_in[q];
        if (own) a.lpsi_out[q] = r ? av.bh * (-gh + lp) : lp;
        if (r) lb += av.chr * (-gh + lp);
    }
    return make_float2(la, lb);
}

// Grid (ceil(n2 / 30), ceil(n1 / 14), ceil(n0 / seg)), block (32, 16). The loads of lambda_E and
// the class id run two planes ahead and those of lambda_H one plane ahead of their use.
template <typename CID>
__global__ void __launch_bounds__(32 * ADJ_ROWS, 2) k_adj_step(AdjArgs a, int seg) {
    __shared__ float es[2][ADJ_ROWS][32];   // la_E[0], lb_E[2] of each row (read by the row below)
    __shared__ float hs[2][ADJ_ROWS][32];   // la_H[0], lb_H[2] of each row (read by the row above)
    __shared__ AdjSm sm;
    const Geom& g = a.g;
    const int lane = threadIdx.x, w = threadIdx.y;
    const int k = int(blockIdx.x) * ADJ_KOWN + lane - 1;
    const int j = int(blockIdx.y) * ADJ_TJ + w - 1;
    if (w == 0) adj_sm_fill(sm.z, lane, g.ax[2] + min(max(k, 0), g.n2 - 1));
    if (w == 1 && lane < ADJ_ROWS) {
        const int jr = int(blockIdx.y) * ADJ_TJ + lane - 1;
        adj_sm_fill(sm.y, lane, g.ax[1] + min(max(jr, 0), g.n1 - 1));
    }
    __syncthreads();
    const AdjAt at{&sm, w, lane};
    const int i0 = int(blockIdx.z) * seg, i1 = min(i0 + seg, g.n0);
    const bool in = j >= 0 && k >= 0 && j < g.n1 && k < g.n2;
    const bool own = in && lane >= 1 && lane <= ADJ_KOWN && w >= 1 && w <= ADJ_TJ;
    const bool hrow = in && lane <= ADJ_KOWN && w <= ADJ_TJ;   // forms lambda_H' and the H-edge terms
    const long long plane = (long long)g.n1 * g.p2, col = (long long)j * g.p2 + k;
    constexpr unsigned FULL = 0xffffffffu;
    float ea[3], eb[3], le[3];   // E-edge terms and ca lambda_E of plane i
    adj_e_all<CID>(a, at, i0, j, k, in, own, ea, eb, le);
    float pa2 = 0.f, pb1 = 0.f;  // la_H[2], lb_H[1] of plane i - 1
    if (i0 > 0) {
        // the H-edge terms of plane i0 - 1 that plane i0 reads, from the inputs
        float qa[3], qb[3], ql[3];
        adj_e_all<CID>(a, at, i0 - 1, j, k, in, false, qa, qb, ql);
        es[0][w][lane] = qa[0];
        const float sb0 = __shfl_down_sync(FULL, qb[0], 1);
        __syncthreads();
        if (hrow) {
            const long long id = (i0 - 1) * plane + col;
            const float h1 = a.lH_in[g.cs + id] + ((qa[2] - ea[2]) + (qb[0] - sb0));
            const float h2 = a.lH_in[2 * g.cs + id] + ((qa[0] - es[0][w + 1][lane]) + (qb[1] - eb[1]));
            pb1 = adj_h_terms(a, at, 1, i0 - 1, j, k, h1, false).y;
            pa2 = adj_h_terms(a, at, 2, i0 - 1, j, k, h2, false).x;
        }
        __syncthreads();
    }
    float fe[3], fh[3] = {0.f, 0.f, 0.f};   // lambda_E of plane i + 1, lambda_H of plane i
    unsigned fc;                            // class id of plane i + 1
    adj_e_load<CID>(a, (i0 + 1) * plane + col, in && i0 + 1 < g.n0, fe, fc);
    if (hrow) {
        const long long id = i0 * plane + col;
        fh[0] = a.lH_in[id];
        fh[1] = a.lH_in[g.cs + id];
        fh[2] = a.lH_in[2 * g.cs + id];
    }
    for (int i = i0; i < i1; ++i) {
        const float l[3] = {fe[0], fe[1], fe[2]}, hc[3] = {fh[0], fh[1], fh[2]};
        const unsigned cid = fc;
        adj_e_load<CID>(a, (i + 2) * plane + col, in && i + 2 < g.n0, fe, fc);
        if (hrow && i + 1 < i1) {
            const long long id = (i + 1) * plane + col;
            fh[0] = a.lH_in[id];
            fh[1] = a.lH_in[g.cs + id];
            fh[2] = a.lH_in[2 * g.cs + id];
        }
        float na[3], nb[3], nle[3];
        adj_e_from(a, at, i + 1, j, k, in && i + 1 < g.n0, own && i + 1 < i1, l, cid, na, nb, nle);
        es[0][w][lane] = ea[0];
        es[1][w][lane] = eb[2];
        const float sa1 = __shfl_down_sync(FULL, ea[1], 1);   // la_E[1] at k + 1
        const float sb0 = __shfl_down_sync(FULL, eb[0], 1);   // lb_E[0] at k + 1
        __syncthreads();
        float ha[3] = {0.f, 0.f, 0.f}, hb[3] = {0.f, 0.f, 0.f};
        if (hrow) {
            const long long id = i * plane + col;
            const float h0 = hc[0] + ((ea[1] - sa1) + (eb[2] - es[1][w + 1][lane]));
            const float h1 = hc[1] + ((ea[2] - na[2]) + (eb[0] - sb0));
            const float h2 = hc[2] + ((ea[0] - es[0][w + 1][lane]) + (eb[1] - nb[1]));
            if (own) {
                a.lH_out[id] = h0;
                a.lH_out[g.cs + id] = h1;
                a.lH_out[2 * g.cs + id] = h2;
            }
            const float2 t0 = adj_h_terms(a, at, 0, i, j, k, h0, own);
            const float2 t1 = adj_h_terms(a, at, 1, i, j, k, h1, own);
            const float2 t2 = adj_h_terms(a, at, 2, i, j, k, h2, own);
            ha[0] = t0.x; hb[0] = t0.y;
            ha[1] = t1.x; hb[1] = t1.y;
            ha[2] = t2.x; hb[2] = t2.y;
        }
        hs[0][w][lane] = ha[0];
        hs[1][w][lane] = hb[2];
        const float ua1 = __shfl_up_sync(FULL, ha[1], 1);   // la_H[1] at k - 1
        const float ub0 = __shfl_up_sync(FULL, hb[0], 1);   // lb_H[0] at k - 1
        __syncthreads();
        if (own) {
            const long long id = i * plane + col;
            a.lE_out[id] = le[0] + ((ua1 - ha[1]) + (hs[1][w - 1][lane] - hb[2]));
            a.lE_out[g.cs + id] = le[1] + ((pa2 - ha[2]) + (ub0 - hb[0]));
            a.lE_out[2 * g.cs + id] = le[2] + ((hs[0][w - 1][lane] - ha[0]) + (pb1 - hb[1]));
        }
        pa2 = ha[2];
        pb1 = hb[1];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            ea[c] = na[c];
            eb[c] = nb[c];
            le[c] = nle[c];
        }
    }
}

// Transpose of the Debye ADE that follows the march (cpu.rs:239-260, debye_post_edge): per Debye
// edge, E' = E* - cb sum_k (1 + b_k)/2 s_k and s_k' = b_k s_k + dd c_k (E' - E_old), E_old the
// step's input. Given lambda_E' (in lE, in place) and lambda_s' (in ls, in place):
//   d = sum_k dd c_k lambda_s'_k;  lambda_E* = lambda_E' + d;  lambda_s_k = b_k lambda_s'_k
//   - cb (1 + b_k)/2 lambda_E*;  and lambda_E_old gains -d, kept in `old` for k_adj_debye_post,
// which adds it to the march transpose's output (E_old is the step's input E).
template <typename CID>
__global__ void k_adj_debye_pre(const long long* __restrict__ f, const float* __restrict__ dd, int count,
                                const CID* __restrict__ node_class, const DevCoef* __restrict__ classes, long long cs,
                                const float* __restrict__ table, float* __restrict__ ls, float* __restrict__ lE,
                                float* __restrict__ old) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const long long fi = f[q];
    const int c = int(fi / cs);
    const long long id = fi - c * cs;
    const float cb = classes[node_class[id]].cb[c];
    const int np = int(table[0]);
    const float w = dd[q];
    float d = 0.0f;
    for (int k = 0; k < np; ++k) d += w * table[2 + 2 * k] * ls[(long long)k * count + q];
    const float le = lE[fi] + d;
    lE[fi] = le;
    for (int k = 0; k < np; ++k) {
        const long long p = (long long)k * count + q;
        ls[p] = table[1 + 2 * k] * ls[p] - cb * (0.5f * (1.0f + table[1 + 2 * k])) * le;
    }
    old[q] = -d;
}

__global__ void k_adj_debye_post(const long long* __restrict__ f, int count, const float* __restrict__ old,
                                 float* __restrict__ lE) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < count) lE[f[q]] += old[q];
}

// dJ/d(state after step n) of the flux objective on the plane window: per window node four
// complex weights (Px, Py for Ex, Ey; Qx, Qy for Hx, Hy) times the step's DFT phase factors
// (the same per-step table the forward DFT used, frequency 0).
__device__ __forceinline__ void adj_inject(const Geom& g, int t, int plane_k, int i0, int wi, int j0, int wj,
                                           const float* __restrict__ w, const float* __restrict__ dft, int nf,
                                           long long n, float* __restrict__ lE, float* __restrict__ lH) {
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

__global__ void k_adj_inject(Geom g, int plane_k, int i0, int wi, int j0, int wj, const float* __restrict__ w,
                             const float* __restrict__ dft, int nf, long long n, float* __restrict__ lE,
                             float* __restrict__ lH) {
    adj_inject(g, blockIdx.x * blockDim.x + threadIdx.x, plane_k, i0, wi, j0, wj, w, dft, nf, n, lE, lH);
}

// dJ/dca and dJ/dcb of every design edge: the adjoint of E^n+1 times E^n and S^n, summed in f64.
__device__ __forceinline__ void adj_grad(const Geom& g, int t, const int4* __restrict__ edges, int n,
                                         const float* __restrict__ lE, const float* __restrict__ hist_e,
                                         const float* __restrict__ hist_s, long long slot, double* __restrict__ ga,
                                         double* __restrict__ gb) {
    if (t >= n) return;
    const int4 d = edges[t];
    const long long id = ((long long)d.y * g.n1 + d.z) * g.p2 + d.w;
    const double l = lE[d.x * g.cs + id];
    ga[t] += l * double(hist_e[slot * n + t]);
    gb[t] += l * double(hist_s[slot * n + t]);
}

__global__ void k_adj_grad(Geom g, const int4* __restrict__ edges, int n, const float* __restrict__ lE,
                           const float* __restrict__ hist_e, const float* __restrict__ hist_s, long long slot,
                           double* __restrict__ ga, double* __restrict__ gb) {
    adj_grad(g, blockIdx.x * blockDim.x + threadIdx.x, edges, n, lE, hist_e, hist_s, slot, ga, gb);
}

// Both of a sweep step's small parts in one launch, where no design edge is a window node of the
// plane (so the gradient reads no lambda_E the source writes): blocks [0, wblocks) add the
// source (k_adj_inject), the rest accumulate the gradient (k_adj_grad). 128 threads per block.
__global__ void k_adj_source_grad(Geom g, int plane_k, int i0, int wi, int j0, int wj, const float* __restrict__ w,
                                  const float* __restrict__ dft, int nf, long long n_step, float* __restrict__ lE,
                                  float* __restrict__ lH, unsigned wblocks, const int4* __restrict__ edges, int nd,
                                  const float* __restrict__ hist_e, const float* __restrict__ hist_s, long long slot,
                                  double* __restrict__ ga, double* __restrict__ gb) {
    if (blockIdx.x < wblocks)
        adj_inject(g, blockIdx.x * blockDim.x + threadIdx.x, plane_k, i0, wi, j0, wj, w, dft, nf, n_step, lE, lH);
    else
        adj_grad(g, (blockIdx.x - wblocks) * blockDim.x + threadIdx.x, edges, nd, lE, hist_e, hist_s, slot, ga, gb);
}

}  // namespace fg
