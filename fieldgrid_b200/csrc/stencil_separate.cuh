// The unfused field update: one kernel for H, one for E, each in place, with the CPML psi
// recursions (sims-field cpu.rs:48-167). It mirrors the reference's "separate" step
// (run.rs:638-657, Extras.fused_e = false) and serves as the plain baseline the fused march in
// stencil_fused.cuh is checked and timed against.
#pragma once

#include "kernels.cuh"

namespace fg {

// H_c -= k_mu * [(dE_v/du) inv_d_u + psi_u - (dE_u/dv) inv_d_v - psi_v]   (cpu.rs:65-102)
template <int C>
__device__ __forceinline__ void h_update_one(const Geom& g, const int p[3], long long id, const long long st[3],
                                             const float* __restrict__ e, float* __restrict__ h, float* __restrict__ psi,
                                             float k_mu) {
    constexpr int U = (C + 1) % 3, V = (C + 2) % 3;
    const int nu = U == 0 ? g.n0 : (U == 1 ? g.n1 : g.n2);
    const int nv = V == 0 ? g.n0 : (V == 1 ? g.n1 : g.n2);
    if (p[U] + 1 >= nu || p[V] + 1 >= nv) return;
    const float ev = e[V * g.cs + id + st[U]] - e[V * g.cs + id];
    const float eu = e[U * g.cs + id + st[V]] - e[U * g.cs + id];
    const AxisNode* au = g.ax[U] + p[U];
    const AxisNode* av = g.ax[V] + p[V];
    float t1 = ev * __ldg(&au->inv_d);
    float t2 = eu * __ldg(&av->inv_d);
    if (g.pml > 0) {
        const int su = __ldg(&au->slot_h);
        if (su >= 0) {
            const long long q = g.psi_off[9 + C * 3 + U] + psi_at(g, U, p[0], p[1], p[2], su);
            const float r = __ldg(&au->bh) * psi[q] + __ldg(&au->ch) * ev * __ldg(&au->raw_inv_d);
            psi[q] = r;
            t1 += r;
        }
        const int sv = __ldg(&av->slot_h);
        if (sv >= 0) {
            const long long q = g.psi_off[9 + C * 3 + V] + psi_at(g, V, p[0], p[1], p[2], sv);
            const float r = __ldg(&av->bh) * psi[q] + __ldg(&av->ch) * eu * __ldg(&av->raw_inv_d);
            psi[q] = r;
            t2 += r;
        }
    }
    h[C * g.cs + id] -= k_mu * (t1 - t2);
}

// E_c = ca E_c + cb [(dH_v/du) inv_dd_u + psi_u - (dH_u/dv) inv_dd_v - psi_v], skipped where
// cb == 0 (cpu.rs:125-162)
template <int C>
__device__ __forceinline__ void e_update_one(const Geom& g, const int p[3], long long id, const long long st[3],
                                             const DevCoef& cf, const float* __restrict__ h, float* __restrict__ e,
                                             float* __restrict__ psi) {
    constexpr int U = (C + 1) % 3, V = (C + 2) % 3;
    const float cb = cf.cb[C];
    if (cb == 0.0f || p[U] == 0 || p[V] == 0) return;
    const float hv = h[V * g.cs + id] - h[V * g.cs + id - st[U]];
    const float hu = h[U * g.cs + id] - h[U * g.cs + id - st[V]];
    const AxisNode* au = g.ax[U] + p[U];
    const AxisNode* av = g.ax[V] + p[V];
    float t1 = hv * __ldg(&au->inv_dd);
    float t2 = hu * __ldg(&av->inv_dd);
    if (g.pml > 0) {
        const int su = __ldg(&au->slot_e);
        if (su >= 0) {
            const long long q = g.psi_off[C * 3 + U] + psi_at(g, U, p[0], p[1], p[2], su);
            const float r = __ldg(&au->be) * psi[q] + __ldg(&au->ce) * hv * __ldg(&au->raw_inv_dd);
            psi[q] = r;
            t1 += r;
        }
        const int sv = __ldg(&av->slot_e);
        if (sv >= 0) {
            const long long q = g.psi_off[C * 3 + V] + psi_at(g, V, p[0], p[1], p[2], sv);
            const float r = __ldg(&av->be) * psi[q] + __ldg(&av->ce) * hu * __ldg(&av->raw_inv_dd);
            psi[q] = r;
            t2 += r;
        }
    }
    float& f = e[C * g.cs + id];
    f = cf.ca[C] * f + cb * (t1 - t2);
}

// Grid (ceil(n2/64), ceil(n1/4), n0), block (64, 4). Its first thread opens step n by raising
// the step counter to n + 1; later kernels of the step read n from it.
__global__ void __launch_bounds__(256) k_update_h(Geom g, const float* __restrict__ e, float* __restrict__ h,
                                                  float* __restrict__ psi, float k_mu, unsigned* counter) {
    if ((blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0) *counter += 1u;
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= g.n2 || j >= g.n1) return;
    const int p[3] = {i, j, k};
    const long long st[3] = {(long long)g.n1 * g.p2, g.p2, 1};
    const long long id = ((long long)i * g.n1 + j) * g.p2 + k;
    h_update_one<0>(g, p, id, st, e, h, psi, k_mu);
    h_update_one<1>(g, p, id, st, e, h, psi, k_mu);
    h_update_one<2>(g, p, id, st, e, h, psi, k_mu);
}

template <typename CID>
__global__ void __launch_bounds__(256) k_update_e(Geom g, const CID* __restrict__ node_class,
                                                  const DevCoef* __restrict__ classes, const float* __restrict__ h,
                                                  float* __restrict__ e, float* __restrict__ psi) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y * blockDim.y + threadIdx.y;
    const int i = blockIdx.z;
    if (k >= g.n2 || j >= g.n1) return;
    const int p[3] = {i, j, k};
    const long long st[3] = {(long long)g.n1 * g.p2, g.p2, 1};
    const long long id = ((long long)i * g.n1 + j) * g.p2 + k;
    const DevCoef cf = classes[node_class[id]];
    e_update_one<0>(g, p, id, st, cf, h, e, psi);
    e_update_one<1>(g, p, id, st, cf, h, e, psi);
    e_update_one<2>(g, p, id, st, cf, h, e, psi);
}

}  // namespace fg
