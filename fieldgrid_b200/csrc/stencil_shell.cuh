// The CPML shell of the fused step: every node outside the clean box the TMA march covers (the
// absorbing slabs and a one-node ring inside them), updated out of place by two plain kernels.
// One thread owns one node and its three components; the arithmetic, operation order and guards
// are those of the reference's CPU step (sims-field cpu.rs:48-167), as in the other pipelines:
//   k_shell_h: H_out from E_in, H_in and the input set of H psi slabs (written to the output set);
//   k_shell_e: E_out from E_in and the new H (the clean box's H written by the march, the shell's
//              by k_shell_h), with the E psi slabs updated in place.
// Run order within a step: the march and k_shell_h (independent), then k_shell_e.
#pragma once

#include "kernels.cuh"

namespace fg {

// Up to six boxes [lo, hi) covering the shell; start[q] counts the nodes of boxes before q.
struct ShellBoxes {
    int n;
    int lo[6][3], hi[6][3];
    long long start[7];
};

// The node of shell index t, k fastest inside each box.
__device__ __forceinline__ void shell_node(const ShellBoxes& b, long long t, int p[3]) {
    int q = 0;
    while (q + 1 < b.n && t >= b.start[q + 1]) ++q;
    long long l = t - b.start[q];
    const int w2 = b.hi[q][2] - b.lo[q][2], w1 = b.hi[q][1] - b.lo[q][1];
    p[2] = b.lo[q][2] + int(l % w2);
    l /= w2;
    p[1] = b.lo[q][1] + int(l % w1);
    p[0] = b.lo[q][0] + int(l / w1);
}

// H_c = H_c - k_mu [(dE_v/du) inv_d_u + psi_u - (dE_u/dv) inv_d_v - psi_v]   (cpu.rs:65-102)
template <int C>
__device__ __forceinline__ void h_shell_one(const Geom& g, const int p[3], long long id, const long long st[3],
                                            const float* __restrict__ e, const float* __restrict__ h_in,
                                            float* __restrict__ h_out, const float* __restrict__ psi_in,
                                            float* __restrict__ psi_out, float k_mu) {
    constexpr int U = (C + 1) % 3, V = (C + 2) % 3;
    const int nu = U == 0 ? g.n0 : (U == 1 ? g.n1 : g.n2);
    const int nv = V == 0 ? g.n0 : (V == 1 ? g.n1 : g.n2);
    float hv = h_in[C * g.cs + id];
    if (p[U] + 1 < nu && p[V] + 1 < nv) {
        const float ev = e[V * g.cs + id + st[U]] - e[V * g.cs + id];
        const float eu = e[U * g.cs + id + st[V]] - e[U * g.cs + id];
        const AxisNode* au = g.ax[U] + p[U];
        const AxisNode* av = g.ax[V] + p[V];
        float t1 = ev * __ldg(&au->inv_d);
        float t2 = eu * __ldg(&av->inv_d);
        const int su = __ldg(&au->slot_h);
        if (su >= 0) {
            const long long q = g.psi_off[9 + C * 3 + U] + psi_at(g, U, p[0], p[1], p[2], su);
            const float r = __ldg(&au->bh) * psi_in[q] + __ldg(&au->ch) * ev * __ldg(&au->raw_inv_d);
            psi_out[q] = r;
            t1 += r;
        }
        const int sv = __ldg(&av->slot_h);
        if (sv >= 0) {
            const long long q = g.psi_off[9 + C * 3 + V] + psi_at(g, V, p[0], p[1], p[2], sv);
            const float r = __ldg(&av->bh) * psi_in[q] + __ldg(&av->ch) * eu * __ldg(&av->raw_inv_d);
            psi_out[q] = r;
            t2 += r;
        }
        hv = hv - k_mu * (t1 - t2);
    }
    h_out[C * g.cs + id] = hv;
}

// E_c = ca E_c + cb [(dH_v/du) inv_dd_u + psi_u - (dH_u/dv) inv_dd_v - psi_v], kept where
// cb == 0 (cpu.rs:125-162)
template <int C>
__device__ __forceinline__ void e_shell_one(const Geom& g, const int p[3], long long id, const long long st[3],
                                            const DevCoef& cf, const float* __restrict__ h,
                                            const float* __restrict__ e_in, float* __restrict__ e_out,
                                            float* __restrict__ psi) {
    constexpr int U = (C + 1) % 3, V = (C + 2) % 3;
    const float cb = cf.cb[C];
    float ev = e_in[C * g.cs + id];
    if (cb != 0.0f && p[U] != 0 && p[V] != 0) {
        const float hv = h[V * g.cs + id] - h[V * g.cs + id - st[U]];
        const float hu = h[U * g.cs + id] - h[U * g.cs + id - st[V]];
        const AxisNode* au = g.ax[U] + p[U];
        const AxisNode* av = g.ax[V] + p[V];
        float t1 = hv * __ldg(&au->inv_dd);
        float t2 = hu * __ldg(&av->inv_dd);
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
        ev = cf.ca[C] * ev + cb * (t1 - t2);
    }
    e_out[C * g.cs + id] = ev;
}

constexpr int SHELL_THREADS = 256;

__global__ void __launch_bounds__(SHELL_THREADS) k_shell_h(Geom g, ShellBoxes b, const float* __restrict__ e_in,
                                                           const float* __restrict__ h_in, float* __restrict__ h_out,
                                                           const float* __restrict__ psi_in, float* __restrict__ psi_out,
                                                           float k_mu) {
    const long long t = (long long)blockIdx.x * SHELL_THREADS + threadIdx.x;
    if (t >= b.start[b.n]) return;
    int p[3];
    shell_node(b, t, p);
    const long long st[3] = {(long long)g.n1 * g.p2, g.p2, 1};
    const long long id = ((long long)p[0] * g.n1 + p[1]) * g.p2 + p[2];
    h_shell_one<0>(g, p, id, st, e_in, h_in, h_out, psi_in, psi_out, k_mu);
    h_shell_one<1>(g, p, id, st, e_in, h_in, h_out, psi_in, psi_out, k_mu);
    h_shell_one<2>(g, p, id, st, e_in, h_in, h_out, psi_in, psi_out, k_mu);
}

template <typename CID>
__global__ void __launch_bounds__(SHELL_THREADS) k_shell_e(Geom g, ShellBoxes b, const CID* __restrict__ node_class,
                                                           const DevCoef* __restrict__ classes,
                                                           const float* __restrict__ h, const float* __restrict__ e_in,
                                                           float* __restrict__ e_out, float* __restrict__ psi) {
    const long long t = (long long)blockIdx.x * SHELL_THREADS + threadIdx.x;
    if (t >= b.start[b.n]) return;
    int p[3];
    shell_node(b, t, p);
    const long long st[3] = {(long long)g.n1 * g.p2, g.p2, 1};
    const long long id = ((long long)p[0] * g.n1 + p[1]) * g.p2 + p[2];
    const DevCoef cf = classes[node_class[id]];
    e_shell_one<0>(g, p, id, st, cf, h, e_in, e_out, psi);
    e_shell_one<1>(g, p, id, st, cf, h, e_in, e_out, psi);
    e_shell_one<2>(g, p, id, st, cf, h, e_in, e_out, psi);
}

}  // namespace fg
