// The CPML shell of the fused step: every node outside the clean box the TMA march covers (the
// absorbing slabs and a one-node ring inside them), updated out of place by two plain kernels.
// One warp walks one row of shell nodes along k, a lane owning a node and its three components;
// the arithmetic, operation order and guards are those of the reference's CPU step (sims-field
// cpu.rs:48-167), as in the other pipelines:
//   k_shell_h: H_out from E_in, H_in and the input set of H psi slabs (written to the output set);
//   k_shell_e: E_out from E_in and the new H (the clean box's H written by the march, the shell's
//              by k_shell_h), with the E psi slabs along x and y updated in place.
// The z slabs (derivative along k) are read from pz_in and written to pz_out, which are the psi
// arrays themselves (in place for E, the two H sets) or, when the step keeps its z-slab psi in
// time slots, the slot of the step's input and the slot of its output.
// Run order within a step: the march and k_shell_h (independent), then k_shell_e.
#pragma once

#include "kernels.cuh"

namespace fg {

// The shell as rows of nodes along k, one warp per row:
//   A: planes [0, xa) and [xb, n0), every row j, every column;
//   B: planes [xa, xb), rows [0, ya) and [yb, n1), every column;
//   C: planes [xa, xb), rows [ya, yb), the two strips of columns [0, za) and [zb, n2).
struct ShellRows {
    int xa, xb, ya, yb, za, zb;
    unsigned ra, rb, rc;      // rows in A, B, C
};

// Row r's (i, j); `strips` when the row covers only the two k strips.
__device__ __forceinline__ void shell_row(const Geom& g, const ShellRows& b, unsigned r, int& i, int& j, bool& strips) {
    if (r < b.ra) {
        const unsigned pi = r / unsigned(g.n1);
        j = int(r - pi * unsigned(g.n1));
        i = int(pi) < b.xa ? int(pi) : b.xb + (int(pi) - b.xa);
        strips = false;
    } else if (r < b.ra + b.rb) {
        r -= b.ra;
        const unsigned ny = unsigned(b.ya + g.n1 - b.yb);
        const unsigned pi = r / ny, jj = r - pi * ny;
        i = b.xa + int(pi);
        j = int(jj) < b.ya ? int(jj) : b.yb + (int(jj) - b.ya);
        strips = false;
    } else {
        r -= b.ra + b.rb;
        const unsigned ny = unsigned(b.yb - b.ya);
        const unsigned pi = r / ny;
        i = b.xa + int(pi);
        j = b.ya + int(r - pi * ny);
        strips = true;
    }
}

// The k axis's factors as separate arrays of n2 entries: a warp walking a row along k reads each
// as one coalesced line (an AxisNode per lane would be a 40-byte-stride gather per field).
struct KAxis {
    const float *inv_d, *inv_dd, *raw_inv_d, *raw_inv_dd, *be, *ce, *bh, *ch;
    const int *slot_e, *slot_h;
};

// The factors of node k that an H (F = 1) or E (F = 0) update reads; the CPML ones only inside
// the layer.
struct KNode {
    float inv, raw, b, c;
    int slot;
};

template <int F>
__device__ __forceinline__ KNode k_node(const KAxis& kx, int k) {
    KNode n;
    n.inv = F ? kx.inv_d[k] : kx.inv_dd[k];
    n.slot = F ? kx.slot_h[k] : kx.slot_e[k];
    n.raw = n.b = n.c = 0.f;
    if (n.slot >= 0) {
        n.raw = F ? kx.raw_inv_d[k] : kx.raw_inv_dd[k];
        n.b = F ? kx.bh[k] : kx.be[k];
        n.c = F ? kx.ch[k] : kx.ce[k];
    }
    return n;
}

// One CPML term, r = b psi + c d raw (cpu.rs:73-99, :135-159), in the reference's operation order.
__device__ __forceinline__ float cpml_term(float b, float psi, float c, float d, float raw) { return b * psi + c * d * raw; }

constexpr int SHELL_THREADS = 256;   // 8 rows per block
// k_shell_h is held to 64 registers (4 blocks per SM, 32 warps: a few bytes spill) for more loads in
// flight: 10 % faster at 512^3 than at its natural 80 registers (3 blocks); k_shell_e at 64 was 3 %
// slower and keeps its 80.

// The new H of one row of shell nodes (cpu.rs:48-107): H_c = H_c - k_mu [(dE_v/du) inv_d_u + psi_u
// - (dE_u/dv) inv_d_v - psi_v], each psi_a updated where the node's slot along a is live. All loads
// of a node come before its stores.
__device__ __forceinline__ void shell_h_row(const Geom& g, const ShellRows& b, const KAxis& kx, unsigned r,
                                            const float* __restrict__ e_in, const float* __restrict__ h_in,
                                            float* __restrict__ h_out, const float* __restrict__ psi_in,
                                            float* __restrict__ psi_out, const float* __restrict__ pz_in,
                                            float* __restrict__ pz_out, float k_mu) {
    if (r >= b.ra + b.rb + b.rc) return;
    int i, j;
    bool strips;
    shell_row(g, b, r, i, j, strips);
    const int len = strips ? b.za + (g.n2 - b.zb) : g.n2;
    const AxisNode ai = g.ax[0][i], aj = g.ax[1][j];     // uniform over the warp
    const bool in_i = i + 1 < g.n0, in_j = j + 1 < g.n1;
    const long long cs = g.cs;
    const long long row = ((long long)i * g.n1 + j) * g.p2;
    const long long si = (long long)g.n1 * g.p2, sj = g.p2;
    // psi offsets of this row in the x and y slabs (psi_idx, sim.rs:659-665); the z slab per node
    const long long px = ai.slot_h >= 0 ? ((long long)ai.slot_h * g.n1 + j) * g.n2 : 0;
    const long long py = aj.slot_h >= 0 ? ((long long)i * (2 * g.pml) + aj.slot_h) * g.n2 : 0;
    const long long pz = ((long long)i * g.n1 + j) * g.pw;
    for (int q = int(threadIdx.x & 31); q < len; q += 32) {
        const int k = strips && q >= b.za ? b.zb + (q - b.za) : q;
        const KNode ak = k_node<1>(kx, k);
        const bool in_k = k + 1 < g.n2;
        const long long id = row + k;
        const bool run0 = in_j && in_k, run1 = in_k && in_i, run2 = in_i && in_j;
        const float ex = e_in[id], ey = e_in[cs + id], ez = e_in[2 * cs + id];
        const float ez_j = in_j ? e_in[2 * cs + id + sj] : 0.f, ex_j = in_j ? e_in[id + sj] : 0.f;
        const float ey_k = in_k ? e_in[cs + id + 1] : 0.f, ex_k = in_k ? e_in[id + 1] : 0.f;
        const float ez_i = in_i ? e_in[2 * cs + id + si] : 0.f, ey_i = in_i ? e_in[cs + id + si] : 0.f;
        float hx = h_in[id], hy = h_in[cs + id], hz = h_in[2 * cs + id];
        // psi of the input set, by (component, axis): Hx (j, k), Hy (k, i), Hz (i, j)
        const long long o0j = g.psi_off[9 + 0 * 3 + 1] + py + k, o0k = g.psi_off[9 + 0 * 3 + 2] + pz + ak.slot;
        const long long o1k = g.psi_off[9 + 1 * 3 + 2] + pz + ak.slot, o1i = g.psi_off[9 + 1 * 3 + 0] + px + k;
        const long long o2i = g.psi_off[9 + 2 * 3 + 0] + px + k, o2j = g.psi_off[9 + 2 * 3 + 1] + py + k;
        const bool lj = aj.slot_h >= 0, lk = ak.slot >= 0, li = ai.slot_h >= 0;
        const float s0j = run0 && lj ? psi_in[o0j] : 0.f, s0k = run0 && lk ? pz_in[o0k] : 0.f;
        const float s1k = run1 && lk ? pz_in[o1k] : 0.f, s1i = run1 && li ? psi_in[o1i] : 0.f;
        const float s2i = run2 && li ? psi_in[o2i] : 0.f, s2j = run2 && lj ? psi_in[o2j] : 0.f;
        if (run0) {   // Hx: U = j, V = k
            const float ev = ez_j - ez, eu = ey_k - ey;
            float t1 = ev * aj.inv_d, t2 = eu * ak.inv;
            if (lj) { const float rr = cpml_term(aj.bh, s0j, aj.ch, ev, aj.raw_inv_d); psi_out[o0j] = rr; t1 += rr; }
            if (lk) { const float rr = cpml_term(ak.b, s0k, ak.c, eu, ak.raw); pz_out[o0k] = rr; t2 += rr; }
            hx = hx - k_mu * (t1 - t2);
        }
        if (run1) {   // Hy: U = k, V = i
            const float ev = ex_k - ex, eu = ez_i - ez;
            float t1 = ev * ak.inv, t2 = eu * ai.inv_d;
            if (lk) { const float rr = cpml_term(ak.b, s1k, ak.c, ev, ak.raw); pz_out[o1k] = rr; t1 += rr; }
            if (li) { const float rr = cpml_term(ai.bh, s1i, ai.ch, eu, ai.raw_inv_d); psi_out[o1i] = rr; t2 += rr; }
            hy = hy - k_mu * (t1 - t2);
        }
        if (run2) {   // Hz: U = i, V = j
            const float ev = ey_i - ey, eu = ex_j - ex;
            float t1 = ev * ai.inv_d, t2 = eu * aj.inv_d;
            if (li) { const float rr = cpml_term(ai.bh, s2i, ai.ch, ev, ai.raw_inv_d); psi_out[o2i] = rr; t1 += rr; }
            if (lj) { const float rr = cpml_term(aj.bh, s2j, aj.ch, eu, aj.raw_inv_d); psi_out[o2j] = rr; t2 += rr; }
            hz = hz - k_mu * (t1 - t2);
        }
        h_out[id] = hx;
        h_out[cs + id] = hy;
        h_out[2 * cs + id] = hz;
    }
}

// The new E of one row of shell nodes (cpu.rs:109-167): E_c = ca E_c + cb [(dH_v/du) inv_dd_u +
// psi_u - (dH_u/dv) inv_dd_v - psi_v], kept where cb == 0; the E psi slabs are updated in place,
// so every psi read of a node precedes its writes.
template <typename CID>
__device__ __forceinline__ void shell_e_row(const Geom& g, const ShellRows& b, const KAxis& kx, unsigned r,
                                            const CID* __restrict__ node_class, const DevCoef* __restrict__ classes,
                                            const float* __restrict__ h, const float* __restrict__ e_in,
                                            float* __restrict__ e_out, float* __restrict__ psi, const float* pz_in,
                                            float* pz_out) {
    if (r >= b.ra + b.rb + b.rc) return;
    int i, j;
    bool strips;
    shell_row(g, b, r, i, j, strips);
    const int len = strips ? b.za + (g.n2 - b.zb) : g.n2;
    const AxisNode ai = g.ax[0][i], aj = g.ax[1][j];
    const long long cs = g.cs;
    const long long row = ((long long)i * g.n1 + j) * g.p2;
    const long long si = (long long)g.n1 * g.p2, sj = g.p2;
    const long long px = ai.slot_e >= 0 ? ((long long)ai.slot_e * g.n1 + j) * g.n2 : 0;
    const long long py = aj.slot_e >= 0 ? ((long long)i * (2 * g.pml) + aj.slot_e) * g.n2 : 0;
    const long long pz = ((long long)i * g.n1 + j) * g.pw;
    for (int q = int(threadIdx.x & 31); q < len; q += 32) {
        const int k = strips && q >= b.za ? b.zb + (q - b.za) : q;
        const KNode ak = k_node<0>(kx, k);
        const long long id = row + k;
        const DevCoef cf = classes[node_class[id]];
        const bool run0 = cf.cb[0] != 0.0f && j > 0 && k > 0;
        const bool run1 = cf.cb[1] != 0.0f && k > 0 && i > 0;
        const bool run2 = cf.cb[2] != 0.0f && i > 0 && j > 0;
        const float hx = h[id], hy = h[cs + id], hz = h[2 * cs + id];
        const float hz_j = j > 0 ? h[2 * cs + id - sj] : 0.f, hx_j = j > 0 ? h[id - sj] : 0.f;
        const float hy_k = k > 0 ? h[cs + id - 1] : 0.f, hx_k = k > 0 ? h[id - 1] : 0.f;
        const float hz_i = i > 0 ? h[2 * cs + id - si] : 0.f, hy_i = i > 0 ? h[cs + id - si] : 0.f;
        float ex = e_in[id], ey = e_in[cs + id], ez = e_in[2 * cs + id];
        const long long o0j = g.psi_off[0 * 3 + 1] + py + k, o0k = g.psi_off[0 * 3 + 2] + pz + ak.slot;
        const long long o1k = g.psi_off[1 * 3 + 2] + pz + ak.slot, o1i = g.psi_off[1 * 3 + 0] + px + k;
        const long long o2i = g.psi_off[2 * 3 + 0] + px + k, o2j = g.psi_off[2 * 3 + 1] + py + k;
        const bool lj = aj.slot_e >= 0, lk = ak.slot >= 0, li = ai.slot_e >= 0;
        const float s0j = run0 && lj ? psi[o0j] : 0.f, s0k = run0 && lk ? pz_in[o0k] : 0.f;
        const float s1k = run1 && lk ? pz_in[o1k] : 0.f, s1i = run1 && li ? psi[o1i] : 0.f;
        const float s2i = run2 && li ? psi[o2i] : 0.f, s2j = run2 && lj ? psi[o2j] : 0.f;
        if (run0) {   // Ex: U = j, V = k
            const float hv = hz - hz_j, hu = hy - hy_k;
            float t1 = hv * aj.inv_dd, t2 = hu * ak.inv;
            if (lj) { const float rr = cpml_term(aj.be, s0j, aj.ce, hv, aj.raw_inv_dd); psi[o0j] = rr; t1 += rr; }
            if (lk) { const float rr = cpml_term(ak.b, s0k, ak.c, hu, ak.raw); pz_out[o0k] = rr; t2 += rr; }
            ex = cf.ca[0] * ex + cf.cb[0] * (t1 - t2);
        }
        if (run1) {   // Ey: U = k, V = i
            const float hv = hx - hx_k, hu = hz - hz_i;
            float t1 = hv * ak.inv, t2 = hu * ai.inv_dd;
            if (lk) { const float rr = cpml_term(ak.b, s1k, ak.c, hv, ak.raw); pz_out[o1k] = rr; t1 += rr; }
            if (li) { const float rr = cpml_term(ai.be, s1i, ai.ce, hu, ai.raw_inv_dd); psi[o1i] = rr; t2 += rr; }
            ey = cf.ca[1] * ey + cf.cb[1] * (t1 - t2);
        }
        if (run2) {   // Ez: U = i, V = j
            const float hv = hy - hy_i, hu = hx - hx_j;
            float t1 = hv * ai.inv_dd, t2 = hu * aj.inv_dd;
            if (li) { const float rr = cpml_term(ai.be, s2i, ai.ce, hv, ai.raw_inv_dd); psi[o2i] = rr; t1 += rr; }
            if (lj) { const float rr = cpml_term(aj.be, s2j, aj.ce, hu, aj.raw_inv_dd); psi[o2j] = rr; t2 += rr; }
            ez = cf.ca[2] * ez + cf.cb[2] * (t1 - t2);
        }
        e_out[id] = ex;
        e_out[cs + id] = ey;
        e_out[2 * cs + id] = ez;
    }
}

__global__ void __launch_bounds__(SHELL_THREADS, 4) k_shell_h(Geom g, ShellRows b, KAxis kx, const float* __restrict__ e_in,
                                                           const float* __restrict__ h_in, float* __restrict__ h_out,
                                                           const float* __restrict__ psi_in, float* __restrict__ psi_out,
                                                           const float* __restrict__ pz_in, float* __restrict__ pz_out,
                                                           float k_mu) {
    shell_h_row(g, b, kx, blockIdx.x * (SHELL_THREADS / 32) + (threadIdx.x >> 5), e_in, h_in, h_out, psi_in, psi_out,
                pz_in, pz_out, k_mu);
}

// k_shell_h in blocks of four rows (128 threads, 64 registers): the launch that runs beside the
// march in a captured step, one block of it fitting on an SM next to two march blocks (2 x 288
// threads x 96 registers + 128 x 64 of the 65,536), so the shell's latency-bound row walks fill
// the march's idle issue slots instead of following it.
constexpr int SHELL_SIDE_THREADS = 128;
__global__ void __launch_bounds__(SHELL_SIDE_THREADS, 8) k_shell_h_side(Geom g, ShellRows b, KAxis kx,
                                                                  const float* __restrict__ e_in,
                                                                  const float* __restrict__ h_in,
                                                                  float* __restrict__ h_out,
                                                                  const float* __restrict__ psi_in,
                                                                  float* __restrict__ psi_out,
                                                                  const float* __restrict__ pz_in,
                                                                  float* __restrict__ pz_out, float k_mu) {
    shell_h_row(g, b, kx, blockIdx.x * (SHELL_SIDE_THREADS / 32) + (threadIdx.x >> 5), e_in, h_in, h_out, psi_in,
                psi_out, pz_in, pz_out, k_mu);
}

template <typename CID>
__global__ void __launch_bounds__(SHELL_THREADS) k_shell_e(Geom g, ShellRows b, KAxis kx, const CID* __restrict__ node_class,
                                                           const DevCoef* __restrict__ classes,
                                                           const float* __restrict__ h, const float* __restrict__ e_in,
                                                           float* __restrict__ e_out, float* __restrict__ psi,
                                                           const float* pz_in, float* pz_out) {
    shell_e_row<CID>(g, b, kx, blockIdx.x * (SHELL_THREADS / 32) + (threadIdx.x >> 5), node_class, classes, h, e_in,
                     e_out, psi, pz_in, pz_out);
}

// One grid's shell in a merged batch launch: its geometry, rows and buffers per input set (the
// pointers of the single-grid launches in the fused step of that parity), and its first block.
struct ShellGrid {
    Geom g;
    ShellRows b;
    KAxis kx;
    const void* node_class;
    const DevCoef* classes;
    const float* e_in[2];
    const float* h_in[2];
    float* e_out[2];
    float* h_out[2];
    const float* psi_h_in[2];
    float* psi_h_out[2];
    float* psi;
    float k_mu;
    int block0;
};

// The shells of many grids in one launch (k_shell_h / k_shell_e per grid): block b walks rows of
// grid block_grid[b].
__global__ void __launch_bounds__(SHELL_THREADS, 4) k_batch_shell_h(const ShellGrid* __restrict__ grids,
                                                                 const int* __restrict__ block_grid, int parity) {
    const ShellGrid& G = grids[block_grid[blockIdx.x]];
    const unsigned r = unsigned(int(blockIdx.x) - G.block0) * (SHELL_THREADS / 32) + (threadIdx.x >> 5);
    shell_h_row(G.g, G.b, G.kx, r, G.e_in[parity], G.h_in[parity], G.h_out[parity], G.psi_h_in[parity],
                G.psi_h_out[parity], G.psi_h_in[parity], G.psi_h_out[parity], G.k_mu);
}

template <typename CID>
__global__ void __launch_bounds__(SHELL_THREADS) k_batch_shell_e(const ShellGrid* __restrict__ grids,
                                                              const int* __restrict__ block_grid, int parity) {
    const ShellGrid& G = grids[block_grid[blockIdx.x]];
    const unsigned r = unsigned(int(blockIdx.x) - G.block0) * (SHELL_THREADS / 32) + (threadIdx.x >> 5);
    shell_e_row<CID>(G.g, G.b, G.kx, r, static_cast<const CID*>(G.node_class), G.classes, G.h_out[parity],
                     G.e_in[parity], G.e_out[parity], G.psi, G.psi, G.psi);
}

}  // namespace fg
