// The fused E+H step: one kernel reads (E, H) of step n and writes (E, H) of step n+1.
//
// A block owns a TJ x TK tile of (j, k) columns and marches along x (i) over SEG planes. Per plane
// every thread forms the new H of its node (3 components, CPML psi included), stores it to the
// output buffer and to a shared-memory tile; the H the tile's E update needs from the neighbours
// at j-1 and k-1 is recomputed from the inputs (read-only, no psi write), and the H of plane i-1
// stays in registers from the previous iteration. After one barrier every thread forms the new E
// of its node from the tile. E, H and the H psi slabs ping-pong between two buffer sets, so a
// block never reads what another block writes in the same launch; the E psi slabs are updated in
// place by their owner only.
//
// Per node and step this reads E and H once and writes them once (48 B), plus one class id
// (1 or 2 B) and the psi slabs inside the CPML. It is the reference's fused_step
// (fdtd.wgsl:186-330, run.rs:616-637) re-thought for the B200: one barrier per plane with a
// double-buffered tile, psi ping-pong only where halos read it, and a coefficient class per node.
#pragma once

#include <string>

#include "kernels.cuh"

namespace fg {

struct FusedShape {
    int tk = 32, tj = 8, seg = 32;
};

struct FusedArgs {
    Geom g;
    const void* node_class;
    const DevCoef* classes;
    const float* __restrict__ e_in;
    const float* __restrict__ h_in;
    float* __restrict__ e_out;
    float* __restrict__ h_out;
    float* __restrict__ psi_e;        // base of all slabs; E slabs updated in place
    const float* __restrict__ psi_h_in;   // base pointers such that + psi_off[9 + ...] is the H slab
    float* __restrict__ psi_h_out;
    float k_mu;
    unsigned* counter;
};

template <int A>
__device__ __forceinline__ int dim_of(const Geom& g) { return A == 0 ? g.n0 : (A == 1 ? g.n1 : g.n2); }

template <int A>
__device__ __forceinline__ long long stride_of(const Geom& g) {
    return A == 0 ? (long long)g.n1 * g.p2 : (A == 1 ? (long long)g.p2 : 1ll);
}

// New H_C at node (i, j, k) from the step's inputs (cpu.rs:65-102). `own` nodes also write psi.
template <int C>
__device__ __forceinline__ float h_new(const FusedArgs& a, int i, int j, int k, bool own) {
    constexpr int U = (C + 1) % 3, V = (C + 2) % 3;
    const Geom& g = a.g;
    const int p[3] = {i, j, k};
    const long long id = ((long long)i * g.n1 + j) * g.p2 + k;
    const float hin = a.h_in[C * g.cs + id];
    if (p[U] + 1 >= dim_of<U>(g) || p[V] + 1 >= dim_of<V>(g)) return hin;
    const float e_v = a.e_in[V * g.cs + id];
    const float e_u = a.e_in[U * g.cs + id];
    const float ev = a.e_in[V * g.cs + id + stride_of<U>(g)] - e_v;
    const float eu = a.e_in[U * g.cs + id + stride_of<V>(g)] - e_u;
    const AxisNode* au = g.ax[U] + p[U];
    const AxisNode* av = g.ax[V] + p[V];
    float t1 = ev * __ldg(&au->inv_d);
    float t2 = eu * __ldg(&av->inv_d);
    if (g.pml > 0) {
        const int su = __ldg(&au->slot_h);
        if (su >= 0) {
            const long long q = g.psi_off[9 + C * 3 + U] + psi_at(g, U, i, j, k, su);
            const float r = __ldg(&au->bh) * a.psi_h_in[q] + __ldg(&au->ch) * ev * __ldg(&au->raw_inv_d);
            if (own) a.psi_h_out[q] = r;
            t1 += r;
        }
        const int sv = __ldg(&av->slot_h);
        if (sv >= 0) {
            const long long q = g.psi_off[9 + C * 3 + V] + psi_at(g, V, i, j, k, sv);
            const float r = __ldg(&av->bh) * a.psi_h_in[q] + __ldg(&av->ch) * eu * __ldg(&av->raw_inv_d);
            if (own) a.psi_h_out[q] = r;
            t2 += r;
        }
    }
    return hin - a.k_mu * (t1 - t2);
}

// New E_C at an owned node from the H differences hv (along U) and hu (along V) (cpu.rs:125-162).
template <int C>
__device__ __forceinline__ float e_new(const FusedArgs& a, const int p[3], float e_own, float ca, float cb, float hv,
                                       float hu) {
    constexpr int U = (C + 1) % 3, V = (C + 2) % 3;
    if (cb == 0.0f || p[U] == 0 || p[V] == 0) return e_own;
    const Geom& g = a.g;
    const AxisNode* au = g.ax[U] + p[U];
    const AxisNode* av = g.ax[V] + p[V];
    float t1 = hv * __ldg(&au->inv_dd);
    float t2 = hu * __ldg(&av->inv_dd);
    if (g.pml > 0) {
        const int su = __ldg(&au->slot_e);
        if (su >= 0) {
            const long long q = g.psi_off[C * 3 + U] + psi_at(g, U, p[0], p[1], p[2], su);
            const float r = __ldg(&au->be) * a.psi_e[q] + __ldg(&au->ce) * hv * __ldg(&au->raw_inv_dd);
            a.psi_e[q] = r;
            t1 += r;
        }
        const int sv = __ldg(&av->slot_e);
        if (sv >= 0) {
            const long long q = g.psi_off[C * 3 + V] + psi_at(g, V, p[0], p[1], p[2], sv);
            const float r = __ldg(&av->be) * a.psi_e[q] + __ldg(&av->ce) * hu * __ldg(&av->raw_inv_dd);
            a.psi_e[q] = r;
            t2 += r;
        }
    }
    return ca * e_own + cb * (t1 - t2);
}

// One tile (bx, by) of TJ x TK columns over planes [i0, i1): the block's whole march. The block
// is (TK, TJ) threads; `hs` is its double-buffered H tile.
template <typename CID, int TK, int TJ>
__device__ __forceinline__ void fused_tile(const FusedArgs& a, float (&hs)[2][3][TJ + 1][TK + 1], int bx, int by, int i0,
                                           int i1) {
    const Geom& g = a.g;
    const int lk = threadIdx.x, lj = threadIdx.y;
    const int k = bx * TK + lk;
    const int j = by * TJ + lj;
    const bool live = k < g.n2 && j < g.n1;
    const CID* cls = static_cast<const CID*>(a.node_class);
    float prev_y = 0.0f, prev_z = 0.0f;
    if (live && i0 > 0) {
        prev_y = h_new<1>(a, i0 - 1, j, k, false);
        prev_z = h_new<2>(a, i0 - 1, j, k, false);
    }
    const int halo_j = by * TJ + lk;  // row served by the k-1 halo lanes
    for (int i = i0; i < i1; ++i) {
        const int o = i & 1;
        float hx = 0.f, hy = 0.f, hz = 0.f;
        if (live) {
            const long long id = ((long long)i * g.n1 + j) * g.p2 + k;
            hx = h_new<0>(a, i, j, k, true);
            hy = h_new<1>(a, i, j, k, true);
            hz = h_new<2>(a, i, j, k, true);
            a.h_out[id] = hx;
            a.h_out[g.cs + id] = hy;
            a.h_out[2 * g.cs + id] = hz;
            hs[o][0][lj + 1][lk + 1] = hx;
            hs[o][1][lj + 1][lk + 1] = hy;
            hs[o][2][lj + 1][lk + 1] = hz;
            if (lj == 0 && j > 0) {
                hs[o][0][0][lk + 1] = h_new<0>(a, i, j - 1, k, false);
                hs[o][2][0][lk + 1] = h_new<2>(a, i, j - 1, k, false);
            }
        }
        if (lj == 1 % TJ && lk < TJ && halo_j < g.n1 && bx > 0) {
            const int ck = bx * TK - 1;
            hs[o][0][lk + 1][0] = h_new<0>(a, i, halo_j, ck, false);
            hs[o][1][lk + 1][0] = h_new<1>(a, i, halo_j, ck, false);
        }
        __syncthreads();
        if (live) {
            const long long id = ((long long)i * g.n1 + j) * g.p2 + k;
            const int p[3] = {i, j, k};
            const DevCoef cf = a.classes[cls[id]];
            const float hx_j = hs[o][0][lj][lk + 1];
            const float hz_j = hs[o][2][lj][lk + 1];
            const float hx_k = hs[o][0][lj + 1][lk];
            const float hy_k = hs[o][1][lj + 1][lk];
            const float ex = a.e_in[id], ey = a.e_in[g.cs + id], ez = a.e_in[2 * g.cs + id];
            a.e_out[id] = e_new<0>(a, p, ex, cf.ca[0], cf.cb[0], hz - hz_j, hy - hy_k);
            a.e_out[g.cs + id] = e_new<1>(a, p, ey, cf.ca[1], cf.cb[1], hx - hx_k, hz - prev_z);
            a.e_out[2 * g.cs + id] = e_new<2>(a, p, ez, cf.ca[2], cf.cb[2], hy - prev_y, hx - hx_j);
            prev_y = hy;
            prev_z = hz;
        }
    }
}

template <typename CID, int TK, int TJ>
__global__ void __launch_bounds__(TK* TJ) k_fused_step(FusedArgs a, int seg) {
    __shared__ float hs[2][3][TJ + 1][TK + 1];
    if ((blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0) *a.counter += 1u;
    const int i0 = blockIdx.z * seg;
    fused_tile<CID, TK, TJ>(a, hs, blockIdx.x, blockIdx.y, i0, min(i0 + seg, a.g.n0));
}

// The fused step over the tiles that cover a box of nodes only: tiles (bx0 + x, by0 + y), planes
// [i_lo, i_hi) in segments of `seg`. Nodes outside the box keep whatever the output buffers held
// (the caller reads only nodes whose inputs the box kept correct: a dependency cone).
template <typename CID, int TK, int TJ>
__global__ void __launch_bounds__(TK* TJ) k_fused_box(FusedArgs a, int seg, int bx0, int by0, int i_lo, int i_hi) {
    __shared__ float hs[2][3][TJ + 1][TK + 1];
    if ((blockIdx.x | blockIdx.y | blockIdx.z | threadIdx.x | threadIdx.y) == 0) *a.counter += 1u;
    const int i0 = i_lo + int(blockIdx.z) * seg;
    fused_tile<CID, TK, TJ>(a, hs, bx0 + int(blockIdx.x), by0 + int(blockIdx.y), i0, min(i0 + seg, i_hi));
}

inline FusedShape choose_shape(const Geom& g, int /*cid_bytes*/, bool /*wires*/) {
    FusedShape s;
    s.tk = 32;
    s.tj = 8;
    // enough x-segments for several waves of blocks on 148 SMs, at most 64 planes each
    long long tiles = (long long)((g.n2 + s.tk - 1) / s.tk) * ((g.n1 + s.tj - 1) / s.tj);
    int seg = 64;
    while (seg > 8 && tiles * ((g.n0 + seg - 1) / seg) < 148 * 8) seg /= 2;
    s.seg = seg;
    return s;
}

inline std::string fused_name(const FusedShape& s) {
    return "fused march, tile " + std::to_string(s.tj) + "x" + std::to_string(s.tk) + ", " + std::to_string(s.seg) +
           " planes per block";
}

inline int launch_fused(const FusedShape& s, int cid_bytes, const Geom& g, const void* node_class, const DevCoef* classes,
                        const float* e_in, const float* h_in, float* e_out, float* h_out, float* psi_e,
                        const float* psi_h_in, float* psi_h_out, float k_mu, unsigned* counter, bool /*wires*/,
                        cudaStream_t st) {
    FusedArgs a{g, node_class, classes, e_in, h_in, e_out, h_out, psi_e, psi_h_in, psi_h_out, k_mu, counter};
    constexpr int TK = 32, TJ = 8;
    dim3 blk(TK, TJ, 1);
    dim3 grd((g.n2 + TK - 1) / TK, (g.n1 + TJ - 1) / TJ, (g.n0 + s.seg - 1) / s.seg);
    switch (cid_bytes) {
        case 1: k_fused_step<uint8_t, TK, TJ><<<grd, blk, 0, st>>>(a, s.seg); break;
        case 2: k_fused_step<uint16_t, TK, TJ><<<grd, blk, 0, st>>>(a, s.seg); break;
        default: k_fused_step<uint32_t, TK, TJ><<<grd, blk, 0, st>>>(a, s.seg); break;
    }
    return cudaPeekAtLastError() == cudaSuccess ? 0 : 1;
}

// launch_fused over the box of nodes [lo, hi) (each lo < hi, inside the grid).
inline int launch_fused_box(int cid_bytes, const Geom& g, const void* node_class, const DevCoef* classes,
                            const float* e_in, const float* h_in, float* e_out, float* h_out, float* psi_e,
                            const float* psi_h_in, float* psi_h_out, float k_mu, unsigned* counter, const int lo[3],
                            const int hi[3], cudaStream_t st) {
    FusedArgs a{g, node_class, classes, e_in, h_in, e_out, h_out, psi_e, psi_h_in, psi_h_out, k_mu, counter};
    constexpr int TK = 32, TJ = 8;
    const int bx0 = lo[2] / TK, bx1 = (hi[2] + TK - 1) / TK, by0 = lo[1] / TJ, by1 = (hi[1] + TJ - 1) / TJ;
    const int planes = hi[0] - lo[0];
    const long long tiles = (long long)(bx1 - bx0) * (by1 - by0);
    // x-segments for several waves of blocks on 148 SMs, 2 to 64 planes: a small box runs short
    // segments, since a block's march is a chain of per-plane latencies
    int seg = 64;
    while (seg > 2 && tiles * ((planes + seg - 1) / seg) < 148 * 8) seg /= 2;
    dim3 blk(TK, TJ, 1);
    dim3 grd(unsigned(bx1 - bx0), unsigned(by1 - by0), unsigned((planes + seg - 1) / seg));
    switch (cid_bytes) {
        case 1: k_fused_box<uint8_t, TK, TJ><<<grd, blk, 0, st>>>(a, seg, bx0, by0, lo[0], hi[0]); break;
        case 2: k_fused_box<uint16_t, TK, TJ><<<grd, blk, 0, st>>>(a, seg, bx0, by0, lo[0], hi[0]); break;
        default: k_fused_box<uint32_t, TK, TJ><<<grd, blk, 0, st>>>(a, seg, bx0, by0, lo[0], hi[0]); break;
    }
    return cudaPeekAtLastError() == cudaSuccess ? 0 : 1;
}

}  // namespace fg
