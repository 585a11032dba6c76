// The fused E+H step fed by the Tensor Memory Accelerator: the engine's main stencil on the B200.
//
// A block owns a TJ x TK tile of (j, k) columns and marches along x over a segment of planes.
// One producer warp streams, per plane p, three boxes into a ring of shared-memory stages with
// cp.async.bulk.tensor (4-D maps over (k, j, i, component)):
//   E(p)     rows j0-1 .. j0+TJ,   columns k0-4 .. k0+TK+3 (all 3 components)
//   H_in(p)  rows j0-1 .. j0+TJ-1, columns k0-4 .. k0+TK-1 (all 3 components)
//   class(p) rows j0   .. j0+TJ-1, columns k0   .. k0+TK-1 (the node class ids)
// Box origins in k are rounded down to 16 bytes; rows or planes outside the grid arrive as zeros.
// Eight consumer warps then, per plane i:
//   1. form the new H on the tile and on its j-1 row and k-1 column (the halo the E update needs;
//      halo points are recomputed, read-only) from the E(i), E(i+1) and H_in(i) boxes, into a
//      triple-buffered H tile; owned points go to the output buffer;
//   2. after one barrier, form the new E of the tile from the H tile of plane i and of plane i-1.
// Each node's E and H are read from DRAM once and written once per step (48 B) plus its class id;
// the halo reads hit L2. The CPML psi recursions run only on tiles/planes inside the absorbing
// layer (a block-uniform test), with the E slabs in place and the H slabs ping-ponged like the
// fields. Mbarrier waits are bounded by the global timer: a wait that runs out raises the error
// word and the block leaves without starting new work.
#pragma once

#include <cuda.h>

#include <string>

#include "kernels.cuh"

namespace fg {

namespace tma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits for the phase of the given parity to complete; false after `limit_ns` without it.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint64_t limit_ns) {
    if (mbar_try_wait(bar, parity)) return true;
    const uint64_t t0 = global_ns();
    while (!mbar_try_wait(bar, parity))
        if (global_ns() - t0 > limit_ns) return false;
    return true;
}

__device__ __forceinline__ void load_4d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z, int w) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5, %6}], [%2];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z), "r"(w)
        : "memory");
}

__device__ __forceinline__ void load_3d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y, int z) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%3, %4, %5}], [%2];" ::"r"(smem_u32(dst)),
        "l"(map), "r"(smem_u32(bar)), "r"(x), "r"(y), "r"(z)
        : "memory");
}

// Consumer-only barrier (named barrier 1) that also ORs a flag across the consumers.
__device__ __forceinline__ bool consumers_sync_or(bool flag, int count) {
    int out;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.s32 p, %1, 0;\n\t"
        "barrier.cta.red.or.pred q, 1, %2, p;\n\t"
        "selp.s32 %0, 1, 0, q;\n\t}"
        : "=r"(out)
        : "r"(int(flag)), "r"(count)
        : "memory");
    return out != 0;
}

constexpr uint64_t WAIT_LIMIT_NS = 2000000000ull;  // 2 s: far beyond any legitimate copy

}  // namespace tma

// Shared-memory layout of one block (tile TJ x TK, TJ + 1 consumer warps' worth of rows).
// With LOCAL, class ids are 8-bit indices into a per-block table of at most LOCAL_CLASSES
// (ca[3], cb[3]) records that the block keeps in shared memory.
constexpr int LOCAL_CLASSES = 256;

template <int TJ, int TK, typename CID, int STAGES, int SEGMAX, bool LOCAL = false, bool PML = true>
struct TmaLayout {
    static constexpr int EW = TK + 8, ER = TJ + 2;   // E box: columns k0-4 .. k0+TK+3, rows j0-1 .. j0+TJ
    static constexpr int HW = TK + 8, HR = TJ + 1;   // H box: columns k0-4 .. k0+TK+3, rows j0-1 .. j0+TJ-1
    static constexpr int CW = TK + 16, CR = TJ;      // class box: columns k0 .. k0+TK+15, rows j0 .. j0+TJ-1
    static constexpr int NW = TK + 4, NR = TJ + 1;   // new-H tile: column k at k-k0+2, row j at j-j0+1
    static constexpr int E_BYTES = 3 * ER * EW * 4;
    static constexpr int H_BYTES = 3 * HR * HW * 4;
    static constexpr int C_BYTES = CR * CW * int(sizeof(CID));
    __host__ __device__ static constexpr int al(int b) { return (b + 127) & ~127; }
    // staged z-slab psi (tiles that reach the k layer): per field a box of 2 components x
    // (TJ + 1) rows (j0-1 .. j0+TJ-1) x pw slots, pw <= PZW
    static constexpr int PZW = 32;
    static constexpr int PZ_FIELD = 2 * (TJ + 1) * PZW * 4;
    static constexpr int PZ_OFF = al(E_BYTES) + al(H_BYTES) + al(C_BYTES);
    static constexpr int STAGE = PZ_OFF + (PML ? 2 * PZ_FIELD : 0);
    static constexpr int TX = E_BYTES + H_BYTES + C_BYTES;  // bytes one stage's field copies deliver
    static constexpr int HN = al(3 * NR * NW * 4);
    static constexpr int NAX = (TJ + 2) + (TK + 4) + (SEGMAX + 2);
    static constexpr int AX = al(NAX * int(sizeof(AxisNode)));
    static constexpr int BARS = al(2 * STAGES * 8);
    static constexpr int LT = LOCAL ? al(LOCAL_CLASSES * 6 * 4) : 0;  // the block's coefficient table
    static constexpr int TOTAL = STAGES * STAGE + 2 * HN + AX + BARS + LT + 128;
};

struct TmaArgs {
    Geom g;
    const DevCoef* classes;
    float* __restrict__ e_out;
    float* __restrict__ h_out;
    float* __restrict__ psi_e;           // E slabs, in place
    const float* __restrict__ psi_h_in;  // H slabs of the step's input set
    float* __restrict__ psi_h_out;
    float k_mu;
    int pz;                              // the z-slab psi boxes are staged (pml > 0, pw <= PZW)
    const int4* blocks;                  // per block: (k0, j0, i0, i1) of its tile and x-segment
    int block0;                          // this launch's first entry of `blocks`
    int bump;                            // this launch raises the step counter (the step's first kernel)
    const float* tables;                 // LOCAL: per block (entry of `blocks`), LOCAL_CLASSES x (ca[3], cb[3])
    unsigned* counter;
    int* error;
};

// The E values around one point that its H update needs (own, +j, +k, +i neighbours).
struct ENb {
    float x, y, z;        // own
    float z_jp, x_jp;     // Ez, Ex at j+1
    float y_kp, x_kp;     // Ey, Ex at k+1
    float z_ip, y_ip;     // Ez, Ey at i+1
};

struct PtAxes {           // the axis factors of one point
    const AxisNode* aj;
    const AxisNode* ak;
    bool jn, kn, pml;     // j+1 / k+1 inside the grid; j or k inside the absorbing layer
};

// The plane-dependent parts of the psi offsets (psi_idx, sim.rs:659-665) at plane i: the x slab
// (slot*n1 + j)*n2 + k splits into slot*n1*n2 + (j*n2 + k), the y slab (i*2pml + slot)*n2 + k
// into i*2pml*n2 + (slot*n2 + k), the z slab (i*n1 + j)*pw + slot into i*n1*pw + (j*pw + slot);
// the bracketed parts are 32-bit and formed per point.
struct PsiPlane {
    long long bie, bih, bj, bk;
};

__device__ __forceinline__ PsiPlane psi_plane(const Geom& g, int i, const AxisNode& ai) {
    const long long w = 2 * g.pml, nn12 = (long long)g.n1 * g.n2;
    return PsiPlane{(long long)ai.slot_e * nn12, (long long)ai.slot_h * nn12, (long long)i * w * g.n2,
                    (long long)i * g.n1 * g.pw};
}

// Offset inside slab (field F: 0 = E, 1 = H; derivative axis A) of point (j, k) whose slot along
// A is `slot`.
template <int F>
__device__ __forceinline__ long long psi_off_of(const Geom& g, const PsiPlane& b, int A, int j, int k, int slot) {
    if (A == 0) return (F ? b.bih : b.bie) + (j * g.n2 + k);
    if (A == 1) return b.bj + (slot * g.n2 + k);
    return b.bk + (j * g.pw + slot);
}

struct CoefRef {          // three ca then three cb
    float ca[3], cb[3];
};

// The psi entries of the x and y slabs (derivative axes 0 and 1) that one point reads, fetched
// before any update of the plane is written: the E slabs are updated in place, so a load issued
// after a store through the same pointer would wait for it, and a chain of such round trips per
// point is what an interleaved gather costs. v[A][0] belongs to curl component A+1, v[A][1] to
// A+2 (mod 3). Axes 0 and 1 are uniform over a warp (one plane, one row).
struct PsiG {
    float v[2][2];
};

template <int F>   // 0: the E slabs, 1: the H slabs of the step's input set
__device__ __forceinline__ PsiG psi_gather(const TmaArgs& a, const AxisNode& ai, const AxisNode& aj,
                                           const PsiPlane& pp, int j, int k) {
    PsiG r{{{0.f, 0.f}, {0.f, 0.f}}};
    const Geom& g = a.g;
    const float* src = F ? a.psi_h_in : a.psi_e;
    const int si = F ? ai.slot_h : ai.slot_e, sj = F ? aj.slot_h : aj.slot_e;
    if (si >= 0) {
        const long long o = psi_off_of<F>(g, pp, 0, j, k, si);
        r.v[0][0] = src[g.psi_off[F * 9 + 1 * 3 + 0] + o];
        r.v[0][1] = src[g.psi_off[F * 9 + 2 * 3 + 0] + o];
    }
    if (sj >= 0) {
        const long long o = psi_off_of<F>(g, pp, 1, j, k, sj);
        r.v[1][0] = src[g.psi_off[F * 9 + 2 * 3 + 1] + o];
        r.v[1][1] = src[g.psi_off[F * 9 + 0 * 3 + 1] + o];
    }
    return r;
}

// The z-slab (derivative axis 2) entries of one point: from the block's staged box when the
// producer copied it (`zrow` = the point's row in the box, `zc` = the component stride), else
// from the slab itself.
template <int F>
__device__ __forceinline__ void psi_z(const TmaArgs& a, const PsiPlane& pp, const float* zrow, int zc, int j, int k,
                                      int sl, float& va, float& vb) {
    if (zrow) {
        va = zrow[sl];
        vb = zrow[zc + sl];
    } else {
        const Geom& g = a.g;
        const float* src = F ? a.psi_h_in : a.psi_e;
        const long long o = psi_off_of<F>(g, pp, 2, j, k, sl);
        va = src[g.psi_off[F * 9 + 0 * 3 + 2] + o];
        vb = src[g.psi_off[F * 9 + 1 * 3 + 2] + o];
    }
}

// The CPML terms of derivative axis A at an H point (cpu.rs:65-102), given its psi entries va
// (curl component CA = A+1) and vb (CB = A+2): they go to t[CA][1] and t[CB][0]; owned points
// store the new psi. Nothing happens where the point's slot along A is outside the layer.
template <int A>
__device__ __forceinline__ void h_apply(const TmaArgs& a, const AxisNode& an, float va, float vb,
                                        const float (&d)[3][2], float (&t)[3][2], const bool (&run)[3],
                                        const PsiPlane& pp, int j, int k, bool own) {
    constexpr int CA = (A + 1) % 3, CB = (A + 2) % 3;
    const int sl = an.slot_h;
    if (sl < 0) return;
    const Geom& g = a.g;
    const long long o = psi_off_of<1>(g, pp, A, j, k, sl);
    if (run[CA]) {
        const float r = an.bh * va + an.ch * d[CA][1] * an.raw_inv_d;
        if (own) a.psi_h_out[g.psi_off[9 + CA * 3 + A] + o] = r;
        t[CA][1] += r;
    }
    if (run[CB]) {
        const float r = an.bh * vb + an.ch * d[CB][0] * an.raw_inv_d;
        if (own) a.psi_h_out[g.psi_off[9 + CB * 3 + A] + o] = r;
        t[CB][0] += r;
    }
}

// New H at one point (the update of cpu.rs:48-107). A point inside the CPML (`pml`) adds the psi
// terms of each derivative axis whose slot is live to t where the reference does.
__device__ __forceinline__ void h_node(const TmaArgs& a, const ENb& n, float& hx, float& hy, float& hz,
                                       const PtAxes& q, const AxisNode& ai, const PsiPlane& pp, bool in, bool pml,
                                       const PsiG& gv, const float* zrow, int zc, int j, int k, bool own) {
    const AxisNode* ax[3] = {&ai, q.aj, q.ak};            // by axis 0 (i), 1 (j), 2 (k)
    const float d[3][2] = {{n.z_jp - n.z, n.y_kp - n.y}, {n.x_kp - n.x, n.z_ip - n.z}, {n.y_ip - n.y, n.x_jp - n.x}};
    const bool run[3] = {q.jn && q.kn, q.kn && in, in && q.jn};
    float t[3][2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int u = 0; u < 2; ++u) t[c][u] = d[c][u] * ax[(c + 1 + u) % 3]->inv_d;
    if (pml) {
        h_apply<0>(a, ai, gv.v[0][0], gv.v[0][1], d, t, run, pp, j, k, own);
        h_apply<1>(a, *q.aj, gv.v[1][0], gv.v[1][1], d, t, run, pp, j, k, own);
        const int sk = q.ak->slot_h;
        if (sk >= 0) {
            float va, vb;
            psi_z<1>(a, pp, zrow, zc, j, k, sk, va, vb);
            h_apply<2>(a, *q.ak, va, vb, d, t, run, pp, j, k, own);
        }
    }
    if (run[0]) hx = hx - a.k_mu * (t[0][0] - t[0][1]);
    if (run[1]) hy = hy - a.k_mu * (t[1][0] - t[1][1]);
    if (run[2]) hz = hz - a.k_mu * (t[2][0] - t[2][1]);
}

// The CPML terms of derivative axis A at an owned E point (cpu.rs:125-162), E slabs in place.
template <int A>
__device__ __forceinline__ void e_apply(const TmaArgs& a, const AxisNode& an, float va, float vb,
                                        const float (&d)[3][2], float (&t)[3][2], const bool (&run)[3],
                                        const PsiPlane& pp, int j, int k) {
    constexpr int CA = (A + 1) % 3, CB = (A + 2) % 3;
    const int sl = an.slot_e;
    if (sl < 0) return;
    const Geom& g = a.g;
    const long long o = psi_off_of<0>(g, pp, A, j, k, sl);
    if (run[CA]) {
        const float r = an.be * va + an.ce * d[CA][1] * an.raw_inv_dd;
        a.psi_e[g.psi_off[CA * 3 + A] + o] = r;
        t[CA][1] += r;
    }
    if (run[CB]) {
        const float r = an.be * vb + an.ce * d[CB][0] * an.raw_inv_dd;
        a.psi_e[g.psi_off[CB * 3 + A] + o] = r;
        t[CB][0] += r;
    }
}

// New E at one owned point (cpu.rs:109-167); h*_jm / h*_km are the new H at j-1 / k-1, py / pz
// the H of plane i-1. Same structure as h_node.
__device__ __forceinline__ void e_node(const TmaArgs& a, const CoefRef& cf, float& ex, float& ey, float& ez,
                                       float hx, float hy, float hz, float hz_jm, float hx_jm, float hy_km,
                                       float hx_km, float py, float pz, const PtAxes& q, const AxisNode& ai,
                                       const PsiPlane& pp, bool pml, const PsiG& gv, const float* zrow, int zc,
                                       int i, int j, int k) {
    const AxisNode* ax[3] = {&ai, q.aj, q.ak};
    const float d[3][2] = {{hz - hz_jm, hy - hy_km}, {hx - hx_km, hz - pz}, {hy - py, hx - hx_jm}};
    const bool run[3] = {cf.cb[0] != 0.0f && j > 0 && k > 0, cf.cb[1] != 0.0f && k > 0 && i > 0,
                         cf.cb[2] != 0.0f && i > 0 && j > 0};
    float t[3][2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int u = 0; u < 2; ++u) t[c][u] = d[c][u] * ax[(c + 1 + u) % 3]->inv_dd;
    if (pml) {
        e_apply<0>(a, ai, gv.v[0][0], gv.v[0][1], d, t, run, pp, j, k);
        e_apply<1>(a, *q.aj, gv.v[1][0], gv.v[1][1], d, t, run, pp, j, k);
        const int sk = q.ak->slot_e;
        if (sk >= 0) {
            float va, vb;
            psi_z<0>(a, pp, zrow, zc, j, k, sk, va, vb);
            e_apply<2>(a, *q.ak, va, vb, d, t, run, pp, j, k);
        }
    }
    if (run[0]) ex = cf.ca[0] * ex + cf.cb[0] * (t[0][0] - t[0][1]);
    if (run[1]) ey = cf.ca[1] * ey + cf.cb[1] * (t[1][0] - t[1][1]);
    if (run[2]) ez = cf.ca[2] * ez + cf.cb[2] * (t[2][0] - t[2][1]);
}

constexpr int TMA_CONSUMERS = 256;

// Tile TJ = 7 rows x TK = 64 columns; consumer warp w computes row j0 + w - 1 (warp 0: the halo
// row j0 - 1), each lane a pair of columns k0 + 2 lane, +1. Warp 0 lanes 0..TJ-1 also take the
// halo column k0 - 1, lanes TJ..2TJ-1 the column k0 + TK when the tile owns it (a grid whose
// node count along k is 64t + 1).
// The coefficients of class `id`: from the block's shared table or from the global table.
template <bool LOCAL>
__device__ __forceinline__ CoefRef coef_of(const TmaArgs& a, const float* lt, unsigned id) {
    CoefRef c;
    if constexpr (LOCAL) {
        const float* t = lt + id * 6;
#pragma unroll
        for (int q = 0; q < 3; ++q) { c.ca[q] = t[q]; c.cb[q] = t[3 + q]; }
    } else {
        const DevCoef d = a.classes[id];
#pragma unroll
        for (int q = 0; q < 3; ++q) { c.ca[q] = d.ca[q]; c.cb[q] = d.cb[q]; }
    }
    return c;
}

// PML = false: the block's tile, halo and planes hold no CPML node, and the kernel carries no
// psi code at all; PML = true: the blocks that reach the absorbing layer.
template <int TJ, int TK, typename CID, int STAGES, int SEGMAX, bool LOCAL, int MINB, bool PML>
__global__ void __launch_bounds__(TMA_CONSUMERS + 32, MINB)
    k_tma_step(const __grid_constant__ CUtensorMap map_e, const __grid_constant__ CUtensorMap map_h,
               const __grid_constant__ CUtensorMap map_c, const __grid_constant__ CUtensorMap map_pze,
               const __grid_constant__ CUtensorMap map_pzh, TmaArgs a) {
    static_assert(TJ + 1 == TMA_CONSUMERS / 32 && TK == 64, "one warp per row, one column pair per lane");
    using L = TmaLayout<TJ, TK, CID, STAGES, SEGMAX, LOCAL, PML>;
    static_assert(!LOCAL || sizeof(CID) == 1, "local class ids are 8-bit");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* base = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~uintptr_t(127));
    unsigned char* stages = base;
    float* hn_all = reinterpret_cast<float*>(base + STAGES * L::STAGE);
    AxisNode* axj = reinterpret_cast<AxisNode*>(base + STAGES * L::STAGE + 2 * L::HN);  // rows j0-1 .. j0+TJ
    AxisNode* axk = axj + (TJ + 2);                                                    // cols k0-1 .. k0+TK+2
    AxisNode* axi = axk + (TK + 4);                                                    // planes p_first .. i1
    uint64_t* full = reinterpret_cast<uint64_t*>(base + STAGES * L::STAGE + 2 * L::HN + L::AX);
    uint64_t* empty = full + STAGES;
    float* lt = reinterpret_cast<float*>(base + STAGES * L::STAGE + 2 * L::HN + L::AX + L::BARS);

    const Geom& g = a.g;
    const int tid = threadIdx.x;
    const int bid = a.block0 + int(blockIdx.x);
    const int4 bd = a.blocks[bid];
    const int k0 = bd.x, j0 = bd.y, i0 = bd.z, i1 = bd.w;
    const int p_first = i0 > 0 ? i0 - 1 : 0;   // plane i0-1 supplies H(i0-1) for the first E update
    const int p_last = i1;                     // E(i1) for the last H update (zeros past the grid)
    const bool redge = k0 + TK == g.n2 - 1;    // the last tile of a grid with 64t + 1 nodes along k
    if (a.bump && (blockIdx.x | tid) == 0) *a.counter += 1u;

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            tma::mbar_init(&full[s], 1);
            tma::mbar_init(&empty[s], TMA_CONSUMERS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int q = tid; q < L::NAX; q += blockDim.x) {
        AxisNode v;
        if (q < TJ + 2) v = g.ax[1][min(max(j0 - 1 + q, 0), g.n1 - 1)];
        else if (q < TJ + 2 + TK + 4) v = g.ax[2][min(max(k0 - 1 + (q - TJ - 2), 0), g.n2 - 1)];
        else v = g.ax[0][min(p_first + (q - TJ - 2 - TK - 4), g.n0 - 1)];
        axj[q] = v;
    }
    if constexpr (LOCAL) {
        const float* src = a.tables + (long long)bid * (LOCAL_CLASSES * 6);
        for (int q = tid; q < LOCAL_CLASSES * 6; q += blockDim.x) lt[q] = src[q];
    }
    __syncthreads();
    // the tile (with its halo column and right-edge column) reaches the k layer: z boxes staged
    bool kz = false;
    if (PML && a.pz)
        for (int q = 0; q < TK + 2; ++q) kz = kz || axk[q].slot_h >= 0 || axk[q].slot_e >= 0;
    const int zc = (TJ + 1) * g.pw;   // component stride inside a staged z box

    if (tid >= TMA_CONSUMERS) {
        // producer warp: one lane issues the copies
        if (tid != TMA_CONSUMERS) return;
        for (int p = p_first; p <= p_last; ++p) {
            const int u = p - p_first, s = u % STAGES, n = u / STAGES;
            if (!tma::mbar_wait(&empty[s], uint32_t((n & 1) ^ 1), tma::WAIT_LIMIT_NS)) {
                atomicExch(a.error, 1);
                for (int q = max(p_first, p - STAGES); q < p; ++q) {
                    const int uq = q - p_first;
                    tma::mbar_wait(&full[uq % STAGES], uint32_t((uq / STAGES) & 1), tma::WAIT_LIMIT_NS);
                }
                return;
            }
            unsigned char* st = stages + s * L::STAGE;
            const bool zp = PML && kz && p < i1;   // plane i1 supplies E only
            tma::mbar_expect_tx(&full[s], L::TX + (zp ? 2 * 2 * zc * 4 : 0));
            tma::load_4d(st, &map_e, &full[s], k0 - 4, j0 - 1, p, 0);
            tma::load_4d(st + L::al(L::E_BYTES), &map_h, &full[s], k0 - 4, j0 - 1, p, 0);
            tma::load_3d(st + L::al(L::E_BYTES) + L::al(L::H_BYTES), &map_c, &full[s], k0, j0, p);
            if (zp) {
                tma::load_4d(st + L::PZ_OFF, &map_pze, &full[s], 0, j0 - 1, p, 0);
                tma::load_4d(st + L::PZ_OFF + L::PZ_FIELD, &map_pzh, &full[s], 0, j0 - 1, p, 0);
            }
        }
        return;
    }

    // ---- consumers
    constexpr int EC = L::ER * L::EW, HC = L::HR * L::HW, NC = L::NR * L::NW;
    const int w = tid >> 5, lane = tid & 31;
    const int r = w - 1;              // tile row of this warp's pair (-1: the halo row)
    const int c = 2 * lane;           // first column of the pair
    const int jj = j0 + r, kk = k0 + c;
    const bool row_live = jj >= 0 && jj < g.n1;
    const bool live0 = row_live && kk < g.n2, live1 = row_live && kk + 1 < g.n2;
    const bool own_row = r >= 0;
    const AxisNode* rj = axj + (r + 1);
    PtAxes q0{rj, axk + (c + 1), jj + 1 < g.n1, kk + 1 < g.n2, false};
    PtAxes q1{rj, axk + (c + 2), jj + 1 < g.n1, kk + 2 < g.n2, false};
    const bool pml_j = PML && (rj->slot_e >= 0 || rj->slot_h >= 0);
    q0.pml = pml_j || (PML && (q0.ak->slot_e >= 0 || q0.ak->slot_h >= 0));
    q1.pml = pml_j || (PML && (q1.ak->slot_e >= 0 || q1.ak->slot_h >= 0));
    const int eo = (r + 1) * L::EW + c + 4, ho = (r + 1) * L::HW + c + 4, no = (r + 1) * L::NW + c + 2;
    const unsigned goff = unsigned(max(jj, 0)) * unsigned(g.p2) + unsigned(kk);
    // warp 0 extras: the k-1 halo column (lanes 0..TJ-1), the owned right-edge column (lanes
    // TJ..2TJ-1) and that column's j-1 halo point (lane 2TJ)
    const int xr = lane < TJ ? lane : (lane < 2 * TJ ? lane - TJ : -1);  // row of the extra point
    const int xc = lane < TJ ? -1 : TK;                                   // column of the extra point
    const bool xtra = w == 0 && ((lane < TJ && k0 > 0) || (lane >= TJ && lane <= 2 * TJ && redge)) &&
                      j0 + xr >= 0 && j0 + xr < g.n1;
    const bool xown = xtra && lane >= TJ && lane < 2 * TJ;                // the right-edge points are owned
    const int xj = j0 + xr, xk = k0 + xc;
    PtAxes qx{axj + (xr + 1), axk + (xc + 1), xj + 1 < g.n1, xk + 1 < g.n2, false};
    qx.pml = PML && (qx.aj->slot_e >= 0 || qx.aj->slot_h >= 0 || qx.ak->slot_e >= 0 || qx.ak->slot_h >= 0);
    const int xeo = (xr + 1) * L::EW + xc + 4, xho = (xr + 1) * L::HW + xc + 4, xno = (xr + 1) * L::NW + xc + 2;
    const unsigned xgoff = unsigned(min(xj, g.n1 - 1)) * unsigned(g.p2) + unsigned(max(xk, 0));

    float py0 = 0.f, pz0 = 0.f, py1 = 0.f, pz1 = 0.f, pyx = 0.f, pzx = 0.f;  // H of plane i-1
    bool bad = false;
    for (int p = p_first; p < i1; ++p) {
        const int u = p - p_first;
        const int s = u % STAGES, s1 = (u + 1) % STAGES;
        const bool pre = p < i0;  // the plane before the segment: H only, nothing written
        if (!tma::mbar_wait(&full[s], uint32_t((u / STAGES) & 1), tma::WAIT_LIMIT_NS)) bad = true;
        if (!tma::mbar_wait(&full[s1], uint32_t(((u + 1) / STAGES) & 1), tma::WAIT_LIMIT_NS)) bad = true;
        const float* E = reinterpret_cast<const float*>(stages + s * L::STAGE);
        const float* E1 = reinterpret_cast<const float*>(stages + s1 * L::STAGE);
        const float* H = reinterpret_cast<const float*>(stages + s * L::STAGE + L::al(L::E_BYTES));
        const CID* CL = reinterpret_cast<const CID*>(stages + s * L::STAGE + L::al(L::E_BYTES) + L::al(L::H_BYTES));
        const float* ZE = PML && kz ? reinterpret_cast<const float*>(stages + s * L::STAGE + L::PZ_OFF) : nullptr;
        const float* ZH = kz ? ZE + L::PZ_FIELD / 4 : nullptr;
        float* hn = hn_all + (u & 1) * (L::HN / 4);
        const int i = p;
        const AxisNode& ai = axi[u];
        const bool pml_i = PML && (ai.slot_e >= 0 || ai.slot_h >= 0);
        const bool in = i + 1 < g.n0;
        const long long plane = (long long)i * g.n1 * g.p2;
        const bool own = own_row && !pre;
        const PsiPlane pp = psi_plane(g, i, ai);

        // 1. new H: the pair (two columns), and warp 0's extra point; x/y-slab psi fetched first
        PsiG gh0{}, gh1{}, ghx{};
        if (live0 && (q0.pml || pml_i)) gh0 = psi_gather<1>(a, ai, *q0.aj, pp, jj, kk);
        if (live1 && (q1.pml || pml_i)) gh1 = psi_gather<1>(a, ai, *q1.aj, pp, jj, kk + 1);
        if (xtra && (qx.pml || pml_i)) ghx = psi_gather<1>(a, ai, *qx.aj, pp, xj, xk);
        const float* zh0 = ZH ? ZH + (r + 1) * g.pw : nullptr;
        ENb nb0, nb1;
        float hx0 = 0.f, hy0 = 0.f, hz0 = 0.f, hx1 = 0.f, hy1 = 0.f, hz1 = 0.f;
        if (live0) {
            const float2 x = *reinterpret_cast<const float2*>(E + eo);
            const float2 y = *reinterpret_cast<const float2*>(E + EC + eo);
            const float2 z = *reinterpret_cast<const float2*>(E + 2 * EC + eo);
            const float2 zj = *reinterpret_cast<const float2*>(E + 2 * EC + eo + L::EW);
            const float2 xj = *reinterpret_cast<const float2*>(E + eo + L::EW);
            const float2 zi = *reinterpret_cast<const float2*>(E1 + 2 * EC + eo);
            const float2 yi = *reinterpret_cast<const float2*>(E1 + EC + eo);
            const float y2 = E[EC + eo + 2], x2 = E[eo + 2];
            nb0 = ENb{x.x, y.x, z.x, zj.x, xj.x, y.y, x.y, zi.x, yi.x};
            nb1 = ENb{x.y, y.y, z.y, zj.y, xj.y, y2, x2, zi.y, yi.y};
            const float2 hx = *reinterpret_cast<const float2*>(H + ho);
            const float2 hy = *reinterpret_cast<const float2*>(H + HC + ho);
            const float2 hz = *reinterpret_cast<const float2*>(H + 2 * HC + ho);
            hx0 = hx.x; hy0 = hy.x; hz0 = hz.x;
            hx1 = hx.y; hy1 = hy.y; hz1 = hz.y;
            h_node(a, nb0, hx0, hy0, hz0, q0, ai, pp, in, q0.pml || pml_i, gh0, zh0, zc, jj, kk, own);
            if (live1) h_node(a, nb1, hx1, hy1, hz1, q1, ai, pp, in, q1.pml || pml_i, gh1, zh0, zc, jj, kk + 1, own);
            *reinterpret_cast<float2*>(hn + no) = make_float2(hx0, hx1);
            *reinterpret_cast<float2*>(hn + NC + no) = make_float2(hy0, hy1);
            *reinterpret_cast<float2*>(hn + 2 * NC + no) = make_float2(hz0, hz1);
            if (own) {
                // a dead second column is padding and stays zero
                float* o = a.h_out + plane + goff;
                *reinterpret_cast<float2*>(o) = make_float2(hx0, live1 ? hx1 : 0.f);
                *reinterpret_cast<float2*>(o + g.cs) = make_float2(hy0, live1 ? hy1 : 0.f);
                *reinterpret_cast<float2*>(o + 2 * g.cs) = make_float2(hz0, live1 ? hz1 : 0.f);
            }
        }
        ENb nx;
        float hxx = 0.f, hyx = 0.f, hzx = 0.f;
        if (xtra) {
            const float* e0 = E + xeo;
            nx = ENb{e0[0], e0[EC], e0[2 * EC], e0[2 * EC + L::EW], e0[L::EW], e0[EC + 1], e0[1], E1[2 * EC + xeo],
                     E1[EC + xeo]};
            hxx = H[xho];
            hyx = H[HC + xho];
            hzx = H[2 * HC + xho];
            const bool xo = xown && !pre;
            h_node(a, nx, hxx, hyx, hzx, qx, ai, pp, in, qx.pml || pml_i, ghx, ZH ? ZH + (xr + 1) * g.pw : nullptr, zc,
                   xj, xk, xo);
            hn[xno] = hxx;
            hn[NC + xno] = hyx;
            hn[2 * NC + xno] = hzx;
            if (xo) {
                float* o = a.h_out + plane + xgoff;
                o[0] = hxx;
                o[g.cs] = hyx;
                o[2 * g.cs] = hzx;
            }
        }
        if (tma::consumers_sync_or(bad, TMA_CONSUMERS)) {
            if (tid == 0) atomicExch(a.error, 2);
            return;
        }

        // 2. new E on the owned points; every x/y-slab psi read precedes the in-place writes
        if (!pre) {
            PsiG ge0{}, ge1{}, gex{};
            if (own_row && live0 && (q0.pml || pml_i)) ge0 = psi_gather<0>(a, ai, *q0.aj, pp, jj, kk);
            if (own_row && live1 && (q1.pml || pml_i)) ge1 = psi_gather<0>(a, ai, *q1.aj, pp, jj, kk + 1);
            if (xown && (qx.pml || pml_i)) gex = psi_gather<0>(a, ai, *qx.aj, pp, xj, xk);
            const float* ze0 = ZE ? ZE + (r + 1) * g.pw : nullptr;
            if (own_row && live0) {
                // the pair's two class ids in one aligned load (c is even)
                unsigned id0, id1;
                if constexpr (sizeof(CID) == 1) {
                    const unsigned v = *reinterpret_cast<const uint16_t*>(CL + r * L::CW + c);
                    id0 = v & 0xffu;
                    id1 = v >> 8;
                } else if constexpr (sizeof(CID) == 2) {
                    const unsigned v = *reinterpret_cast<const uint32_t*>(CL + r * L::CW + c);
                    id0 = v & 0xffffu;
                    id1 = v >> 16;
                } else {
                    id0 = CL[r * L::CW + c];
                    id1 = CL[r * L::CW + c + 1];
                }
                const CoefRef cf0 = coef_of<LOCAL>(a, lt, id0);
                const float2 hzj = *reinterpret_cast<const float2*>(hn + 2 * NC + no - L::NW);
                const float2 hxj = *reinterpret_cast<const float2*>(hn + no - L::NW);
                const float hyk = hn[NC + no - 1], hxk = hn[no - 1];
                float ex0 = nb0.x, ey0 = nb0.y, ez0 = nb0.z;
                e_node(a, cf0, ex0, ey0, ez0, hx0, hy0, hz0, hzj.x, hxj.x, hyk, hxk, py0, pz0, q0, ai, pp, q0.pml || pml_i,
                       ge0, ze0, zc, i, jj, kk);
                float ex1 = 0.f, ey1 = 0.f, ez1 = 0.f;
                if (live1) {
                    const CoefRef cf1 = coef_of<LOCAL>(a, lt, id1);
                    ex1 = nb1.x; ey1 = nb1.y; ez1 = nb1.z;
                    e_node(a, cf1, ex1, ey1, ez1, hx1, hy1, hz1, hzj.y, hxj.y, hy0, hx0, py1, pz1, q1, ai, pp,
                           q1.pml || pml_i, ge1, ze0, zc, i, jj, kk + 1);
                }
                float* o = a.e_out + plane + goff;
                *reinterpret_cast<float2*>(o) = make_float2(ex0, ex1);
                *reinterpret_cast<float2*>(o + g.cs) = make_float2(ey0, ey1);
                *reinterpret_cast<float2*>(o + 2 * g.cs) = make_float2(ez0, ez1);
            }
            if (xown) {
                const CoefRef cf = coef_of<LOCAL>(a, lt, CL[xr * L::CW + xc]);
                float ex = nx.x, ey = nx.y, ez = nx.z;
                e_node(a, cf, ex, ey, ez, hxx, hyx, hzx, hn[2 * NC + xno - L::NW], hn[xno - L::NW], hn[NC + xno - 1],
                       hn[xno - 1], pyx, pzx, qx, ai, pp, qx.pml || pml_i, gex, ZE ? ZE + (xr + 1) * g.pw : nullptr, zc,
                       i, xj, xk);
                float* o = a.e_out + plane + xgoff;
                o[0] = ex;
                o[g.cs] = ey;
                o[2 * g.cs] = ez;
            }
        }
        py0 = hy0; pz0 = hz0; py1 = hy1; pz1 = hz1; pyx = hyx; pzx = hzx;
        tma::mbar_arrive(&empty[s]);
    }
    // the last plane's stage (E(i1)) was waited on by the final iteration; nothing is in flight
}

// Host side ---------------------------------------------------------------------------------

struct TmaPlan {
    CUtensorMap e[2], h[2], c;   // per input parity
    CUtensorMap pze, pzh[2];     // the z-slab psi: E slabs, H slabs of the input set per parity
    bool pz = false;
    int tj = 8, tk = 64, seg = 64;
    int n_clean = 0, n_layer = 0;  // blocks of the clean kernel (listed first) and of the layer kernel
    int shape = 0;               // index into the engine's kernel shapes
    int smem = 0;
    bool ok = false;
    std::string why;
};

}  // namespace fg
