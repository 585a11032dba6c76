// The fused E+H step fed by the Tensor Memory Accelerator: the engine's main stencil on the B200.
//
// A block owns a TJ x TK tile of (j, k) columns and marches along x over a segment of planes.
// One producer warp streams, per plane p, three boxes into a ring of shared-memory stages with
// cp.async.bulk.tensor (4-D maps over (k, j, i, component)):
//   E(p)     rows j0-1 .. j0+TJ,   columns k0-4 .. k0+TK+3 (all 3 components)
//   H_in(p)  rows j0-1 .. j0+TJ-1, columns k0-4 .. k0+TK-1 (all 3 components)
//   class(p) rows j0   .. j0+TJ-1, columns from k0 rounded down to 16 (the node class ids)
// Box origins in k are rounded down to 16 bytes; rows or planes outside the grid arrive as zeros.
// Eight consumer warps then, per plane i:
//   1. form the new H on the tile and on its j-1 row and k-1 column (the halo the E update needs;
//      halo points are recomputed, read-only) from the E(i), E(i+1) and H_in(i) boxes, into a
//      triple-buffered H tile; owned points go to the output buffer;
//   2. after one barrier, form the new E of the tile from the H tile of plane i and of plane i-1.
// Each node's E and H are read from DRAM once and written once per step (48 B) plus its class id.
// The kernel covers the clean box, where no CPML term arises; the shell kernels update the rest.
// Mbarrier waits are bounded by the global timer: a wait that runs out raises the error word and
// the block leaves without starting new work.
#pragma once

#include <cuda.h>

#include <string>

#include "kernels.cuh"

namespace fg {

namespace tma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return uint32_t(__cvta_generic_to_shared(p)); }

// The first 128-byte boundary at or after p (a dynamic shared-memory array). The offset is added to
// the array's own pointer, so the compiler still sees a shared-memory address and emits shared
// loads and stores (an integer round trip of the pointer would leave generic accesses).
__device__ __forceinline__ unsigned char* align128(unsigned char* p) { return p + ((128u - (smem_u32(p) & 127u)) & 127u); }

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
constexpr uint64_t WAIT_LIMIT_MIN_NS = 1000000ull;  // the shortest limit a run may ask for (1 ms)

}  // namespace tma

// Shared-memory layout of one block (tile TJ x TK, TJ + 1 consumer warps' worth of rows).
// With LOCAL, class ids are 8-bit indices into a per-block table of at most LOCAL_CLASSES
// (ca[3], cb[3]) records that the block keeps in shared memory.
constexpr int LOCAL_CLASSES = 256;

template <int TJ, int TK, typename CID, int STAGES, int SEGMAX, bool LOCAL = false, bool ZL = false>
struct TmaLayout {
    static constexpr int EW = TK + 8, ER = TJ + 2;   // E box: columns k0-4 .. k0+TK+3, rows j0-1 .. j0+TJ
    static constexpr int HW = TK + 8, HR = TJ + 1;   // H box: columns k0-4 .. k0+TK+3, rows j0-1 .. j0+TJ-1
    static constexpr int CW = TK + 16, CR = TJ;      // class box: columns (k0 & ~15) + 0 .. 79, rows j0 .. j0+TJ-1
    static constexpr int NW = TK + 4, NR = TJ + 1;   // new-H tile: column k at k-k0+2, row j at j-j0+1
    static constexpr int E_BYTES = 3 * ER * EW * 4;
    static constexpr int H_BYTES = 3 * HR * HW * 4;
    static constexpr int C_BYTES = CR * CW * int(sizeof(CID));
    __host__ __device__ static constexpr int al(int b) { return (b + 127) & ~127; }
    // ZL (tiles that reach the k layer): per field a staged z-slab box of 2 components x
    // (TJ + 1) rows (j0-1 .. j0+TJ-1) x pw slots, pw <= PZW
    static constexpr int PZW = 32;
    static constexpr int PZ_FIELD = 2 * (TJ + 1) * PZW * 4;
    static constexpr int PZ_OFF = al(E_BYTES) + al(H_BYTES) + al(C_BYTES);
    static constexpr int STAGE = PZ_OFF + (ZL ? 2 * PZ_FIELD : 0);
    static constexpr int TX = E_BYTES + H_BYTES + C_BYTES;  // bytes one stage's field copies deliver
    static constexpr int HN = al(3 * NR * NW * 4);
    static constexpr int NAX = (TJ + 2) + (TK + 4) + (SEGMAX + 2);
    static constexpr int AX = al(NAX * int(sizeof(AxisNode)));
    static constexpr int BARS = al(2 * STAGES * 8);
    // the block's coefficient table, then (a folded Debye ADE) its entries' Debye masks
    static constexpr int LT = LOCAL ? al(LOCAL_CLASSES * 6 * 4 + LOCAL_CLASSES) : 0;
    // ZL: per consumer warp, the k-layer CPML terms of its row (two components x TK columns)
    static constexpr int ZR = al((TJ + 1) * 2 * TK * 4);
    // ZL: the k factors (b, c, raw) of the block's columns k0-1 .. k0+TK+2, for H then for E
    static constexpr int ZK = al(2 * (TK + 4) * 16);
    static constexpr int TOTAL = STAGES * STAGE + 2 * HN + AX + BARS + LT + ZR + ZK + 128;
};

struct TmaArgs {
    Geom g;
    const DevCoef* classes;
    float* __restrict__ e_out;
    float* __restrict__ h_out;
    float k_mu;
    int kbeg, jend, kend;                // the clean box: rows < jend, columns kbeg .. kend-1 are owned
    const int4* blocks;                  // per block: (k0, j0, i0, i1) of its tile and x-segment
    const int2* own_rows;                // per block: the rows [x, y) it writes; null: [j0, jend)
    int block0;                          // this launch's first entry of `blocks`
    int bump;                            // this launch opens the step (raises the step counter)
    float* psi_e;                        // ZL: the E psi slabs (z slabs updated in place)
    float* psi_h_out;                    // ZL: the H psi slabs of the output set
    const float* tables;                 // LOCAL: per block (entry of `blocks`), LOCAL_CLASSES x (ca[3], cb[3])
    unsigned* counter;
    int* error;
    unsigned long long wait_ns;          // the limit of every mbarrier wait (2 s in normal runs)
    float neg0;                          // -0.0f (the packed products' addend, see f2::mul)
    int stall_plane;                     // test knob, -1 in normal runs: the full barrier of this
                                         // plane expects 16 bytes more than its copies deliver, so
                                         // the waits on it run out (the failure path under test)
    // the Debye ADE folded into the E half (FOLD): the edges at the nodes the block's column
    // pairs write, in march order (setup_kernels.cuh)
    const uint8_t* lmask;                // per block: LOCAL_CLASSES masks, bit c: E_c is a Debye edge
    const int* drow;                     // per (block, owned plane, row): the row's first folded edge
    const float* fdd;                    // dd per folded edge
    float* fstate;                       // pole state per folded edge, pole-major (nfold per pole)
    int nfold, npoles;
    float db[2], dc[2];                  // the pole table: b_k and c_k (k_debye_post_cb's table)
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
    bool jn, kn;          // j+1 / k+1 inside the grid
};

struct CoefRef {          // three ca then three cb
    float ca[3], cb[3];
};

// The k-layer CPML term of one point (cpu.rs:65-102 for H, :125-162 for E) for the two curl
// components that differentiate along k (CA = 0 in t[0][1], CB = 1 in t[1][0]), with the old psi
// from the block's staged z box (`zrow` = the point's row, `zc` = the component stride); owned
// points store the new psi (H: to the output set; E: in place).
template <int F>   // 1: H (bh, ch, raw_inv_d), 0: E (be, ce, raw_inv_dd)
__device__ __forceinline__ void z_terms(const TmaArgs& a, const AxisNode& ak, const float (&d)[3][2],
                                        float (&t)[3][2], bool run0, bool run1, const float* zrow, int zc, int i,
                                        int j, bool own) {
    const int sl = F ? ak.slot_h : ak.slot_e;
    if (sl < 0) return;
    const Geom& g = a.g;
    const float bb = F ? ak.bh : ak.be, cc = F ? ak.ch : ak.ce, raw = F ? ak.raw_inv_d : ak.raw_inv_dd;
    const long long o = ((long long)i * g.n1 + j) * g.pw + sl;
    float* dst = F ? a.psi_h_out : a.psi_e;
    if (run0) {
        const float r = bb * zrow[sl] + cc * d[0][1] * raw;
        if (own) dst[g.psi_off[F * 9 + 0 * 3 + 2] + o] = r;
        t[0][1] += r;
    }
    if (run1) {
        const float r = bb * zrow[zc + sl] + cc * d[1][0] * raw;
        if (own) dst[g.psi_off[F * 9 + 1 * 3 + 2] + o] = r;
        t[1][0] += r;
    }
}

// New H at one point outside the CPML (the update of cpu.rs:48-107 with no psi term).
template <bool ZL = false>
__device__ __forceinline__ void h_node(const TmaArgs& a, const ENb& n, float& hx, float& hy, float& hz,
                                       const PtAxes& q, const AxisNode& ai, bool in, const float* zrow = nullptr,
                                       int zc = 0, int i = 0, int j = 0, bool own = false) {
    const AxisNode* ax[3] = {&ai, q.aj, q.ak};            // by axis 0 (i), 1 (j), 2 (k)
    const float d[3][2] = {{n.z_jp - n.z, n.y_kp - n.y}, {n.x_kp - n.x, n.z_ip - n.z}, {n.y_ip - n.y, n.x_jp - n.x}};
    float t[3][2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int u = 0; u < 2; ++u) t[c][u] = d[c][u] * ax[(c + 1 + u) % 3]->inv_d;
    if constexpr (ZL) z_terms<1>(a, *q.ak, d, t, q.jn && q.kn, q.kn && in, zrow, zc, i, j, own);
    if (q.jn && q.kn) hx = hx - a.k_mu * (t[0][0] - t[0][1]);
    if (q.kn && in) hy = hy - a.k_mu * (t[1][0] - t[1][1]);
    if (in && q.jn) hz = hz - a.k_mu * (t[2][0] - t[2][1]);
}

// New E at one owned point outside the CPML (cpu.rs:109-167); h*_jm / h*_km are the new H at
// j-1 / k-1, py / pz the H of plane i-1.
template <bool ZL = false>
__device__ __forceinline__ void e_node(const TmaArgs& a, const CoefRef& cf, float& ex, float& ey, float& ez, float hx,
                                       float hy, float hz, float hz_jm, float hx_jm, float hy_km, float hx_km,
                                       float py, float pz, const PtAxes& q, const AxisNode& ai, int i, int j, int k,
                                       const float* zrow = nullptr, int zc = 0) {
    const AxisNode* ax[3] = {&ai, q.aj, q.ak};
    const float d[3][2] = {{hz - hz_jm, hy - hy_km}, {hx - hx_km, hz - pz}, {hy - py, hx - hx_jm}};
    float t[3][2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int u = 0; u < 2; ++u) t[c][u] = d[c][u] * ax[(c + 1 + u) % 3]->inv_dd;
    const bool run0 = cf.cb[0] != 0.0f && j > 0 && k > 0, run1 = cf.cb[1] != 0.0f && k > 0 && i > 0;
    if constexpr (ZL) z_terms<0>(a, *q.ak, d, t, run0, run1, zrow, zc, i, j, true);
    if (run0) ex = cf.ca[0] * ex + cf.cb[0] * (t[0][0] - t[0][1]);
    if (run1) ey = cf.ca[1] * ey + cf.cb[1] * (t[1][0] - t[1][1]);
    if (cf.cb[2] != 0.0f && i > 0 && j > 0) ez = cf.ca[2] * ez + cf.cb[2] * (t[2][0] - t[2][1]);
}

constexpr int TMA_CONSUMERS = 256;

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

// Pairs of f32 in one instruction (sm_100's packed FP32: add/sub .rn .f32x2 and products as a fused
// multiply-add of -0). Each lane of the pair is rounded as the scalar operation would be (round to
// nearest, never fused with another operation), so a pair update gives the scalar update's bits.
namespace f2 {
__device__ __forceinline__ float2 add(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "add.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
__device__ __forceinline__ float2 sub(float2 a, float2 b) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return d;
}
// The product as fma(a, b, z) with z = (-0, -0): one rounding, the product's own (x + (-0) = x for
// every x, signed zeros included). The assembler contracts a packed mul.rn with a following packed
// add or sub into one fused operation (one rounding where the scalar path rounds twice), and it
// would drop a literal -0 addend and contract again; z therefore comes from a kernel argument, whose
// value it cannot see, and the product stays a fused operation of its own.
__device__ __forceinline__ float2 mul(float2 a, float2 b, float2 z) {
    float2 d;
    asm("{\n\t.reg .b64 ra, rb, rz, rd;\n\tmov.b64 ra, {%2, %3};\n\tmov.b64 rb, {%4, %5};\n\t"
        "mov.b64 rz, {%6, %7};\n\tfma.rn.f32x2 rd, ra, rb, rz;\n\tmov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(d.x), "=f"(d.y) : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y), "f"(z.x), "f"(z.y));
    return d;
}
__device__ __forceinline__ float2 bc(float v) { return make_float2(v, v); }
__device__ __forceinline__ float2 pick(bool px, bool py, float2 n, float2 o) {
    return make_float2(px ? n.x : o.x, py ? n.y : o.y);
}
}  // namespace f2

// The pair's E around its H updates: own (x, y, z), +j (zj, xj), +k (yk, xk: the columns c + 1 and
// c + 2), +i (zi, yi).
struct EPair {
    float2 x, y, z, zj, xj, yk, xk, zi, yi;
};

// New H of a column pair outside the CPML (h_node on both columns at once); dk, kn per column.
// ZL: zr points at the pair's k-layer terms in its warp's row buffer (component 0 at zr, 1 at
// zr + zs), formed by the row's dense pass; zf bit 0 / 1: column c / c + 1 has a live H slot.
template <bool ZL>
__device__ __forceinline__ void h_pair(const TmaArgs& a, float2 mz, const EPair& n, float2& hx, float2& hy, float2& hz, float di,
                                       float dj, float2 dk, bool jn, bool kn0, bool kn1, bool in, bool live1,
                                       const float* zr, int zs, unsigned zf) {
    using namespace f2;
    const float2 d00 = sub(n.zj, n.z), d01 = sub(n.yk, n.y);
    const float2 d10 = sub(n.xk, n.x), d11 = sub(n.zi, n.z);
    const float2 d20 = sub(n.yi, n.y), d21 = sub(n.xj, n.x);
    float2 t00 = mul(d00, bc(dj), mz), t01 = mul(d01, dk, mz);
    float2 t10 = mul(d10, dk, mz), t11 = mul(d11, bc(di), mz);
    const float2 t20 = mul(d20, bc(di), mz), t21 = mul(d21, bc(dj), mz);
    if constexpr (ZL) {
        if (zf & 3u) {   // z_terms<1>'s additions, in its order (t += r after the product)
            const float2 r0 = *reinterpret_cast<const float2*>(zr), r1 = *reinterpret_cast<const float2*>(zr + zs);
            if ((zf & 1u) && jn && kn0) t01.x = t01.x + r0.x;
            if ((zf & 1u) && kn0 && in) t10.x = t10.x + r1.x;
            if (live1 && (zf & 2u) && jn && kn1) t01.y = t01.y + r0.y;
            if (live1 && (zf & 2u) && kn1 && in) t10.y = t10.y + r1.y;
        }
    }
    const float2 km = bc(a.k_mu);
    const float2 nx = sub(hx, mul(km, sub(t00, t01), mz));
    const float2 ny = sub(hy, mul(km, sub(t10, t11), mz));
    const float2 nz = sub(hz, mul(km, sub(t20, t21), mz));
    hx = pick(jn && kn0, jn && kn1 && live1, nx, hx);
    hy = pick(kn0 && in, kn1 && in && live1, ny, hy);
    hz = pick(in && jn, in && jn && live1, nz, hz);
}

// New E of a column pair outside the CPML (e_node on both columns); hj: H at j - 1, hk: H at k - 1
// (columns c - 1 and c), p: H of plane i - 1. ZL: as h_pair, zf bit 2 / 3: column c / c + 1 has a
// live E slot.
template <bool ZL>
__device__ __forceinline__ void e_pair(const TmaArgs& a, float2 mz, const CoefRef& c0, const CoefRef& c1, float2& ex, float2& ey,
                                       float2& ez, float2 hx, float2 hy, float2 hz, float2 hzj, float2 hxj, float2 hyk,
                                       float2 hxk, float2 py, float2 pz, float ei, float ej, float2 ek, int i, int j,
                                       int k, bool live1, const float* zr, int zs, unsigned zf) {
    using namespace f2;
    const float2 d00 = sub(hz, hzj), d01 = sub(hy, hyk);
    const float2 d10 = sub(hx, hxk), d11 = sub(hz, pz);
    const float2 d20 = sub(hy, py), d21 = sub(hx, hxj);
    float2 t00 = mul(d00, bc(ej), mz), t01 = mul(d01, ek, mz);
    float2 t10 = mul(d10, ek, mz), t11 = mul(d11, bc(ei), mz);
    const float2 t20 = mul(d20, bc(ei), mz), t21 = mul(d21, bc(ej), mz);
    const bool r00 = c0.cb[0] != 0.0f && j > 0 && k > 0, r01 = live1 && c1.cb[0] != 0.0f && j > 0;
    const bool r10 = c0.cb[1] != 0.0f && k > 0 && i > 0, r11 = live1 && c1.cb[1] != 0.0f && i > 0;
    const bool r20 = c0.cb[2] != 0.0f && i > 0 && j > 0, r21 = live1 && c1.cb[2] != 0.0f && i > 0 && j > 0;
    if constexpr (ZL) {
        if (zf & 12u) {   // z_terms<0>'s additions
            const float2 r0 = *reinterpret_cast<const float2*>(zr), r1 = *reinterpret_cast<const float2*>(zr + zs);
            if ((zf & 4u) && r00) t01.x = t01.x + r0.x;
            if ((zf & 4u) && r10) t10.x = t10.x + r1.x;
            if ((zf & 8u) && r01) t01.y = t01.y + r0.y;
            if ((zf & 8u) && r11) t10.y = t10.y + r1.y;
        }
    }
    const float2 nx = add(mul(make_float2(c0.ca[0], c1.ca[0]), ex, mz), mul(make_float2(c0.cb[0], c1.cb[0]), sub(t00, t01), mz));
    const float2 ny = add(mul(make_float2(c0.ca[1], c1.ca[1]), ey, mz), mul(make_float2(c0.cb[1], c1.cb[1]), sub(t10, t11), mz));
    const float2 nz = add(mul(make_float2(c0.ca[2], c1.ca[2]), ez, mz), mul(make_float2(c0.cb[2], c1.cb[2]), sub(t20, t21), mz));
    ex = pick(r00, r01, nx, ex);
    ey = pick(r10, r11, ny, ey);
    ez = pick(r20, r21, nz, ez);
}

// The fused step on the clean box: every point a block computes (its tile, halo row j0-1, halo
// column k0-1 and halo plane i0-1) lies outside the CPML, so no psi term appears; the absorbing
// shell around the box is updated by the shell kernels (stencil_shell.cuh).
// Tile TJ = 7 rows x TK = 64 columns; consumer warp w computes row j0 + w - 1 (warp 0: the halo
// row j0 - 1), each lane a pair of columns k0 + 2 lane, +1. Warp 0 lanes 0..TJ-1 also take the
// halo column k0 - 1, lanes TJ..2TJ-1 the column k0 + TK when the tile owns it (a clean box
// reaching the end of a grid whose node count along k is 64t + 1). Points past jend / kend are
// computed when they exist in the grid but never written, and so are the first tile's columns
// below kbeg; kbeg and kend are even (unless kend = n2), so a column pair is owned whole.
// ZL = true: tiles that reach the k layer (in clean rows and planes): the producer also stages
// the z-slab psi of every plane, and points inside the layer add their k-layer CPML terms.
// A block descriptor's k0 carries this bit when the tile reaches the k layer.
constexpr int TMA_ZL_TILE = 1 << 30;

// One block's march; ZL: the tile reaches the k layer. The shared-memory layout is the ZL one for
// both (the z boxes sit past the field boxes of each stage), so one launch runs both kinds of tile
// in the block list's order: neighbouring tiles march together and share their halo columns in L2.
// One folded Debye edge of a one-pole model (k_debye_post_cb's arithmetic, in its order): e is the
// edge's new E, old its E before the step, w its dd and st its pole state (both loaded before the
// H half); the new state goes to q.
__device__ __forceinline__ void fold_edge(const TmaArgs& a, float& e, float old, float cb, float w, float st, int q) {
    float s0 = 0.0f;
    s0 += 0.5f * (1.0f + a.db[0]) * st;
    const float next = e - cb * s0;
    e = next;
    const float de = next - old;
    a.fstate[q] = a.db[0] * st + w * a.dc[0] * de;
}

template <int TJ, int TK, typename CID, int STAGES, int SEGMAX, bool LOCAL, bool ZL, bool FOLD = false>
__device__ __forceinline__ void tma_march(const CUtensorMap& map_e, const CUtensorMap& map_h, const CUtensorMap& map_c,
                                          const CUtensorMap& map_pze, const CUtensorMap& map_pzh, const TmaArgs& a,
                                          unsigned char* base) {
    static_assert(TJ + 1 == TMA_CONSUMERS / 32 && TK == 64, "one warp per row, one column pair per lane");
    using L = TmaLayout<TJ, TK, CID, STAGES, SEGMAX, LOCAL, true>;
    static_assert(!LOCAL || sizeof(CID) == 1, "local class ids are 8-bit");
    unsigned char* stages = base;
    float* hn_all = reinterpret_cast<float*>(base + STAGES * L::STAGE);
    AxisNode* axj = reinterpret_cast<AxisNode*>(base + STAGES * L::STAGE + 2 * L::HN);  // rows j0-1 .. j0+TJ
    AxisNode* axk = axj + (TJ + 2);                                                    // cols k0-1 .. k0+TK+2
    AxisNode* axi = axk + (TK + 4);                                                    // planes p_first .. i1
    uint64_t* full = reinterpret_cast<uint64_t*>(base + STAGES * L::STAGE + 2 * L::HN + L::AX);
    uint64_t* empty = full + STAGES;
    float* lt = reinterpret_cast<float*>(base + STAGES * L::STAGE + 2 * L::HN + L::AX + L::BARS);
    float* zr_all = reinterpret_cast<float*>(base + STAGES * L::STAGE + 2 * L::HN + L::AX + L::BARS + L::LT);
    float4* zkh = reinterpret_cast<float4*>(base + STAGES * L::STAGE + 2 * L::HN + L::AX + L::BARS + L::LT + L::ZR);
    float4* zke = zkh + (TK + 4);

    const Geom& g = a.g;
    const int tid = threadIdx.x;
    const int bid = a.block0 + int(blockIdx.x);
    const int4 bd = a.blocks[bid];
    const int k0 = bd.x & ~TMA_ZL_TILE, j0 = bd.y, i0 = bd.z, i1 = bd.w;
    const int p_first = i0 > 0 ? i0 - 1 : 0;   // plane i0-1 supplies H(i0-1) for the first E update
    const int p_last = i1;                     // E(i1) for the last H update (zeros past the grid)
    const bool redge = a.kend == g.n2 && k0 + TK == g.n2 - 1;
    if (a.bump && (blockIdx.x | tid) == 0) *a.counter += 1u;   // the step's first kernel opens step n
    const int zc = (TJ + 1) * g.pw;   // ZL: the component stride inside a staged z box

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
        if constexpr (ZL) {
            if (q >= TJ + 2 && q < TJ + 2 + TK + 4) {
                zkh[q - TJ - 2] = make_float4(v.bh, v.ch, v.raw_inv_d, 0.f);
                zke[q - TJ - 2] = make_float4(v.be, v.ce, v.raw_inv_dd, 0.f);
            }
        }
    }
    if constexpr (LOCAL) {
        const float* src = a.tables + (long long)bid * (LOCAL_CLASSES * 6);
        for (int q = tid; q < LOCAL_CLASSES * 6; q += blockDim.x) lt[q] = src[q];
    }
    uint8_t* lm = reinterpret_cast<uint8_t*>(lt + LOCAL_CLASSES * 6);   // FOLD: the entries' Debye masks
    if constexpr (FOLD) {
        static_assert(LOCAL, "the folded Debye ADE reads its masks from the per-block tables");
        for (int q = tid; q < LOCAL_CLASSES; q += blockDim.x) lm[q] = a.lmask[(long long)bid * LOCAL_CLASSES + q];
    }
    __syncthreads();

    if (tid >= TMA_CONSUMERS) {
        // producer warp: one lane issues the copies
        if (tid != TMA_CONSUMERS) return;
        for (int p = p_first; p <= p_last; ++p) {
            const int u = p - p_first, s = u % STAGES, n = u / STAGES;
            if (!tma::mbar_wait(&empty[s], uint32_t((n & 1) ^ 1), a.wait_ns)) {
                atomicExch(a.error, 1);
                // the copies already issued land before the block leaves (bounded waits)
                for (int q = max(p_first, p - STAGES); q < p; ++q) {
                    const int uq = q - p_first;
                    tma::mbar_wait(&full[uq % STAGES], uint32_t((uq / STAGES) & 1), a.wait_ns);
                }
                return;
            }
            unsigned char* st = stages + s * L::STAGE;
            const bool zp = ZL && p < i1;   // plane i1 supplies E only
            tma::mbar_expect_tx(&full[s], L::TX + (zp ? 2 * 2 * zc * 4 : 0) + (p == a.stall_plane ? 16 : 0));
            tma::load_4d(st, &map_e, &full[s], k0 - 4, j0 - 1, p, 0);
            tma::load_4d(st + L::al(L::E_BYTES), &map_h, &full[s], k0 - 4, j0 - 1, p, 0);
            tma::load_3d(st + L::al(L::E_BYTES) + L::al(L::H_BYTES), &map_c, &full[s], k0 & ~15, j0, p);
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
    const int2 orow = a.own_rows ? a.own_rows[bid] : make_int2(j0, a.jend);
    const bool own_row = r >= 0 && jj >= orow.x && jj < orow.y && kk >= a.kbeg && kk < a.kend;   // the pair is written
    const AxisNode* rj = axj + (r + 1);
    const PtAxes q0{rj, axk + (c + 1), jj + 1 < g.n1, kk + 1 < g.n2};
    const PtAxes q1{rj, axk + (c + 2), jj + 1 < g.n1, kk + 2 < g.n2};
    const int eo = (r + 1) * L::EW + c + 4, ho = (r + 1) * L::HW + c + 4, no = (r + 1) * L::NW + c + 2;
    const unsigned goff = unsigned(max(jj, 0)) * unsigned(g.p2) + unsigned(kk);
    // warp 0 extras: the k-1 halo column (lanes 0..TJ-1), the owned right-edge column (lanes
    // TJ..2TJ-1) and that column's j-1 halo point (lane 2TJ)
    const int xr = lane < TJ ? lane : (lane < 2 * TJ ? lane - TJ : -1);  // row of the extra point
    const int xc = lane < TJ ? -1 : TK;                                   // column of the extra point
    const bool xtra = w == 0 && ((lane < TJ && k0 > 0) || (lane >= TJ && lane <= 2 * TJ && redge)) &&
                      j0 + xr >= 0 && j0 + xr < g.n1;
    const bool xown = xtra && lane >= TJ && lane < 2 * TJ && j0 + xr >= orow.x && j0 + xr < orow.y;  // right-edge points are owned
    const int xj = j0 + xr, xk = k0 + xc;
    const PtAxes qx{axj + (xr + 1), axk + (xc + 1), xj + 1 < g.n1, xk + 1 < g.n2};
    const int xeo = (xr + 1) * L::EW + xc + 4, xho = (xr + 1) * L::HW + xc + 4, xno = (xr + 1) * L::NW + xc + 2;
    const unsigned xgoff = unsigned(min(xj, g.n1 - 1)) * unsigned(g.p2) + unsigned(max(xk, 0));

    // the pair's axis factors, kept in registers (the i factors are read per plane)
    const float dj = rj->inv_d, ej = rj->inv_dd;
    const float2 dk2 = make_float2(q0.ak->inv_d, q1.ak->inv_d), ek2 = make_float2(q0.ak->inv_dd, q1.ak->inv_dd);
    float2 pyp = make_float2(0.f, 0.f), pzp = make_float2(0.f, 0.f);   // the pair's H of plane i-1
    const float2 mz = make_float2(a.neg0, a.neg0);
    float pyx = 0.f, pzx = 0.f;                                         // warp 0's extra point's
    bool bad = false;
    // ZL: the tile columns [zc0, zc1) with a live k slot (the layer is contiguous within a tile),
    // the pair's slot flags (bits 0/1: H slot of column c / c + 1, bits 2/3: E slot) and the warp's
    // row buffer of k-layer terms (component 0 at column c, component 1 at TK + c)
    int zc0 = TK, zc1 = 0;
    unsigned zf = 0;
    float* zw = zr_all + w * (2 * TK);
    if constexpr (ZL) {
        const AxisNode &z0 = axk[c + 1], &z1 = axk[c + 2];
        const bool in0 = kk < g.n2, in1 = kk + 1 < g.n2;
        zf = (in0 && z0.slot_h >= 0 ? 1u : 0u) | (in1 && z1.slot_h >= 0 ? 2u : 0u) |
             (in0 && z0.slot_e >= 0 ? 4u : 0u) | (in1 && z1.slot_e >= 0 ? 8u : 0u);
        const bool h0 = (zf & 5u) != 0, h1 = (zf & 10u) != 0;
        zc0 = int(__reduce_min_sync(0xffffffffu, unsigned(h0 ? c : (h1 ? c + 1 : TK))));
        zc1 = int(__reduce_max_sync(0xffffffffu, unsigned(h1 ? c + 2 : (h0 ? c + 1 : 0))));
    }
    // ZL: the lane's own item of the dense passes (t = lane < 2 (zc1 - zc0)), its plane-invariant
    // parts formed once: bit 0 the H term is live (all but the i+1 test), 1 it is stored, 2 the E
    // term is live (all but the class's cb and the i > 0 test); bits 8-14 the column, 15 the
    // component, 16-23 the H slot, 24-31 the E slot; zoe / zoh its offsets in the E box / new-H tile
    unsigned zi = 0;
    int zoe = 0, zoh = 0;
    if constexpr (ZL) {
        const int nz = zc1 - zc0;
        if (lane < 2 * nz) {
            const int cp = lane >= nz ? 1 : 0, cc = zc0 + lane - cp * nz, kq = k0 + cc, kp = k0 + (cc & ~1);
            const AxisNode& ak = axk[cc + 1];
            const bool kn = kq + 1 < g.n2;
            const bool opt = r >= 0 && jj >= orow.x && jj < orow.y && kp >= a.kbeg && kp < a.kend;
            const bool hl = row_live && kq < g.n2 && ak.slot_h >= 0 && (cp ? kn : q0.jn && kn);
            const bool el = opt && row_live && kq < g.n2 && ak.slot_e >= 0 && kq > 0 && (cp || jj > 0);
            zi = (hl ? 1u : 0u) | (hl && opt ? 2u : 0u) | (el ? 4u : 0u) | (unsigned(cc) << 8) | (unsigned(cp) << 15) |
                 (unsigned(max(ak.slot_h, 0)) << 16) | (unsigned(max(ak.slot_e, 0)) << 24);
            zoe = (r + 1) * L::EW + cc + 4 + (cp ? 0 : EC);
            zoh = (r + 1) * L::NW + cc + 2 + (cp ? 0 : NC);
        }
    }
    // FOLD: the row's first folded edge in the next owned plane, loaded a plane ahead
    int fnext = 0;
    if constexpr (FOLD) {
        if (r >= 0) fnext = a.drow[(long long)bid * SEGMAX * 8 + r];
    }
    for (int p = p_first; p < i1; ++p) {
        const int u = p - p_first;
        const int s = u % STAGES, s1 = (u + 1) % STAGES;
        const bool pre = p < i0;  // the plane before the segment: H only, nothing written
        if (!tma::mbar_wait(&full[s], uint32_t((u / STAGES) & 1), a.wait_ns)) bad = true;
        if (!tma::mbar_wait(&full[s1], uint32_t(((u + 1) / STAGES) & 1), a.wait_ns)) bad = true;
        const float* E = reinterpret_cast<const float*>(stages + s * L::STAGE);
        const float* E1 = reinterpret_cast<const float*>(stages + s1 * L::STAGE);
        const float* H = reinterpret_cast<const float*>(stages + s * L::STAGE + L::al(L::E_BYTES));
        // the class box starts at k0 rounded down to 16 ids: column k sits at k - k0 + (k0 & 15)
        const CID* CL = reinterpret_cast<const CID*>(stages + s * L::STAGE + L::al(L::E_BYTES) + L::al(L::H_BYTES)) +
                        (k0 & 15);
        float* hn = hn_all + (u & 1) * (L::HN / 4);
        const float* ZE = ZL ? reinterpret_cast<const float*>(stages + s * L::STAGE + L::PZ_OFF) : nullptr;
        const float* ZH = ZL ? ZE + L::PZ_FIELD / 4 : nullptr;
        const int i = p;
        const AxisNode& ai = axi[u];
        const bool in = i + 1 < g.n0;
        const long long plane = (long long)i * g.n1 * g.p2;
        const bool own = own_row && !pre;

        // the pair's two class ids in one aligned load (c is even)
        unsigned id0 = 0, id1 = 0;
        if (!pre && own_row && live0) {
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
        }
        // FOLD: the pair's folded Debye edges (column c's components, then column c + 1's), their
        // numbers (a scan over the row's lanes) and their dd and state, loaded before the H half so
        // that it hides the loads
        unsigned fm = 0;           // bits 0-2: column c's components, 3-5: column c + 1's
        int fq = 0;
        float fw[6], fs[6];
        if constexpr (FOLD) {
            if (!pre) {
                if (own_row && live0) fm = unsigned(lm[id0]) | (live1 ? unsigned(lm[id1]) << 3 : 0u);
                const int cnt = __popc(fm);
                int x = cnt;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, x, d);
                    if (lane >= d) x += y;
                }
                fq = fnext + (x - cnt);
                int q = fq;
#pragma unroll
                for (int t = 0; t < 6; ++t) {
                    fw[t] = 0.f;
                    fs[t] = 0.f;
                    if (fm >> t & 1u) {
                        fw[t] = a.fdd[q];
                        fs[t] = a.fstate[q];
                        ++q;
                    }
                }
                if (r >= 0 && p + 1 < i1) fnext = a.drow[((long long)bid * SEGMAX + (p + 1 - i0)) * 8 + r];
            }
        }

        // ZL: the row's k-layer H terms (z_terms<1> on every live point of the row's layer columns),
        // one lane per (component, column): component 0 is Hx's (dEy/dk), 1 is Hy's (dEx/dk)
        if constexpr (ZL) {
            const int nz = zc1 - zc0;
            const long long zpl = (long long)i * g.n1 * g.pw;   // the plane's first z-slab row
            __syncwarp();
            if ((zi & 1u) && (!(zi & 0x8000u) || in)) {
                const int cc = int(zi >> 8 & 127u), cp = int(zi >> 15 & 1u), sl = int(zi >> 16 & 255u);
                const float4 f = zkh[cc + 1];
                const float d = E[zoe + 1] - E[zoe];
                const float rv = f.x * ZH[(r + 1) * g.pw + cp * zc + sl] + f.y * d * f.z;
                zw[cp * TK + cc] = rv;
                if ((zi & 2u) && !pre)
                    a.psi_h_out[(cp ? g.psi_off[9 + 1 * 3 + 2] : g.psi_off[9 + 0 * 3 + 2]) + zpl + (jj * g.pw + sl)] = rv;
            }
            for (int t = lane + 32; t < 2 * nz; t += 32) {   // layers wider than 16 columns in a tile
                const int cp = t >= nz ? 1 : 0, cc = zc0 + t - cp * nz, kq = k0 + cc;
                const AxisNode& ak = axk[cc + 1];
                const int sl = ak.slot_h;
                const bool kn = kq + 1 < g.n2;
                if (row_live && kq < g.n2 && sl >= 0 && (cp ? kn && in : q0.jn && kn)) {
                    const int off = (r + 1) * L::EW + cc + 4 + (cp ? 0 : EC);
                    const float d = E[off + 1] - E[off];
                    const float rv = ak.bh * ZH[(r + 1) * g.pw + cp * zc + sl] + ak.ch * d * ak.raw_inv_d;
                    zw[cp * TK + cc] = rv;
                    const int kp = k0 + (cc & ~1);
                    if (!pre && r >= 0 && jj >= orow.x && jj < orow.y && kp >= a.kbeg && kp < a.kend)
                        a.psi_h_out[g.psi_off[9 + cp * 3 + 2] + ((long long)i * g.n1 + jj) * g.pw + sl] = rv;
                }
            }
            __syncwarp();
        }

        // 1. new H: the pair (two columns, one packed update), and warp 0's extra point
        EPair nb{};
        float2 hxp = make_float2(0.f, 0.f), hyp = hxp, hzp = hxp;
        if (live0) {
            nb.x = *reinterpret_cast<const float2*>(E + eo);
            nb.y = *reinterpret_cast<const float2*>(E + EC + eo);
            nb.z = *reinterpret_cast<const float2*>(E + 2 * EC + eo);
            nb.zj = *reinterpret_cast<const float2*>(E + 2 * EC + eo + L::EW);
            nb.xj = *reinterpret_cast<const float2*>(E + eo + L::EW);
            nb.zi = *reinterpret_cast<const float2*>(E1 + 2 * EC + eo);
            nb.yi = *reinterpret_cast<const float2*>(E1 + EC + eo);
            nb.yk = make_float2(nb.y.y, E[EC + eo + 2]);
            nb.xk = make_float2(nb.x.y, E[eo + 2]);
            hxp = *reinterpret_cast<const float2*>(H + ho);
            hyp = *reinterpret_cast<const float2*>(H + HC + ho);
            hzp = *reinterpret_cast<const float2*>(H + 2 * HC + ho);
            h_pair<ZL>(a, mz, nb, hxp, hyp, hzp, ai.inv_d, dj, dk2, q0.jn, q0.kn, q1.kn, in, live1, zw + c, TK, zf);
            *reinterpret_cast<float2*>(hn + no) = hxp;
            *reinterpret_cast<float2*>(hn + NC + no) = hyp;
            *reinterpret_cast<float2*>(hn + 2 * NC + no) = hzp;
            if (own) {
                // a dead second column is padding past n2 and stays zero
                float* o = a.h_out + plane + goff;
                *reinterpret_cast<float2*>(o) = make_float2(hxp.x, live1 ? hxp.y : 0.f);
                *reinterpret_cast<float2*>(o + g.cs) = make_float2(hyp.x, live1 ? hyp.y : 0.f);
                *reinterpret_cast<float2*>(o + 2 * g.cs) = make_float2(hzp.x, live1 ? hzp.y : 0.f);
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
            h_node<ZL>(a, nx, hxx, hyx, hzx, qx, ai, in, ZL ? ZH + (xr + 1) * g.pw : nullptr, zc, i, xj, xown && !pre);
            hn[xno] = hxx;
            hn[NC + xno] = hyx;
            hn[2 * NC + xno] = hzx;
            if (xown && !pre) {
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

        // 2. new E on the owned points
        // ZL: the row's k-layer E terms (z_terms<0> on its owned live points, psi updated in place):
        // component 0 is Ex's (dHy/dk), 1 is Ey's (dHx/dk), from the new H tile
        if constexpr (ZL) {
            if (!pre) {
                const int nz = zc1 - zc0;
                const long long zpl = (long long)i * g.n1 * g.pw;
                __syncwarp();
                if (zi & 4u) {
                    const int cc = int(zi >> 8 & 127u), cp = int(zi >> 15 & 1u), sl = int(zi >> 24);
                    const CoefRef cf = coef_of<LOCAL>(a, lt, CL[r * L::CW + cc]);
                    if ((cp ? cf.cb[1] : cf.cb[0]) != 0.0f && (!cp || i > 0)) {
                        const float4 f = zke[cc + 1];
                        const float d = hn[zoh] - hn[zoh - 1];
                        const float rv = f.x * ZE[(r + 1) * g.pw + cp * zc + sl] + f.y * d * f.z;
                        zw[cp * TK + cc] = rv;
                        a.psi_e[(cp ? g.psi_off[1 * 3 + 2] : g.psi_off[0 * 3 + 2]) + zpl + (jj * g.pw + sl)] = rv;
                    }
                }
                for (int t = lane + 32; t < 2 * nz; t += 32) {
                    const int cp = t >= nz ? 1 : 0, cc = zc0 + t - cp * nz, kq = k0 + cc, kp = k0 + (cc & ~1);
                    const AxisNode& ak = axk[cc + 1];
                    const int sl = ak.slot_e;
                    if (r >= 0 && row_live && kq < g.n2 && sl >= 0 && jj >= orow.x && jj < orow.y && kp >= a.kbeg &&
                        kp < a.kend) {
                        const CoefRef cf = coef_of<LOCAL>(a, lt, CL[r * L::CW + cc]);
                        if ((cp ? cf.cb[1] : cf.cb[0]) != 0.0f && kq > 0 && (cp ? i > 0 : jj > 0)) {
                            const int off = (r + 1) * L::NW + cc + 2 + (cp ? 0 : NC);
                            const float d = hn[off] - hn[off - 1];
                            const float rv = ak.be * ZE[(r + 1) * g.pw + cp * zc + sl] + ak.ce * d * ak.raw_inv_dd;
                            zw[cp * TK + cc] = rv;
                            a.psi_e[g.psi_off[cp * 3 + 2] + ((long long)i * g.n1 + jj) * g.pw + sl] = rv;
                        }
                    }
                }
                __syncwarp();
            }
        }
        if (!pre) {
            if (own_row && live0) {
                const CoefRef cf0 = coef_of<LOCAL>(a, lt, id0);
                const CoefRef cf1 = coef_of<LOCAL>(a, lt, live1 ? id1 : id0);
                const float2 hzj = *reinterpret_cast<const float2*>(hn + 2 * NC + no - L::NW);
                const float2 hxj = *reinterpret_cast<const float2*>(hn + no - L::NW);
                const float2 hyk = make_float2(hn[NC + no - 1], hyp.x), hxk = make_float2(hn[no - 1], hxp.x);
                // a dead second column keeps E = 0
                float2 ex = make_float2(nb.x.x, live1 ? nb.x.y : 0.f), ey = make_float2(nb.y.x, live1 ? nb.y.y : 0.f);
                float2 ez = make_float2(nb.z.x, live1 ? nb.z.y : 0.f);
                e_pair<ZL>(a, mz, cf0, cf1, ex, ey, ez, hxp, hyp, hzp, hzj, hxj, hyk, hxk, pyp, pzp, ai.inv_dd, ej, ek2, i,
                           jj, kk, live1, zw + c, TK, zf);
                if constexpr (FOLD) {
                    if (fm) {   // in the fill's order: column c's components, then column c + 1's
                        int q = fq;
                        if (fm & 1u) fold_edge(a, ex.x, nb.x.x, cf0.cb[0], fw[0], fs[0], q++);
                        if (fm & 2u) fold_edge(a, ey.x, nb.y.x, cf0.cb[1], fw[1], fs[1], q++);
                        if (fm & 4u) fold_edge(a, ez.x, nb.z.x, cf0.cb[2], fw[2], fs[2], q++);
                        if (fm & 8u) fold_edge(a, ex.y, nb.x.y, cf1.cb[0], fw[3], fs[3], q++);
                        if (fm & 16u) fold_edge(a, ey.y, nb.y.y, cf1.cb[1], fw[4], fs[4], q++);
                        if (fm & 32u) fold_edge(a, ez.y, nb.z.y, cf1.cb[2], fw[5], fs[5], q++);
                    }
                }
                float* o = a.e_out + plane + goff;
                *reinterpret_cast<float2*>(o) = ex;
                *reinterpret_cast<float2*>(o + g.cs) = ey;
                *reinterpret_cast<float2*>(o + 2 * g.cs) = ez;
            }
            if (xown) {
                const CoefRef cf = coef_of<LOCAL>(a, lt, CL[xr * L::CW + xc]);
                float ex = nx.x, ey = nx.y, ez = nx.z;
                e_node<ZL>(a, cf, ex, ey, ez, hxx, hyx, hzx, hn[2 * NC + xno - L::NW], hn[xno - L::NW],
                           hn[NC + xno - 1], hn[xno - 1], pyx, pzx, qx, ai, i, xj, xk,
                           ZL ? ZE + (xr + 1) * g.pw : nullptr, zc);
                float* o = a.e_out + plane + xgoff;
                o[0] = ex;
                o[g.cs] = ey;
                o[2 * g.cs] = ez;
            }
        }
        pyp = hyp; pzp = hzp; pyx = hyx; pzx = hzx;
        tma::mbar_arrive(&empty[s]);
    }
    // the last plane's stage (E(i1)) was waited on by the final iteration; nothing is in flight
}

template <int TJ, int TK, typename CID, int STAGES, int SEGMAX, bool LOCAL, int MINB, bool FOLD = false>
__global__ void __launch_bounds__(TMA_CONSUMERS + 32, MINB)
    k_tma_step(const __grid_constant__ CUtensorMap map_e, const __grid_constant__ CUtensorMap map_h,
               const __grid_constant__ CUtensorMap map_c, const __grid_constant__ CUtensorMap map_pze,
               const __grid_constant__ CUtensorMap map_pzh, TmaArgs a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* base = tma::align128(smem_raw);
    if (a.blocks[a.block0 + int(blockIdx.x)].x & TMA_ZL_TILE)
        tma_march<TJ, TK, CID, STAGES, SEGMAX, LOCAL, true, FOLD>(map_e, map_h, map_c, map_pze, map_pzh, a, base);
    else
        tma_march<TJ, TK, CID, STAGES, SEGMAX, LOCAL, false, FOLD>(map_e, map_h, map_c, map_pze, map_pzh, a, base);
}

// One grid of a merged batch launch (k_batch_tma): its tensor maps (64-byte aligned in HBM; a
// copy reads them there as it reads kernel parameters) and its march arguments for each input
// set. block0 is minus the grid's first block in the launch, so a.block0 + blockIdx.x indexes the
// grid's own block list; bump is 0 (the batch opens every grid's step before the march).
struct alignas(128) TmaGrid {
    CUtensorMap e[2], h[2], c, pze, pzh[2];
    TmaArgs a[2];
};

// The TMA march over the clean boxes of many grids in one launch: block b marches a tile of grid
// block_grid[b] with that grid's maps and arguments (copied to shared memory first). One launch
// serves the grids with per-block class tables (LOCAL), another those with global class ids.
template <int TJ, int TK, typename CID, int STAGES, int SEGMAX, bool LOCAL, int MINB>
__global__ void __launch_bounds__(TMA_CONSUMERS + 32, MINB)
    k_batch_tma(const TmaGrid* __restrict__ grids, const int* __restrict__ block_grid, int parity) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    __shared__ __align__(16) TmaArgs sa;
    unsigned char* base = tma::align128(smem_raw);
    const TmaGrid& G = grids[block_grid[blockIdx.x]];
    static_assert(sizeof(TmaArgs) % 4 == 0, "TmaArgs copies as words");
    const int* src = reinterpret_cast<const int*>(&G.a[parity]);
    int* dst = reinterpret_cast<int*>(&sa);
    for (int q = threadIdx.x; q < int(sizeof(TmaArgs) / 4); q += blockDim.x) dst[q] = src[q];
    __syncthreads();
    if (sa.blocks[sa.block0 + int(blockIdx.x)].x & TMA_ZL_TILE)
        tma_march<TJ, TK, CID, STAGES, SEGMAX, LOCAL, true>(G.e[parity], G.h[parity], G.c, G.pze, G.pzh[parity], sa, base);
    else
        tma_march<TJ, TK, CID, STAGES, SEGMAX, LOCAL, false>(G.e[parity], G.h[parity], G.c, G.pze, G.pzh[parity], sa, base);
}

// Host side ---------------------------------------------------------------------------------

struct TmaPlan {
    CUtensorMap e[2], h[2], c;   // per input parity
    CUtensorMap pze, pzh[2];     // the z-slab psi: E slabs, H slabs of the input set per parity
    bool pz = false;
    int tj = 8, tk = 64, seg = 64;
    int blocks = 0;              // blocks of the clean box
    int zblocks = 0;             // of them, the last ones: tiles that reach the k layer
    int shape = 0;               // index into the engine's kernel shapes
    int smem = 0;
    bool ok = false;
    std::string why;
};

}  // namespace fg
