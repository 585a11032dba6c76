// Two time steps per x-sweep (temporal blocking of depth 2) over the interior of the grid.
//
// A block owns a 14 x 64 tile of (j, k) columns over a segment of x-planes [i0, i1) and turns the
// fields of step n (buffer set A) into those of step n + 2 (set C) in one pass, so each node's E
// and H are read from HBM once and written once per two steps. Per x-plane t the consumer warps
// form, on shrinking (j, k) regions (rows / columns relative to the tile's origin):
//   H1 = H^{n+1/2}(t)    rows -2 .. 14, columns -2 .. 64    from E^n(t), E^n(t+1), H^{n-1/2}(t)
//   E1 = E^{n+1}(t)      rows -1 .. 14, columns -1 .. 64    from H1(t) and H1(t-1)
//   H2 = H^{n+3/2}(t-1)  rows -1 .. 13, columns -1 .. 63    from E1(t-1) and E1(t)
//   E2 = E^{n+2}(t-1)    rows  0 .. 13, columns  0 .. 63    from H2(t-1) and H2(t-2)
// (column 64 joins H2 and E2 in a tile that ends the grid with n2 = 64 t + 1 nodes). The regions
// are what the step-(n+2) update of the tile needs, so every block computes its halo itself and
// blocks never wait for each other. The update of each node is that of the one-step kernels
// (cpu.rs:48-167, with the Debye ADE of cpu.rs:239-260 and the k-layer CPML of the z slabs), in the
// same operation order, so both paths give the same bits.
//
// One producer warp streams, per x-plane, E^n (rows -2 .. 15), H^{n-1/2} (rows -2 .. 14), the
// block's class ids and, in tiles that reach the k layer, the z-slab psi of E and H into a ring of
// shared-memory stages with cp.async.bulk.tensor. 17 main warps own one row each (row w - 2), a
// lane the columns lane and lane + 32; 2 edge warps take the 51 points of the extra columns -2, -1
// and 64. A point is always computed by the same thread, so each point's values of the previous
// x-plane stay in registers; neighbours go through shared memory.
//
// Tiles whose halo (two nodes around the tile and two planes around the segment) would reach an
// x- or y-layer of the CPML, a port, probe loop, source or inductor are not run here; the one-step
// kernels update them (and the CPML shell) twice, and two-step tiles next to those ("rim") write
// their step-(n+1) fields (set B) as well so the one-step kernels can read their neighbours.
// The psi of the z slabs and the Debye state live in three time slots: the step from t reads slot
// t mod 3 and writes slot (t + 1) mod 3, so a block's halo never reads a value another block has
// already moved on.
#pragma once

#include "stencil_tma.cuh"

namespace fg {

constexpr int TB_TJ = 14, TB_TK = 64;
constexpr int TB_MAIN = 17;                      // main warps: row w - 2
constexpr int TB_EDGE = 2;                       // edge warps: 51 points of columns -2, -1, 64
constexpr int TB_CONSUMERS = (TB_MAIN + TB_EDGE) * 32;
constexpr int TB_THREADS = TB_CONSUMERS + 32;    // + the producer warp
constexpr int TB_EDGE_POINTS = 51;
constexpr int TB_PZW = 32;                       // z-slab psi row pitch in shared memory (>= pw)
constexpr int TB_CW = 80;                        // class-id row pitch (columns -1 .. 78)
constexpr int TB_SEGMAX = 64;
constexpr int TB_NPMAX = 2;                      // Debye poles the two-step mode takes
constexpr int TB_REC = 12;                       // floats per class record: ca[3], cb[3], dd[3], 3 pad

template <int STAGES>
struct Tb2Layout {
    static constexpr int EW = 72, ER = 18;       // E^n box: columns -4 .. 67, rows -2 .. 15
    static constexpr int HW = 72, HR = 17;       // H^{n-1/2} box: columns -4 .. 67, rows -2 .. 14
    static constexpr int CR = 16;                // class box: rows -1 .. 14, TB_CW columns
    static constexpr int ZHR = 17, ZER = 16;     // z-slab psi boxes: H rows -2 .. 14, E rows -1 .. 14
    static constexpr int BW = 68;                // working buffers' row pitch
    static constexpr int E_BYTES = 3 * ER * EW * 4;
    static constexpr int H_BYTES = 3 * HR * HW * 4;
    static constexpr int C_BYTES = CR * TB_CW;
    __host__ __device__ static constexpr int al(int b) { return (b + 127) & ~127; }
    static constexpr int ZH_BYTES_MAX = 2 * ZHR * TB_PZW * 4;
    static constexpr int ZE_BYTES_MAX = 2 * ZER * TB_PZW * 4;
    static constexpr int OFF_H = al(E_BYTES);
    static constexpr int OFF_C = OFF_H + al(H_BYTES);
    static constexpr int OFF_ZH = OFF_C + al(C_BYTES);
    static constexpr int OFF_ZE = OFF_ZH + al(ZH_BYTES_MAX);
    static constexpr int STAGE = OFF_ZE + al(ZE_BYTES_MAX);
    static constexpr int H1 = al(3 * 17 * BW * 4);           // rows -2 .. 14, columns -2 .. 65
    static constexpr int E1 = al(3 * 16 * BW * 4);           // rows -1 .. 14, columns -1 .. 66 (x2)
    static constexpr int H2 = al(3 * 15 * BW * 4);           // rows -1 .. 13, columns -1 .. 66
    static constexpr int ZH1 = al(2 * 17 * TB_PZW * 4);      // psi H^{n+1/2} of the z slabs (x2)
    static constexpr int ZE1 = al(2 * 16 * TB_PZW * 4);      // psi E^{n+1} of the z slabs (x2)
    static constexpr int NAX = 18 + 68 + (TB_SEGMAX + 4);    // j rows -2 .. 15, k columns -2 .. 65, planes
    static constexpr int AX = al(NAX * int(sizeof(AxisNode)));
    static constexpr int LT = al(LOCAL_CLASSES * TB_REC * 4);   // the block's class records
    static constexpr int BARS = al(2 * STAGES * 8);
    static constexpr int OFF_WORK = STAGES * STAGE;
    static constexpr int OFF_E1 = OFF_WORK + H1;
    static constexpr int OFF_H2 = OFF_E1 + 2 * E1;
    static constexpr int OFF_ZH1 = OFF_H2 + H2;
    static constexpr int OFF_ZE1 = OFF_ZH1 + 2 * ZH1;
    static constexpr int OFF_AX = OFF_ZE1 + 2 * ZE1;
    static constexpr int OFF_LT = OFF_AX + AX;
    static constexpr int OFF_BARS = OFF_LT + LT;
    static constexpr int TOTAL = OFF_BARS + BARS + 128;
};

struct Tb2Args {
    Geom g;
    float k_mu;
    const int4* blocks;          // per block: (k0 | TMA_ZL_TILE | TB_RIM, j0, i0, i1)
    const int* id_base;          // per block: its first plane in the block-major class-id array
    const float* tables;         // per block: LOCAL_CLASSES records of TB_REC floats (ca, cb, dd)
    float* e_out1;               // set B (step n + 1): written by rim tiles only
    float* h_out1;
    float* e_out2;               // set C (step n + 2)
    float* h_out2;
    float* pz_e1;                // z-slab psi, slot of step n + 1 (bases for the psi_off offsets)
    float* pz_h1;
    float* pz_e2;                // slot of step n + 2
    float* pz_h2;
    const unsigned* dbase;       // per device node: its first Debye edge (Debye nodes only)
    const float* dstate_in;      // Debye state, slots of steps n, n + 1, n + 2: [edge * np + pole]
    float* dstate_1;
    float* dstate_2;
    const float* dtable;         // [np, (b_k, c_k) ...] as the one-step Debye kernel reads it
    int* error;
    unsigned long long wait_ns;
};

constexpr int TB_RIM = 1 << 29;  // block flag: also write the step-(n+1) fields of the owned nodes

namespace tb {

// The (ca, cb, dd) record of a local class.
struct Coef9 {
    float ca[3], cb[3], dd[3];
};

__device__ __forceinline__ Coef9 coef9(const float* lt, unsigned id) {
    const float4* t = reinterpret_cast<const float4*>(lt + id * TB_REC);
    const float4 v0 = t[0], v1 = t[1], v2 = t[2];
    Coef9 c;
    c.ca[0] = v0.x; c.ca[1] = v0.y; c.ca[2] = v0.z;
    c.cb[0] = v0.w; c.cb[1] = v1.x; c.cb[2] = v1.y;
    c.dd[0] = v1.z; c.dd[1] = v1.w; c.dd[2] = v2.x;
    return c;
}

// Axis factors of one point.
struct Fac {
    float di, dj, dk;      // inv_d of the i, j, k axes (H update)
    float ei, ej, ek;      // inv_dd (E update)
};

// H at one point (cpu.rs:65-102): h[c] -= k_mu (t[c][0] - t[c][1]), t[c][u] = d[c][u] inv_d of
// axis (c + 1 + u) mod 3; d from E at the point (e0) and at +j (ej), +k (ek), +i (ei). Hx and Hy
// need k + 1 inside the grid (kn); i and j stay inside in this kernel. With ZL the k-layer CPML
// terms join t[0][1] and t[1][0] (psi of the previous half step in zin; the new psi in z0, z1).
template <bool ZL>
__device__ __forceinline__ void h_point(float k_mu, const Fac& f, const float (&e0)[3], float ej_z, float ej_x,
                                        float ek_y, float ek_x, float ei_z, float ei_y, float (&h)[3], bool kn,
                                        const AxisNode* ak, const float* zin0, const float* zin1, float& z0,
                                        float& z1) {
    const float d00 = ej_z - e0[2], d01 = ek_y - e0[1];
    const float d10 = ek_x - e0[0], d11 = ei_z - e0[2];
    const float d20 = ei_y - e0[1], d21 = ej_x - e0[0];
    float t00 = d00 * f.dj, t01 = d01 * f.dk;
    float t10 = d10 * f.dk, t11 = d11 * f.di;
    const float t20 = d20 * f.di, t21 = d21 * f.dj;
    if constexpr (ZL) {
        const int sl = ak->slot_h;
        if (sl >= 0 && kn) {
            z0 = ak->bh * zin0[sl] + ak->ch * d01 * ak->raw_inv_d;
            t01 += z0;
            z1 = ak->bh * zin1[sl] + ak->ch * d10 * ak->raw_inv_d;
            t10 += z1;
        }
    }
    if (kn) {
        h[0] = h[0] - k_mu * (t00 - t01);
        h[1] = h[1] - k_mu * (t10 - t11);
    }
    h[2] = h[2] - k_mu * (t20 - t21);
}

// E at one point (cpu.rs:125-162): e[c] = ca e[c] + cb (t[c][0] - t[c][1]) where cb != 0; Ex and Ey
// need k > 0 (kp). hj, hk: H at -j, -k; hi: H of plane i - 1 (y, z). With ZL the k-layer CPML terms
// of the components that run join t[0][1] and t[1][0] (new psi in z0, z1; 0 for one that does not
// run, whose psi never changes from 0).
template <bool ZL>
__device__ __forceinline__ void e_point(const Fac& f, const Coef9& cf, float (&e)[3], const float (&h)[3], float hj_z,
                                        float hj_x, float hk_y, float hk_x, float hi_y, float hi_z, bool kp,
                                        const AxisNode* ak, const float* zin0, const float* zin1, float& z0,
                                        float& z1) {
    const float d00 = h[2] - hj_z, d01 = h[1] - hk_y;
    const float d10 = h[0] - hk_x, d11 = h[2] - hi_z;
    const float d20 = h[1] - hi_y, d21 = h[0] - hj_x;
    float t00 = d00 * f.ej, t01 = d01 * f.ek;
    float t10 = d10 * f.ek, t11 = d11 * f.ei;
    const float t20 = d20 * f.ei, t21 = d21 * f.ej;
    const bool run0 = cf.cb[0] != 0.0f && kp, run1 = cf.cb[1] != 0.0f && kp;
    if constexpr (ZL) {
        const int sl = ak->slot_e;
        if (sl >= 0) {
            if (run0) {
                z0 = ak->be * zin0[sl] + ak->ce * d01 * ak->raw_inv_dd;
                t01 += z0;
            }
            if (run1) {
                z1 = ak->be * zin1[sl] + ak->ce * d10 * ak->raw_inv_dd;
                t10 += z1;
            }
        }
    }
    if (run0) e[0] = cf.ca[0] * e[0] + cf.cb[0] * (t00 - t01);
    if (run1) e[1] = cf.ca[1] * e[1] + cf.cb[1] * (t10 - t11);
    if (cf.cb[2] != 0.0f) e[2] = cf.ca[2] * e[2] + cf.cb[2] * (t20 - t21);
}

// The Debye ADE of one point's Debye edges (cpu.rs:239-260, as the one-step kernel forms it):
// e -= cb sum_k (1 + b_k)/2 s_k, then s_k' = b_k s_k + dd c_k (e - e_old), for the components with
// dd != 0 in component order; their states follow each other from edge `base` on.
__device__ __forceinline__ void debye_point(const Coef9& cf, float (&e)[3], const float (&e_old)[3], unsigned base,
                                            const float* table, const float* sin, float* sout) {
    const int np = int(table[0]);
    unsigned q = base;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        if (cf.dd[c] == 0.0f) continue;
        float s0 = 0.0f;
        for (int k = 0; k < np; ++k) s0 += 0.5f * (1.0f + table[1 + 2 * k]) * sin[(size_t)q * np + k];
        const float next = e[c] - cf.cb[c] * s0;
        e[c] = next;
        const float de = next - e_old[c];
        const float w = cf.dd[c];
        if (sout)
            for (int k = 0; k < np; ++k)
                sout[(size_t)q * np + k] = table[1 + 2 * k] * sin[(size_t)q * np + k] + w * table[2 + 2 * k] * de;
        ++q;
    }
}

__device__ __forceinline__ bool has_debye(const Coef9& cf) { return cf.dd[0] != 0.0f || cf.dd[1] != 0.0f || cf.dd[2] != 0.0f; }

}  // namespace tb

// One block's two-step march. ZL: the tile reaches the k layer (z-slab psi staged and updated).
template <int STAGES, bool ZL>
__device__ __forceinline__ void tb2_march(const CUtensorMap& map_e, const CUtensorMap& map_h, const CUtensorMap& map_c,
                                          const CUtensorMap& map_zh, const CUtensorMap& map_ze, const Tb2Args& a,
                                          unsigned char* base) {
    using L = Tb2Layout<STAGES>;
    const Geom& g = a.g;
    const int tid = threadIdx.x;
    const int4 bd = a.blocks[blockIdx.x];
    const bool rim = (bd.x & TB_RIM) != 0;
    const int k0 = bd.x & ~(TMA_ZL_TILE | TB_RIM), j0 = bd.y, i0 = bd.z, i1 = bd.w;
    const int p_first = i0 - 2, p_last = i1 + 1;       // planes streamed
    const bool redge = k0 + TB_TK == g.n2 - 1;         // column 64 is the grid's last node, owned here
    const int pw = g.pw;

    float* h1s = reinterpret_cast<float*>(base + L::OFF_WORK);
    float* e1s = reinterpret_cast<float*>(base + L::OFF_E1);
    float* h2s = reinterpret_cast<float*>(base + L::OFF_H2);
    float* zh1s = reinterpret_cast<float*>(base + L::OFF_ZH1);
    float* ze1s = reinterpret_cast<float*>(base + L::OFF_ZE1);
    AxisNode* axj = reinterpret_cast<AxisNode*>(base + L::OFF_AX);   // rows -2 .. 15
    AxisNode* axk = axj + 18;                                        // columns -2 .. 65
    AxisNode* axi = axk + 68;                                        // planes p_first ..
    float* lt = reinterpret_cast<float*>(base + L::OFF_LT);
    uint64_t* full = reinterpret_cast<uint64_t*>(base + L::OFF_BARS);
    uint64_t* empty = full + STAGES;

    if (tid == 0) {
        for (int s = 0; s < STAGES; ++s) {
            tma::mbar_init(&full[s], 1);
            tma::mbar_init(&empty[s], TB_CONSUMERS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    for (int q = tid; q < L::NAX; q += blockDim.x) {
        AxisNode v;
        if (q < 18) v = g.ax[1][min(max(j0 - 2 + q, 0), g.n1 - 1)];
        else if (q < 18 + 68) v = g.ax[2][min(max(k0 - 2 + (q - 18), 0), g.n2 - 1)];
        else v = g.ax[0][min(p_first + (q - 86), g.n0 - 1)];
        axj[q] = v;
    }
    {
        const float4* src = reinterpret_cast<const float4*>(a.tables + (long long)blockIdx.x * (LOCAL_CLASSES * TB_REC));
        float4* dst = reinterpret_cast<float4*>(lt);
        for (int q = tid; q < LOCAL_CLASSES * TB_REC / 4; q += blockDim.x) dst[q] = src[q];
    }
    __syncthreads();

    const int idb = a.id_base[blockIdx.x];
    const int zhb = 2 * L::ZHR * pw * 4, zeb = 2 * L::ZER * pw * 4;   // bytes of the staged z boxes

    if (tid >= TB_CONSUMERS) {
        if (tid != TB_CONSUMERS) return;
        for (int p = p_first; p <= p_last; ++p) {
            const int u = p - p_first, s = u % STAGES, n = u / STAGES;
            if (!tma::mbar_wait(&empty[s], uint32_t((n & 1) ^ 1), a.wait_ns)) {
                atomicExch(a.error, 3);
                // the copies already issued land before the block leaves (bounded waits)
                for (int q = max(p_first, p - STAGES); q < p; ++q) {
                    const int uq = q - p_first;
                    tma::mbar_wait(&full[uq % STAGES], uint32_t((uq / STAGES) & 1), a.wait_ns);
                }
                return;
            }
            unsigned char* st = base + s * L::STAGE;
            const bool cls = p >= i0 - 1 && p <= i1;          // planes whose E1 is formed
            const bool zh = ZL && p <= i1, ze = ZL && cls;
            tma::mbar_expect_tx(&full[s], L::E_BYTES + L::H_BYTES + (cls ? L::C_BYTES : 0) + (zh ? zhb : 0) +
                                              (ze ? zeb : 0));
            tma::load_4d(st, &map_e, &full[s], k0 - 4, j0 - 2, p, 0);
            tma::load_4d(st + L::OFF_H, &map_h, &full[s], k0 - 4, j0 - 2, p, 0);
            if (cls) tma::load_3d(st + L::OFF_C, &map_c, &full[s], 0, 0, idb + (p - (i0 - 1)));
            if (zh) tma::load_4d(st + L::OFF_ZH, &map_zh, &full[s], 0, j0 - 2, p, 0);
            if (ze) tma::load_4d(st + L::OFF_ZE, &map_ze, &full[s], 0, j0 - 1, p, 0);
        }
        return;
    }

    // ---- consumers
    const int w = tid >> 5, lane = tid & 31;
    const bool main_w = w < TB_MAIN;
    constexpr int EC = L::ER * L::EW, HC = L::HR * L::HW, BW = L::BW;
    constexpr int H1C = 17 * BW, E1C = 16 * BW, H2C = 15 * BW;
    // The points of this thread. Main warps: row w - 2, columns lane and lane + 32 (a warp's lanes
    // touch 32 consecutive words of every buffer: no bank conflicts). Edge warps: one point each.
    int npt, r, cpt[2];
    if (main_w) {
        npt = 2;
        r = w - 2;
        cpt[0] = lane;
        cpt[1] = lane + 32;
    } else {
        const int q = (w - TB_MAIN) * 32 + lane;
        npt = q < TB_EDGE_POINTS ? 1 : 0;
        const int sel = q / 17;
        r = q % 17 - 2;
        cpt[0] = sel == 0 ? -2 : (sel == 1 ? -1 : 64);
        cpt[1] = cpt[0];
    }
    const int jj = j0 + r;
    // the half steps each point takes part in (the two points of a main thread share them)
    bool do_h1 = npt > 0, do_e1, do_h2, do_e2;
    if (main_w) {
        do_e1 = r >= -1;
        do_h2 = r >= -1 && r <= 13;
        do_e2 = r >= 0 && r <= 13;
    } else {
        const int c = cpt[0];
        do_e1 = npt > 0 && c != -2 && r >= -1;
        do_h2 = npt > 0 && r >= -1 && r <= 13 && (c == -1 || (c == 64 && redge));
        do_e2 = npt > 0 && r >= 0 && r <= 13 && c == 64 && redge;
    }
    const bool own_row = r >= 0 && r < TB_TJ;
    // per point: liveness, guards, k-axis factors; the second point of a main thread sits 32
    // columns right of the first, so its offsets are the first's + 32
    const int c0 = cpt[0];
    bool live[2], kn[2], kp[2], own[2];
    float dk[2], ek[2];
    const AxisNode& aj = axj[r + 2];
    const float dj = aj.inv_d, ej = aj.inv_dd;
#pragma unroll
    for (int q = 0; q < 2; ++q) {
        const int c = c0 + 32 * q;
        const int k = k0 + c;
        live[q] = q < npt && k >= 0 && k < g.n2;
        kn[q] = k + 1 < g.n2;
        kp[q] = k > 0;
        own[q] = live[q] && own_row && (c < TB_TK || (c == TB_TK && redge)) && c >= 0;
        const AxisNode* an = axk + min(max(c + 2, 0), 67);
        dk[q] = an->inv_d;
        ek[q] = an->inv_dd;
    }
    const int eo0 = (r + 2) * L::EW + (c0 + 4);    // E^n / H^{n-1/2} boxes (same pitch)
    const int b20 = (r + 2) * BW + (c0 + 2);       // H1 buffer (rows -2 ..)
    const int b10 = (r + 1) * BW + (c0 + 1);       // E1 and H2 buffers (rows -1 ..)
    const int cl0 = (r + 1) * TB_CW + (c0 + 1);    // class ids
    const long long rowg = (long long)jj * g.p2 + (k0 + c0);
    const long long psi_row = (long long)jj * pw;   // + plane * n1 * pw

    float h1p[2][3] = {{0, 0, 0}, {0, 0, 0}};   // H1 of the previous plane at the point
    float h2p[2][3] = {{0, 0, 0}, {0, 0, 0}};   // H2 of the previous plane at the point
    unsigned cidp[2] = {0u, 0u};                // the point's class id in the previous plane
    bool bad = false;

    for (int t = p_first; t <= i1; ++t) {
        const int u = t - p_first;
        const int s = u % STAGES, s1 = (u + 1) % STAGES;
        if (!tma::mbar_wait(&full[s], uint32_t((u / STAGES) & 1), a.wait_ns)) bad = true;
        if (!tma::mbar_wait(&full[s1], uint32_t(((u + 1) / STAGES) & 1), a.wait_ns)) bad = true;
        const float* E0 = reinterpret_cast<const float*>(base + s * L::STAGE);
        const float* E0n = reinterpret_cast<const float*>(base + s1 * L::STAGE);
        const float* H0 = reinterpret_cast<const float*>(base + s * L::STAGE + L::OFF_H);
        const unsigned char* CL = base + s * L::STAGE + L::OFF_C;
        const float* ZH0 = reinterpret_cast<const float*>(base + s * L::STAGE + L::OFF_ZH);
        const float* ZE0 = reinterpret_cast<const float*>(base + s * L::STAGE + L::OFF_ZE);
        const float di = axi[u].inv_d, ei = axi[u].inv_dd;
        const float dim = axi[u > 0 ? u - 1 : 0].inv_d, eim = axi[u > 0 ? u - 1 : 0].inv_dd;
        float* e1cur = e1s + (t & 1) * (L::E1 / 4);
        const float* e1prv = e1s + ((t - 1) & 1) * (L::E1 / 4);
        float* zh1cur = zh1s + (t & 1) * (L::ZH1 / 4);
        const float* zh1prv = zh1s + ((t - 1) & 1) * (L::ZH1 / 4);
        float* ze1cur = ze1s + (t & 1) * (L::ZE1 / 4);
        const float* ze1prv = ze1s + ((t - 1) & 1) * (L::ZE1 / 4);
        const long long plane = (long long)t * g.n1 * g.p2 + rowg;
        const long long planem = (long long)(t - 1) * g.n1 * g.p2 + rowg;
        const long long zp = (long long)t * g.n1 * pw + psi_row, zpm = (long long)(t - 1) * g.n1 * pw + psi_row;
        const bool owned_t = t >= i0 && t < i1;       // plane t is owned (H1, E1 rim writes)
        const bool owned_tm = t - 1 >= i0 && t - 1 < i1;

        // 1. H1(t)
        float h1c[2][3] = {{0, 0, 0}, {0, 0, 0}};
        if (do_h1) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (!live[q]) continue;
                const int o = eo0 + 32 * q;
                const float e0[3] = {E0[o], E0[EC + o], E0[2 * EC + o]};
                float h[3] = {H0[o], H0[HC + o], H0[2 * HC + o]};
                const tb::Fac f{di, dj, dk[q], 0.f, 0.f, 0.f};
                const float* zin0 = ZH0 + (r + 2) * pw;
                float z0 = 0.f, z1 = 0.f;
                tb::h_point<ZL>(a.k_mu, f, e0, E0[2 * EC + o + L::EW], E0[o + L::EW], E0[EC + o + 1], E0[o + 1],
                                E0n[2 * EC + o], E0n[EC + o], h, kn[q], (axk + min(max(c0 + 32 * q + 2, 0), 67)), zin0, zin0 + L::ZHR * pw, z0, z1);
                const int bo = b20 + 32 * q;
                h1s[bo] = h[0];
                h1s[H1C + bo] = h[1];
                h1s[2 * H1C + bo] = h[2];
                h1c[q][0] = h[0];
                h1c[q][1] = h[1];
                h1c[q][2] = h[2];
                const int sl = ZL ? (axk + min(max(c0 + 32 * q + 2, 0), 67))->slot_h : -1;
                if (ZL && sl >= 0 && kn[q]) {
                    zh1cur[(r + 2) * TB_PZW + sl] = z0;
                    zh1cur[17 * TB_PZW + (r + 2) * TB_PZW + sl] = z1;
                }
                if (rim && own[q] && owned_t) {
                    float* out = a.h_out1 + plane + 32 * q;
                    out[0] = h[0];
                    out[g.cs] = h[1];
                    out[2 * g.cs] = h[2];
                    if (ZL && sl >= 0 && kn[q]) {
                        a.pz_h1[g.psi_off[9 + 0 * 3 + 2] + zp + sl] = z0;
                        a.pz_h1[g.psi_off[9 + 1 * 3 + 2] + zp + sl] = z1;
                    }
                }
            }
        }
        if (tma::consumers_sync_or(bad, TB_CONSUMERS)) {
            if (tid == 0) atomicExch(a.error, 4);
            return;
        }

        // 2. E1(t) (from plane i0 - 1 on)
        const bool e1_plane = t >= i0 - 1;
        float e1c[2][3] = {{0, 0, 0}, {0, 0, 0}};
        unsigned cidc[2] = {0u, 0u};
        if (do_e1 && e1_plane) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (!live[q]) continue;
                const int o = eo0 + 32 * q, bo = b20 + 32 * q;
                const float e_old[3] = {E0[o], E0[EC + o], E0[2 * EC + o]};
                float e[3] = {e_old[0], e_old[1], e_old[2]};
                cidc[q] = CL[cl0 + 32 * q];
                const tb::Coef9 cf = tb::coef9(lt, cidc[q]);
                const tb::Fac f{0.f, 0.f, 0.f, ei, ej, ek[q]};
                const float* zin0 = ZE0 + (r + 1) * pw;
                float z0 = 0.f, z1 = 0.f;
                tb::e_point<ZL>(f, cf, e, h1c[q], h1s[2 * H1C + bo - BW], h1s[bo - BW], h1s[H1C + bo - 1], h1s[bo - 1],
                                h1p[q][1], h1p[q][2], kp[q], (axk + min(max(c0 + 32 * q + 2, 0), 67)), zin0, zin0 + L::ZER * pw, z0, z1);
                const bool keep = own[q] && owned_t;
                if (tb::has_debye(cf)) {
                    // owned points keep s^{n+1} for their E2 (slot of step n + 1)
                    tb::debye_point(cf, e, e_old, a.dbase[plane + 32 * q], a.dtable, a.dstate_in,
                                    keep ? a.dstate_1 : nullptr);
                }
                const int bo1 = b10 + 32 * q;
                e1cur[bo1] = e[0];
                e1cur[E1C + bo1] = e[1];
                e1cur[2 * E1C + bo1] = e[2];
                e1c[q][0] = e[0];
                e1c[q][1] = e[1];
                e1c[q][2] = e[2];
                const int sl = ZL ? (axk + min(max(c0 + 32 * q + 2, 0), 67))->slot_e : -1;
                if (ZL && sl >= 0) {
                    ze1cur[(r + 1) * TB_PZW + sl] = z0;
                    ze1cur[16 * TB_PZW + (r + 1) * TB_PZW + sl] = z1;
                }
                if (rim && keep) {
                    float* out = a.e_out1 + plane + 32 * q;
                    out[0] = e[0];
                    out[g.cs] = e[1];
                    out[2 * g.cs] = e[2];
                    if (ZL && sl >= 0) {
                        a.pz_e1[g.psi_off[0 * 3 + 2] + zp + sl] = z0;
                        a.pz_e1[g.psi_off[1 * 3 + 2] + zp + sl] = z1;
                    }
                }
            }
        }
        // the stage of plane t has been read for the last time (E^n(t) also fed H1(t - 1), done)
        tma::mbar_arrive(&empty[s]);

        // 3. H2(t - 1) (planes i0 - 1 .. i1 - 1)
        const bool h2_plane = t - 1 >= i0 - 1;
        float h2c[2][3] = {{0, 0, 0}, {0, 0, 0}};
        if (do_h2 && h2_plane) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (!live[q]) continue;
                const int bo1 = b10 + 32 * q;
                const float e0[3] = {e1prv[bo1], e1prv[E1C + bo1], e1prv[2 * E1C + bo1]};
                float h[3] = {h1p[q][0], h1p[q][1], h1p[q][2]};
                const tb::Fac f{dim, dj, dk[q], 0.f, 0.f, 0.f};
                const float* zin0 = zh1prv + (r + 2) * TB_PZW;
                float z0 = 0.f, z1 = 0.f;
                tb::h_point<ZL>(a.k_mu, f, e0, e1prv[2 * E1C + bo1 + BW], e1prv[bo1 + BW], e1prv[E1C + bo1 + 1],
                                e1prv[bo1 + 1], e1c[q][2], e1c[q][1], h, kn[q], (axk + min(max(c0 + 32 * q + 2, 0), 67)), zin0, zin0 + 17 * TB_PZW, z0,
                                z1);
                h2s[bo1] = h[0];
                h2s[H2C + bo1] = h[1];
                h2s[2 * H2C + bo1] = h[2];
                h2c[q][0] = h[0];
                h2c[q][1] = h[1];
                h2c[q][2] = h[2];
                if (own[q] && owned_tm) {
                    float* out = a.h_out2 + planem + 32 * q;
                    out[0] = h[0];
                    out[g.cs] = h[1];
                    out[2 * g.cs] = h[2];
                    const int sl = ZL ? (axk + min(max(c0 + 32 * q + 2, 0), 67))->slot_h : -1;
                    if (ZL && sl >= 0 && kn[q]) {
                        a.pz_h2[g.psi_off[9 + 0 * 3 + 2] + zpm + sl] = z0;
                        a.pz_h2[g.psi_off[9 + 1 * 3 + 2] + zpm + sl] = z1;
                    }
                }
            }
        }
        if (tma::consumers_sync_or(bad, TB_CONSUMERS)) {
            if (tid == 0) atomicExch(a.error, 4);
            return;
        }

        // 4. E2(t - 1) (owned planes i0 .. i1 - 1)
        if (do_e2 && owned_tm) {
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                if (!own[q]) continue;
                const int bo1 = b10 + 32 * q;
                const float e_old[3] = {e1prv[bo1], e1prv[E1C + bo1], e1prv[2 * E1C + bo1]};
                float e[3] = {e_old[0], e_old[1], e_old[2]};
                const tb::Coef9 cf = tb::coef9(lt, cidp[q]);
                const tb::Fac f{0.f, 0.f, 0.f, eim, ej, ek[q]};
                const float* zin0 = ze1prv + (r + 1) * TB_PZW;
                float z0 = 0.f, z1 = 0.f;
                tb::e_point<ZL>(f, cf, e, h2c[q], h2s[2 * H2C + bo1 - BW], h2s[bo1 - BW], h2s[H2C + bo1 - 1],
                                h2s[bo1 - 1], h2p[q][1], h2p[q][2], kp[q], (axk + min(max(c0 + 32 * q + 2, 0), 67)), zin0, zin0 + 16 * TB_PZW, z0, z1);
                if (tb::has_debye(cf))
                    tb::debye_point(cf, e, e_old, a.dbase[planem + 32 * q], a.dtable, a.dstate_1, a.dstate_2);
                float* out = a.e_out2 + planem + 32 * q;
                out[0] = e[0];
                out[g.cs] = e[1];
                out[2 * g.cs] = e[2];
                const int sl = ZL ? (axk + min(max(c0 + 32 * q + 2, 0), 67))->slot_e : -1;
                if (ZL && sl >= 0) {
                    a.pz_e2[g.psi_off[0 * 3 + 2] + zpm + sl] = z0;
                    a.pz_e2[g.psi_off[1 * 3 + 2] + zpm + sl] = z1;
                }
            }
        }
        // this plane's values become the previous plane's
#pragma unroll
        for (int q = 0; q < 2; ++q) {
            cidp[q] = cidc[q];
            for (int cc = 0; cc < 3; ++cc) {
                h1p[q][cc] = h1c[q][cc];
                h2p[q][cc] = h2c[q][cc];
            }
        }
    }
}

template <int STAGES>
__global__ void __launch_bounds__(TB_THREADS, 1)
    k_tb2_step(const __grid_constant__ CUtensorMap map_e, const __grid_constant__ CUtensorMap map_h,
               const __grid_constant__ CUtensorMap map_c, const __grid_constant__ CUtensorMap map_zh,
               const __grid_constant__ CUtensorMap map_ze, Tb2Args a) {
    extern __shared__ __align__(128) unsigned char smem_raw[];
    unsigned char* base = tma::align128(smem_raw);
    if (a.blocks[blockIdx.x].x & TMA_ZL_TILE)
        tb2_march<STAGES, true>(map_e, map_h, map_c, map_zh, map_ze, a, base);
    else
        tb2_march<STAGES, false>(map_e, map_h, map_c, map_zh, map_ze, a, base);
}

}  // namespace fg
