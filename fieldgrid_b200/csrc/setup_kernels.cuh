// Device-side parts of session set-up (pack(), run.rs:205-376, in the device layout): the
// per-block class tables of the TMA march and the Debye edge list, both formed in HBM from the
// node classes once they are uploaded, so the host neither builds nor uploads them.
#pragma once

#include <cstdint>

#include "host.hpp"
#include "kernels.cuh"
#include "stencil_tma.cuh"

namespace fg {

constexpr int LC_SLOTS = 512;                 // open-addressing slots per block region
constexpr unsigned LC_EMPTY = 0xffffffffu;

// One CTA per march block region (its owned rows and columns over its planes): the distinct
// global classes of the region, ranked in increasing id order, become the region's table of at
// most LOCAL_CLASSES (ca[3], cb[3]) entries and each owned node's 8-bit local id. With node masks
// (dmask: bit c set where the node's E_c carries a Debye edge) the entries are the distinct
// (class, mask) pairs and lmask gets each entry's mask. A region with more entries sets *over and
// writes nothing; the host then keeps the global ids. Classes are below 2^29 - 1 with masks.
template <typename CID>
__global__ void __launch_bounds__(256) k_local_classes(const CID* __restrict__ node_class,
                                                       const DevCoef* __restrict__ classes,
                                                       const int4* __restrict__ blocks, const int2* __restrict__ own,
                                                       int n1, int n2, int p2, int tk, int lo2, int hi2,
                                                       uint8_t* __restrict__ ids, float* __restrict__ tables,
                                                       int* over, const uint8_t* __restrict__ dmask = nullptr,
                                                       uint8_t* __restrict__ lmask = nullptr) {
    __shared__ unsigned keys[LC_SLOTS];
    __shared__ unsigned short rank[LC_SLOTS];
    __shared__ int count;
    const int r = blockIdx.x;
    const int4 b = blocks[r];
    const int k0 = b.x & ~TMA_ZL_TILE, i0 = b.z, i1 = b.w;
    const int kbeg = max(k0, lo2);
    int kend = min(k0 + tk, hi2);
    if (hi2 == n2 && k0 + tk == n2 - 1) kend = n2;   // the owned right-edge column
    const int jbeg = own[r].x, jend = own[r].y;
    for (int q = threadIdx.x; q < LC_SLOTS; q += blockDim.x) keys[q] = LC_EMPTY;
    if (threadIdx.x == 0) count = 0;
    __syncthreads();
    volatile unsigned* vkeys = keys;
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int nj = max(jend - jbeg, 0);
    const int rows = (i1 - i0) * nj;

    // pass 1: insert every owned node's class (a lane skips a repeat of its previous one)
    bool full = false;
    unsigned last = LC_EMPTY;
    for (int row = w; row < rows && !full; row += nw) {
        const size_t base = (size_t(i0 + row / nj) * n1 + size_t(jbeg + row % nj)) * p2;
        for (int k = kbeg + lane; k < kend && !full; k += 32) {
            const unsigned gid = unsigned(node_class[base + k]) | (dmask ? unsigned(dmask[base + k]) << 29 : 0u);
            if (gid == last) continue;
            last = gid;
            unsigned h = (gid * 2654435761u) & (LC_SLOTS - 1);
            for (int probe = 0;; ++probe) {
                if (probe == LC_SLOTS) { full = true; break; }
                unsigned cur = vkeys[h];
                if (cur == LC_EMPTY) {
                    cur = atomicCAS(&keys[h], LC_EMPTY, gid);
                    if (cur == LC_EMPTY) { atomicAdd(&count, 1); break; }
                }
                if (cur == gid) break;
                h = (h + 1) & (LC_SLOTS - 1);
            }
        }
    }
    if (__syncthreads_or(full) || count > LOCAL_CLASSES) {
        if (threadIdx.x == 0) atomicExch(over, 1);
        return;
    }

    // ranks (the number of smaller keys) and the region's table
    float* tab = tables + size_t(r) * (LOCAL_CLASSES * 6);
    for (int q = threadIdx.x; q < LC_SLOTS; q += blockDim.x) {
        const unsigned key = keys[q];
        if (key == LC_EMPTY) continue;
        int rk = 0;
        for (int t = 0; t < LC_SLOTS; ++t) rk += (keys[t] != LC_EMPTY && keys[t] < key) ? 1 : 0;
        rank[q] = (unsigned short)rk;
        const DevCoef c = classes[dmask ? (key & 0x1fffffffu) : key];
        if (lmask) lmask[size_t(r) * LOCAL_CLASSES + rk] = uint8_t(key >> 29);
#pragma unroll
        for (int m = 0; m < 3; ++m) {
            tab[rk * 6 + m] = c.ca[m];
            tab[rk * 6 + 3 + m] = c.cb[m];
        }
    }
    __syncthreads();

    // pass 2: the local ids (every key is present, so each lookup ends within LC_SLOTS probes)
    last = LC_EMPTY;
    uint8_t last_id = 0;
    for (int row = w; row < rows; row += nw) {
        const size_t base = (size_t(i0 + row / nj) * n1 + size_t(jbeg + row % nj)) * p2;
        for (int k = kbeg + lane; k < kend; k += 32) {
            const unsigned gid = unsigned(node_class[base + k]) | (dmask ? unsigned(dmask[base + k]) << 29 : 0u);
            if (gid != last) {
                unsigned h = (gid * 2654435761u) & (LC_SLOTS - 1);
                for (int probe = 0; probe < LC_SLOTS && keys[h] != gid; ++probe) h = (h + 1) & (LC_SLOTS - 1);
                last = gid;
                last_id = uint8_t(rank[h]);
            }
            ids[base + k] = last_id;
        }
    }
}

// The Debye edge list of the one-step scheme from the host's edge records (run.rs:291-295): the
// device index of each edge's E component, its dd in f32 and the cb of its node class.
template <typename CID>
__global__ void k_debye_lists(const DebyeEdge* __restrict__ edges, long long ne, const CID* __restrict__ node_class,
                              const DevCoef* __restrict__ classes, long long n2, long long p2, long long cs,
                              long long* __restrict__ f, float* __restrict__ dd, float* __restrict__ cb) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ne;
         q += (long long)gridDim.x * blockDim.x) {
        const DebyeEdge d = edges[q];
        const long long dev = (long long)(d.id / uint64_t(n2)) * p2 + (long long)(d.id % uint64_t(n2));
        f[q] = (long long)d.comp * cs + dev;
        dd[q] = float(d.dd);
        cb[q] = classes[unsigned(node_class[dev])].cb[d.comp];
    }
}

// The Debye records as staged to the device: the E component in the top two bits and the device
// node index below (grids of fewer than 2^30 device nodes), dd already rounded to f32 (the
// conversion k_debye_lists makes). 8 bytes against the host record's 24.
struct PackedDebye {
    uint32_t key;
    float dd;
};

template <typename CID>
__global__ void k_debye_lists_packed(const PackedDebye* __restrict__ edges, long long ne,
                                     const CID* __restrict__ node_class, const DevCoef* __restrict__ classes,
                                     long long cs, long long* __restrict__ f, float* __restrict__ dd,
                                     float* __restrict__ cb) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ne;
         q += (long long)gridDim.x * blockDim.x) {
        const PackedDebye d = edges[q];
        const unsigned comp = d.key >> 30;
        const long long dev = (long long)(d.key & 0x3fffffffu);
        f[q] = (long long)comp * cs + dev;
        dd[q] = d.dd;
        cb[q] = classes[unsigned(node_class[dev])].cb[comp];
    }
}

// ---- the Debye ADE folded into the TMA march's E half ----
//
// Folded edges are the Debye edges at the nodes a march block writes through its column pairs
// (owned rows and planes, columns kbeg .. kend - 1 of the tile): the march applies their ADE right
// after their E update. They are numbered per block, owned plane and row, and within a row by
// column then component: the order the march's lanes meet them (a lane's two columns, each's
// components in turn). The other Debye edges (the shell's, a tile's right-edge column) keep the
// edge-list kernel.

constexpr unsigned FOLD_TAKEN = 0x7fc0f01du;   // a NaN payload no dd has: marks a folded edge

// Each Debye edge's component bit in its node's byte (4 nodes per word) and its dd in the
// per-(component, node) scratch ddn (the layout of a field buffer).
__global__ void k_debye_node_mask(const long long* __restrict__ f, const float* __restrict__ dd, long long ne,
                                  long long cs, unsigned* __restrict__ mask_words, float* __restrict__ ddn) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ne;
         q += (long long)gridDim.x * blockDim.x) {
        const long long fi = f[q];
        const long long c = fi / cs, dev = fi - c * cs;
        atomicOr(&mask_words[dev >> 2], (1u << unsigned(c)) << unsigned((dev & 3) * 8));
        ddn[fi] = dd[q];
    }
}

// One CTA per block, a warp per (owned plane, row) at a time, a lane per column pair as in the
// march: COUNT writes each row's folded-edge count to rows[(block * segmax + plane) * 8 + row];
// FILL takes rows as the exclusive prefix sums and writes each folded edge's dd in march order,
// marking it taken in ddn.
template <bool FILL>
__global__ void __launch_bounds__(256) k_fold_rows(const int4* __restrict__ blocks, const int2* __restrict__ own,
                                                   int n1, int n2, int p2, int tj, int tk, int kbeg, int kend,
                                                   int segmax, const uint8_t* __restrict__ dmask, long long cs,
                                                   int* __restrict__ rows, float* __restrict__ ddn,
                                                   float* __restrict__ fdd) {
    const int bid = blockIdx.x;
    const int4 b = blocks[bid];
    const int k0 = b.x & ~TMA_ZL_TILE, j0 = b.y, i0 = b.z, i1 = b.w;
    const int2 orow = own[bid];
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int kk = k0 + 2 * lane;
    for (int u = 0; u < i1 - i0; ++u)
        for (int r = w; r < tj; r += nw) {
            const int jj = j0 + r;
            const bool owned = jj >= orow.x && jj < orow.y && kk >= kbeg && kk < kend && kk < n2 && 2 * lane < tk;
            const bool live1 = kk + 1 < n2;
            const long long dev = ((long long)(i0 + u) * n1 + jj) * p2 + kk;
            unsigned m0 = 0, m1 = 0;
            if (owned) {
                m0 = dmask[dev];
                m1 = live1 ? dmask[dev + 1] : 0u;
            }
            const int cnt = __popc(m0) + __popc(m1);
            int x = cnt;
            for (int d = 1; d < 32; d <<= 1) {
                const int y = __shfl_up_sync(0xffffffffu, x, d);
                if (lane >= d) x += y;
            }
            const long long idx = ((long long)bid * segmax + u) * 8 + r;
            if (!FILL) {
                const int total = __shfl_sync(0xffffffffu, x, 31);
                if (lane == 0) rows[idx] = total;
            } else if (cnt) {
                long long q = (long long)rows[idx] + (x - cnt);
                for (int col = 0; col < 2; ++col) {
                    const unsigned m = col ? m1 : m0;
                    for (int c = 0; c < 3; ++c)
                        if (m >> c & 1u) {
                            float* slot = ddn + (long long)c * cs + dev + col;
                            fdd[q++] = *slot;
                            *slot = __uint_as_float(FOLD_TAKEN);
                        }
                }
            }
        }
}

// 1 for the Debye edges the march does not fold (their list stays), 0 for the folded ones.
__global__ void k_debye_unfolded(const long long* __restrict__ f, long long ne, const float* __restrict__ ddn,
                                 int* __restrict__ keep) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ne;
         q += (long long)gridDim.x * blockDim.x)
        keep[q] = __float_as_uint(ddn[f[q]]) == FOLD_TAKEN ? 0 : 1;
}

// The unfolded edges' list entries at their positions in the compacted list (pos: exclusive
// prefix sums of keep).
__global__ void k_debye_compact(const long long* __restrict__ f, const float* __restrict__ dd,
                                const float* __restrict__ cb, const int* __restrict__ keep,
                                const int* __restrict__ pos, long long ne, long long* __restrict__ f2,
                                float* __restrict__ dd2, float* __restrict__ cb2) {
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < ne;
         q += (long long)gridDim.x * blockDim.x)
        if (keep[q]) {
            const int p = pos[q];
            f2[p] = f[q];
            dd2[p] = dd[q];
            cb2[p] = cb[q];
        }
}

}  // namespace fg
