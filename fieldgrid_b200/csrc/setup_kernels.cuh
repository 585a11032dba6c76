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
// most LOCAL_CLASSES (ca[3], cb[3]) entries and each owned node's 8-bit local id. A region with
// more classes sets *over and writes nothing; the host then keeps the global ids.
template <typename CID>
__global__ void __launch_bounds__(256) k_local_classes(const CID* __restrict__ node_class,
                                                       const DevCoef* __restrict__ classes,
                                                       const int4* __restrict__ blocks, const int2* __restrict__ own,
                                                       int n1, int n2, int p2, int tk, int lo2, int hi2,
                                                       uint8_t* __restrict__ ids, float* __restrict__ tables,
                                                       int* over) {
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
            const unsigned gid = unsigned(node_class[base + k]);
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
        const DevCoef c = classes[key];
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
            const unsigned gid = unsigned(node_class[base + k]);
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

}  // namespace fg
