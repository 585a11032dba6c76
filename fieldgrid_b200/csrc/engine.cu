// The device side of one run: buffers in HBM, the per-step kernel sequence, CUDA-graph capture of
// the step loop, energy checks and read-back. This is the B200 counterpart of run.rs:390-758
// (buffers, pipelines, dispatch loop) with pack() (run.rs:205-376) folded into session_new.
#include <cuda_runtime.h>

#include <algorithm>
#include <parallel/algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <set>
#include <type_traits>
#include <string>
#include <vector>

#include "../../include/fieldgrid.h"
#include "engine.hpp"
#include "kernels.cuh"
#include "stencil_fused.cuh"
#include "stencil_separate.cuh"
#include "stencil_shell.cuh"
#include "stencil_tma.cuh"
#include "stencil_tb2.cuh"
#include "setup_kernels.cuh"
#include "adjoint_kernels.cuh"

#include <cudaTypedefs.h>
#include <cub/cub.cuh>

namespace fg {

#define FG_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);                              \
            return FG_ERR_CUDA;                                                                    \
        }                                                                                          \
    } while (0)

int gpu_open(int device, Gpu** out, std::string& err) {
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        err = std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "none found");
        return FG_ERR_NO_DEVICE;
    }
    if (device < 0) device = 0;
    if (device >= count) {
        err = "CUDA device " + std::to_string(device) + " does not exist";
        return FG_ERR_NO_DEVICE;
    }
    FG_CUDA(cudaSetDevice(device));
    cudaDeviceProp prop;
    FG_CUDA(cudaGetDeviceProperties(&prop, device));
    auto* g = new Gpu;
    g->device = device;
    g->name = prop.name;
    *out = g;
    return FG_OK;
}

void gpu_close(Gpu* g) {
    if (!g) return;
    cudaSetDevice(g->device);
    if (g->spare) cudaFree(g->spare);
    for (int b = 0; b < 2; ++b) {
        if (g->stage_ev[b]) {
            cudaEventSynchronize(static_cast<cudaEvent_t>(g->stage_ev[b]));
            cudaEventDestroy(static_cast<cudaEvent_t>(g->stage_ev[b]));
        }
        if (g->stage[b]) cudaFreeHost(g->stage[b]);
    }
    delete g;
}

static constexpr size_t STAGE_BYTES = size_t(32) << 20;

// Host -> device through the two pinned staging buffers: fill(buf, off, n) writes bytes [off,
// off + n) of the destination's contents into buf; it runs on the host threads (OpenMP, 1 MB
// parts) while the previous buffer's copy is in flight.
template <class Fill>
int staged_fill(Gpu* g, void* dst, size_t bytes, cudaStream_t st, Fill&& fill) {
    for (int b = 0; b < 2; ++b) {
        if (!g->stage[b]) {
            cudaError_t e = cudaHostAlloc(&g->stage[b], STAGE_BYTES, cudaHostAllocDefault);
            if (e != cudaSuccess) return int(e);
            cudaEvent_t ev;
            e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
            if (e != cudaSuccess) return int(e);
            g->stage_ev[b] = ev;
        }
    }
    char* d8 = static_cast<char*>(dst);
    int b = 0;
    for (size_t off = 0; off < bytes; off += STAGE_BYTES, b ^= 1) {
        const size_t n = std::min(STAGE_BYTES, bytes - off);
        cudaEvent_t ev = static_cast<cudaEvent_t>(g->stage_ev[b]);
        cudaError_t e = cudaEventSynchronize(ev);   // the buffer's previous transfer has finished
        if (e != cudaSuccess) return int(e);
        char* buf = static_cast<char*>(g->stage[b]);
        const long long parts = (long long)((n + (size_t(1) << 20) - 1) >> 20);
#pragma omp parallel for schedule(static)
        for (long long q = 0; q < parts; ++q) {
            const size_t a = size_t(q) << 20, m = std::min(size_t(1) << 20, n - a);
            fill(buf + a, off + a, m);
        }
        e = cudaMemcpyAsync(d8 + off, buf, n, cudaMemcpyHostToDevice, st);
        if (e != cudaSuccess) return int(e);
        e = cudaEventRecord(ev, st);
        if (e != cudaSuccess) return int(e);
    }
    // the source may be reused as soon as it has been copied into the staging buffers
    return int(cudaSuccess);
}

int staged_upload(Gpu* g, void* dst, const void* src, size_t bytes, void* stream) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (bytes < (size_t(4) << 20)) return int(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st));
    const char* s8 = static_cast<const char*>(src);
    return staged_fill(g, dst, bytes, st, [s8](char* buf, size_t off, size_t n) { std::memcpy(buf, s8 + off, n); });
}

struct Session {
    Gpu* gpu = nullptr;
    cudaStream_t stream = nullptr;
    Geom geom{};
    StepConst sc{};
    bool fused = true;
    int cid_bytes = 1;
    // device buffers (sub-allocations of one arena)
    char* arena = nullptr;
    size_t arena_bytes = 0;
    float *e = nullptr, *h = nullptr, *e2 = nullptr, *h2 = nullptr;
    float *psi = nullptr, *psi_h2 = nullptr;
    void* node_class = nullptr;
    DevCoef* classes = nullptr;
    AxisNode* axes = nullptr;
    unsigned* counter = nullptr;
    float* series = nullptr;
    float* plane = nullptr;
    float* ntff = nullptr;
    unsigned* patch = nullptr;
    DevSource* sources = nullptr;
    DevInductor* inductors = nullptr;
    DevProbe* probes = nullptr;
    DevPortEdge* port_edges = nullptr;
    DevLoop* loops = nullptr;
    DevWire* wires = nullptr;
    DevSheet* sheets = nullptr;
    float* branch = nullptr;
    float* currents = nullptr;
    long long* debye_f = nullptr;
    float* debye_dd = nullptr;
    float* debye_cb = nullptr;      // each Debye edge's cb
    float* debye_old = nullptr;
    float* debye_state = nullptr;
    float* debye_table = nullptr;
    double* partial = nullptr;
    int* error = nullptr;           // set by a kernel whose bounded wait ran out
    TmaPlan tma;                    // the TMA-fed fused step, when it applies
    uint8_t* local_ids = nullptr;   // per node: index into its block region's coefficient table
    int4* tma_blocks = nullptr;     // the TMA march's blocks over the clean box
    std::vector<int4> tma_plan_blocks;  // the same list on the host
    int clean_lo[3] = {0, 0, 0}, clean_hi[3] = {0, 0, 0};
    ShellRows shell{};              // the CPML shell around the clean box
    KAxis kax{};                    // the k axis as separate arrays, for the shell kernels
    std::vector<float> kaxis_host;
    // adjoint support: the design edges and the ring of their recorded E^n and curl terms
    int n_design = 0;
    int4* design = nullptr;
    float *hist_e = nullptr, *hist_s = nullptr;
    int hist_cap = 0;
    long long* hist_base = nullptr;
    // what a reset to step 0 restores
    int n_poles = 0;
    size_t currents_len = 0;
    std::vector<DevInductor> ind_host;
    float* tables = nullptr;        // per block region: LOCAL_CLASSES x (ca[3], cb[3])
    bool local = false;
    // the Debye ADE folded into the TMA march (setup_kernels.cuh): per-block entry masks, row
    // offsets, dd and pole state of the folded edges; the list keeps the others
    bool fold = false;
    uint8_t* lmask = nullptr;
    int* drow = nullptr;
    float* fdd = nullptr;
    float* fstate = nullptr;
    int nfold = 0;
    float fdb[2] = {0.f, 0.f}, fdc[2] = {0.f, 0.f};
    // counts
    int n_sources = 0, n_inductors = 0, n_ports = 0, n_wires = 0, n_sheets = 0, n_debye = 0, n_patches = 0;
    int plane_k = 0;
    uint64_t plane_len = 0, ntff_len = 0, series_len = 0;
    long long psi_total = 0, psi_hbase = 0;
    double t0 = 0, tau = 0;
    uint64_t steps = 0;
    uint64_t launches = 0;
    FusedShape shape{};
    std::string variant;
    uint64_t h2d_bytes = 0, d2h_bytes = 0;
    // when set, enqueue_step records an event before every launch (per-kernel timing)
    std::vector<std::pair<const char*, cudaEvent_t>>* marks = nullptr;
    // graphs
    int graph_steps = 0;
    cudaGraphExec_t graph_many = nullptr;
    cudaGraphExec_t graph_two = nullptr;   // an even pair, for the ping-pong parity
    cudaGraphExec_t graph_one[2] = {nullptr, nullptr};
    // re-runs (the adjoint's segment recomputation): steps without the outputs the run already
    // holds (plane DFT, port series, NTFF)
    bool quiet = false;
    bool design_in_steps = true;   // the normal steps record the design history too
    // march with the direct-load fused kernel even where a TMA plan exists (a batch's graph
    // branches of small grids: one launch instead of march + shell)
    bool direct = false;
    // with `direct`: march only the tiles over the box [box_lo, box_hi) (the adjoint's re-runs
    // inside the design history's dependency cone)
    bool boxed = false;
    int box_lo[3] = {0, 0, 0}, box_hi[3] = {0, 0, 0};
    // the march's mbarrier wait limit and its test knob (TmaArgs::stall_plane); set at creation
    // from FIELDGRID_TEST_WAIT_NS / FIELDGRID_TEST_STALL_PLANE, which only the failure-path test sets
    unsigned long long wait_ns = tma::WAIT_LIMIT_NS;
    int stall_plane = -1;
    int2* tma_own = nullptr;        // per block of the one-step march: the rows it writes
    // ---- the two-step mode (stencil_tb2.cuh). Step t reads field set, z-slab psi slot and Debye
    // state slot t mod 3 and writes (t + 1) mod 3; the x/y slabs keep the one-step scheme (E in
    // place, H by the parity of t). A double step is the two-step march over the interior tiles
    // beside one step of the remaining tiles and the shell (second stream), then one more step of
    // those.
    bool slots = false;
    float *e3 = nullptr, *h3 = nullptr;              // the third field set
    float* zslot[3] = {nullptr, nullptr, nullptr};   // z-slab psi by time slot (psi_off offsets)
    float* dslot[3] = {nullptr, nullptr, nullptr};   // Debye state by time slot: [edge * np + pole]
    unsigned* dbase = nullptr;                       // per device node: its first Debye edge
    long long* dd_f = nullptr;                       // Debye edges in node order, those of the one-step
    unsigned* dd_s = nullptr;                        // tiles and shell first (dd_c of them), then the
    float* dd_w = nullptr;                           // two-step tiles' (dd_all in all): field index,
    float* dd_cb = nullptr;                          // state index, weight, cb
    int dd_c = 0, dd_all = 0;
    int4* c_blocks = nullptr;                        // the one-step tiles of a double step
    int2* c_own = nullptr;
    float* c_tables = nullptr;
    int n_cblocks = 0;
    int4* tb_blocks = nullptr;                       // the two-step tiles
    int* tb_idbase = nullptr;
    uint8_t* tb_ids = nullptr;
    float* tb_tables = nullptr;
    int n_tb = 0, tb_zblocks = 0, tb_rim = 0, tb_smem = 0;
    size_t tb_planes = 0;                            // planes of the block-major class-id array
    CUtensorMap tbm_e[3], tbm_h[3], tbm_c, tbm_zh[3], tbm_ze[3];   // the two-step march's maps
    CUtensorMap d1_e[3], d1_h[3], d1_pze[3], d1_pzh[3];            // the one-step march's, per set/slot
    cudaStream_t side = nullptr;
    cudaEvent_t fork_ev = nullptr, join_ev = nullptr;
    // graph-captured fused steps: the plane DFT and the NTFF accumulation of step n run on `aux`
    // beside step n + 1 (which only reads the fields they read); step n + 2, which overwrites those
    // fields, waits for them (aux_done of the same parity), and every captured graph joins them
    cudaStream_t aux = nullptr;
    cudaEvent_t aux_ready[2] = {nullptr, nullptr}, aux_done[2] = {nullptr, nullptr};
    bool aux_on = false, aux_pending[2] = {false, false};
    // captured TMA steps with a CPML shell: k_shell_h runs on `shell_st` beside the march (it reads
    // the step's inputs only), at the lowest priority and the march at the highest, so that its
    // blocks take the room two march blocks leave on an SM; k_shell_e joins both
    cudaStream_t shell_st = nullptr;
    cudaEvent_t shell_fork = nullptr, shell_join = nullptr;
    int prio_lo = 0, prio_hi = 0;
    bool capturing = false;
    std::map<int, cudaGraphExec_t> slot_graphs;      // captured steps by (kind, phase t mod 6)
    std::vector<void*> extra_allocs;
};

static constexpr int ENERGY_BLOCKS = 1024;
// Steps per sweep when FIELDGRID_STEP_DEPTH (1 or 2) does not say: 2 runs the two-step march where
// a Sim qualifies for it.
static constexpr int STEP_DEPTH_DEFAULT = 1;

namespace {

template <typename T>
T* carve(char*& cur, size_t count) {
    T* p = reinterpret_cast<T*>(cur);
    size_t bytes = ((count * sizeof(T)) + 255) & ~size_t(255);
    cur += std::max<size_t>(bytes, 256);
    return p;
}

size_t carve_size(size_t bytes) { return std::max<size_t>((bytes + 255) & ~size_t(255), 256); }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no link against libcuda).
PFN_cuTensorMapEncodeTiled_v12000 encode_tiled() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

bool encode(CUtensorMap* m, CUtensorMapDataType dt, void* base, int rank, const cuuint64_t* dims,
            const cuuint64_t* strides, const cuuint32_t* box, std::string& why) {
    auto fn = encode_tiled();
    if (!fn) { why = "cuTensorMapEncodeTiled is unavailable"; return false; }
    cuuint32_t es[5] = {1, 1, 1, 1, 1};
    CUtensorMapL2promotion promo = CU_TENSOR_MAP_L2_PROMOTION_L2_256B;
    if (const char* v = std::getenv("FIELDGRID_TMA_L2PROMO")) {
        const int b = std::atoi(v);
        promo = b == 0 ? CU_TENSOR_MAP_L2_PROMOTION_NONE
              : b == 64 ? CU_TENSOR_MAP_L2_PROMOTION_L2_64B
              : b == 128 ? CU_TENSOR_MAP_L2_PROMOTION_L2_128B : CU_TENSOR_MAP_L2_PROMOTION_L2_256B;
    }
    CUresult r = fn(m, dt, cuuint32_t(rank), base, dims, strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, promo, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) { why = "cuTensorMapEncodeTiled failed (" + std::to_string(int(r)) + ")"; return false; }
    return true;
}

constexpr int TMA_TJ = 7, TMA_TK = 64, TMA_STAGES = 3, TMA_SEGMAX = 64;

// Kernel shapes the step can run with: stages of the copy ring and the blocks per SM the register
// budget is cut for. Shape 0 is the default; the others are tried by the tuner.
struct TmaShape {
    int stages, minb;
};
constexpr TmaShape TMA_SHAPES[] = {{4, 2}, {3, 3}, {2, 3}};
constexpr int TMA_NSHAPES = 3;

template <typename CID, bool LOCAL, int ST>
using TmaLS = TmaLayout<TMA_TJ, TMA_TK, CID, ST, TMA_SEGMAX, LOCAL, true>;
template <typename CID, bool LOCAL = false>
using TmaL = TmaLS<CID, LOCAL, TMA_STAGES>;
template <typename CID, bool LOCAL, int SHAPE, bool FOLD = false>
constexpr auto tma_kernel_s =
    k_tma_step<TMA_TJ, TMA_TK, CID, TMA_SHAPES[SHAPE].stages, TMA_SEGMAX, LOCAL, TMA_SHAPES[SHAPE].minb, FOLD>;

template <typename CID, bool LOCAL, int SHAPE>
int tma_smem_s() { return TmaLS<CID, LOCAL, TMA_SHAPES[SHAPE].stages>::TOTAL; }

// Calls f(kernel, smem bytes) with the instantiation for (class-id width, local tables, shape,
// the folded Debye ADE).
template <typename F>
bool with_tma_kernel(int cid_bytes, bool local, bool fold, int shape, F&& f) {
    auto go = [&](auto sh) {
        constexpr int S = decltype(sh)::value;
        if (local && fold) return f(tma_kernel_s<uint8_t, true, S, true>, tma_smem_s<uint8_t, true, S>());
        if (local) return f(tma_kernel_s<uint8_t, true, S>, tma_smem_s<uint8_t, true, S>());
        if (cid_bytes == 1) return f(tma_kernel_s<uint8_t, false, S>, tma_smem_s<uint8_t, false, S>());
        if (cid_bytes == 2) return f(tma_kernel_s<uint16_t, false, S>, tma_smem_s<uint16_t, false, S>());
        return f(tma_kernel_s<uint32_t, false, S>, tma_smem_s<uint32_t, false, S>());
    };
    switch (shape) {
        case 0: return go(std::integral_constant<int, 0>{});
        case 1: return go(std::integral_constant<int, 1>{});
        default: return go(std::integral_constant<int, 2>{});
    }
}

// Tiles along k over [za, zb): when the range reaches n2 and spans 64t + 1 nodes, t tiles, the
// last owning the extra column.
inline int tma_ktiles(int za, int zb, int n2) {
    const int w = zb - za;
    return (zb == n2 && w > TMA_TK && w % TMA_TK == 1) ? (w - 1) / TMA_TK : (w + TMA_TK - 1) / TMA_TK;
}

// The fused TMA march covers the clean box [lo, hi): no node the march computes there (its tiles
// and their halo row, column and plane) has a live CPML slot, so the march carries no psi term.
// The box starts one node past the low layer, so the halo stays outside it. Along k it starts on
// an even node and ends on one unless it reaches n2, so column pairs are owned whole; the tiles
// start at that node rounded down to 8 (a 32-byte sector: row writes of every tile but the first
// fill whole sectors; the E and H boxes start at k0 - 4 floats, on 16 bytes; the class-id box at
// k0 rounded down to 16 ids), and the first tile leaves its columns below the box unwritten. The shell around it (the layer and a one-node ring) goes to
// the shell kernels. Blocks are (k0, j0, i0, i1): a TJ x TK tile over one x-segment.
struct CleanPlan {
    std::vector<int4> blocks;    // k0 | TMA_ZL_TILE for the zblocks tiles that reach the k layer
    std::vector<int2> own;       // per block: the rows [x, y) it writes (its tile's rows inside the box)
    int zblocks = 0;
    int seg = 0;                 // planes per block (at most)
    int lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
    int kbase = 0;               // the tile grid's origin along k: lo[2] rounded down to 8 nodes
    ShellRows shell{};
    bool ok = false;
};

// [a, b) along one axis such that no node of [a - 1, b) has a live slot; false when empty.
bool clean_range(const Axis& ax, int n, int& a, int& b) {
    auto hot = [&](int i) { return ax.node[size_t(i)].slot_e >= 0 || ax.node[size_t(i)].slot_h >= 0; };
    int lead = 0;
    while (lead < n && hot(lead)) ++lead;
    int trail = n;
    while (trail > lead && hot(trail - 1)) --trail;
    a = lead > 0 ? lead + 1 : 0;
    b = trail;
    for (int i = std::max(a - 1, 0); i < b; ++i)
        if (hot(i)) return false;
    return a < b;
}

// With z_layer (the z-slab psi fits the march's staged boxes) the box spans every column of its
// rows and planes, and tiles that reach the k layer run the ZL instantiation.
// With `anchor` >= 0 the tiles' rows are laid out so that a tile starts at row `anchor` (the
// first tile may start below the box and own fewer rows), and `segs` (when not empty) gives the
// x-segments explicitly: the two-step march pairs these tiles and reuses these segments.
CleanPlan plan_clean(const HostSim& sim, const Geom& g, bool z_layer, int seg_fixed, int anchor = -1,
                     const std::vector<int2>& segs = {}) {
    CleanPlan out;
    const int n[3] = {g.n0, g.n1, g.n2};
    for (int a = 0; a < 3; ++a)
        if (!clean_range(sim.ax[a], n[a], out.lo[a], out.hi[a]) && !(a == 2 && z_layer)) return out;
    if (z_layer) {
        out.lo[2] = 0;
        out.hi[2] = g.n2;
    }
    out.lo[2] = (out.lo[2] + 1) & ~1;
    if (out.hi[2] < g.n2) out.hi[2] = out.lo[2] + ((out.hi[2] - out.lo[2]) & ~1);
    if (out.lo[2] >= out.hi[2]) return out;
    out.kbase = out.lo[2] & ~7;
    const int kt = tma_ktiles(out.kbase, out.hi[2], g.n2);
    // tile rows: from the box's first row, or laid out around `anchor`
    const int jfirst = anchor < 0 ? out.lo[1] : anchor - TMA_TJ * ((anchor - out.lo[1] + TMA_TJ - 1) / TMA_TJ);
    const int jt = (out.hi[1] - jfirst + TMA_TJ - 1) / TMA_TJ;
    const int xw = out.hi[0] - out.lo[0];
    // x-planes per block: enough blocks for several waves of 3 blocks per SM, at most TMA_SEGMAX
    int seg = TMA_SEGMAX;
    while (seg > 8 && (long long)kt * jt * ((xw + seg - 1) / seg) < 148 * 3 * 6) seg /= 2;
    if (seg_fixed > 0) seg = std::min(seg_fixed, TMA_SEGMAX);
    std::vector<int2> sg = segs;
    if (sg.empty()) {
        const int ns = (xw + seg - 1) / seg;
        for (int q = 0; q < ns; ++q)
            sg.push_back(make_int2(out.lo[0] + int((long long)xw * q / ns), out.lo[0] + int((long long)xw * (q + 1) / ns)));
    }
    out.seg = 0;
    for (const int2& v : sg) out.seg = std::max(out.seg, v.y - v.x);
    auto hot_k = [&](int k) { return sim.ax[2].node[size_t(k)].slot_e >= 0 || sim.ax[2].node[size_t(k)].slot_h >= 0; };
    for (const int2& v : sg) {
        const int i0 = v.x, i1 = v.y;
        for (int by = 0; by < jt; ++by)
            for (int bx = 0; bx < kt; ++bx) {
                const int k0 = out.kbase + bx * TMA_TK;
                const int j0 = jfirst + by * TMA_TJ;
                bool edge = false;   // a column of the tile, its halo column or right-edge column is in the layer
                for (int k = std::max(k0 - 1, 0); k <= std::min(k0 + TMA_TK, g.n2 - 1); ++k) edge = edge || hot_k(k);
                out.zblocks += edge;
                out.blocks.push_back(make_int4(edge ? (k0 | TMA_ZL_TILE) : k0, j0, i0, i1));
                out.own.push_back(make_int2(std::max(j0, out.lo[1]), std::min(j0 + TMA_TJ, out.hi[1])));
            }
    }
    // the shell rows around the clean box
    ShellRows& sr = out.shell;
    sr.xa = out.lo[0]; sr.xb = out.hi[0];
    sr.ya = out.lo[1]; sr.yb = out.hi[1];
    sr.za = out.lo[2]; sr.zb = out.hi[2];
    sr.ra = unsigned((sr.xa + g.n0 - sr.xb) * g.n1);
    sr.rb = unsigned((sr.xb - sr.xa) * (sr.ya + g.n1 - sr.yb));
    sr.rc = (sr.za > 0 || sr.zb < g.n2) ? unsigned((sr.xb - sr.xa) * (sr.yb - sr.ya)) : 0u;
    out.ok = true;
    return out;
}

// Builds the tensor maps of the TMA step: E and H of both buffer sets, and the class ids.
void plan_tma(Session& s) {
    TmaPlan& t = s.tma;
    t.ok = false;
    const Geom& g = s.geom;
    if (!s.fused) { t.why = "separate step"; return; }
    if (const char* v = std::getenv("FIELDGRID_NO_TMA"); v && v[0] == '1') { t.why = "disabled by FIELDGRID_NO_TMA"; return; }
    int dev = 0, major = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (major < 10) { t.why = "needs sm_100"; return; }
    if (g.n2 < 2 || g.n1 < 2) { t.why = "grid too thin"; return; }
    t.tj = TMA_TJ;
    t.tk = TMA_TK;
    t.shape = 0;
    if (const char* v = std::getenv("FIELDGRID_TMA_SHAPE")) t.shape = std::min(std::max(std::atoi(v), 0), TMA_NSHAPES - 1);
    const cuuint64_t dims[4] = {cuuint64_t(g.n2), cuuint64_t(g.n1), cuuint64_t(g.n0), 3};
    const cuuint64_t strides[3] = {cuuint64_t(g.p2) * 4, cuuint64_t(g.n1) * g.p2 * 4, cuuint64_t(g.cs) * 4};
    const cuuint32_t box_e[4] = {cuuint32_t(TmaL<float>::EW), cuuint32_t(TmaL<float>::ER), 1, 3};
    const cuuint32_t box_h[4] = {cuuint32_t(TmaL<float>::HW), cuuint32_t(TmaL<float>::HR), 1, 3};
    float* es[2] = {s.e, s.e2};
    float* hs[2] = {s.h, s.h2};
    for (int q = 0; q < 2; ++q) {
        if (!encode(&t.e[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, es[q], 4, dims, strides, box_e, t.why)) return;
        if (!encode(&t.h[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, hs[q], 4, dims, strides, box_h, t.why)) return;
    }
    const int b = s.local ? 1 : s.cid_bytes;
    const CUtensorMapDataType dt = b == 1 ? CU_TENSOR_MAP_DATA_TYPE_UINT8
                                 : (b == 2 ? CU_TENSOR_MAP_DATA_TYPE_UINT16 : CU_TENSOR_MAP_DATA_TYPE_UINT32);
    const cuuint64_t cdims[3] = {cuuint64_t(g.n2), cuuint64_t(g.n1), cuuint64_t(g.n0)};
    const cuuint64_t cstr[2] = {cuuint64_t(g.p2) * b, cuuint64_t(g.n1) * g.p2 * b};
    const cuuint32_t cbox[3] = {cuuint32_t(TmaL<float>::CW), cuuint32_t(TmaL<float>::CR), 1};
    if (!encode(&t.c, dt, s.local ? (void*)s.local_ids : s.node_class, 3, cdims, cstr, cbox, t.why)) return;
    // z-slab psi for the k-layer tiles: (slot, j, i, component) over each field's two adjacent z slabs
    t.pz = t.zblocks > 0;
    if (t.pz) {
        const long long zlen = g.psi_off[1 * 3 + 2] - g.psi_off[0 * 3 + 2];  // slab stride, 128-byte multiple
        const cuuint64_t zd[4] = {cuuint64_t(g.pw), cuuint64_t(g.n1), cuuint64_t(g.n0), 2};
        const cuuint64_t zs[3] = {cuuint64_t(g.pw) * 4, cuuint64_t(g.n1) * g.pw * 4, cuuint64_t(zlen) * 4};
        const cuuint32_t zb[4] = {cuuint32_t(g.pw), cuuint32_t(TMA_TJ + 1), 1, 2};
        if (!encode(&t.pze, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, s.psi + g.psi_off[0 * 3 + 2], 4, zd, zs, zb, t.why)) return;
        float* hsets[2] = {s.psi, s.psi_h2};  // the H slabs read by a step whose input set is 0 / 1
        for (int q = 0; q < 2; ++q)
            if (!encode(&t.pzh[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, hsets[q] + g.psi_off[9 + 0 * 3 + 2], 4, zd, zs, zb,
                        t.why))
                return;
    }
    cudaError_t ce = cudaSuccess;
    for (int sh = 0; sh < TMA_NSHAPES && ce == cudaSuccess; ++sh)
        with_tma_kernel(b, s.local, s.fold, sh, [&](auto kern, int smem) {
            ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
            if (sh == t.shape) t.smem = smem;
            return true;
        });
    if (ce != cudaSuccess) { t.why = std::string("cudaFuncSetAttribute: ") + cudaGetErrorString(ce); return; }
    if (!s.tma_blocks) { t.why = "no block list"; return; }
    // every TMA box origin along k must sit on 16 bytes: k0 - 4 floats, and k0 & ~15 class ids
    for (const int4& bk : s.tma_plan_blocks)
        if ((bk.x & ~TMA_ZL_TILE) % 8 != 0) { t.why = "internal: unaligned tile origin"; return; }
    t.ok = true;
}

int launch_tma(Session& s, int parity, float* e_out, float* h_out, float* psi_h_out) {
    const TmaPlan& t = s.tma;
    TmaArgs a{s.geom, s.classes, e_out, h_out, s.sc.k_mu, s.clean_lo[2], s.clean_hi[1], s.clean_hi[2], s.tma_blocks,
              s.tma_own, 0, 1, s.psi, psi_h_out, s.tables, s.counter, s.error, s.wait_ns, -0.0f, s.stall_plane};
    if (s.fold) {
        a.lmask = s.lmask;
        a.drow = s.drow;
        a.fdd = s.fdd;
        a.fstate = s.fstate;
        a.nfold = s.nfold;
        a.npoles = s.n_poles;
        for (int k = 0; k < 2; ++k) { a.db[k] = s.fdb[k]; a.dc[k] = s.fdc[k]; }
    }
    // without k-layer tiles the last two maps are never read
    const CUtensorMap& pze = t.pz ? t.pze : t.c;
    const CUtensorMap& pzh = t.pz ? t.pzh[parity] : t.c;
    with_tma_kernel(s.cid_bytes, s.local, s.fold, t.shape, [&](auto kern, int smem) {
        if (s.capturing && s.shell_st) {
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3(unsigned(t.blocks));
            cfg.blockDim = dim3(TMA_CONSUMERS + 32);
            cfg.dynamicSmemBytes = size_t(smem);
            cfg.stream = s.stream;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributePriority;
            at[0].val.priority = s.prio_hi;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            cudaLaunchKernelEx(&cfg, kern, t.e[parity], t.h[parity], t.c, pze, pzh, a);
        } else {
            kern<<<unsigned(t.blocks), TMA_CONSUMERS + 32, smem, s.stream>>>(t.e[parity], t.h[parity], t.c, pze, pzh, a);
        }
        return true;
    });
    return cudaPeekAtLastError() == cudaSuccess ? 0 : 1;
}

// One time step. `parity` selects the ping-pong direction of the fused step (input = parity 0
// buffers on even steps). The separate step updates in place.
int enqueue_step(Session& s, int parity, std::string& err) {
    const Geom& g = s.geom;
    cudaStream_t st = s.stream;
    auto mark = [&](const char* name) {
        if (!s.marks) return;
        cudaEvent_t ev;
        cudaEventCreate(&ev);
        cudaEventRecord(ev, st);
        s.marks->push_back({name, ev});
    };
    float *e_in = s.e, *h_in = s.h, *e_out = s.e, *h_out = s.h;
    if (s.fused && parity) { e_in = s.e2; h_in = s.h2; e_out = s.e; h_out = s.h; }
    else if (s.fused) { e_out = s.e2; h_out = s.h2; }
    if (!s.fused) {
        dim3 blk(64, 4, 1), grd((g.n2 + 63) / 64, (g.n1 + 3) / 4, g.n0);
        mark("update_h");
        k_update_h<<<grd, blk, 0, st>>>(g, s.e, s.h, s.psi, s.sc.k_mu, s.counter);
        if (s.n_wires) { mark("wire_h"); k_wire_h<<<(s.n_wires + 127) / 128, 128, 0, st>>>(s.wires, s.n_wires, s.e, s.h); }
        if (s.n_sheets) { mark("sheet_pre"); k_sheet_pre<<<(s.n_sheets + 127) / 128, 128, 0, st>>>(s.sheets, s.n_sheets, s.e, s.h); }
        if (s.n_debye) { mark("debye_pre"); k_debye_pre<<<(s.n_debye + 255) / 256, 256, 0, st>>>(s.debye_f, s.n_debye, s.e, s.debye_old); }
        mark("update_e");
        switch (s.cid_bytes) {
            case 1: k_update_e<uint8_t><<<grd, blk, 0, st>>>(g, (const uint8_t*)s.node_class, s.classes, s.h, s.e, s.psi); break;
            case 2: k_update_e<uint16_t><<<grd, blk, 0, st>>>(g, (const uint16_t*)s.node_class, s.classes, s.h, s.e, s.psi); break;
            default: k_update_e<uint32_t><<<grd, blk, 0, st>>>(g, (const uint32_t*)s.node_class, s.classes, s.h, s.e, s.psi); break;
        }
    } else {
        if (s.n_wires) {
            // thin-wire terms join H before the march reads it (run.rs:620-623); E is the step's input
            mark("wire_h");
            k_wire_h<<<(s.n_wires + 127) / 128, 128, 0, st>>>(s.wires, s.n_wires, e_in, h_in);
        }
        if (s.aux_on && s.aux_pending[parity]) {   // this step overwrites what step n - 2's extras read
            FG_CUDA(cudaStreamWaitEvent(st, s.aux_done[parity], 0));
            s.aux_pending[parity] = false;
        }
        const bool tma = s.tma.ok && !s.direct;
        const unsigned shell_rows = s.shell.ra + s.shell.rb + s.shell.rc;
        const bool shell_side = tma && shell_rows > 0 && s.capturing && s.shell_st;
        if (shell_side) {
            // the shell's H update beside the march (both read only the step's inputs)
            FG_CUDA(cudaEventRecord(s.shell_fork, st));
            FG_CUDA(cudaStreamWaitEvent(s.shell_st, s.shell_fork, 0));
            const unsigned gs = (shell_rows + SHELL_SIDE_THREADS / 32 - 1) / (SHELL_SIDE_THREADS / 32);
            cudaLaunchConfig_t cfg{};
            cfg.gridDim = dim3(gs);
            cfg.blockDim = dim3(SHELL_SIDE_THREADS);
            cfg.stream = s.shell_st;
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributePriority;
            at[0].val.priority = s.prio_lo;
            cfg.attrs = at;
            cfg.numAttrs = 1;
            FG_CUDA(cudaLaunchKernelEx(&cfg, k_shell_h_side, g, s.shell, s.kax, (const float*)e_in, (const float*)h_in,
                                       h_out, (const float*)(parity ? s.psi_h2 : s.psi), parity ? s.psi : s.psi_h2,
                                       (const float*)(parity ? s.psi_h2 : s.psi), parity ? s.psi : s.psi_h2,
                                       s.sc.k_mu));
            FG_CUDA(cudaEventRecord(s.shell_join, s.shell_st));
        }
        mark("fused_step");
        int rc = s.direct && s.boxed
                     ? launch_fused_box(s.cid_bytes, g, s.node_class, s.classes, e_in, h_in, e_out, h_out, s.psi,
                                        parity ? s.psi_h2 : s.psi, parity ? s.psi : s.psi_h2, s.sc.k_mu, s.counter,
                                        s.box_lo, s.box_hi, st)
                 : tma
                     ? launch_tma(s, parity, e_out, h_out, parity ? s.psi : s.psi_h2)
                     : launch_fused(s.shape, s.cid_bytes, g, s.node_class, s.classes, e_in, h_in, e_out, h_out, s.psi,
                                    parity ? s.psi_h2 : s.psi, parity ? s.psi : s.psi_h2, s.sc.k_mu, s.counter,
                                    s.n_wires > 0, st);
        if (rc) { err = "fused step launch failed"; return FG_ERR_CUDA; }
        if (tma && shell_rows > 0) {
            // the CPML shell around the march's clean box, one warp per row
            const unsigned gb = (shell_rows + SHELL_THREADS / 32 - 1) / (SHELL_THREADS / 32);
            if (shell_side) {
                FG_CUDA(cudaStreamWaitEvent(st, s.shell_join, 0));
            } else {
                mark("shell_h");
                k_shell_h<<<gb, SHELL_THREADS, 0, st>>>(g, s.shell, s.kax, e_in, h_in, h_out, parity ? s.psi_h2 : s.psi,
                                                        parity ? s.psi : s.psi_h2, parity ? s.psi_h2 : s.psi,
                                                        parity ? s.psi : s.psi_h2, s.sc.k_mu);
            }
            mark("shell_e");
            switch (s.cid_bytes) {
                case 1: k_shell_e<uint8_t><<<gb, SHELL_THREADS, 0, st>>>(g, s.shell, s.kax, (const uint8_t*)s.node_class, s.classes, h_out, e_in, e_out, s.psi, s.psi, s.psi); break;
                case 2: k_shell_e<uint16_t><<<gb, SHELL_THREADS, 0, st>>>(g, s.shell, s.kax, (const uint16_t*)s.node_class, s.classes, h_out, e_in, e_out, s.psi, s.psi, s.psi); break;
                default: k_shell_e<uint32_t><<<gb, SHELL_THREADS, 0, st>>>(g, s.shell, s.kax, (const uint32_t*)s.node_class, s.classes, h_out, e_in, e_out, s.psi, s.psi, s.psi); break;
            }
        }
        if (s.n_sheets) {
            mark("sheet_pre");
            k_sheet_pre<<<(s.n_sheets + 127) / 128, 128, 0, st>>>(s.sheets, s.n_sheets, e_in, h_out);
        }
    }
    float* e_now = s.fused ? e_out : s.e;
    float* h_now = s.fused ? h_out : s.h;
    if (s.n_sheets) mark("sheet_post");
    if (s.n_sheets) k_sheet_post<<<(s.n_sheets + 127) / 128, 128, 0, st>>>(s.sheets, s.n_sheets, s.branch, s.currents, e_now);
    if (s.n_debye) {
        mark("debye_post");
        const float* saved = s.fused ? nullptr : s.debye_old;
        k_debye_post_cb<<<(s.n_debye + 255) / 256, 256, 0, st>>>(s.debye_f, s.debye_dd, s.debye_cb, s.n_debye, saved,
                                                                 e_in, s.debye_table, s.debye_state, e_now);
    }
    const bool lumped = s.n_sources || s.n_inductors, probes = s.n_ports && !s.quiet;
    if (lumped && probes && s.n_ports == 1) {
        // one port: its source and its probe in one launch
        mark("lumped_probe");
        k_lumped_probe<<<1, 256, 0, st>>>(s.sources, s.n_sources, s.inductors, s.n_inductors, s.sc, s.counter, e_now,
                                          s.probes, s.port_edges, s.loops, g.cs, h_now, s.series);
    } else {
        if (lumped) mark("lumped");
        if (lumped) k_lumped<<<1, 256, 0, st>>>(s.sources, s.n_sources, s.inductors, s.n_inductors, s.sc, s.counter, e_now);
        if (probes) mark("probe");
        if (probes) k_probe<<<s.n_ports, 256, 0, st>>>(s.probes, s.port_edges, s.loops, g.cs, e_now, h_now, s.counter, s.sc, s.series);
    }
    const bool branch = s.aux_on && s.fused && (s.plane_len || s.ntff_len) && !s.quiet;
    cudaStream_t xs = branch ? s.aux : st;
    const int xpar = branch ? parity : -1;
    if (branch) {
        FG_CUDA(cudaEventRecord(s.aux_ready[parity], st));
        FG_CUDA(cudaStreamWaitEvent(s.aux, s.aux_ready[parity], 0));
    }
    if (s.plane_len && !s.quiet) {
        long long q = (long long)g.n0 * g.n1;
        mark("field_dft");
        k_field_dft<<<unsigned((q + 127) / 128), 128, 0, xs>>>(g, s.plane_k, s.sc, s.counter, xpar, e_now, h_now, s.plane);
    }
    if (s.ntff_len && !s.quiet) mark("ntff");
    if (s.ntff_len && !s.quiet)
        k_ntff<<<(s.n_patches + 127) / 128, 128, 0, xs>>>(s.patch, s.n_patches, g.cs, s.sc, s.counter, xpar, e_now,
                                                          h_now, s.ntff);
    if (branch) {
        FG_CUDA(cudaEventRecord(s.aux_done[parity], s.aux));
        s.aux_pending[parity] = true;
    }
    if (s.n_design && s.fused && (s.quiet || s.design_in_steps)) {
        mark("design_record");
        k_design_record<<<(s.n_design + 127) / 128, 128, 0, st>>>(g, s.design, s.n_design, e_in, h_now, s.psi, s.counter,
                                                                   s.hist_base, s.hist_cap, s.hist_e, s.hist_s);
    }
    mark(nullptr);
    return FG_OK;
}

uint64_t count_launches(const Session& s) {
    if (s.slots) {
        // a double step: the two-step march and twice (march, shell H and E, Debye, sources+probes)
        const uint64_t one = 1 + ((s.shell.ra + s.shell.rb + s.shell.rc) ? 2 : 0) + (s.dd_c > 0 ? 1 : 0) +
                             ((s.n_sources || s.n_inductors) && s.n_ports == 1 ? 1
                              : uint64_t(s.n_sources || s.n_inductors) + uint64_t(s.n_ports > 0));
        return (1 + 2 * one + 1) / 2;
    }
    uint64_t n = 1;  // the field update (fused) or H update (separate)
    if (s.tma.ok && !s.direct && s.shell.ra + s.shell.rb + s.shell.rc > 0) n += 2;  // the CPML shell around the TMA march
    if (!s.fused) n += 1 + (s.n_debye ? 1 : 0);
    if (s.n_wires) n++;
    if (s.n_sheets) n += 2;
    if (s.n_debye) n++;
    const bool lumped = s.n_sources || s.n_inductors;
    if (lumped) n++;
    if (s.n_ports && !(lumped && s.n_ports == 1)) n++;   // one port: with the source in one launch
    if (s.plane_len) n++;
    if (s.ntff_len) n++;
    if (s.n_design && s.fused && s.design_in_steps) n++;
    return n;
}

int capture(Session& s, int steps, int parity0, cudaGraphExec_t* out, std::string& err) {
    cudaGraph_t graph;
    FG_CUDA(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal));
    int rc = FG_OK;
    s.aux_on = s.aux != nullptr;
    s.capturing = true;
    for (int q = 0; q < steps && rc == FG_OK; ++q) rc = enqueue_step(s, (parity0 + q) & 1, err);
    s.capturing = false;
    for (int p = 0; p < 2; ++p)   // the graph ends with its extras joined
        if (s.aux_pending[p]) {
            if (rc == FG_OK && cudaStreamWaitEvent(s.stream, s.aux_done[p], 0) != cudaSuccess) rc = FG_ERR_CUDA;
            s.aux_pending[p] = false;
        }
    s.aux_on = false;
    cudaError_t ce = cudaStreamEndCapture(s.stream, &graph);
    if (rc) return rc;
    if (ce != cudaSuccess) { err = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ce); return FG_ERR_CUDA; }
    ce = cudaGraphInstantiate(out, graph, s.shell_st ? cudaGraphInstantiateFlagUseNodePriority : 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) { err = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ce); return FG_ERR_CUDA; }
    return FG_OK;
}

// ---- the two-step mode: plan --------------------------------------------------------------

// The layout of a double step over the clean box: the two-step tiles (14 x 64 columns over
// x-segments, each tile the pair of one-step tiles it replaces) and the one-step tiles left beside
// them. Tiles whose halo (two nodes and two planes around them) would reach a node with its own
// per-step terms (a port edge, a probe loop, a source or an inductor) or would need more than
// LOCAL_CLASSES coefficient classes stay one-step. Two-step tiles next to a one-step tile (or the
// shell) write their step-(n+1) fields as well ("rim").
struct SlotPlan {
    bool ok = false;
    std::string why;
    CleanPlan cp;                       // the one-step plan, rows and segments aligned with the tiles
    std::vector<int4> tb;               // two-step tiles: k0 | TMA_ZL_TILE | TB_RIM, j0, i0, i1
    std::vector<int> idbase;            // per two-step tile: its first plane in `ids`
    std::vector<uint8_t> ids;           // block-major class ids: [plane][16 rows][TB_CW columns]
    std::vector<float> tables;          // per two-step tile: LOCAL_CLASSES records of TB_REC floats
    std::vector<int> cidx;              // one-step tiles of a double step (indices into cp.blocks)
    std::vector<long long> dd_f;        // Debye edges in node order: one-step ones first
    std::vector<unsigned> dd_s;
    std::vector<float> dd_w, dd_cb;
    int dd_c = 0;
    int zblocks = 0, rim = 0;
};

SlotPlan plan_slots(const HostSim& sim, const Geom& g, bool z_layer, const std::vector<uint64_t>& special) {
    SlotPlan P;
    const int n[3] = {g.n0, g.n1, g.n2};
    int lo[3], hi[3];
    for (int a = 0; a < 3; ++a)
        if (!clean_range(sim.ax[a], n[a], lo[a], hi[a]) && !(a == 2 && z_layer)) { P.why = "no clean box"; return P; }
    // rows: the tile's halo rows j0 - 2 .. j0 + 15 stay in the clean rows [ya - 1, yb) and off the
    // grid's first and last rows (j0 >= 2, j0 + 16 <= n1); planes likewise
    const int ja = std::max(lo[1] + 1, 2);
    const int jlim = std::min(hi[1], g.n1) - 2;
    const int J = jlim > ja ? (jlim - ja) / TB_TJ : 0;
    const int ia = std::max(lo[0] + 1, 2), ib = std::min(hi[0] - 2, g.n0 - 2);
    if (J < 1 || ib - ia < 4) { P.why = "the interior is too small for two-step tiles"; return P; }
    std::vector<int2> rsegs, segs;
    {
        const int w = ib - ia, ns = (w + TB_SEGMAX - 1) / TB_SEGMAX;
        for (int q = 0; q < ns; ++q) rsegs.push_back(make_int2(ia + int((long long)w * q / ns), ia + int((long long)w * (q + 1) / ns)));
    }
    if (lo[0] < ia) segs.push_back(make_int2(lo[0], ia));
    segs.insert(segs.end(), rsegs.begin(), rsegs.end());
    if (ib < hi[0]) segs.push_back(make_int2(ib, hi[0]));
    P.cp = plan_clean(sim, g, z_layer, 0, ja, segs);
    if (!P.cp.ok) { P.why = "no clean box"; return P; }
    const CleanPlan& cp = P.cp;
    const int kt = tma_ktiles(cp.kbase, cp.hi[2], g.n2);
    const int NS = int(rsegs.size());
    auto flat = [&](int sg, int q, int bx) { return (size_t(sg) * J + q) * kt + bx; };
    std::vector<uint8_t> on(size_t(NS) * J * kt, 1);
    // halo of a tile: planes [i0 - 2, i1 + 2), rows [j0 - 2, j0 + 16), columns [k0 - 2, k0 + 66)
    for (uint64_t id : special) {
        const int i = int(id / (uint64_t(g.n1) * g.n2)), j = int((id / g.n2) % g.n1), k = int(id % g.n2);
        for (int sg = 0; sg < NS; ++sg) {
            if (i < rsegs[sg].x - 2 || i >= rsegs[sg].y + 2) continue;
            for (int q = 0; q < J; ++q) {
                const int j0 = ja + TB_TJ * q;
                if (j < j0 - 2 || j >= j0 + 16) continue;
                for (int bx = 0; bx < kt; ++bx) {
                    const int k0 = cp.kbase + TB_TK * bx;
                    if (k >= k0 - 2 && k < k0 + 66) on[flat(sg, q, bx)] = 0;
                }
            }
        }
    }
    // Debye edges in node order; per node its first edge (or none)
    const size_t nn = sim.nn, n1 = g.n1, n2 = g.n2;
    std::vector<std::pair<uint64_t, uint32_t>> order;   // (id, comp)
    order.reserve(sim.debye_edges.size());
    for (const auto& q : sim.debye_edges) order.push_back({q.id, q.comp});
    std::vector<size_t> perm(order.size());
    for (size_t q = 0; q < perm.size(); ++q) perm[q] = q;
    __gnu_parallel::sort(perm.begin(), perm.end(), [&](size_t x, size_t y) { return order[x] < order[y]; });
    std::vector<uint32_t> dfirst;
    if (!sim.debye_edges.empty()) {
        dfirst.resize(nn);
#pragma omp parallel for schedule(static)
        for (long long q = 0; q < (long long)nn; ++q) dfirst[size_t(q)] = 0xffffffffu;
    }
    for (size_t e = 0; e < perm.size(); ++e) {
        const uint64_t id = sim.debye_edges[perm[e]].id;
        if (dfirst[id] == 0xffffffffu) dfirst[id] = uint32_t(e);
    }
    auto dd_of = [&](uint64_t id, float (&dd)[3]) {
        dd[0] = dd[1] = dd[2] = 0.f;
        if (dfirst.empty() || dfirst[id] == 0xffffffffu) return;
        for (size_t e = dfirst[id]; e < perm.size() && sim.debye_edges[perm[e]].id == id; ++e)
            dd[sim.debye_edges[perm[e]].comp] = float(sim.debye_edges[perm[e]].dd);
    };
    // per candidate tile: its coefficient classes over the region whose E it forms
    // (planes i0 - 1 .. i1, rows j0 - 1 .. j0 + 14, columns k0 - 1 .. k0 + 64)
    const long long cand = (long long)NS * J * kt;
    std::vector<float> ctab(size_t(cand) * LOCAL_CLASSES * TB_REC, 0.f);
    std::vector<size_t> cand_idbase(static_cast<size_t>(cand));
    {
        size_t acc = 0;
        for (long long c = 0; c < cand; ++c) {
            cand_idbase[size_t(c)] = acc;
            const int sg = int(c / ((long long)J * kt));
            acc += size_t(rsegs[sg].y - rsegs[sg].x + 2);
        }
        P.ids.resize(acc * 16 * TB_CW);   // each candidate clears and fills its own planes below
    }
#pragma omp parallel for schedule(dynamic, 4)
    for (long long c = 0; c < cand; ++c) {
        if (!on[size_t(c)]) continue;
        const int sg = int(c / ((long long)J * kt)), q = int((c / kt) % J), bx = int(c % kt);
        const int i0 = rsegs[sg].x, i1 = rsegs[sg].y, j0 = ja + TB_TJ * q, k0 = cp.kbase + TB_TK * bx;
        struct Key { uint32_t gid; float dd[3]; };
        Key keys[512];
        bool used[512] = {};
        uint8_t vals[512];
        int count = 0;
        bool over = false;
        float* tab = ctab.data() + size_t(c) * LOCAL_CLASSES * TB_REC;
        uint8_t* idp = P.ids.data() + cand_idbase[size_t(c)] * 16 * TB_CW;
        std::memset(idp, 0, size_t(i1 - i0 + 2) * 16 * TB_CW);
        Key last{0xffffffffu, {0.f, 0.f, 0.f}};   // runs of equal keys along a row skip the hash
        uint8_t last_val = 0;
        for (int i = i0 - 1; i <= i1 && !over; ++i)
            for (int r = -1; r < 15 && !over; ++r)
                for (int cc = -1; cc < 65; ++cc) {
                    const int j = j0 + r, k = k0 + cc;
                    if (k < 0 || k >= g.n2) continue;
                    const uint64_t id = (uint64_t(i) * n1 + uint64_t(j)) * n2 + uint64_t(k);
                    Key key;
                    key.gid = sim.cls(id);
                    dd_of(id, key.dd);
                    if (key.gid == last.gid && std::memcmp(key.dd, last.dd, 12) == 0) {
                        idp[(size_t(i - (i0 - 1)) * 16 + size_t(r + 1)) * TB_CW + size_t(cc + 1)] = last_val;
                        continue;
                    }
                    uint32_t hsh = key.gid * 2654435761u;
                    for (int t = 0; t < 3; ++t) {
                        uint32_t b;
                        std::memcpy(&b, &key.dd[t], 4);
                        hsh ^= b * (0x9e3779b9u + 2u * uint32_t(t));
                        hsh *= 0x85ebca6bu;
                    }
                    uint32_t h = hsh & 511u;
                    while (used[h] && !(keys[h].gid == key.gid && std::memcmp(keys[h].dd, key.dd, 12) == 0)) h = (h + 1) & 511u;
                    if (!used[h]) {
                        if (count == LOCAL_CLASSES) { over = true; break; }
                        used[h] = true;
                        keys[h] = key;
                        vals[h] = uint8_t(count);
                        const Coef& cf = sim.classes[key.gid];
                        for (int t = 0; t < 3; ++t) {
                            tab[count * TB_REC + t] = cf.ca[t];
                            tab[count * TB_REC + 3 + t] = cf.cb[t];
                            tab[count * TB_REC + 6 + t] = key.dd[t];
                        }
                        ++count;
                    }
                    idp[(size_t(i - (i0 - 1)) * 16 + size_t(r + 1)) * TB_CW + size_t(cc + 1)] = vals[h];
                    last = key;
                    last_val = vals[h];
                }
        if (over) on[size_t(c)] = 0;
    }
    // the rim: a tile with a one-step node (or the shell) within two nodes
    auto is_on = [&](int sg, int q, int bx) {
        if (sg < 0 || sg >= NS || q < 0 || q >= J) return false;
        if (bx < 0 || bx >= kt) return true;   // past the grid's k ends: no node there
        return on[flat(sg, q, bx)] != 0;
    };
    std::vector<size_t> cand_of_tb;
    for (int sg = 0; sg < NS; ++sg)
        for (int q = 0; q < J; ++q)
            for (int bx = 0; bx < kt; ++bx) {
                if (!on[flat(sg, q, bx)]) continue;
                bool rim = false;
                for (int ds = -1; ds <= 1 && !rim; ++ds)
                    for (int dq = -1; dq <= 1 && !rim; ++dq)
                        for (int db = -1; db <= 1 && !rim; ++db)
                            if (!is_on(sg + ds, q + dq, bx + db)) rim = true;
                const int k0 = cp.kbase + TB_TK * bx;
                bool zl = false;
                for (int k = std::max(k0 - 2, 0); k <= std::min(k0 + 65, g.n2 - 1); ++k)
                    zl = zl || sim.ax[2].node[size_t(k)].slot_e >= 0 || sim.ax[2].node[size_t(k)].slot_h >= 0;
                P.zblocks += zl;
                P.rim += rim;
                P.tb.push_back(make_int4(k0 | (zl ? TMA_ZL_TILE : 0) | (rim ? TB_RIM : 0), ja + TB_TJ * q, rsegs[sg].x,
                                         rsegs[sg].y));
                cand_of_tb.push_back(flat(sg, q, bx));
            }
    if (P.tb.empty()) { P.why = "no two-step tile"; return P; }
    // the tiles kept point into the candidates' id planes (a dropped candidate leaves its planes
    // unused); their tables are gathered in tile order
    {
        std::vector<float> tabs(P.tb.size() * LOCAL_CLASSES * TB_REC);
        for (size_t b = 0; b < P.tb.size(); ++b) {
            const size_t c = cand_of_tb[b];
            P.idbase.push_back(int(cand_idbase[c]));
            std::memcpy(tabs.data() + b * LOCAL_CLASSES * TB_REC, ctab.data() + c * LOCAL_CLASSES * TB_REC,
                        LOCAL_CLASSES * TB_REC * 4);
        }
        P.tables.swap(tabs);
    }
    // one-step tiles of a double step: those of the one-step plan no two-step tile replaces
    std::vector<int> seg_of(size_t(g.n0), -1);
    for (int sg = 0; sg < NS; ++sg)
        for (int i = rsegs[sg].x; i < rsegs[sg].y; ++i) seg_of[size_t(i)] = sg;
    auto two_step = [&](int i, int j, int k) {   // node (i, j, k) belongs to a two-step tile
        const int sg = seg_of[size_t(i)];
        if (sg < 0 || j < ja || j >= ja + TB_TJ * J) return false;
        int bx = (k - cp.kbase) / TB_TK;
        if (bx >= kt) bx = kt - 1;   // the last tile's extra column
        return bx >= 0 && on[flat(sg, (j - ja) / TB_TJ, bx)] != 0;
    };
    for (size_t b = 0; b < cp.blocks.size(); ++b) {
        const int4 bk = cp.blocks[b];
        const int k0 = bk.x & ~TMA_ZL_TILE;
        if (cp.own[b].x >= cp.own[b].y || !two_step(bk.z, cp.own[b].x, std::max(k0, cp.kbase)))
            P.cidx.push_back(int(b));
    }
    // Debye edges: one-step ones first (each node's first edge is found on the device)
    std::vector<size_t> first_c, first_r;
    for (size_t e = 0; e < perm.size(); ++e) {
        const auto& q = sim.debye_edges[perm[e]];
        const int i = int(q.id / (n1 * n2)), j = int((q.id / n2) % n1), k = int(q.id % n2);
        (two_step(i, j, k) ? first_r : first_c).push_back(e);
    }
    auto devid = [&](uint64_t id) { return (long long)(id / n2) * g.p2 + (long long)(id % n2); };
    for (auto* list : {&first_c, &first_r})
        for (size_t e : *list) {
            const auto& q = sim.debye_edges[perm[e]];
            P.dd_f.push_back((long long)q.comp * g.cs + devid(q.id));
            P.dd_s.push_back(uint32_t(e));
            P.dd_w.push_back(float(q.dd));
            P.dd_cb.push_back(sim.cb(q.comp, q.id));
        }
    P.dd_c = int(first_c.size());
    P.ok = true;
    return P;
}

bool encode_tb2_maps(Session& s, std::string& why) {
    const Geom& g = s.geom;
    float* E[3] = {s.e, s.e2, s.e3};
    float* H[3] = {s.h, s.h2, s.h3};
    const cuuint64_t dims[4] = {cuuint64_t(g.n2), cuuint64_t(g.n1), cuuint64_t(g.n0), 3};
    const cuuint64_t strides[3] = {cuuint64_t(g.p2) * 4, cuuint64_t(g.n1) * g.p2 * 4, cuuint64_t(g.cs) * 4};
    using L = Tb2Layout<3>;
    const cuuint32_t box_e[4] = {cuuint32_t(L::EW), cuuint32_t(L::ER), 1, 3};
    const cuuint32_t box_h[4] = {cuuint32_t(L::HW), cuuint32_t(L::HR), 1, 3};
    const cuuint32_t box_e1[4] = {cuuint32_t(TmaL<float>::EW), cuuint32_t(TmaL<float>::ER), 1, 3};
    const cuuint32_t box_h1[4] = {cuuint32_t(TmaL<float>::HW), cuuint32_t(TmaL<float>::HR), 1, 3};
    const long long zlen = g.psi_off[1 * 3 + 2] - g.psi_off[0 * 3 + 2];
    const cuuint64_t zd[4] = {cuuint64_t(g.pw), cuuint64_t(g.n1), cuuint64_t(g.n0), 2};
    const cuuint64_t zs[3] = {cuuint64_t(g.pw) * 4, cuuint64_t(g.n1) * g.pw * 4, cuuint64_t(zlen) * 4};
    const cuuint32_t zbh[4] = {cuuint32_t(g.pw), cuuint32_t(L::ZHR), 1, 2};
    const cuuint32_t zbe[4] = {cuuint32_t(g.pw), cuuint32_t(L::ZER), 1, 2};
    const cuuint32_t zb1[4] = {cuuint32_t(g.pw), cuuint32_t(TMA_TJ + 1), 1, 2};
    for (int q = 0; q < 3; ++q) {
        if (!encode(&s.tbm_e[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, E[q], 4, dims, strides, box_e, why)) return false;
        if (!encode(&s.tbm_h[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, H[q], 4, dims, strides, box_h, why)) return false;
        if (!encode(&s.d1_e[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, E[q], 4, dims, strides, box_e1, why)) return false;
        if (!encode(&s.d1_h[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, H[q], 4, dims, strides, box_h1, why)) return false;
        if (g.pml > 0) {
            float* ze = s.zslot[q] + g.psi_off[0 * 3 + 2];
            float* zh = s.zslot[q] + g.psi_off[9 + 0 * 3 + 2];
            if (!encode(&s.tbm_zh[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, zh, 4, zd, zs, zbh, why)) return false;
            if (!encode(&s.tbm_ze[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, ze, 4, zd, zs, zbe, why)) return false;
            if (!encode(&s.d1_pze[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, ze, 4, zd, zs, zb1, why)) return false;
            if (!encode(&s.d1_pzh[q], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, zh, 4, zd, zs, zb1, why)) return false;
        } else {
            s.tbm_zh[q] = s.tbm_ze[q] = s.d1_pze[q] = s.d1_pzh[q] = s.tma.c;   // never read without a CPML
        }
    }
    const cuuint64_t cd[3] = {cuuint64_t(TB_CW), 16, cuuint64_t(s.tb_planes)};
    const cuuint64_t cs2[2] = {cuuint64_t(TB_CW), cuuint64_t(16 * TB_CW)};
    const cuuint32_t cb[3] = {cuuint32_t(TB_CW), 16, 1};
    return encode(&s.tbm_c, CU_TENSOR_MAP_DATA_TYPE_UINT8, s.tb_ids, 3, cd, cs2, cb, why);
}

// The one-step march's launch over a block list, from set a to set b.
void launch_tma_slots(Session& s, bool all, int a, int b, cudaStream_t st) {
    float* E[3] = {s.e, s.e2, s.e3};
    float* H[3] = {s.h, s.h2, s.h3};
    TmaArgs args{s.geom, s.classes, E[b], H[b], s.sc.k_mu, s.clean_lo[2], s.clean_hi[1], s.clean_hi[2],
                 all ? s.tma_blocks : s.c_blocks, all ? s.tma_own : s.c_own, 0, 1, s.zslot[b], s.zslot[b],
                 all ? s.tables : s.c_tables, s.counter, s.error, s.wait_ns, -0.0f, s.stall_plane};
    const unsigned nb = unsigned(all ? s.tma.blocks : s.n_cblocks);
    with_tma_kernel(s.cid_bytes, s.local, false, s.tma.shape, [&](auto kern, int smem) {
        kern<<<nb, TMA_CONSUMERS + 32, smem, st>>>(s.d1_e[a], s.d1_h[a], s.tma.c, s.d1_pze[a], s.d1_pzh[a], args);
        return true;
    });
}

// The per-step terms after the field update (sources and inductors, then the port probes), as
// enqueue_step forms them.
void enqueue_lumped(Session& s, float* e_now, float* h_now, cudaStream_t st) {
    const Geom& g = s.geom;
    const bool lumped = s.n_sources || s.n_inductors, probes = s.n_ports && !s.quiet;
    if (lumped && probes && s.n_ports == 1) {
        k_lumped_probe<<<1, 256, 0, st>>>(s.sources, s.n_sources, s.inductors, s.n_inductors, s.sc, s.counter, e_now,
                                          s.probes, s.port_edges, s.loops, g.cs, h_now, s.series);
    } else {
        if (lumped) k_lumped<<<1, 256, 0, st>>>(s.sources, s.n_sources, s.inductors, s.n_inductors, s.sc, s.counter, e_now);
        if (probes) k_probe<<<s.n_ports, 256, 0, st>>>(s.probes, s.port_edges, s.loops, g.cs, e_now, h_now, s.counter, s.sc, s.series);
    }
}

// One step t -> t + 1 of the one-step kernels in the slot scheme: the march over all one-step
// tiles (all) or over those left beside the two-step tiles, the shell, Debye, sources, probes.
void enqueue_slot_one(Session& s, uint64_t t, bool all, cudaStream_t st,
                      std::vector<std::pair<const char*, cudaEvent_t>>* marks, bool last = true) {
    auto mark = [&](const char* name) {
        if (!marks) return;
        cudaEvent_t ev;
        cudaEventCreate(&ev);
        cudaEventRecord(ev, st);
        marks->push_back({name, ev});
    };
    const Geom& g = s.geom;
    const int a = int(t % 3), b = int((t + 1) % 3), par = int(t & 1);
    float* E[3] = {s.e, s.e2, s.e3};
    float* H[3] = {s.h, s.h2, s.h3};
    mark(all ? "fused_step" : "edge_step");
    launch_tma_slots(s, all, a, b, st);
    const unsigned shell_rows = s.shell.ra + s.shell.rb + s.shell.rc;
    if (shell_rows > 0) {
        const unsigned gb = (shell_rows + SHELL_THREADS / 32 - 1) / (SHELL_THREADS / 32);
        mark("shell_h");
        k_shell_h<<<gb, SHELL_THREADS, 0, st>>>(g, s.shell, s.kax, E[a], H[a], H[b], par ? s.psi_h2 : s.psi,
                                                par ? s.psi : s.psi_h2, s.zslot[a], s.zslot[b], s.sc.k_mu);
        mark("shell_e");
        switch (s.cid_bytes) {
            case 1: k_shell_e<uint8_t><<<gb, SHELL_THREADS, 0, st>>>(g, s.shell, s.kax, (const uint8_t*)s.node_class, s.classes, H[b], E[a], E[b], s.psi, s.zslot[a], s.zslot[b]); break;
            case 2: k_shell_e<uint16_t><<<gb, SHELL_THREADS, 0, st>>>(g, s.shell, s.kax, (const uint16_t*)s.node_class, s.classes, H[b], E[a], E[b], s.psi, s.zslot[a], s.zslot[b]); break;
            default: k_shell_e<uint32_t><<<gb, SHELL_THREADS, 0, st>>>(g, s.shell, s.kax, (const uint32_t*)s.node_class, s.classes, H[b], E[a], E[b], s.psi, s.zslot[a], s.zslot[b]); break;
        }
    }
    const int nd = all ? s.dd_all : s.dd_c;
    if (nd > 0) {
        mark("debye_post");
        k_debye_slots<<<(nd + 255) / 256, 256, 0, st>>>(s.dd_f, s.dd_s, s.dd_w, s.dd_cb, nd, E[a], s.debye_table,
                                                        s.dslot[a], s.dslot[b], E[b]);
    }
    if (s.n_sources || s.n_inductors || (s.n_ports && !s.quiet)) mark("lumped_probe");
    enqueue_lumped(s, E[b], H[b], st);
    if (last) mark(nullptr);
}

// Steps t -> t + 2: the two-step march over the interior tiles, beside (on the side stream when
// `fork`) the first one-step update of the other tiles and the shell; then the second.
void enqueue_slot_double(Session& s, uint64_t t, cudaStream_t st, bool fork,
                         std::vector<std::pair<const char*, cudaEvent_t>>* marks) {
    const int a = int(t % 3), b = int((t + 1) % 3), c = int((t + 2) % 3);
    float* E[3] = {s.e, s.e2, s.e3};
    float* H[3] = {s.h, s.h2, s.h3};
    Tb2Args ta{s.geom, s.sc.k_mu, s.tb_blocks, s.tb_idbase, s.tb_tables, E[b], H[b], E[c], H[c], s.zslot[b],
               s.zslot[b], s.zslot[c], s.zslot[c], s.dbase, s.dslot[a], s.dslot[b], s.dslot[c], s.debye_table,
               s.error, s.wait_ns};
    if (fork) {
        cudaEventRecord(s.fork_ev, st);
        cudaStreamWaitEvent(s.side, s.fork_ev, 0);
        enqueue_slot_one(s, t, false, s.side, nullptr);
        cudaEventRecord(s.join_ev, s.side);
    }
    if (marks) {
        cudaEvent_t ev;
        cudaEventCreate(&ev);
        cudaEventRecord(ev, st);
        marks->push_back({"two_step", ev});
    }
    k_tb2_step<3><<<unsigned(s.n_tb), TB_THREADS, s.tb_smem, st>>>(s.tbm_e[a], s.tbm_h[a], s.tbm_c, s.tbm_zh[a],
                                                                   s.tbm_ze[a], ta);
    if (fork) cudaStreamWaitEvent(st, s.join_ev, 0);
    else enqueue_slot_one(s, t, false, st, marks, false);
    enqueue_slot_one(s, t + 1, false, st, marks);
}

// The captured graph of `kind` (0: one step, 1: a double step, 2: 24 double steps) starting at a
// step of the given phase (t mod 6), captured on first use.
int slot_graph(Session& s, int kind, int phase, cudaGraphExec_t* out, std::string& err) {
    const int key = kind * 8 + phase;
    auto it = s.slot_graphs.find(key);
    if (it != s.slot_graphs.end()) { *out = it->second; return FG_OK; }
    FG_CUDA(cudaStreamSynchronize(s.stream));
    cudaGraph_t graph;
    FG_CUDA(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeThreadLocal));
    if (kind == 0) enqueue_slot_one(s, uint64_t(phase), true, s.stream, nullptr);
    else
        for (int q = 0; q < (kind == 1 ? 1 : 24); ++q) enqueue_slot_double(s, uint64_t(phase + 2 * q), s.stream, true, nullptr);
    cudaError_t ce = cudaStreamEndCapture(s.stream, &graph);
    if (ce != cudaSuccess) { err = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ce); return FG_ERR_CUDA; }
    cudaGraphExec_t ex;
    ce = cudaGraphInstantiate(&ex, graph, 0);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) { err = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ce); return FG_ERR_CUDA; }
    s.slot_graphs[key] = ex;
    *out = ex;
    return FG_OK;
}

// Device buffers, tensor maps and launch settings of the two-step mode.
int setup_slots(Session& s, const HostSim& sim, const SlotPlan& sp, long long psi_total, std::string& err) {
    const Geom& g = s.geom;
    auto alloc = [&](void** p, size_t bytes) -> int {
        FG_CUDA(cudaMalloc(p, std::max<size_t>(bytes, 256)));
        s.extra_allocs.push_back(*p);
        return FG_OK;
    };
    auto upload = [&](void* dst, const void* src, size_t bytes) -> int {
        if (bytes) FG_CUDA(cudaError_t(staged_upload(s.gpu, dst, src, bytes, s.stream)));
        s.h2d_bytes += bytes;
        return FG_OK;
    };
    const size_t fb = size_t(3 * g.cs) * 4;
    const size_t np = std::max<size_t>(sim.poles.size(), 1);
    const size_t ne = sp.dd_f.size();
    const size_t pz = size_t(std::max<long long>(psi_total, 1)) * 4;
    int rc = FG_OK;
    rc |= alloc((void**)&s.e3, fb);
    rc |= alloc((void**)&s.h3, fb);
    for (int q = 0; q < 3; ++q) {
        rc |= alloc((void**)&s.zslot[q], pz);
        rc |= alloc((void**)&s.dslot[q], std::max<size_t>(ne * np, 1) * 4);
    }
    if (rc) return rc;
    const size_t nnp = size_t(g.n0) * g.n1 * size_t(g.p2);
    if (ne) {
        rc |= alloc((void**)&s.dbase, nnp * 4);
        rc |= alloc((void**)&s.dd_f, ne * 8);
        rc |= alloc((void**)&s.dd_s, ne * 4);
        rc |= alloc((void**)&s.dd_w, ne * 4);
        rc |= alloc((void**)&s.dd_cb, ne * 4);
    }
    std::vector<int4> cb;
    std::vector<int2> co;
    std::vector<float> ct;
    for (int b : sp.cidx) {
        cb.push_back(sp.cp.blocks[size_t(b)]);
        co.push_back(sp.cp.own[size_t(b)]);
    }
    // the one-step tiles' coefficient tables, in the order of the double step's list
    std::vector<float> all_tables(size_t(s.tma.blocks) * LOCAL_CLASSES * 6);
    FG_CUDA(cudaMemcpy(all_tables.data(), s.tables, all_tables.size() * 4, cudaMemcpyDeviceToHost));
    for (int b : sp.cidx)
        ct.insert(ct.end(), all_tables.begin() + size_t(b) * LOCAL_CLASSES * 6,
                  all_tables.begin() + size_t(b + 1) * LOCAL_CLASSES * 6);
    rc |= alloc((void**)&s.c_blocks, cb.size() * sizeof(int4));
    rc |= alloc((void**)&s.c_own, co.size() * sizeof(int2));
    rc |= alloc((void**)&s.c_tables, ct.size() * 4);
    rc |= alloc((void**)&s.tb_blocks, sp.tb.size() * sizeof(int4));
    rc |= alloc((void**)&s.tb_idbase, sp.idbase.size() * 4);
    rc |= alloc((void**)&s.tb_ids, sp.ids.size());
    rc |= alloc((void**)&s.tb_tables, sp.tables.size() * 4);
    if (rc) return rc;
    for (float* p : {s.e3, s.h3}) FG_CUDA(cudaMemsetAsync(p, 0, fb, s.stream));
    for (int q = 0; q < 3; ++q) {
        FG_CUDA(cudaMemsetAsync(s.zslot[q], 0, pz, s.stream));
        FG_CUDA(cudaMemsetAsync(s.dslot[q], 0, std::max<size_t>(ne * np, 1) * 4, s.stream));
    }
    if (ne) {
        rc |= upload(s.dd_f, sp.dd_f.data(), ne * 8);
        rc |= upload(s.dd_s, sp.dd_s.data(), ne * 4);
        rc |= upload(s.dd_w, sp.dd_w.data(), ne * 4);
        rc |= upload(s.dd_cb, sp.dd_cb.data(), ne * 4);
    }
    rc |= upload(s.c_blocks, cb.data(), cb.size() * sizeof(int4));
    rc |= upload(s.c_own, co.data(), co.size() * sizeof(int2));
    rc |= upload(s.c_tables, ct.data(), ct.size() * 4);
    rc |= upload(s.tb_blocks, sp.tb.data(), sp.tb.size() * sizeof(int4));
    rc |= upload(s.tb_idbase, sp.idbase.data(), sp.idbase.size() * 4);
    rc |= upload(s.tb_ids, sp.ids.data(), sp.ids.size());
    rc |= upload(s.tb_tables, sp.tables.data(), sp.tables.size() * 4);
    if (rc) return rc;
    if (ne) {
        // each Debye node's first edge: the smallest state index among its edges
        FG_CUDA(cudaMemsetAsync(s.dbase, 0xff, nnp * 4, s.stream));
        k_debye_base<<<unsigned((ne + 255) / 256), 256, 0, s.stream>>>(s.dd_f, s.dd_s, (long long)ne, g.cs, s.dbase);
        FG_CUDA(cudaGetLastError());
    }
    FG_CUDA(cudaStreamSynchronize(s.stream));
    s.n_cblocks = int(cb.size());
    s.n_tb = int(sp.tb.size());
    s.tb_zblocks = sp.zblocks;
    s.tb_rim = sp.rim;
    s.dd_c = sp.dd_c;
    s.dd_all = int(ne);
    s.tb_planes = sp.ids.size() / (16 * TB_CW);
    // every tile's boxes and halo stay inside the grid and its buffers: origins along k on 16 bytes
    // (k0 - 4 floats, k0 a multiple of 8), planes i0 - 2 .. i1 + 1 and rows j0 - 2 .. j0 + 15 inside,
    // its class planes inside the id array, the z-slab rows inside the staged pitch
    if (g.pw > TB_PZW || sim.poles.size() > size_t(TB_NPMAX) || s.n_cblocks == 0) {
        err = "internal: two-step limits";
        return FG_ERR_INVALID;
    }
    for (size_t b = 0; b < sp.tb.size(); ++b) {
        const int4 t = sp.tb[b];
        const int k0 = t.x & ~(TMA_ZL_TILE | TB_RIM);
        const bool okb = k0 % 8 == 0 && k0 >= 0 && k0 < g.n2 && t.z >= 2 && t.w + 2 <= g.n0 && t.w > t.z &&
                         t.w - t.z <= TB_SEGMAX && t.y >= 2 && t.y + 16 <= g.n1 &&
                         size_t(sp.idbase[b]) + size_t(t.w - t.z + 2) <= s.tb_planes;
        if (!okb) { err = "internal: a two-step tile outside its limits"; return FG_ERR_INVALID; }
    }
    for (unsigned q : sp.dd_s)
        if (size_t(q) >= ne) { err = "internal: a Debye state index outside the state"; return FG_ERR_INVALID; }
    std::string why;
    if (!encode_tb2_maps(s, why)) { err = "two-step march: " + why; return FG_ERR_CUDA; }
    s.tb_smem = Tb2Layout<3>::TOTAL;
    FG_CUDA(cudaFuncSetAttribute(k_tb2_step<3>, cudaFuncAttributeMaxDynamicSharedMemorySize, s.tb_smem));
    FG_CUDA(cudaStreamCreateWithFlags(&s.side, cudaStreamNonBlocking));
    FG_CUDA(cudaEventCreateWithFlags(&s.fork_ev, cudaEventDisableTiming));
    FG_CUDA(cudaEventCreateWithFlags(&s.join_ev, cudaEventDisableTiming));
    s.slots = true;
    return FG_OK;
}

}  // namespace

// Wall-clock phases of session_new, printed to stderr when FIELDGRID_SETUP_TIMES=1.
struct PhaseClock {
    bool on = false;
    std::chrono::steady_clock::time_point t0 = std::chrono::steady_clock::now(), last = t0;
    std::string text;
    PhaseClock() { const char* v = std::getenv("FIELDGRID_SETUP_TIMES"); on = v && v[0] == '1'; }
    void mark(const char* what) {
        if (!on) return;
        const auto now = std::chrono::steady_clock::now();
        text += std::string(" ") + what + " " +
                std::to_string(std::chrono::duration<double, std::milli>(now - last).count()).substr(0, 6) + " ms;";
        last = now;
    }
    ~PhaseClock() {
        if (on) std::fprintf(stderr, "session_new:%s total %.1f ms\n", text.c_str(),
                             std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count());
    }
};

int session_new(Gpu* gpu, const HostSim& sim, const RunSpec& rs, Session** out, std::string& err) {
    PhaseClock clk;
    *out = nullptr;
    if (!gpu) { err = "no GPU: this engine has no CPU path"; return FG_ERR_NO_DEVICE; }
    FG_CUDA(cudaSetDevice(gpu->device));
    if (rs.driven >= sim.port_src.size()) { err = "the driven port does not exist"; return FG_ERR_INVALID; }
    auto s = std::make_unique<Session>();
    s->gpu = gpu;
    s->fused = rs.fused;
    const size_t n0 = sim.n[0], n1 = sim.n[1], n2 = sim.n[2], nn = sim.nn;
    if (n0 >= (1u << 31) || n1 >= (1u << 31) || n2 >= (1u << 31)) { err = "grid dimension too large"; return FG_ERR_INVALID; }
    Geom& g = s->geom;
    g.n0 = int(n0); g.n1 = int(n1); g.n2 = int(n2);
    g.pml = int(sim.pml);
    g.nn = (long long)nn;
    g.p2 = int((n2 + 31) & ~size_t(31));
    const size_t nnp = n0 * n1 * size_t(g.p2);   // device nodes, rows padded to the pitch
    g.cs = (long long)((nnp + 31) & ~size_t(31));
    const long long cs = g.cs;
    // reference node id (i*n1 + j)*n2 + k -> device node id (i*n1 + j)*p2 + k
    auto dev = [&](uint64_t id) { return (long long)(id / n2) * g.p2 + (long long)(id % n2); };
    auto fidx = [&](uint64_t key) { return (long long)(key / nn) * cs + dev(key % nn); };

    // psi slabs (run.rs:214-225): the 12 (field, component, axis) slabs of the reference, E
    // first, then H; per field the two z slabs (components 0 and 1, derivative along k) first and
    // adjacent, each slab 128-byte aligned, z-slab rows padded to pw slots
    g.pw = int((2 * sim.pml + 3) & ~size_t(3));
    long long psi_total = 0, psi_hbase = 0;
    for (int e = 0; e < 2; ++e) {
        if (e == 1) psi_hbase = psi_total;
        static const int order[6][2] = {{0, 2}, {1, 2}, {0, 1}, {1, 0}, {2, 0}, {2, 1}};  // (comp, axis)
        for (int c = 0; c < 3; ++c) g.psi_off[e * 9 + c * 3 + c] = psi_total;  // unused (axis == comp)
        for (const auto& ca : order) {
            g.psi_off[e * 9 + ca[0] * 3 + ca[1]] = psi_total;
            if (sim.pml > 0) {
                size_t m[3] = {n0, n1, n2};
                m[ca[1]] = ca[1] == 2 ? size_t(g.pw) : 2 * sim.pml;
                psi_total += (long long)((m[0] * m[1] * m[2] + 31) & ~size_t(31));
            }
        }
    }
    s->psi_total = psi_total;
    s->psi_hbase = psi_hbase;
    const long long psi_h = psi_total - psi_hbase;  // the H slabs, ping-ponged in the fused step

    // class ids narrowed to the smallest width that holds them
    const size_t ncls = sim.classes.size();
    s->cid_bytes = ncls <= 256 ? 1 : (ncls <= 65536 ? 2 : 4);
    if (rs.cid_bytes > s->cid_bytes) s->cid_bytes = rs.cid_bytes == 2 ? 2 : 4;

    // sparse lists (pack, run.rs:243-340)
    std::vector<DevSource> src;
    for (auto& q : sim.port_src[rs.driven]) src.push_back(DevSource{(long long)q.comp * cs + dev(q.id), q.src});
    std::vector<DevInductor> ind;
    for (auto& q : sim.inductors) ind.push_back(DevInductor{(long long)q.comp * cs + dev(q.id), q.ke, q.ki, 0.f});
    std::vector<DevWire> wires;
    for (auto& w : sim.wires) {
        DevWire d;
        d.h = fidx(w.h);
        for (int t = 0; t < 4; ++t) { d.e[t] = fidx(w.e[t]); d.c[t] = w.c[t]; }
        wires.push_back(d);
    }
    std::vector<DevSheet> sheets;
    for (auto& q : sim.sheets) {  // run.rs:261-289: z-directed sheets and k == 0 are skipped
        if (q.comp == 2 || q.id % n2 == 0) continue;
        long long hc = q.comp == 0 ? 1 : 0;
        DevSheet d{};
        d.f = (long long)q.comp * cs + dev(q.id);
        d.ha = hc * cs + dev(q.id);
        d.hb = hc * cs + dev(q.id) - 1;
        d.len = float(q.len);
        d.c = float(q.c);
        d.r = float(q.r);
        d.adaptive = q.adaptive ? 1.f : 0.f;
        d.ma = 0.5f;
        d.mb = 0.5f;
        d.face_a = unsigned(q.faces[0]);
        d.face_b = unsigned(q.faces[1]);
        sheets.push_back(d);
    }
    // the Debye edge list of the one-step scheme is formed on the device (below)
    std::vector<float> debye_table{float(sim.poles.size())};
    for (auto& [x, a] : sim.poles) {
        double d = 1.0 + 0.5 * x * sim.dt;
        debye_table.push_back(float((1.0 - 0.5 * x * sim.dt) / d));
        debye_table.push_back(float(EPS0 * a * x / d));
    }
    // nodes with per-step terms of their own (a two-step tile's halo must not reach them)
    std::vector<uint64_t> special;
    for (auto& q : sim.port_src[rs.driven]) special.push_back(q.id);
    for (auto& q : sim.inductors) special.push_back(q.id);
    for (auto& p : sim.ports)
        for (auto& col : p.columns)
            for (auto& e : col) special.push_back(sim.idx(e.at[0], e.at[1], e.at[2]));
    std::vector<DevProbe> probes;
    std::vector<DevPortEdge> pedges;
    std::vector<DevLoop> loops;
    for (auto& p : sim.ports) {  // run.rs:305-340 with port_loop (run.rs:102-127)
        const int axis = int(p.columns[0][0].comp);
        const int u = (axis + 1) % 3, v = (axis + 2) % 3;
        const auto& mid = p.columns[p.columns.size() / 2];
        DevProbe d{axis, int(pedges.size()), 0, int(loops.size()), 0};
        const double polarity = p.reference_above ? -1.0 : 1.0;
        const double weight = polarity / double(p.columns.size());
        for (auto& col : p.columns)
            for (auto& e : col)
                pedges.push_back(DevPortEdge{dev(sim.idx(e.at[0], e.at[1], e.at[2])),
                                             float(sim.ax[axis].d[e.at[axis]] * weight)});
        d.count = int(pedges.size()) - d.first;
        double height = 0.0;
        for (auto& e : mid) height += sim.ax[axis].d[e.at[axis]];
        std::set<std::pair<size_t, size_t>> nodes;
        for (auto& c : p.columns) nodes.insert({c[0].at[u], c[0].at[v]});
        for (auto& e : mid) {
            const size_t k = e.at[axis];
            const double share = polarity * sim.ax[axis].d[k] / height;
            auto at = [&](size_t a, size_t b) {
                size_t q[3];
                q[u] = a; q[v] = b; q[axis] = k;
                return sim.idx(q[0], q[1], q[2]);
            };
            std::map<std::pair<size_t, int>, int> turns;
            for (auto [a, b] : nodes) {
                turns[{at(a, b), v}] += 1;
                turns[{at(a - 1, b), v}] -= 1;
                turns[{at(a, b), u}] -= 1;
                turns[{at(a, b - 1), u}] += 1;
            }
            for (auto& [kc, t] : turns) {
                if (t == 0) continue;
                const size_t id = kc.first;
                special.push_back(uint64_t(id));
                const int comp = kc.second;
                const size_t pc = comp == 0 ? id / (n1 * n2) : (comp == 1 ? (id / n2) % n1 : id % n2);
                const double w = double(t) * sim.ax[comp].dd[pc];
                loops.push_back(DevLoop{(long long)comp * cs + dev(id), float(w * share)});
            }
        }
        d.loop_count = int(loops.size()) - d.loop_first;
        probes.push_back(d);
    }
    for (auto& p : sim.ports)  // run.rs:341-343, on the reference's node ids
        for (auto& col : p.columns)
            for (auto& e : col)
                if (float(sim.idx(e.at[0], e.at[1], e.at[2])) >= float(1u << 24)) {
                    err = "grid too large for f32 port indices";
                    return FG_ERR_PORT_INDEX;
                }

    clk.mark("lists");
    pulse_shape(rs.fc, s->t0, s->tau);
    StepConst& sc = s->sc;
    sc.k_mu = float(sim.dt / MU0);
    sc.dt = float(sim.dt);
    sc.t0 = float(s->t0);
    sc.tau = float(s->tau);
    sc.w0 = float(2.0 * PI * rs.f0);
    sc.nf = int(std::min<size_t>(rs.freqs.size(), 4));
    for (int q = 0; q < 4; ++q) sc.omega[q] = q < sc.nf ? float(2.0 * PI * rs.freqs[q]) : 0.f;
    sc.cap = unsigned(std::min<uint64_t>(rs.max_steps, 0xffffffffu));
    sc.ports = int(sim.ports.size());
    s->n_sources = int(src.size());
    s->n_inductors = int(ind.size());
    s->n_ports = int(probes.size());
    s->n_wires = int(wires.size());
    s->n_sheets = int(sheets.size());
    s->plane_k = int(rs.has_plane_k ? rs.plane_k : 0);
    s->plane_len = rs.has_plane_k ? uint64_t(n0) * n1 * sc.nf * 10 : 0;
    if (rs.has_plane_k && rs.plane_k >= n2) { err = "plane_k is outside the grid"; return FG_ERR_INVALID; }
    s->n_patches = rs.has_ntff ? int(rs.ntff.size() / 13) : 0;
    s->ntff_len = (s->n_patches > 0 && sc.nf > 0) ? uint64_t(s->n_patches) * sc.nf * 12 : 0;
    for (size_t q = 0; q < size_t(s->n_patches) * 13; ++q)
        if (q % 13 != 0 && rs.ntff[q] >= nn) { err = "an NTFF patch index is outside the grid"; return FG_ERR_INVALID; }
    s->series_len = uint64_t(sc.cap) * sc.ports * 2;
    // per-step pulse and phase tables (host libm, f32, the reference's expressions)
    std::vector<float> t_pulse(sc.cap), t_dft(size_t(sc.cap) * sc.nf * 4), t_far(size_t(sc.cap) * sc.nf * 4);
    {
        const float dt = sc.dt, t0 = sc.t0, tau = sc.tau, w0 = sc.w0;
        const int nf = sc.nf;
        const float* om = sc.omega;
#pragma omp parallel for schedule(static)
        for (long long n = 0; n < (long long)sc.cap; ++n) {
            const float t = (float(n) + 0.5f) * dt;
            const float x = (t - t0) / tau;
            t_pulse[n] = std::exp(-x * x) * std::cos(w0 * (t - t0));
            const float te = (float(n) + 1.0f) * dt, th = (float(n) + 0.5f) * dt;
            for (int k = 0; k < nf; ++k) {
                float* d = &t_dft[(size_t(n) * nf + k) * 4];
                d[0] = std::cos(om[k] * te) * dt;
                d[1] = -std::sin(om[k] * te) * dt;
                d[2] = std::cos(om[k] * th) * dt;
                d[3] = -std::sin(om[k] * th) * dt;
                float* f = &t_far[(size_t(n) * nf + k) * 4];
                f[0] = std::cos(-om[k] * te) * dt;
                f[1] = std::sin(-om[k] * te) * dt;
                f[2] = std::cos(-om[k] * th) * dt;
                f[3] = std::sin(-om[k] * th) * dt;
            }
        }
    }
    const size_t states = sim.sheet_states;
    const size_t nr_nc = sim.sheet_table.size() >= 2 ? size_t(sim.sheet_table[0]) + 2 * size_t(sim.sheet_table[1]) : 0;
    (void)states;

    clk.mark("tables");
    // per-region class tables for the TMA step (fused runs on sm_100), formed on the device below
    CleanPlan cp;
    SlotPlan sp;
    const bool z_layer = g.pml > 0 && g.pw <= TmaL<float>::PZW;
    if (s->fused && rs.tma && !(std::getenv("FIELDGRID_NO_TMA") && std::getenv("FIELDGRID_NO_TMA")[0] == '1')) {
        // the two-step mode: graph-stepped fused runs with no wires, sheets, NTFF, plane DFT, design
        // history, and at most TB_NPMAX Debye poles, on sm_100 (FIELDGRID_STEP_DEPTH=1 or 2 chooses)
        int dev = 0, major = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
        const char* dv = std::getenv("FIELDGRID_STEP_DEPTH");
        const int depth = dv && (dv[0] == '1' || dv[0] == '2') ? dv[0] - '0' : STEP_DEPTH_DEFAULT;
        const bool want = depth == 2 && rs.graphs && major >= 10 && s->n_wires == 0 && s->n_sheets == 0 &&
                          s->plane_len == 0 && s->ntff_len == 0 && !(rs.design && !rs.design->empty()) &&
                          sim.poles.size() <= size_t(TB_NPMAX) && (g.pml == 0 || z_layer);
        if (want) sp = plan_slots(sim, g, z_layer, special);
        cp = sp.ok ? sp.cp : plan_clean(sim, g, z_layer, rs.tma_seg);
        s->local = cp.ok;
    }
    clk.mark("plans");
    // the one-step Debye list exists in the two-step mode too: its fallback when the slot set-up
    // does not apply (a region with more classes than a local table)
    const size_t nd = sim.debye_edges.size();
    s->n_debye = int(nd);
    // size the arena
    const size_t fields = size_t(3 * cs);
    size_t need = 0;
    const int field_sets = s->fused ? 2 : 1;
    need += carve_size(fields * 4) * 2 * field_sets;
    need += carve_size(size_t(std::max<long long>(psi_total, 1)) * 4);
    if (s->fused) need += carve_size(size_t(std::max<long long>(psi_h, 1)) * 4);
    need += carve_size(nnp * size_t(s->cid_bytes));
    need += carve_size(ncls * sizeof(DevCoef));
    need += carve_size((n0 + n1 + n2) * sizeof(AxisNode));
    need += carve_size(10 * n2 * 4);
    need += carve_size(64);
    need += carve_size(std::max<uint64_t>(s->series_len, 1) * 4);
    need += carve_size(std::max<uint64_t>(s->plane_len, 1) * 4);
    need += carve_size(std::max<uint64_t>(s->ntff_len, 1) * 4);
    need += carve_size(std::max<size_t>(rs.ntff.size(), 1) * 4);
    need += carve_size(std::max<size_t>(src.size(), 1) * sizeof(DevSource));
    need += carve_size(std::max<size_t>(ind.size(), 1) * sizeof(DevInductor));
    need += carve_size(std::max<size_t>(probes.size(), 1) * sizeof(DevProbe));
    need += carve_size(std::max<size_t>(pedges.size(), 1) * sizeof(DevPortEdge));
    need += carve_size(std::max<size_t>(loops.size(), 1) * sizeof(DevLoop));
    need += carve_size(std::max<size_t>(wires.size(), 1) * sizeof(DevWire));
    need += carve_size(std::max<size_t>(sheets.size(), 1) * sizeof(DevSheet));
    need += carve_size(std::max<size_t>(sim.sheet_table.size(), 1) * 4);
    need += carve_size(std::max<size_t>(sheets.size() * nr_nc, 1) * 4);
    need += carve_size(std::max<size_t>(nd, 1) * 8);
    need += carve_size(std::max<size_t>(nd, 1) * 4) * 3;
    need += carve_size(std::max<size_t>(nd * sim.poles.size(), 1) * 4);
    // the host records, set-up only: packed to 8 bytes while staged where the device nodes allow
    const bool pack_debye = nnp < (size_t(1) << 30);
    need += carve_size(std::max<size_t>(nd, 1) * (pack_debye ? sizeof(PackedDebye) : sizeof(DebyeEdge)));
    need += carve_size(debye_table.size() * 4);
    need += carve_size(std::max<size_t>(t_pulse.size(), 1) * 4);
    need += carve_size(std::max<size_t>(t_dft.size(), 1) * 4) * 2;
    need += carve_size(ENERGY_BLOCKS * 8);
    need += carve_size(64);
    const size_t local_tables = cp.blocks.size() * LOCAL_CLASSES * 6;
    if (s->local) need += carve_size(nnp) + carve_size(local_tables * 4);
    need += carve_size(64);
    need += carve_size(cp.blocks.size() * sizeof(int4));
    need += carve_size(cp.own.size() * sizeof(int2));
    // the device's spare arena serves when it holds the need with at most a quarter (+64 MB) more
    Gpu* gp = s->gpu;
    if (gp->spare && !(gp->spare_bytes >= need && gp->spare_bytes <= need + need / 4 + (size_t(64) << 20))) {
        cudaFree(gp->spare);
        gp->spare = nullptr;
        gp->spare_bytes = 0;
    }
    if (!gp->spare) {
        size_t free_b = 0, total_b = 0;
        FG_CUDA(cudaMemGetInfo(&free_b, &total_b));
        if (need + (size_t(256) << 20) > free_b) {
            err = std::to_string(sim.cells()) + " cells is more than this GPU can hold";
            return FG_ERR_TOO_LARGE;
        }
    }
    FG_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
    if (gp->spare) {
        s->arena = static_cast<char*>(gp->spare);
        gp->spare = nullptr;
        gp->spare_bytes = 0;
    } else {
        FG_CUDA(cudaMalloc(&s->arena, need));
    }
    clk.mark("malloc");
    s->arena_bytes = need;
    char* cur = s->arena;
    s->e = carve<float>(cur, fields);
    s->h = carve<float>(cur, fields);
    if (s->fused) { s->e2 = carve<float>(cur, fields); s->h2 = carve<float>(cur, fields); }
    s->psi = carve<float>(cur, size_t(std::max<long long>(psi_total, 1)));
    if (s->fused) {
        // the H slabs of the second set live at psi_h2 + psi_hbase so the same offsets apply
        float* hb = carve<float>(cur, size_t(std::max<long long>(psi_h, 1)));
        s->psi_h2 = hb - psi_hbase;
    }
    s->node_class = carve<char>(cur, nnp * size_t(s->cid_bytes));
    s->classes = carve<DevCoef>(cur, ncls);
    s->axes = carve<AxisNode>(cur, n0 + n1 + n2);
    float* kax = carve<float>(cur, 10 * n2);   // the k axis as separate arrays (KAxis)
    s->counter = carve<unsigned>(cur, 16);
    s->series = carve<float>(cur, std::max<uint64_t>(s->series_len, 1));
    s->plane = carve<float>(cur, std::max<uint64_t>(s->plane_len, 1));
    s->ntff = carve<float>(cur, std::max<uint64_t>(s->ntff_len, 1));
    s->patch = carve<unsigned>(cur, std::max<size_t>(rs.ntff.size(), 1));
    s->sources = carve<DevSource>(cur, std::max<size_t>(src.size(), 1));
    s->inductors = carve<DevInductor>(cur, std::max<size_t>(ind.size(), 1));
    s->probes = carve<DevProbe>(cur, std::max<size_t>(probes.size(), 1));
    s->port_edges = carve<DevPortEdge>(cur, std::max<size_t>(pedges.size(), 1));
    s->loops = carve<DevLoop>(cur, std::max<size_t>(loops.size(), 1));
    s->wires = carve<DevWire>(cur, std::max<size_t>(wires.size(), 1));
    s->sheets = carve<DevSheet>(cur, std::max<size_t>(sheets.size(), 1));
    s->branch = carve<float>(cur, std::max<size_t>(sim.sheet_table.size(), 1));
    s->currents = carve<float>(cur, std::max<size_t>(sheets.size() * nr_nc, 1));
    s->debye_f = carve<long long>(cur, std::max<size_t>(nd, 1));
    s->debye_dd = carve<float>(cur, std::max<size_t>(nd, 1));
    s->debye_cb = carve<float>(cur, std::max<size_t>(nd, 1));
    s->debye_old = carve<float>(cur, std::max<size_t>(nd, 1));
    s->debye_state = carve<float>(cur, std::max<size_t>(nd * sim.poles.size(), 1));
    void* debye_raw = carve<char>(cur, std::max<size_t>(nd, 1) * (pack_debye ? sizeof(PackedDebye) : sizeof(DebyeEdge)));
    s->debye_table = carve<float>(cur, debye_table.size());
    float* d_pulse = carve<float>(cur, std::max<size_t>(t_pulse.size(), 1));
    float* d_dft = carve<float>(cur, std::max<size_t>(t_dft.size(), 1));
    float* d_far = carve<float>(cur, std::max<size_t>(t_far.size(), 1));
    sc.pulse = d_pulse;
    sc.dft = d_dft;
    sc.far = d_far;
    s->partial = carve<double>(cur, ENERGY_BLOCKS);
    s->error = carve<int>(cur, 16);
    if (s->local) {
        s->local_ids = carve<uint8_t>(cur, nnp);
        s->tables = carve<float>(cur, local_tables);
    }
    int* setup_flag = carve<int>(cur, 16);
    if (!cp.blocks.empty()) s->tma_blocks = carve<int4>(cur, cp.blocks.size());
    if (!cp.own.empty()) s->tma_own = carve<int2>(cur, cp.own.size());
    s->tma_plan_blocks = cp.blocks;
    s->tma.blocks = int(cp.blocks.size());
    s->tma.zblocks = cp.zblocks;
    s->tma.seg = cp.seg;
    s->shell = cp.shell;
    for (int q = 0; q < 3; ++q) { s->clean_lo[q] = cp.lo[q]; s->clean_hi[q] = cp.hi[q]; }
    if (size_t(cur - s->arena) > need) { err = "internal: arena overflow"; return FG_ERR_INVALID; }

    cudaStream_t st = s->stream;
    clk.mark("alloc");
    FG_CUDA(cudaMemsetAsync(s->arena, 0, need, st));
    // node classes, narrowed and laid out with the row pitch while they are staged for the upload
    {
        const uint32_t* src32 = sim.node_class.data();     // one of the two holds the ids
        const uint16_t* src16 = sim.node_class16.data();
        const bool s16 = !sim.node_class16.empty();
        const int cb = s->cid_bytes;
        const size_t p2 = size_t(g.p2);
        // columns [k0, kn) of row r into o as cb-byte ids, the pitch padding (k >= n2) zero
        auto row = [&](auto* in, auto* o, size_t k0, size_t kn) {
            using T = std::remove_pointer_t<decltype(o)>;
            const size_t kv = std::min(kn, n2);
            for (size_t k = k0; k < kv; ++k) o[k - k0] = T(in[k]);
            for (size_t k = std::max(k0, n2); k < kn; ++k) o[k - k0] = T(0);
        };
        auto narrow = [&](char* buf, size_t off, size_t n) {
            // bytes [off, off + n) of the pitched array: elements off / cb .. (off + n) / cb
            const size_t e0 = off / size_t(cb), e1 = (off + n) / size_t(cb);
            size_t e = e0;
            while (e < e1) {
                const size_t r = e / p2, k0 = e % p2, kn = std::min(p2, k0 + (e1 - e));
                char* o = buf + (e - e0) * size_t(cb);
                if (s16) {
                    const uint16_t* in = src16 + r * n2;
                    if (cb == 1) row(in, reinterpret_cast<uint8_t*>(o), k0, kn);
                    else if (cb == 2) row(in, reinterpret_cast<uint16_t*>(o), k0, kn);
                    else row(in, reinterpret_cast<uint32_t*>(o), k0, kn);
                } else {
                    const uint32_t* in = src32 + r * n2;
                    if (cb == 1) row(in, reinterpret_cast<uint8_t*>(o), k0, kn);
                    else if (cb == 2) row(in, reinterpret_cast<uint16_t*>(o), k0, kn);
                    else row(in, reinterpret_cast<uint32_t*>(o), k0, kn);
                }
                e += kn - k0;
            }
        };
        const size_t bytes = nnp * size_t(cb);
        FG_CUDA(cudaError_t(staged_fill(s->gpu, s->node_class, bytes, st, narrow)));
        s->h2d_bytes += bytes;
    }
    clk.mark("classes_up");
    std::vector<DevCoef> dcls(ncls);
    for (size_t q = 0; q < ncls; ++q) {
        for (int c = 0; c < 3; ++c) { dcls[q].ca[c] = sim.classes[q].ca[c]; dcls[q].cb[c] = sim.classes[q].cb[c]; }
        dcls[q].pad0 = dcls[q].pad1 = 0.f;
    }
    FG_CUDA(cudaMemcpyAsync(s->classes, dcls.data(), ncls * sizeof(DevCoef), cudaMemcpyHostToDevice, st));
    FG_CUDA(cudaStreamSynchronize(st));
    std::vector<AxisNode> axes;
    for (int a = 0; a < 3; ++a) axes.insert(axes.end(), sim.ax[a].node.begin(), sim.ax[a].node.end());
    FG_CUDA(cudaMemcpyAsync(s->axes, axes.data(), axes.size() * sizeof(AxisNode), cudaMemcpyHostToDevice, st));
    g.ax[0] = s->axes;
    g.ax[1] = s->axes + n0;
    g.ax[2] = s->axes + n0 + n1;
    {
        std::vector<float> kv(10 * n2);
        for (size_t k = 0; k < n2; ++k) {
            const AxisNode& a = sim.ax[2].node[k];
            const float f[8] = {a.inv_d, a.inv_dd, a.raw_inv_d, a.raw_inv_dd, a.be, a.ce, a.bh, a.ch};
            for (int q = 0; q < 8; ++q) kv[q * n2 + k] = f[q];
            std::memcpy(&kv[8 * n2 + k], &a.slot_e, 4);
            std::memcpy(&kv[9 * n2 + k], &a.slot_h, 4);
        }
        FG_CUDA(cudaMemcpyAsync(kax, kv.data(), kv.size() * 4, cudaMemcpyHostToDevice, st));
        s->kaxis_host = std::move(kv);   // the copy must outlive the asynchronous upload
        s->kax = KAxis{kax, kax + n2, kax + 2 * n2, kax + 3 * n2, kax + 4 * n2, kax + 5 * n2, kax + 6 * n2,
                       kax + 7 * n2, reinterpret_cast<const int*>(kax + 8 * n2), reinterpret_cast<const int*>(kax + 9 * n2)};
    }
    s->h2d_bytes += ncls * sizeof(DevCoef) + axes.size() * sizeof(AxisNode);
    auto up = [&](void* dst, const void* srcp, size_t bytes) -> int {
        s->h2d_bytes += bytes;
        if (bytes) FG_CUDA(cudaError_t(staged_upload(s->gpu, dst, srcp, bytes, st)));
        return FG_OK;
    };
    int rc = FG_OK;
    // the patch records word-major (k_ntff): word m of patch g at m * patches + g
    std::vector<uint32_t> patch_dev(rs.ntff.size());
    const size_t npatch = rs.ntff.size() / 13;
    for (size_t q = 0; q < rs.ntff.size(); ++q)
        patch_dev[(q % 13) * npatch + q / 13] = q % 13 == 0 ? rs.ntff[q] : uint32_t(dev(rs.ntff[q]));
    if (!rs.ntff.empty() && 3ull * uint64_t(cs) >= (1ull << 32)) { err = "the NTFF box needs 64-bit indices on this grid"; return FG_ERR_UNSUPPORTED; }
    rc |= up(s->patch, patch_dev.data(), patch_dev.size() * 4);
    rc |= up(s->sources, src.data(), src.size() * sizeof(DevSource));
    rc |= up(s->inductors, ind.data(), ind.size() * sizeof(DevInductor));
    rc |= up(s->probes, probes.data(), probes.size() * sizeof(DevProbe));
    rc |= up(s->port_edges, pedges.data(), pedges.size() * sizeof(DevPortEdge));
    rc |= up(s->loops, loops.data(), loops.size() * sizeof(DevLoop));
    rc |= up(s->wires, wires.data(), wires.size() * sizeof(DevWire));
    rc |= up(s->sheets, sheets.data(), sheets.size() * sizeof(DevSheet));
    rc |= up(s->branch, sim.sheet_table.data(), sim.sheet_table.size() * 4);
    if (pack_debye && nd) {
        const DebyeEdge* de = sim.debye_edges.data();
        const size_t p2 = size_t(g.p2);
        auto pack = [&](char* buf, size_t off, size_t n) {   // whole records: 1 MB parts hold 2^17 of them
            PackedDebye* o = reinterpret_cast<PackedDebye*>(buf);
            const size_t q0 = off / sizeof(PackedDebye), q1 = (off + n) / sizeof(PackedDebye);
            // the edges run in node order within a component: the row of the previous edge (its
            // first node rb, its index r) serves until an edge leaves it, so few edges divide
            uint64_t rb = 0, r = 0;   // row 0; an edge before rb wraps past n2 and divides
            for (size_t q = q0; q < q1; ++q) {
                const DebyeEdge& d = de[q];
                if (d.id - rb >= n2) {
                    r = d.id / n2;
                    rb = r * n2;
                }
                const size_t dv = r * p2 + (d.id - rb);
                o[q - q0] = PackedDebye{uint32_t(d.comp) << 30 | uint32_t(dv), float(d.dd)};
            }
        };
        const size_t bytes = nd * sizeof(PackedDebye);
        if (cudaError_t(staged_fill(s->gpu, debye_raw, bytes, st, pack)) != cudaSuccess) return FG_ERR_CUDA;
        s->h2d_bytes += bytes;
    } else {
        rc |= up(debye_raw, sim.debye_edges.data(), nd * sizeof(DebyeEdge));
    }
    rc |= up(s->debye_table, debye_table.data(), debye_table.size() * 4);
    rc |= up(d_pulse, t_pulse.data(), t_pulse.size() * 4);
    if (!cp.blocks.empty()) rc |= up(s->tma_blocks, cp.blocks.data(), cp.blocks.size() * sizeof(int4));
    if (!cp.own.empty()) rc |= up(s->tma_own, cp.own.data(), cp.own.size() * sizeof(int2));
    rc |= up(d_dft, t_dft.data(), t_dft.size() * 4);
    rc |= up(d_far, t_far.data(), t_far.size() * 4);
    if (rc) return FG_ERR_CUDA;
    // the Debye list and the per-block class tables from the uploaded node classes
    auto with_cid = [&](auto fn) {
        if (s->cid_bytes == 1) fn(static_cast<const uint8_t*>(s->node_class));
        else if (s->cid_bytes == 2) fn(static_cast<const uint16_t*>(s->node_class));
        else fn(static_cast<const uint32_t*>(s->node_class));
    };
    if (nd)
        with_cid([&](auto nc) {
            const unsigned grid = unsigned(std::min<size_t>((nd + 255) / 256, size_t(148) * 16));
            if (pack_debye)
                k_debye_lists_packed<<<grid, 256, 0, st>>>(static_cast<const PackedDebye*>(debye_raw), (long long)nd, nc,
                                                           s->classes, (long long)cs, s->debye_f, s->debye_dd,
                                                           s->debye_cb);
            else
                k_debye_lists<<<grid, 256, 0, st>>>(static_cast<const DebyeEdge*>(debye_raw), (long long)nd, nc,
                                                    s->classes, (long long)n2, (long long)g.p2, (long long)cs,
                                                    s->debye_f, s->debye_dd, s->debye_cb);
        });
    // the Debye ADE folded into the march (opt-in, FIELDGRID_DEBYE_FOLD=1: at 513^3 the march's
    // added per-plane work cost more than the separate list kernel): graph-stepped one-step TMA runs
    // with per-block tables, one pole, no sheets and no design history
    const char* fv = std::getenv("FIELDGRID_DEBYE_FOLD");
    bool fold = nd > 0 && s->local && !cp.blocks.empty() && !sp.ok && rs.graphs && s->fused && sim.poles.size() == 1 &&
                s->n_sheets == 0 && !(rs.design && !rs.design->empty()) && ncls + 1 < (size_t(1) << 29) &&
                fv && fv[0] == '1';
    std::vector<void*> scratch;   // set-up only
    struct Scratch {
        std::vector<void*>& v;
        ~Scratch() { for (void* p : v) cudaFree(p); }
    } scratch_guard{scratch};
    auto grab = [&](void** p, size_t bytes, bool keep) -> bool {
        if (cudaMalloc(p, std::max<size_t>(bytes, 4)) != cudaSuccess) { cudaGetLastError(); return false; }
        (keep ? s->extra_allocs : scratch).push_back(*p);
        return true;
    };
    uint8_t* dmask = nullptr;
    float* ddn = nullptr;
    if (fold) fold = grab((void**)&dmask, (nnp + 3) & ~size_t(3), false) && grab((void**)&ddn, size_t(3 * cs) * 4, false) &&
                     grab((void**)&s->lmask, cp.blocks.size() * LOCAL_CLASSES, true);
    if (fold) {
        FG_CUDA(cudaMemsetAsync(dmask, 0, (nnp + 3) & ~size_t(3), st));
        const unsigned grid = unsigned(std::min<size_t>((nd + 255) / 256, size_t(148) * 16));
        k_debye_node_mask<<<grid, 256, 0, st>>>(s->debye_f, s->debye_dd, (long long)nd, (long long)cs,
                                                reinterpret_cast<unsigned*>(dmask), ddn);
    }
    if (s->local && !cp.blocks.empty())
        with_cid([&](auto nc) {
            k_local_classes<<<unsigned(cp.blocks.size()), 256, 0, st>>>(nc, s->classes, s->tma_blocks, s->tma_own, g.n1,
                                                                       g.n2, g.p2, TMA_TK, cp.lo[2], cp.hi[2],
                                                                       s->local_ids, s->tables, setup_flag,
                                                                       fold ? dmask : nullptr,
                                                                       fold ? s->lmask : nullptr);
        });
    FG_CUDA(cudaGetLastError());
    int over = 0;
    FG_CUDA(cudaMemcpyAsync(&over, setup_flag, sizeof(int), cudaMemcpyDeviceToHost, st));
    FG_CUDA(cudaStreamSynchronize(st));
    if (over) {   // a region holds more classes than a local table: global ids, the list's Debye ADE
        s->local = false;
        fold = false;
    }
    if (fold) {
        // each (block, owned plane, row)'s folded edges, their offsets, their dd in march order
        const size_t nrow = cp.blocks.size() * size_t(TMA_SEGMAX) * 8;
        int *counts = nullptr, *keep = nullptr, *pos = nullptr;
        void* tmp = nullptr;
        size_t tmp_bytes = 0, tmp2 = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, counts, s->drow, int(nrow), st);
        cub::DeviceScan::ExclusiveSum(nullptr, tmp2, keep, pos, int(nd), st);
        fold = grab((void**)&counts, nrow * 4, false) && grab((void**)&s->drow, nrow * 4, true) &&
               grab((void**)&keep, nd * 4, false) && grab((void**)&pos, nd * 4, false) &&
               grab(&tmp, std::max(tmp_bytes, tmp2), false);
        if (fold) {
            FG_CUDA(cudaMemsetAsync(counts, 0, nrow * 4, st));
            const unsigned nb = unsigned(cp.blocks.size());
            k_fold_rows<false><<<nb, 256, 0, st>>>(s->tma_blocks, s->tma_own, g.n1, g.n2, g.p2, TMA_TJ, TMA_TK, cp.lo[2],
                                                  cp.hi[2], TMA_SEGMAX, dmask, (long long)cs, counts, ddn, nullptr);
            tmp_bytes = std::max(tmp_bytes, tmp2);
            FG_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, counts, s->drow, int(nrow), st));
            int tail[2] = {0, 0};
            FG_CUDA(cudaMemcpyAsync(&tail[0], s->drow + nrow - 1, 4, cudaMemcpyDeviceToHost, st));
            FG_CUDA(cudaMemcpyAsync(&tail[1], counts + nrow - 1, 4, cudaMemcpyDeviceToHost, st));
            FG_CUDA(cudaStreamSynchronize(st));
            s->nfold = tail[0] + tail[1];
            const size_t np = sim.poles.size();
            fold = grab((void**)&s->fdd, size_t(s->nfold) * 4, true) &&
                   grab((void**)&s->fstate, size_t(s->nfold) * np * 4, true);
        }
        if (fold) {
            FG_CUDA(cudaMemsetAsync(s->fstate, 0, std::max<size_t>(size_t(s->nfold) * sim.poles.size() * 4, 4), st));
            const unsigned nb = unsigned(cp.blocks.size());
            k_fold_rows<true><<<nb, 256, 0, st>>>(s->tma_blocks, s->tma_own, g.n1, g.n2, g.p2, TMA_TJ, TMA_TK, cp.lo[2],
                                                 cp.hi[2], TMA_SEGMAX, dmask, (long long)cs, s->drow, ddn, s->fdd);
            // the edges left to the list, compacted in list order
            const unsigned grid = unsigned(std::min<size_t>((nd + 255) / 256, size_t(148) * 16));
            k_debye_unfolded<<<grid, 256, 0, st>>>(s->debye_f, (long long)nd, ddn, keep);
            tmp_bytes = std::max(tmp_bytes, tmp2);
            FG_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, keep, pos, int(nd), st));
            int tail[2] = {0, 0};
            FG_CUDA(cudaMemcpyAsync(&tail[0], pos + nd - 1, 4, cudaMemcpyDeviceToHost, st));
            FG_CUDA(cudaMemcpyAsync(&tail[1], keep + nd - 1, 4, cudaMemcpyDeviceToHost, st));
            FG_CUDA(cudaStreamSynchronize(st));
            const size_t nres = size_t(tail[0]) + size_t(tail[1]);
            if (size_t(s->nfold) + nres != nd) { err = "internal: folded and listed Debye edges do not add up"; return FG_ERR_INVALID; }
            long long* f2 = nullptr;
            float *dd2 = nullptr, *cb2 = nullptr;
            if (!grab((void**)&f2, nres * 8, true) || !grab((void**)&dd2, nres * 4, true) || !grab((void**)&cb2, nres * 4, true)) {
                err = "out of device memory for the Debye list";
                return FG_ERR_CUDA;
            }
            k_debye_compact<<<grid, 256, 0, st>>>(s->debye_f, s->debye_dd, s->debye_cb, keep, pos, (long long)nd, f2, dd2,
                                                  cb2);
            FG_CUDA(cudaGetLastError());
            FG_CUDA(cudaStreamSynchronize(st));
            s->debye_f = f2;
            s->debye_dd = dd2;
            s->debye_cb = cb2;
            s->n_debye = int(nres);
            for (size_t k = 0; k < std::min<size_t>(sim.poles.size(), 2); ++k) {
                s->fdb[k] = debye_table[1 + 2 * k];
                s->fdc[k] = debye_table[2 + 2 * k];
            }
        }
    }
    s->fold = fold;
    FG_CUDA(cudaStreamSynchronize(st));   // the scratch goes with scratch_guard

    clk.mark("upload");
    if (rs.design && !rs.design->empty()) {
        if (!s->fused) { err = "design recording needs the fused step"; return FG_ERR_INVALID; }
        s->n_design = int(rs.design->size());
        s->design_in_steps = rs.design_in_steps;
        s->hist_cap = std::max(rs.hist_cap, 1);
        const size_t hb = size_t(s->hist_cap) * size_t(s->n_design) * 4;
        FG_CUDA(cudaMalloc(&s->design, rs.design->size() * sizeof(int4)));
        FG_CUDA(cudaMalloc(&s->hist_e, hb));
        FG_CUDA(cudaMalloc(&s->hist_s, hb));
        FG_CUDA(cudaMalloc(&s->hist_base, sizeof(long long)));
        FG_CUDA(cudaMemcpy(s->design, rs.design->data(), rs.design->size() * sizeof(int4), cudaMemcpyHostToDevice));
        FG_CUDA(cudaMemset(s->hist_base, 0, sizeof(long long)));
    }
    s->shape = choose_shape(g, s->cid_bytes, s->n_wires > 0);
    if (const char* v = std::getenv("FIELDGRID_TEST_WAIT_NS"))
        s->wait_ns = std::min<unsigned long long>(std::max<unsigned long long>(std::strtoull(v, nullptr, 10),
                                                                               tma::WAIT_LIMIT_MIN_NS), tma::WAIT_LIMIT_NS);
    if (const char* v = std::getenv("FIELDGRID_TEST_STALL_PLANE")) s->stall_plane = std::atoi(v);
    plan_tma(*s);
    clk.mark("tma_maps");
    if (sp.ok && s->tma.ok && s->local) {
        rc = setup_slots(*s, sim, sp, psi_total, err);
        if (rc) { session_free(s.release()); return rc; }
    }
    if (s->slots)
        s->variant = "two-step march over " + std::to_string(s->n_tb) + " tiles of 14x64 (" + std::to_string(s->tb_zblocks) +
                     " reaching the k layer, " + std::to_string(s->tb_rim) + " at the rim) beside the one-step TMA march on " +
                     std::to_string(s->n_cblocks) + " tiles of 7x64 and a CPML shell of " +
                     std::to_string(s->shell.ra + s->shell.rb + s->shell.rc) + " rows, " +
                     std::to_string(s->dd_all) + " Debye edges in time slots";
    else if (s->tma.ok)
        s->variant = "TMA fused march, tile " + std::to_string(s->tma.tj) + "x" + std::to_string(s->tma.tk) + ", " +
                     std::to_string(s->tma.seg) + " planes per block, " + std::to_string(s->tma.blocks) +
                     " blocks on the clean box (" + std::to_string(s->tma.zblocks) + " reaching the k layer), CPML shell of " +
                     std::to_string(s->shell.ra + s->shell.rb + s->shell.rc) + " rows, " +
                     std::to_string(TMA_SHAPES[s->tma.shape].stages) + " stages, " +
                     std::to_string(TMA_SHAPES[s->tma.shape].minb) + " blocks/SM, " +
                     (s->local ? "per-block class tables" : "global class table") +
                     (s->fold ? ", Debye ADE folded into the march for " + std::to_string(s->nfold) + " edges (" +
                                    std::to_string(s->n_debye) + " on the list)"
                              : std::string());
    else
        s->variant = s->fused ? fused_name(s->shape) + " (" + s->tma.why + ")" : std::string("separate H+E, 64x4 threads");
    s->launches = count_launches(*s);
    s->n_poles = int(sim.poles.size());
    s->currents_len = sheets.size() * nr_nc;
    s->ind_host = ind;
    clk.mark("slots");
    if (s->slots) {
        // single and double steps of every phase now; the 48-step graphs on first use
        for (int kind = 0; kind < 2 && !rc; ++kind)
            for (int ph = 0; ph < 6 && !rc; ++ph) {
                cudaGraphExec_t gx;
                rc = slot_graph(*s, kind, ph, &gx, err);
            }
        if (rc) { session_free(s.release()); return rc; }
    }
    clk.mark("graphs_slots");
    struct Done {   // the graph captures below are the last phase
        PhaseClock& c;
        ~Done() { c.mark("graphs"); }
    } done{clk};
    {
        // the shell's H update beside the march in captured steps, the
        // session's own graphs or a batch's branches (FIELDGRID_SHELL_SIDE=0: after it)
        const char* sv = std::getenv("FIELDGRID_SHELL_SIDE");
        const bool off = sv && sv[0] == '0';
        if (!off && !s->slots && s->fused && s->tma.ok && !s->direct && s->shell.ra + s->shell.rb + s->shell.rc > 0) {
            FG_CUDA(cudaDeviceGetStreamPriorityRange(&s->prio_lo, &s->prio_hi));
            FG_CUDA(cudaStreamCreateWithPriority(&s->shell_st, cudaStreamNonBlocking, s->prio_lo));
            FG_CUDA(cudaEventCreateWithFlags(&s->shell_fork, cudaEventDisableTiming));
            FG_CUDA(cudaEventCreateWithFlags(&s->shell_join, cudaEventDisableTiming));
        }
    }
    if (!rs.graphs || s->slots) {
        *out = s.release();
        return FG_OK;
    }
    if (s->fused && (s->plane_len || s->ntff_len) && s->n_wires == 0 && s->n_sheets == 0) {
        FG_CUDA(cudaStreamCreateWithFlags(&s->aux, cudaStreamNonBlocking));
        for (int p = 0; p < 2; ++p) {
            FG_CUDA(cudaEventCreateWithFlags(&s->aux_ready[p], cudaEventDisableTiming));
            FG_CUDA(cudaEventCreateWithFlags(&s->aux_done[p], cudaEventDisableTiming));
        }
    }
    // graphs: a pair and singles now, a block of even length (the fused step alternates buffers)
    // when a run first steps that far (a short run never needs it)
    s->graph_steps = 32;
    rc = capture(*s, 2, 0, &s->graph_two, err);
    if (!rc) rc = capture(*s, 1, 0, &s->graph_one[0], err);
    if (!rc && s->fused) rc = capture(*s, 1, 1, &s->graph_one[1], err);
    if (rc) { session_free(s.release()); return rc; }
    *out = s.release();
    return FG_OK;
}

void session_free(Session* s) {
    if (!s) return;
    if (s->gpu) cudaSetDevice(s->gpu->device);
    if (s->stream) cudaStreamSynchronize(s->stream);
    if (s->graph_many) cudaGraphExecDestroy(s->graph_many);
    if (s->graph_two) cudaGraphExecDestroy(s->graph_two);
    for (auto& gx : s->graph_one)
        if (gx) cudaGraphExecDestroy(gx);
    for (auto& kv : s->slot_graphs) cudaGraphExecDestroy(kv.second);
    for (void* p : s->extra_allocs) cudaFree(p);
    if (s->side) cudaStreamDestroy(s->side);
    if (s->shell_st) cudaStreamDestroy(s->shell_st);
    if (s->shell_fork) cudaEventDestroy(s->shell_fork);
    if (s->shell_join) cudaEventDestroy(s->shell_join);
    if (s->fork_ev) cudaEventDestroy(s->fork_ev);
    if (s->join_ev) cudaEventDestroy(s->join_ev);
    if (s->aux) cudaStreamDestroy(s->aux);
    for (int p = 0; p < 2; ++p) {
        if (s->aux_ready[p]) cudaEventDestroy(s->aux_ready[p]);
        if (s->aux_done[p]) cudaEventDestroy(s->aux_done[p]);
    }
    if (s->arena) {   // kept as the device's spare (the stream is idle), or released
        Gpu* gp = s->gpu;
        if (gp && !gp->spare) {
            gp->spare = s->arena;
            gp->spare_bytes = s->arena_bytes;
        } else {
            cudaFree(s->arena);
        }
    }
    cudaFree(s->design);
    cudaFree(s->hist_e);
    cudaFree(s->hist_s);
    cudaFree(s->hist_base);
    if (s->stream) cudaStreamDestroy(s->stream);
    delete s;
}

// Back to step 0: fields, psi, Debye and sheet state, inductor currents, records and the step
// counter cleared; coefficients and element lists kept.
int session_reset(Session* s, std::string& err) {
    FG_CUDA(cudaSetDevice(s->gpu->device));
    cudaStream_t st = s->stream;
    const size_t fb = size_t(3 * s->geom.cs) * 4;
    for (float* p : {s->e, s->h, s->e2, s->h2, s->e3, s->h3})
        if (p) FG_CUDA(cudaMemsetAsync(p, 0, fb, st));
    if (s->slots)
        for (int q = 0; q < 3; ++q) {
            FG_CUDA(cudaMemsetAsync(s->zslot[q], 0, size_t(std::max<long long>(s->psi_total, 1)) * 4, st));
            FG_CUDA(cudaMemsetAsync(s->dslot[q], 0, std::max<size_t>(size_t(s->dd_all) * size_t(std::max(s->n_poles, 1)), 1) * 4, st));
        }
    FG_CUDA(cudaMemsetAsync(s->psi, 0, size_t(std::max<long long>(s->psi_total, 1)) * 4, st));
    if (s->fused && s->psi_total > s->psi_hbase)
        FG_CUDA(cudaMemsetAsync(s->psi_h2 + s->psi_hbase, 0, size_t(s->psi_total - s->psi_hbase) * 4, st));
    FG_CUDA(cudaMemsetAsync(s->counter, 0, 16 * sizeof(unsigned), st));
    FG_CUDA(cudaMemsetAsync(s->series, 0, std::max<uint64_t>(s->series_len, 1) * 4, st));
    FG_CUDA(cudaMemsetAsync(s->plane, 0, std::max<uint64_t>(s->plane_len, 1) * 4, st));
    FG_CUDA(cudaMemsetAsync(s->ntff, 0, std::max<uint64_t>(s->ntff_len, 1) * 4, st));
    if (s->n_debye) {
        FG_CUDA(cudaMemsetAsync(s->debye_old, 0, size_t(s->n_debye) * 4, st));
        FG_CUDA(cudaMemsetAsync(s->debye_state, 0, size_t(s->n_debye) * size_t(std::max(s->n_poles, 1)) * 4, st));
    }
    if (s->fold && s->nfold)
        FG_CUDA(cudaMemsetAsync(s->fstate, 0, size_t(s->nfold) * size_t(std::max(s->n_poles, 1)) * 4, st));
    if (s->currents_len) FG_CUDA(cudaMemsetAsync(s->currents, 0, s->currents_len * 4, st));
    if (!s->ind_host.empty())
        FG_CUDA(cudaMemcpyAsync(s->inductors, s->ind_host.data(), s->ind_host.size() * sizeof(DevInductor),
                                cudaMemcpyHostToDevice, st));
    FG_CUDA(cudaStreamSynchronize(st));
    s->steps = 0;
    return FG_OK;
}

int session_step(Session* s, uint64_t k, std::string& err) {
    if (!s->slots && !s->graph_one[0]) { err = "this session steps only as part of a batch"; return FG_ERR_INVALID; }
    FG_CUDA(cudaSetDevice(s->gpu->device));
    uint64_t done = 0;
    if (s->slots) {
        // 48 steps (24 double steps) keep the phase t mod 6 of the sets, slots and parity
        while (done < k) {
            const uint64_t left = k - done;
            const int kind = left >= 48 ? 2 : (left >= 2 ? 1 : 0);
            cudaGraphExec_t gx;
            int rc = slot_graph(*s, kind, int(s->steps % 6), &gx, err);
            if (rc) return rc;
            FG_CUDA(cudaGraphLaunch(gx, s->stream));
            const uint64_t n = kind == 2 ? 48 : (kind == 1 ? 2 : 1);
            done += n;
            s->steps += n;
        }
        FG_CUDA(cudaGetLastError());
        return FG_OK;
    }
    // the fused step alternates buffers: a whole graph block needs an even start
    while (done < k) {
        const uint64_t left = k - done;
        const int parity = s->fused ? int(s->steps & 1) : 0;
        if (parity == 0 && left >= uint64_t(s->graph_steps)) {
            if (!s->graph_many) {
                const int rc = capture(*s, s->graph_steps, 0, &s->graph_many, err);
                if (rc) return rc;
            }
            FG_CUDA(cudaGraphLaunch(s->graph_many, s->stream));
            done += s->graph_steps;
            s->steps += s->graph_steps;
        } else if (parity == 0 && left >= 2) {
            FG_CUDA(cudaGraphLaunch(s->graph_two, s->stream));
            done += 2;
            s->steps += 2;
        } else {
            FG_CUDA(cudaGraphLaunch(s->graph_one[parity], s->stream));
            done += 1;
            s->steps += 1;
        }
    }
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

int session_sync(Session* s, std::string& err) {
    FG_CUDA(cudaSetDevice(s->gpu->device));
    FG_CUDA(cudaStreamSynchronize(s->stream));
    return FG_OK;
}

// The buffers that hold the latest fields: after an odd number of fused steps, the second set.
static void latest(const Session* s, float** e, float** h) {
    if (s->slots) {
        float* E[3] = {s->e, s->e2, s->e3};
        float* H[3] = {s->h, s->h2, s->h3};
        *e = E[s->steps % 3];
        *h = H[s->steps % 3];
        return;
    }
    if (s->fused && (s->steps & 1)) { *e = s->e2; *h = s->h2; }
    else { *e = s->e; *h = s->h; }
}

int session_energy(Session* s, double* out, std::string& err) {
    FG_CUDA(cudaSetDevice(s->gpu->device));
    float *e, *h;
    latest(s, &e, &h);
    k_energy<<<ENERGY_BLOCKS, 256, 0, s->stream>>>(s->geom, e, h, s->partial);
    FG_CUDA(cudaGetLastError());
    std::vector<double> part(ENERGY_BLOCKS);
    FG_CUDA(cudaMemcpyAsync(part.data(), s->partial, ENERGY_BLOCKS * 8, cudaMemcpyDeviceToHost, s->stream));
    s->d2h_bytes += ENERGY_BLOCKS * 8;
    FG_CUDA(cudaStreamSynchronize(s->stream));
    int flag = 0;
    FG_CUDA(cudaMemcpy(&flag, s->error, sizeof(int), cudaMemcpyDeviceToHost));
    if (flag) {
        err = "a bounded wait in the fused step ran out (code " + std::to_string(flag) + ")";
        return FG_ERR_CUDA;
    }
    double sum = 0.0;
    for (double v : part) sum += v;
    *out = sum;
    return FG_OK;
}

uint64_t session_steps(const Session* s) { return s->steps; }

int session_read(Session* s, const std::string& which, float* dst, uint64_t len, std::string& err) {
    FG_CUDA(cudaSetDevice(s->gpu->device));
    FG_CUDA(cudaStreamSynchronize(s->stream));
    auto copy = [&](const float* src, uint64_t n) -> int {
        if (n > len) { err = "destination too small for " + which; return FG_ERR_INVALID; }
        if (n) FG_CUDA(cudaMemcpy(dst, src, n * 4, cudaMemcpyDeviceToHost));
        s->d2h_bytes += n * 4;
        return FG_OK;
    };
    if (which == "series") {
        uint64_t n = std::min<uint64_t>(s->steps, s->sc.cap) * uint64_t(s->sc.ports) * 2;
        return copy(s->series, n);
    }
    if (which == "plane") return copy(s->plane, s->plane_len);
    if (which == "ntff") {
        // the device keeps (frequency, value) major; the record is patch major (cpu.rs:363-415)
        if (s->ntff_len > len) { err = "destination too small for ntff"; return FG_ERR_INVALID; }
        std::vector<float> t(s->ntff_len);
        if (s->ntff_len) FG_CUDA(cudaMemcpy(t.data(), s->ntff, s->ntff_len * 4, cudaMemcpyDeviceToHost));
        s->d2h_bytes += s->ntff_len * 4;
        const uint64_t P = uint64_t(s->n_patches), per = uint64_t(s->sc.nf) * 12;
        for (uint64_t g = 0; g < P; ++g)
            for (uint64_t m = 0; m < per; ++m) dst[g * per + m] = t[m * P + g];
        return FG_OK;
    }
    if (which == "e" || which == "h") {
        float *e, *h;
        latest(s, &e, &h);
        const float* src = which == "e" ? e : h;
        const uint64_t nn = uint64_t(s->geom.nn);
        if (3 * nn > len) { err = "destination too small for " + which; return FG_ERR_INVALID; }
        const Geom& g = s->geom;
        for (int c = 0; c < 3; ++c)
            FG_CUDA(cudaMemcpy2D(dst + c * nn, size_t(g.n2) * 4, src + c * g.cs, size_t(g.p2) * 4, size_t(g.n2) * 4,
                                 size_t(g.n0) * g.n1, cudaMemcpyDeviceToHost));
        s->d2h_bytes += 3 * nn * 4;
        return FG_OK;
    }
    err = "unknown buffer " + which;
    return FG_ERR_INVALID;
}

void* session_stream(Session* s) { return s->stream; }
uint64_t session_launches_per_step(const Session* s) { return s->launches; }
uint64_t session_device_bytes(const Session* s) { return s->arena_bytes; }
const char* session_variant(const Session* s) { return s->variant.c_str(); }
uint64_t session_ports(const Session* s) { return uint64_t(s->sc.ports); }
uint64_t session_plane_len(const Session* s) { return s->plane_len; }
uint64_t session_ntff_len(const Session* s) { return s->ntff_len; }
double session_t0(const Session* s) { return s->t0; }

int session_kernel_times(Session* s, uint64_t steps, std::vector<std::pair<std::string, double>>& out,
                         std::string& err);

// Per-kernel device times, printed like report_kernel_times (run.rs:153-176). It steps the
// session, so the run loop calls it only after its last step.
void session_profile(Session* s) {
    std::string err;
    std::vector<std::pair<std::string, double>> t;
    if (session_kernel_times(s, 20, t, err)) {
        std::fprintf(stderr, "fdtd kernel times unavailable: %s\n", err.c_str());
        return;
    }
    double step = 0.0;
    for (auto& [name, ms] : t) {
        std::fprintf(stderr, "fdtd kernel %s: %.1f us over 20 launches\n", name.c_str(), 1e3 * ms);
        step += ms;
    }
    std::fprintf(stderr, "fdtd kernel time per step: %.1f us (%s)\n", 1e3 * step, s->variant.c_str());
}

// Launches `steps` steps one kernel at a time with an event before each launch.
int session_kernel_times(Session* s, uint64_t steps, std::vector<std::pair<std::string, double>>& out,
                         std::string& err) {
    FG_CUDA(cudaSetDevice(s->gpu->device));
    std::vector<std::pair<const char*, cudaEvent_t>> marks;
    std::vector<std::pair<std::string, double>> sums;
    std::vector<int> counts;
    // the two-step mode times double steps (one stream) and reports each kernel's time per step
    const uint64_t per = s->slots ? 2 : 1;
    for (uint64_t q = 0; q < steps; q += per) {
        marks.clear();
        if (s->slots) {
            enqueue_slot_double(*s, s->steps, s->stream, false, &marks);
        } else {
            s->marks = &marks;
            int rc = enqueue_step(*s, s->fused ? int(s->steps & 1) : 0, err);
            s->marks = nullptr;
            if (rc) return rc;
        }
        s->steps += per;
        FG_CUDA(cudaStreamSynchronize(s->stream));
        for (size_t m = 0; m + 1 < marks.size(); ++m) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, marks[m].second, marks[m + 1].second);
            if (sums.size() <= m) { sums.push_back({marks[m].first, 0.0}); counts.push_back(0); }
            sums[m].second += ms;
            counts[m] += 1;
        }
        for (auto& mk : marks) cudaEventDestroy(mk.second);
    }
    out.clear();
    for (size_t m = 0; m < sums.size(); ++m) {
        const double ms = sums[m].second / std::max(counts[m], 1) / double(per);
        bool merged = false;   // a kernel that runs twice in a double step: its two launches summed
        for (auto& o : out)
            if (o.first == sums[m].first) { o.second += ms; merged = true; }
        if (!merged) out.push_back({sums[m].first, ms});
    }
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

uint64_t session_h2d_bytes(const Session* s) { return s->h2d_bytes; }
uint64_t session_d2h_bytes(const Session* s) { return s->d2h_bytes; }

}  // namespace fg

#include "adjoint.cuh"
#include "batch.cuh"
#include "fp64_forward.cuh"
