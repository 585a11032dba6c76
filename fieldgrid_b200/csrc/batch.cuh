// Many independent grids of uneven sizes stepped together: one persistent launch per step marches
// every grid's tiles from a shared work-list, then one launch each applies every grid's Debye
// edges, sources and port probes, and the step loop is captured in a CUDA graph. Each grid keeps
// its own buffers, coefficients, CPML and element lists (a Session built without graphs), so the
// arithmetic is per grid exactly that of stepping it alone with the direct-load march.
//
// Work items: for grid b, tiles_k x tiles_j tiles of TJ x TK columns times ceil(n0 / seg) x-segments;
// item numbers are prefix-summed over the grids, and a block takes the next item from an atomic
// counter (reset at the start of every step), finds its grid by binary search over the prefix
// sums, and marches that tile (fused_tile, stencil_fused.cuh). Large grids therefore fill the GPU
// while small ones finish in the same launch, with no per-grid launch or tail.
//
// Merged mode (tile 5): one launch of the TMA march over every grid's clean box (k_batch_tma: the
// grids' tensor maps and march arguments in HBM, one block per tile of any grid), one launch each
// of the two CPML shell kernels over every grid's shell rows, then the Debye, source and probe
// launches above: seven launches per step for the whole batch, with each grid's arithmetic that of
// its own TMA step.
//
// The autotuner times a few steps of each candidate (tile shape, blocks per SM of the persistent
// launch, planes per item; graph branches; the merged launches) on the real batch, keeps the
// fastest, resets every grid to step 0 and captures the graphs with it.
//
// Included at the end of engine.cu (it builds on Session).
#pragma once

namespace fg {

struct BatchInstance {
    FusedArgs a[2];                 // the march's arguments for input set 0 / 1
    int tiles_k, tiles_j, seg;
    const long long* debye_f;
    const float* debye_dd;
    int n_debye;
    const float* debye_table;
    float* debye_state;
    const DevSource* src;
    int ns;
    DevInductor* ind;
    int ni;
    StepConst sc;
    unsigned* counter;
    const DevProbe* probes;
    const DevPortEdge* pe;
    const DevLoop* lp;
    int n_ports;
    float* series;
    float* e[2];
    float* h[2];
    int opens;                      // 1: k_batch_begin opens this grid's step (0: its own march does)
};

// the index b with first[b] <= t < first[b + 1]
__device__ __forceinline__ int batch_find(const long long* __restrict__ first, int n, long long t) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (first[mid] <= t) lo = mid;
        else hi = mid;
    }
    return lo;
}

// Opens step n of every grid (the counters the later kernels read) and rewinds the work-list.
__global__ void k_batch_begin(const BatchInstance* __restrict__ bi, int n, unsigned long long* queue) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n && bi[t].opens) *bi[t].counter += 1u;
    if (t == 0) *queue = 0ull;
}

template <typename CID, int TK, int TJ>
__global__ void __launch_bounds__(TK* TJ) k_batch_march(const BatchInstance* __restrict__ bi,
                                                        const long long* __restrict__ first, int n,
                                                        unsigned long long* queue, int parity) {
    __shared__ float hs[2][3][TJ + 1][TK + 1];
    __shared__ long long item;
    const long long total = first[n];
    for (;;) {
        __syncthreads();   // the previous item's tile is read no more
        if (threadIdx.x == 0 && threadIdx.y == 0) item = (long long)atomicAdd(queue, 1ull);
        __syncthreads();
        const long long it = item;
        if (it >= total) return;
        const int b = batch_find(first, n, it);
        const BatchInstance& in = bi[b];
        const long long l = it - first[b];
        const int per = in.tiles_k * in.tiles_j;
        const int bz = int(l / per), r = int(l - (long long)bz * per);
        const int i0 = bz * in.seg;
        const FusedArgs& a = in.a[parity];
        fused_tile<CID, TK, TJ>(a, hs, r % in.tiles_k, r / in.tiles_k, i0, min(i0 + in.seg, a.g.n0));
    }
}

template <typename CID>
__global__ void k_batch_debye(const BatchInstance* __restrict__ bi, const long long* __restrict__ first, int n,
                              int parity) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= first[n]) return;
    const int b = batch_find(first, n, t);
    const BatchInstance& in = bi[b];
    debye_post_edge<CID>(int(t - first[b]), in.debye_f, in.debye_dd, in.n_debye, nullptr, in.e[parity],
                         static_cast<const CID*>(in.a[0].node_class), in.a[0].classes, in.a[0].g.cs, in.debye_table,
                         in.debye_state, in.e[1 - parity]);
}

// one block per grid
__global__ void k_batch_lumped(const BatchInstance* __restrict__ bi, int parity) {
    const BatchInstance& in = bi[blockIdx.x];
    lumped_block(in.src, in.ns, in.ind, in.ni, in.sc, in.counter, in.e[1 - parity]);
}

// one block per port of any grid
__global__ void __launch_bounds__(256) k_batch_probe(const BatchInstance* __restrict__ bi,
                                                     const long long* __restrict__ first, int n, int parity) {
    const int b = batch_find(first, n, blockIdx.x);
    const BatchInstance& in = bi[b];
    probe_block(int(blockIdx.x - first[b]), in.probes, in.pe, in.lp, in.a[0].g.cs, in.e[1 - parity],
                in.h[1 - parity], in.counter, in.sc, in.series);
}

struct BatchShape {
    int tile = 0;             // 0: 32 x 8, 1: 64 x 4, 2: 32 x 4 (TK x TJ); 3: graph branches; 4: the same
                              // with the direct-load march for the small grids
    int blocks_per_sm = 0;    // persistent blocks per SM; 0: the occupancy limit
    int seg = 32;             // x-planes per work item; tile 4: the grids of fewer than seg thousand
                              // nodes march direct (0: all)
};

// tile 3 is the other execution mode: one graph branch per grid, each running that grid's own
// step (TMA march where it has a clean box, CPML shell, Debye, sources, probes) on its stream;
// branches run concurrently
constexpr int BATCH_BRANCHES = 3;          // graph branches, each grid's own step (TMA march + shell)
constexpr int BATCH_BRANCHES_DIRECT = 4;   // graph branches with the direct-load fused march
constexpr int BATCH_MERGED = 5;            // one TMA march and one shell launch over all grids

constexpr int BATCH_TILES[3][2] = {{32, 8}, {64, 4}, {32, 4}};

struct Batch {
    Gpu* gpu = nullptr;
    cudaStream_t stream = nullptr;
    std::vector<Session*> s;
    int cid_bytes = 1;
    BatchShape shape{};
    BatchInstance* d_inst = nullptr;
    long long* d_items = nullptr;   // n + 1 prefix sums of work items
    long long* d_edges = nullptr;   // n + 1 prefix sums of Debye edges
    long long* d_ports = nullptr;   // n + 1 prefix sums of ports
    unsigned long long* d_queue = nullptr;
    std::vector<BatchInstance> inst;
    long long total_edges = 0, total_ports = 0;
    int persistent_blocks = 0;
    uint64_t steps = 0;
    int graph_steps = 0;
    cudaGraphExec_t graph_many = nullptr, graph_one[2] = {nullptr, nullptr};
    double tuned_ms = 0;      // ms per step of the chosen shape while tuning
    std::vector<std::pair<BatchShape, double>> trials;
    cudaEvent_t fork = nullptr;        // graph branches: the fork and one join per grid
    std::vector<cudaEvent_t> join;
    // merged mode
    bool merged_ok = false;
    std::string merged_why;
    TmaGrid* d_tma = nullptr;          // the merged grids: per-block class tables first, then global ids
    int* d_tma_block = nullptr;        // per march block: its grid
    int tma_blocks = 0, tma_blocks_local = 0;   // blocks in all, blocks of the first launch
    ShellGrid* d_shell = nullptr;
    int* d_shell_block = nullptr;      // per shell block: its grid
    int shell_blocks = 0;
    std::vector<int> merged_rest;      // grids the merged launches leave to their own direct-load march
};

constexpr auto batch_tma_local =
    k_batch_tma<TMA_TJ, TMA_TK, uint8_t, TMA_SHAPES[0].stages, TMA_SEGMAX, true, TMA_SHAPES[0].minb>;
template <typename CID>
constexpr auto batch_tma_global = k_batch_tma<TMA_TJ, TMA_TK, CID, TMA_SHAPES[0].stages, TMA_SEGMAX, false, TMA_SHAPES[0].minb>;

// f(kernel, smem) for the merged march of grids with (local) or without per-block tables
template <typename F>
void with_batch_tma(bool local, int cid_bytes, F&& f) {
    if (local) f(batch_tma_local, tma_smem_s<uint8_t, true, 0>());
    else if (cid_bytes == 1) f(batch_tma_global<uint8_t>, tma_smem_s<uint8_t, false, 0>());
    else if (cid_bytes == 2) f(batch_tma_global<uint16_t>, tma_smem_s<uint16_t, false, 0>());
    else f(batch_tma_global<uint32_t>, tma_smem_s<uint32_t, false, 0>());
}

// The merged mode's descriptors: the grids with per-block class tables march in one launch, those
// with global class ids in a second (as each grid's own session chose); a grid without a TMA march
// (no clean box) runs its own direct-load march in the step.
int batch_merged_setup(Batch& B, std::string& err) {
    B.merged_ok = false;
    B.merged_rest.clear();
    B.tma_blocks_local = 0;
    std::vector<TmaGrid> tg;
    std::vector<int> tblock, sblock;
    std::vector<ShellGrid> sg;
    std::vector<size_t> order;   // the grids with tables first
    for (int pass = 0; pass < 2; ++pass)
        for (size_t b = 0; b < B.s.size(); ++b)
            if (B.s[b]->tma.ok && B.s[b]->tma.shape == 0 && B.s[b]->local == (pass == 0)) order.push_back(b);
    for (size_t b = 0; b < B.s.size(); ++b)
        if (!B.s[b]->tma.ok || B.s[b]->tma.shape != 0) B.merged_rest.push_back(int(b));
    for (size_t b : order) {
        Session& s = *B.s[b];
        if (s.local) B.tma_blocks_local = int(tblock.size()) + s.tma.blocks;
        const TmaPlan& t = s.tma;
        TmaGrid G{};
        for (int p = 0; p < 2; ++p) { G.e[p] = t.e[p]; G.h[p] = t.h[p]; G.pzh[p] = t.pz ? t.pzh[p] : t.c; }
        G.c = t.c;
        G.pze = t.pz ? t.pze : t.c;
        // the grid's first block in its launch (the second launch starts after the local grids' blocks)
        const int first = int(tblock.size()) - (s.local ? 0 : B.tma_blocks_local);
        for (int p = 0; p < 2; ++p) {   // launch_tma's arguments for input set p
            float* e_out = p ? s.e : s.e2;
            float* h_out = p ? s.h : s.h2;
            float* psi_h_out = p ? s.psi : s.psi_h2;
            G.a[p] = TmaArgs{s.geom, s.classes, e_out, h_out, s.sc.k_mu, s.clean_lo[2], s.clean_hi[1], s.clean_hi[2],
                             s.tma_blocks, s.tma_own, -first, 0, s.psi, psi_h_out, s.tables, s.counter, s.error,
                             s.wait_ns, -0.0f, s.stall_plane};
        }
        // blocks index the merged grids (tg), not the batch's grids: some of those march on their own
        const int gi = int(tg.size());
        tg.push_back(G);
        for (int q = 0; q < t.blocks; ++q) tblock.push_back(gi);
        const unsigned rows = s.shell.ra + s.shell.rb + s.shell.rc;
        if (rows) {
            ShellGrid S{};
            S.g = s.geom;
            S.b = s.shell;
            S.kx = s.kax;
            S.node_class = s.node_class;
            S.classes = s.classes;
            for (int p = 0; p < 2; ++p) {
                S.e_in[p] = p ? s.e2 : s.e;
                S.h_in[p] = p ? s.h2 : s.h;
                S.e_out[p] = p ? s.e : s.e2;
                S.h_out[p] = p ? s.h : s.h2;
                S.psi_h_in[p] = p ? s.psi_h2 : s.psi;
                S.psi_h_out[p] = p ? s.psi : s.psi_h2;
            }
            S.psi = s.psi;
            S.k_mu = s.sc.k_mu;
            S.block0 = int(sblock.size());
            const unsigned nb = (rows + SHELL_THREADS / 32 - 1) / (SHELL_THREADS / 32);
            for (unsigned q = 0; q < nb; ++q) sblock.push_back(int(sg.size()));
            sg.push_back(S);
        }
    }
    // every block's grid and its index in that grid's block list, checked before any launch
    for (size_t q = 0; q < tblock.size(); ++q) {
        const int gi = tblock[q];
        const long long launch_q = (long long)q - (q >= size_t(B.tma_blocks_local) ? B.tma_blocks_local : 0);
        const long long local = launch_q + tg[size_t(gi)].a[0].block0;
        const Session* owner = nullptr;
        for (Session* x : B.s)
            if (x->tma_blocks == tg[size_t(gi)].a[0].blocks) owner = x;
        if (gi < 0 || size_t(gi) >= tg.size() || !owner || local < 0 || local >= owner->tma.blocks ||
            tg[size_t(gi)].a[0].block0 != tg[size_t(gi)].a[1].block0) {
            err = "internal: a merged march block outside its grid's block list";
            return FG_ERR_INVALID;
        }
    }
    for (size_t q = 0; q < sblock.size(); ++q) {
        const int gi = sblock[q];
        const ShellGrid& S = sg[size_t(gi)];
        const long long rows = (long long)(q - size_t(S.block0)) * (SHELL_THREADS / 32);
        if (gi < 0 || size_t(gi) >= sg.size() || rows < 0 || rows >= (long long)(S.b.ra + S.b.rb + S.b.rc)) {
            err = "internal: a merged shell block outside its grid's rows";
            return FG_ERR_INVALID;
        }
    }
    cudaError_t ce = cudaSuccess;
    for (bool local : {true, false})
        with_batch_tma(local, B.cid_bytes, [&](auto kern, int smem) {
            if (ce == cudaSuccess) ce = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
        });
    FG_CUDA(ce);
    FG_CUDA(cudaMalloc(&B.d_tma, std::max<size_t>(tg.size(), 1) * sizeof(TmaGrid)));
    FG_CUDA(cudaMalloc(&B.d_tma_block, std::max<size_t>(tblock.size(), 1) * sizeof(int)));
    FG_CUDA(cudaMalloc(&B.d_shell, std::max<size_t>(sg.size(), 1) * sizeof(ShellGrid)));
    FG_CUDA(cudaMalloc(&B.d_shell_block, std::max<size_t>(sblock.size(), 1) * sizeof(int)));
    if (!tg.empty()) {
        FG_CUDA(cudaMemcpy(B.d_tma, tg.data(), tg.size() * sizeof(TmaGrid), cudaMemcpyHostToDevice));
        FG_CUDA(cudaMemcpy(B.d_tma_block, tblock.data(), tblock.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    if (!sg.empty()) {
        FG_CUDA(cudaMemcpy(B.d_shell, sg.data(), sg.size() * sizeof(ShellGrid), cudaMemcpyHostToDevice));
        FG_CUDA(cudaMemcpy(B.d_shell_block, sblock.data(), sblock.size() * sizeof(int), cudaMemcpyHostToDevice));
    }
    B.tma_blocks = int(tblock.size());
    B.shell_blocks = int(sblock.size());
    B.merged_ok = true;
    return FG_OK;
}

template <typename F>
bool with_batch_march(int cid_bytes, int tile, F&& f) {
    auto go = [&](auto cid) {
        using C = decltype(cid);
        switch (tile) {
            case 1: return f(k_batch_march<C, 64, 4>, 64, 4);
            case 2: return f(k_batch_march<C, 32, 4>, 32, 4);
            default: return f(k_batch_march<C, 32, 8>, 32, 8);
        }
    };
    if (cid_bytes == 1) return go(uint8_t{});
    if (cid_bytes == 2) return go(uint16_t{});
    return go(uint32_t{});
}

// Work items of every grid for a shape; uploads the per-grid tiling and the prefix sums.
int batch_apply_shape(Batch& B, const BatchShape& sh, std::string& err) {
    for (Session* s : B.s) {
        s->direct = sh.tile == BATCH_BRANCHES_DIRECT && (sh.seg <= 0 || s->geom.nn < 1000LL * sh.seg);
        // the other grids fill the GPU: long x-segments, few halo planes
        if (s->direct) s->shape.seg = 64;
    }
    for (size_t b = 0; b < B.inst.size(); ++b) B.inst[b].opens = 1;
    if (sh.tile == BATCH_MERGED) {
        if (!B.merged_ok) { err = "merged batch launches: " + B.merged_why; return FG_ERR_INVALID; }
        for (int b : B.merged_rest) B.inst[size_t(b)].opens = 0;   // their own march opens their step
        FG_CUDA(cudaMemcpy(B.d_inst, B.inst.data(), B.inst.size() * sizeof(BatchInstance), cudaMemcpyHostToDevice));
    }
    if (sh.tile >= BATCH_BRANCHES) {
        B.shape = sh;
        return FG_OK;
    }
    const int TK = BATCH_TILES[sh.tile][0], TJ = BATCH_TILES[sh.tile][1];
    std::vector<long long> items(B.s.size() + 1, 0);
    for (size_t b = 0; b < B.s.size(); ++b) {
        const Geom& g = B.s[b]->geom;
        BatchInstance& in = B.inst[b];
        in.tiles_k = (g.n2 + TK - 1) / TK;
        in.tiles_j = (g.n1 + TJ - 1) / TJ;
        in.seg = std::min(sh.seg, g.n0);
        items[b + 1] = items[b] + (long long)in.tiles_k * in.tiles_j * ((g.n0 + in.seg - 1) / in.seg);
    }
    FG_CUDA(cudaMemcpy(B.d_inst, B.inst.data(), B.inst.size() * sizeof(BatchInstance), cudaMemcpyHostToDevice));
    FG_CUDA(cudaMemcpy(B.d_items, items.data(), items.size() * 8, cudaMemcpyHostToDevice));
    int occ = 0;
    cudaError_t ce = cudaSuccess;
    with_batch_march(B.cid_bytes, sh.tile, [&](auto kern, int tk, int tj) {
        ce = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, tk * tj, 0);
        return true;
    });
    if (ce != cudaSuccess) { err = std::string("cudaOccupancyMaxActiveBlocksPerMultiprocessor: ") + cudaGetErrorString(ce); return FG_ERR_CUDA; }
    int sms = 0;
    FG_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, B.gpu->device));
    const int per_sm = sh.blocks_per_sm > 0 ? std::min(sh.blocks_per_sm, std::max(occ, 1)) : std::max(occ, 1);
    B.persistent_blocks = per_sm * sms;
    B.shape = sh;
    return FG_OK;
}

int batch_enqueue_step(Batch& B, int parity, std::string& err) {
    cudaStream_t st = B.stream;
    const int n = int(B.s.size());
    if (B.shape.tile >= BATCH_BRANCHES && B.shape.tile != BATCH_MERGED) {
        // fork every grid's stream from the batch stream, step it there, join back
        FG_CUDA(cudaEventRecord(B.fork, st));
        for (int b = 0; b < n; ++b) {
            Session& S = *B.s[size_t(b)];
            FG_CUDA(cudaStreamWaitEvent(S.stream, B.fork, 0));
            const int rc = enqueue_step(S, parity, err);
            if (rc) return rc;
            FG_CUDA(cudaEventRecord(B.join[size_t(b)], S.stream));
            FG_CUDA(cudaStreamWaitEvent(st, B.join[size_t(b)], 0));
        }
        return FG_OK;
    }
    k_batch_begin<<<(n + 127) / 128, 128, 0, st>>>(B.d_inst, n, B.d_queue);
    if (B.shape.tile == BATCH_MERGED) {
        // every grid's march (its input set `parity`), then every grid's shell H and E; the grids
        // left out march on their own
        const int nl = B.tma_blocks_local, ng = B.tma_blocks - B.tma_blocks_local;
        if (nl > 0)
            with_batch_tma(true, B.cid_bytes, [&](auto kern, int smem) {
                kern<<<unsigned(nl), TMA_CONSUMERS + 32, smem, st>>>(B.d_tma, B.d_tma_block, parity);
            });
        if (ng > 0)   // the second launch's blocks start at block nl of the list: offset the index
            with_batch_tma(false, B.cid_bytes, [&](auto kern, int smem) {
                kern<<<unsigned(ng), TMA_CONSUMERS + 32, smem, st>>>(B.d_tma, B.d_tma_block + nl, parity);
            });
        for (int b : B.merged_rest) {
            Session& S = *B.s[size_t(b)];
            float *e_in = parity ? S.e2 : S.e, *h_in = parity ? S.h2 : S.h;
            float *e_out = parity ? S.e : S.e2, *h_out = parity ? S.h : S.h2;
            if (launch_fused(S.shape, S.cid_bytes, S.geom, S.node_class, S.classes, e_in, h_in, e_out, h_out, S.psi,
                             parity ? S.psi_h2 : S.psi, parity ? S.psi : S.psi_h2, S.sc.k_mu, S.counter, false, st)) {
                err = "fused step launch failed";
                return FG_ERR_CUDA;
            }
        }
        if (B.shell_blocks > 0) {
            k_batch_shell_h<<<unsigned(B.shell_blocks), SHELL_THREADS, 0, st>>>(B.d_shell, B.d_shell_block, parity);
            switch (B.cid_bytes) {
                case 1: k_batch_shell_e<uint8_t><<<unsigned(B.shell_blocks), SHELL_THREADS, 0, st>>>(B.d_shell, B.d_shell_block, parity); break;
                case 2: k_batch_shell_e<uint16_t><<<unsigned(B.shell_blocks), SHELL_THREADS, 0, st>>>(B.d_shell, B.d_shell_block, parity); break;
                default: k_batch_shell_e<uint32_t><<<unsigned(B.shell_blocks), SHELL_THREADS, 0, st>>>(B.d_shell, B.d_shell_block, parity); break;
            }
        }
    } else {
        with_batch_march(B.cid_bytes, B.shape.tile, [&](auto kern, int tk, int tj) {
            kern<<<B.persistent_blocks, dim3(tk, tj), 0, st>>>(B.d_inst, B.d_items, n, B.d_queue, parity);
            return true;
        });
    }
    if (B.total_edges > 0) {
        const unsigned blocks = unsigned((B.total_edges + 255) / 256);
        switch (B.cid_bytes) {
            case 1: k_batch_debye<uint8_t><<<blocks, 256, 0, st>>>(B.d_inst, B.d_edges, n, parity); break;
            case 2: k_batch_debye<uint16_t><<<blocks, 256, 0, st>>>(B.d_inst, B.d_edges, n, parity); break;
            default: k_batch_debye<uint32_t><<<blocks, 256, 0, st>>>(B.d_inst, B.d_edges, n, parity); break;
        }
    }
    k_batch_lumped<<<n, 256, 0, st>>>(B.d_inst, parity);
    if (B.total_ports > 0) k_batch_probe<<<unsigned(B.total_ports), 256, 0, st>>>(B.d_inst, B.d_ports, n, parity);
    const cudaError_t ce = cudaPeekAtLastError();
    if (ce != cudaSuccess) { err = std::string("batched step launch: ") + cudaGetErrorString(ce); return FG_ERR_CUDA; }
    return FG_OK;
}

void batch_free(Batch* B) {
    if (!B) return;
    if (B->gpu) cudaSetDevice(B->gpu->device);
    if (B->stream) cudaStreamSynchronize(B->stream);
    if (B->graph_many) cudaGraphExecDestroy(B->graph_many);
    for (auto& gx : B->graph_one)
        if (gx) cudaGraphExecDestroy(gx);
    cudaFree(B->d_inst);
    cudaFree(B->d_items);
    cudaFree(B->d_edges);
    cudaFree(B->d_ports);
    cudaFree(B->d_queue);
    cudaFree(B->d_tma);
    cudaFree(B->d_tma_block);
    cudaFree(B->d_shell);
    cudaFree(B->d_shell_block);
    for (Session* s : B->s) session_free(s);
    if (B->fork) cudaEventDestroy(B->fork);
    for (cudaEvent_t e : B->join) cudaEventDestroy(e);
    if (B->stream) cudaStreamDestroy(B->stream);
    delete B;
}

int batch_capture(Batch& B, int steps, int parity0, cudaGraphExec_t* out, std::string& err) {
    cudaGraph_t graph;
    FG_CUDA(cudaStreamBeginCapture(B.stream, cudaStreamCaptureModeThreadLocal));
    int rc = FG_OK;
    if (B.shape.tile >= BATCH_BRANCHES && B.shape.tile != BATCH_MERGED) {
        // the grids are independent: each branch runs all the graph's steps, one join at the end
        FG_CUDA(cudaEventRecord(B.fork, B.stream));
        for (size_t b = 0; b < B.s.size() && rc == FG_OK; ++b) {
            Session& S = *B.s[b];
            FG_CUDA(cudaStreamWaitEvent(S.stream, B.fork, 0));
            S.capturing = S.shell_st != nullptr;   // the grid's shell H update beside its march
            for (int q = 0; q < steps && rc == FG_OK; ++q) rc = enqueue_step(S, (parity0 + q) & 1, err);
            S.capturing = false;
            FG_CUDA(cudaEventRecord(B.join[b], S.stream));
            FG_CUDA(cudaStreamWaitEvent(B.stream, B.join[b], 0));
        }
    }
    for (int q = 0; q < steps && rc == FG_OK && (B.shape.tile < BATCH_BRANCHES || B.shape.tile == BATCH_MERGED); ++q)
        rc = batch_enqueue_step(B, (parity0 + q) & 1, err);
    cudaError_t ce = cudaStreamEndCapture(B.stream, &graph);
    if (rc) return rc;
    if (ce != cudaSuccess) { err = std::string("cudaStreamEndCapture: ") + cudaGetErrorString(ce); return FG_ERR_CUDA; }
    ce = cudaGraphInstantiate(out, graph, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(graph);
    if (ce != cudaSuccess) { err = std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ce); return FG_ERR_CUDA; }
    return FG_OK;
}

int batch_reset(Batch& B, std::string& err) {
    for (Session* s : B.s) {
        const int rc = session_reset(s, err);
        if (rc) return rc;
    }
    B.steps = 0;
    return FG_OK;
}

int batch_step(Batch& B, uint64_t k, std::string& err) {
    FG_CUDA(cudaSetDevice(B.gpu->device));
    uint64_t done = 0;
    while (done < k) {
        const int parity = int(B.steps & 1);
        if (parity == 0 && k - done >= uint64_t(B.graph_steps) && B.graph_many) {
            FG_CUDA(cudaGraphLaunch(B.graph_many, B.stream));
            done += B.graph_steps;
            B.steps += B.graph_steps;
        } else {
            FG_CUDA(cudaGraphLaunch(B.graph_one[parity], B.stream));
            done += 1;
            B.steps += 1;
        }
    }
    for (Session* s : B.s) s->steps = B.steps;   // for session_read's choice of the latest buffers
    FG_CUDA(cudaGetLastError());
    return FG_OK;
}

// opt: a fixed shape (tune = false) or the tuner's candidates (tune = true).
int batch_new(Gpu* gpu, const std::vector<const HostSim*>& sims, const std::vector<RunSpec>& specs, bool tune,
              const BatchShape& fixed, int graph_steps, Batch** out, std::string& err) {
    *out = nullptr;
    if (!gpu) { err = "no GPU: this engine has no CPU path"; return FG_ERR_NO_DEVICE; }
    if (sims.empty() || sims.size() != specs.size()) { err = "a batch needs one run spec per grid"; return FG_ERR_INVALID; }
    FG_CUDA(cudaSetDevice(gpu->device));
    auto B = std::unique_ptr<Batch, void (*)(Batch*)>(new Batch, batch_free);
    B->gpu = gpu;
    FG_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking));
    // one class-id width for all grids
    int cid = 1;
    for (const HostSim* h : sims) cid = std::max(cid, h->classes.size() <= 256 ? 1 : (h->classes.size() <= 65536 ? 2 : 4));
    B->cid_bytes = cid;
    for (size_t b = 0; b < sims.size(); ++b) {
        const HostSim& h = *sims[b];
        if (!h.wires.empty() || !h.sheets.empty()) { err = "grid " + std::to_string(b) + ": a batch takes no thin wires or resistive sheets"; return FG_ERR_INVALID; }
        RunSpec rs = specs[b];
        if (rs.has_plane_k || rs.has_ntff) { err = "grid " + std::to_string(b) + ": a batch records no plane DFT or NTFF"; return FG_ERR_INVALID; }
        rs.fused = true;
        rs.graphs = false;
        rs.cid_bytes = cid;
        rs.tma_seg = 64;   // the other grids fill the GPU: long segments, few halo planes
        Session* s = nullptr;
        const int rc = session_new(gpu, h, rs, &s, err);
        if (rc) { err = "grid " + std::to_string(b) + ": " + err; return rc; }
        B->s.push_back(s);
    }
    // descriptors
    std::vector<long long> edges(sims.size() + 1, 0), ports(sims.size() + 1, 0);
    for (size_t b = 0; b < B->s.size(); ++b) {
        Session& s = *B->s[b];
        BatchInstance in{};
        in.a[0] = FusedArgs{s.geom, s.node_class, s.classes, s.e, s.h, s.e2, s.h2, s.psi, s.psi, s.psi_h2, s.sc.k_mu, s.counter};
        in.a[1] = FusedArgs{s.geom, s.node_class, s.classes, s.e2, s.h2, s.e, s.h, s.psi, s.psi_h2, s.psi, s.sc.k_mu, s.counter};
        in.debye_f = s.debye_f;
        in.debye_dd = s.debye_dd;
        in.n_debye = s.n_debye;
        in.debye_table = s.debye_table;
        in.debye_state = s.debye_state;
        in.src = s.sources;
        in.ns = s.n_sources;
        in.ind = s.inductors;
        in.ni = s.n_inductors;
        in.sc = s.sc;
        in.counter = s.counter;
        in.probes = s.probes;
        in.pe = s.port_edges;
        in.lp = s.loops;
        in.n_ports = s.n_ports;
        in.series = s.series;
        in.e[0] = s.e; in.e[1] = s.e2;
        in.h[0] = s.h; in.h[1] = s.h2;
        in.opens = 1;
        B->inst.push_back(in);
        edges[b + 1] = edges[b] + s.n_debye;
        ports[b + 1] = ports[b] + s.n_ports;
    }
    B->total_edges = edges.back();
    B->total_ports = ports.back();
    const size_t n = B->s.size();
    FG_CUDA(cudaMalloc(&B->d_inst, n * sizeof(BatchInstance)));
    FG_CUDA(cudaMalloc(&B->d_items, (n + 1) * 8));
    FG_CUDA(cudaMalloc(&B->d_edges, (n + 1) * 8));
    FG_CUDA(cudaMalloc(&B->d_ports, (n + 1) * 8));
    FG_CUDA(cudaMalloc(&B->d_queue, 8));
    FG_CUDA(cudaEventCreateWithFlags(&B->fork, cudaEventDisableTiming));
    B->join.assign(n, nullptr);
    for (auto& e : B->join) FG_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    FG_CUDA(cudaMemcpy(B->d_edges, edges.data(), (n + 1) * 8, cudaMemcpyHostToDevice));
    FG_CUDA(cudaMemcpy(B->d_ports, ports.data(), (n + 1) * 8, cudaMemcpyHostToDevice));
    int rc = batch_merged_setup(*B, err);
    if (rc) return rc;
    // the tuner: each candidate runs a warm-up step then a timed block of steps from the live state
    BatchShape best = fixed;
    if (tune) {
        cudaEvent_t e0, e1;
        FG_CUDA(cudaEventCreate(&e0));
        FG_CUDA(cudaEventCreate(&e1));
        double best_ms = 1e300;
        const int timed = 4;
        std::vector<BatchShape> cands;
        for (int tile = 0; tile < 3; ++tile)
            for (int seg : {16, 32, 64})
                for (int bps : {0, 2}) cands.push_back(BatchShape{tile, bps, seg});
        cands.push_back(BatchShape{BATCH_BRANCHES, 0, 0});
        if (B->merged_ok) cands.push_back(BatchShape{BATCH_MERGED, 0, 0});
        for (int below : {0, 300, 1000}) cands.push_back(BatchShape{BATCH_BRANCHES_DIRECT, 0, below});
        for (const BatchShape& sh : cands) {
            if ((rc = batch_apply_shape(*B, sh, err))) break;
            // each candidate is timed as captured graphs of `timed` steps (launch costs included)
            cudaGraphExec_t gx = nullptr;
            if ((rc = batch_capture(*B, timed, 0, &gx, err))) break;
            FG_CUDA(cudaGraphLaunch(gx, B->stream));   // warm-up
            FG_CUDA(cudaEventRecord(e0, B->stream));
            FG_CUDA(cudaGraphLaunch(gx, B->stream));
            FG_CUDA(cudaEventRecord(e1, B->stream));
            FG_CUDA(cudaEventSynchronize(e1));
            cudaGraphExecDestroy(gx);
            float ms = 0;
            FG_CUDA(cudaEventElapsedTime(&ms, e0, e1));
            B->trials.push_back({sh, ms / timed});
            if (ms / timed < best_ms) { best_ms = ms / timed; best = sh; }
        }
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        if (rc) return rc;
        B->tuned_ms = best_ms;
        if (const char* v = std::getenv("FIELDGRID_BATCH_TRIALS"); v && v[0] == '1') {
            std::fprintf(stderr, "batch tuner: %zu grids, %zu march on their own in the merged mode\n", B->s.size(),
                         B->merged_rest.size());
            for (auto& [sh, ms] : B->trials)
                std::fprintf(stderr, "  tile %d blocks/SM %d seg %d: %.3f ms per step\n", sh.tile, sh.blocks_per_sm,
                             sh.seg, ms);
        }
        if ((rc = batch_reset(*B, err))) return rc;
    }
    if ((rc = batch_apply_shape(*B, best, err))) return rc;
    B->graph_steps = std::max(2, graph_steps + (graph_steps & 1));
    if ((rc = batch_capture(*B, B->graph_steps, 0, &B->graph_many, err))) return rc;
    if ((rc = batch_capture(*B, 1, 0, &B->graph_one[0], err))) return rc;
    if ((rc = batch_capture(*B, 1, 1, &B->graph_one[1], err))) return rc;
    *out = B.release();
    return FG_OK;
}

int batch_new_c(Gpu* gpu, const std::vector<const HostSim*>& sims, const std::vector<RunSpec>& specs, bool tune,
                int tile, int blocks_per_sm, int seg, int graph_steps, Batch** out, std::string& err) {
    BatchShape sh;
    sh.tile = std::min(std::max(tile, 0), BATCH_MERGED);
    sh.blocks_per_sm = std::max(blocks_per_sm, 0);
    sh.seg = seg > 0 ? seg : 32;
    return batch_new(gpu, sims, specs, tune, sh, graph_steps > 0 ? graph_steps : 10, out, err);
}

int batch_sync(Batch& B, std::string& err) {
    FG_CUDA(cudaSetDevice(B.gpu->device));
    FG_CUDA(cudaStreamSynchronize(B.stream));
    return FG_OK;
}

int batch_read(Batch& B, uint64_t index, const std::string& which, float* dst, uint64_t len, std::string& err) {
    if (index >= B.s.size()) { err = "no grid " + std::to_string(index) + " in this batch"; return FG_ERR_INVALID; }
    const int rc = batch_sync(B, err);
    if (rc) return rc;
    return session_read(B.s[index], which, dst, len, err);
}

void batch_info(const Batch& B, int* tile, int* blocks_per_sm, int* seg, int* persistent_blocks, double* tuned_ms,
                uint64_t* steps) {
    if (tile) *tile = B.shape.tile;
    if (blocks_per_sm) *blocks_per_sm = B.shape.blocks_per_sm;
    if (seg) *seg = B.shape.seg;
    if (persistent_blocks) *persistent_blocks = B.persistent_blocks;
    if (tuned_ms) *tuned_ms = B.tuned_ms;
    if (steps) *steps = B.steps;
}

uint64_t batch_size(const Batch& B) { return B.s.size(); }

}  // namespace fg
