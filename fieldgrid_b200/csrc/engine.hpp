// Internal interface between the C ABI (capi.cpp) and the CUDA engine (engine.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include <vector_types.h>

#include "host.hpp"

namespace fg {

struct RunSpec {               // pack() inputs that are not part of the Sim (run.rs:205-210)
    uint64_t driven = 0;
    double f0 = 0, fc = 0;
    uint64_t max_steps = 0;
    std::vector<double> freqs;  // first 4 used
    bool has_plane_k = false;
    uint64_t plane_k = 0;
    bool has_ntff = false;
    std::vector<uint32_t> ntff;
    bool fused = true;          // the fused E+H march; false = the separate H and E kernels
    bool profile = false;
    // adjoint support: E edges (comp, i, j, k) whose E^n and curl term every fused step records
    // into a ring of hist_cap slots (slot = step - base)
    const std::vector<int4>* design = nullptr;
    int hist_cap = 0;
    bool design_in_steps = true;   // false: only quiet re-runs (the adjoint's) record the design history
    // batched use: the direct-load march only, no captured graphs, and a class-id width of at
    // least cid_bytes (so instances share one kernel instantiation)
    bool tma = true;
    bool graphs = true;
    int cid_bytes = 0;
    int tma_seg = 0;            // x-planes per march block; 0: enough blocks to fill the GPU alone
};

struct Session;

struct Gpu {
    int device = 0;
    std::string name;
    // pinned staging for host-to-device uploads (allocated on the first large upload): a copy goes
    // through the two buffers in turn, so filling one overlaps the transfer of the other
    void* stage[2] = {nullptr, nullptr};
    void* stage_ev[2] = {nullptr, nullptr};   // cudaEvent_t: the last transfer out of each buffer
    // the arena of the last session freed on this device, kept for the next session of a similar
    // size (runs of one grid after another skip the allocation and its release)
    void* spare = nullptr;
    size_t spare_bytes = 0;
};

// Copies `bytes` from pageable host memory to the device through the Gpu's pinned staging buffers
// (OpenMP copies into them, the transfers overlap the next copy); on return the source may be
// reused. Small copies go straight. Returns a cudaError_t as int.
int staged_upload(Gpu* g, void* dst, const void* src, size_t bytes, void* stream);

// mesh -> grid rasterisation (raster.cu)
int raster_fill(Gpu* gpu, const double* tris, uint64_t ntri, const std::vector<double>* samples, const size_t* dims,
                int order, uint8_t* inside, uint8_t* thin, std::string& err);
int raster_sheet_edges(Gpu* gpu, const double* tris, uint64_t ntri, const std::vector<double>* lines, uint8_t* mask,
                       std::string& err);
bool raster_closed(const double* tris, uint64_t ntri);

int gpu_open(int device, Gpu** out, std::string& err);
void gpu_close(Gpu* g);

int session_new(Gpu* g, const HostSim& sim, const RunSpec& rs, Session** out, std::string& err);
void session_free(Session* s);
int session_step(Session* s, uint64_t k, std::string& err);
int session_sync(Session* s, std::string& err);
int session_energy(Session* s, double* out, std::string& err);
uint64_t session_steps(const Session* s);
int session_read(Session* s, const std::string& which, float* dst, uint64_t len, std::string& err);
void* session_stream(Session* s);
uint64_t session_launches_per_step(const Session* s);
uint64_t session_device_bytes(const Session* s);
const char* session_variant(const Session* s);
uint64_t session_ports(const Session* s);
uint64_t session_plane_len(const Session* s);
uint64_t session_ntff_len(const Session* s);
double session_t0(const Session* s);
void session_profile(Session* s);
int session_kernel_times(Session* s, uint64_t steps, std::vector<std::pair<std::string, double>>& out, std::string& err);
uint64_t session_h2d_bytes(const Session* s);
uint64_t session_d2h_bytes(const Session* s);

// Far field on the device: fields for n directions (6 doubles each).
int far_field_gpu(Gpu* g, const double* pos, const double* area, const double* jm, uint64_t count, double freq,
                  const double* dirs, uint64_t n, double* out, std::string& err);

int sim_try_new(const struct fg_sim_spec* spec, HostSim** out, std::string& err);

// The flux objective J = |F|^2 on a z-plane window at one frequency and, when want_grad, its
// gradient over the permittivity and conductivity of a design box of voxels (adjoint.cuh).
struct FluxSpec {
    uint64_t lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};   // design cells [lo, hi)
    uint64_t plane_k = 0;
    uint64_t win_lo[2] = {0, 0}, win_hi[2] = {0, 0};  // (i, j) nodes of the flux sum
    double freq = 0;
    uint64_t steps = 0;
    uint64_t checkpoints = 0;                          // 0: keep every step's design history
    int transposes = 0;     // 0: one fused adjoint step launch per step; 1: the E and H transposes apart
};

struct FluxResult {
    double J = 0, f_re = 0, f_im = 0;
    double forward_ms = 0, recompute_ms = 0, adjoint_ms = 0;
    double backward_ms = 0;             // the whole backward pass (re-runs and sweeps overlap)
    double setup_ms = 0;                // checks, session, checkpoint and adjoint buffers
    uint64_t segments = 0, segment_len = 0, design_edges = 0;
    std::vector<double> g_eps, g_sig;   // per design cell, k fastest
};

// Batches of independent grids stepped by shared launches (batch.cuh).
struct Batch;
struct BatchShape;
int session_reset(Session* s, std::string& err);
int batch_new_c(Gpu* gpu, const std::vector<const HostSim*>& sims, const std::vector<RunSpec>& specs, bool tune,
                int tile, int blocks_per_sm, int seg, int graph_steps, Batch** out, std::string& err);
void batch_free(Batch* b);
int batch_step(Batch& b, uint64_t k, std::string& err);
int batch_sync(Batch& b, std::string& err);
int batch_read(Batch& b, uint64_t index, const std::string& which, float* dst, uint64_t len, std::string& err);
void batch_info(const Batch& b, int* tile, int* blocks_per_sm, int* seg, int* persistent_blocks, double* tuned_ms,
                uint64_t* steps);
uint64_t batch_size(const Batch& b);

int flux_gradient(Gpu* gpu, const HostSim& sim, uint64_t driven, double f0, double fc, const FluxSpec& sp,
                  bool want_grad, FluxResult& res, std::string& err);
// count flux gradients on one GPU, `group` at a time with their phases enqueued together
int flux_gradient_batch(Gpu* gpu, const std::vector<const HostSim*>& sims, const std::vector<uint64_t>& driven,
                        const std::vector<std::pair<double, double>>& pulses, const std::vector<FluxSpec>& specs,
                        int group, std::vector<FluxResult>& out, std::string& err);
// The same objective from an FP64 forward on the device (fp64_forward.cuh).
int flux_objective64(Gpu* gpu, const HostSim& sim, uint64_t driven, double f0, double fc, const FluxSpec& sp,
                     FluxResult& res, std::string& err);

}  // namespace fg
