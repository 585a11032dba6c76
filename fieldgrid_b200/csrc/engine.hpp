// Internal interface between the C ABI (capi.cpp) and the CUDA engine (engine.cu).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

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
};

struct Session;

struct Gpu {
    int device = 0;
    std::string name;
};

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

}  // namespace fg
