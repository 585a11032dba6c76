// The field energy of caller-owned device arrays without any device allocation.
//
// Some callers cannot allocate device memory at the point where they need this number: a host
// framework's operator callback that runs while the framework's own caching allocator owns the
// device memory, or a loop that must not take the implicit device-wide synchronisation that
// cudaMalloc/cudaFree bring. fg_energy_noalloc serves them: its per-block partial sums live in the
// file-scope array below, which exists once per device for the lifetime of the process.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/fieldgrid.h"

namespace fg {
void set_last_error(const std::string& msg);
}

// Scratch: one f64 partial per block of the first pass. 4096 x 8 B = 32 KB per device.
static __device__ __align__(256) double g_energy_partials[FG_ENERGY_NOALLOC_MAX_BLOCKS];

namespace {

constexpr int NOALLOC_THREADS = 256;
constexpr unsigned long long MIN_CHUNK = 2048;   // elements per block at least

// First pass: block b sums E^2 + (376.73 H)^2 over elements [b*chunk, min((b+1)*chunk, n)) of
// both arrays into g_energy_partials[b] (every slot the second pass reads is written here first,
// so nothing has to be cleared between calls).
__global__ void k_energy_partials(const float* __restrict__ e, const float* __restrict__ h, unsigned long long n,
                                  unsigned long long chunk, double* partials) {
    __shared__ double red[NOALLOC_THREADS];
    const unsigned long long lo = (unsigned long long)blockIdx.x * chunk;
    const unsigned long long hi = lo + chunk < n ? lo + chunk : n;
    double acc = 0.0;
    for (unsigned long long q = lo + threadIdx.x; q < hi; q += blockDim.x) {
        const double x = double(e[q]);
        const double y = double(h[q]) * 376.73;
        acc += x * x + y * y;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partials[blockIdx.x] = red[0];
}

// Second pass: one block adds the `blocks` partials into *out.
__global__ void k_energy_total(const double* partials, int blocks, double* out) {
    __shared__ double red[NOALLOC_THREADS];
    double acc = 0.0;
    for (int q = threadIdx.x; q < blocks; q += blockDim.x) acc += partials[q];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = red[0];
}

// The device address of g_energy_partials, looked up once per device. In host code the name
// g_energy_partials is only a host-side stand-in, never a device address.
constexpr int MAX_DEVICES = 64;
std::mutex g_lock;
double* g_scratch[MAX_DEVICES] = {};

int scratch_of(int device, double** out, std::string& err) {
    std::lock_guard<std::mutex> lk(g_lock);
    if (device < 0 || device >= MAX_DEVICES) {
        err = "device index out of range";
        return FG_ERR_INVALID;
    }
    if (!g_scratch[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_energy_partials);
        if (e != cudaSuccess) {
            err = std::string("cudaGetSymbolAddress(g_energy_partials): ") + cudaGetErrorString(e);
            return FG_ERR_CUDA;
        }
        g_scratch[device] = static_cast<double*>(p);
    }
    *out = g_scratch[device];
    return FG_OK;
}

}  // namespace

extern "C" int fg_energy_noalloc(const float* e, const float* h, uint64_t n, double* out, void* stream) {
    if (!out || (n > 0 && (!e || !h))) {   // an empty array may come as a null pointer
        fg::set_last_error("fg_energy_noalloc: null pointer");
        return FG_ERR_INVALID;
    }
    const unsigned long long limit = (unsigned long long)FG_ENERGY_NOALLOC_MAX_BLOCKS * FG_ENERGY_NOALLOC_CHUNK;
    if (n > limit) {
        fg::set_last_error("fg_energy_noalloc: " + std::to_string(n) + " elements exceed the maximum of " +
                           std::to_string(limit) + " this entry point's fixed scratch covers");
        return FG_ERR_INVALID;
    }
    // Elements per block, chosen per call so that small and large arrays both spread over the
    // GPU: n split over at most FG_ENERGY_NOALLOC_MAX_BLOCKS blocks, at least MIN_CHUNK elements
    // each, a multiple of the block size. At the limit this is FG_ENERGY_NOALLOC_CHUNK.
    unsigned long long chunk = (n + FG_ENERGY_NOALLOC_MAX_BLOCKS - 1) / FG_ENERGY_NOALLOC_MAX_BLOCKS;
    if (chunk < MIN_CHUNK) chunk = MIN_CHUNK;
    chunk = (chunk + NOALLOC_THREADS - 1) / NOALLOC_THREADS * NOALLOC_THREADS;
    const unsigned long long blocks = (n + chunk - 1) / chunk;
    int device = 0;
    cudaError_t ce = cudaGetDevice(&device);
    if (ce != cudaSuccess) {
        fg::set_last_error(std::string("cudaGetDevice: ") + cudaGetErrorString(ce));
        return FG_ERR_NO_DEVICE;
    }
    double* partials = nullptr;
    std::string err;
    int rc = scratch_of(device, &partials, err);
    if (rc) {
        fg::set_last_error(err);
        return rc;
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (blocks > 0)
        k_energy_partials<<<unsigned(blocks), NOALLOC_THREADS, 0, st>>>(e, h, n, chunk, partials);
    k_energy_total<<<1, NOALLOC_THREADS, 0, st>>>(partials, int(blocks), out);
    ce = cudaGetLastError();
    if (ce != cudaSuccess) {
        fg::set_last_error(std::string("fg_energy_noalloc launch: ") + cudaGetErrorString(ce));
        return FG_ERR_CUDA;
    }
    return FG_OK;
}
