// Far field of the NTFF box on the device: Far::field (sims-field ntff.rs:90-116) for many
// directions at once. One block per direction sums the patch currents with their phase
// e^{j k r.r'} in f64 (the host transform's precision); the patch table (positions, areas and the
// 12 current doubles per patch) is read by every block and stays in L2.
#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "../../include/fieldgrid.h"
#include "engine.hpp"

namespace fg {

namespace {

constexpr int FAR_THREADS = 256;

__global__ void __launch_bounds__(FAR_THREADS) k_far_field(const double* __restrict__ pos, const double* __restrict__ area,
                                                           const double* __restrict__ jm, long long count, double kw,
                                                           const double* __restrict__ dirs, double* __restrict__ out) {
    __shared__ double red[12][FAR_THREADS / 32];
    const double* dir = dirs + 3 * (long long)blockIdx.x;
    const double d0 = dir[0], d1 = dir[1], d2 = dir[2];
    double acc[12];
#pragma unroll
    for (int q = 0; q < 12; ++q) acc[q] = 0.0;
    for (long long i = threadIdx.x; i < count; i += blockDim.x) {
        const double* p = pos + 3 * i;
        const double arg = kw * (d0 * p[0] + d1 * p[1] + d2 * p[2]);
        double s, c;
        sincos(arg, &s, &c);
        const double a = area[i];
        const double ph0 = a * c, ph1 = a * s;
        const double* x = jm + 12 * i;
#pragma unroll
        for (int q = 0; q < 12; q += 2) {
            acc[q] += x[q] * ph0 - x[q + 1] * ph1;
            acc[q + 1] += x[q] * ph1 + x[q + 1] * ph0;
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int q = 0; q < 12; ++q) {
        double v = acc[q];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
        if (lane == 0) red[q][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double nn[3][2], ll[3][2];
        for (int q = 0; q < 12; ++q) {
            double v = 0.0;
            for (int w = 0; w < FAR_THREADS / 32; ++w) v += red[q][w];
            if (q < 6) nn[q / 2][q % 2] = v;
            else ll[(q - 6) / 2][q % 2] = v;
        }
        const double d[3] = {d0, d1, d2};
        double rn0 = 0, rn1 = 0;
        for (int c = 0; c < 3; ++c) { rn0 += nn[c][0] * d[c]; rn1 += nn[c][1] * d[c]; }
        const double eta0 = 376.730313668;
        const double scale = kw / (4.0 * 3.14159265358979323846);
        const double rl[3][2] = {{d[1] * ll[2][0] - d[2] * ll[1][0], d[1] * ll[2][1] - d[2] * ll[1][1]},
                                 {d[2] * ll[0][0] - d[0] * ll[2][0], d[2] * ll[0][1] - d[0] * ll[2][1]},
                                 {d[0] * ll[1][0] - d[1] * ll[0][0], d[0] * ll[1][1] - d[1] * ll[0][1]}};
        double* o = out + 6 * (long long)blockIdx.x;
        for (int c = 0; c < 3; ++c) {
            const double p0 = nn[c][0] - rn0 * d[c], p1 = nn[c][1] - rn1 * d[c];
            o[2 * c] = (rl[c][0] - p0 * eta0) * scale;
            o[2 * c + 1] = (rl[c][1] - p1 * eta0) * scale;
        }
    }
}

}  // namespace

int far_field_gpu(Gpu* g, const double* pos, const double* area, const double* jm, uint64_t count, double freq,
                  const double* dirs, uint64_t n, double* out, std::string& err) {
    if (n == 0) return FG_OK;
    auto check = [&](cudaError_t e, const char* what) {
        if (e != cudaSuccess) { err = std::string(what) + ": " + cudaGetErrorString(e); return false; }
        return true;
    };
    if (!check(cudaSetDevice(g->device), "cudaSetDevice")) return FG_ERR_CUDA;
    const size_t bytes = (5 * count + 12 * count + 3 * n + 6 * n) * sizeof(double) + 1024;
    char* buf = nullptr;
    if (!check(cudaMalloc(&buf, bytes), "cudaMalloc")) return FG_ERR_CUDA;
    double* d_pos = reinterpret_cast<double*>(buf);
    double* d_area = d_pos + 3 * count;
    double* d_jm = d_area + count;
    double* d_dirs = d_jm + 12 * count;
    double* d_out = d_dirs + 3 * n;
    bool ok = check(cudaMemcpy(d_pos, pos, 3 * count * 8, cudaMemcpyHostToDevice), "cudaMemcpy") &&
              check(cudaMemcpy(d_area, area, count * 8, cudaMemcpyHostToDevice), "cudaMemcpy") &&
              check(cudaMemcpy(d_jm, jm, 12 * count * 8, cudaMemcpyHostToDevice), "cudaMemcpy") &&
              check(cudaMemcpy(d_dirs, dirs, 3 * n * 8, cudaMemcpyHostToDevice), "cudaMemcpy");
    if (ok) {
        const double kw = 2.0 * 3.14159265358979323846 * freq / 299792458.0;
        for (uint64_t first = 0; first < n && ok; first += 65535) {
            const uint64_t m = std::min<uint64_t>(65535, n - first);
            k_far_field<<<unsigned(m), FAR_THREADS>>>(d_pos, d_area, d_jm, (long long)count, kw, d_dirs + 3 * first,
                                                       d_out + 6 * first);
            ok = check(cudaGetLastError(), "k_far_field");
        }
        ok = ok && check(cudaMemcpy(out, d_out, 6 * n * 8, cudaMemcpyDeviceToHost), "cudaMemcpy");
    }
    cudaFree(buf);
    return ok ? FG_OK : FG_ERR_CUDA;
}

}  // namespace fg
