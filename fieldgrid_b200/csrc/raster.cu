// Mesh -> grid rasterisation on the device: the ray-parity fill of crates/sims-field/src/raster.rs
// (fill :24-104, solid_edges :145-160, solid_cells :162-173, sheet_edges :186-264) over the
// bounding-volume hierarchy of crates/sims-field/src/bvh.rs, and the closed-mesh check (:127-143)
// on the host.
//
// Layout: the triangles (9 f64 each) and the hierarchy's nodes live in HBM; one thread per sample
// column casts the column's ray through the hierarchy (an explicit stack), pairs its crossings and
// marks the samples between each pair (inside) or, for a pair with no sample between, the sample
// nearest its middle (thin); sheet_edges runs one block per triangle over the nodes near it. Every
// mark is a byte store of 1, so the order in which threads mark does not change the masks. The
// arithmetic is the reference's f64 arithmetic in its operation order (the build has no a*b+c
// contraction), so the masks equal the reference's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/fieldgrid.h"
#include "engine.hpp"

namespace fg {
namespace raster {

struct Node {                 // bvh.rs:4-10
    double lo[3], hi[3];
    int start, count;         // the node's range of `order`
    int left, right;          // children (-1: a leaf)
};

constexpr int STACK = 64;                  // traversal stack depth (a hierarchy of median splits
                                           // over 2^31 triangles is 30 levels deep)
constexpr int MAX_CROSSINGS = 1 << 20;     // per column

// Bvh::build (bvh.rs:62-93): median split along the longest axis of the node's box, leaves of at
// most 4 triangles.
struct Builder {
    const double* tri;
    std::vector<int> order;
    std::vector<Node> nodes;
    int depth = 0;

    double centre(int i, int axis) const {
        const double* t = tri + size_t(i) * 9;
        return (t[axis] + t[3 + axis] + t[6 + axis]) / 3.0;
    }
    int build(int start, int end, int level) {
        depth = std::max(depth, level);
        Node n{};
        for (int a = 0; a < 3; ++a) { n.lo[a] = INFINITY; n.hi[a] = -INFINITY; }
        for (int q = start; q < end; ++q)
            for (int p = 0; p < 3; ++p)
                for (int a = 0; a < 3; ++a) {
                    const double v = tri[size_t(order[q]) * 9 + p * 3 + a];
                    n.lo[a] = std::fmin(n.lo[a], v);
                    n.hi[a] = std::fmax(n.hi[a], v);
                }
        n.start = start;
        n.count = end - start;
        n.left = n.right = -1;
        const int index = int(nodes.size());
        nodes.push_back(n);
        if (end - start <= 4) return index;
        const double ex[3] = {n.hi[0] - n.lo[0], n.hi[1] - n.lo[1], n.hi[2] - n.lo[2]};
        const int axis = (ex[0] >= ex[1] && ex[0] >= ex[2]) ? 0 : (ex[1] >= ex[2] ? 1 : 2);
        const int middle = (start + end) / 2;
        std::nth_element(order.begin() + start, order.begin() + middle, order.begin() + end,
                         [&](int a, int b) { return centre(a, axis) < centre(b, axis); });
        const int l = build(start, middle, level + 1);
        const int r = build(middle, end, level + 1);
        nodes[size_t(index)].left = l;
        nodes[size_t(index)].right = r;
        return index;
    }
};

__device__ __forceinline__ void dsub(const double* a, const double* b, double* o) {
    o[0] = a[0] - b[0]; o[1] = a[1] - b[1]; o[2] = a[2] - b[2];
}
__device__ __forceinline__ double ddot(const double* a, const double* b) { return a[0] * b[0] + a[1] * b[1] + a[2] * b[2]; }
__device__ __forceinline__ void dcross(const double* a, const double* b, double* o) {
    o[0] = a[1] * b[2] - a[2] * b[1];
    o[1] = a[2] * b[0] - a[0] * b[2];
    o[2] = a[0] * b[1] - a[1] * b[0];
}

// hit (bvh.rs:156-177): the ray parameter of a triangle crossing, or NaN for none.
__device__ double hit(const double* t, const double* origin, const double* dir) {
    double e1[3], e2[3], p[3], s[3], q[3];
    dsub(t + 3, t, e1);
    dsub(t + 6, t, e2);
    dcross(dir, e2, p);
    const double det = ddot(e1, p);
    if (fabs(det) < 1.0e-18) return NAN;
    const double inv = 1.0 / det;
    dsub(origin, t, s);
    const double u = ddot(s, p) * inv;
    if (!(u >= -1.0e-9 && u <= 1.0 + 1.0e-9)) return NAN;
    dcross(s, e1, q);
    const double v = ddot(dir, q) * inv;
    if (v < -1.0e-9 || u + v > 1.0 + 1.0e-9) return NAN;
    return ddot(e2, q) * inv;
}

// Bvh::slab (bvh.rs:95-110); fmax / fmin pass over NaN as Rust's f64::max / min do.
__device__ __forceinline__ bool slab(const Node& n, const double* o, const double* inv, double limit) {
    double near = 0.0, far = limit;
    for (int k = 0; k < 3; ++k) {
        const double t1 = (n.lo[k] - o[k]) * inv[k];
        const double t2 = (n.hi[k] - o[k]) * inv[k];
        const double a = t1 < t2 ? t1 : t2, b = t1 < t2 ? t2 : t1;
        near = fmax(near, a);
        far = fmin(far, b);
        if (near > far) return false;
    }
    return true;
}

// Bvh::ray (bvh.rs:112-154): the nearest crossing with t > least (INFINITY: none). *bad is set
// when the stack would overflow.
__device__ double ray(const Node* nodes, const int* order, const double* tri, const double* o, const double* dir,
                      double least, bool* bad) {
    double best = INFINITY;
    const double inv[3] = {1.0 / dir[0], 1.0 / dir[1], 1.0 / dir[2]};
    int stack[STACK];
    int top = 0;
    stack[top++] = 0;
    while (top > 0) {
        const Node n = nodes[stack[--top]];
        if (!slab(n, o, inv, best)) continue;
        if (n.left >= 0) {
            if (top + 2 > STACK) { *bad = true; return INFINITY; }
            stack[top++] = n.left;
            stack[top++] = n.right;
        } else {
            for (int q = n.start; q < n.start + n.count; ++q) {
                const double t = hit(tri + size_t(order[q]) * 9, o, dir);
                if (t > least && t < best) best = t;      // NaN compares false
            }
        }
    }
    return best;
}

// slice::partition_point over a sorted line: the first index whose sample fails `below`.
__device__ __forceinline__ int count_below(const double* line, int n, double v, bool or_equal) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const bool in = or_equal ? line[mid] <= v : line[mid] < v;
        if (in) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// grid::nearest (grid.rs:48-55)
__device__ int nearest(const double* line, int n, double v) {
    const int i = count_below(line, n, v, false);
    if (i >= 1 && i < n) {
        if (fabs(v - line[i - 1]) <= fabs(line[i] - v)) return i - 1;
    } else if (i >= 1) {
        return i - 1;
    }
    return min(i, max(n - 1, 0));
}

struct FillAxis {
    const double* line[3];     // the sample lines of the three axes
    int n[3];
    int axis, u, v;
    int us, wide, vs, tall;    // the columns' sample spans along u and v
    double step[3];
    double start;
    double reach0, reach1;
    int order;                 // 0: (i m1 + j) m2 + k, 1: i + (j + k m1) m0
    long long m[3];            // the dimensions of the index space
};

__device__ __forceinline__ size_t index_of(const FillAxis& f, const int* c) {
    if (f.order == 0) return (size_t(c[0]) * f.m[1] + c[1]) * f.m[2] + c[2];
    return size_t(c[0]) + (size_t(c[1]) + size_t(c[2]) * f.m[1]) * f.m[0];
}

// fill's column loop (raster.rs:52-99), one thread per column.
__global__ void k_fill_axis(FillAxis f, const Node* nodes, const int* order, const double* tri, uint8_t* inside,
                            uint8_t* thin, int* error) {
    const long long col = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (col >= (long long)f.wide * f.tall) return;
    int cell[3] = {0, 0, 0};
    cell[f.u] = f.us + int(col % f.wide);
    cell[f.v] = f.vs + int(col / f.wide);
    double from[3], dir[3] = {0.0, 0.0, 0.0};
    from[f.u] = f.line[f.u][cell[f.u]] + f.step[f.u] * 1.234567e-6;
    from[f.v] = f.line[f.v][cell[f.v]] + f.step[f.v] * 2.345678e-6;
    from[f.axis] = f.start;
    dir[f.axis] = 1.0;
    const double* line = f.line[f.axis];
    const int n = f.n[f.axis];
    bool bad = false;
    double last = 0.0, a = 0.0;
    bool open = false;      // a crossing waits for its pair
    auto pair = [&](double pa, double pb) {
        const int first = count_below(line, n, pa, false);
        const int last_n = count_below(line, n, pb, true);   // partition_point(s <= b); last = that - 1
        if (last_n >= 1 && first <= last_n - 1) {
            if (f.axis == 0)
                for (int k = first; k <= last_n - 1; ++k) {
                    int c[3] = {cell[0], cell[1], cell[2]};
                    c[f.axis] = k;
                    inside[index_of(f, c)] = 1;
                }
        } else if (isfinite(pb)) {
            const double middle = 0.5 * (pa + pb);
            if (middle >= f.reach0 && middle < f.reach1) {
                int c[3] = {cell[0], cell[1], cell[2]};
                c[f.axis] = nearest(line, n, middle);
                thin[index_of(f, c)] = 1;
            }
        }
    };
    for (int q = 0; q < MAX_CROSSINGS; ++q) {
        const double t = ray(nodes, order, tri, from, dir, last + f.step[f.axis] * 1.0e-9, &bad);
        if (bad) { atomicExch(error, 1); return; }
        if (!isfinite(t)) break;
        const double x = f.start + t;
        if (open) pair(a, x);
        else a = x;
        open = !open;
        last = t;
        if (q + 1 == MAX_CROSSINGS) { atomicExch(error, 2); return; }
    }
    if (open) pair(a, INFINITY);
}

struct SheetArgs {
    const double* line[3];
    int n[3];
};

__device__ int cell_of(const double* line, int n, double v) {   // grid::cell_of (grid.rs:57-59)
    const int i = max(count_below(line, n, v, true) - 1, 0);
    return min(i, max(n - 2, 0));
}

__device__ double local_size(const double* line, int n, int i, bool centre) {   // raster.rs:175-184
    if (centre) return line[min(i + 1, n - 1)] - line[min(i, n - 2)];
    const double before = i > 0 ? line[i] - line[i - 1] : line[1] - line[0];
    const double after = i + 1 < n ? line[i + 1] - line[i] : line[n - 1] - line[n - 2];
    return 0.5 * (before + after);
}

// sheet_edges (raster.rs:186-264): one block per triangle, its threads over the nodes near it.
__global__ void k_sheet_edges(SheetArgs g, const double* tris, long long ntri, uint8_t* mask) {
    for (long long ti = blockIdx.x; ti < ntri; ti += gridDim.x) {
        const double* t = tris + ti * 9;
        double e0[3], e1[3], normal[3];
        dsub(t + 3, t, e0);
        dsub(t + 6, t, e1);
        dcross(e0, e1, normal);
        const double area2 = sqrt(ddot(normal, normal));
        if (area2 <= 1e-30) continue;
        const double nrm[3] = {normal[0] / area2, normal[1] / area2, normal[2] / area2};
        double lo[3], hi[3];
        const double inf = INFINITY;
        for (int a = 0; a < 3; ++a) {
            lo[a] = fmin(fmin(fmin(inf, t[a]), t[3 + a]), t[6 + a]);
            hi[a] = fmax(fmax(fmax(-inf, t[a]), t[3 + a]), t[6 + a]);
        }
        const double d00 = ddot(e0, e0), d01 = ddot(e0, e1), d11 = ddot(e1, e1);
        const double det = d00 * d11 - d01 * d01;
        const size_t nn = size_t(g.n[0]) * g.n[1] * g.n[2];
        for (int c = 0; c < 3; ++c) {
            if (fabs(nrm[c]) >= 0.75) continue;
            int first[3], count[3];
            for (int a = 0; a < 3; ++a) {
                const double* line = g.line[a];
                const int n = g.n[a];
                const int il = cell_of(line, n, lo[a]), ih = cell_of(line, n, hi[a]);
                const double reach = fmax(line[il + 1] - line[il], line[ih + 1] - line[ih]);
                const int f0 = count_below(line, n, lo[a] - reach, false);
                int l0 = count_below(line, n, hi[a] + reach, true);
                if (a == c) l0 = min(l0, n - 1);
                first[a] = f0;
                count[a] = max(l0 - f0, 0);
            }
            const long long total = (long long)count[0] * count[1] * count[2];
            for (long long q = threadIdx.x; q < total; q += blockDim.x) {
                const int p[3] = {first[0] + int(q / ((long long)count[1] * count[2])),
                                  first[1] + int((q / count[2]) % count[1]), first[2] + int(q % count[2])};
                if (p[c] + 1 >= g.n[c]) continue;
                double mid[3], h[3];
                for (int a = 0; a < 3; ++a) {
                    const double* l = g.line[a];
                    mid[a] = a == c ? 0.5 * (l[p[a]] + l[p[a] + 1]) : l[p[a]];
                    h[a] = local_size(l, g.n[a], p[a], a == c);
                }
                double sum = 0.0;
                for (int a = 0; a < 3; ++a) sum = sum + fabs(nrm[a]) * h[a];
                const double tol = 0.5 * sum;
                double r[3];
                dsub(mid, t, r);
                const double d = ddot(r, nrm);
                const double eps = 1e-9 * tol;
                if (d <= eps - tol || d > tol + eps) continue;
                const double nd[3] = {nrm[0] * d, nrm[1] * d, nrm[2] * d};
                double m1[3], qv[3];
                dsub(mid, nd, m1);
                dsub(m1, t, qv);
                const double q0 = ddot(qv, e0), q1 = ddot(qv, e1);
                const double v = (d11 * q0 - d01 * q1) / det;
                const double w = (d00 * q1 - d01 * q0) / det;
                const double slack = 1e-9;
                if (v >= -slack && w >= -slack && v + w <= 1.0 + slack)
                    mask[size_t(c) * nn + (size_t(p[0]) * g.n[1] + p[1]) * g.n[2] + p[2]] = 1;
            }
        }
    }
}

// spacing (raster.rs:13-15): the smallest positive gap of a line (INFINITY when none).
double spacing(const std::vector<double>& line) {
    double s = INFINITY;
    for (size_t i = 0; i + 1 < line.size(); ++i) {
        const double d = line[i + 1] - line[i];
        if (d > 0.0) s = std::fmin(s, d);
    }
    return s;
}

size_t partition(const std::vector<double>& line, double v, bool or_equal) {
    return size_t(std::partition_point(line.begin(), line.end(),
                                       [&](double x) { return or_equal ? x <= v : x < v; }) - line.begin());
}

}  // namespace raster

#define RS_CUDA(call)                                                                              \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) {                                                                   \
            err = std::string(#call) + ": " + cudaGetErrorString(e_);                              \
            return FG_ERR_CUDA;                                                                    \
        }                                                                                          \
    } while (0)

// fill (raster.rs:24-104) on the device: inside / thin get 1 at the filled samples, indexed in the
// space of dimensions dims (order 0: (i m1 + j) m2 + k, 1: i + (j + k m1) m0; every sample index
// is below its dimension); thin is then cleared where inside is set.
int raster_fill(Gpu* gpu, const double* tris, uint64_t ntri, const std::vector<double>* samples, const size_t* dims,
                int order, uint8_t* inside, uint8_t* thin, std::string& err) {
    using namespace raster;
    for (int a = 0; a < 3; ++a)
        if (samples[a].size() > dims[a]) { err = "a sample line is longer than its index dimension"; return FG_ERR_INVALID; }
    const size_t total = dims[0] * dims[1] * dims[2];
    std::memset(inside, 0, total);
    std::memset(thin, 0, total);
    if (ntri == 0 || total == 0) return FG_OK;
    if (ntri >= (uint64_t(1) << 31)) { err = "too many triangles"; return FG_ERR_INVALID; }
    RS_CUDA(cudaSetDevice(gpu->device));
    Builder b;
    b.tri = tris;
    b.order.resize(size_t(ntri));
    for (size_t q = 0; q < ntri; ++q) b.order[q] = int(q);
    b.build(0, int(ntri), 1);
    if (b.depth >= STACK / 2) { err = "the mesh's hierarchy is too deep"; return FG_ERR_INVALID; }
    const Node& root = b.nodes[0];
    double low[3], high[3];
    for (int a = 0; a < 3; ++a) { low[a] = root.lo[a]; high[a] = root.hi[a]; }
    double step[3];
    for (int a = 0; a < 3; ++a) {
        const double s = spacing(samples[a]);
        step[a] = std::isfinite(s) ? s : std::fmax(std::fmax(high[0] - low[0], high[1] - low[1]), 1.0);
    }
    int sp0[3], sp1[3];
    for (int a = 0; a < 3; ++a) {   // span (raster.rs:17-22)
        const std::vector<double>& line = samples[a];
        if (line.empty()) return FG_OK;
        const size_t last_sample = line.size() - 1;
        size_t first = partition(line, low[a], true);
        first = first >= 1 ? first - 1 : 0;
        first = first >= 2 ? first - 2 : 0;
        const size_t last = std::min(partition(line, high[a], false) + 2, last_sample);
        if (first > last) return FG_OK;
        sp0[a] = int(first);
        sp1[a] = int(last);
    }
    cudaStream_t st;
    RS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct Bufs {
        void* p[8] = {};
        cudaStream_t st;
        ~Bufs() {
            cudaStreamSynchronize(st);
            for (void* q : p) if (q) cudaFree(q);
            cudaStreamDestroy(st);
        }
    } m;
    m.st = st;
    const size_t lens[3] = {samples[0].size(), samples[1].size(), samples[2].size()};
    RS_CUDA(cudaMalloc(&m.p[0], b.nodes.size() * sizeof(Node)));
    RS_CUDA(cudaMalloc(&m.p[1], b.order.size() * sizeof(int)));
    RS_CUDA(cudaMalloc(&m.p[2], size_t(ntri) * 9 * sizeof(double)));
    RS_CUDA(cudaMalloc(&m.p[3], (lens[0] + lens[1] + lens[2]) * sizeof(double)));
    RS_CUDA(cudaMalloc(&m.p[4], total));
    RS_CUDA(cudaMalloc(&m.p[5], total));
    RS_CUDA(cudaMalloc(&m.p[6], 64));
    RS_CUDA(cudaMemcpyAsync(m.p[0], b.nodes.data(), b.nodes.size() * sizeof(Node), cudaMemcpyHostToDevice, st));
    RS_CUDA(cudaMemcpyAsync(m.p[1], b.order.data(), b.order.size() * sizeof(int), cudaMemcpyHostToDevice, st));
    RS_CUDA(cudaMemcpyAsync(m.p[2], tris, size_t(ntri) * 9 * sizeof(double), cudaMemcpyHostToDevice, st));
    double* dl = static_cast<double*>(m.p[3]);
    RS_CUDA(cudaMemcpyAsync(dl, samples[0].data(), lens[0] * 8, cudaMemcpyHostToDevice, st));
    RS_CUDA(cudaMemcpyAsync(dl + lens[0], samples[1].data(), lens[1] * 8, cudaMemcpyHostToDevice, st));
    RS_CUDA(cudaMemcpyAsync(dl + lens[0] + lens[1], samples[2].data(), lens[2] * 8, cudaMemcpyHostToDevice, st));
    RS_CUDA(cudaMemsetAsync(m.p[4], 0, total, st));
    RS_CUDA(cudaMemsetAsync(m.p[5], 0, total, st));
    RS_CUDA(cudaMemsetAsync(m.p[6], 0, 64, st));
    for (int axis = 0; axis < 3; ++axis) {
        FillAxis f{};
        f.line[0] = dl;
        f.line[1] = dl + lens[0];
        f.line[2] = dl + lens[0] + lens[1];
        for (int a = 0; a < 3; ++a) { f.n[a] = int(lens[a]); f.step[a] = step[a]; }
        f.axis = axis;
        f.u = (axis + 1) % 3;
        f.v = (axis + 2) % 3;
        f.us = sp0[f.u];
        f.wide = sp1[f.u] - sp0[f.u] + 1;
        f.vs = sp0[f.v];
        f.tall = sp1[f.v] - sp0[f.v] + 1;
        const std::vector<double>& line = samples[axis];
        f.start = std::fmin(line[0], low[axis]) - 2.0 * step[axis];
        f.reach0 = line[0] - step[axis] * 0.5;
        f.reach1 = line[line.size() - 1] + step[axis] * 0.5;
        f.order = order;
        for (int a = 0; a < 3; ++a) f.m[a] = (long long)dims[a];
        const long long cols = (long long)f.wide * f.tall;
        k_fill_axis<<<unsigned((cols + 127) / 128), 128, 0, st>>>(
            f, static_cast<const Node*>(m.p[0]), static_cast<const int*>(m.p[1]), static_cast<const double*>(m.p[2]),
            static_cast<uint8_t*>(m.p[4]), static_cast<uint8_t*>(m.p[5]), static_cast<int*>(m.p[6]));
        RS_CUDA(cudaGetLastError());
    }
    int error = 0;
    RS_CUDA(cudaMemcpyAsync(&error, m.p[6], sizeof(int), cudaMemcpyDeviceToHost, st));
    RS_CUDA(cudaMemcpyAsync(inside, m.p[4], total, cudaMemcpyDeviceToHost, st));
    RS_CUDA(cudaMemcpyAsync(thin, m.p[5], total, cudaMemcpyDeviceToHost, st));
    RS_CUDA(cudaStreamSynchronize(st));
    if (error) {
        err = error == 1 ? "the mesh's hierarchy is too deep" : "a column crosses the mesh too often";
        return FG_ERR_INVALID;
    }
    for (size_t q = 0; q < total; ++q)
        if (inside[q]) thin[q] = 0;      // raster.rs:100-103: thin samples that are not inside
    return FG_OK;
}

int raster_sheet_edges(Gpu* gpu, const double* tris, uint64_t ntri, const std::vector<double>* lines, uint8_t* mask,
                       std::string& err) {
    using namespace raster;
    const size_t nn = lines[0].size() * lines[1].size() * lines[2].size();
    std::memset(mask, 0, 3 * nn);
    if (ntri == 0 || nn == 0) return FG_OK;
    for (int a = 0; a < 3; ++a)
        if (lines[a].size() < 2) { err = "a grid axis needs two lines"; return FG_ERR_INVALID; }
    RS_CUDA(cudaSetDevice(gpu->device));
    cudaStream_t st;
    RS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct Bufs {
        void* p[3] = {};
        cudaStream_t st;
        ~Bufs() {
            cudaStreamSynchronize(st);
            for (void* q : p) if (q) cudaFree(q);
            cudaStreamDestroy(st);
        }
    } m;
    m.st = st;
    const size_t lens[3] = {lines[0].size(), lines[1].size(), lines[2].size()};
    RS_CUDA(cudaMalloc(&m.p[0], size_t(ntri) * 9 * sizeof(double)));
    RS_CUDA(cudaMalloc(&m.p[1], (lens[0] + lens[1] + lens[2]) * sizeof(double)));
    RS_CUDA(cudaMalloc(&m.p[2], 3 * nn));
    RS_CUDA(cudaMemcpyAsync(m.p[0], tris, size_t(ntri) * 9 * sizeof(double), cudaMemcpyHostToDevice, st));
    double* dl = static_cast<double*>(m.p[1]);
    RS_CUDA(cudaMemcpyAsync(dl, lines[0].data(), lens[0] * 8, cudaMemcpyHostToDevice, st));
    RS_CUDA(cudaMemcpyAsync(dl + lens[0], lines[1].data(), lens[1] * 8, cudaMemcpyHostToDevice, st));
    RS_CUDA(cudaMemcpyAsync(dl + lens[0] + lens[1], lines[2].data(), lens[2] * 8, cudaMemcpyHostToDevice, st));
    RS_CUDA(cudaMemsetAsync(m.p[2], 0, 3 * nn, st));
    SheetArgs g{};
    g.line[0] = dl;
    g.line[1] = dl + lens[0];
    g.line[2] = dl + lens[0] + lens[1];
    for (int a = 0; a < 3; ++a) g.n[a] = int(lens[a]);
    const unsigned blocks = unsigned(std::min<uint64_t>(ntri, 148 * 32));
    k_sheet_edges<<<blocks, 256, 0, st>>>(g, static_cast<const double*>(m.p[0]), (long long)ntri,
                                          static_cast<uint8_t*>(m.p[2]));
    RS_CUDA(cudaGetLastError());
    RS_CUDA(cudaMemcpyAsync(mask, m.p[2], 3 * nn, cudaMemcpyDeviceToHost, st));
    RS_CUDA(cudaStreamSynchronize(st));
    return FG_OK;
}

// closed (raster.rs:127-143): every edge of the non-degenerate triangles, keyed by its quantised
// end points, is shared by an even number of them.
bool raster_closed(const double* tris, uint64_t ntri) {
    if (ntri == 0) return false;
    double lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint64_t q = 0; q < ntri * 3; ++q)
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::fmin(lo[a], tris[q * 3 + a]);
            hi[a] = std::fmax(hi[a], tris[q * 3 + a]);
        }
    double size = 0.0;
    for (int a = 0; a < 3; ++a) size = std::fmax(size, hi[a] - lo[a]);
    size = std::fmax(size, 1e-30);
    const double base = std::fmin(std::fmin(lo[0], lo[1]), lo[2]);
    struct Key {
        int64_t a[3], b[3];
        bool operator==(const Key& o) const { return std::memcmp(this, &o, sizeof(Key)) == 0; }
    };
    struct Hash {
        size_t operator()(const Key& k) const {
            uint64_t h = 1469598103934665603ull;
            const int64_t* v = k.a;
            for (int q = 0; q < 6; ++q) h = (h ^ uint64_t(v[q])) * 1099511628211ull;
            return size_t(h);
        }
    };
    std::unordered_map<Key, uint32_t, Hash> edges;
    auto key = [&](const double* p, int64_t* o) {
        for (int a = 0; a < 3; ++a) o[a] = int64_t(std::round((p[a] - base) / size * 1e9));
    };
    for (uint64_t t = 0; t < ntri; ++t) {
        int64_t k[3][3];
        for (int v = 0; v < 3; ++v) key(tris + t * 9 + v * 3, k[v]);
        auto same = [&](int x, int y) { return k[x][0] == k[y][0] && k[x][1] == k[y][1] && k[x][2] == k[y][2]; };
        if (same(0, 1) || same(1, 2) || same(0, 2)) continue;
        const int pairs[3][2] = {{0, 1}, {1, 2}, {2, 0}};
        for (auto& pr : pairs) {
            const int64_t* a = k[pr[0]];
            const int64_t* b = k[pr[1]];
            const bool less = std::lexicographical_compare(a, a + 3, b, b + 3);
            Key e;
            std::memcpy(e.a, less ? a : b, sizeof e.a);
            std::memcpy(e.b, less ? b : a, sizeof e.b);
            edges[e] += 1;
        }
    }
    if (edges.empty()) return false;
    for (auto& kv : edges)
        if (kv.second % 2 != 0) return false;
    return true;
}

}  // namespace fg
