// Device-side types and the per-step kernels other than the field stencil: thin-wire H terms,
// resistive sheets, Debye ADE, lumped sources and inductors, port V/I probes, the plane DFT, the
// NTFF accumulation and the energy reduction. Each names the reference code it restates
// (crates/sims-field/src/fdtd/cpu.rs, the CPU path whose results are the parity target).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "host.hpp"

namespace fg {

// Node geometry shared by every kernel. On the device a row of n2 nodes is stored with pitch p2
// (n2 rounded up to 32, so rows start 128-byte aligned and TMA strides are legal): the device
// node index is (i*n1 + j)*p2 + k. Fields are component-major with component stride cs
// (>= n0*n1*p2). The psi slabs follow the reference's layout (sim.rs:659-665), except that a
// z slab (derivative along k) pads its rows of 2 pml slots to pw, a multiple of 4, so its rows
// are whole 16-byte units for the TMA; slabs start 128-byte aligned, and each field's two z
// slabs sit next to each other (one box brings both components).
struct Geom {
    int n0, n1, n2;
    int p2;
    int pml;
    int pw;                     // z-slab row pitch: 2 pml rounded up to 4
    long long nn;               // real nodes n0*n1*n2
    long long cs;
    const AxisNode* ax[3];
    long long psi_off[18];  // offsets of the 12 psi slabs: [field*9 + comp*3 + axis], field 0 = E, 1 = H
};

// A node's three (ca, cb) pairs as the kernels read them: 32 bytes, two 16-byte loads.
struct __align__(16) DevCoef {
    float ca[3];
    float pad0;
    float cb[3];
    float pad1;
};

struct DevSheet {           // pack() sheet record (run.rs:259-289), named
    long long f, ha, hb;    // field indices (comp*cs + id)
    float len, c, r, adaptive;
    float aa, bb, ab, ma, mb, old, i_old;
    unsigned face_a, face_b;
};

struct DevSource { long long f; float src; };           // run.rs:243-246
struct DevInductor { long long f; float ke, ki, cur; };  // run.rs:247-250
struct DevPortEdge { long long id; float w; };           // run.rs:314-317
struct DevLoop { long long f; float w; };                // run.rs:326-328 (f = (3+comp-3)*cs + id)
struct DevProbe { int comp, first, count, loop_first, loop_count; };
struct DevWire { long long h; long long e[4]; float c[4]; };

struct StepConst {          // per-run scalars (run.rs:433-464 Params)
    float k_mu, dt, t0, tau, w0;
    int nf;
    float omega[4];
    unsigned cap;
    int ports;
    // Per-step tables formed on the host with the same f32 libm calls as the reference's CPU path
    // (cpu.rs:262-265, :344-353, :370-405), for steps below `cap`:
    const float* pulse;     // [cap]             pulse((n + 1/2) dt)
    const float* dft;       // [cap][nf][4]      cos(w te) dt, -sin(w te) dt, cos(w th) dt, -sin(w th) dt
    const float* far;       // [cap][nf][4]      cos(-w te) dt, sin(-w te) dt, cos(-w th) dt, sin(-w th) dt
};

__device__ __forceinline__ long long psi_at(const Geom& g, int a, int i, int j, int k, int s) {
    if (a == 0) return ((long long)s * g.n1 + j) * g.n2 + k;
    if (a == 1) return ((long long)i * (2 * g.pml) + s) * g.n2 + k;
    return ((long long)i * g.n1 + j) * g.pw + s;
}

// The step index n of the running step: the first kernel of step n raised the counter to n + 1.
__device__ __forceinline__ unsigned step_index(const unsigned* counter) { return *(volatile const unsigned*)counter - 1u; }

// The step index for a kernel that may run beside the next step's kernels (the next step's first
// kernel opens step n + 1 by incrementing the counter, and the step after that waits for this
// kernel): the step of parity `parity` among the two the counter can show (parity -1: the kernel
// runs in order, the counter's step).
__device__ __forceinline__ unsigned step_of(const unsigned* counter, int parity) {
    const unsigned n = step_index(counter);
    return (parity < 0 || int(n & 1u) == parity) ? n : n - 1u;
}

// cpu.rs:270-273: h[w.h] += sum of four c*E terms, after the H update, with E not yet updated.
__global__ void k_wire_h(const DevWire* __restrict__ w, int count, const float* __restrict__ e, float* __restrict__ h) {
    int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= count) return;
    DevWire x = w[s];
    float t0 = x.c[0] * e[x.e[0]], t1 = x.c[1] * e[x.e[1]], t2 = x.c[2] * e[x.e[2]], t3 = x.c[3] * e[x.e[3]];
    h[x.h] += ((t0 + t1) + t2) + t3;
}

// cpu.rs:169-193 on one sheet edge: before the E update, with the new H.
__device__ __forceinline__ void sheet_before(DevSheet& s, float old, float ha, float hb) {
    s.old = old;
    float aa = s.aa + ha * ha, bb = s.bb + hb * hb, ab = s.ab + ha * hb;
    s.aa = aa;
    s.bb = bb;
    s.ab = ab;
    float sum = aa + bb;
    if (sum <= 1e-30f) return;
    float scale = 1.0f;
    if (s.adaptive != 0.0f) {
        scale = s.ma + s.mb;
        float tot = aa + bb - 2.0f * ab;
        if (tot > 1e-30f) scale = fminf(fmaxf(sum / tot, 0.5f), 4.0f);
    }
    s.ma = scale * aa / sum;
    s.mb = scale * bb / sum;
}

__global__ void k_sheet_pre(DevSheet* __restrict__ sh, int count, const float* __restrict__ e, const float* __restrict__ h) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    DevSheet s = sh[q];
    sheet_before(s, e[s.f], h[s.ha], h[s.hb]);
    sh[q] = s;
}

// cpu.rs:195-237: the sheet current from the branch table after the E update.
__global__ void k_sheet_post(DevSheet* __restrict__ sh, int count, const float* __restrict__ br, float* __restrict__ cur,
                             float* __restrict__ e) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    DevSheet s = sh[q];
    const int nr = int(br[0]), nc = int(br[1]);
    const int stride = 2 + nr + 2 * nc, faces = 4 + 2 * nr + 4 * nc;
    const int fa = faces + int(s.face_a) * stride, fb = faces + int(s.face_b) * stride;
    const long long base = (long long)q * (nr + 2 * nc);
    const float ma = s.ma, mb = s.mb;
    float hist = (ma * br[fa + 1] + mb * br[fb + 1]) * s.i_old;
    for (int k = 0; k < nr; ++k) hist -= (ma * br[fa + 2 + k] + mb * br[fb + 2 + k]) * cur[base + k];
    for (int k = 0; k < nc; ++k) {
        int o = 2 + nr + 2 * k;
        float cr = ma * br[fa + o] + mb * br[fb + o];
        float ci = ma * br[fa + o + 1] + mb * br[fb + o + 1];
        long long u = base + nr + 2 * k;
        hist -= cr * cur[u] - ci * cur[u + 1];
    }
    float a = s.r * (ma * br[fa] + mb * br[fb]);
    float ef = e[s.f];
    float ibar = (0.5f * s.len * (ef + s.old) + s.r * hist) / (a + 0.5f * s.len * s.c);
    e[s.f] = ef - s.c * ibar;
    s.i_old = 2.0f * ibar - s.i_old;
    for (int k = 0; k < nr; ++k) {
        int p = 4 + 2 * k;
        cur[base + k] = br[p] * cur[base + k] + br[p + 1] * ibar;
    }
    for (int k = 0; k < nc; ++k) {
        int p = 4 + 2 * nr + 4 * k;
        long long u = base + nr + 2 * k;
        float ur = cur[u], ui = cur[u + 1];
        cur[u] = br[p] * ur - br[p + 1] * ui + br[p + 2] * ibar;
        cur[u + 1] = br[p] * ui + br[p + 1] * ur + br[p + 3] * ibar;
    }
    sh[q] = s;
}

// cpu.rs:281-283: the E of each Debye edge before the E update.
__global__ void k_debye_pre(const long long* __restrict__ f, int count, const float* __restrict__ e, float* __restrict__ old) {
    int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q < count) old[q] = e[f[q]];
}

// cpu.rs:239-260: E -= cb * sum_k 0.5 (1 + b_k) s_k; s_k = b_k s_k + dd c_k (E_new - E_old).
// `eold` is either the saved copy (separate step) or the step's input buffer (fused step).
template <typename CID>
__device__ __forceinline__ void debye_post_edge(int q, const long long* __restrict__ f, const float* __restrict__ dd,
                                                int count, const float* __restrict__ eold_saved,
                                                const float* __restrict__ eold_field, const CID* __restrict__ node_class,
                                                const DevCoef* __restrict__ classes, long long cs,
                                                const float* __restrict__ table, float* __restrict__ state,
                                                float* __restrict__ e) {
    const long long fi = f[q];
    const int c = int(fi / cs);
    const long long id = fi - c * cs;
    const float cb = classes[node_class[id]].cb[c];
    const float old = eold_saved ? eold_saved[q] : eold_field[fi];
    const int np = int(table[0]);
    float s0 = 0.0f;
    for (int k = 0; k < np; ++k) s0 += 0.5f * (1.0f + table[1 + 2 * k]) * state[(long long)k * count + q];
    const float next = e[fi] - cb * s0;
    e[fi] = next;
    const float de = next - old;
    const float w = dd[q];
    for (int k = 0; k < np; ++k) {
        long long p = (long long)k * count + q;
        state[p] = table[1 + 2 * k] * state[p] + w * table[2 + 2 * k] * de;
    }
}

// debye_post_edge with each edge's cb given (cbq, formed once at set-up): no class-id lookup
// between the edge list and the arithmetic, so every load of an edge issues at once.
__global__ void k_debye_post_cb(const long long* __restrict__ f, const float* __restrict__ dd,
                                const float* __restrict__ cbq, int count, const float* __restrict__ eold_saved,
                                const float* __restrict__ eold_field, const float* __restrict__ table,
                                float* __restrict__ state, float* __restrict__ e) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const long long fi = f[q];
    const float cb = cbq[q];
    const float old = eold_saved ? eold_saved[q] : eold_field[fi];
    const int np = int(table[0]);
    float s0 = 0.0f;
    for (int k = 0; k < np; ++k) s0 += 0.5f * (1.0f + table[1 + 2 * k]) * state[(long long)k * count + q];
    const float next = e[fi] - cb * s0;
    e[fi] = next;
    const float de = next - old;
    const float w = dd[q];
    for (int k = 0; k < np; ++k) {
        long long p = (long long)k * count + q;
        state[p] = table[1 + 2 * k] * state[p] + w * table[2 + 2 * k] * de;
    }
}


// The Debye ADE of k_debye_post_cb for edges whose pole state lives in time slots: edge q's state
// is s_in[sidx[q] * np + k] before the step and s_out[...] after it (the steps of the two-step mode
// keep three slots, so no kernel reads a state another has already advanced).
__global__ void k_debye_slots(const long long* __restrict__ f, const unsigned* __restrict__ sidx,
                              const float* __restrict__ dd, const float* __restrict__ cbq, int count,
                              const float* __restrict__ eold, const float* __restrict__ table,
                              const float* __restrict__ s_in, float* __restrict__ s_out, float* __restrict__ e) {
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const long long fi = f[q];
    const float cb = cbq[q];
    const float old = eold[fi];
    const int np = int(table[0]);
    const size_t b = size_t(sidx[q]) * size_t(np);
    float s0 = 0.0f;
    for (int k = 0; k < np; ++k) s0 += 0.5f * (1.0f + table[1 + 2 * k]) * s_in[b + k];
    const float next = e[fi] - cb * s0;
    e[fi] = next;
    const float de = next - old;
    const float w = dd[q];
    for (int k = 0; k < np; ++k) s_out[b + k] = table[1 + 2 * k] * s_in[b + k] + w * table[2 + 2 * k] * de;
}

// Per Debye node (device index), the state index of its first edge: the smallest index among the
// node's edges (f = comp * cs + node, sidx = the edge's state index); dbase starts at all ones.
__global__ void k_debye_base(const long long* __restrict__ f, const unsigned* __restrict__ sidx, long long count,
                             long long cs, unsigned* __restrict__ dbase) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    atomicMin(dbase + (f[q] % cs), sidx[q]);
}

// cpu.rs:262-265
__device__ __forceinline__ float pulse_at(const StepConst& sc, float t) {
    float x = (t - sc.t0) / sc.tau;
    return expf(-x * x) * cosf(sc.w0 * (t - sc.t0));
}

// cpu.rs:291-303: the driven port's soft source at t = (n + 1/2) dt, then the inductor ADE.
// One block; the source edges of a port are distinct, as are the inductor edges.
__device__ __forceinline__ void lumped_block(const DevSource* __restrict__ src, int ns, DevInductor* __restrict__ ind,
                                             int ni, const StepConst& sc, const unsigned* __restrict__ counter,
                                             float* __restrict__ e) {
    const unsigned n = step_index(counter);
    const float p = n < sc.cap ? sc.pulse[n] : pulse_at(sc, (float(n) + 0.5f) * sc.dt);
    for (int q = threadIdx.x; q < ns; q += blockDim.x) {
        DevSource s = src[q];
        e[s.f] -= s.src * p;
    }
    __syncthreads();
    for (int q = threadIdx.x; q < ni; q += blockDim.x) {
        DevInductor d = ind[q];
        float x = e[d.f] - d.ke * d.cur;
        e[d.f] = x;
        ind[q].cur = d.cur + d.ki * x;
    }
}

__global__ void k_lumped(const DevSource* __restrict__ src, int ns, DevInductor* __restrict__ ind, int ni,
                         StepConst sc, const unsigned* __restrict__ counter, float* __restrict__ e) {
    lumped_block(src, ns, ind, ni, sc, counter, e);
}

// cpu.rs:309-334: per port V = -sum E*w over its edges and I = sum H*w around the loop, summed
// in f64 like the CPU path; one block per port.
__device__ __forceinline__ void probe_block(int port, const DevProbe* __restrict__ defs,
                                            const DevPortEdge* __restrict__ pe, const DevLoop* __restrict__ lp,
                                            long long cs, const float* __restrict__ e, const float* __restrict__ h,
                                            const unsigned* __restrict__ counter, const StepConst& sc,
                                            float* __restrict__ series) {
    __shared__ double sv[256], si[256];
    const DevProbe d = defs[port];
    double v = 0.0, cur = 0.0;
    for (int q = threadIdx.x; q < d.count; q += blockDim.x) {
        DevPortEdge x = pe[d.first + q];
        v -= double(e[(long long)d.comp * cs + x.id] * x.w);
    }
    for (int q = threadIdx.x; q < d.loop_count; q += blockDim.x) {
        DevLoop x = lp[d.loop_first + q];
        cur += double(h[x.f] * x.w);
    }
    sv[threadIdx.x] = v;
    si[threadIdx.x] = cur;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            sv[threadIdx.x] += sv[threadIdx.x + s];
            si[threadIdx.x] += si[threadIdx.x + s];
        }
        __syncthreads();
    }
    const unsigned n = step_index(counter);
    if (threadIdx.x == 0 && n < sc.cap) {
        long long o = ((long long)n * sc.ports + port) * 2;
        series[o] = float(sv[0]);
        series[o + 1] = float(si[0]);
    }
}

__global__ void k_probe(const DevProbe* __restrict__ defs, const DevPortEdge* __restrict__ pe, const DevLoop* __restrict__ lp,
                        long long cs, const float* __restrict__ e, const float* __restrict__ h,
                        const unsigned* __restrict__ counter, StepConst sc, float* __restrict__ series) {
    probe_block(blockIdx.x, defs, pe, lp, cs, e, h, counter, sc, series);
}

// The driven port's source (and inductors) then the probe of a Sim's single port, in one block:
// lumped_block's writes are visible to probe_block after the block barrier.
__global__ void k_lumped_probe(const DevSource* __restrict__ src, int ns, DevInductor* __restrict__ ind, int ni,
                               StepConst sc, const unsigned* __restrict__ counter, float* __restrict__ e,
                               const DevProbe* __restrict__ defs, const DevPortEdge* __restrict__ pe,
                               const DevLoop* __restrict__ lp, long long cs, const float* __restrict__ h,
                               float* __restrict__ series) {
    lumped_block(src, ns, ind, ni, sc, counter, e);
    __syncthreads();
    probe_block(0, defs, pe, lp, cs, e, h, counter, sc, series);
}

// cpu.rs:336-361: running DFT of Ex, Ey, Ez (at (n+1) dt) and Hx, Hy (at (n+1/2) dt) on the
// z-plane k = plane_k; phases formed in f32 like the CPU path.
__global__ void k_field_dft(Geom g, int plane_k, StepConst sc, const unsigned* __restrict__ counter, int parity,
                            const float* __restrict__ e, const float* __restrict__ h, float* __restrict__ acc) {
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= (long long)g.n0 * g.n1) return;
    const unsigned n = step_of(counter, parity);
    const float te = (float(n) + 1.0f) * sc.dt, th = (float(n) + 0.5f) * sc.dt;
    const long long id = q * g.p2 + plane_k;
    const float f[5] = {e[id], e[g.cs + id], e[2 * g.cs + id], h[id], h[g.cs + id]};
    float* out = acc + q * sc.nf * 10;
    for (int k = 0; k < sc.nf; ++k) {
        const float w = sc.omega[k];
        float ce0, ce1, ch0, ch1;
        if (n < sc.cap) {
            const float* t = sc.dft + ((long long)n * sc.nf + k) * 4;
            ce0 = t[0]; ce1 = t[1]; ch0 = t[2]; ch1 = t[3];
        } else {
            ce0 = cosf(w * te) * sc.dt; ce1 = -sinf(w * te) * sc.dt;
            ch0 = cosf(w * th) * sc.dt; ch1 = -sinf(w * th) * sc.dt;
        }
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            const float p0 = c >= 3 ? ch0 : ce0, p1 = c >= 3 ? ch1 : ce1;
            out[k * 10 + 2 * c] += f[c] * p0;
            out[k * 10 + 2 * c + 1] += f[c] * p1;
        }
    }
}

// cpu.rs:363-415: per NTFF patch, tangential E (2-edge mean) and H (4-edge mean), J = n x H,
// M = E x n, accumulated with dt e^{-j w t}. Component-major on the device so a warp's loads and
// stores coalesce: the patch record's word m of patch g at pidx[m * patches + g], accumulator
// (frequency k, value c of 12) at acc[(k * 12 + c) * patches + g] (read back in the reference's
// patch-major order).
__global__ void k_ntff(const unsigned* __restrict__ pidx, int patches, long long cs, StepConst sc,
                       const unsigned* __restrict__ counter, int parity, const float* __restrict__ e,
                       const float* __restrict__ h, float* __restrict__ acc) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= patches) return;
    const unsigned n = step_of(counter, parity);
    unsigned b[13];
#pragma unroll
    for (int m = 0; m < 13; ++m) b[m] = pidx[(long long)m * patches + g];
    const unsigned meta = b[0];
    const int axis = meta & 3;
    const float side = (meta & 4) ? 1.0f : -1.0f;
    const int u = (axis + 1) % 3, v = (axis + 2) % 3;
    float ef[3] = {0, 0, 0}, hf[3] = {0, 0, 0};
    ef[u] = 0.5f * (e[u * cs + b[1]] + e[u * cs + b[2]]);
    ef[v] = 0.5f * (e[v * cs + b[3]] + e[v * cs + b[4]]);
    hf[u] = 0.25f * (h[u * cs + b[5]] + h[u * cs + b[6]] + h[u * cs + b[7]] + h[u * cs + b[8]]);
    hf[v] = 0.25f * (h[v * cs + b[9]] + h[v * cs + b[10]] + h[v * cs + b[11]] + h[v * cs + b[12]]);
    float nrm[3] = {0, 0, 0};
    nrm[axis] = side;
    const float jv[3] = {nrm[1] * hf[2] - nrm[2] * hf[1], nrm[2] * hf[0] - nrm[0] * hf[2], nrm[0] * hf[1] - nrm[1] * hf[0]};
    const float mv[3] = {ef[1] * nrm[2] - ef[2] * nrm[1], ef[2] * nrm[0] - ef[0] * nrm[2], ef[0] * nrm[1] - ef[1] * nrm[0]};
    const float te = (float(n) + 1.0f) * sc.dt, th = (float(n) + 0.5f) * sc.dt;
    for (int k = 0; k < sc.nf; ++k) {
        const float wf = sc.omega[k];
        float pe0, pe1, ph0, ph1;
        if (n < sc.cap) {
            const float* t = sc.far + ((long long)n * sc.nf + k) * 4;
            pe0 = t[0]; pe1 = t[1]; ph0 = t[2]; ph1 = t[3];
        } else {
            pe0 = cosf(-wf * te) * sc.dt; pe1 = sinf(-wf * te) * sc.dt;
            ph0 = cosf(-wf * th) * sc.dt; ph1 = sinf(-wf * th) * sc.dt;
        }
        float* o = acc + (long long)k * 12 * patches + g;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            o[(long long)(2 * c) * patches] += ph0 * jv[c];
            o[(long long)(2 * c + 1) * patches] += ph1 * jv[c];
            o[(long long)(6 + 2 * c) * patches] += pe0 * mv[c];
            o[(long long)(6 + 2 * c + 1) * patches] += pe1 * mv[c];
        }
    }
}

// cpu.rs:417-421: sum of E^2 + (376.73 H)^2 in f64, one partial per block. Row padding and the
// component tail hold zeros and add nothing.
__global__ void k_energy(Geom g, const float* __restrict__ e, const float* __restrict__ h, double* __restrict__ partial) {
    __shared__ double s[256];
    double acc = 0.0;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (int c = 0; c < 3; ++c) {
        const float* ec = e + c * g.cs;
        const float* hc = h + c * g.cs;
        for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < g.cs; q += stride) {
            double x = double(ec[q]);
            double y = double(hc[q]) * 376.73;
            acc += x * x + y * y;
        }
    }
    s[threadIdx.x] = acc;
    __syncthreads();
    for (int k = blockDim.x / 2; k > 0; k >>= 1) {
        if (threadIdx.x < k) s[threadIdx.x] += s[threadIdx.x + k];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = s[0];
}

}  // namespace fg
