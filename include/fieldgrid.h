/*
 * fieldgrid.h — C ABI of the B200-native Yee-grid FDTD engine.
 *
 * This is the drop-in boundary for the `sims_field::fdtd` solve of v0l/fieldgrid
 * (crate `sims-field`, files `src/fdtd/{sim.rs,run.rs,cpu.rs,ntff.rs}`, `src/gpu.rs`).
 * Every entry point below names the reference item it stands in for. The ABI uses
 * plain C types only: pointers, sizes, and the POD structs declared here. Strings
 * returned in `err` buffers are the reference's own `Err(String)` texts, so a
 * caller that matches on them (the reference's tests do) keeps working.
 *
 * Ownership: every handle is created and freed by this library. Input arrays are
 * borrowed for the duration of the call only. Handles are not thread-safe; distinct
 * handles are independent. There is no CPU fallback: with no CUDA device every
 * device entry point returns FG_ERR_NO_DEVICE.
 *
 * Index conventions are the reference's: node counts n = grid.dims() (cells + 1 per
 * axis), node id = (i*n1 + j)*n2 + k (k fastest), fields are component-major
 * (field[c*nn + id]) and materials are per cell ((n0-1)(n1-1)(n2-1), same order).
 */
#ifndef FIELDGRID_H
#define FIELDGRID_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes. Each non-zero code comes with a message (err buffer / fg_last_error). */
#define FG_OK 0
#define FG_ERR_INVALID 1      /* malformed argument (null pointer, bad index, ...) */
#define FG_ERR_SETUP 2        /* Sim::try_new refused, e.g. the thin-wire radius text */
#define FG_ERR_NO_DEVICE 3    /* no usable CUDA device: this library never falls back to the CPU */
#define FG_ERR_TOO_LARGE 4    /* "{cells} cells is more than this GPU can hold" */
#define FG_ERR_PORT_INDEX 5   /* "grid too large for f32 port indices" (run.rs:341-343) */
#define FG_ERR_UNSTABLE 6     /* "the FDTD run went unstable" (run.rs:734-738) */
#define FG_ERR_CANCELLED 7    /* "cancelled": the progress callback returned 0 (run.rs:742-744) */
#define FG_ERR_CUDA 8         /* a CUDA runtime call failed; the message names it */
#define FG_ERR_UNSUPPORTED 9  /* a request this build does not implement */

/* ---- opaque handles ---------------------------------------------------------------- */
typedef struct fg_gpu fg_gpu;         /* sims_field::Gpu (gpu.rs:36-41): one CUDA device + stream */
typedef struct fg_sim fg_sim;         /* sims_field::fdtd::Sim (sim.rs:173-189), host-side */
typedef struct fg_record fg_record;   /* sims_field::fdtd::Record (run.rs:52-59) */
typedef struct fg_session fg_session; /* device-resident state of one run (run.rs:390-758 buffers) */
typedef struct fg_far fg_far;         /* sims_field::fdtd::Far (ntff.rs:67-74) */

/* ---- setup inputs (sim.rs) ----------------------------------------------------------- */
typedef struct fg_edge {              /* Edge (sim.rs:145-149) */
    uint32_t comp;
    uint32_t reserved;
    uint64_t at[3];
} fg_edge;

enum fg_element_kind {                /* Element (sim.rs:151-156) */
    FG_RESISTOR = 0,
    FG_CAPACITOR = 1,
    FG_INDUCTOR = 2
};

typedef struct fg_lumped {            /* Lumped (sim.rs:158-163) */
    const char* name;
    const fg_edge* edges;
    uint64_t n_edges;
    int32_t element;                  /* fg_element_kind */
    int32_t reserved;
    double value;                     /* ohm, farad or henry */
} fg_lumped;

typedef struct fg_port {              /* PortDef (sim.rs:165-171); columns flattened */
    const char* name;
    const fg_edge* edges;             /* all columns back to back */
    const uint64_t* column_len;       /* n_columns entries */
    uint64_t n_columns;
    double r;
    int32_t reference_above;
    int32_t reserved;
} fg_port;

typedef struct fg_resistive {         /* Resistive (sim.rs:208-215) */
    uint32_t comp;
    int32_t adaptive;
    uint64_t id;                      /* node id of the edge */
    double r;
    uint64_t faces[2];
} fg_resistive;

typedef struct fg_wire {              /* one Media.wires entry (Edge, radius) (sim.rs:240) */
    fg_edge edge;
    double radius;
} fg_wire;

/* pec(comp, at) of Sim::try_new (sim.rs:355). Return non-zero for a PEC edge. */
typedef int (*fg_pec_fn)(void* user, uint32_t comp, const uint64_t at[3]);

typedef struct fg_sim_spec {          /* the arguments of Sim::try_new (sim.rs:352-360) */
    const double* x; uint64_t nx;     /* Grid (grid.rs:2-7): node lines */
    const double* y; uint64_t ny;
    const double* z; uint64_t nz;
    uint64_t pml;
    const float* eps;                 /* Materials (sim.rs:217-222), one value per cell; */
    const float* sigma;               /* NULL means Materials::new's default */
    const float* inf;                 /* (eps 1, sigma 0, inf 1, debye 0) */
    const float* debye;
    const uint8_t* pec_mask;          /* 3*nn bytes, comp-major, non-zero = PEC; may be NULL */
    fg_pec_fn pec_fn;                 /* alternative to pec_mask; both NULL = no PEC edges */
    void* pec_user;
    const fg_lumped* lumped; uint64_t n_lumped;
    const fg_port* ports; uint64_t n_ports;
    const fg_resistive* resistive; uint64_t n_resistive;
    const float* sheet_table; uint64_t sheet_table_len;   /* Media.sheets (sim.rs:224-234); */
    uint64_t sheet_states;                                /* NULL table = Sheets::default() */
    const double* debye_poles; uint64_t n_debye_poles;    /* Media.debye: (x, a) pairs */
    const fg_wire* wires; uint64_t n_wires;               /* Media.wires */
} fg_sim_spec;

/* ---- run inputs (run.rs:34-50) -------------------------------------------------------- */
typedef struct fg_pulse {             /* Pulse (run.rs:47-50) */
    double f0;
    double fc;
} fg_pulse;

typedef struct fg_extras {            /* Extras (run.rs:34-45) */
    uint64_t min_steps;
    uint64_t max_steps;
    double decay_db;
    const double* freqs; uint64_t n_freqs;   /* the first 4 are used */
    int32_t has_plane_k;                     /* plane_k: Option<usize> */
    int32_t fused_e;                         /* 1: the fused E+H march; 0: separate H and E kernels */
    uint64_t plane_k;
    const uint32_t* ntff; uint64_t ntff_len; /* patches(...).gpu, 13 u32 per patch; NULL = None */
    uint64_t check_every;                    /* 0 = 1000 */
    int32_t profile;                         /* print per-kernel device times to stderr */
    int32_t keep_fields;                     /* also return the final E/H in the record */
} fg_extras;

/* progress(steps, decay_db) of run (run.rs:396). Return 0 to cancel. */
typedef int (*fg_progress_fn)(void* user, uint64_t steps, double decay_db);

/* ---- library -------------------------------------------------------------------------- */
const char* fg_version(void);
/* The message of the last failed call on this thread. */
const char* fg_last_error(void);

/* ---- device (gpu.rs) -------------------------------------------------------------------- */
/* Gpu::open / open_blocking (gpu.rs:86-108). device < 0 picks device 0. */
int fg_gpu_open(int device, fg_gpu** out, char* err, size_t errlen);
void fg_gpu_close(fg_gpu* g);
/* Gpu.name (gpu.rs:40); copies at most len-1 bytes. */
int fg_gpu_name(const fg_gpu* g, char* dst, size_t len);

/* ---- setup (sim.rs) --------------------------------------------------------------------- */
/* Sim::try_new (sim.rs:352-554). On failure *out stays NULL and err holds the reference text. */
int fg_sim_try_new(const fg_sim_spec* spec, fg_sim** out, char* err, size_t errlen);
void fg_sim_free(fg_sim* sim);
/* Sim.dt (sim.rs:176), Sim::dims (sim.rs:637-639). */
double fg_sim_dt(const fg_sim* sim);
void fg_sim_dims(const fg_sim* sim, uint64_t n[3]);
/* Lengths of Sim.port_src[port] / inductors / sheets / debye_edges / wires / ports (sim.rs:180-188). */
uint64_t fg_sim_count(const fg_sim* sim, const char* what);
/* Sim.ca[comp] / Sim.cb[comp] (sim.rs:177-178): nn floats each into caller buffers. */
int fg_sim_coefs(const fg_sim* sim, uint32_t comp, float* ca, float* cb);
/* Sim.wires (sim.rs:191-195) as 9 u32 per wire: h, then (e, coeff bits) x 4 (run.rs:251-258). */
int fg_sim_wires(const fg_sim* sim, uint32_t* dst, uint64_t len);
/* Number of distinct (ca, cb) node triples the engine's coefficient table holds. */
uint64_t fg_sim_coef_classes(const fg_sim* sim);

/* time_step (sim.rs:133-137) of a grid given by its node lines. */
double fg_time_step(const double* x, uint64_t nx, const double* y, uint64_t ny,
                    const double* z, uint64_t nz);

/* ---- the solve (run.rs) ------------------------------------------------------------------ */
/* run / run_blocking (run.rs:379-397). g == NULL is the `None` of the Option<&Gpu> entry
 * and returns FG_ERR_NO_DEVICE: there is no CPU path in this library. */
int fg_run(fg_gpu* g, const fg_sim* sim, uint64_t driven, const fg_pulse* pulse,
           const fg_extras* extras, fg_progress_fn progress, void* user,
           fg_record** out, char* err, size_t errlen);

/* Record fields (run.rs:52-59). Pointers stay valid until fg_record_free. */
uint64_t fg_record_steps(const fg_record* r);
uint64_t fg_record_ports(const fg_record* r);
double fg_record_decay_db(const fg_record* r);
const float* fg_record_series(const fg_record* r, uint64_t* len);
const float* fg_record_plane(const fg_record* r, uint64_t* len);
const float* fg_record_ntff(const fg_record* r, uint64_t* len);
/* Final E and H (3*nn each, reference layout) when extras.keep_fields was set; else NULL. */
const float* fg_record_e(const fg_record* r, uint64_t* len);
const float* fg_record_h(const fg_record* r, uint64_t* len);
/* Bytes the run copied host->device (the packed grid: class ids, tables, lists) and
 * device->host (energy partials, series, plane, ntff, fields). */
void fg_record_transfer(const fg_record* r, uint64_t* h2d, uint64_t* d2h);
void fg_record_free(fg_record* r);

/* ---- device-resident session: the buffers of one run, stepped explicitly ------------------
 * fg_run is fg_session_new + chunks of fg_session_step + energy checks + reads. The session
 * keeps every buffer in HBM between calls, so a caller can time the step loop alone. */
int fg_session_new(fg_gpu* g, const fg_sim* sim, uint64_t driven, const fg_pulse* pulse,
                   const fg_extras* extras, fg_session** out, char* err, size_t errlen);
/* Enqueue k time steps on the session's stream (CUDA-graph replays); does not wait. */
int fg_session_step(fg_session* s, uint64_t k);
/* Wait for the session's stream. */
int fg_session_sync(fg_session* s);
/* Sum of E^2 + (376.73 H)^2 over the current fields (cpu.rs:417-421), waits. */
int fg_session_energy(fg_session* s, double* out);
/* Steps taken so far. */
uint64_t fg_session_steps(const fg_session* s);
/* Copy results out: which = "series" (steps*ports*2), "plane", "ntff", "e", "h" (3*nn each,
 * reference layout). len is the number of floats the caller's buffer holds. */
int fg_session_read(fg_session* s, const char* which, float* dst, uint64_t len);
/* The CUDA stream the session launches on (a cudaStream_t), for event timing. */
void* fg_session_stream(fg_session* s);
/* Kernel launches one time step enqueues (for launch accounting). */
uint64_t fg_session_launches_per_step(const fg_session* s);
/* Device bytes the session holds. */
uint64_t fg_session_device_bytes(const fg_session* s);
/* Per-kernel device times of `steps` steps launched one kernel at a time with CUDA events
 * between the launches (the report of run.rs:153-176). Fills up to `cap` entries of names
 * (each up to 63 chars + NUL, 64 bytes per entry) and mean ms per launch; *count = kernels per
 * step. The steps count as steps of the run. */
int fg_session_kernel_times(fg_session* s, uint64_t steps, char* names, double* ms, uint64_t cap, uint64_t* count);
/* Name of the stencil kernel variant in use and its tile shape. */
const char* fg_session_variant(const fg_session* s);
void fg_session_free(fg_session* s);

/* ---- field energy without device allocation --------------------------------------------
 * No counterpart in the reference. For callers that cannot allocate device memory when they need
 * the energy of a field (e.g. an operator callback running while a host framework's caching
 * allocator owns the device memory, or a loop that must avoid the device-wide synchronisation of
 * cudaMalloc/cudaFree): sum over q < n of e[q]^2 + (376.73 h[q])^2, each term and the sum in f64,
 * written to *out; n = 0 gives 0, and e and h may then be NULL. e, h and out are device pointers
 * owned by the caller; the call allocates nothing. Its per-block partial sums live in one fixed
 * array of FG_ENERGY_NOALLOC_MAX_BLOCKS doubles (32 KB) per device, held from the library's load
 * until process exit; each call splits its n elements over at most that many blocks, and n is
 * limited to FG_ENERGY_NOALLOC_MAX_BLOCKS * FG_ENERGY_NOALLOC_CHUNK (2^32): larger n is refused
 * with FG_ERR_INVALID. The first call on a device looks up that array's device address and keeps
 * it (make that call before any stream capture); after cudaDeviceReset on that device the kept
 * address is stale, so do not call this entry point again in that process. Every call uses the
 * same array: calls that overlap on the GPU (different streams, or host threads on one device)
 * race; calls ordered on one stream are safe. Work is enqueued on `stream` (NULL = the default
 * stream); read *out after that stream is synchronised. */
#define FG_ENERGY_NOALLOC_MAX_BLOCKS 4096
#define FG_ENERGY_NOALLOC_CHUNK (1u << 20)
int fg_energy_noalloc(const float* e, const float* h, uint64_t n, double* out, void* stream);

/* ---- near-to-far field (ntff.rs) -------------------------------------------------------- */
/* patches(sim, inset).gpu (ntff.rs:11-59): 13 u32 per patch. Call with dst == NULL to get the
 * count of patches in *count, then again with a buffer of 13*count u32 (and pos/area of
 * 3*count / count doubles, each may be NULL). */
int fg_patches(const fg_sim* sim, uint64_t inset, uint32_t* dst, double* pos, double* area,
               uint64_t* count);
/* Far::load (ntff.rs:77-88) from a record's ntff accumulators. */
int fg_far_load(const double* pos, const double* area, uint64_t count, const float* acc,
                uint64_t nf, uint64_t k, double freq, double scale_re, double scale_im,
                fg_far** out);
void fg_far_free(fg_far* f);
/* Far::field (ntff.rs:90-116) for n directions (3 doubles each) -> 6 doubles each
 * (re, im of x, y, z), computed on the GPU when g != NULL. */
int fg_far_field(fg_gpu* g, const fg_far* f, const double* dirs, uint64_t n, double* out);
/* Far::intensity (ntff.rs:118-120) for n directions. */
int fg_far_intensity(fg_gpu* g, const fg_far* f, const double* dirs, uint64_t n, double* out);
/* Far::radiated (ntff.rs:122-136): total radiated power and peak intensity. */
int fg_far_radiated(fg_gpu* g, const fg_far* f, uint64_t steps, double* total, double* peak);

/* ---- port spectra (sims-antenna/src/fdtd/mod.rs:229-266, finish) -------------------------
 * The running DFT of one port's V/I series at nf frequencies, in f64: V(f) = sum_n V_n dt
 * e^{-j w (n+1) dt}, I(f) = sum_n I_n dt e^{-j w (n+1/2) dt}, w = 2 pi f. series is the record's
 * (steps * ports * 2) floats; v and i receive nf (re, im) pairs. The caller forms Z = V/I,
 * S11 = (Z - 50)/(Z + 50) and P_in = Re(V conj(I))/2 from them, as finish does. Host code. */
int fg_port_spectra(const float* series, uint64_t steps, uint64_t ports, uint64_t port, double dt,
                    const double* freqs, uint64_t nf, double* v, double* i);

/* ---- adjoint: the gradient of a flux objective over a box of design voxels ----
 * No counterpart in the reference (sims_field::fdtd has no adjoint). The objective is
 * J = |F|^2, F = sum over the (i, j) window of the z-plane plane_k of
 * dA (Ex^ conj(Hy^) - Ey^ conj(Hx^)), with Ex^..Hy^ the running DFT at `freq` that run() keeps for
 * Extras.plane_k (cpu.rs:336-361) and dA = dd_x(i) dd_y(j). The gradient is over the relative
 * permittivity and the conductivity of every cell of the design box (the Materials arrays),
 * exact for the f32 update as the device runs it (a discrete adjoint), from one forward run on the
 * fused step and one backward sweep. checkpoints = 0 keeps each step's E and curl term on the
 * design edges; checkpoints = c keeps the full field state at the start of about c segments and
 * re-runs each segment before sweeping it (sqrt(steps) checkpoints: segment recomputation).
 * The design box must stay off the grid boundary and off PEC, lumped, port and Debye edges; the
 * Sim may hold Debye media outside the design box (their ADE is transposed in the backward sweep
 * and carried by the checkpoints), but no inductors, thin wires or resistive sheets. */
typedef struct fg_flux_spec {
    uint64_t design_lo[3], design_hi[3];  /* design cells [lo, hi), cell indices as in Materials */
    uint64_t plane_k;                     /* node index of the flux plane along z */
    uint64_t window_lo[2], window_hi[2];  /* (i, j) nodes summed; window_hi {0, 0}: those inside the CPML */
    double freq;                          /* Hz */
    uint64_t steps;
    uint64_t checkpoints;
    int32_t precision;                    /* 0 or 32: the f32 update; 64: the objective alone from an FP64
                                             forward (f64 fields, psi, coefficients, pulse and DFT) */
    int32_t transposes;                   /* 0: each adjoint step one fused launch; 1: the E and H transposes
                                             as two launches (slower; the same sums, bit for bit) */
} fg_flux_spec;

typedef struct fg_flux_result {
    double objective, flux_re, flux_im;   /* J, and F */
    double forward_ms, recompute_ms, adjoint_ms;   /* the parts' device times (re-runs and sweeps overlap) */
    double backward_ms;                   /* the backward pass as a whole */
    double setup_ms;                      /* checks, device session, checkpoint and adjoint buffers */
    uint64_t segments, segment_len, design_edges;
} fg_flux_result;

/* grad_eps, grad_sigma: one entry per design cell, (i, j, k) order with k fastest; both NULL to
 * compute the objective alone. */
int fg_flux_gradient(fg_gpu* g, const fg_sim* sim, uint64_t driven, const fg_pulse* pulse,
                     const fg_flux_spec* spec, fg_flux_result* out, double* grad_eps, double* grad_sigma,
                     char* err, size_t errlen);

/* Many flux gradients on one GPU: no counterpart in the reference. count independent runs, each a
 * Sim with its own driven port, pulse and flux spec (precision 32), in groups of `group` runs (0:
 * 16) whose phases are enqueued together, each run on its own streams: the forwards, then each
 * objective as its forward ends, then the backward sweeps (the next group's set-up and forwards
 * overlap them). A group holds fewer runs when the free device memory would not hold the next. Each run's results (out[q], and the gradients over spec q's design cells in
 * grad_eps[q], grad_sigma[q]) are those of running it alone with fg_flux_gradient. The first
 * failing run ends the call; its error names the run. */
int fg_flux_gradient_batch(fg_gpu* g, const fg_sim* const* sims, const uint64_t* driven, const fg_pulse* pulses,
                           const fg_flux_spec* specs, uint64_t count, int group, fg_flux_result* out,
                           double* const* grad_eps, double* const* grad_sigma, char* err, size_t errlen);

/* ---- batches: many independent grids stepped together ----
 * No counterpart in the reference (it runs one Sim per run() call). Each grid is a Sim with its
 * own driven port and pulse; every step runs one persistent launch that marches the tiles of all
 * grids from a shared work-list (the direct-load fused march), then one launch each for all
 * grids' Debye edges, sources and port probes, captured in a CUDA graph; or (tile 3) one graph
 * branch per grid, each running that grid's own fused step on its stream, concurrently; or (tile 5)
 * one launch of the TMA march over every grid's clean box and one of each CPML shell kernel over
 * every grid's shell, then the shared Debye, source and probe launches. Each
 * grid's results are those of stepping it alone (fused step). Grids with thin wires or resistive
 * sheets, or that ask for a plane DFT or NTFF, are refused. With tune = 1 the batch times each
 * candidate (work-list tile 32x8, 64x4 or 32x4 with its persistent blocks per SM and x-planes per
 * work item, both kinds of graph branches and the merged launches) as a captured graph of a few steps, keeps the fastest and
 * resets every grid to step 0; with tune = 0 it uses the shape given. */
typedef struct fg_batch fg_batch;
typedef struct fg_batch_options {
    int tune;
    int tile;                /* work-list march 0: 32x8, 1: 64x4, 2: 32x4 (k x j); 3: graph branches;
                                4: graph branches, the grids of fewer than seg thousand nodes (all: seg 0)
                                with the direct-load march (one launch per grid-step); 5: merged TMA march
                                and shell launches over all grids */
    int blocks_per_sm;       /* 0: the occupancy limit */
    int seg;                 /* x-planes per work item; 0: 32 */
    int graph_steps;         /* steps per captured graph; 0: 10 */
} fg_batch_options;

int fg_batch_new(fg_gpu* g, const fg_sim* const* sims, const uint64_t* driven, const fg_pulse* pulses,
                 uint64_t count, uint64_t max_steps, const fg_batch_options* opt, fg_batch** out,
                 char* err, size_t errlen);
int fg_batch_step(fg_batch* b, uint64_t steps, char* err, size_t errlen);
int fg_batch_sync(fg_batch* b);
/* which: "series", "e" or "h" of grid `index` (as fg_session_read) */
int fg_batch_read(fg_batch* b, uint64_t index, const char* which, float* dst, uint64_t len, char* err, size_t errlen);
/* the shape in use (opt), the persistent launch's blocks, the tuned step time (ms) and steps taken */
int fg_batch_info(const fg_batch* b, fg_batch_options* opt, int* persistent_blocks, double* tuned_ms, uint64_t* steps);
void fg_batch_free(fg_batch* b);

/* ---- mesh -> grid rasterisation (crates/sims-field/src/raster.rs, bvh.rs) -----------------
 * Triangles are ntri x 3 vertices x 3 f64 (x, y, z). Masks are bytes, 1 = marked. The ray casts
 * and the sheet sweep run on the GPU in the reference's f64 arithmetic; g must be open. */
/* fill (raster.rs:24-104) over the sample lines s0 (n0), s1 (n1), s2 (n2): inside / thin get the
 * samples filled by ray parity / kept as thin skins (thin excludes inside), indexed over the
 * samples themselves in order 0 = (i n1 + j) n2 + k or 1 = i + (j + k n1) n0. */
int fg_raster_fill(fg_gpu* g, const double* tris, uint64_t ntri, const double* s0, uint64_t n0, const double* s1,
                   uint64_t n1, const double* s2, uint64_t n2, int order, uint8_t* inside, uint8_t* thin,
                   char* err, size_t errlen);
/* solid_edges (raster.rs:145-160): per component c, the E edges (node index (i ny + j) nz + k,
 * mask c * nx ny nz + node) whose midpoints the closed mesh holds, on the grid lines x, y, z. */
int fg_raster_solid_edges(fg_gpu* g, const double* tris, uint64_t ntri, const double* x, uint64_t nx,
                          const double* y, uint64_t ny, const double* z, uint64_t nz, uint8_t* mask,
                          char* err, size_t errlen);
/* solid_cells (raster.rs:162-173): the cells ((i (ny-1) + j) (nz-1) + k) whose centres the closed
 * mesh holds. */
int fg_raster_solid_cells(fg_gpu* g, const double* tris, uint64_t ntri, const double* x, uint64_t nx,
                          const double* y, uint64_t ny, const double* z, uint64_t nz, uint8_t* mask,
                          char* err, size_t errlen);
/* sheet_edges (raster.rs:186-264): per component, the E edges a triangle sheet passes through
 * (mask as fg_raster_solid_edges). */
int fg_raster_sheet_edges(fg_gpu* g, const double* tris, uint64_t ntri, const double* x, uint64_t nx,
                          const double* y, uint64_t ny, const double* z, uint64_t nz, uint8_t* mask,
                          char* err, size_t errlen);
/* closed (raster.rs:127-143): 1 when every edge of the mesh is shared by an even number of its
 * triangles, 0 otherwise (and for an empty mesh). Host code. */
int fg_raster_closed(const double* tris, uint64_t ntri);

#ifdef __cplusplus
}
#endif

#endif /* FIELDGRID_H */
