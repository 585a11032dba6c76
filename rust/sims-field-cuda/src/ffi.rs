//! Declarations matching include/fieldgrid.h (the C ABI of libfieldgrid.so), field for field.
#![allow(dead_code)]
use std::os::raw::{c_char, c_int, c_void};

#[repr(C)]
#[derive(Clone, Copy)]
pub struct FgEdge { pub comp: u32, pub reserved: u32, pub at: [u64; 3] }

pub const FG_RESISTOR: i32 = 0;
pub const FG_CAPACITOR: i32 = 1;
pub const FG_INDUCTOR: i32 = 2;

#[repr(C)]
pub struct FgLumped {
    pub name: *const c_char, pub edges: *const FgEdge, pub n_edges: u64,
    pub element: i32, pub reserved: i32, pub value: f64,
}

#[repr(C)]
pub struct FgPort {
    pub name: *const c_char, pub edges: *const FgEdge, pub column_len: *const u64, pub n_columns: u64,
    pub r: f64, pub reference_above: i32, pub reserved: i32,
}

#[repr(C)]
pub struct FgResistive { pub comp: u32, pub adaptive: i32, pub id: u64, pub r: f64, pub faces: [u64; 2] }

#[repr(C)]
pub struct FgWire { pub edge: FgEdge, pub radius: f64 }

pub type FgPecFn = Option<unsafe extern "C" fn(*mut c_void, u32, *const u64) -> c_int>;

#[repr(C)]
pub struct FgSimSpec {
    pub x: *const f64, pub nx: u64, pub y: *const f64, pub ny: u64, pub z: *const f64, pub nz: u64,
    pub pml: u64,
    pub eps: *const f32, pub sigma: *const f32, pub inf: *const f32, pub debye: *const f32,
    pub pec_mask: *const u8, pub pec_fn: FgPecFn, pub pec_user: *mut c_void,
    pub lumped: *const FgLumped, pub n_lumped: u64,
    pub ports: *const FgPort, pub n_ports: u64,
    pub resistive: *const FgResistive, pub n_resistive: u64,
    pub sheet_table: *const f32, pub sheet_table_len: u64, pub sheet_states: u64,
    pub debye_poles: *const f64, pub n_debye_poles: u64,
    pub wires: *const FgWire, pub n_wires: u64,
}

#[repr(C)]
pub struct FgPulse { pub f0: f64, pub fc: f64 }

#[repr(C)]
pub struct FgExtras {
    pub min_steps: u64, pub max_steps: u64, pub decay_db: f64,
    pub freqs: *const f64, pub n_freqs: u64,
    pub has_plane_k: i32, pub fused_e: i32, pub plane_k: u64,
    pub ntff: *const u32, pub ntff_len: u64,
    pub check_every: u64, pub profile: i32, pub keep_fields: i32,
}

#[repr(C)]
pub struct FgFluxSpec {
    pub design_lo: [u64; 3], pub design_hi: [u64; 3], pub plane_k: u64,
    pub window_lo: [u64; 2], pub window_hi: [u64; 2], pub freq: f64,
    pub steps: u64, pub checkpoints: u64, pub precision: i32, pub transposes: i32,
}

#[repr(C)]
#[derive(Default)]
pub struct FgFluxResult {
    pub objective: f64, pub flux_re: f64, pub flux_im: f64,
    pub forward_ms: f64, pub recompute_ms: f64, pub adjoint_ms: f64, pub backward_ms: f64, pub setup_ms: f64,
    pub segments: u64, pub segment_len: u64, pub design_edges: u64,
}

pub enum FgGpu {}
pub enum FgSim {}
pub enum FgRecord {}
pub enum FgFar {}

pub type FgProgress = Option<unsafe extern "C" fn(*mut c_void, u64, f64) -> c_int>;

extern "C" {
    pub fn fg_last_error() -> *const c_char;
    pub fn fg_gpu_open(device: c_int, out: *mut *mut FgGpu, err: *mut c_char, errlen: usize) -> c_int;
    pub fn fg_gpu_close(g: *mut FgGpu);
    pub fn fg_sim_try_new(spec: *const FgSimSpec, out: *mut *mut FgSim, err: *mut c_char, errlen: usize) -> c_int;
    pub fn fg_sim_free(s: *mut FgSim);
    pub fn fg_sim_dt(s: *const FgSim) -> f64;
    pub fn fg_sim_dims(s: *const FgSim, n: *mut u64);
    pub fn fg_run(g: *mut FgGpu, s: *const FgSim, driven: u64, p: *const FgPulse, x: *const FgExtras,
                  progress: FgProgress, user: *mut c_void, out: *mut *mut FgRecord,
                  err: *mut c_char, errlen: usize) -> c_int;
    pub fn fg_record_steps(r: *const FgRecord) -> u64;
    pub fn fg_record_ports(r: *const FgRecord) -> u64;
    pub fn fg_record_decay_db(r: *const FgRecord) -> f64;
    pub fn fg_record_series(r: *const FgRecord, len: *mut u64) -> *const f32;
    pub fn fg_record_plane(r: *const FgRecord, len: *mut u64) -> *const f32;
    pub fn fg_record_ntff(r: *const FgRecord, len: *mut u64) -> *const f32;
    pub fn fg_record_free(r: *mut FgRecord);
    pub fn fg_patches(s: *const FgSim, inset: u64, dst: *mut u32, pos: *mut f64, area: *mut f64,
                      count: *mut u64) -> c_int;
    pub fn fg_far_load(pos: *const f64, area: *const f64, count: u64, acc: *const f32, nf: u64, k: u64,
                       freq: f64, scale_re: f64, scale_im: f64, out: *mut *mut FgFar) -> c_int;
    pub fn fg_far_free(f: *mut FgFar);
    pub fn fg_far_field(g: *mut FgGpu, f: *const FgFar, dirs: *const f64, n: u64, out: *mut f64) -> c_int;
    pub fn fg_far_radiated(g: *mut FgGpu, f: *const FgFar, steps: u64, total: *mut f64, peak: *mut f64) -> c_int;
    pub fn fg_port_spectra(series: *const f32, steps: u64, ports: u64, port: u64, dt: f64, freqs: *const f64,
                           nf: u64, v: *mut f64, i: *mut f64) -> c_int;
    pub fn fg_flux_gradient(g: *mut FgGpu, s: *const FgSim, driven: u64, p: *const FgPulse,
                            spec: *const FgFluxSpec, out: *mut FgFluxResult, grad_eps: *mut f64,
                            grad_sigma: *mut f64, err: *mut c_char, errlen: usize) -> c_int;
}
