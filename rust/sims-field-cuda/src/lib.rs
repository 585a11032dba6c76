//! sims_field::fdtd on the B200 engine: `Sim::try_new`, `run` (the `Option<&Gpu>` entry of
//! run.rs:390-397), `patches`, `Far` and `backward` (the flux-objective adjoint, which the
//! reference does not have), over the C ABI of include/fieldgrid.h. The argument types are the
//! reference's own (sims_field::fdtd::{Materials, Lumped, PortDef, Resistive, Media, Pulse, Extras,
//! Record}), so a caller switches by changing the path of `run`. `None` for the GPU returns the
//! ABI's error: the engine has no CPU path.
mod ffi;

use ffi::*;
use sims_field::fdtd::{Element, Extras, Lumped, Materials, Media, PortDef, Pulse, Record, Resistive};
use sims_field::Grid;
use std::ffi::{CStr, CString};
use std::os::raw::{c_char, c_int, c_void};

fn err_text(buf: &[c_char]) -> String {
    unsafe { CStr::from_ptr(buf.as_ptr()) }.to_string_lossy().into_owned()
}

/// One CUDA device (gpu.rs:36-41's role).
pub struct Gpu { raw: *mut FgGpu }

impl Gpu {
    pub fn open(device: i32) -> Result<Gpu, String> {
        let mut raw = std::ptr::null_mut();
        let mut err = [0 as c_char; 1024];
        let rc = unsafe { fg_gpu_open(device, &mut raw, err.as_mut_ptr(), err.len()) };
        if rc != 0 { return Err(err_text(&err)); }
        Ok(Gpu { raw })
    }
}

impl Drop for Gpu {
    fn drop(&mut self) { unsafe { fg_gpu_close(self.raw) } }
}

/// The engine's Sim: the set-up of sim.rs:352-554 done by the library from the same inputs.
pub struct Sim { raw: *mut FgSim, pub grid: Grid }

impl Sim {
    /// Sim::try_new (sim.rs:352-361) with the reference's arguments and error texts.
    pub fn try_new(grid: Grid, mats: &Materials, pec: &dyn Fn(usize, [usize; 3]) -> bool, lumped: &[Lumped],
                   ports: Vec<PortDef>, resistive: &[Resistive], media: Media) -> Result<Sim, String> {
        let edge = |e: &sims_field::fdtd::Edge| FgEdge {
            comp: e.comp as u32, reserved: 0, at: [e.at[0] as u64, e.at[1] as u64, e.at[2] as u64],
        };
        let names: Vec<CString> = lumped.iter().map(|l| CString::new(l.name.clone()).unwrap_or_default())
            .chain(ports.iter().map(|p| CString::new(p.name.clone()).unwrap_or_default())).collect();
        let l_edges: Vec<Vec<FgEdge>> = lumped.iter().map(|l| l.edges.iter().map(edge).collect()).collect();
        let f_lumped: Vec<FgLumped> = lumped.iter().enumerate().map(|(q, l)| {
            let (element, value) = match l.element {
                Element::Resistor(v) => (FG_RESISTOR, v),
                Element::Capacitor(v) => (FG_CAPACITOR, v),
                Element::Inductor(v) => (FG_INDUCTOR, v),
            };
            FgLumped { name: names[q].as_ptr(), edges: l_edges[q].as_ptr(), n_edges: l_edges[q].len() as u64,
                       element, reserved: 0, value }
        }).collect();
        let p_edges: Vec<Vec<FgEdge>> = ports.iter().map(|p| p.columns.iter().flatten().map(edge).collect()).collect();
        let p_cols: Vec<Vec<u64>> = ports.iter().map(|p| p.columns.iter().map(|c| c.len() as u64).collect()).collect();
        let f_ports: Vec<FgPort> = ports.iter().enumerate().map(|(q, p)| FgPort {
            name: names[lumped.len() + q].as_ptr(), edges: p_edges[q].as_ptr(), column_len: p_cols[q].as_ptr(),
            n_columns: p_cols[q].len() as u64, r: p.r, reference_above: p.reference_above as i32, reserved: 0,
        }).collect();
        let f_res: Vec<FgResistive> = resistive.iter().map(|r| FgResistive {
            comp: r.comp as u32, adaptive: r.adaptive as i32, id: r.id as u64, r: r.r,
            faces: [r.faces[0] as u64, r.faces[1] as u64],
        }).collect();
        let poles: Vec<f64> = media.debye.poles.iter().flat_map(|&(x, a)| [x, a]).collect();
        let f_wires: Vec<FgWire> = media.wires.iter().map(|(e, r)| FgWire { edge: edge(e), radius: *r }).collect();
        unsafe extern "C" fn pec_tramp(user: *mut c_void, comp: u32, at: *const u64) -> c_int {
            let f = &*(user as *const &dyn Fn(usize, [usize; 3]) -> bool);
            let a = std::slice::from_raw_parts(at, 3);
            f(comp as usize, [a[0] as usize, a[1] as usize, a[2] as usize]) as c_int
        }
        let pec_ref: &dyn Fn(usize, [usize; 3]) -> bool = pec;
        let spec = FgSimSpec {
            x: grid.x.as_ptr(), nx: grid.x.len() as u64, y: grid.y.as_ptr(), ny: grid.y.len() as u64,
            z: grid.z.as_ptr(), nz: grid.z.len() as u64, pml: grid.pml as u64,
            eps: mats.eps.as_ptr(), sigma: mats.sigma.as_ptr(), inf: mats.inf.as_ptr(), debye: mats.debye.as_ptr(),
            pec_mask: std::ptr::null(), pec_fn: Some(pec_tramp), pec_user: &pec_ref as *const _ as *mut c_void,
            lumped: f_lumped.as_ptr(), n_lumped: f_lumped.len() as u64,
            ports: f_ports.as_ptr(), n_ports: f_ports.len() as u64,
            resistive: f_res.as_ptr(), n_resistive: f_res.len() as u64,
            sheet_table: media.sheets.table.as_ptr(), sheet_table_len: media.sheets.table.len() as u64,
            sheet_states: media.sheets.states as u64,
            debye_poles: poles.as_ptr(), n_debye_poles: media.debye.poles.len() as u64,
            wires: f_wires.as_ptr(), n_wires: f_wires.len() as u64,
        };
        let mut raw = std::ptr::null_mut();
        let mut err = [0 as c_char; 1024];
        let rc = unsafe { fg_sim_try_new(&spec, &mut raw, err.as_mut_ptr(), err.len()) };
        if rc != 0 { return Err(err_text(&err)); }
        Ok(Sim { raw, grid })
    }

    /// Sim::new (sim.rs:339-350): panics on error as the reference does.
    pub fn new(grid: Grid, mats: &Materials, pec: &dyn Fn(usize, [usize; 3]) -> bool, lumped: &[Lumped],
               ports: Vec<PortDef>, resistive: &[Resistive], media: Media) -> Sim {
        Sim::try_new(grid, mats, pec, lumped, ports, resistive, media).unwrap_or_else(|e| panic!("{e}"))
    }

    pub fn dt(&self) -> f64 { unsafe { fg_sim_dt(self.raw) } }
}

impl Drop for Sim {
    fn drop(&mut self) { unsafe { fg_sim_free(self.raw) } }
}

struct ExtrasFfi { x: FgExtras, _freqs: Vec<f64>, _ntff: Vec<u32> }

fn extras_ffi(e: &Extras) -> ExtrasFfi {
    let freqs = e.freqs.clone();
    let ntff = e.ntff.clone().unwrap_or_default();
    let x = FgExtras {
        min_steps: e.min_steps as u64, max_steps: e.max_steps as u64, decay_db: e.decay_db,
        freqs: freqs.as_ptr(), n_freqs: freqs.len() as u64,
        has_plane_k: e.plane_k.is_some() as i32, fused_e: e.fused_e as i32, plane_k: e.plane_k.unwrap_or(0) as u64,
        ntff: if e.ntff.is_some() { ntff.as_ptr() } else { std::ptr::null() }, ntff_len: ntff.len() as u64,
        check_every: e.check_every as u64, profile: e.profile as i32, keep_fields: 0,
    };
    ExtrasFfi { x, _freqs: freqs, _ntff: ntff }
}

fn copy_out(r: *const FgRecord, f: unsafe extern "C" fn(*const FgRecord, *mut u64) -> *const f32) -> Vec<f32> {
    let mut n = 0u64;
    let p = unsafe { f(r, &mut n) };
    if p.is_null() || n == 0 { return Vec::new(); }
    unsafe { std::slice::from_raw_parts(p, n as usize) }.to_vec()
}

/// run (run.rs:390-397) / run_blocking (run.rs:379-388) on the B200 engine.
pub fn run(g: Option<&Gpu>, sim: &Sim, driven: usize, pulse: &Pulse, extras: &Extras,
           progress: &mut dyn FnMut(usize, f64) -> bool) -> Result<Record, String> {
    unsafe extern "C" fn tramp(user: *mut c_void, steps: u64, decay: f64) -> c_int {
        let f = &mut *(user as *mut &mut dyn FnMut(usize, f64) -> bool);
        f(steps as usize, decay) as c_int
    }
    let mut cb: &mut dyn FnMut(usize, f64) -> bool = progress;
    let x = extras_ffi(extras);
    let p = FgPulse { f0: pulse.f0, fc: pulse.fc };
    let mut rec = std::ptr::null_mut();
    let mut err = [0 as c_char; 1024];
    let graw = g.map(|g| g.raw).unwrap_or(std::ptr::null_mut());
    let rc = unsafe {
        fg_run(graw, sim.raw, driven as u64, &p, &x.x, Some(tramp), &mut cb as *mut _ as *mut c_void, &mut rec,
               err.as_mut_ptr(), err.len())
    };
    if rc != 0 { return Err(err_text(&err)); }
    let out = Record {
        steps: unsafe { fg_record_steps(rec) } as usize,
        ports: unsafe { fg_record_ports(rec) } as usize,
        series: copy_out(rec, fg_record_series),
        decay_db: unsafe { fg_record_decay_db(rec) },
        plane: copy_out(rec, fg_record_plane),
        ntff: copy_out(rec, fg_record_ntff),
    };
    unsafe { fg_record_free(rec) };
    Ok(out)
}

/// patches (ntff.rs:11-59): the NTFF box `inset` cells inside the CPML.
pub fn patches(sim: &Sim, inset: usize) -> sims_field::fdtd::Patches {
    let mut count = 0u64;
    unsafe { fg_patches(sim.raw, inset as u64, std::ptr::null_mut(), std::ptr::null_mut(), std::ptr::null_mut(), &mut count) };
    let n = count as usize;
    let mut gpu = vec![0u32; 13 * n];
    let mut pos = vec![0f64; 3 * n];
    let mut area = vec![0f64; n];
    unsafe { fg_patches(sim.raw, inset as u64, gpu.as_mut_ptr(), pos.as_mut_ptr(), area.as_mut_ptr(), &mut count) };
    sims_field::fdtd::Patches { pos: pos.chunks(3).map(|c| [c[0], c[1], c[2]]).collect(), area, gpu }
}

/// The flux objective of a design box and its gradient (no counterpart in the reference): see
/// fg_flux_gradient in include/fieldgrid.h. Returns (J, dJ/deps_r, dJ/dsigma) over the design cells.
pub struct FluxSpec {
    pub design_lo: [usize; 3], pub design_hi: [usize; 3], pub plane_k: usize, pub freq: f64,
    pub steps: usize, pub checkpoints: usize,
}

pub fn backward(g: &Gpu, sim: &Sim, driven: usize, pulse: &Pulse, spec: &FluxSpec)
                -> Result<(f64, Vec<f64>, Vec<f64>), String> {
    let cells: usize = (0..3).map(|a| spec.design_hi[a] - spec.design_lo[a]).product();
    let s = FgFluxSpec {
        design_lo: spec.design_lo.map(|v| v as u64), design_hi: spec.design_hi.map(|v| v as u64),
        plane_k: spec.plane_k as u64, window_lo: [0, 0], window_hi: [0, 0], freq: spec.freq,
        steps: spec.steps as u64, checkpoints: spec.checkpoints as u64, precision: 32, transposes: 0,
    };
    let p = FgPulse { f0: pulse.f0, fc: pulse.fc };
    let mut out = FgFluxResult::default();
    let mut ge = vec![0f64; cells];
    let mut gs = vec![0f64; cells];
    let mut err = [0 as c_char; 1024];
    let rc = unsafe {
        fg_flux_gradient(g.raw, sim.raw, driven as u64, &p, &s, &mut out, ge.as_mut_ptr(), gs.as_mut_ptr(),
                         err.as_mut_ptr(), err.len())
    };
    if rc != 0 { return Err(err_text(&err)); }
    Ok((out.objective, ge, gs))
}
