//! Rust binding of the B200 Barnes-Hut engine (`libgalaxy_bh.so`, C ABI in
//! `include/galaxy_bh.h`).
//!
//! The reference's host drives its Barnes-Hut evolution through
//! `NbodyGpu` (runtime/src/nbody_gpu.rs:312-1114) and `ParallelTreeRuntime`
//! (runtime/src/nbody_parallel.rs:93-993) over wgpu.  This crate exposes the
//! same steps with the same method names over the CUDA engine: `ffi` is the
//! raw `extern "C"` block (one declaration per header function), and
//! `Device`, `EvolvingState`, `ParallelTree`, `Batch` and `Server` are safe
//! owners that free their handle on Drop, as the reference's structs do.
//! Records keep the frozen layouts of nbody_gpu.rs:22-83 byte for byte, so a
//! caller holding the reference's `bytemuck::Pod` records can pass them
//! through `bytemuck::cast_slice` unchanged.
//!
//! Errors carry the engine's status code and its thread-local message, the
//! counterpart of the reference's `Result<_, String>` texts.
#![allow(non_camel_case_types)]

use std::marker::PhantomData;
use std::os::raw::{c_char, c_int};

pub const NO_CHILD: u32 = 0xffff_ffff;
pub const FLAG_COMPENSATED: u32 = 1;
pub const FLAG_POTENTIAL: u32 = 2;
pub const FLAG_NO_STATS: u32 = 4;

// ---- frozen transfer records (nbody_gpu.rs:22-83) -------------------------

/// nbody_gpu.rs:24-27: info = body_count, cell_count, root_index, reserved;
/// physics = theta, softening, G, reserved.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct BhSettings {
    pub info: [u32; 4],
    pub physics: [f32; 4],
}

/// nbody_gpu.rs:31-34: x, y, mass, reserved | Morton position, reserved x3.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct GpuBody {
    pub position_mass: [f32; 4],
    pub meta: [u32; 4],
}

/// nbody_gpu.rs:38-40: Morton code, body index, 0, 0.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct GpuEntry {
    pub data: [u32; 4],
}

/// nbody_gpu.rs:44-49.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct GpuCell {
    pub center_half_mass: [f32; 4],
    pub com: [f32; 4],
    pub range_depth: [u32; 4],
    pub children: [u32; 4],
}

/// nbody_gpu.rs:53-55: ax, ay, 0, 0.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct GpuAccel {
    pub value: [f32; 4],
}

/// nbody_gpu.rs:66-69: x, y, mass, reserved | vx, vy, reserved x2.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct GpuEvolveState {
    pub position_mass: [f32; 4],
    pub velocity: [f32; 4],
}

/// nbody_gpu.rs:80-83 (data = cell_count, body_count, max_depth, flags).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct TreeMeta {
    pub data: [u32; 4],
    pub bounds: [f32; 4],
}

// ---- configuration, timings, counters ------------------------------------

/// Config of nbody/src/lib.rs:27-67 plus engine flags (FLAG_*).
#[repr(C)]
#[derive(Clone, Copy, Debug, PartialEq)]
pub struct BhConfig {
    pub theta: f64,
    pub softening: f64,
    pub g: f64,
    pub bucket: u32,
    pub max_depth: u32,
    pub flags: u32,
    pub reserved: u32,
}

/// StageTiming of nbody_gpu.rs:125-130 (seconds).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct BhStageTiming {
    pub transfer_seconds: f64,
    pub dispatch_seconds: f64,
    pub readback_seconds: f64,
}

/// ParallelTreeBuildTiming of nbody_parallel.rs:45-53 (seconds).
#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct BhBuildTiming {
    pub bounds_seconds: f64,
    pub morton_seconds: f64,
    pub radix_seconds: f64,
    pub positions_seconds: f64,
    pub topology_seconds: f64,
    pub aggregate_seconds: f64,
}

/// ForceStats of nbody/src/lib.rs:102-107 plus two engine counters.
#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct BhForceStats {
    pub visited_nodes: u64,
    pub approximated_cells: u64,
    pub direct_terms: u64,
    pub exact_mac_fallbacks: u64,
    pub warp_iterations: u64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, PartialEq)]
pub struct BhTuning {
    pub radix_bits: u32,
    pub traverse_warps: u32,
    pub reserved: [u32; 2],
}

#[repr(C)]
#[derive(Clone, Copy, Debug, PartialEq)]
pub struct BhServeConfig {
    pub budget_bytes: u64,
    pub round_steps: u32,
    pub max_members: u32,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct BhServeResult {
    pub request_id: u64,
    pub n: u32,
    pub status: u32,
    pub steps: u32,
    pub reserved: u32,
    pub submitted_s: f64,
    pub admitted_s: f64,
    pub finished_s: f64,
}

#[repr(C)]
#[derive(Clone, Copy, Debug, Default, PartialEq)]
pub struct BhServeStats {
    pub rounds: u64,
    pub particle_steps: u64,
    pub completed: u64,
    pub busy_seconds: f64,
    pub elapsed_seconds: f64,
    pub admit_seconds: f64,
    pub solve_seconds: f64,
    pub form_seconds: f64,
    pub readback_seconds: f64,
}

/// The raw C ABI, one declaration per function of include/galaxy_bh.h.
pub mod ffi {
    use super::{BhBuildTiming, BhConfig, BhForceStats, BhServeConfig, BhServeResult,
                BhServeStats, BhSettings, BhStageTiming, BhTuning, GpuAccel, GpuBody, GpuCell,
                GpuEntry, GpuEvolveState, TreeMeta};
    use std::ffi::c_void;
    use std::os::raw::{c_char, c_int};

    #[repr(C)]
    pub struct bh_device {
        _private: [u8; 0],
    }
    #[repr(C)]
    pub struct bh_state {
        _private: [u8; 0],
    }
    #[repr(C)]
    pub struct bh_tree {
        _private: [u8; 0],
    }
    #[repr(C)]
    pub struct bh_batch {
        _private: [u8; 0],
    }
    #[repr(C)]
    pub struct bh_server {
        _private: [u8; 0],
    }

    extern "C" {
        pub fn galaxy_bh_last_error(buf: *mut c_char, len: usize) -> usize;
        pub fn galaxy_bh_wait_probe(dev: *mut bh_device, spin_cycles: u64) -> c_int;
        pub fn galaxy_bh_abi_version() -> u32;
        pub fn galaxy_bh_device_open(ordinal: c_int, out: *mut *mut bh_device) -> c_int;
        pub fn galaxy_bh_device_close(dev: *mut bh_device) -> c_int;
        pub fn galaxy_bh_device_info(dev: *mut bh_device, buf: *mut c_char, len: usize) -> c_int;
        pub fn galaxy_bh_device_stream(dev: *mut bh_device, stream: *mut *mut c_void) -> c_int;
        pub fn galaxy_bh_state_create(dev: *mut bh_device, host: *const GpuEvolveState, n: u32,
                                      out: *mut *mut bh_state, timing: *mut BhStageTiming)
                                      -> c_int;
        pub fn galaxy_bh_state_destroy(st: *mut bh_state) -> c_int;
        pub fn galaxy_bh_state_count(st: *mut bh_state, n: *mut u32) -> c_int;
        pub fn galaxy_bh_state_bytes(st: *mut bh_state, bytes: *mut u64) -> c_int;
        pub fn galaxy_bh_kick_drift(dev: *mut bh_device, st: *mut bh_state, dt: f64,
                                    timing: *mut BhStageTiming) -> c_int;
        pub fn galaxy_bh_final_kick(dev: *mut bh_device, st: *mut bh_state, dt: f64,
                                    timing: *mut BhStageTiming) -> c_int;
        pub fn galaxy_bh_final_kick_drift(dev: *mut bh_device, st: *mut bh_state, dt: f64,
                                          timing: *mut BhStageTiming) -> c_int;
        pub fn galaxy_bh_read_state(dev: *mut bh_device, st: *mut bh_state,
                                    out: *mut GpuEvolveState, n: u32,
                                    timing: *mut BhStageTiming) -> c_int;
        pub fn galaxy_bh_read_accel(dev: *mut bh_device, st: *mut bh_state, out: *mut GpuAccel,
                                    n: u32, timing: *mut BhStageTiming) -> c_int;
        pub fn galaxy_bh_write_state(dev: *mut bh_device, st: *mut bh_state,
                                     host: *const GpuEvolveState, n: u32) -> c_int;
        pub fn galaxy_bh_tree_create(dev: *mut bh_device, st: *mut bh_state, cfg: *const BhConfig,
                                     out: *mut *mut bh_tree) -> c_int;
        pub fn galaxy_bh_tree_destroy(tree: *mut bh_tree) -> c_int;
        pub fn galaxy_bh_tree_rebuild(dev: *mut bh_device, st: *mut bh_state, tree: *mut bh_tree,
                                      cfg: *const BhConfig, timing: *mut BhBuildTiming) -> c_int;
        pub fn galaxy_bh_force(dev: *mut bh_device, st: *mut bh_state, tree: *mut bh_tree,
                               cfg: *const BhConfig, timing: *mut BhStageTiming) -> c_int;
        pub fn galaxy_bh_force_stats(dev: *mut bh_device, tree: *mut bh_tree,
                                     out: *mut BhForceStats) -> c_int;
        pub fn galaxy_bh_force_f64(dev: *mut bh_device, st: *mut bh_state, tree: *mut bh_tree,
                                   cfg: *const BhConfig, accel: *mut f64, abs_sum: *mut f64,
                                   stats: *mut BhForceStats) -> c_int;
        pub fn galaxy_bh_read_tree_evidence(dev: *mut bh_device, tree: *mut bh_tree,
                                            meta: *mut TreeMeta, entries: *mut GpuEntry,
                                            bodies: *mut GpuBody, n: u32, cells: *mut GpuCell,
                                            cell_capacity: u32, cell_count: *mut u32) -> c_int;
        pub fn galaxy_bh_tree_buffer_bytes(tree: *mut bh_tree, bytes: *mut u64) -> c_int;
        pub fn galaxy_bh_tree_footprint(n: u32, cfg: *const BhConfig, bytes: *mut u64) -> c_int;
        pub fn galaxy_bh_traverse_packed(dev: *mut bh_device, settings: *const BhSettings,
                                         bodies: *const GpuBody, n: u32,
                                         entries: *const GpuEntry, cells: *const GpuCell,
                                         cell_count: u32, out: *mut GpuAccel,
                                         timing: *mut BhStageTiming) -> c_int;
        pub fn galaxy_bh_force_into(dev: *mut bh_device, st: *mut bh_state,
                                    settings: *const BhSettings, bodies: *const GpuBody,
                                    entries: *const GpuEntry, cells: *const GpuCell,
                                    cell_count: u32, timing: *mut BhStageTiming) -> c_int;
        pub fn galaxy_bh_step(dev: *mut bh_device, st: *mut bh_state, tree: *mut bh_tree,
                              cfg: *const BhConfig, dt: f64, nsteps: u32) -> c_int;
        pub fn galaxy_bh_direct_probes(dev: *mut bh_device, st: *mut bh_state,
                                       cfg: *const BhConfig, probes: *const u32, nprobes: u32,
                                       out: *mut f64) -> c_int;
        pub fn galaxy_bh_conservation(dev: *mut bh_device, st: *mut bh_state,
                                      out: *mut f64) -> c_int;
        pub fn galaxy_bh_conservation_noalloc(state: *const GpuEvolveState,
                                              potential: *const f32, n: u32, sums: *mut f64,
                                              stream: *mut c_void) -> c_int;
        pub fn galaxy_bh_batch_create(dev: *mut bh_device, states: *const *mut bh_state,
                                      cfgs: *const BhConfig, count: u32,
                                      out: *mut *mut bh_batch) -> c_int;
        pub fn galaxy_bh_batch_destroy(batch: *mut bh_batch) -> c_int;
        pub fn galaxy_bh_batch_solve(dev: *mut bh_device, batch: *mut bh_batch) -> c_int;
        pub fn galaxy_bh_batch_step(dev: *mut bh_device, batch: *mut bh_batch, dts: *const f64,
                                    nsteps: u32) -> c_int;
        pub fn galaxy_bh_batch_bytes(batch: *mut bh_batch, bytes: *mut u64) -> c_int;
        pub fn galaxy_bh_serve_start(ordinal: c_int, config: *const BhServeConfig,
                                     out: *mut *mut bh_server) -> c_int;
        pub fn galaxy_bh_serve_submit(server: *mut bh_server, host: *const GpuEvolveState,
                                      n: u32, cfg: *const BhConfig, dt: f64, steps: u32,
                                      request_id: *mut u64) -> c_int;
        pub fn galaxy_bh_serve_poll(server: *mut bh_server, timeout_ms: u32,
                                    result: *mut BhServeResult, out: *mut GpuEvolveState,
                                    capacity: u32) -> c_int;
        pub fn galaxy_bh_serve_stats(server: *mut bh_server, out: *mut BhServeStats) -> c_int;
        pub fn galaxy_bh_serve_stop(server: *mut bh_server) -> c_int;
        pub fn galaxy_bh_batch_tune(batch: *mut bh_batch, tuning: *const BhTuning) -> c_int;
        pub fn galaxy_bh_tree_tune(tree: *mut bh_tree, tuning: *const BhTuning) -> c_int;
        pub fn galaxy_bh_batch_footprint(counts: *const u32, cfgs: *const BhConfig, count: u32,
                                         bytes: *mut u64) -> c_int;
    }
}

// ---- errors ----------------------------------------------------------------

/// A failed call: the bh_status code and the engine's message.
#[derive(Clone, Debug, PartialEq)]
pub struct Error {
    pub status: i32,
    pub message: String,
}

impl std::fmt::Display for Error {
    fn fmt(&self, f: &mut std::fmt::Formatter<'_>) -> std::fmt::Result {
        write!(f, "{} (status {})", self.message, self.status)
    }
}

impl std::error::Error for Error {}

pub type Result<T> = std::result::Result<T, Error>;

fn check(rc: c_int) -> Result<()> {
    if rc == 0 {
        return Ok(());
    }
    let mut buf = vec![0u8; 1024];
    let len = unsafe { ffi::galaxy_bh_last_error(buf.as_mut_ptr() as *mut c_char, buf.len()) };
    buf.truncate(len.min(1023));
    Err(Error { status: rc, message: String::from_utf8_lossy(&buf).into_owned() })
}

fn count_u32(len: usize, what: &str) -> Result<u32> {
    u32::try_from(len).map_err(|_| Error {
        status: 1,
        message: format!("{what} count does not fit u32"),
    })
}

// ---- safe owners -------------------------------------------------------------

/// NbodyGpu::new (nbody_gpu.rs:331) and ParallelTreeRuntime::new
/// (nbody_parallel.rs:156): one CUDA device and its stream.
pub struct Device {
    raw: *mut ffi::bh_device,
}

/// An evolving state resident on the device (nbody_gpu.rs:786).
pub struct EvolvingState<'d> {
    raw: *mut ffi::bh_state,
    count: u32,
    _dev: PhantomData<&'d Device>,
}

/// A GPU-built tree of one evolving state (nbody_parallel.rs:361).
pub struct ParallelTree<'d> {
    raw: *mut ffi::bh_tree,
    _dev: PhantomData<&'d Device>,
}

/// The tree evidence of nbody_parallel.rs:929-988 (cells in CPU preorder).
pub struct TreeEvidence {
    pub meta: TreeMeta,
    pub entries: Vec<GpuEntry>,
    pub bodies: Vec<GpuBody>,
    pub cells: Vec<GpuCell>,
}

/// Many independent simulations advanced with one launch per stage.
pub struct Batch<'d> {
    raw: *mut ffi::bh_batch,
    _dev: PhantomData<&'d Device>,
}

impl Device {
    pub fn new(ordinal: i32) -> Result<Self> {
        let mut raw = std::ptr::null_mut();
        check(unsafe { ffi::galaxy_bh_device_open(ordinal, &mut raw) })?;
        Ok(Self { raw })
    }

    /// NbodyGpu::info (nbody_gpu.rs:298-310): a JSON adapter description.
    pub fn info(&self) -> Result<String> {
        let mut buf = vec![0u8; 4096];
        check(unsafe {
            ffi::galaxy_bh_device_info(self.raw, buf.as_mut_ptr() as *mut c_char, buf.len())
        })?;
        let end = buf.iter().position(|&b| b == 0).unwrap_or(buf.len());
        Ok(String::from_utf8_lossy(&buf[..end]).into_owned())
    }

    pub fn create_evolving_state(&self, records: &[GpuEvolveState])
                                 -> Result<(EvolvingState<'_>, BhStageTiming)> {
        let n = count_u32(records.len(), "body")?;
        let mut raw = std::ptr::null_mut();
        let mut t = BhStageTiming::default();
        check(unsafe {
            ffi::galaxy_bh_state_create(self.raw, records.as_ptr(), n, &mut raw, &mut t)
        })?;
        Ok((EvolvingState { raw, count: n, _dev: PhantomData }, t))
    }

    pub fn kick_drift(&self, s: &EvolvingState<'_>, dt: f64) -> Result<BhStageTiming> {
        let mut t = BhStageTiming::default();
        check(unsafe { ffi::galaxy_bh_kick_drift(self.raw, s.raw, dt, &mut t) })?;
        Ok(t)
    }

    pub fn final_kick(&self, s: &EvolvingState<'_>, dt: f64) -> Result<BhStageTiming> {
        let mut t = BhStageTiming::default();
        check(unsafe { ffi::galaxy_bh_final_kick(self.raw, s.raw, dt, &mut t) })?;
        Ok(t)
    }

    /// final_kick then kick_drift in one pass (bit-identical to the two calls).
    pub fn final_kick_drift(&self, s: &EvolvingState<'_>, dt: f64) -> Result<BhStageTiming> {
        let mut t = BhStageTiming::default();
        check(unsafe { ffi::galaxy_bh_final_kick_drift(self.raw, s.raw, dt, &mut t) })?;
        Ok(t)
    }

    pub fn read_evolving_state(&self, s: &EvolvingState<'_>)
                               -> Result<(Vec<GpuEvolveState>, BhStageTiming)> {
        let mut out = vec![GpuEvolveState::default(); s.count as usize];
        let mut t = BhStageTiming::default();
        check(unsafe {
            ffi::galaxy_bh_read_state(self.raw, s.raw, out.as_mut_ptr(), s.count, &mut t)
        })?;
        Ok((out, t))
    }

    pub fn read_evolving_accelerations(&self, s: &EvolvingState<'_>)
                                       -> Result<(Vec<GpuAccel>, BhStageTiming)> {
        let mut out = vec![GpuAccel::default(); s.count as usize];
        let mut t = BhStageTiming::default();
        check(unsafe {
            ffi::galaxy_bh_read_accel(self.raw, s.raw, out.as_mut_ptr(), s.count, &mut t)
        })?;
        Ok((out, t))
    }

    pub fn write_evolving_state(&self, s: &EvolvingState<'_>, records: &[GpuEvolveState])
                                -> Result<()> {
        let n = count_u32(records.len(), "body")?;
        check(unsafe { ffi::galaxy_bh_write_state(self.raw, s.raw, records.as_ptr(), n) })
    }

    /// NbodyGpu::traverse (nbody_gpu.rs:640-780) over a packed flat tree.
    pub fn traverse(&self, settings: &BhSettings, bodies: &[GpuBody], entries: &[GpuEntry],
                    cells: &[GpuCell]) -> Result<(Vec<GpuAccel>, BhStageTiming)> {
        let n = count_u32(bodies.len(), "body")?;
        let nc = count_u32(cells.len(), "cell")?;
        let mut out = vec![GpuAccel::default(); bodies.len()];
        let mut t = BhStageTiming::default();
        check(unsafe {
            ffi::galaxy_bh_traverse_packed(self.raw, settings, bodies.as_ptr(), n,
                                           entries.as_ptr(), cells.as_ptr(), nc,
                                           out.as_mut_ptr(), &mut t)
        })?;
        Ok((out, t))
    }

    /// NbodyGpu::force_into (nbody_gpu.rs:854-938).
    pub fn force_into(&self, s: &EvolvingState<'_>, settings: &BhSettings, bodies: &[GpuBody],
                      entries: &[GpuEntry], cells: &[GpuCell]) -> Result<BhStageTiming> {
        let nc = count_u32(cells.len(), "cell")?;
        let mut t = BhStageTiming::default();
        check(unsafe {
            ffi::galaxy_bh_force_into(self.raw, s.raw, settings, bodies.as_ptr(),
                                      entries.as_ptr(), cells.as_ptr(), nc, &mut t)
        })?;
        Ok(t)
    }

    /// FP64 direct accelerations of probe bodies (lib.rs:315-329).
    pub fn direct_probes(&self, s: &EvolvingState<'_>, cfg: &BhConfig, probes: &[u32])
                         -> Result<Vec<[f64; 2]>> {
        let k = count_u32(probes.len(), "probe")?;
        let mut out = vec![[0.0f64; 2]; probes.len()];
        check(unsafe {
            ffi::galaxy_bh_direct_probes(self.raw, s.raw, cfg, probes.as_ptr(), k,
                                         out.as_mut_ptr() as *mut f64)
        })?;
        Ok(out)
    }

    /// FP64 invariants: mass, com_x, com_y, px, py, lz, kinetic, potential,
    /// sum m|v|, total energy.
    pub fn conservation(&self, s: &EvolvingState<'_>) -> Result<[f64; 10]> {
        let mut out = [0.0f64; 10];
        check(unsafe { ffi::galaxy_bh_conservation(self.raw, s.raw, out.as_mut_ptr()) })?;
        Ok(out)
    }

    /// ParallelTreeRuntime::create_tree (nbody_parallel.rs:361-493).
    pub fn create_tree(&self, s: &EvolvingState<'_>, cfg: &BhConfig) -> Result<ParallelTree<'_>> {
        let mut raw = std::ptr::null_mut();
        check(unsafe { ffi::galaxy_bh_tree_create(self.raw, s.raw, cfg, &mut raw) })?;
        Ok(ParallelTree { raw, _dev: PhantomData })
    }

    /// ParallelTreeRuntime::rebuild (nbody_parallel.rs:555-826).
    pub fn rebuild(&self, s: &EvolvingState<'_>, tree: &ParallelTree<'_>, cfg: &BhConfig)
                   -> Result<BhBuildTiming> {
        let mut t = BhBuildTiming::default();
        check(unsafe { ffi::galaxy_bh_tree_rebuild(self.raw, s.raw, tree.raw, cfg, &mut t) })?;
        Ok(t)
    }

    /// ParallelTreeRuntime::force (nbody_parallel.rs:828-897).
    pub fn force(&self, s: &EvolvingState<'_>, tree: &ParallelTree<'_>, cfg: &BhConfig)
                 -> Result<BhStageTiming> {
        let mut t = BhStageTiming::default();
        check(unsafe { ffi::galaxy_bh_force(self.raw, s.raw, tree.raw, cfg, &mut t) })?;
        Ok(t)
    }

    pub fn force_stats(&self, tree: &ParallelTree<'_>) -> Result<BhForceStats> {
        let mut out = BhForceStats::default();
        check(unsafe { ffi::galaxy_bh_force_stats(self.raw, tree.raw, &mut out) })?;
        Ok(out)
    }

    /// flat_accelerations_from_tree (flat.rs:270-371) in f64 on the device:
    /// (ax, ay) per body and the sum of each body's term magnitudes.
    pub fn force_f64(&self, s: &EvolvingState<'_>, tree: &ParallelTree<'_>, cfg: &BhConfig)
                     -> Result<(Vec<[f64; 2]>, Vec<f64>, BhForceStats)> {
        let mut acc = vec![[0.0f64; 2]; s.count as usize];
        let mut abs_sum = vec![0.0f64; s.count as usize];
        let mut st = BhForceStats::default();
        check(unsafe {
            ffi::galaxy_bh_force_f64(self.raw, s.raw, tree.raw, cfg,
                                     acc.as_mut_ptr() as *mut f64, abs_sum.as_mut_ptr(),
                                     &mut st)
        })?;
        Ok((acc, abs_sum, st))
    }

    /// ParallelTreeRuntime::read_evidence (nbody_parallel.rs:929-988).
    pub fn read_evidence(&self, tree: &ParallelTree<'_>, n: u32) -> Result<TreeEvidence> {
        let mut meta = TreeMeta::default();
        let mut count = 0u32;
        check(unsafe {
            ffi::galaxy_bh_read_tree_evidence(self.raw, tree.raw, &mut meta,
                                              std::ptr::null_mut(), std::ptr::null_mut(), 0,
                                              std::ptr::null_mut(), 0, &mut count)
        })?;
        let mut entries = vec![GpuEntry::default(); n as usize];
        let mut bodies = vec![GpuBody::default(); n as usize];
        let mut cells = vec![GpuCell::default(); count as usize];
        check(unsafe {
            ffi::galaxy_bh_read_tree_evidence(self.raw, tree.raw, &mut meta, entries.as_mut_ptr(),
                                              bodies.as_mut_ptr(), n, cells.as_mut_ptr(), count,
                                              &mut count)
        })?;
        Ok(TreeEvidence { meta, entries, bodies, cells })
    }

    /// The reference loop (galaxy-bh-gpu-tree-parallel.rs:345-350) fused:
    /// nsteps KDK steps; rebuild + force must have run once.
    pub fn step(&self, s: &EvolvingState<'_>, tree: &ParallelTree<'_>, cfg: &BhConfig, dt: f64,
                nsteps: u32) -> Result<()> {
        check(unsafe { ffi::galaxy_bh_step(self.raw, s.raw, tree.raw, cfg, dt, nsteps) })
    }

    pub fn create_batch(&self, states: &[&EvolvingState<'_>], cfgs: &[BhConfig])
                        -> Result<Batch<'_>> {
        if states.len() != cfgs.len() {
            return Err(Error { status: 1, message: "one config per state".into() });
        }
        let raws: Vec<*mut ffi::bh_state> = states.iter().map(|s| s.raw).collect();
        let count = count_u32(raws.len(), "state")?;
        let mut raw = std::ptr::null_mut();
        check(unsafe {
            ffi::galaxy_bh_batch_create(self.raw, raws.as_ptr(), cfgs.as_ptr(), count, &mut raw)
        })?;
        Ok(Batch { raw, _dev: PhantomData })
    }

    pub fn batch_solve(&self, batch: &Batch<'_>) -> Result<()> {
        check(unsafe { ffi::galaxy_bh_batch_solve(self.raw, batch.raw) })
    }

    pub fn batch_step(&self, batch: &Batch<'_>, dts: &[f64], nsteps: u32) -> Result<()> {
        check(unsafe { ffi::galaxy_bh_batch_step(self.raw, batch.raw, dts.as_ptr(), nsteps) })
    }
}

impl Drop for Device {
    fn drop(&mut self) {
        unsafe { ffi::galaxy_bh_device_close(self.raw) };
    }
}

impl EvolvingState<'_> {
    pub fn count(&self) -> u32 {
        self.count
    }

    /// NbodyGpu::evolving_buffer_bytes (nbody_gpu.rs:1116).
    pub fn buffer_bytes(&self) -> Result<u64> {
        let mut v = 0u64;
        check(unsafe { ffi::galaxy_bh_state_bytes(self.raw, &mut v) })?;
        Ok(v)
    }
}

impl Drop for EvolvingState<'_> {
    fn drop(&mut self) {
        unsafe { ffi::galaxy_bh_state_destroy(self.raw) };
    }
}

impl ParallelTree<'_> {
    /// ParallelTreeRuntime::buffer_bytes (nbody_parallel.rs:990-992).
    pub fn buffer_bytes(&self) -> Result<u64> {
        let mut v = 0u64;
        check(unsafe { ffi::galaxy_bh_tree_buffer_bytes(self.raw, &mut v) })?;
        Ok(v)
    }

    pub fn tune(&self, tuning: &BhTuning) -> Result<()> {
        check(unsafe { ffi::galaxy_bh_tree_tune(self.raw, tuning) })
    }
}

impl Drop for ParallelTree<'_> {
    fn drop(&mut self) {
        unsafe { ffi::galaxy_bh_tree_destroy(self.raw) };
    }
}

impl Batch<'_> {
    pub fn bytes(&self) -> Result<u64> {
        let mut v = 0u64;
        check(unsafe { ffi::galaxy_bh_batch_bytes(self.raw, &mut v) })?;
        Ok(v)
    }

    pub fn tune(&self, tuning: &BhTuning) -> Result<()> {
        check(unsafe { ffi::galaxy_bh_batch_tune(self.raw, tuning) })
    }
}

impl Drop for Batch<'_> {
    fn drop(&mut self) {
        unsafe { ffi::galaxy_bh_batch_destroy(self.raw) };
    }
}

/// The continuous-batching server (no counterpart in the reference).
pub struct Server {
    raw: *mut ffi::bh_server,
}

// The server's submit/poll/stats are documented as callable from any thread.
unsafe impl Send for Server {}
unsafe impl Sync for Server {}

impl Server {
    pub fn start(ordinal: i32, config: &BhServeConfig) -> Result<Self> {
        let mut raw = std::ptr::null_mut();
        check(unsafe { ffi::galaxy_bh_serve_start(ordinal, config, &mut raw) })?;
        Ok(Self { raw })
    }

    pub fn submit(&self, records: &[GpuEvolveState], cfg: &BhConfig, dt: f64, steps: u32)
                  -> Result<u64> {
        let n = count_u32(records.len(), "body")?;
        let mut id = 0u64;
        check(unsafe {
            ffi::galaxy_bh_serve_submit(self.raw, records.as_ptr(), n, cfg, dt, steps, &mut id)
        })?;
        Ok(id)
    }

    /// Waits up to timeout_ms for a finished request; Ok(None) on timeout.
    pub fn poll(&self, timeout_ms: u32, out: &mut Vec<GpuEvolveState>)
                -> Result<Option<BhServeResult>> {
        let mut r = BhServeResult::default();
        let cap = count_u32(out.len(), "body")?;
        let rc = unsafe {
            ffi::galaxy_bh_serve_poll(self.raw, timeout_ms, &mut r, out.as_mut_ptr(), cap)
        };
        if rc == 5 {
            return Ok(None); // BH_TIMEOUT: nothing finished yet
        }
        if rc == 1 && r.n as usize > out.len() {
            // the result needs more room; it stays queued
            out.resize(r.n as usize, GpuEvolveState::default());
            return self.poll(timeout_ms, out);
        }
        check(rc)?;
        out.truncate(r.n as usize);
        Ok(Some(r))
    }

    pub fn stats(&self) -> Result<BhServeStats> {
        let mut s = BhServeStats::default();
        check(unsafe { ffi::galaxy_bh_serve_stats(self.raw, &mut s) })?;
        Ok(s)
    }
}

impl Drop for Server {
    fn drop(&mut self) {
        unsafe { ffi::galaxy_bh_serve_stop(self.raw) };
    }
}

/// Device bytes a tree of n bodies under cfg needs (the receipt validator's
/// tree-buffer formula for this engine).
pub fn tree_footprint(n: u32, cfg: &BhConfig) -> Result<u64> {
    let mut v = 0u64;
    check(unsafe { ffi::galaxy_bh_tree_footprint(n, cfg, &mut v) })?;
    Ok(v)
}

pub fn batch_footprint(counts: &[u32], cfgs: &[BhConfig]) -> Result<u64> {
    let count = count_u32(counts.len(), "state")?;
    let mut v = 0u64;
    check(unsafe { ffi::galaxy_bh_batch_footprint(counts.as_ptr(), cfgs.as_ptr(), count, &mut v) })?;
    Ok(v)
}

pub fn abi_version() -> u32 {
    unsafe { ffi::galaxy_bh_abi_version() }
}

#[cfg(test)]
mod tests {
    use super::*;

    #[test]
    fn record_sizes_match_the_frozen_layouts() {
        assert_eq!(std::mem::size_of::<BhSettings>(), 32);
        assert_eq!(std::mem::size_of::<GpuBody>(), 32);
        assert_eq!(std::mem::size_of::<GpuEntry>(), 16);
        assert_eq!(std::mem::size_of::<GpuCell>(), 64);
        assert_eq!(std::mem::size_of::<GpuAccel>(), 16);
        assert_eq!(std::mem::size_of::<GpuEvolveState>(), 32);
        assert_eq!(std::mem::size_of::<TreeMeta>(), 32);
        assert_eq!(std::mem::size_of::<BhConfig>(), 40);
        assert_eq!(std::mem::size_of::<BhServeResult>(), 48);
    }
}
