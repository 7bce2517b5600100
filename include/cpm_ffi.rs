// cpm_ffi.rs — Rust declarations of the C ABI in include/cpm.h, for the reference crate's
// `cuda` cargo feature: copy to src/cuda_ffi.rs (with `mod cuda_ffi;` in main.rs) and link
// libcpm_cuda.so from build.rs. Every `pub fn` here matches a declaration of include/cpm.h
// (same name, same parameter count; checked by tests/test_integration_decls.py).
#![cfg(feature = "cuda")]
use std::ffi::{c_char, c_int, c_void, CStr};

#[repr(C)] pub struct CpmCtx { _p: [u8; 0] }
#[repr(C)] pub struct CpmSim { _p: [u8; 0] }
#[repr(C)] #[derive(Clone, Copy)] pub struct CpmCosmology { pub omega_r: f32, pub omega_m: f32, pub omega_l: f32, pub h0: f32 }
#[repr(C)] #[derive(Clone, Copy)] pub struct CpmForceSplit { pub r_split: f32, pub r_cut: f32, pub softening: f32, pub theta: f32 }
#[repr(C)] pub struct CpmSimParams {
    pub cosmo: CpmCosmology, pub box_size: f32, pub mesh_n: c_int, pub n_particles: usize,
    pub use_tree: c_int, pub split: CpmForceSplit, pub flags: u32,
}

extern "C" {
    pub fn cpm_last_error(ctx: *const CpmCtx) -> *const c_char;
    pub fn cpm_ctx_create(n_mesh: c_int, box_size: f32, max_particles: usize, flags: u32, out: *mut *mut CpmCtx) -> c_int;
    pub fn cpm_ctx_destroy(ctx: *mut CpmCtx) -> c_int;
    pub fn cpm_mesh_deposit(ctx: *mut CpmCtx, x3: *const f32, n: usize, mass: f32, cells_out: *mut f32) -> c_int;
    pub fn cpm_mesh_interpolate(ctx: *mut CpmCtx, cells: *const f32, x3: *const f32, n: usize, out: *mut f32) -> c_int;
    pub fn cpm_mesh_interpolate3(ctx: *mut CpmCtx, gx: *const f32, gy: *const f32, gz: *const f32,
                                 x3: *const f32, n: usize, out3: *mut f32) -> c_int;
    pub fn cpm_fft3(ctx: *mut CpmCtx, data: *mut c_void, n: c_int, inverse: c_int) -> c_int;
    pub fn cpm_poisson_accel(ctx: *mut CpmCtx, delta: *const f32, n: c_int, cosmo: *const CpmCosmology, a: f32,
                             r_split: f32, gx: *mut f32, gy: *mut f32, gz: *mut f32) -> c_int;
    pub fn cpm_tree_accel(ctx: *mut CpmCtx, x3: *const f32, n: usize, box_size: f32, split: *const CpmForceSplit,
                          k: f32, acc3: *mut f32) -> c_int;
    pub fn cpm_sim_create(p: *const CpmSimParams, x3: *const f32, p3: *const f32, a0: f32, out: *mut *mut CpmSim) -> c_int;
    pub fn cpm_sim_step_host(sim: *mut CpmSim, a1: f32, x3: *mut f32, p3: *mut f32) -> c_int;
    pub fn cpm_sim_get_state(sim: *mut CpmSim, x3: *mut f32, p3: *mut f32, acc3: *mut f32, delta: *mut f32, a: *mut f32) -> c_int;
    pub fn cpm_sim_snapshot(sim: *mut CpmSim, speeds: *mut f32, densities: *mut f32, rsd3: *mut f32,
                            grid: *mut f32, grid_n: *mut c_int, max_speed: *mut f32) -> c_int;
    pub fn cpm_sim_power_spectrum(sim: *mut CpmSim, n_shells: c_int, k_mean: *mut f64, p_mean: *mut f64,
                                  counts: *mut u64) -> c_int;
    pub fn cpm_fft_supported(n: c_int) -> c_int;
    pub fn cpm_sim_destroy(sim: *mut CpmSim) -> c_int;
    // integrator.rs:117-126 `density_contrast`, fft.rs:86-95 `wavenumber`, tree.rs:40-57
    pub fn cpm_density_contrast(ctx: *mut CpmCtx, x3: *const f32, n: usize, delta_out: *mut f32) -> c_int;
    pub fn cpm_wavenumber(i: usize, n: usize, box_size: f32) -> f32;
    pub fn cpm_force_split_with(box_size: f32, mesh_n: usize, particles_per_side: usize, softening_scale: f32,
                                theta: f32) -> CpmForceSplit;
    pub fn cpm_short_range_factor(r: f32, r_split: f32) -> f32;
    // ics.rs:119-182 `zeldovich`, runner.rs:209-225 `init_simulation`, frame.rs:30-55 `downsample_grid`
    pub fn cpm_ics_zeldovich(n_side: c_int, box_size: f32, cosmo: *const CpmCosmology, n_s: f32, sigma8: f32,
                             a_init: f32, seed: u64, x3: *mut f32, p3: *mut f32) -> c_int;
    pub fn cpm_sim_create_zeldovich(p: *const CpmSimParams, n_side: c_int, n_s: f32, sigma8: f32, a0: f32,
                                    seed: u64, out: *mut *mut CpmSim) -> c_int;
    pub fn cpm_sim_set_state(sim: *mut CpmSim, x3: *const f32, p3: *const f32) -> c_int;
    pub fn cpm_density_grid(ctx: *mut CpmCtx, delta: *const f32, n: c_int, grid: *mut f32, grid_n: *mut c_int) -> c_int;
    // no counterpart in the reference: P(k) of particles (the estimator of the test ics.rs:213-266)
    pub fn cpm_power_spectrum(ctx: *mut CpmCtx, x3: *const f32, n: usize, n_shells: c_int, k_mean: *mut f64,
                              p_mean: *mut f64, counts: *mut u64) -> c_int;
}

pub const CPM_SIM_FIXED_POINT: u32 = 0x1;
pub const CPM_SIM_DECONVOLVE: u32 = 0x2;
pub const CPM_SIM_TIMING: u32 = 0x4;
pub const CPM_SIM_NO_GRAPH: u32 = 0x8;
pub const CPM_SIM_QUADRUPOLE: u32 = 0x10;
pub const CPM_SIM_NO_AUTOTUNE: u32 = 0x20;

/// The reference panics where the C ABI returns an error (e.g. poisson.rs:35); keep that.
pub fn check(rc: c_int, ctx: *const CpmCtx) {
    if rc != 0 {
        let msg = unsafe { CStr::from_ptr(cpm_last_error(ctx)) }.to_string_lossy();
        panic!("libcpm_cuda error {rc}: {msg}");
    }
}
