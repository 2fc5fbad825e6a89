// ldsc_b200.rs -- Rust FFI declarations of the C ABI in ldsc_b200.h, for
// ldsc-rs (copy to src/b200.rs).  Struct field order and types follow the
// header one for one; the host test suite checks the field names against it.
use std::os::raw::{c_char, c_int, c_void};

#[repr(C)] pub struct LdscCtx { _p: [u8; 0] }
#[repr(C)] pub struct LdscPanel { _p: [u8; 0] }

#[repr(C)]
pub struct LdscProgress { pub chunks_done: u64, pub chunks_total: u64,
                          pub snps_done: u64, pub snps_total: u64, pub chunk_wall_ms: f64 }

#[repr(C)]
pub struct LdscPerf { pub m: u64, pub n_indiv: u64, pub bed_read_secs: f64, pub norm_secs: f64,
                      pub sketch_secs: f64, pub bb_dot_secs: f64, pub ab_dot_secs: f64,
                      pub ring_store_secs: f64, pub n_pairs: u64, pub n_tiles: u64,
                      pub kernel_launches: u32, pub gram_kind: u32, pub device_ms: f64,
                      pub contract_secs: f64, pub layout_secs: f64 }

#[repr(C)]
pub struct LdscL2Args {
    pub n_snp: u64, pub bed_idx: *const u64, pub chr: *const u8, pub cm: *const f64,
    pub bp: *const u32, pub window_mode: i32, pub window_size: f64, pub window_snps: u64,
    pub chunk_size: u32, pub global_pass: i32, pub snp_level_masking: i32, pub precision: i32,
    pub use_f32: i32, pub sketch_d: u32, pub sketch_maf_aware: i32,
    pub keep_iids: *const i64, pub n_keep: u64, pub annot: *const f64, pub n_annot: u32,
    pub has_pq_exp: i32, pub pq_exp: f64, pub yes_really: i32,
    pub on_progress: Option<extern "C" fn(*const LdscProgress, *mut c_void)>,
    pub progress_user: *mut c_void,
    // resident-panel extensions (zero = off)
    pub row_begin: u64, pub annot_on_device: i32, pub annot_ld: u64, pub out_on_device: i32,
}

#[repr(C)]
pub struct LdscH2Args { pub n_snp: u64, pub n_traits: u32, pub n_blocks: u32,
                        pub chi2: *const f64, pub n_per_snp: *const f64, pub n_scalar: *const f64,
                        pub ref_l2: *const f64, pub w_l2: *const f64, pub m_snps: f64,
                        pub fixed_intercept: i32, pub intercept: f64, pub want_lambda_gc: i32,
                        pub device_pointers: i32, pub two_step: i32, pub two_step_cutoff: f64 }
#[repr(C)]
pub struct LdscH2Result { pub h2: f64, pub h2_se: f64, pub intercept: f64, pub intercept_se: f64,
                          pub mean_chi2: f64, pub lambda_gc: f64, pub ratio: f64, pub ratio_se: f64,
                          pub coef: f64, pub coef_se: f64 }
#[repr(C)]
pub struct LdscRgArgs { pub n_snp: u64, pub n_pairs: u32, pub n_blocks: u32,
                        pub z1: *const f64, pub z2: *const f64, pub n1: *const f64, pub n2: *const f64,
                        pub ref_l2: *const f64, pub w_l2: *const f64, pub m_snps: f64,
                        pub device_pointers: i32 }
#[repr(C)]
pub struct LdscH2pArgs { pub n_snp: u64, pub n_traits: u32, pub n_annot: u32, pub n_blocks: u32,
                         pub chi2: *const f64, pub n_per_snp: *const f64, pub n_scalar: *const f64,
                         pub ref_l2: *const f64, pub ref_ld: u64, pub w_l2: *const f64,
                         pub m_vec: *const f64, pub fixed_intercept: i32, pub intercept: f64,
                         pub chisq_max: *const f64, pub device_pointers: i32,
                         pub est: *mut f64, pub cov: *mut f64, pub delete_values: *mut f64,
                         pub h2_annot: *mut f64 }
#[repr(C)]
pub struct LdscH2pResult { pub h2_total: f64, pub h2_total_se: f64, pub intercept: f64,
                           pub intercept_se: f64, pub n_mean: f64, pub mean_chi2: f64,
                           pub n_obs: u64, pub n_blocks: u32 }
#[repr(C)]
pub struct LdscRgResult { pub rg: f64, pub rg_se: f64, pub z: f64, pub p: f64, pub gencov: f64,
                          pub gencov_se: f64, pub gencov_intercept: f64, pub gencov_intercept_se: f64,
                          pub h2_1: f64, pub h2_1_se: f64, pub h2_2: f64, pub h2_2_se: f64,
                          pub mean_z1z2: f64 }

#[link(name = "ldsc_b200")]
extern "C" {
    pub fn ldsc_ctx_create(device: c_int, flags: u32, out: *mut *mut LdscCtx) -> c_int;
    pub fn ldsc_ctx_destroy(ctx: *mut LdscCtx) -> c_int;
    pub fn ldsc_last_error(ctx: *const LdscCtx, buf: *mut c_char, len: usize) -> c_int;
    pub fn ldsc_panel_upload(ctx: *mut LdscCtx, body: *const u8, bytes: u64, n_indiv: u64,
                             n_snp: u64, out: *mut *mut LdscPanel) -> c_int;
    pub fn ldsc_panel_destroy(p: *mut LdscPanel) -> c_int;
    pub fn ldsc_l2_run(ctx: *mut LdscCtx, p: *const LdscPanel, a: *const LdscL2Args,
                       l2_out: *mut f64, maf_out: *mut f64, perf: *mut LdscPerf) -> c_int;
    pub fn ldsc_l2_from_bed(ctx: *mut LdscCtx, bed: *const u8, len: u64, n_indiv: u64,
                            a: *const LdscL2Args, l2_out: *mut f64, maf_out: *mut f64,
                            perf: *mut LdscPerf) -> c_int;
    pub fn ldsc_h2_batch(ctx: *mut LdscCtx, a: *const LdscH2Args, out: *mut LdscH2Result) -> c_int;
    pub fn ldsc_rg_batch(ctx: *mut LdscCtx, a: *const LdscRgArgs, out: *mut LdscRgResult) -> c_int;
    pub fn ldsc_h2_partitioned(ctx: *mut LdscCtx, a: *const LdscH2pArgs, out: *mut LdscH2pResult) -> c_int;
    pub fn ldsc_l2_left_limits(a: *const LdscL2Args, left_out: *mut i64) -> c_int;
    pub fn ldsc_l2_workspace_bytes(a: *const LdscL2Args, n_indiv: u64, bytes: *mut u64) -> c_int;
    pub fn ldsc_l2_int8_noalloc(d_rows: *const u8, pitch: u64, n_indiv: u64, n_snp: u64,
                                left: *const i64, d_l2: *mut f64, d_maf: *mut f64,
                                stream: *mut c_void) -> c_int;
    pub fn ldsc_noalloc_last_error(buf: *mut c_char, len: usize) -> c_int;
}
