//! Raw bindings of include/fgf_cuda.h (libfgfcuda.so). Every call returns an
//! `fgfc_status`; `fgfc_last_error` holds the message of the last failure on
//! the calling thread.
#![allow(non_camel_case_types)]
use std::os::raw::{c_char, c_int, c_void};

pub type fgfc_stream = *mut c_void;
pub type fgfc_field = c_int;
pub type fgfc_status = c_int;
pub type fgfc_kernel = c_int;

pub const FGFC_GF8B: fgfc_field = 0;
pub const FGFC_GF8D: fgfc_field = 1;
pub const FGFC_GF16: fgfc_field = 2;
pub const FGFC_GF32: fgfc_field = 3;
pub const FGFC_FP8: fgfc_field = 4;
pub const FGFC_FP16: fgfc_field = 5;
pub const FGFC_FP32: fgfc_field = 6;
pub const FGFC_GF64: fgfc_field = 7;
pub const FGFC_FP64: fgfc_field = 8;

pub const FGFC_OK: fgfc_status = 0;
pub const FGFC_ERR_WIDTH: fgfc_status = 1;
pub const FGFC_ERR_LENGTH: fgfc_status = 2;
pub const FGFC_ERR_ROWS: fgfc_status = 3;
pub const FGFC_ERR_COEFFS: fgfc_status = 4;
pub const FGFC_ERR_SOURCE: fgfc_status = 5;
pub const FGFC_ERR_PLAN_DIMS: fgfc_status = 6;
pub const FGFC_ERR_OVERLAP: fgfc_status = 7;
pub const FGFC_ERR_BOUNDS: fgfc_status = 8;
pub const FGFC_ERR_ALIGN: fgfc_status = 9;
pub const FGFC_ERR_OVERFLOW: fgfc_status = 10;
pub const FGFC_ERR_ARG: fgfc_status = 11;
pub const FGFC_ERR_LIMIT: fgfc_status = 12;
pub const FGFC_ERR_CUDA: fgfc_status = 13;
pub const FGFC_ERR_NOMEM: fgfc_status = 14;

pub const FGFC_KERNEL_AUTO: fgfc_kernel = 0;
pub const FGFC_KERNEL_NIBBLE: fgfc_kernel = 1;
pub const FGFC_KERNEL_BYTE: fgfc_kernel = 2;
pub const FGFC_KERNEL_GF2MMA: fgfc_kernel = 3;

#[repr(C)]
pub struct fgfc_plan {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct fgfc_batch {
    _opaque: [u8; 0],
}
#[repr(C)]
pub struct fgfc_server {
    _opaque: [u8; 0],
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct fgfc_term {
    pub coeffs: *const u32,
    pub ncoeffs: usize,
    pub src: *const u8,
    pub src_len: usize,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct fgfc_slice {
    pub ptr: *const u8,
    pub len: usize,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct fgfc_matrix_job {
    pub plan: *const fgfc_plan,
    pub srcs: *const fgfc_slice,
    pub nsrcs: usize,
    pub dst: *mut u8,
    pub dst_len: usize,
    pub row_starts: *const usize,
    pub nrows: usize,
    pub row_len: usize,
    pub overwrite: c_int,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct fgfc_noalloc_job {
    pub coeffs: *const u32,
    pub srcs: *const fgfc_slice,
    pub nsrcs: usize,
    pub dst: *mut u8,
    pub dst_len: usize,
    pub row_starts: *const usize,
    pub nrows: usize,
    pub row_len: usize,
    pub overwrite: c_int,
}

#[repr(C)]
#[derive(Clone, Copy, Default)]
pub struct fgfc_server_config {
    pub hbm_budget: usize,
    pub staging_bytes: usize,
    pub max_batch: usize,
    pub max_inflight: usize,
    pub plan_cache: usize,
    pub max_launch_bytes: usize,
    pub plain: c_int,
    pub device: c_int,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct fgfc_request {
    pub field: fgfc_field,
    pub coeffs: *const u32,
    pub srcs: *const fgfc_slice,
    pub nsrcs: usize,
    pub dst: *mut u8,
    pub dst_len: usize,
    pub row_starts: *const usize,
    pub nrows: usize,
    pub row_len: usize,
    pub overwrite: c_int,
}

#[repr(C)]
#[derive(Clone, Copy)]
pub struct fgfc_rebuild_request {
    pub field: fgfc_field,
    pub parity: *const u32,
    pub k: usize,
    pub m: usize,
    pub survivors: *const usize,
    pub srcs: *const fgfc_slice,
    pub erased: *const usize,
    pub nerased: usize,
    pub dst: *mut u8,
    pub dst_len: usize,
    pub row_starts: *const usize,
    pub row_len: usize,
}

#[repr(C)]
#[derive(Clone, Copy, Default, Debug)]
pub struct fgfc_server_stats {
    pub completed: u64,
    pub failed: u64,
    pub launches: u64,
    pub plan_hits: u64,
    pub plan_misses: u64,
    pub source_bytes: u64,
    pub peak_device_bytes: u64,
    pub max_batch_seen: u64,
    pub p50_us: f64,
    pub p99_us: f64,
    pub mean_us: f64,
    pub max_us: f64,
    pub busy_s: f64,
    pub queue_us: f64,
    pub launch_us: f64,
}

pub const FGFC_NOALLOC_SCRATCH_BYTES: usize = 8 << 20;
pub const FGFC_NOALLOC_MAX_ROWS_GF8: usize = 16;

extern "C" {
    pub fn fgfc_last_error() -> *const c_char;
    pub fn fgfc_version() -> *const c_char;
    pub fn fgfc_limits(max_sources: *mut usize, max_rows: *mut usize);
    pub fn fgfc_field_bytes(field: fgfc_field) -> usize;
    pub fn fgfc_device_check(clear: c_int) -> fgfc_status;

    pub fn fgfc_plan_create(field: fgfc_field, rows: usize, cols: usize, coeffs: *const u32,
                            out: *mut *mut fgfc_plan) -> fgfc_status;
    pub fn fgfc_coeff_create(field: fgfc_field, coeff: u32, out: *mut *mut fgfc_plan) -> fgfc_status;
    pub fn fgfc_plan_create_u64(field: fgfc_field, rows: usize, cols: usize, coeffs: *const u64,
                                out: *mut *mut fgfc_plan) -> fgfc_status;
    pub fn fgfc_coeff_create_u64(field: fgfc_field, coeff: u64, out: *mut *mut fgfc_plan) -> fgfc_status;
    pub fn fgfc_plan_destroy(plan: *mut fgfc_plan);
    pub fn fgfc_plan_dimensions(plan: *const fgfc_plan, rows: *mut usize, cols: *mut usize) -> fgfc_status;
    pub fn fgfc_plan_len(plan: *const fgfc_plan) -> usize;
    pub fn fgfc_plan_field(plan: *const fgfc_plan) -> fgfc_field;
    pub fn fgfc_plan_values(plan: *const fgfc_plan, out: *mut u32) -> fgfc_status;
    pub fn fgfc_plan_get_at(plan: *const fgfc_plan, row: usize, col: usize, out: *mut u32) -> fgfc_status;
    pub fn fgfc_plan_values_u64(plan: *const fgfc_plan, out: *mut u64) -> fgfc_status;
    pub fn fgfc_plan_get_at_u64(plan: *const fgfc_plan, row: usize, col: usize, out: *mut u64) -> fgfc_status;

    pub fn fgfc_add_assign(field: fgfc_field, dst: *mut u8, dst_len: usize, src: *const u8, src_len: usize,
                           stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_add(field: fgfc_field, dst: *mut u8, dst_len: usize, coeff: u32, src: *const u8,
                        src_len: usize, stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_add_with(dst: *mut u8, dst_len: usize, coeff: *const fgfc_plan, src: *const u8,
                             src_len: usize, stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_into(field: fgfc_field, dst: *mut u8, dst_len: usize, coeff: u32, src: *const u8,
                         src_len: usize, stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_into_with(dst: *mut u8, dst_len: usize, coeff: *const fgfc_plan, src: *const u8,
                              src_len: usize, stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_assign(field: fgfc_field, dst: *mut u8, dst_len: usize, coeff: u32,
                           stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_assign_with(dst: *mut u8, dst_len: usize, coeff: *const fgfc_plan,
                                stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_elementwise(field: fgfc_field, dst: *mut u8, dst_len: usize, a: *const u8, a_len: usize,
                                b: *const u8, b_len: usize, stream: fgfc_stream) -> fgfc_status;

    pub fn fgfc_mul_add_scatter(field: fgfc_field, rows: *mut u8, rows_len: usize, row_len: usize,
                                coeffs: *const u32, ncoeffs: usize, src: *const u8, src_len: usize,
                                stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_add_scatter_with(rows: *mut u8, rows_len: usize, row_len: usize, plan: *const fgfc_plan,
                                     src: *const u8, src_len: usize, stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_add_gather(field: fgfc_field, dst: *mut u8, dst_len: usize, coeffs: *const u32,
                               ncoeffs: usize, srcs: *const fgfc_slice, nsrcs: usize,
                               stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_add_gather_with(dst: *mut u8, dst_len: usize, plan: *const fgfc_plan, srcs: *const fgfc_slice,
                                    nsrcs: usize, stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_dot_product(field: fgfc_field, dst: *mut u8, dst_len: usize, coeffs: *const u32, ncoeffs: usize,
                            srcs: *const fgfc_slice, nsrcs: usize, stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_dot_product_with(dst: *mut u8, dst_len: usize, plan: *const fgfc_plan, srcs: *const fgfc_slice,
                                 nsrcs: usize, stream: fgfc_stream) -> fgfc_status;

    pub fn fgfc_mul_add_matrix(field: fgfc_field, rows: *mut u8, rows_len: usize, row_len: usize, nrows: usize,
                               terms: *const fgfc_term, nterms: usize, stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_add_matrix_with(rows: *mut u8, rows_len: usize, row_len: usize, nrows: usize,
                                    plan: *const fgfc_plan, srcs: *const fgfc_slice, nsrcs: usize,
                                    stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_dot_product_matrix(field: fgfc_field, rows: *mut u8, rows_len: usize, row_len: usize,
                                   nrows: usize, terms: *const fgfc_term, nterms: usize,
                                   stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_dot_product_matrix_with(rows: *mut u8, rows_len: usize, row_len: usize, nrows: usize,
                                        plan: *const fgfc_plan, srcs: *const fgfc_slice, nsrcs: usize,
                                        stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_add_matrix_scattered(field: fgfc_field, dst: *mut u8, dst_len: usize, row_len: usize,
                                         row_starts: *const usize, nrows: usize, terms: *const fgfc_term,
                                         nterms: usize, stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_mul_add_matrix_scattered_with(dst: *mut u8, dst_len: usize, row_len: usize,
                                              row_starts: *const usize, nrows: usize, plan: *const fgfc_plan,
                                              srcs: *const fgfc_slice, nsrcs: usize,
                                              stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_dot_product_matrix_scattered_with(dst: *mut u8, dst_len: usize, row_len: usize,
                                                  row_starts: *const usize, nrows: usize,
                                                  plan: *const fgfc_plan, srcs: *const fgfc_slice, nsrcs: usize,
                                                  stream: fgfc_stream) -> fgfc_status;

    pub fn fgfc_cauchy_matrix(field: fgfc_field, m: usize, k: usize, x0: u32, out: *mut u32) -> fgfc_status;
    pub fn fgfc_decode_matrix(field: fgfc_field, parity: *const u32, k: usize, m: usize, survivors: *const usize,
                              erased: *const usize, nerased: usize, out: *mut u32) -> fgfc_status;
    pub fn fgfc_decode_plan_create(field: fgfc_field, parity: *const u32, k: usize, m: usize,
                                   survivors: *const usize, erased: *const usize, nerased: usize,
                                   out: *mut *mut fgfc_plan) -> fgfc_status;

    pub fn fgfc_batch_create(out: *mut *mut fgfc_batch) -> fgfc_status;
    pub fn fgfc_batch_destroy(batch: *mut fgfc_batch);
    pub fn fgfc_batch_set_graphs(batch: *mut fgfc_batch, enable: c_int) -> fgfc_status;
    pub fn fgfc_batch_run(batch: *mut fgfc_batch, jobs: *const fgfc_matrix_job, njobs: usize,
                          stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_batch_stats(batch: *const fgfc_batch, launches: *mut usize, items: *mut usize,
                            graph_replayed: *mut c_int) -> fgfc_status;
    pub fn fgfc_run_jobs_serial(jobs: *const fgfc_matrix_job, njobs: usize, stream: fgfc_stream) -> fgfc_status;
    pub fn fgfc_batch_run_noalloc(field: fgfc_field, jobs: *const fgfc_noalloc_job, njobs: usize,
                                  stream: fgfc_stream) -> fgfc_status;

    pub fn fgfc_tune_force(kernel: fgfc_kernel) -> fgfc_status;
    pub fn fgfc_tune_choice(field: fgfc_field, nsrcs: usize, nrows: usize, row_len: usize) -> fgfc_kernel;
    pub fn fgfc_tune_usable(kernel: fgfc_kernel, field: fgfc_field, nsrcs: usize, nrows: usize) -> c_int;
    pub fn fgfc_tune_shape(field: fgfc_field, nsrcs: usize, nrows: usize, row_len: usize,
                           out: *mut fgfc_kernel) -> fgfc_status;
    pub fn fgfc_tune_set_tile(elem_bytes: usize, groups: usize, cols: u32) -> fgfc_status;
    pub fn fgfc_tune_tile(elem_bytes: usize, groups: usize) -> u32;
    pub fn fgfc_tune_batch_tiles(batch: *mut fgfc_batch, jobs: *const fgfc_matrix_job, njobs: usize,
                                 stream: fgfc_stream, us_before: *mut f64, us_after: *mut f64) -> fgfc_status;
    pub fn fgfc_tune_save(path: *const c_char) -> fgfc_status;
    pub fn fgfc_tune_load(path: *const c_char) -> fgfc_status;
    pub fn fgfc_tune_clear();

    pub fn fgfc_server_create(cfg: *const fgfc_server_config, out: *mut *mut fgfc_server) -> fgfc_status;
    pub fn fgfc_server_submit(server: *mut fgfc_server, req: *const fgfc_request, ticket: *mut u64) -> fgfc_status;
    pub fn fgfc_server_submit_rebuild(server: *mut fgfc_server, req: *const fgfc_rebuild_request,
                                      ticket: *mut u64) -> fgfc_status;
    pub fn fgfc_server_wait(server: *mut fgfc_server, ticket: u64) -> fgfc_status;
    pub fn fgfc_server_poll(server: *mut fgfc_server, ticket: u64, done: *mut c_int) -> fgfc_status;
    pub fn fgfc_server_drain(server: *mut fgfc_server) -> fgfc_status;
    pub fn fgfc_server_get_stats(server: *mut fgfc_server, out: *mut fgfc_server_stats, reset: c_int) -> fgfc_status;
    pub fn fgfc_server_destroy(server: *mut fgfc_server);
}
