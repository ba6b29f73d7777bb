//! Batched submissions (`fgfc_batch_*`): many stripes of uneven field, k, m
//! and shard length in one persistent launch per class, replayed as a CUDA
//! graph when the structure repeats. No reference counterpart.
use std::ptr;

use crate::device::{DeviceSlice, DeviceSliceMut, Stream};
use crate::ops::{CudaField, Plan};
use crate::{check, sys};

/// One stripe: the arguments of one dot_product_matrix_with (overwrite),
/// mul_add_matrix_with (accumulate) or, with `row_starts`, the scattered
/// forms.
pub struct Job<'a, F: CudaField> {
    pub plan: &'a Plan<F>,
    pub srcs: Vec<DeviceSlice<'a>>,
    pub dst: DeviceSliceMut<'a>,
    pub row_len: usize,
    pub nrows: usize,
    pub overwrite: bool,
    pub row_starts: Option<Vec<usize>>,
}

pub struct Batch {
    raw: *mut sys::fgfc_batch,
}

impl Batch {
    pub fn new() -> Self {
        let mut raw = ptr::null_mut();
        check(unsafe { sys::fgfc_batch_create(&mut raw) });
        Self { raw }
    }

    pub fn set_graphs(&mut self, enable: bool) {
        check(unsafe { sys::fgfc_batch_set_graphs(self.raw, enable as i32) });
    }

    /// Enqueue every job on `stream`; jobs must not write memory another job reads or writes.
    #[track_caller]
    pub fn run<F: CudaField>(&mut self, jobs: &mut [Job<'_, F>], stream: Stream) {
        let srcs = job_slices(jobs);
        let raws = raw_jobs(jobs, &srcs);
        check(unsafe { sys::fgfc_batch_run(self.raw, raws.as_ptr(), raws.len(), stream.0) });
    }

    /// `fgfc_tune_batch_tiles`: measure the work-list tile shapes on this
    /// submission (run repeatedly, so its jobs must be safe to rerun) and keep
    /// the fastest per class; returns the device time in microseconds with the
    /// starting and with the chosen tiles.
    #[track_caller]
    pub fn tune_tiles<F: CudaField>(&mut self, jobs: &mut [Job<'_, F>], stream: Stream) -> (f64, f64) {
        let srcs = job_slices(jobs);
        let raws = raw_jobs(jobs, &srcs);
        let (mut before, mut after) = (0.0, 0.0);
        check(unsafe {
            sys::fgfc_tune_batch_tiles(self.raw, raws.as_ptr(), raws.len(), stream.0, &mut before, &mut after)
        });
        (before, after)
    }
}

fn job_slices<F: CudaField>(jobs: &[Job<'_, F>]) -> Vec<Vec<sys::fgfc_slice>> {
    jobs.iter().map(|j| j.srcs.iter().map(|s| s.raw()).collect()).collect()
}

fn raw_jobs<F: CudaField>(jobs: &mut [Job<'_, F>], srcs: &[Vec<sys::fgfc_slice>]) -> Vec<sys::fgfc_matrix_job> {
    jobs.iter_mut()
        .zip(srcs)
        .map(|(j, s)| sys::fgfc_matrix_job {
            plan: j.plan.as_raw(),
            srcs: s.as_ptr(),
            nsrcs: s.len(),
            dst: j.dst.as_mut_ptr(),
            dst_len: j.dst.len(),
            row_starts: j.row_starts.as_ref().map_or(ptr::null(), |r| r.as_ptr()),
            nrows: j.nrows,
            row_len: j.row_len,
            overwrite: j.overwrite as i32,
        })
        .collect()
}

impl Default for Batch {
    fn default() -> Self {
        Self::new()
    }
}

impl Drop for Batch {
    fn drop(&mut self) {
        unsafe { sys::fgfc_batch_destroy(self.raw) };
    }
}
