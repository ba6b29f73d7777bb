//! The serving loop (`fgfc_server_*`): continuous batching of matrix calls
//! over host or device buffers, a device plan cache keyed by matrix hash, an
//! HBM admission budget, page-locked staging and p50/p99 latency. No
//! reference counterpart.
use std::ptr;

use crate::{check, sys};

pub use crate::sys::{fgfc_request as Request, fgfc_rebuild_request as RebuildRequest,
                     fgfc_server_config as Config, fgfc_server_stats as Stats};

pub struct Server {
    raw: *mut sys::fgfc_server,
}

// SAFETY: the server's entry points are thread-safe.
unsafe impl Send for Server {}
unsafe impl Sync for Server {}

impl Server {
    #[track_caller]
    pub fn new(cfg: &Config) -> Self {
        let mut raw = ptr::null_mut();
        check(unsafe { sys::fgfc_server_create(cfg, &mut raw) });
        Self { raw }
    }

    /// # Safety
    /// The request's buffers must stay valid and untouched until it completes.
    #[track_caller]
    pub unsafe fn submit(&self, req: &Request) -> u64 {
        let mut t = 0;
        check(unsafe { sys::fgfc_server_submit(self.raw, req, &mut t) });
        t
    }

    /// # Safety
    /// As [`Server::submit`].
    #[track_caller]
    pub unsafe fn submit_rebuild(&self, req: &RebuildRequest) -> u64 {
        let mut t = 0;
        check(unsafe { sys::fgfc_server_submit_rebuild(self.raw, req, &mut t) });
        t
    }

    #[track_caller]
    pub fn wait(&self, ticket: u64) {
        check(unsafe { sys::fgfc_server_wait(self.raw, ticket) });
    }

    pub fn drain(&self) {
        check(unsafe { sys::fgfc_server_drain(self.raw) });
    }

    pub fn stats(&self, reset: bool) -> Stats {
        let mut s = Stats::default();
        check(unsafe { sys::fgfc_server_get_stats(self.raw, &mut s, reset as i32) });
        s
    }
}

impl Drop for Server {
    fn drop(&mut self) {
        unsafe { sys::fgfc_server_destroy(self.raw) };
    }
}
