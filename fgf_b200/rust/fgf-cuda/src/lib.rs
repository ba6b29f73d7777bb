//! `fgf-cuda`: the packed-vector `ops` AXPY family of the `fgf` crate over
//! device buffers on NVIDIA B200 (sm_100a).
//!
//! Every function of `fgf::ops` (src/ops.rs:323-1017 of fgf 0.4.0) has a
//! counterpart in [`ops`] with the same name, argument order and panic
//! messages; byte slices become [`DeviceSlice`] / [`DeviceSliceMut`] and the
//! calls are enqueued on the calling thread's current [`Stream`]. Results are
//! bit-identical to `fgf::ops` on the same bytes. Underneath is the C ABI of
//! `libfgfcuda.so` ([`sys`], declared in include/fgf_cuda.h), which reports
//! errors as status codes; this crate turns them back into the reference's
//! panics.
//!
//! Beyond the reference: batched submissions ([`batch`]), coding and decode
//! matrices ([`codes`]), kernel-family choice ([`tune`]) and the serving loop
//! ([`serve`]).
#![deny(unsafe_op_in_unsafe_fn)]

pub mod batch;
pub mod codes;
mod device;
pub mod ops;
pub mod serve;
pub mod sys;
pub mod tune;

pub use device::{DeviceSlice, DeviceSliceMut, Stream};
pub use ops::{Coeff, CoeffRef, CudaField, Plan, PreparedCoefficient};

/// The library's message for the last failed call on this thread.
pub fn last_error() -> String {
    // SAFETY: fgfc_last_error returns a NUL-terminated thread-local string.
    unsafe { std::ffi::CStr::from_ptr(sys::fgfc_last_error()) }.to_string_lossy().into_owned()
}

/// Panics with the library's message unless `st` is FGFC_OK (the reference
/// panics on the same conditions with the same text).
#[track_caller]
pub(crate) fn check(st: sys::fgfc_status) {
    if st != sys::FGFC_OK {
        panic!("{}", last_error());
    }
}
