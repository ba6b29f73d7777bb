//! Kernel-family choice (`fgfc_tune_*`): split-nibble tables, byte tables or
//! the tensor-core GF(2) contraction; all give the same bytes.
use std::ffi::CString;

use crate::ops::CudaField;
use crate::{check, sys};

#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub enum Kernel {
    Auto,
    Nibble,
    Byte,
    Gf2Mma,
}

impl Kernel {
    fn raw(self) -> sys::fgfc_kernel {
        match self {
            Kernel::Auto => sys::FGFC_KERNEL_AUTO,
            Kernel::Nibble => sys::FGFC_KERNEL_NIBBLE,
            Kernel::Byte => sys::FGFC_KERNEL_BYTE,
            Kernel::Gf2Mma => sys::FGFC_KERNEL_GF2MMA,
        }
    }
    fn from_raw(k: sys::fgfc_kernel) -> Self {
        match k {
            sys::FGFC_KERNEL_NIBBLE => Kernel::Nibble,
            sys::FGFC_KERNEL_BYTE => Kernel::Byte,
            sys::FGFC_KERNEL_GF2MMA => Kernel::Gf2Mma,
            _ => Kernel::Auto,
        }
    }
}

/// Process-wide override for A/B runs (Auto restores the tuned choice).
pub fn force(kernel: Kernel) {
    check(unsafe { sys::fgfc_tune_force(kernel.raw()) });
}

pub fn choice<F: CudaField>(nsrcs: usize, nrows: usize, row_len: usize) -> Kernel {
    Kernel::from_raw(unsafe { sys::fgfc_tune_choice(F::ID, nsrcs, nrows, row_len) })
}

/// Measure every usable family on this shape and record the winner.
pub fn tune_shape<F: CudaField>(nsrcs: usize, nrows: usize, row_len: usize) -> Kernel {
    let mut k = 0;
    check(unsafe { sys::fgfc_tune_shape(F::ID, nsrcs, nrows, row_len, &mut k) });
    Kernel::from_raw(k)
}

/// Element-vector columns per thread per work item of a batched
/// split-nibble class (`fgfc_tune_set_tile`: 1, 2, 4, 8 or 16; 0 = built-in).
pub fn set_tile(elem_bytes: usize, groups: usize, cols: u32) {
    check(unsafe { sys::fgfc_tune_set_tile(elem_bytes, groups, cols) });
}

pub fn tile(elem_bytes: usize, groups: usize) -> u32 {
    unsafe { sys::fgfc_tune_tile(elem_bytes, groups) }
}

pub fn save(path: &str) {
    let p = CString::new(path).expect("tune::save: path contains NUL");
    check(unsafe { sys::fgfc_tune_save(p.as_ptr()) });
}

pub fn load(path: &str) {
    let p = CString::new(path).expect("tune::load: path contains NUL");
    check(unsafe { sys::fgfc_tune_load(p.as_ptr()) });
}
