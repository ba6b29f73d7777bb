//! Coding and decode matrices for systematic codes [I_k ; C]
//! (`fgfc_cauchy_matrix`, `fgfc_decode_matrix`, `fgfc_decode_plan_create`).
//! The reference leaves these recipes to its callers (src/lib.rs:115-116);
//! inverses follow its inv(0) = 0 convention. The library's matrices are
//! 32-bit: the 8-byte fields are refused (their coefficient plans are built
//! from 64-bit values with `Plan::matrix`).
use std::ptr;

use crate::ops::{CudaField, Plan};
use crate::{check, sys};

/// Row-major m x k parity matrix c[i][j] = inv(x_i + y_j), x_i = x0 + i, y_j = j.
#[track_caller]
pub fn cauchy<F: CudaField>(m: usize, k: usize, x0: u32) -> Vec<F::Elem> {
    let mut out = vec![0u32; m * k];
    check(unsafe { sys::fgfc_cauchy_matrix(F::ID, m, k, x0, out.as_mut_ptr()) });
    out.into_iter().map(|v| F::from_raw(u64::from(v))).collect()
}

/// Decode rows (k x erased.len(), term-major) for rebuilding `erased` from the
/// k shards `survivors` of the code [I_k ; parity] (parity row-major m x k).
#[track_caller]
pub fn decode_matrix<F: CudaField>(parity: &[F::Elem], k: usize, survivors: &[usize], erased: &[usize]) -> Vec<F::Elem> {
    assert_eq!(survivors.len(), k, "decode_matrix: {} survivors for k = {k}", survivors.len());
    let m = parity.len() / k;
    let p: Vec<u32> = parity.iter().map(|&c| F::to_raw(c) as u32).collect();
    let mut out = vec![0u32; k * erased.len()];
    check(unsafe {
        sys::fgfc_decode_matrix(F::ID, p.as_ptr(), k, m, survivors.as_ptr(), erased.as_ptr(), erased.len(),
                                out.as_mut_ptr())
    });
    out.into_iter().map(|v| F::from_raw(u64::from(v))).collect()
}

/// The decode rows as a device plan of dimensions (k, erased.len()).
#[track_caller]
pub fn decode_plan<F: CudaField>(parity: &[F::Elem], k: usize, survivors: &[usize], erased: &[usize]) -> Plan<F> {
    assert_eq!(survivors.len(), k, "decode_plan: {} survivors for k = {k}", survivors.len());
    let m = parity.len() / k;
    let p: Vec<u32> = parity.iter().map(|&c| F::to_raw(c) as u32).collect();
    let mut raw = ptr::null_mut();
    check(unsafe {
        sys::fgfc_decode_plan_create(F::ID, p.as_ptr(), k, m, survivors.as_ptr(), erased.as_ptr(), erased.len(),
                                     &mut raw)
    });
    Plan::adopt(raw, k, erased.len())
}
