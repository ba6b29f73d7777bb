//! The `fgf::ops` surface over device buffers (fgf 0.4.0, src/ops.rs).
//!
//! Same function names, argument order and meaning as the reference; `&[u8]`
//! becomes [`DeviceSlice`], `&mut [u8]` becomes [`DeviceSliceMut`], and each
//! call is enqueued on the thread's current [`Stream`] (stream-ordered,
//! asynchronous). The library validates exactly what the reference asserts and
//! these wrappers panic with the same messages (e.g. "mul_add: dst is 8 bytes
//! but src is 4 bytes").
use std::marker::PhantomData;
use std::ptr;

use fgf::fan_paar::{fp16, fp32, fp64, fp8, FanPaar16, FanPaar32, FanPaar64, FanPaar8};
use fgf::field::{gf16, gf32, gf64, gf8b, gf8d, Field, Gf16, Gf32, Gf64, Gf8B, Gf8D};

use crate::device::{DeviceSlice, DeviceSliceMut, Stream};
use crate::{check, sys};

/// A field the device library implements: its ABI code and element <-> u64.
/// `WIDE` marks the 8-byte fields, whose 64-bit coefficients reach the
/// library only through plans (the raw entry points take 32-bit values).
pub trait CudaField: Field {
    const ID: sys::fgfc_field;
    const WIDE: bool = false;
    fn to_raw(e: Self::Elem) -> u64;
    fn from_raw(v: u64) -> Self::Elem;
}

impl CudaField for Gf8B {
    const ID: sys::fgfc_field = sys::FGFC_GF8B;
    fn to_raw(e: gf8b::Elem) -> u64 {
        u64::from(e.0)
    }
    fn from_raw(v: u64) -> gf8b::Elem {
        gf8b::Elem(v as u8)
    }
}

impl CudaField for Gf8D {
    const ID: sys::fgfc_field = sys::FGFC_GF8D;
    fn to_raw(e: gf8d::Elem) -> u64 {
        u64::from(e.0)
    }
    fn from_raw(v: u64) -> gf8d::Elem {
        gf8d::Elem(v as u8)
    }
}

impl CudaField for Gf16 {
    const ID: sys::fgfc_field = sys::FGFC_GF16;
    fn to_raw(e: gf16::Elem) -> u64 {
        u64::from(e.0)
    }
    fn from_raw(v: u64) -> gf16::Elem {
        gf16::Elem(v as u16)
    }
}

impl CudaField for Gf32 {
    const ID: sys::fgfc_field = sys::FGFC_GF32;
    fn to_raw(e: gf32::Elem) -> u64 {
        u64::from(e.0)
    }
    fn from_raw(v: u64) -> gf32::Elem {
        gf32::Elem(v as u32)
    }
}

impl CudaField for FanPaar8 {
    const ID: sys::fgfc_field = sys::FGFC_FP8;
    fn to_raw(e: fp8::Elem) -> u64 {
        u64::from(e.0)
    }
    fn from_raw(v: u64) -> fp8::Elem {
        fp8::Elem(v as u8)
    }
}

impl CudaField for FanPaar16 {
    const ID: sys::fgfc_field = sys::FGFC_FP16;
    fn to_raw(e: fp16::Elem) -> u64 {
        u64::from(e.0)
    }
    fn from_raw(v: u64) -> fp16::Elem {
        fp16::Elem(v as u16)
    }
}

impl CudaField for FanPaar32 {
    const ID: sys::fgfc_field = sys::FGFC_FP32;
    fn to_raw(e: fp32::Elem) -> u64 {
        u64::from(e.0)
    }
    fn from_raw(v: u64) -> fp32::Elem {
        fp32::Elem(v as u32)
    }
}

impl CudaField for Gf64 {
    const ID: sys::fgfc_field = sys::FGFC_GF64;
    const WIDE: bool = true;
    fn to_raw(e: gf64::Elem) -> u64 {
        e.0
    }
    fn from_raw(v: u64) -> gf64::Elem {
        gf64::Elem(v)
    }
}

impl CudaField for FanPaar64 {
    const ID: sys::fgfc_field = sys::FGFC_FP64;
    const WIDE: bool = true;
    fn to_raw(e: fp64::Elem) -> u64 {
        e.0
    }
    fn from_raw(v: u64) -> fp64::Elem {
        fp64::Elem(v)
    }
}

/// 32-bit coefficients for the raw entry points (every field but the 8-byte
/// ones, whose raw forms below go through a plan).
fn raw<F: CudaField>(coeffs: &[F::Elem]) -> Vec<u32> {
    coeffs.iter().map(|&c| F::to_raw(c) as u32).collect()
}

fn stream() -> sys::fgfc_stream {
    Stream::current().0
}

fn slices(srcs: &[DeviceSlice<'_>]) -> Vec<sys::fgfc_slice> {
    srcs.iter().map(|s| s.raw()).collect()
}

// ---------------------------------------------------------------- plans

/// `ops::Plan<F>` (src/ops.rs:158-276): coefficients prepared once, with
/// their product tables (and, where the shape allows, the GF(2) bit matrix of
/// the tensor-core kernel) uploaded to the device. A matrix plan has one row
/// per source term and one column per destination row.
pub struct Plan<F: CudaField> {
    raw: *mut sys::fgfc_plan,
    values: Vec<F::Elem>,
    rows: usize,
    cols: usize,
    _f: PhantomData<F>,
}

// SAFETY: the library's plans are immutable after creation and usable from
// any host thread.
unsafe impl<F: CudaField> Send for Plan<F> {}
unsafe impl<F: CudaField> Sync for Plan<F> {}

impl<F: CudaField> Plan<F> {
    /// `Plan::new` (src/ops.rs:176-190): a one-row plan.
    pub fn new(coeffs: &[F::Elem]) -> Self {
        Self::matrix(1, coeffs.len(), coeffs)
    }

    /// `Plan::matrix` (src/ops.rs:198-212).
    #[track_caller]
    pub fn matrix(rows: usize, cols: usize, coeffs: &[F::Elem]) -> Self {
        let expected = rows.checked_mul(cols).expect("Plan::matrix: dimensions overflow");
        assert_eq!(coeffs.len(), expected, "Plan::matrix: {} coefficients for {rows}x{cols} matrix", coeffs.len());
        let v: Vec<u64> = coeffs.iter().map(|&c| F::to_raw(c)).collect();
        let mut p = ptr::null_mut();
        // SAFETY: v holds rows * cols values; p receives a new plan.
        check(unsafe { sys::fgfc_plan_create_u64(F::ID, rows, cols, v.as_ptr(), &mut p) });
        Self { raw: p, values: coeffs.to_vec(), rows, cols, _f: PhantomData }
    }

    pub(crate) fn adopt(raw: *mut sys::fgfc_plan, rows: usize, cols: usize) -> Self {
        let mut v = vec![0u64; rows * cols];
        // SAFETY: the plan holds rows * cols values.
        check(unsafe { sys::fgfc_plan_values_u64(raw, v.as_mut_ptr()) });
        Self { raw, values: v.into_iter().map(F::from_raw).collect(), rows, cols, _f: PhantomData }
    }

    pub fn len(&self) -> usize {
        self.values.len()
    }
    pub fn is_empty(&self) -> bool {
        self.values.is_empty()
    }
    pub fn dimensions(&self) -> (usize, usize) {
        (self.rows, self.cols)
    }
    pub fn get(&self, index: usize) -> Option<CoeffRef<'_, F>> {
        (index < self.values.len()).then(|| CoeffRef { plan: self, index })
    }
    pub fn get_at(&self, row: usize, col: usize) -> Option<CoeffRef<'_, F>> {
        (row < self.rows && col < self.cols).then(|| CoeffRef { plan: self, index: row * self.cols + col })
    }
    pub fn coeffs(&self) -> impl ExactSizeIterator<Item = CoeffRef<'_, F>> {
        (0..self.values.len()).map(move |index| CoeffRef { plan: self, index })
    }
    pub fn row(&self, row: usize) -> Option<impl ExactSizeIterator<Item = CoeffRef<'_, F>> + '_> {
        (row < self.rows).then(move || (row * self.cols..(row + 1) * self.cols).map(move |index| CoeffRef { plan: self, index }))
    }
    pub fn values(&self) -> impl ExactSizeIterator<Item = F::Elem> + '_ {
        self.values.iter().copied()
    }
    pub fn as_raw(&self) -> *const sys::fgfc_plan {
        self.raw
    }
}

impl<F: CudaField> Drop for Plan<F> {
    fn drop(&mut self) {
        // SAFETY: the plan was created by the library and is dropped once.
        unsafe { sys::fgfc_plan_destroy(self.raw) };
    }
}

/// `ops::Coeff<F>` (src/ops.rs:44-73): one prepared coefficient.
pub struct Coeff<F: CudaField> {
    plan: Plan<F>,
}

impl<F: CudaField> Coeff<F> {
    pub fn new(coeff: F::Elem) -> Self {
        Self { plan: Plan::new(&[coeff]) }
    }
    pub fn value(&self) -> F::Elem {
        self.plan.values[0]
    }
}

/// `ops::CoeffRef` (src/ops.rs:127-156): a borrowed entry of a plan.
#[derive(Clone, Copy)]
pub struct CoeffRef<'a, F: CudaField> {
    plan: &'a Plan<F>,
    index: usize,
}

impl<F: CudaField> CoeffRef<'_, F> {
    pub fn value(self) -> F::Elem {
        self.plan.values[self.index]
    }
}

/// `ops::PreparedCoefficient` (src/ops.rs:98-156): a [`Coeff`], or an entry of
/// a [`Plan`] (a one-entry plan is used as is; another entry is prepared as
/// a one-coefficient plan on use).
pub trait PreparedCoefficient<F: CudaField> {
    fn value(&self) -> F::Elem;
    #[doc(hidden)]
    fn with_plan<R>(&self, f: impl FnOnce(*const sys::fgfc_plan) -> R) -> R;
}

impl<F: CudaField> PreparedCoefficient<F> for Coeff<F> {
    fn value(&self) -> F::Elem {
        Coeff::value(self)
    }
    fn with_plan<R>(&self, f: impl FnOnce(*const sys::fgfc_plan) -> R) -> R {
        f(self.plan.raw)
    }
}

impl<F: CudaField> PreparedCoefficient<F> for CoeffRef<'_, F> {
    fn value(&self) -> F::Elem {
        CoeffRef::value(*self)
    }
    fn with_plan<R>(&self, f: impl FnOnce(*const sys::fgfc_plan) -> R) -> R {
        if self.plan.len() == 1 {
            f(self.plan.raw)
        } else {
            let one = Plan::<F>::new(&[CoeffRef::value(*self)]);
            f(one.raw)
        }
    }
}

// ---------------------------------------------------------------- single row

/// `ops::add_assign` (src/ops.rs:323): `dst ^= src`.
#[track_caller]
pub fn add_assign<F: CudaField>(dst: &mut DeviceSliceMut<'_>, src: &DeviceSlice<'_>) {
    // SAFETY: device ranges valid per DeviceSlice's contract.
    check(unsafe { sys::fgfc_add_assign(F::ID, dst.as_mut_ptr(), dst.len(), src.as_ptr(), src.len(), stream()) });
}

/// `ops::sub_assign` (src/ops.rs:333): the same as add_assign in characteristic 2.
#[track_caller]
pub fn sub_assign<F: CudaField>(dst: &mut DeviceSliceMut<'_>, src: &DeviceSlice<'_>) {
    add_assign::<F>(dst, src)
}

/// `ops::mul_add` (src/ops.rs:342): `dst ^= coeff * src`.
#[track_caller]
pub fn mul_add<F: CudaField>(dst: &mut DeviceSliceMut<'_>, coeff: F::Elem, src: &DeviceSlice<'_>) {
    if F::WIDE {
        return mul_add_with(dst, &Coeff::<F>::new(coeff), src);
    }
    check(unsafe {
        sys::fgfc_mul_add(F::ID, dst.as_mut_ptr(), dst.len(), F::to_raw(coeff) as u32, src.as_ptr(), src.len(), stream())
    });
}

/// `ops::mul_add_with` (src/ops.rs:359).
#[track_caller]
pub fn mul_add_with<F: CudaField>(dst: &mut DeviceSliceMut<'_>, coeff: &impl PreparedCoefficient<F>, src: &DeviceSlice<'_>) {
    let (d, n) = (dst.as_mut_ptr(), dst.len());
    check(coeff.with_plan(|p| unsafe { sys::fgfc_mul_add_with(d, n, p, src.as_ptr(), src.len(), stream()) }));
}

/// `ops::mul_into` (src/ops.rs:381): `dst = coeff * src`.
#[track_caller]
pub fn mul_into<F: CudaField>(dst: &mut DeviceSliceMut<'_>, coeff: F::Elem, src: &DeviceSlice<'_>) {
    if F::WIDE {
        return mul_into_with(dst, &Coeff::<F>::new(coeff), src);
    }
    check(unsafe {
        sys::fgfc_mul_into(F::ID, dst.as_mut_ptr(), dst.len(), F::to_raw(coeff) as u32, src.as_ptr(), src.len(), stream())
    });
}

/// `ops::mul_into_with` (src/ops.rs:399).
#[track_caller]
pub fn mul_into_with<F: CudaField>(dst: &mut DeviceSliceMut<'_>, coeff: &impl PreparedCoefficient<F>, src: &DeviceSlice<'_>) {
    let (d, n) = (dst.as_mut_ptr(), dst.len());
    check(coeff.with_plan(|p| unsafe { sys::fgfc_mul_into_with(d, n, p, src.as_ptr(), src.len(), stream()) }));
}

/// `ops::mul_assign` (src/ops.rs:422): `dst *= coeff`.
#[track_caller]
pub fn mul_assign<F: CudaField>(dst: &mut DeviceSliceMut<'_>, coeff: F::Elem) {
    if F::WIDE {
        return mul_assign_with(dst, &Coeff::<F>::new(coeff));
    }
    check(unsafe { sys::fgfc_mul_assign(F::ID, dst.as_mut_ptr(), dst.len(), F::to_raw(coeff) as u32, stream()) });
}

/// `ops::mul_assign_with` (src/ops.rs:439).
#[track_caller]
pub fn mul_assign_with<F: CudaField>(dst: &mut DeviceSliceMut<'_>, coeff: &impl PreparedCoefficient<F>) {
    let (d, n) = (dst.as_mut_ptr(), dst.len());
    check(coeff.with_plan(|p| unsafe { sys::fgfc_mul_assign_with(d, n, p, stream()) }));
}

/// `ops::mul_elementwise` (src/ops.rs:953): `dst[i] = a[i] * b[i]`.
#[track_caller]
pub fn mul_elementwise<F: CudaField>(dst: &mut DeviceSliceMut<'_>, a: &DeviceSlice<'_>, b: &DeviceSlice<'_>) {
    check(unsafe {
        sys::fgfc_mul_elementwise(F::ID, dst.as_mut_ptr(), dst.len(), a.as_ptr(), a.len(), b.as_ptr(), b.len(), stream())
    });
}

// ---------------------------------------------------------------- one-to-many / many-to-one

/// `ops::mul_add_scatter` (src/ops.rs:461): `rows[j] ^= coeffs[j] * src`.
#[track_caller]
pub fn mul_add_scatter<F: CudaField>(rows: &mut DeviceSliceMut<'_>, row_len: usize, coeffs: &[F::Elem], src: &DeviceSlice<'_>) {
    if F::WIDE && !coeffs.is_empty() {
        return mul_add_scatter_with(rows, row_len, &Plan::<F>::new(coeffs), src);
    }
    let c = raw::<F>(coeffs);
    check(unsafe {
        sys::fgfc_mul_add_scatter(F::ID, rows.as_mut_ptr(), rows.len(), row_len, c.as_ptr(), c.len(), src.as_ptr(),
                                  src.len(), stream())
    });
}

/// `ops::mul_add_scatter_with` (src/ops.rs:493).
#[track_caller]
pub fn mul_add_scatter_with<F: CudaField>(rows: &mut DeviceSliceMut<'_>, row_len: usize, plan: &Plan<F>, src: &DeviceSlice<'_>) {
    check(unsafe {
        sys::fgfc_mul_add_scatter_with(rows.as_mut_ptr(), rows.len(), row_len, plan.raw, src.as_ptr(), src.len(), stream())
    });
}

/// `ops::mul_add_gather` (src/ops.rs:533): `dst ^= sum coeffs[i] * srcs[i]`.
#[track_caller]
pub fn mul_add_gather<F: CudaField>(dst: &mut DeviceSliceMut<'_>, coeffs: &[F::Elem], srcs: &[DeviceSlice<'_>]) {
    if F::WIDE && !coeffs.is_empty() && coeffs.len() == srcs.len() {
        return mul_add_gather_with(dst, &Plan::<F>::new(coeffs), srcs);
    }
    let c = raw::<F>(coeffs);
    let s = slices(srcs);
    check(unsafe {
        sys::fgfc_mul_add_gather(F::ID, dst.as_mut_ptr(), dst.len(), c.as_ptr(), c.len(), s.as_ptr(), s.len(), stream())
    });
}

/// `ops::mul_add_gather_with` (src/ops.rs:563).
#[track_caller]
pub fn mul_add_gather_with<F: CudaField>(dst: &mut DeviceSliceMut<'_>, plan: &Plan<F>, srcs: &[DeviceSlice<'_>]) {
    let s = slices(srcs);
    check(unsafe { sys::fgfc_mul_add_gather_with(dst.as_mut_ptr(), dst.len(), plan.raw, s.as_ptr(), s.len(), stream()) });
}

/// `ops::dot_product` (src/ops.rs:597): `dst = sum coeffs[i] * srcs[i]`.
#[track_caller]
pub fn dot_product<F: CudaField>(dst: &mut DeviceSliceMut<'_>, coeffs: &[F::Elem], srcs: &[DeviceSlice<'_>]) {
    if F::WIDE && !coeffs.is_empty() && coeffs.len() == srcs.len() {
        return dot_product_with(dst, &Plan::<F>::new(coeffs), srcs);
    }
    let c = raw::<F>(coeffs);
    let s = slices(srcs);
    check(unsafe {
        sys::fgfc_dot_product(F::ID, dst.as_mut_ptr(), dst.len(), c.as_ptr(), c.len(), s.as_ptr(), s.len(), stream())
    });
}

/// `ops::dot_product_with` (src/ops.rs:632).
#[track_caller]
pub fn dot_product_with<F: CudaField>(dst: &mut DeviceSliceMut<'_>, plan: &Plan<F>, srcs: &[DeviceSlice<'_>]) {
    let s = slices(srcs);
    check(unsafe { sys::fgfc_dot_product_with(dst.as_mut_ptr(), dst.len(), plan.raw, s.as_ptr(), s.len(), stream()) });
}

// ---------------------------------------------------------------- many-to-many

/// For an 8-byte field: the terms as a (sources, rows) plan and their
/// sources, when every term carries `nrows` coefficients (otherwise the raw
/// entry point reports the shape error).
fn wide_terms<'a, F: CudaField>(terms: &[(&[F::Elem], DeviceSlice<'a>)], nrows: usize)
                                -> Option<(Plan<F>, Vec<DeviceSlice<'a>>)> {
    if !F::WIDE || terms.is_empty() || terms.iter().any(|(c, _)| c.len() != nrows) {
        return None;
    }
    let vals: Vec<F::Elem> = terms.iter().flat_map(|(c, _)| c.iter().copied()).collect();
    Some((Plan::matrix(terms.len(), nrows, &vals), terms.iter().map(|(_, s)| *s).collect()))
}

fn terms<F: CudaField>(terms: &[(&[F::Elem], DeviceSlice<'_>)]) -> (Vec<Vec<u32>>, Vec<sys::fgfc_term>) {
    let coeffs: Vec<Vec<u32>> = terms.iter().map(|(c, _)| raw::<F>(c)).collect();
    let raws = terms
        .iter()
        .zip(&coeffs)
        .map(|((_, s), c)| sys::fgfc_term { coeffs: c.as_ptr(), ncoeffs: c.len(), src: s.as_ptr(), src_len: s.len() })
        .collect();
    (coeffs, raws)
}

/// `ops::mul_add_matrix` (src/ops.rs:675): `rows[j] ^= sum_t c[t][j] * src_t`.
#[track_caller]
pub fn mul_add_matrix<F: CudaField>(rows: &mut DeviceSliceMut<'_>, row_len: usize, nrows: usize,
                                    terms_: &[(&[F::Elem], DeviceSlice<'_>)]) {
    if let Some((plan, srcs)) = wide_terms::<F>(terms_, nrows) {
        return mul_add_matrix_with(rows, row_len, nrows, &plan, &srcs);
    }
    let (_keep, t) = terms::<F>(terms_);
    check(unsafe {
        sys::fgfc_mul_add_matrix(F::ID, rows.as_mut_ptr(), rows.len(), row_len, nrows, t.as_ptr(), t.len(), stream())
    });
}

/// `ops::mul_add_matrix_with` (src/ops.rs:720); plan dimensions (sources, rows).
#[track_caller]
pub fn mul_add_matrix_with<F: CudaField>(rows: &mut DeviceSliceMut<'_>, row_len: usize, nrows: usize, plan: &Plan<F>,
                                         srcs: &[DeviceSlice<'_>]) {
    let s = slices(srcs);
    check(unsafe {
        sys::fgfc_mul_add_matrix_with(rows.as_mut_ptr(), rows.len(), row_len, nrows, plan.raw, s.as_ptr(), s.len(),
                                      stream())
    });
}

/// `ops::dot_product_matrix` (src/ops.rs:773): the overwrite form.
#[track_caller]
pub fn dot_product_matrix<F: CudaField>(rows: &mut DeviceSliceMut<'_>, row_len: usize, nrows: usize,
                                        terms_: &[(&[F::Elem], DeviceSlice<'_>)]) {
    if let Some((plan, srcs)) = wide_terms::<F>(terms_, nrows) {
        return dot_product_matrix_with(rows, row_len, nrows, &plan, &srcs);
    }
    let (_keep, t) = terms::<F>(terms_);
    check(unsafe {
        sys::fgfc_dot_product_matrix(F::ID, rows.as_mut_ptr(), rows.len(), row_len, nrows, t.as_ptr(), t.len(), stream())
    });
}

/// `ops::dot_product_matrix_with` (src/ops.rs:823): the RS encode entry point.
#[track_caller]
pub fn dot_product_matrix_with<F: CudaField>(rows: &mut DeviceSliceMut<'_>, row_len: usize, nrows: usize,
                                             plan: &Plan<F>, srcs: &[DeviceSlice<'_>]) {
    let s = slices(srcs);
    check(unsafe {
        sys::fgfc_dot_product_matrix_with(rows.as_mut_ptr(), rows.len(), row_len, nrows, plan.raw, s.as_ptr(), s.len(),
                                          stream())
    });
}

/// `ops::mul_add_matrix_scattered` (src/ops.rs:887): row j at `dst[row_starts[j]..]`.
#[track_caller]
pub fn mul_add_matrix_scattered<F: CudaField>(dst: &mut DeviceSliceMut<'_>, row_len: usize, row_starts: &[usize],
                                              terms_: &[(&[F::Elem], DeviceSlice<'_>)]) {
    if let Some((plan, srcs)) = wide_terms::<F>(terms_, row_starts.len()) {
        return mul_add_matrix_scattered_with(dst, row_len, row_starts, &plan, &srcs);
    }
    let (_keep, t) = terms::<F>(terms_);
    check(unsafe {
        sys::fgfc_mul_add_matrix_scattered(F::ID, dst.as_mut_ptr(), dst.len(), row_len, row_starts.as_ptr(),
                                           row_starts.len(), t.as_ptr(), t.len(), stream())
    });
}

/// Extension (no reference counterpart): the scattered op driven by a plan.
#[track_caller]
pub fn mul_add_matrix_scattered_with<F: CudaField>(dst: &mut DeviceSliceMut<'_>, row_len: usize, row_starts: &[usize],
                                                   plan: &Plan<F>, srcs: &[DeviceSlice<'_>]) {
    let s = slices(srcs);
    check(unsafe {
        sys::fgfc_mul_add_matrix_scattered_with(dst.as_mut_ptr(), dst.len(), row_len, row_starts.as_ptr(),
                                                row_starts.len(), plan.raw, s.as_ptr(), s.len(), stream())
    });
}

/// Extension (no reference counterpart): the overwrite form of the scattered
/// op, equal to zeroing the rows and then mul_add_matrix_scattered.
#[track_caller]
pub fn dot_product_matrix_scattered_with<F: CudaField>(dst: &mut DeviceSliceMut<'_>, row_len: usize,
                                                       row_starts: &[usize], plan: &Plan<F>,
                                                       srcs: &[DeviceSlice<'_>]) {
    let s = slices(srcs);
    check(unsafe {
        sys::fgfc_dot_product_matrix_scattered_with(dst.as_mut_ptr(), dst.len(), row_len, row_starts.as_ptr(),
                                                    row_starts.len(), plan.raw, s.as_ptr(), s.len(), stream())
    });
}
