//! Device buffers and streams.
use std::cell::Cell;
use std::marker::PhantomData;

/// A borrowed range of device memory, the counterpart of `&[u8]`.
#[derive(Clone, Copy, Debug)]
pub struct DeviceSlice<'a> {
    ptr: *const u8,
    len: usize,
    _life: PhantomData<&'a [u8]>,
}

/// A borrowed range of writable device memory, the counterpart of `&mut [u8]`.
#[derive(Debug)]
pub struct DeviceSliceMut<'a> {
    ptr: *mut u8,
    len: usize,
    _life: PhantomData<&'a mut [u8]>,
}

impl<'a> DeviceSlice<'a> {
    /// # Safety
    /// `ptr..ptr + len` must be device memory of the current device that
    /// stays allocated and is not written by the GPU while borrowed.
    pub unsafe fn from_raw(ptr: *const u8, len: usize) -> Self {
        Self { ptr, len, _life: PhantomData }
    }
    pub fn len(&self) -> usize {
        self.len
    }
    pub fn is_empty(&self) -> bool {
        self.len == 0
    }
    pub fn as_ptr(&self) -> *const u8 {
        self.ptr
    }
    /// Sub-range `[start, start + len)`.
    pub fn slice(&self, start: usize, len: usize) -> DeviceSlice<'a> {
        assert!(start <= self.len && len <= self.len - start, "DeviceSlice::slice out of range");
        // SAFETY: a sub-range of a valid borrowed range.
        unsafe { DeviceSlice::from_raw(self.ptr.add(start), len) }
    }
    pub(crate) fn raw(&self) -> crate::sys::fgfc_slice {
        crate::sys::fgfc_slice { ptr: self.ptr, len: self.len }
    }
}

impl<'a> DeviceSliceMut<'a> {
    /// # Safety
    /// `ptr..ptr + len` must be device memory of the current device that
    /// stays allocated, with no other access while borrowed.
    pub unsafe fn from_raw(ptr: *mut u8, len: usize) -> Self {
        Self { ptr, len, _life: PhantomData }
    }
    pub fn len(&self) -> usize {
        self.len
    }
    pub fn is_empty(&self) -> bool {
        self.len == 0
    }
    pub fn as_mut_ptr(&mut self) -> *mut u8 {
        self.ptr
    }
    pub fn as_slice(&self) -> DeviceSlice<'_> {
        // SAFETY: the same range, borrowed immutably.
        unsafe { DeviceSlice::from_raw(self.ptr, self.len) }
    }
}

/// A CUDA stream handle (`cudaStream_t`); the null stream is the default.
#[derive(Clone, Copy, Debug, PartialEq, Eq)]
pub struct Stream(pub crate::sys::fgfc_stream);

// SAFETY: a stream handle is an opaque token the CUDA runtime accepts from
// any host thread.
unsafe impl Send for Stream {}
unsafe impl Sync for Stream {}

thread_local! {
    static CURRENT: Cell<crate::sys::fgfc_stream> = const { Cell::new(std::ptr::null_mut()) };
}

impl Stream {
    pub const DEFAULT: Stream = Stream(std::ptr::null_mut());
    /// Calls of `ops` on this thread are enqueued on `self` from now on.
    pub fn make_current(self) {
        CURRENT.with(|c| c.set(self.0));
    }
    pub fn current() -> Stream {
        Stream(CURRENT.with(|c| c.get()))
    }
}
