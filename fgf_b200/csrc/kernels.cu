// kernels.cu -- sm_100a kernels of libfgfcuda.so.
//
// One kernel family computes every shape of the reference's `ops` AXPY
// family (src/ops.rs:342-941): rows[j] (^)= XOR_t c[t][j] * src_t, with the
// destination rows given as pointers (contiguous or scattered) and
// overwrite (dot_product*) or accumulate (mul_add*) semantics.
//
// Arithmetic: multiplying a packed element by a fixed coefficient is linear
// over its byte subfield, so every output byte is an XOR of products of
// source bytes with constants (gf_host.hpp: coeff_byte_matrix). Products are
// read from split-nibble tables in shared memory: per (source, source byte
// plane, group of 4 output bytes) a 16-entry table for the low nibble and
// one for the high nibble, each entry a 32-bit word carrying the products
// for 4 output bytes at once (4 Gf8 rows, 2 Gf16 rows or 1 Gf32 row). Every
// table row is replicated across the 32 banks so a warp's lookups never
// conflict, and one PRMT forms each lookup address from the nibble, the
// lane and the table slot. The destination tile stays in registers while all
// sources are folded in, as the reference's blocked CPU kernels do
// (src/kernel/x86/gf8.rs:2208-2315), and is written once.
#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>
#include <map>
#include <mutex>
#include <utility>

#include "fast_core.cuh"
#include "internal.hpp"

namespace fgfc {

namespace {

// Copy compact tables for this launch into the replicated shared layout:
// word index i of the shared area is slot (i >> 10), nibble row
// ((i >> 6) & 15), half ((i >> 5) & 1), lane (i & 31). The compact words are
// staged in shared memory first (one independent load per thread) and each
// entry's 32 lane copies are written as 8 identical 16-byte stores.
template <int E, int G>
__device__ __forceinline__ void fill_tables(const MatrixLaunch& a) {
  const uint32_t nslots = a.k * E * G;
  uint32_t* stage = reinterpret_cast<uint32_t*>(g_smem) + nslots * 1024u;
  for (uint32_t i = threadIdx.x; i < nslots * kCompactWords; i += blockDim.x) {
    const uint32_t slot = i >> 5;  // (t * E + p) * G + g
    const uint32_t src = ((slot / G) * a.gstride + a.g0 + slot % G) * kCompactWords + (i & 31u);
    stage[i] = a.tables ? __ldg(a.tables + src) : a.inline_tab[src];
  }
  __syncthreads();
  uint4* st4 = reinterpret_cast<uint4*>(g_smem);
#pragma unroll 4
  for (uint32_t i = threadIdx.x; i < nslots * 256u; i += blockDim.x) {
    const uint32_t v = stage[(i >> 8) * kCompactWords + ((i >> 3) & 1u) * 16u + ((i >> 4) & 15u)];
    st4[i] = make_uint4(v, v, v, v);
  }
}

// Per-source lookup context: the byte pattern that places each byte's slot
// (low 4 bits) next to its nibble, and per plane the register supplying the
// lane offset (byte 0) and the 64 KiB page of the slot (bytes 2..3).
template <int E, int G>
struct SrcCtx {
  uint32_t pat;
  uint32_t lr[E];
  __device__ __forceinline__ SrcCtx(uint32_t t, uint32_t lane4) {
    pat = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const uint32_t s = (t * E + (b % E)) * G;
      pat |= (s & 15u) << (8 * b + 4);
    }
#pragma unroll
    for (int p = 0; p < E; ++p) {
      const uint32_t s = (t * E + p) * G;
      lr[p] = lane4 | ((s >> 4) << 16);
    }
  }
};

// Fold the 4 source bytes of word `w` (whole elements) into the
// accumulators of their elements: acc[g][e0 + b / E] for byte b.
template <int E, int G, int NE>
__device__ __forceinline__ void fold_word(uint32_t w, const SrcCtx<E, G>& c, uint32_t (&acc)[G][NE],
                                          int e0) {
  const uint32_t xl = (w & 0x0F0F0F0Fu) | c.pat;
  const uint32_t xh = ((w >> 4) & 0x0F0F0F0Fu) | c.pat;
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const uint32_t sel = 0x7604u | (static_cast<uint32_t>(b) << 4);
    const uint32_t al = prmt(xl, c.lr[b % E], sel);
    const uint32_t ah = prmt(xh, c.lr[b % E], sel);
#pragma unroll
    for (int g = 0; g < G; ++g)
      acc[g][e0 + b / E] ^= lds_at(al + g * kSlotBytes) ^ lds_at(ah + g * kSlotBytes + 128);
  }
}

// Assemble output word q (16-byte step: q < 4; scalar step: q = 0) of row
// rr of group g from the element accumulators.
template <int E, int G, int NE>
__device__ __forceinline__ uint32_t out_word(const uint32_t (&acc)[G][NE], int g, int rr, int q) {
  if (E == 1) {
    const uint32_t a0 = acc[g][4 * q], a1 = acc[g][4 * q + 1], a2 = acc[g][4 * q + 2],
                   a3 = acc[g][4 * q + 3];
    const uint32_t s01 = (rr < 2) ? prmt(a0, a1, 0x5140u) : prmt(a0, a1, 0x7362u);
    const uint32_t s23 = (rr < 2) ? prmt(a2, a3, 0x5140u) : prmt(a2, a3, 0x7362u);
    return (rr & 1) ? prmt(s01, s23, 0x7632u) : prmt(s01, s23, 0x5410u);
  } else if (E == 2) {
    return prmt(acc[g][2 * q], acc[g][2 * q + 1], rr ? 0x7632u : 0x5410u);
  } else {
    return acc[g][q];
  }
}

// SHIFT: some row is not at the sources' offset within 16 bytes. Then whole
// warps iterate together (the row stores shuffle between lanes) and lanes
// past the end reload the last column; otherwise each thread runs alone.
template <int E, int G, bool OVR, bool SHIFT>
__global__ void __launch_bounds__(512, (16 / E) * G <= 16 ? 2 : 1)
    matrix_vec_kernel(const __grid_constant__ MatrixLaunch a) {
  constexpr int NE = 16 / E;  // elements per 16-byte step
  constexpr int R = 4 / E;    // rows per group
  fill_tables<E, G>(a);
  __syncthreads();
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lane4 = lane * 4u;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t vb = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x - (SHIFT ? lane : 0u);
       vb < a.nvec; vb += stride) {
    const uint64_t v = SHIFT ? vb + lane : vb;
    const bool valid = !SHIFT || v < a.nvec;
    const uint64_t off = a.head + (valid ? v : a.nvec - 1) * 16u;
    uint32_t acc[G][NE];
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int e = 0; e < NE; ++e) acc[g][e] = 0;
    uint4 cur = ldg16(a.src[0] + off);
    for (uint32_t t = 0; t < a.k; ++t) {
      uint4 nxt = cur;
      if (t + 1 < a.k) nxt = ldg16(a.src[t + 1] + off);
      const SrcCtx<E, G> c(t, lane4);
      fold_word<E, G, NE>(cur.x, c, acc, 0 * (4 / E));
      fold_word<E, G, NE>(cur.y, c, acc, 1 * (4 / E));
      fold_word<E, G, NE>(cur.z, c, acc, 2 * (4 / E));
      fold_word<E, G, NE>(cur.w, c, acc, 3 * (4 / E));
      cur = nxt;
    }
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        const uint32_t row = g * R + rr;
        uint4 o;
        o.x = out_word<E, G, NE>(acc, g, rr, 0);
        o.y = out_word<E, G, NE>(acc, g, rr, 1);
        o.z = out_word<E, G, NE>(acc, g, rr, 2);
        o.w = out_word<E, G, NE>(acc, g, rr, 3);
        if constexpr (SHIFT) {
          const bool rv = valid && row < a.nrows;
          store_vec16(rv ? a.dst[row] + off : nullptr, o, rv, OVR);
        } else {
          if (row < a.nrows) put16(a.dst[row] + off, o, OVR);
        }
      }
  }
}

// Scalar path: 4-byte groups with byte loads and stores, for the unaligned
// head and tail of the vector body and for buffers whose pointers do not
// share an alignment. Ranges [r0s, r0e) and [r1s, r1e) of every row; each
// range starts on an element boundary.
struct ScalarRanges {
  uint64_t r0s, r0e, r1s, r1e;
};

template <int E, int G, bool OVR>
__global__ void __launch_bounds__(256) matrix_scalar_kernel(const __grid_constant__ MatrixLaunch a,
                                                            ScalarRanges rg) {
  constexpr int R = 4 / E;
  fill_tables<E, G>(a);
  __syncthreads();
  const uint32_t lane4 = (threadIdx.x & 31u) * 4u;
  const uint64_t n0 = (rg.r0e - rg.r0s + 3) / 4, n1 = (rg.r1e - rg.r1s + 3) / 4;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n0 + n1;
       i += stride) {
    const uint64_t off = i < n0 ? rg.r0s + 4 * i : rg.r1s + 4 * (i - n0);
    const uint64_t end = i < n0 ? rg.r0e : rg.r1e;
    const int nb = static_cast<int>(end - off < 4 ? end - off : 4);
    uint32_t acc[G][4 / E];
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int e = 0; e < 4 / E; ++e) acc[g][e] = 0;
    for (uint32_t t = 0; t < a.k; ++t) {
      const uint8_t* s = a.src[t] + off;
      uint32_t w = 0;
      for (int b = 0; b < nb; ++b) w |= static_cast<uint32_t>(s[b]) << (8 * b);
      const SrcCtx<E, G> c(t, lane4);
      fold_word<E, G, 4 / E>(w, c, acc, 0);
    }
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int rr = 0; rr < R; ++rr) {
        const uint32_t row = g * R + rr;
        if (row >= a.nrows) continue;
        uint32_t o;
        if (E == 1) {
          o = prmt(prmt(acc[g][0], acc[g][1], rr < 2 ? 0x5140u : 0x7362u),
                   prmt(acc[g][2], acc[g][3], rr < 2 ? 0x5140u : 0x7362u),
                   (rr & 1) ? 0x7632u : 0x5410u);
        } else if (E == 2) {
          o = prmt(acc[g][0], acc[g][1], rr ? 0x7632u : 0x5410u);
        } else {
          o = acc[g][0];
        }
        uint8_t* d = a.dst[row] + off;
        for (int b = 0; b < nb; ++b) {
          const uint8_t v = static_cast<uint8_t>(o >> (8 * b));
          d[b] = OVR ? v : static_cast<uint8_t>(d[b] ^ v);
        }
      }
  }
}

// ---------------------------------------------------------------- byte-table kernel
//
// Gf8, at most 4 rows, K <= 14 sources: the RS(10,4) encode / reconstruct
// shape and the single-row ops (fast_core.cuh). Chosen per call by the tuner
// (tune.cpp): short rows use the nibble kernel, whose tables fill faster.

template <int K, bool OVR, bool SHIFT>
__global__ void __launch_bounds__(kFastThreads, 1) matrix_fast_kernel(const __grid_constant__ MatrixLaunch a) {
  fill_fast<K>(a.tables, a.inline_tab, a.gstride, a.g0);
  const FastRegs r;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const uint32_t lane = threadIdx.x & 31u;
  // SHIFT: whole warps iterate together (see matrix_vec_kernel)
  for (uint64_t vb = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x - (SHIFT ? lane : 0u);
       vb < a.nvec; vb += stride) {
    const uint64_t v = SHIFT ? vb + lane : vb;
    const bool valid = !SHIFT || v < a.nvec;
    const uint64_t off = a.head + (valid ? v : a.nvec - 1) * 16u;
    if (v + stride < a.nvec) {  // this thread's next column: into L2 now
#pragma unroll
      for (int t = 0; t < K; ++t) prefetch_l2(a.src[t] + off + stride * 16u);
    }
    uint32_t w[K][4];
#pragma unroll
    for (int t = 0; t < K; ++t) {
      const uint4 x = ldg16(a.src[t] + off);
      w[t][0] = x.x;
      w[t][1] = x.y;
      w[t][2] = x.z;
      w[t][3] = x.w;
    }
    uint32_t acc[16];
#pragma unroll
    for (int e = 0; e < 16; ++e) acc[e] = 0;
    fast_fold<K, 4>(w, acc, r);
    if constexpr (SHIFT)
      store_col4_any(acc, a.dst, a.nrows, off, OVR, valid);
    else
      store_col4(acc, a.dst, a.nrows, off, OVR);
  }
}

template <int K, bool OVR, bool SHIFT>
cudaError_t launch_fast_k(const MatrixLaunch& a, cudaStream_t s) {
  cudaError_t e = ensure_smem_attr(reinterpret_cast<const void*>(matrix_fast_kernel<K, OVR, SHIFT>),
                                   FastLayout<K>::smem);
  if (e != cudaSuccess) return e;
  const uint64_t want = (a.nvec + kFastThreads - 1) / kFastThreads;
  const uint64_t cap = static_cast<uint64_t>(sm_count());
  const unsigned blocks = static_cast<unsigned>(want < cap ? want : cap);
  matrix_fast_kernel<K, OVR, SHIFT><<<blocks, kFastThreads, FastLayout<K>::smem, s>>>(a);
  return cudaGetLastError();
}

template <bool OVR, bool SHIFT>
cudaError_t launch_fast_s(const MatrixLaunch& a, cudaStream_t s) {
  switch (a.k) {
    case 1: return launch_fast_k<1, OVR, SHIFT>(a, s);
    case 2: return launch_fast_k<2, OVR, SHIFT>(a, s);
    case 3: return launch_fast_k<3, OVR, SHIFT>(a, s);
    case 4: return launch_fast_k<4, OVR, SHIFT>(a, s);
    case 5: return launch_fast_k<5, OVR, SHIFT>(a, s);
    case 6: return launch_fast_k<6, OVR, SHIFT>(a, s);
    case 7: return launch_fast_k<7, OVR, SHIFT>(a, s);
    case 8: return launch_fast_k<8, OVR, SHIFT>(a, s);
    case 9: return launch_fast_k<9, OVR, SHIFT>(a, s);
    case 10: return launch_fast_k<10, OVR, SHIFT>(a, s);
    case 11: return launch_fast_k<11, OVR, SHIFT>(a, s);
    case 12: return launch_fast_k<12, OVR, SHIFT>(a, s);
    case 13: return launch_fast_k<13, OVR, SHIFT>(a, s);
    case 14: return launch_fast_k<14, OVR, SHIFT>(a, s);
    default: return cudaErrorInvalidValue;
  }
}

template <bool OVR>
cudaError_t launch_fast(const MatrixLaunch& a, cudaStream_t s) {
  return a.shift ? launch_fast_s<OVR, true>(a, s) : launch_fast_s<OVR, false>(a, s);
}

template <int E, int G, bool OVR>
cudaError_t launch_one(const MatrixLaunch& a, cudaStream_t s, bool byte_tables) {
  constexpr int kSmemMax = kMaxSlots * (kSlotBytes + kCompactWords * 4);
  for (const void* fn : {reinterpret_cast<const void*>(matrix_vec_kernel<E, G, OVR, false>),
                         reinterpret_cast<const void*>(matrix_vec_kernel<E, G, OVR, true>),
                         reinterpret_cast<const void*>(matrix_scalar_kernel<E, G, OVR>)}) {
    cudaError_t e = ensure_smem_attr(fn, kSmemMax);
    if (e != cudaSuccess) return e;
  }
  const size_t smem = static_cast<size_t>(a.k) * E * G * (kSlotBytes + kCompactWords * 4);
  const int sms = sm_count();
  if (E == 1 && G == 1 && a.k <= 14 && a.nvec && byte_tables) {
    cudaError_t e = launch_fast<OVR>(a, s);
    if (e != cudaSuccess) return e;
  } else if (a.nvec) {
    int occ = 0;
    auto kern = a.shift ? matrix_vec_kernel<E, G, OVR, true> : matrix_vec_kernel<E, G, OVR, false>;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 512, smem);
    if (e != cudaSuccess) return e;
    const int occ_vec = occ > 0 ? occ : 1;
    uint64_t want = (a.nvec + 511) / 512;
    uint64_t cap = static_cast<uint64_t>(sms) * occ_vec;
    const unsigned blocks = static_cast<unsigned>(want < cap ? want : cap);
    kern<<<blocks, 512, smem, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  ScalarRanges rg;
  rg.r0s = 0;
  rg.r0e = a.head;
  rg.r1s = a.head + a.nvec * 16;
  rg.r1e = a.len;
  const uint64_t ngroups = (rg.r0e - rg.r0s + 3) / 4 + (rg.r1e - rg.r1s + 3) / 4;
  if (ngroups) {
    uint64_t want = (ngroups + 255) / 256;
    uint64_t cap = static_cast<uint64_t>(sms) * 2;
    const unsigned blocks = static_cast<unsigned>(want < cap ? want : cap);
    matrix_scalar_kernel<E, G, OVR><<<blocks, 256, smem, s>>>(a, rg);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

template <int E, bool OVR>
cudaError_t launch_e(int groups, const MatrixLaunch& a, cudaStream_t s, bool bt) {
  switch (groups) {
    case 1: return launch_one<E, 1, OVR>(a, s, bt);
    case 2: return launch_one<E, 2, OVR>(a, s, bt);
    case 3: return launch_one<E, 3, OVR>(a, s, bt);
    case 4: return launch_one<E, 4, OVR>(a, s, bt);
    default: return cudaErrorInvalidValue;
  }
}

// ---------------------------------------------------------------- helpers

__global__ void xor_kernel(uint8_t* __restrict__ dst, const uint8_t* __restrict__ src, uint64_t len,
                           uint64_t head, uint64_t nvec) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (uint64_t v = tid; v < nvec; v += stride) {
    uint4* d = reinterpret_cast<uint4*>(dst + head + 16 * v);
    const uint4 x = ldg16(src + head + 16 * v);
    uint4 y = *d;
    y.x ^= x.x;
    y.y ^= x.y;
    y.z ^= x.z;
    y.w ^= x.w;
    *d = y;
  }
  const uint64_t tail0 = head + 16 * nvec;
  for (uint64_t i = tid; i < head + (len - tail0); i += stride) {
    const uint64_t o = i < head ? i : tail0 + (i - head);
    dst[o] ^= src[o];
  }
}

__constant__ uint8_t c_exp[2][512];
__constant__ uint8_t c_log[2][256];
// __constant__ memory is per device: the tables are uploaded once per device.
constexpr int kMaxDevices = 64;
std::atomic<bool> g_const_ready[kMaxDevices];
std::mutex g_const_mu;

__device__ __forceinline__ uint8_t emul(const uint8_t* ex, const uint8_t* lg, uint8_t x, uint8_t y) {
  return (x && y) ? ex[lg[x] + lg[y]] : 0;
}

template <int F>
__global__ void elementwise_kernel(uint8_t* dst, const uint8_t* a, const uint8_t* b, uint64_t nelem) {
  __shared__ uint8_t ex[512];
  __shared__ uint8_t lg[256];
  constexpr int sel = (F == kGf8D) ? 1 : 0;
  for (int i = threadIdx.x; i < 512; i += blockDim.x) ex[i] = c_exp[sel][i];
  for (int i = threadIdx.x; i < 256; i += blockDim.x) lg[i] = c_log[sel][i];
  __syncthreads();
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nelem;
       i += stride) {
    if (F == kGf8B || F == kGf8D) {
      dst[i] = emul(ex, lg, a[i], b[i]);
    } else if (F == kGf16) {
      const uint8_t x0 = a[2 * i], x1 = a[2 * i + 1], y0 = b[2 * i], y1 = b[2 * i + 1];
      const uint8_t ac = emul(ex, lg, x0, y0), bd = emul(ex, lg, x1, y1);
      dst[2 * i] = ac ^ emul(ex, lg, 0x20, bd);
      dst[2 * i + 1] = emul(ex, lg, x0 ^ x1, y0 ^ y1) ^ ac;
    } else {
      auto m16 = [&](uint16_t x, uint16_t y) -> uint16_t {
        const uint8_t p0 = x & 0xFF, p1 = x >> 8, q0 = y & 0xFF, q1 = y >> 8;
        const uint8_t ac = emul(ex, lg, p0, q0), bd = emul(ex, lg, p1, q1);
        const uint8_t lo = ac ^ emul(ex, lg, 0x20, bd);
        const uint8_t hi = emul(ex, lg, p0 ^ p1, q0 ^ q1) ^ ac;
        return static_cast<uint16_t>(lo | (hi << 8));
      };
      const uint16_t xa = a[4 * i] | (a[4 * i + 1] << 8), xb = a[4 * i + 2] | (a[4 * i + 3] << 8);
      const uint16_t ya = b[4 * i] | (b[4 * i + 1] << 8), yb = b[4 * i + 2] | (b[4 * i + 3] << 8);
      const uint16_t ac = m16(xa, ya), bd = m16(xb, yb);
      const uint16_t lo = ac ^ m16(0x2000, bd);
      const uint16_t hi = m16(xa ^ xb, ya ^ yb) ^ ac;
      dst[4 * i] = lo & 0xFF;
      dst[4 * i + 1] = lo >> 8;
      dst[4 * i + 2] = hi & 0xFF;
      dst[4 * i + 3] = hi >> 8;
    }
  }
}

}  // namespace

int sm_count() {
  static std::atomic<int> sms[kMaxDevices];
  int dev = 0;
  cudaGetDevice(&dev);
  const bool cached = dev >= 0 && dev < kMaxDevices;
  int v = cached ? sms[dev].load(std::memory_order_relaxed) : 0;
  if (v > 0) return v;
  cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
  if (v <= 0) v = 148;
  if (cached) sms[dev].store(v, std::memory_order_relaxed);
  return v;
}

// cudaFuncSetAttribute acts on the current device only, so the opt-in to
// more than 48 KiB of dynamic shared memory is recorded per (device, kernel)
// and taken under a lock: plans, batch runners and servers may target any
// device from any host thread.
cudaError_t ensure_smem_attr(const void* fn, int bytes) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  static std::mutex mu;
  static std::map<std::pair<int, const void*>, int> done;
  std::lock_guard<std::mutex> lk(mu);
  const auto key = std::make_pair(dev, fn);
  const auto it = done.find(key);
  if (it != done.end() && it->second >= bytes) return cudaSuccess;
  e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) done[key] = bytes;
  return e;
}

cudaError_t launch_matrix(int field, int groups, bool overwrite, const MatrixLaunch& a,
                          cudaStream_t s, bool bt) {
  const int E = field_bytes(field);
  if (E == 1) return overwrite ? launch_e<1, true>(groups, a, s, bt) : launch_e<1, false>(groups, a, s, bt);
  if (E == 2) return overwrite ? launch_e<2, true>(groups, a, s, bt) : launch_e<2, false>(groups, a, s, bt);
  if (E == 4) return overwrite ? launch_e<4, true>(groups, a, s, bt) : launch_e<4, false>(groups, a, s, bt);
  return cudaErrorInvalidValue;
}

cudaError_t launch_zero_rows(uint8_t* const* rows, int n, uint64_t len, cudaStream_t s) {
  for (int j = 0; j < n; ++j) {
    cudaError_t e = cudaMemsetAsync(rows[j], 0, len, s);
    if (e != cudaSuccess) return e;
  }
  return cudaSuccess;
}

cudaError_t launch_xor(uint8_t* dst, const uint8_t* src, uint64_t len, cudaStream_t s) {
  if (!len) return cudaSuccess;
  const uint64_t ad = reinterpret_cast<uintptr_t>(dst) & 15, as = reinterpret_cast<uintptr_t>(src) & 15;
  uint64_t head = 0, nvec = 0;
  if (ad == as) {
    head = (16 - ad) & 15;
    if (head > len) head = len;
    nvec = (len - head) / 16;
  } else {
    head = len;
  }
  const uint64_t work = nvec + head + (len - head - 16 * nvec);
  uint64_t want = (work + 255) / 256, cap = static_cast<uint64_t>(sm_count()) * 8;
  xor_kernel<<<static_cast<unsigned>(want < cap ? want : cap), 256, 0, s>>>(dst, src, len, head, nvec);
  return cudaGetLastError();
}

cudaError_t launch_elementwise(int field, uint8_t* dst, const uint8_t* a, const uint8_t* b,
                               uint64_t len, cudaStream_t s) {
  if (!len) return cudaSuccess;
  int dev = 0;
  cudaError_t de = cudaGetDevice(&dev);
  if (de != cudaSuccess) return de;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (!g_const_ready[dev].load(std::memory_order_acquire)) {
    std::lock_guard<std::mutex> lk(g_const_mu);
    uint8_t ex[2][512], lg[2][256];
    const Gf8Log* t[2] = {&gf8b_tab(), &gf8d_tab()};
    for (int w = 0; w < 2; ++w) {
      for (int i = 0; i < 512; ++i) ex[w][i] = t[w]->exp[i];
      for (int i = 0; i < 256; ++i) lg[w][i] = t[w]->log[i];
    }
    cudaError_t e = cudaMemcpyToSymbol(c_exp, ex, sizeof(ex));
    if (e != cudaSuccess) return e;
    e = cudaMemcpyToSymbol(c_log, lg, sizeof(lg));
    if (e != cudaSuccess) return e;
    g_const_ready[dev].store(true, std::memory_order_release);
  }
  const uint64_t nelem = len / field_bytes(field);
  uint64_t want = (nelem + 255) / 256, cap = static_cast<uint64_t>(sm_count()) * 8;
  const unsigned blocks = static_cast<unsigned>(want < cap ? want : cap);
  switch (field) {
    case kGf8B: elementwise_kernel<kGf8B><<<blocks, 256, 0, s>>>(dst, a, b, nelem); break;
    case kGf8D: elementwise_kernel<kGf8D><<<blocks, 256, 0, s>>>(dst, a, b, nelem); break;
    case kGf16: elementwise_kernel<kGf16><<<blocks, 256, 0, s>>>(dst, a, b, nelem); break;
    case kGf32: elementwise_kernel<kGf32><<<blocks, 256, 0, s>>>(dst, a, b, nelem); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace fgfc
