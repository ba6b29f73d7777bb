// kernels.cu -- sm_100a kernels of libfgfcuda.so.
//
// One kernel family computes every shape of the reference's `ops` AXPY
// family (src/ops.rs:342-941): rows[j] (^)= XOR_t c[t][j] * src_t, with the
// destination rows given as pointers (contiguous or scattered) and
// overwrite (dot_product*) or accumulate (mul_add*) semantics.
//
// Arithmetic: multiplying a packed element by a fixed coefficient is linear
// over GF(2) in every field here, so every output byte is an XOR of fixed
// linear maps of the source bytes (gf_host.hpp: coeff_images). Products are
// read from split-nibble tables in shared memory: per (source, source byte
// plane, group of 4 output bytes) a 16-entry table for the low nibble and
// one for the high nibble, each entry a 32-bit word carrying the products
// for 4 output bytes at once (4 one-byte, 2 two-byte or 1 four-byte rows). Every
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

// Per-device caches (SM count) are arrays indexed by device ordinal.
constexpr int kMaxDevices = 64;

// ---- mul_elementwise: products of two vectors, without tables.
//
// GF(2^8) products of 4 byte lanes of a 32-bit word at once by shifts and
// XORs: x * y = XOR over the set bits b of y of x * 2^b, where x * 2 is the
// byte-wise shift left reduced by the field polynomial in the lanes whose
// bit 7 falls out. A permute whose selector nibble is 8 + i copies the top
// bit of byte i over the whole byte, so each byte mask costs one PRMT.
// Gf16 and Gf32 use their tower identities over these byte products:
//   (a + b u)(c + d u) = (ac + 0x20 bd) + ((a + b)(c + d) + ac) u      (Gf16)
//   (A + B v)(C + D v) = (AC + 0x2000 BD) + ((A + B)(C + D) + AC) v   (Gf32)
// (src/field/gf16.rs:54-60, src/field/gf32.rs:36-42). No lookups means no
// shared-memory bank conflicts; the kernel is bound by HBM for Gf8.

__device__ __forceinline__ uint32_t prmt_sign(uint32_t a, uint32_t sel) {
  uint32_t d;
  asm("prmt.b32 %0, %1, 0, %2;" : "=r"(d) : "r"(a), "r"(sel));
  return d;
}

// 4 byte lanes times 2, reduced by the polynomial whose low byte is R.
template <uint32_t R>
__device__ __forceinline__ uint32_t xtime4(uint32_t x) {
  return ((x & 0x7F7F7F7Fu) << 1) ^ (prmt_sign(x, 0xBA98u) & (R * 0x01010101u));
}

// 4 independent GF(2^8) products (byte lane i of x times byte lane i of y).
template <uint32_t R>
__device__ __forceinline__ uint32_t gmul4(uint32_t x, uint32_t y) {
  uint32_t acc = 0;
#pragma unroll
  for (int b = 0; b < 8; ++b) {
    acc ^= x & prmt_sign(y << (7 - b), 0xBA98u);  // lanes whose bit b of y is set
    if (b < 7) x = xtime4<R>(x);
  }
  return acc;
}

// Two Gf16 products per word: elements [a, b] in bytes 0-1 and 2-3.
__device__ __forceinline__ uint32_t gmul16x2(uint32_t x, uint32_t y) {
  const uint32_t p = gmul4<0x1Bu>(x, y);                                   // [ac, bd, ...]
  const uint32_t q = gmul4<0x1Bu>(x ^ prmt(x, 0u, 0x2301u), y ^ prmt(y, 0u, 0x2301u));  // [(a+b)(c+d), ...]
  uint32_t c = p;                                                          // 0x20 * p: five doublings
#pragma unroll
  for (int i = 0; i < 5; ++i) c = xtime4<0x1Bu>(c);
  // [ac + 0x20 bd, (a+b)(c+d) + ac] per element
  return prmt(p, p, 0x2200u) ^ prmt(c, q, 0x7351u);
}

// The Gf16 products of two words at once (r1 = x1 * y1, r2 = x2 * y2, two
// elements each): the four cross products (a + b)(c + d) share one byte
// product pass instead of filling half of two.
__device__ __forceinline__ void gmul16x2_pair(uint32_t x1, uint32_t y1, uint32_t x2, uint32_t y2, uint32_t& r1,
                                              uint32_t& r2) {
  const uint32_t p1 = gmul4<0x1Bu>(x1, y1), p2 = gmul4<0x1Bu>(x2, y2);  // [ac, bd, ac, bd]
  const uint32_t xs = prmt(x1 ^ (x1 >> 8), x2 ^ (x2 >> 8), 0x6420u);      // a + b of the 4 elements
  const uint32_t ys = prmt(y1 ^ (y1 >> 8), y2 ^ (y2 >> 8), 0x6420u);
  const uint32_t q = gmul4<0x1Bu>(xs, ys);                                 // (a+b)(c+d) of the 4 elements
  uint32_t c = prmt(p1, p2, 0x7531u);                                      // the 4 bd, then 0x20 bd:
#pragma unroll
  for (int i = 0; i < 5; ++i) c = xtime4<0x1Bu>(c);                        // five doublings
  r1 = prmt(p1, p1, 0x2200u) ^ prmt(c, q, 0x5140u);
  r2 = prmt(p2, p2, 0x2200u) ^ prmt(c, q, 0x7362u);
}

// 0x2000 times each Gf16 lane (a + b u) of a word: 0x20 0x20 b + 0x20 (a + b) u.
// The hi lanes (a + b) take 5 doublings and the lo lanes (b) 10: the first 5
// run on both at once.
__device__ __forceinline__ uint32_t gmul2000x2(uint32_t v) {
  uint32_t w = ((v ^ (v << 8)) & 0xFF00FF00u) | ((v >> 8) & 0x00FF00FFu);
#pragma unroll
  for (int i = 0; i < 5; ++i) w = xtime4<0x1Bu>(w);
  uint32_t lo = w & 0x00FF00FFu;
#pragma unroll
  for (int i = 0; i < 5; ++i) lo = xtime4<0x1Bu>(lo);
  return (w & 0xFF00FF00u) | lo;
}

// One Gf32 product per word: [A, B] as Gf16 halves.
__device__ __forceinline__ uint32_t gmul32(uint32_t x, uint32_t y) {
  uint32_t p, q;                                                           // [AC, BD], [(A+B)(C+D), ..]
  gmul16x2_pair(x, y, x ^ prmt(x, 0u, 0x1032u), y ^ prmt(y, 0u, 0x1032u), p, q);
  const uint32_t c = gmul2000x2(p);                                        // [0x2000 AC, 0x2000 BD]
  return prmt(p ^ (c >> 16), q ^ p, 0x5410u);                             // [AC + 0x2000 BD, (A+B)(C+D) + AC]
}

// One word of 32-bit lanes holding 4 bytes of each vector (a whole number of
// elements: 4 Gf8, 2 Gf16, 1 Gf32).
template <int F>
__device__ __forceinline__ uint32_t emul_word(uint32_t x, uint32_t y) {
  if (F == kGf8B) return gmul4<0x1Bu>(x, y);
  if (F == kGf8D) return gmul4<0x1Du>(x, y);
  if (F == kGf16) return gmul16x2(x, y);
  return gmul32(x, y);
}

// Vector path: dst, a and b share their offset within 16 bytes and the first
// `head` bytes (a whole number of elements) run through the scalar path, so
// the body is 16-byte loads and stores; `nvec` 16-byte vectors follow.
// Scalar path (head, tail, or every element when the offsets differ): one
// element per thread step, its bytes gathered into the low lanes of a word.
template <int F>
__global__ void elementwise_kernel(uint8_t* __restrict__ dst, const uint8_t* __restrict__ a,
                                   const uint8_t* __restrict__ b, uint64_t len, uint64_t head, uint64_t nvec) {
  constexpr int E = (F == kGf16) ? 2 : (F == kGf32 ? 4 : 1);
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  for (uint64_t v = tid; v < nvec; v += stride) {
    const uint64_t o = head + 16 * v;
    const uint4 x = ldg16(a + o), y = ldg16(b + o);
    uint4 r;
    if (F == kGf16) {  // pairs of words share their cross-product pass
      gmul16x2_pair(x.x, y.x, x.y, y.y, r.x, r.y);
      gmul16x2_pair(x.z, y.z, x.w, y.w, r.z, r.w);
    } else {
      r.x = emul_word<F>(x.x, y.x);
      r.y = emul_word<F>(x.y, y.y);
      r.z = emul_word<F>(x.z, y.z);
      r.w = emul_word<F>(x.w, y.w);
    }
    *reinterpret_cast<uint4*>(dst + o) = r;
  }
  const uint64_t tail0 = head + 16 * nvec;
  const uint64_t nscalar = (head + (len - tail0)) / E;
  for (uint64_t i = tid; i < nscalar; i += stride) {
    const uint64_t o = i * E < head ? i * E : tail0 + (i * E - head);
    uint32_t x = 0, y = 0;
#pragma unroll
    for (int k = 0; k < E; ++k) {
      x |= static_cast<uint32_t>(a[o + k]) << (8 * k);
      y |= static_cast<uint32_t>(b[o + k]) << (8 * k);
    }
    const uint32_t r = emul_word<F>(x, y);
#pragma unroll
    for (int k = 0; k < E; ++k) dst[o + k] = static_cast<uint8_t>(r >> (8 * k));
  }
}

// ---- mul_elementwise over the Fan-Paar towers. Byte products use the
// byte level's log/exp tables (generator 0x2d) and a byte times the byte
// level's top generator alpha uses a 256-entry table; the 16-, 32- and 64-bit
// levels follow the Karatsuba recursion of the tower X^2 + alpha X + 1
// (src/field/fan_paar.rs:80-94, 122-134). Tables: 1 KiB, staged from
// constant memory into shared memory per CTA.
__constant__ uint8_t c_fp_tab[1024];  // exp[0..510) | pad | log[256] | alpha[256]

struct FpTab {
  const uint8_t* exp;
  const uint8_t* log;
  const uint8_t* alpha;
  __device__ __forceinline__ uint32_t m8(uint32_t a, uint32_t b) const {
    return (a && b) ? exp[log[a] + log[b]] : 0u;
  }
  __device__ __forceinline__ uint32_t alpha16(uint32_t v) const {  // v * alpha at the 16-bit level
    return (v >> 8) | (((v & 0xFFu) ^ alpha[v >> 8]) << 8);
  }
  __device__ __forceinline__ uint32_t m16(uint32_t x, uint32_t y) const {
    const uint32_t a0 = x & 0xFFu, a1 = x >> 8, b0 = y & 0xFFu, b1 = y >> 8;
    const uint32_t z0 = m8(a0, b0), z2 = m8(a1, b1), z1 = m8(a0 ^ a1, b0 ^ b1) ^ z0 ^ z2;
    return (z0 ^ z2) | ((z1 ^ alpha[z2]) << 8);
  }
  __device__ __forceinline__ uint32_t m32(uint32_t x, uint32_t y) const {
    const uint32_t a0 = x & 0xFFFFu, a1 = x >> 16, b0 = y & 0xFFFFu, b1 = y >> 16;
    const uint32_t z0 = m16(a0, b0), z2 = m16(a1, b1), z1 = m16(a0 ^ a1, b0 ^ b1) ^ z0 ^ z2;
    return (z0 ^ z2) | ((z1 ^ alpha16(z2)) << 16);
  }
  __device__ __forceinline__ uint32_t alpha32(uint32_t v) const {  // v * alpha at the 32-bit level
    return (v >> 16) | (((v & 0xFFFFu) ^ alpha16(v >> 16)) << 16);
  }
  __device__ __forceinline__ uint64_t m64(uint64_t x, uint64_t y) const {
    const uint32_t a0 = static_cast<uint32_t>(x), a1 = static_cast<uint32_t>(x >> 32);
    const uint32_t b0 = static_cast<uint32_t>(y), b1 = static_cast<uint32_t>(y >> 32);
    const uint32_t z0 = m32(a0, b0), z2 = m32(a1, b1), z1 = m32(a0 ^ a1, b0 ^ b1) ^ z0 ^ z2;
    return static_cast<uint64_t>(z0 ^ z2) | (static_cast<uint64_t>(z1 ^ alpha32(z2)) << 32);
  }
};

template <int E>
__global__ void elementwise_fp_kernel(uint8_t* __restrict__ dst, const uint8_t* __restrict__ a,
                                      const uint8_t* __restrict__ b, uint64_t nelem) {
  __shared__ uint8_t tab[1024];
  for (int i = threadIdx.x; i < 1024; i += blockDim.x) tab[i] = c_fp_tab[i];
  __syncthreads();
  const FpTab T{tab, tab + 512, tab + 768};
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nelem; i += stride) {
    uint64_t x = 0, y = 0;
#pragma unroll
    for (int k = 0; k < E; ++k) {
      x |= static_cast<uint64_t>(a[E * i + k]) << (8 * k);
      y |= static_cast<uint64_t>(b[E * i + k]) << (8 * k);
    }
    const uint64_t r = E == 1   ? T.m8(static_cast<uint32_t>(x), static_cast<uint32_t>(y))
                       : E == 2 ? T.m16(static_cast<uint32_t>(x), static_cast<uint32_t>(y))
                       : E == 4 ? T.m32(static_cast<uint32_t>(x), static_cast<uint32_t>(y))
                                : T.m64(x, y);
#pragma unroll
    for (int k = 0; k < E; ++k) dst[E * i + k] = static_cast<uint8_t>(r >> (8 * k));
  }
}

// 0x20000000 times a Gf32 element [A, B] (Gf16 halves): v = 0x2000 in the
// high half, so (A + B v) 0x2000 v = 0x2000 0x2000 B + 0x2000 (A + B) v.
__device__ __forceinline__ uint32_t gmul20000000(uint32_t w) {
  const uint32_t u = ((w ^ (w << 16)) & 0xFFFF0000u) | (w >> 16);  // [B, A + B]
  const uint32_t u1 = gmul2000x2(u);                                 // [0x2000 B, 0x2000 (A + B)]
  return (u1 & 0xFFFF0000u) | (gmul2000x2(u1) & 0x0000FFFFu);
}

__device__ __forceinline__ uint64_t ld8(const uint8_t* p) {
  if ((reinterpret_cast<uintptr_t>(p) & 7u) == 0) return *reinterpret_cast<const uint64_t*>(p);
  uint64_t v = 0;
#pragma unroll
  for (int k = 0; k < 8; ++k) v |= static_cast<uint64_t>(p[k]) << (8 * k);
  return v;
}

// GF(2^64) = Gf32[w]/(w^2 + w + 0x20000000): three word-parallel Gf32
// products and one product by the constant (src/field/gf64.rs:120-128),
// that one by doublings.
__global__ void elementwise_gf64_kernel(uint8_t* __restrict__ dst, const uint8_t* __restrict__ a,
                                        const uint8_t* __restrict__ b, uint64_t nelem) {
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t i = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < nelem; i += stride) {
    const uint64_t x = ld8(a + 8 * i), y = ld8(b + 8 * i);
    const uint32_t p = static_cast<uint32_t>(x), q = static_cast<uint32_t>(x >> 32);
    const uint32_t c = static_cast<uint32_t>(y), d = static_cast<uint32_t>(y >> 32);
    const uint32_t ac = gmul32(p, c), bd = gmul32(q, d);
    const uint32_t lo = ac ^ gmul20000000(bd);
    const uint32_t hi = gmul32(p ^ q, c ^ d) ^ ac;
    const uint64_t r = static_cast<uint64_t>(lo) | (static_cast<uint64_t>(hi) << 32);
    uint8_t* o = dst + 8 * i;
    if ((reinterpret_cast<uintptr_t>(o) & 7u) == 0) {
      *reinterpret_cast<uint64_t*>(o) = r;
    } else {
#pragma unroll
      for (int k = 0; k < 8; ++k) o[k] = static_cast<uint8_t>(r >> (8 * k));
    }
  }
}

std::atomic<bool> g_fp_ready[kMaxDevices];
std::mutex g_fp_mu;

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

// Fan-Paar fields: byte tables built on the host from the tower product,
// uploaded once per device.
static cudaError_t launch_elementwise_fp(int field, uint8_t* dst, const uint8_t* a, const uint8_t* b,
                                         uint64_t len, cudaStream_t s) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  if (!g_fp_ready[dev].load(std::memory_order_acquire)) {
    std::lock_guard<std::mutex> lk(g_fp_mu);
    uint8_t tab[1024] = {};
    uint32_t v = 1;
    for (int i = 0; i < 255; ++i) {
      tab[i] = tab[i + 255] = static_cast<uint8_t>(v);
      tab[512 + v] = static_cast<uint8_t>(i);
      v = fp_mul(v, 0x2D, 8);
    }
    for (uint32_t x = 0; x < 256; ++x) tab[768 + x] = static_cast<uint8_t>(fp_mul_alpha(x, 8));
    e = cudaMemcpyToSymbol(c_fp_tab, tab, sizeof tab);
    if (e != cudaSuccess) return e;
    g_fp_ready[dev].store(true, std::memory_order_release);
  }
  const int E = field_bytes(field);
  const uint64_t nelem = len / E;
  uint64_t want = (nelem + 255) / 256, cap = static_cast<uint64_t>(sm_count()) * 8;
  const unsigned blocks = static_cast<unsigned>(want < cap ? want : cap);
  if (E == 1)
    elementwise_fp_kernel<1><<<blocks, 256, 0, s>>>(dst, a, b, nelem);
  else if (E == 2)
    elementwise_fp_kernel<2><<<blocks, 256, 0, s>>>(dst, a, b, nelem);
  else if (E == 4)
    elementwise_fp_kernel<4><<<blocks, 256, 0, s>>>(dst, a, b, nelem);
  else
    elementwise_fp_kernel<8><<<blocks, 256, 0, s>>>(dst, a, b, nelem);
  return cudaGetLastError();
}

cudaError_t launch_elementwise(int field, uint8_t* dst, const uint8_t* a, const uint8_t* b,
                               uint64_t len, cudaStream_t s) {
  if (!len) return cudaSuccess;
  const int E = field_bytes(field);
  if (E <= 0 || len % E) return cudaErrorInvalidValue;
  if (field == kFp8 || field == kFp16 || field == kFp32 || field == kFp64)
    return launch_elementwise_fp(field, dst, a, b, len, s);
  if (field == kGf64) {
    const uint64_t nelem = len / 8;
    uint64_t want = (nelem + 255) / 256, cap = static_cast<uint64_t>(sm_count()) * 8;
    elementwise_gf64_kernel<<<static_cast<unsigned>(want < cap ? want : cap), 256, 0, s>>>(dst, a, b, nelem);
    return cudaGetLastError();
  }
  const uint64_t ad = reinterpret_cast<uintptr_t>(dst) & 15;
  uint64_t head = len, nvec = 0;
  if (ad == (reinterpret_cast<uintptr_t>(a) & 15) && ad == (reinterpret_cast<uintptr_t>(b) & 15)) {
    const uint64_t h = (16 - ad) & 15;
    if (h % E == 0 && h <= len) {
      head = h;
      nvec = (len - h) / 16;
    }
  }
  const uint64_t work = nvec + (len - 16 * nvec) / E;
  uint64_t want = (work + 255) / 256, cap = static_cast<uint64_t>(sm_count()) * 8;
  const unsigned blocks = static_cast<unsigned>(want < cap ? want : cap);
  switch (field) {
    case kGf8B: elementwise_kernel<kGf8B><<<blocks, 256, 0, s>>>(dst, a, b, len, head, nvec); break;
    case kGf8D: elementwise_kernel<kGf8D><<<blocks, 256, 0, s>>>(dst, a, b, len, head, nvec); break;
    case kGf16: elementwise_kernel<kGf16><<<blocks, 256, 0, s>>>(dst, a, b, len, head, nvec); break;
    case kGf32: elementwise_kernel<kGf32><<<blocks, 256, 0, s>>>(dst, a, b, len, head, nvec); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace fgfc
