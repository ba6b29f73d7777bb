// wide.cu -- the matrix ops for the 8-byte fields (GF(2^64), Fan-Paar
// GF(2^64)).
//
// The reference runs these fields on its portable scalar kernel
// (src/kernel/gf64.rs, src/kernel/fan_paar.rs: "every other Fan-Paar field
// ... uses the portable scalar kernel"). Here one kernel computes every
// shape: rows[j] (^)= XOR_t c[t][j] * src_t over 8-byte elements.
//
// Both fields are quadratic over a 4-byte base field (Gf32 for GF(2^64),
// FP32 for Fan-Paar), so with c = c0 + c1 w and x = x0 + x1 w a product
// needs three half-products (Karatsuba): A = c0 x0, B = c1 x1,
// C = (c0 + c1)(x0 + x1), then
//   GF(2^64)  (w^2 = w + beta):        lo = A + beta B,  hi = A + C
//   Fan-Paar  (X^2 = alpha X + 1):     lo = A + B,       hi = A + C + (1 + alpha) B.
// The fix-up is linear, so it is applied once per row to the sums over all
// sources. Each half-product is a GF(2)-linear map on a 32-bit word, read
// from split-nibble tables built on the host (tables.cpp:
// build_wide_tables): 8 lookups per half-product and row, 24 per source
// element and row, against 32 for the map on the whole 8-byte element;
// shared-memory lookups are what bounds this kernel. One thread folds one
// element column: accumulators A, B, C per row in registers, one 8-byte
// write per row. Tables live in shared memory; sources are processed in
// chunks that fit it (later chunks accumulate), rows in chunks of kWideRows.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "internal.hpp"

namespace fgfc {

namespace {

constexpr int kWideRows = 8;                         // rows per launch
constexpr int kWideSrc = 64;                         // sources per launch
constexpr int kWideInlineWords = 7168;               // inline tables: 28 KiB of launch parameters
constexpr size_t kWideSmemBytes = 160 * 1024;        // shared-memory tables per CTA
constexpr int kWideThreads = 256;
constexpr int kFixWords = 4 * kCompactWords;         // fix-up map: 4 input bytes x 32 words

struct WideLaunch {
  const uint32_t* tables;  // device tables [((t * 3 + P) * 4 + p) * gstride + j0 + j][32], or nullptr: inline_tab
  uint32_t gstride, j0;
  uint32_t k, m;           // sources and rows of this launch
  uint32_t ovr;
  uint64_t nelem;          // 8-byte elements per row
  const uint8_t* src[kWideSrc];
  uint8_t* dst[kWideRows];
  uint32_t fix[kFixWords];
  uint32_t inline_tab[kWideInlineWords];
};
static_assert(sizeof(WideLaunch) <= 32000, "launch parameter block too large");

__device__ __forceinline__ uint64_t load8(const uint8_t* p) {
  if ((reinterpret_cast<uintptr_t>(p) & 7u) == 0) return *reinterpret_cast<const uint64_t*>(p);
  uint64_t v = 0;
#pragma unroll
  for (int i = 0; i < 8; ++i) v |= static_cast<uint64_t>(p[i]) << (8 * i);
  return v;
}

__device__ __forceinline__ void store8(uint8_t* p, uint64_t v, bool ovr) {
  if ((reinterpret_cast<uintptr_t>(p) & 7u) == 0) {
    uint64_t* q = reinterpret_cast<uint64_t*>(p);
    *q = ovr ? v : (*q ^ v);
    return;
  }
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const uint8_t b = static_cast<uint8_t>(v >> (8 * i));
    p[i] = ovr ? b : static_cast<uint8_t>(p[i] ^ b);
  }
}

// acc[j] ^= map_j(x) for the M row maps whose input-byte-p tables start at
// tp + p * M * 32 (row j's table j * 32 further on).
template <int M>
__device__ __forceinline__ void fold_half(uint32_t (&acc)[M], const uint32_t* tp, uint32_t x) {
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const uint32_t b = (x >> (8 * p)) & 0xFFu;
    const uint32_t* s = tp + p * M * kCompactWords;
#pragma unroll
    for (int j = 0; j < M; ++j) acc[j] ^= s[j * kCompactWords + (b & 15u)] ^ s[j * kCompactWords + 16 + (b >> 4)];
  }
}

// The fix-up map applied to one word.
__device__ __forceinline__ uint32_t fixup(const uint32_t* fix, uint32_t v) {
  uint32_t r = 0;
#pragma unroll
  for (int p = 0; p < 4; ++p) {
    const uint32_t b = (v >> (8 * p)) & 0xFFu;
    r ^= fix[p * kCompactWords + (b & 15u)] ^ fix[p * kCompactWords + 16 + (b >> 4)];
  }
  return r;
}

// M rows of this launch; FP: the Fan-Paar fix-up (else GF(2^64)'s).
template <int M, bool FP>
__global__ void __launch_bounds__(kWideThreads) wide_kernel(const __grid_constant__ WideLaunch a) {
  extern __shared__ uint32_t tab[];  // [((t * 3 + P) * 4 + p) * M + j][32], then the fix-up map
  const uint32_t* from = a.tables ? a.tables : a.inline_tab;
  const uint32_t nwords = a.k * static_cast<uint32_t>(kWideSlotsPerSrcRow) * M * kCompactWords;
  for (uint32_t i = threadIdx.x; i < nwords; i += blockDim.x) {
    const uint32_t slot = i >> 5, w = i & 31u;
    const uint32_t q = slot / M, j = slot % M;
    tab[i] = from[(static_cast<size_t>(q) * a.gstride + a.j0 + j) * kCompactWords + w];
  }
  uint32_t* fix = tab + nwords;
  for (uint32_t i = threadIdx.x; i < kFixWords; i += blockDim.x) fix[i] = a.fix[i];
  __syncthreads();
  constexpr uint32_t kProd = 4u * M * kCompactWords;  // words of one half-product's tables
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t e = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < a.nelem; e += stride) {
    uint32_t accA[M], accB[M], accC[M];
#pragma unroll
    for (int j = 0; j < M; ++j) accA[j] = accB[j] = accC[j] = 0;
    uint64_t next = load8(a.src[0] + 8 * e);
    for (uint32_t t = 0; t < a.k; ++t) {
      const uint64_t x = next;  // the next source's element is in flight during this one's lookups
      if (t + 1 < a.k) next = load8(a.src[t + 1] + 8 * e);
      const uint32_t x0 = static_cast<uint32_t>(x), x1 = static_cast<uint32_t>(x >> 32);
      const uint32_t* tt = tab + t * 3u * kProd;
      fold_half<M>(accA, tt, x0);
      fold_half<M>(accB, tt + kProd, x1);
      fold_half<M>(accC, tt + 2 * kProd, x0 ^ x1);
    }
#pragma unroll
    for (int j = 0; j < M; ++j) {
      uint32_t lo, hi;
      if (FP) {
        lo = accA[j] ^ accB[j];
        hi = accA[j] ^ accC[j] ^ fixup(fix, accB[j]);
      } else {
        lo = accA[j] ^ fixup(fix, accB[j]);
        hi = accA[j] ^ accC[j];
      }
      store8(a.dst[j] + 8 * e, static_cast<uint64_t>(lo) | (static_cast<uint64_t>(hi) << 32), a.ovr != 0);
    }
  }
}

using WideFn = void (*)(WideLaunch);

template <bool FP>
WideFn wide_kernel_rows(int rows) {
  switch (rows) {
    case 1: return wide_kernel<1, FP>;
    case 2: return wide_kernel<2, FP>;
    case 3: return wide_kernel<3, FP>;
    case 4: return wide_kernel<4, FP>;
    case 5: return wide_kernel<5, FP>;
    case 6: return wide_kernel<6, FP>;
    case 7: return wide_kernel<7, FP>;
    case 8: return wide_kernel<8, FP>;
    default: return nullptr;
  }
}

std::mutex g_wide_mu;

}  // namespace

cudaError_t wide_launch(int field, const uint8_t* const* srcs, size_t k, uint8_t* const* rows, size_t m,
                        const uint64_t* host_coeffs, const uint32_t* dev_tables, size_t gstride, size_t len,
                        bool overwrite, cudaStream_t stream) {
  const size_t nelem = len / 8;
  if (!nelem || !m || !k) return cudaSuccess;
  const bool inl = dev_tables == nullptr;
  const bool fp = field == kFp64;
  static thread_local WideLaunch a;  // large (inline tables): keep off the stack
  build_wide_fixup(field, a.fix);
  for (size_t r0 = 0; r0 < m; r0 += kWideRows) {
    const size_t nr = std::min<size_t>(kWideRows, m - r0);
    const size_t per_src_words = kWideSlotsPerSrcRow * nr * kCompactWords;
    size_t kc = inl ? kWideInlineWords / per_src_words : (kWideSmemBytes / 4 - kFixWords) / per_src_words;
    kc = std::max<size_t>(1, std::min<size_t>({kc, static_cast<size_t>(kWideSrc), k}));
    WideFn fn = fp ? wide_kernel_rows<true>(static_cast<int>(nr)) : wide_kernel_rows<false>(static_cast<int>(nr));
    if (!fn) return cudaErrorInvalidValue;
    for (size_t t0 = 0; t0 < k; t0 += kc) {
      const size_t kk = std::min(kc, k - t0);
      a.k = static_cast<uint32_t>(kk);
      a.m = static_cast<uint32_t>(nr);
      a.ovr = overwrite && t0 == 0 ? 1u : 0u;
      a.nelem = nelem;
      for (size_t t = 0; t < kk; ++t) a.src[t] = srcs[t0 + t];
      for (size_t j = 0; j < nr; ++j) a.dst[j] = rows[r0 + j];
      if (inl) {
        // rows r0 .. r0 + nr of sources t0 .. t0 + kk
        build_wide_tables(field, host_coeffs, m, t0, kk, r0, nr, a.inline_tab);
        a.tables = nullptr;
        a.gstride = static_cast<uint32_t>(nr);
        a.j0 = 0;
      } else {
        a.tables = dev_tables + t0 * kWideSlotsPerSrcRow * gstride * kCompactWords;
        a.gstride = static_cast<uint32_t>(gstride);
        a.j0 = static_cast<uint32_t>(r0);
      }
      const size_t smem = (kk * per_src_words + kFixWords) * 4;
      cudaError_t e = ensure_smem_attr(reinterpret_cast<const void*>(fn), static_cast<int>(smem));
      if (e != cudaSuccess) return e;
      // One wave of resident CTAs: each loads its tables into shared memory once.
      int per_sm = 0;
      if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kWideThreads, smem) != cudaSuccess || per_sm < 1)
        per_sm = 1;
      const uint64_t want = (nelem + kWideThreads - 1) / kWideThreads;
      const unsigned grid =
          static_cast<unsigned>(std::min<uint64_t>(want, static_cast<uint64_t>(sm_count()) * static_cast<uint64_t>(per_sm)));
      {
        std::lock_guard<std::mutex> lk(g_wide_mu);
        fn<<<grid, kWideThreads, smem, stream>>>(a);
        e = cudaGetLastError();
      }
      if (e != cudaSuccess) return e;
    }
  }
  return cudaSuccess;
}

}  // namespace fgfc
