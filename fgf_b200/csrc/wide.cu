// wide.cu -- the matrix ops for the 8-byte fields (GF(2^64), Fan-Paar
// GF(2^64)).
//
// The reference runs these fields on its portable scalar kernel
// (src/kernel/gf64.rs, src/kernel/fan_paar.rs: "every other Fan-Paar field
// ... uses the portable scalar kernel"). Here one kernel computes every
// shape: rows[j] (^)= XOR_t c[t][j] * src_t over 8-byte elements. Products
// come from split-nibble tables built on the host from the images of single
// input bits (gf_host.hpp: coeff_images), the same derivation as for the
// narrower fields: per (source t, input byte p, 4-byte output group g) a
// 16-entry table for the low nibble and one for the high nibble. A row of
// 8-byte elements is two groups. One thread folds one element column: 8 input
// bytes x 2 lookups x 2m groups per source, accumulators in registers, one
// 8-byte write per row. Tables live in shared memory; sources are processed in
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

constexpr int kWideRows = 8;                         // rows per launch (16 groups)
constexpr int kWideSrc = 64;                         // sources per launch
constexpr int kWideInlineWords = 7168;               // inline tables: 28 KiB of launch parameters
constexpr size_t kWideSmemBytes = 160 * 1024;        // shared-memory tables per CTA
constexpr int kWideThreads = 256;

struct WideLaunch {
  const uint32_t* tables;  // device tables [(t * 8 + p) * gstride + g0 + g][32], or nullptr: inline_tab
  uint32_t gstride, g0;
  uint32_t k, m;           // sources and rows of this launch
  uint32_t ovr;
  uint64_t nelem;          // 8-byte elements per row
  const uint8_t* src[kWideSrc];
  uint8_t* dst[kWideRows];
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

// G = 2 m groups per source byte (m rows of this launch).
template <int G>
__global__ void __launch_bounds__(kWideThreads) wide_kernel(const __grid_constant__ WideLaunch a) {
  extern __shared__ uint32_t tab[];  // [(t * 8 + p) * G + g][32]
  const uint32_t* from = a.tables ? a.tables : a.inline_tab;
  const uint32_t nwords = a.k * 8u * G * 32u;
  for (uint32_t i = threadIdx.x; i < nwords; i += blockDim.x) {
    const uint32_t slot = i >> 5, w = i & 31u;
    const uint32_t tp = slot / G, g = slot % G;
    tab[i] = from[(static_cast<size_t>(tp) * a.gstride + a.g0 + g) * 32u + w];
  }
  __syncthreads();
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  for (uint64_t e = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x; e < a.nelem; e += stride) {
    uint32_t acc[G];
#pragma unroll
    for (int g = 0; g < G; ++g) acc[g] = 0;
    uint64_t next = load8(a.src[0] + 8 * e);
    for (uint32_t t = 0; t < a.k; ++t) {
      const uint64_t x = next;  // the next source's element is in flight during this one's lookups
      if (t + 1 < a.k) next = load8(a.src[t + 1] + 8 * e);
      const uint32_t* tt = tab + t * 8u * G * 32u;
#pragma unroll
      for (int p = 0; p < 8; ++p) {
        const uint32_t b = static_cast<uint32_t>(x >> (8 * p)) & 0xFFu;
        const uint32_t* tp = tt + p * G * 32;
#pragma unroll
        for (int g = 0; g < G; ++g) acc[g] ^= tp[g * 32 + (b & 15u)] ^ tp[g * 32 + 16 + (b >> 4)];
      }
    }
#pragma unroll
    for (int j = 0; j < G / 2; ++j)
      if (j < static_cast<int>(a.m))
        store8(a.dst[j] + 8 * e, static_cast<uint64_t>(acc[2 * j]) | (static_cast<uint64_t>(acc[2 * j + 1]) << 32),
               a.ovr != 0);
  }
}

using WideFn = void (*)(WideLaunch);

WideFn wide_kernel_for(int groups) {
  switch (groups) {
    case 2: return wide_kernel<2>;
    case 4: return wide_kernel<4>;
    case 6: return wide_kernel<6>;
    case 8: return wide_kernel<8>;
    case 10: return wide_kernel<10>;
    case 12: return wide_kernel<12>;
    case 14: return wide_kernel<14>;
    case 16: return wide_kernel<16>;
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
  static thread_local WideLaunch a;  // large (inline tables): keep off the stack
  for (size_t r0 = 0; r0 < m; r0 += kWideRows) {
    const size_t nr = std::min<size_t>(kWideRows, m - r0);
    const int G = static_cast<int>(2 * nr);
    const size_t per_src_words = 8u * G * 32u;
    size_t kc = inl ? kWideInlineWords / per_src_words : (kWideSmemBytes / 4) / per_src_words;
    kc = std::max<size_t>(1, std::min<size_t>({kc, static_cast<size_t>(kWideSrc), k}));
    WideFn fn = wide_kernel_for(G);
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
        // groups 2 r0 .. 2 (r0 + nr) of sources t0 .. t0 + kk
        build_compact_tables(field, host_coeffs, m, t0, kk, 2 * r0, G, a.inline_tab);
        a.tables = nullptr;
        a.gstride = static_cast<uint32_t>(G);
        a.g0 = 0;
      } else {
        a.tables = dev_tables + t0 * 8 * gstride * kCompactWords;
        a.gstride = static_cast<uint32_t>(gstride);
        a.g0 = static_cast<uint32_t>(2 * r0);
      }
      const size_t smem = kk * per_src_words * 4;
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
