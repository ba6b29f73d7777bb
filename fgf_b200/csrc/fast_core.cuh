// fast_core.cuh -- device building blocks shared by the single-call kernels
// (kernels.cu) and the persistent batch kernels (batch.cu).
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

#include "internal.hpp"

namespace fgfc {

extern __shared__ __align__(16) uint8_t g_smem[];

__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t s) {
  return __byte_perm(a, b, s);
}

__device__ __forceinline__ uint32_t lds_at(uint32_t off) {
  return *reinterpret_cast<const uint32_t*>(g_smem + off);
}

// Source loads: read-only path without L1 allocation (sources are read once).
__device__ __forceinline__ uint4 ldg16(const uint8_t* p) {
  uint4 v;
  asm volatile("ld.global.nc.L1::no_allocate.v4.u32 {%0,%1,%2,%3}, [%4];"
               : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
               : "l"(p));
  return v;
}

// Pull a line into L2 ahead of its load (the next grid-stride iteration's
// column); this keeps more DRAM requests in flight than the registers of
// 1024-thread CTAs allow.
__device__ __forceinline__ void prefetch_l2(const uint8_t* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }

// ---------------------------------------------------------------- byte-table layout
//
// Gf8 fields with at most 4 rows (one table group) and a compile-time number
// of sources K. Sources t < kByteSrc get a full 256-entry product table (one
// lookup per source byte, 32 KiB with the 32 lane copies; two tables share
// each 64 KiB page, at byte offsets 0 and 128 of every 256-byte row), the
// rest keep split-nibble tables in 4 KiB slots after the three byte-table
// pages. With K fixed every table address is a PRMT of the data byte plus an
// immediate.
constexpr int kByteSrc = 6;
constexpr int kFastMaxK = 14;
constexpr int kFastThreads = 1024;
constexpr uint32_t kNibbleBase = 3u * 65536u;

template <int K>
struct FastLayout {
  static constexpr int NB = K < kByteSrc ? K : kByteSrc;  // byte-table sources
  static constexpr int NN = K - NB;                       // nibble-table sources
  static constexpr uint32_t tables = NN ? kNibbleBase + NN * kSlotBytes : ((NB + 1) / 2) * 65536u;
  static constexpr uint32_t smem = tables + K * kCompactWords * 4u;  // + compact staging
};

// Expand the compact tables of K sources (plan layout: source t at
// ((t * gstride + g0) * 32)) into the byte-table layout. `tables` is a device
// pointer, or null to read `inl` (launch parameters). The compact words are
// staged in shared memory first (one independent load per thread) and every
// entry's 32 lane copies are written as 8 identical 16-byte stores.
template <int K>
__device__ __forceinline__ void fill_fast(const uint32_t* tables, const uint32_t* inl, uint32_t gstride,
                                          uint32_t g0) {
  using L = FastLayout<K>;
  uint32_t* stage = reinterpret_cast<uint32_t*>(g_smem) + L::tables / 4;
  for (uint32_t i = threadIdx.x; i < K * kCompactWords; i += blockDim.x) {
    const uint32_t src = ((i >> 5) * gstride + g0) * kCompactWords + (i & 31u);
    stage[i] = tables ? __ldg(tables + src) : inl[src];
  }
  __syncthreads();
  // byte tables: word index = page * 16384 + x * 64 + half * 32 + lane
  uint4* st4 = reinterpret_cast<uint4*>(g_smem);
#pragma unroll 4
  for (uint32_t i = threadIdx.x; i < L::NB * 2048u; i += blockDim.x) {
    const uint32_t t = i >> 11, x = (i >> 3) & 255u, q = i & 7u;
    const uint32_t v = stage[t * kCompactWords + (x & 15u)] ^ stage[t * kCompactWords + 16u + (x >> 4)];
    st4[(t >> 1) * 4096u + x * 16u + (t & 1u) * 8u + q] = make_uint4(v, v, v, v);
  }
  if constexpr (L::NN > 0) {
#pragma unroll 4
    for (uint32_t i = threadIdx.x; i < L::NN * 256u; i += blockDim.x) {
      const uint32_t v =
          stage[(L::NB + (i >> 8)) * kCompactWords + ((i >> 3) & 1u) * 16u + ((i >> 4) & 15u)];
      st4[kNibbleBase / 16 + i] = make_uint4(v, v, v, v);
    }
  }
  __syncthreads();
}

// Lane / page registers of the byte-table layout.
struct FastRegs {
  uint32_t lrp[3];  // byte-table pages 0..2
  uint32_t lrn;     // nibble slots (page 3)
  __device__ __forceinline__ FastRegs() {
    const uint32_t lane4 = (threadIdx.x & 31u) * 4u;
#pragma unroll
    for (int p = 0; p < 3; ++p) lrp[p] = lane4 | (static_cast<uint32_t>(p) << 16);
    lrn = lane4 | (3u << 16);
  }
};

// Fold NW words (4 bytes each, byte b of word q is element 4q + b) of each
// of the K sources into acc (acc[e] = products for rows 0..3 of element e).
template <int K, int NW>
__device__ __forceinline__ void fast_fold(const uint32_t (&w)[K][NW], uint32_t (&acc)[4 * NW],
                                          const FastRegs& r) {
  using L = FastLayout<K>;
#pragma unroll
  for (int t = 0; t < L::NB; t += 2) {
    const uint32_t lr = r.lrp[t >> 1];
    if (t + 1 < L::NB) {
#pragma unroll
      for (int q = 0; q < NW; ++q)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const uint32_t sel = 0x7604u | (static_cast<uint32_t>(b) << 4);
          acc[4 * q + b] ^= lds_at(prmt(w[t][q], lr, sel)) ^ lds_at(prmt(w[t + 1][q], lr, sel) + 128u);
        }
    } else {
#pragma unroll
      for (int q = 0; q < NW; ++q)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const uint32_t sel = 0x7604u | (static_cast<uint32_t>(b) << 4);
          acc[4 * q + b] ^= lds_at(prmt(w[t][q], lr, sel));
        }
    }
  }
#pragma unroll
  for (int i = 0; i < L::NN; ++i) {
    const uint32_t pat = ((static_cast<uint32_t>(48 + i) & 15u) << 4) * 0x01010101u;
#pragma unroll
    for (int q = 0; q < NW; ++q) {
      const uint32_t xl = (w[L::NB + i][q] & 0x0F0F0F0Fu) | pat;
      const uint32_t xh = ((w[L::NB + i][q] >> 4) & 0x0F0F0F0Fu) | pat;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const uint32_t sel = 0x7604u | (static_cast<uint32_t>(b) << 4);
        acc[4 * q + b] ^= lds_at(prmt(xl, r.lrn, sel)) ^ lds_at(prmt(xh, r.lrn, sel) + 128u);
      }
    }
  }
}

// Row rr (0..3) of one output word from 4 element accumulators (4x4 byte
// transpose: acc[e] holds rows 0..3 of element e).
__device__ __forceinline__ uint32_t row_word4(const uint32_t* acc, int rr) {
  const uint32_t s01 = prmt(acc[0], acc[1], rr < 2 ? 0x5140u : 0x7362u);
  const uint32_t s23 = prmt(acc[2], acc[3], rr < 2 ? 0x5140u : 0x7362u);
  return prmt(s01, s23, (rr & 1) ? 0x7632u : 0x5410u);
}

// ---------------------------------------------------------------- row stores
//
// The vector paths compute 16-byte columns in the alignment of the sources.
// A destination row may start anywhere (contiguous rows of any length put
// row j at j * row_len). When a column's destination is dl = addr & 15 bytes
// past a 16-byte boundary, each lane writes the aligned 16 bytes that end
// inside its column, spliced from the previous lane's column (one warp
// shuffle per word) and its own; the ends of a run of contiguous columns are
// written bytewise. Every byte is written by exactly one lane. All 32 lanes
// of the warp must call store_vec16 together; lanes without a column pass
// valid = false.

constexpr unsigned kFullWarp = 0xffffffffu;

// Bytes [s, s + 16) of the 32-byte concatenation P || V, 0 < s < 16.
__device__ __forceinline__ uint4 splice16(const uint4& P, const uint4& V, uint32_t s) {
  uint32_t c0, c1, c2, c3, c4;
  switch (s >> 2) {
    case 0: c0 = P.x; c1 = P.y; c2 = P.z; c3 = P.w; c4 = V.x; break;
    case 1: c0 = P.y; c1 = P.z; c2 = P.w; c3 = V.x; c4 = V.y; break;
    case 2: c0 = P.z; c1 = P.w; c2 = V.x; c3 = V.y; c4 = V.z; break;
    default: c0 = P.w; c1 = V.x; c2 = V.y; c3 = V.z; c4 = V.w; break;
  }
  const uint32_t r = (s & 3u) * 8u;
  return make_uint4(__funnelshift_r(c0, c1, r), __funnelshift_r(c1, c2, r), __funnelshift_r(c2, c3, r),
                    __funnelshift_r(c3, c4, r));
}

// Bytes [b0, b1) of V to p[0 .. b1 - b0), one byte store each.
__device__ __forceinline__ void put_bytes(uint8_t* p, const uint4& V, uint32_t b0, uint32_t b1, bool ovr) {
  const uint32_t w[4] = {V.x, V.y, V.z, V.w};
#pragma unroll
  for (uint32_t b = 0; b < 16; ++b) {
    if (b < b0 || b >= b1) continue;
    const uint8_t v = static_cast<uint8_t>(w[b >> 2] >> (8 * (b & 3u)));
    uint8_t* q = p + (b - b0);
    *q = ovr ? v : static_cast<uint8_t>(*q ^ v);
  }
}

__device__ __forceinline__ void put16(uint8_t* p, uint4 o, bool ovr) {
  uint4* dp = reinterpret_cast<uint4*>(p);
  if (!ovr) {
    const uint4 d = *dp;
    o.x ^= d.x;
    o.y ^= d.y;
    o.z ^= d.z;
    o.w ^= d.w;
  }
  *dp = o;
}

// Store the 16-byte column o at p (any alignment); accumulate unless ovr.
__device__ __forceinline__ void store_vec16(uint8_t* p, const uint4& o, bool valid, bool ovr) {
  const uint64_t a = reinterpret_cast<uint64_t>(p);
  const uint32_t dl = static_cast<uint32_t>(a) & 15u;
  if (__all_sync(kFullWarp, !valid || dl == 0)) {
    if (valid) put16(p, o, ovr);
    return;
  }
  const uint32_t lane = threadIdx.x & 31u;
  const uint64_t ap = __shfl_up_sync(kFullWarp, a, 1);
  const uint64_t an = __shfl_down_sync(kFullWarp, a, 1);
  const int vp = __shfl_up_sync(kFullWarp, valid ? 1 : 0, 1);
  const int vn = __shfl_down_sync(kFullWarp, valid ? 1 : 0, 1);
  uint4 P;
  P.x = __shfl_up_sync(kFullWarp, o.x, 1);
  P.y = __shfl_up_sync(kFullWarp, o.y, 1);
  P.z = __shfl_up_sync(kFullWarp, o.z, 1);
  P.w = __shfl_up_sync(kFullWarp, o.w, 1);
  if (!valid) return;
  if (dl == 0) {
    put16(p, o, ovr);
    return;
  }
  const bool prev_ok = lane > 0 && vp && ap + 16 == a;
  const bool next_ok = lane < 31 && vn && an == a + 16;
  const uint32_t s = 16u - dl;
  if (prev_ok)
    put16(p - dl, splice16(P, o, s), ovr);  // [p - dl, p + s): previous column's tail, then ours
  else
    put_bytes(p, o, 0, s, ovr);
  if (!next_ok) put_bytes(p + s, o, s, 16, ovr);
}

// Store one 16-byte column of up to 4 rows whose destinations share the
// sources' alignment; accumulate unless overwriting.
__device__ __forceinline__ void store_col4(const uint32_t (&acc)[16], uint8_t* const* dst, uint32_t nrows,
                                           uint64_t off, bool ovr) {
#pragma unroll
  for (int rr = 0; rr < 4; ++rr) {
    if (rr >= static_cast<int>(nrows)) break;
    uint4 o;
    o.x = row_word4(&acc[0], rr);
    o.y = row_word4(&acc[4], rr);
    o.z = row_word4(&acc[8], rr);
    o.w = row_word4(&acc[12], rr);
    put16(dst[rr] + off, o, ovr);
  }
}

// The same for rows at any offset. Called by every lane of the warp;
// `valid` marks lanes holding a column.
__device__ __forceinline__ void store_col4_any(const uint32_t (&acc)[16], uint8_t* const* dst, uint32_t nrows,
                                               uint64_t off, bool ovr, bool valid) {
#pragma unroll
  for (int rr = 0; rr < 4; ++rr) {
    uint4 o;
    o.x = row_word4(&acc[0], rr);
    o.y = row_word4(&acc[4], rr);
    o.z = row_word4(&acc[8], rr);
    o.w = row_word4(&acc[12], rr);
    const bool rv = valid && rr < static_cast<int>(nrows);
    store_vec16(rv ? dst[rr] + off : nullptr, o, rv, ovr);
  }
}

}  // namespace fgfc
