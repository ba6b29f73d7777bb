// batch.cu -- batched submissions: many stripes of uneven field, k, m and
// shard length in one persistent launch per class, driven by a device
// work-list.
//
// A submission is lowered on the host to sub-jobs (all sources of a stripe,
// the rows of at most 4 table groups) and grouped in classes:
//   * Gf8 sub-jobs of at most 4 rows and K <= 14 sources use the byte-table
//     layout (fast_core.cuh), one class per K. When every sub-job of such a
//     class shares one plan, the CTAs load the tables once and grid-stride
//     over the flattened columns of all stripes (the stripes travel in the
//     launch parameters); otherwise they claim work items.
//   * everything else uses split-nibble tables, one class per (element
//     width, groups); tables that do not fit at once are processed in source
//     chunks inside the kernel.
// Work items are (sub-job, part) pairs: part p of P covers the sub-job's
// column vectors p*T + tid + j*P*T (T threads per CTA), so CTAs holding
// consecutive items sweep one window of memory together; the remaining parts
// cover the 4-byte scalar groups of heads, tails and unaligned stripes.
// Persistent CTAs claim items from an atomic counter and reload their
// shared-memory tables only when an item needs a different plan. The
// descriptor blob (jobs, pointers, items, counters) goes to the device in one
// copy, and a submission whose structure repeats replays a captured graph.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/fgf_cuda.h"
#include "fast_core.cuh"
#include "internal.hpp"

namespace fgfc {

namespace {

struct BatchJob {
  const uint32_t* tables;  // plan compact tables (matrix orientation)
  uint64_t len;            // bytes per row
  uint64_t head;           // scalar bytes before the vector body
  uint64_t nvec;           // 16-byte vectors in the body
  uint32_t gstride, g0;    // plan groups per (source, plane); first group of this sub-job
  uint32_t k, nrows;       // sources; rows of this sub-job
  uint32_t ovr;            // 1 = overwrite
  uint32_t src_idx, dst_idx;
  uint32_t nv_items;       // vector items; scalar items follow
};

constexpr int kThreads = 512;
constexpr uint32_t kVecPerItem = 8 * kThreads;
constexpr uint32_t kGroupsPerItem = kThreads;
constexpr uint32_t kFastVecPerItem = 8 * kFastThreads;
constexpr uint32_t kFastGroupsPerItem = kFastThreads;
constexpr uint32_t kClaim = 2;  // items claimed per atomic

// ---------------------------------------------------------------- nibble classes

// Expand compact tables of sources [t0, t0 + kk) into the replicated
// nibble layout (slot = (t * E + p) * G + g, 4 KiB each), via a staging copy.
template <int E, int G>
__device__ void fill_chunk(const BatchJob& J, uint32_t t0, uint32_t kk) {
  const uint32_t nslots = kk * E * G;
  uint32_t* stage = reinterpret_cast<uint32_t*>(g_smem) + kMaxSlots * 1024u;
  __syncthreads();  // previous tables no longer read
  for (uint32_t i = threadIdx.x; i < nslots * kCompactWords; i += blockDim.x) {
    const uint32_t slot = i >> 5;
    const uint32_t tp = t0 * E + slot / G;
    stage[i] = __ldg(J.tables + (tp * J.gstride + J.g0 + slot % G) * kCompactWords + (i & 31u));
  }
  __syncthreads();
  uint4* st4 = reinterpret_cast<uint4*>(g_smem);
#pragma unroll 4
  for (uint32_t i = threadIdx.x; i < nslots * 256u; i += blockDim.x) {
    const uint32_t v = stage[(i >> 8) * kCompactWords + ((i >> 3) & 1u) * 16u + ((i >> 4) & 15u)];
    st4[i] = make_uint4(v, v, v, v);
  }
  __syncthreads();
}

template <int E, int G>
struct Ctx {
  uint32_t pat;
  uint32_t lr[E];
  __device__ __forceinline__ Ctx(uint32_t t, uint32_t lane4) {
    pat = 0;
#pragma unroll
    for (int b = 0; b < 4; ++b) pat |= (((t * E + (b % E)) * G) & 15u) << (8 * b + 4);
#pragma unroll
    for (int p = 0; p < E; ++p) lr[p] = lane4 | ((((t * E + p) * G) >> 4) << 16);
  }
};

template <int E, int G, int NE>
__device__ __forceinline__ void fold(uint32_t w, const Ctx<E, G>& c, uint32_t (&acc)[G][NE], int e0) {
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

template <int E, int G, int NE>
__device__ __forceinline__ uint32_t out_word(const uint32_t (&acc)[G][NE], int g, int rr, int q) {
  if (E == 1) {
    return row_word4(&acc[g][4 * q], rr);
  } else if (E == 2) {
    return prmt(acc[g][2 * q], acc[g][2 * q + 1], rr ? 0x7632u : 0x5410u);
  } else {
    return acc[g][q];
  }
}

// One vector item of a sub-job, for sources [t0, t0 + kk) whose tables are
// resident; `ovr` overwrites, otherwise the destination is accumulated.
// SHIFT: some row is not at the sources' offset within 16 bytes; whole warps
// then iterate together (the row stores shuffle between lanes) and lanes past
// the end reload the last column.
template <int E, int G, bool SHIFT>
__device__ void vector_item(const BatchJob& J, const uint64_t* ptrs, uint32_t part, uint32_t t0,
                            uint32_t kk, bool ovr) {
  constexpr int NE = 16 / E, R = 4 / E;
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lane4 = lane * 4u;
  const uint64_t step = static_cast<uint64_t>(J.nv_items) * blockDim.x;
  for (uint64_t vb = static_cast<uint64_t>(part) * blockDim.x + threadIdx.x - (SHIFT ? lane : 0u); vb < J.nvec;
       vb += step) {
    const uint64_t v = SHIFT ? vb + lane : vb;
    const bool valid = !SHIFT || v < J.nvec;
    const uint64_t off = J.head + (valid ? v : J.nvec - 1) * 16u;
    uint32_t acc[G][NE];
#pragma unroll
    for (int g = 0; g < G; ++g)
#pragma unroll
      for (int e = 0; e < NE; ++e) acc[g][e] = 0;
    const uint8_t* const* srcs = reinterpret_cast<const uint8_t* const*>(ptrs + J.src_idx + t0);
    uint4 cur = ldg16(srcs[0] + off);
    for (uint32_t t = 0; t < kk; ++t) {
      uint4 nxt = cur;
      if (t + 1 < kk) nxt = ldg16(srcs[t + 1] + off);
      const Ctx<E, G> c(t, lane4);
      fold<E, G, NE>(cur.x, c, acc, 0);
      fold<E, G, NE>(cur.y, c, acc, 4 / E);
      fold<E, G, NE>(cur.z, c, acc, 2 * (4 / E));
      fold<E, G, NE>(cur.w, c, acc, 3 * (4 / E));
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
          const bool rv = valid && row < J.nrows;
          store_vec16(rv ? reinterpret_cast<uint8_t*>(ptrs[J.dst_idx + row]) + off : nullptr, o, rv, ovr);
        } else {
          if (row < J.nrows) put16(reinterpret_cast<uint8_t*>(ptrs[J.dst_idx + row]) + off, o, ovr);
        }
      }
  }
}

// One scalar item: 4-byte groups of the head [0, head) and the tail
// [head + 16 * nvec, len) of every row, byte loads and stores.
template <int E, int G>
__device__ void scalar_item(const BatchJob& J, const uint64_t* ptrs, uint32_t part, uint32_t t0,
                            uint32_t kk, bool ovr) {
  constexpr int R = 4 / E;
  const uint32_t lane4 = (threadIdx.x & 31u) * 4u;
  const uint64_t tail0 = J.head + J.nvec * 16u;
  const uint64_t n0 = (J.head + 3) / 4, n1 = (J.len - tail0 + 3) / 4;
  const uint64_t gi = static_cast<uint64_t>(part) * kGroupsPerItem + threadIdx.x;
  // every thread runs the lookups (uniform control flow); only threads with
  // a group in range touch memory
  const bool live = gi < n0 + n1;
  const uint64_t off = !live ? 0 : (gi < n0 ? 4 * gi : tail0 + 4 * (gi - n0));
  const uint64_t end = !live ? 0 : (gi < n0 ? J.head : J.len);
  const int nb = !live ? 0 : static_cast<int>(end - off < 4 ? end - off : 4);
  uint32_t acc[G][4 / E];
#pragma unroll
  for (int g = 0; g < G; ++g)
#pragma unroll
    for (int e = 0; e < 4 / E; ++e) acc[g][e] = 0;
  for (uint32_t t = 0; t < kk; ++t) {
    const uint8_t* s = reinterpret_cast<const uint8_t*>(ptrs[J.src_idx + t0 + t]) + off;
    uint32_t w = 0;
    for (int b = 0; b < nb; ++b) w |= static_cast<uint32_t>(s[b]) << (8 * b);
    const Ctx<E, G> c(t, lane4);
    fold<E, G, 4 / E>(w, c, acc, 0);
  }
  if (!live) return;
#pragma unroll
  for (int g = 0; g < G; ++g)
#pragma unroll
    for (int rr = 0; rr < R; ++rr) {
      const uint32_t row = g * R + rr;
      if (row >= J.nrows) continue;
      uint32_t o;
      if (E == 1) {
        o = row_word4(&acc[g][0], rr);
      } else if (E == 2) {
        o = prmt(acc[g][0], acc[g][1], rr ? 0x7632u : 0x5410u);
      } else {
        o = acc[g][0];
      }
      uint8_t* d = reinterpret_cast<uint8_t*>(ptrs[J.dst_idx + row]) + off;
      for (int b = 0; b < nb; ++b) {
        const uint8_t v = static_cast<uint8_t>(o >> (8 * b));
        d[b] = ovr ? v : static_cast<uint8_t>(d[b] ^ v);
      }
    }
}

// Persistent work-list kernel for one nibble (E, G) class.
template <int E, int G, bool SHIFT>
__global__ void __launch_bounds__(kThreads, 1)
    batch_kernel(const BatchJob* __restrict__ jobs, const uint64_t* __restrict__ ptrs,
                 const uint2* __restrict__ items, uint32_t nitems, uint32_t* counter) {
  __shared__ uint32_t s_item;
  __shared__ const uint32_t* s_tab;
  __shared__ uint32_t s_g0, s_t0;
  const uint32_t kc = kMaxSlots / (E * G);  // sources whose tables fit at once
  if (threadIdx.x == 0) {
    s_tab = nullptr;
    s_g0 = s_t0 = 0xFFFFFFFFu;
  }
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(counter, kClaim);
    __syncthreads();
    const uint32_t first = s_item;
    if (first >= nitems) break;
    for (uint32_t it = first; it < first + kClaim && it < nitems; ++it) {
      const uint2 wi = items[it];
      const BatchJob J = jobs[wi.x];
      const uint32_t nchunks = (J.k + kc - 1) / kc;
      for (uint32_t c = 0; c < nchunks; ++c) {
        const uint32_t t0 = c * kc, kk = min(kc, J.k - t0);
        __syncthreads();
        const bool resident = s_tab == J.tables && s_g0 == J.g0 && s_t0 == t0;
        if (!resident) {
          fill_chunk<E, G>(J, t0, kk);
          if (threadIdx.x == 0) {
            s_tab = J.tables;
            s_g0 = J.g0;
            s_t0 = t0;
          }
        }
        const bool ovr = J.ovr && c == 0;
        if (wi.y < J.nv_items)
          vector_item<E, G, SHIFT>(J, ptrs, wi.y, t0, kk, ovr);
        else
          scalar_item<E, G>(J, ptrs, wi.y - J.nv_items, t0, kk, ovr);
        __syncthreads();  // chunk c's writes precede chunk c + 1's reads of the same rows
      }
    }
  }
}

// ---------------------------------------------------------------- Gf16 by byte half-products

// Gf16 = Gf8B[u]/(u^2 + u + 0x20) (src/field/gf16.rs:143-153): with
// c = c0 + c1 u and x = a + b u, A = c0 a, B = c1 b, C = (c0 + c1)(a + b)
// give c x = (A + 0x20 B) + (A + C) u. Each byte half-product is a Gf8
// nibble fold whose table word holds 4 rows, so an element costs 3 x 2
// lookups per 4 rows instead of 2 x 2 per 2 rows. The tables are those of
// 3 "virtual sources" per source (3t + P, tables.cpp: build_kara16_tables).

// v * 0x20 in every byte of v over Gf8B (x^8 + x^4 + x^3 + x + 1).
__device__ __forceinline__ uint32_t mul20_4(uint32_t v) {
#pragma unroll
  for (int i = 0; i < 5; ++i) v = ((v & 0x7F7F7F7Fu) << 1) ^ (((v >> 7) & 0x01010101u) * 0x1Bu);
  return v;
}

// Row word of elements e, e + 1 (lo and hi words: byte r = row 4q + r).
__device__ __forceinline__ uint32_t k16_word(uint32_t lo0, uint32_t hi0, uint32_t lo1, uint32_t hi1, int r) {
  const uint32_t sel = static_cast<uint32_t>(r) | ((4u + static_cast<uint32_t>(r)) << 4);
  return prmt(prmt(lo0, hi0, sel), prmt(lo1, hi1, sel), 0x5410u);
}

template <int GK, int NE>
__device__ __forceinline__ void k16_finish(uint32_t (&A)[GK][NE], uint32_t (&B)[GK][NE], uint32_t (&C)[GK][NE]) {
#pragma unroll
  for (int q = 0; q < GK; ++q)
#pragma unroll
    for (int e = 0; e < NE; ++e) {
      B[q][e] = A[q][e] ^ mul20_4(B[q][e]);  // lo
      C[q][e] ^= A[q][e];                    // hi
    }
}

template <int GK, bool SHIFT>
__device__ void vector_item_k16(const BatchJob& J, const uint64_t* ptrs, uint32_t part, uint32_t t0, uint32_t kk,
                                bool ovr) {
  const uint32_t lane = threadIdx.x & 31u;
  const uint32_t lane4 = lane * 4u;
  const uint64_t step = static_cast<uint64_t>(J.nv_items) * blockDim.x;
  for (uint64_t vb = static_cast<uint64_t>(part) * blockDim.x + threadIdx.x - (SHIFT ? lane : 0u); vb < J.nvec;
       vb += step) {
    const uint64_t v = SHIFT ? vb + lane : vb;
    const bool valid = !SHIFT || v < J.nvec;
    const uint64_t off = J.head + (valid ? v : J.nvec - 1) * 16u;
    uint32_t A[GK][8], B[GK][8], C[GK][8];
#pragma unroll
    for (int q = 0; q < GK; ++q)
#pragma unroll
      for (int e = 0; e < 8; ++e) A[q][e] = B[q][e] = C[q][e] = 0;
    const uint8_t* const* srcs = reinterpret_cast<const uint8_t* const*>(ptrs + J.src_idx + t0);
    uint4 cur = ldg16(srcs[0] + off);
    for (uint32_t t = 0; t < kk; ++t) {
      uint4 nxt = cur;
      if (t + 1 < kk) nxt = ldg16(srcs[t + 1] + off);
      // low and high bytes of the 8 elements
      const uint32_t a0 = prmt(cur.x, cur.y, 0x6420u), a1 = prmt(cur.z, cur.w, 0x6420u);
      const uint32_t b0 = prmt(cur.x, cur.y, 0x7531u), b1 = prmt(cur.z, cur.w, 0x7531u);
      const Ctx<1, GK> ca(3u * t, lane4), cb(3u * t + 1u, lane4), cc(3u * t + 2u, lane4);
      fold<1, GK, 8>(a0, ca, A, 0);
      fold<1, GK, 8>(a1, ca, A, 4);
      fold<1, GK, 8>(b0, cb, B, 0);
      fold<1, GK, 8>(b1, cb, B, 4);
      fold<1, GK, 8>(a0 ^ b0, cc, C, 0);
      fold<1, GK, 8>(a1 ^ b1, cc, C, 4);
      cur = nxt;
    }
    k16_finish<GK, 8>(A, B, C);
#pragma unroll
    for (int q = 0; q < GK; ++q)
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const uint32_t row = 4 * q + r;
        uint4 o;
        o.x = k16_word(B[q][0], C[q][0], B[q][1], C[q][1], r);
        o.y = k16_word(B[q][2], C[q][2], B[q][3], C[q][3], r);
        o.z = k16_word(B[q][4], C[q][4], B[q][5], C[q][5], r);
        o.w = k16_word(B[q][6], C[q][6], B[q][7], C[q][7], r);
        if constexpr (SHIFT) {
          const bool rv = valid && row < J.nrows;
          store_vec16(rv ? reinterpret_cast<uint8_t*>(ptrs[J.dst_idx + row]) + off : nullptr, o, rv, ovr);
        } else {
          if (row < J.nrows) put16(reinterpret_cast<uint8_t*>(ptrs[J.dst_idx + row]) + off, o, ovr);
        }
      }
  }
}

// Heads and tails: 4-byte groups (two elements) with byte loads and stores.
template <int GK>
__device__ void scalar_item_k16(const BatchJob& J, const uint64_t* ptrs, uint32_t part, uint32_t t0, uint32_t kk,
                                bool ovr) {
  const uint32_t lane4 = (threadIdx.x & 31u) * 4u;
  const uint64_t tail0 = J.head + J.nvec * 16u;
  const uint64_t n0 = (J.head + 3) / 4, n1 = (J.len - tail0 + 3) / 4;
  const uint64_t gi = static_cast<uint64_t>(part) * kGroupsPerItem + threadIdx.x;
  const bool live = gi < n0 + n1;
  const uint64_t off = !live ? 0 : (gi < n0 ? 4 * gi : tail0 + 4 * (gi - n0));
  const uint64_t end = !live ? 0 : (gi < n0 ? J.head : J.len);
  const int nb = !live ? 0 : static_cast<int>(end - off < 4 ? end - off : 4);
  uint32_t A[GK][4], B[GK][4], C[GK][4];
#pragma unroll
  for (int q = 0; q < GK; ++q)
#pragma unroll
    for (int e = 0; e < 4; ++e) A[q][e] = B[q][e] = C[q][e] = 0;
  for (uint32_t t = 0; t < kk; ++t) {
    const uint8_t* s = reinterpret_cast<const uint8_t*>(ptrs[J.src_idx + t0 + t]) + off;
    uint32_t w = 0;
    for (int b = 0; b < nb; ++b) w |= static_cast<uint32_t>(s[b]) << (8 * b);
    const uint32_t a = prmt(w, 0u, 0x4420u), bb = prmt(w, 0u, 0x4431u);  // [a0 a1 0 0], [b0 b1 0 0]
    const Ctx<1, GK> ca(3u * t, lane4), cb(3u * t + 1u, lane4), cc(3u * t + 2u, lane4);
    fold<1, GK, 4>(a, ca, A, 0);
    fold<1, GK, 4>(bb, cb, B, 0);
    fold<1, GK, 4>(a ^ bb, cc, C, 0);
  }
  if (!live) return;
  k16_finish<GK, 4>(A, B, C);
#pragma unroll
  for (int q = 0; q < GK; ++q)
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const uint32_t row = 4 * q + r;
      if (row >= J.nrows) continue;
      const uint32_t o = k16_word(B[q][0], C[q][0], B[q][1], C[q][1], r);
      uint8_t* d = reinterpret_cast<uint8_t*>(ptrs[J.dst_idx + row]) + off;
      for (int b = 0; b < nb; ++b) {
        const uint8_t v = static_cast<uint8_t>(o >> (8 * b));
        d[b] = ovr ? v : static_cast<uint8_t>(d[b] ^ v);
      }
    }
}

// Persistent work-list kernel of a Gf16 half-product class: GK row quads.
template <int GK, bool SHIFT>
__global__ void __launch_bounds__(kThreads, 1)
    batch_kernel_k16(const BatchJob* __restrict__ jobs, const uint64_t* __restrict__ ptrs,
                     const uint2* __restrict__ items, uint32_t nitems, uint32_t* counter) {
  __shared__ uint32_t s_item;
  __shared__ const uint32_t* s_tab;
  __shared__ uint32_t s_g0, s_t0;
  const uint32_t kc = kMaxSlots / (3 * GK);  // sources whose tables fit at once
  if (threadIdx.x == 0) {
    s_tab = nullptr;
    s_g0 = s_t0 = 0xFFFFFFFFu;
  }
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(counter, kClaim);
    __syncthreads();
    const uint32_t first = s_item;
    if (first >= nitems) break;
    for (uint32_t it = first; it < first + kClaim && it < nitems; ++it) {
      const uint2 wi = items[it];
      const BatchJob J = jobs[wi.x];
      const uint32_t nchunks = (J.k + kc - 1) / kc;
      for (uint32_t c = 0; c < nchunks; ++c) {
        const uint32_t t0 = c * kc, kk = min(kc, J.k - t0);
        __syncthreads();
        const bool resident = s_tab == J.tables && s_g0 == J.g0 && s_t0 == t0;
        if (!resident) {
          fill_chunk<1, GK>(J, 3 * t0, 3 * kk);
          if (threadIdx.x == 0) {
            s_tab = J.tables;
            s_g0 = J.g0;
            s_t0 = t0;
          }
        }
        const bool ovr = J.ovr && c == 0;
        if (wi.y < J.nv_items)
          vector_item_k16<GK, SHIFT>(J, ptrs, wi.y, t0, kk, ovr);
        else
          scalar_item_k16<GK>(J, ptrs, wi.y - J.nv_items, t0, kk, ovr);
        __syncthreads();  // chunk c's writes precede chunk c + 1's reads of the same rows
      }
    }
  }
}

// ---------------------------------------------------------------- byte-table classes

// Work-list kernel for Gf8 sub-jobs of at most 4 rows and exactly K sources.
// The plan's tables stay resident across consecutive items of one plan.
template <int K, bool SHIFT>
__global__ void __launch_bounds__(kFastThreads, 1)
    batch_fast_kernel(const BatchJob* __restrict__ jobs, const uint64_t* __restrict__ ptrs,
                      const uint2* __restrict__ items, uint32_t nitems, uint32_t* counter) {
  __shared__ uint32_t s_item;
  __shared__ const uint32_t* s_tab;
  __shared__ uint32_t s_g0;
  __shared__ const uint8_t* s_src[K];
  __shared__ uint8_t* s_dst[4];
  if (threadIdx.x == 0) {
    s_tab = nullptr;
    s_g0 = 0xFFFFFFFFu;
  }
  const FastRegs r;
  for (;;) {
    __syncthreads();
    if (threadIdx.x == 0) s_item = atomicAdd(counter, kClaim);
    __syncthreads();
    const uint32_t first = s_item;
    if (first >= nitems) break;
    for (uint32_t it = first; it < first + kClaim && it < nitems; ++it) {
      const uint2 wi = items[it];
      const BatchJob J = jobs[wi.x];
      __syncthreads();  // the previous item is done with tables and pointers
      const bool resident = s_tab == J.tables && s_g0 == J.g0;
      if (threadIdx.x < K) s_src[threadIdx.x] = reinterpret_cast<const uint8_t*>(ptrs[J.src_idx + threadIdx.x]);
      if (threadIdx.x < J.nrows) s_dst[threadIdx.x] = reinterpret_cast<uint8_t*>(ptrs[J.dst_idx + threadIdx.x]);
      if (!resident) {
        fill_fast<K>(J.tables, nullptr, J.gstride, J.g0);
        if (threadIdx.x == 0) {
          s_tab = J.tables;
          s_g0 = J.g0;
        }
      }
      __syncthreads();
      const bool ovr = J.ovr != 0;
      if (wi.y < J.nv_items) {
        const uint64_t step = static_cast<uint64_t>(J.nv_items) * blockDim.x;
        const uint32_t lane = threadIdx.x & 31u;
        // SHIFT: whole warps iterate together (see vector_item)
        for (uint64_t vb = static_cast<uint64_t>(wi.y) * blockDim.x + threadIdx.x - (SHIFT ? lane : 0u);
             vb < J.nvec; vb += step) {
          const uint64_t v = SHIFT ? vb + lane : vb;
          const bool valid = !SHIFT || v < J.nvec;
          const uint64_t off = J.head + (valid ? v : J.nvec - 1) * 16u;
          if (v + step < J.nvec) {  // this thread's next column: into L2 now
#pragma unroll
            for (int t = 0; t < K; ++t) prefetch_l2(s_src[t] + off + step * 16u);
          }
          uint32_t w[K][4];
#pragma unroll
          for (int t = 0; t < K; ++t) {
            const uint4 x = ldg16(s_src[t] + off);
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
            store_col4_any(acc, s_dst, J.nrows, off, ovr, valid);
          else
            store_col4(acc, s_dst, J.nrows, off, ovr);
        }
      } else {
        const uint64_t tail0 = J.head + J.nvec * 16u;
        const uint64_t n0 = (J.head + 3) / 4, n1 = (J.len - tail0 + 3) / 4;
        const uint64_t gi = static_cast<uint64_t>(wi.y - J.nv_items) * kFastGroupsPerItem + threadIdx.x;
        if (gi < n0 + n1) {
          const uint64_t off = gi < n0 ? 4 * gi : tail0 + 4 * (gi - n0);
          const uint64_t end = gi < n0 ? J.head : J.len;
          const int nb = static_cast<int>(end - off < 4 ? end - off : 4);
          uint32_t w[K][1];
#pragma unroll
          for (int t = 0; t < K; ++t) {
            uint32_t x = 0;
            for (int b = 0; b < nb; ++b) x |= static_cast<uint32_t>(s_src[t][off + b]) << (8 * b);
            w[t][0] = x;
          }
          uint32_t acc[4] = {0, 0, 0, 0};
          fast_fold<K, 1>(w, acc, r);
          for (uint32_t rr = 0; rr < J.nrows; ++rr) {
            const uint32_t o = row_word4(acc, static_cast<int>(rr));
            uint8_t* d = s_dst[rr] + off;
            for (int b = 0; b < nb; ++b) {
              const uint8_t v = static_cast<uint8_t>(o >> (8 * b));
              d[b] = ovr ? v : static_cast<uint8_t>(d[b] ^ v);
            }
          }
        }
      }
    }
  }
}

// Segmented variant for byte-table classes whose sub-jobs have their own
// plans (a batched reconstruct: one decode plan per erasure pattern). The
// class's 16-byte columns are flattened in plan order (vprefix over the
// class's sub-jobs jidx[]) and every CTA takes one contiguous range of equal
// size, in whole rows of blockDim.x columns. A CTA sweeps its range like the
// uniform kernel sweeps the whole class: the threads take consecutive
// columns, so the CTA streams through one window of each source at a time,
// and it loads pointers (and, if the plan differs, tables) only where its
// range crosses into the next sub-job -- once or twice per CTA. Short work
// items claimed from a counter (batch_fast_kernel) drain the memory pipeline
// at every item boundary instead; that kernel keeps the scalar heads and
// tails of the class.
template <int K, bool SHIFT>
__global__ void __launch_bounds__(kFastThreads, 1)
    batch_fast_segment_kernel(const BatchJob* __restrict__ jobs, const uint64_t* __restrict__ ptrs,
                              const uint32_t* __restrict__ jidx, const uint64_t* __restrict__ vprefix,
                              uint32_t njobs) {
  __shared__ const uint32_t* s_tab;
  __shared__ uint32_t s_g0;
  __shared__ const uint8_t* s_src[K];
  __shared__ uint8_t* s_dst[4];
  const uint64_t vtotal = vprefix[njobs];
  const uint64_t rows = (vtotal + blockDim.x - 1) / blockDim.x;
  const uint64_t chunk = (rows + gridDim.x - 1) / gridDim.x * blockDim.x;
  uint64_t v0 = static_cast<uint64_t>(blockIdx.x) * chunk;
  const uint64_t v1 = v0 + chunk < vtotal ? v0 + chunk : vtotal;
  if (v0 >= v1) return;  // the whole CTA: no barrier is skipped by part of it
  // the sub-job holding column v0: the last q with vprefix[q] <= v0
  uint32_t lo = 0, hi = njobs;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) / 2;
    if (vprefix[mid] <= v0) lo = mid; else hi = mid;
  }
  uint32_t q = lo;
  if (threadIdx.x == 0) {
    s_tab = nullptr;
    s_g0 = 0xFFFFFFFFu;
  }
  const FastRegs r;
  const uint32_t lane = threadIdx.x & 31u;
  while (v0 < v1) {
    while (vprefix[q + 1] <= v0) ++q;  // sub-jobs without vectors
    const uint64_t base = vprefix[q];
    const uint64_t vend = vprefix[q + 1] < v1 ? vprefix[q + 1] : v1;
    const BatchJob J = jobs[jidx[q]];
    __syncthreads();  // the previous sub-job is done with tables and pointers
    const bool resident = s_tab == J.tables && s_g0 == J.g0;
    if (threadIdx.x < K) s_src[threadIdx.x] = reinterpret_cast<const uint8_t*>(ptrs[J.src_idx + threadIdx.x]);
    if (threadIdx.x < J.nrows) s_dst[threadIdx.x] = reinterpret_cast<uint8_t*>(ptrs[J.dst_idx + threadIdx.x]);
    if (!resident) {
      fill_fast<K>(J.tables, nullptr, J.gstride, J.g0);
      if (threadIdx.x == 0) {
        s_tab = J.tables;
        s_g0 = J.g0;
      }
    }
    __syncthreads();
    const bool ovr = J.ovr != 0;
    // SHIFT: whole warps iterate together (the row stores shuffle between
    // lanes) and lanes past the end reload the last column
    for (uint64_t ub = v0 + threadIdx.x - (SHIFT ? lane : 0u); ub < vend; ub += blockDim.x) {
      const uint64_t u0 = SHIFT ? ub + lane : ub;
      const bool valid = !SHIFT || u0 < vend;
      const uint64_t u = valid ? u0 : vend - 1;
      const uint64_t off = J.head + (u - base) * 16u;
      if (u + blockDim.x < vend) {  // this thread's next column: into L2 now
#pragma unroll
        for (int t = 0; t < K; ++t) prefetch_l2(s_src[t] + off + blockDim.x * 16u);
      }
      uint32_t w[K][4];
#pragma unroll
      for (int t = 0; t < K; ++t) {
        const uint4 x = ldg16(s_src[t] + off);
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
        store_col4_any(acc, s_dst, J.nrows, off, ovr, valid);
      else
        store_col4(acc, s_dst, J.nrows, off, ovr);
    }
    v0 = vend;
  }
}

// Uniform-plan variant: every sub-job of the class shares one plan, so each
// CTA loads the tables once and grid-strides over the flattened column space
// of all sub-jobs (vector columns first, then scalar groups), exactly like one
// long call. The per-stripe pointers and geometry travel in the launch
// parameters (constant bank), so the per-column job lookup is a few cached
// constant loads instead of a chain of dependent global loads; a class with
// more stripes than one parameter block holds is split into launches.
constexpr int kUniformJobs = 160;

struct UJob {
  const uint8_t* src[kFastMaxK];
  uint8_t* dst[4];
  uint64_t len, head, nvec;
  uint32_t nrows, ovr;
};

struct UniformParams {
  const uint32_t* tables;
  uint32_t gstride, g0, njobs, pad;
  uint64_t vprefix[kUniformJobs + 1];
  uint64_t gprefix[kUniformJobs + 1];
  UJob jobs[kUniformJobs];
};
static_assert(sizeof(UniformParams) <= 32000, "launch parameter block too large");

template <int K, bool SHIFT>
__global__ void __launch_bounds__(kFastThreads, 1)
    batch_fast_uniform_kernel(const __grid_constant__ UniformParams P) {
  fill_fast<K>(P.tables, nullptr, P.gstride, P.g0);
  const FastRegs r;
  const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
  const uint64_t tid = static_cast<uint64_t>(blockIdx.x) * blockDim.x + threadIdx.x;
  const uint64_t vtotal = P.vprefix[P.njobs];
  const uint32_t lane = threadIdx.x & 31u;
  uint32_t j = 0, jn = 0;
  // SHIFT: whole warps iterate together (the row stores shuffle between
  // lanes; a warp may straddle two stripes) and lanes past the end reload the
  // last column
  for (uint64_t ub = tid - (SHIFT ? lane : 0u); ub < vtotal; ub += stride) {
    const uint64_t u0 = SHIFT ? ub + lane : ub;
    const bool valid = !SHIFT || u0 < vtotal;
    const uint64_t u = valid ? u0 : vtotal - 1;
    while (u >= P.vprefix[j + 1]) ++j;
    const UJob& J = P.jobs[j];
    const uint64_t off = J.head + (u - P.vprefix[j]) * 16u;
    const uint64_t un = u + stride;  // this thread's next column: into L2 now
    if (un < vtotal) {
      while (un >= P.vprefix[jn + 1]) ++jn;
      const UJob& JN = P.jobs[jn];
      const uint64_t offn = JN.head + (un - P.vprefix[jn]) * 16u;
#pragma unroll
      for (int t = 0; t < K; ++t) prefetch_l2(JN.src[t] + offn);
    }
    uint32_t w[K][4];
#pragma unroll
    for (int t = 0; t < K; ++t) {
      const uint4 x = ldg16(J.src[t] + off);
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
      store_col4_any(acc, J.dst, J.nrows, off, J.ovr != 0, valid);
    else
      store_col4(acc, J.dst, J.nrows, off, J.ovr != 0);
  }
  const uint64_t gtotal = P.gprefix[P.njobs];
  j = 0;
  for (uint64_t u = tid; u < gtotal; u += stride) {
    while (u >= P.gprefix[j + 1]) ++j;
    const UJob& J = P.jobs[j];
    const uint64_t gi = u - P.gprefix[j];
    const uint64_t tail0 = J.head + J.nvec * 16u;
    const uint64_t n0 = (J.head + 3) / 4;
    const uint64_t off = gi < n0 ? 4 * gi : tail0 + 4 * (gi - n0);
    const uint64_t end = gi < n0 ? J.head : J.len;
    const int nb = static_cast<int>(end - off < 4 ? end - off : 4);
    uint32_t w[K][1];
#pragma unroll
    for (int t = 0; t < K; ++t) {
      uint32_t x = 0;
      for (int bb = 0; bb < nb; ++bb) x |= static_cast<uint32_t>(J.src[t][off + bb]) << (8 * bb);
      w[t][0] = x;
    }
    uint32_t acc[4] = {0, 0, 0, 0};
    fast_fold<K, 1>(w, acc, r);
    for (uint32_t rr = 0; rr < J.nrows; ++rr) {
      const uint32_t o = row_word4(acc, static_cast<int>(rr));
      uint8_t* d = J.dst[rr] + off;
      for (int bb = 0; bb < nb; ++bb) {
        const uint8_t v = static_cast<uint8_t>(o >> (8 * bb));
        d[bb] = J.ovr ? v : static_cast<uint8_t>(d[bb] ^ v);
      }
    }
  }
}

using KernelFn = void (*)(const BatchJob*, const uint64_t*, const uint2*, uint32_t, uint32_t*);
using UniformFn = void (*)(UniformParams);
using SegmentFn = void (*)(const BatchJob*, const uint64_t*, const uint32_t*, const uint64_t*, uint32_t);

template <bool S>
KernelFn kernel_for_s(int E, int G) {
  switch (E * 8 + G) {
    case 8 + 1: return batch_kernel<1, 1, S>;
    case 8 + 2: return batch_kernel<1, 2, S>;
    case 8 + 3: return batch_kernel<1, 3, S>;
    case 8 + 4: return batch_kernel<1, 4, S>;
    case 16 + 1: return batch_kernel<2, 1, S>;
    case 16 + 2: return batch_kernel<2, 2, S>;
    case 16 + 3: return batch_kernel<2, 3, S>;
    case 16 + 4: return batch_kernel<2, 4, S>;
    case 32 + 1: return batch_kernel<4, 1, S>;
    case 32 + 2: return batch_kernel<4, 2, S>;
    case 32 + 3: return batch_kernel<4, 3, S>;
    case 32 + 4: return batch_kernel<4, 4, S>;
    default: return nullptr;
  }
}

KernelFn kernel_for(int E, int G, bool shift) { return shift ? kernel_for_s<true>(E, G) : kernel_for_s<false>(E, G); }

KernelFn kernel_for_k16(int GK, bool shift) {
  if (GK == 1) return shift ? batch_kernel_k16<1, true> : batch_kernel_k16<1, false>;
  if (GK == 2) return shift ? batch_kernel_k16<2, true> : batch_kernel_k16<2, false>;
  return nullptr;
}

#define FGFC_K_CASES(X) X(1) X(2) X(3) X(4) X(5) X(6) X(7) X(8) X(9) X(10) X(11) X(12) X(13) X(14)

KernelFn fast_kernel_for(int K, bool shift) {
  switch (K) {
#define FGFC_CASE(k) \
  case k: return shift ? batch_fast_kernel<k, true> : batch_fast_kernel<k, false>;
    FGFC_K_CASES(FGFC_CASE)
#undef FGFC_CASE
    default: return nullptr;
  }
}

SegmentFn segment_kernel_for(int K, bool shift) {
  switch (K) {
#define FGFC_CASE(k) \
  case k: return shift ? batch_fast_segment_kernel<k, true> : batch_fast_segment_kernel<k, false>;
    FGFC_K_CASES(FGFC_CASE)
#undef FGFC_CASE
    default: return nullptr;
  }
}

UniformFn uniform_kernel_for(int K, bool shift) {
  switch (K) {
#define FGFC_CASE(k) \
  case k: return shift ? batch_fast_uniform_kernel<k, true> : batch_fast_uniform_kernel<k, false>;
    FGFC_K_CASES(FGFC_CASE)
#undef FGFC_CASE
    default: return nullptr;
  }
}

uint32_t fast_smem(int K) {
  switch (K) {
#define FGFC_CASE(k) \
  case k: return FastLayout<k>::smem;
    FGFC_K_CASES(FGFC_CASE)
#undef FGFC_CASE
    default: return 0;
  }
}

constexpr size_t kBatchSmem = kMaxSlots * (kSlotBytes + kCompactWords * 4);

}  // namespace

// ---------------------------------------------------------------- host side

struct BatchClass {
  int E, G;
  int K = 0;                   // > 0: byte-table class of Gf8 sub-jobs with K sources
  std::vector<uint32_t> jobs;  // sub-job indices, plan order
  std::vector<uint2> items;
  std::vector<uint32_t> seg_jobs;   // byte-table class with own plans: sub-jobs with vectors, plan order
  std::vector<uint64_t> seg_prefix; // and the prefix of their vector counts (the segmented launch)
  bool uniform = false;        // byte-table class whose sub-jobs share one plan
  bool shift = false;          // its rows are not all at the sources' offset within 16 bytes
  bool kara = false;           // Gf16 by byte half-products, G = row quads
};

// Descriptor slots used round robin: a submission waits (on the host) only
// for the one kBatchSlots submissions before it, so that many can be queued
// on the GPU at once. With an even count, alternating submissions keep their
// own slots and replay their graphs.
constexpr int kBatchSlots = 4;

struct BatchSlot {
  uint8_t* host = nullptr;  // pinned
  uint8_t* dev = nullptr;
  size_t cap = 0;
  cudaEvent_t done = nullptr;  // the last submission out of this slot finished
  cudaGraphExec_t graph = nullptr;
  std::string key;
};

// Classes of one submission run on side streams forked from the caller's
// stream, so that small classes share the GPU instead of queueing.
constexpr int kSideStreams = 4;

struct BatchState {
  std::vector<UniformParams> uparams;
  BatchSlot slot[kBatchSlots];
  int next = 0;
  bool graphs = true;
  cudaStream_t capture = nullptr;
  cudaStream_t side[kSideStreams] = {};
  cudaEvent_t fork = nullptr, join[kSideStreams] = {};
  size_t last_launches = 0, last_items = 0;
  int last_replayed = 0;
  std::vector<std::pair<int, int>> last_classes;  // nibble (E, G) classes of the last submission
  mutable std::mutex mu;
};

static cudaError_t ensure_slot(BatchSlot& s, size_t bytes) {
  if (s.cap >= bytes) return cudaSuccess;
  if (s.host) cudaFreeHost(s.host);
  if (s.dev) cudaFree(s.dev);
  s.host = nullptr;
  s.dev = nullptr;
  if (s.graph) {
    cudaGraphExecDestroy(s.graph);
    s.graph = nullptr;
  }
  s.key.clear();
  size_t cap = 1 << 16;
  while (cap < bytes) cap <<= 1;
  cudaError_t e = cudaHostAlloc(&s.host, cap, cudaHostAllocDefault);
  if (e != cudaSuccess) return e;
  e = cudaMalloc(&s.dev, cap);
  if (e != cudaSuccess) return e;
  if (!s.done) {
    e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
  }
  s.cap = cap;
  return cudaSuccess;
}

void* batch_state_create() { return new BatchState(); }

void batch_state_destroy(void* p) {
  BatchState* b = static_cast<BatchState*>(p);
  if (!b) return;
  for (auto& s : b->slot) {
    if (s.done) cudaEventSynchronize(s.done);
    if (s.graph) cudaGraphExecDestroy(s.graph);
    if (s.host) cudaFreeHost(s.host);
    if (s.dev) cudaFree(s.dev);
    if (s.done) cudaEventDestroy(s.done);
  }
  if (b->capture) cudaStreamDestroy(b->capture);
  for (int i = 0; i < kSideStreams; ++i) {
    if (b->side[i]) cudaStreamDestroy(b->side[i]);
    if (b->join[i]) cudaEventDestroy(b->join[i]);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  delete b;
}

void batch_state_graphs(void* p, bool on) { static_cast<BatchState*>(p)->graphs = on; }

std::vector<std::pair<int, int>> batch_state_classes(const void* p) {
  const BatchState* b = static_cast<const BatchState*>(p);
  std::lock_guard<std::mutex> lk(b->mu);
  std::vector<std::pair<int, int>> v = b->last_classes;
  std::sort(v.begin(), v.end());
  v.erase(std::unique(v.begin(), v.end()), v.end());
  return v;
}

void batch_state_stats(const void* p, size_t* launches, size_t* items, int* replayed) {
  const BatchState* b = static_cast<const BatchState*>(p);
  if (launches) *launches = b->last_launches;
  if (items) *items = b->last_items;
  if (replayed) *replayed = b->last_replayed;
}

static size_t align16(size_t x) { return (x + 15) & ~static_cast<size_t>(15); }

cudaError_t batch_run(void* state, const std::vector<LoweredJob>& jobs, const std::vector<Gf2Job>& tc,
                      cudaStream_t stream) {
  BatchState* b = static_cast<BatchState*>(state);
  std::lock_guard<std::mutex> lk(b->mu);
  b->last_launches = b->last_items = 0;
  b->last_replayed = 0;
  b->last_classes.clear();
  if (jobs.empty() && tc.empty()) return cudaSuccess;

  // ---- device descriptors, pointer array, classes (sub-jobs in plan order)
  std::vector<BatchJob> dj(jobs.size());
  std::vector<uint64_t> ptrs;
  for (size_t i = 0; i < jobs.size(); ++i) {
    const LoweredJob& L = jobs[i];
    BatchJob& J = dj[i];
    J.tables = L.tables;
    J.len = L.len;
    J.head = L.head;
    J.nvec = L.nvec;
    J.gstride = static_cast<uint32_t>(L.gstride);
    J.g0 = static_cast<uint32_t>(L.g0);
    J.k = static_cast<uint32_t>(L.k);
    J.nrows = static_cast<uint32_t>(L.nrows);
    J.ovr = L.ovr ? 1u : 0u;
    J.src_idx = static_cast<uint32_t>(ptrs.size());
    ptrs.insert(ptrs.end(), L.srcs.begin(), L.srcs.end());
    J.dst_idx = static_cast<uint32_t>(ptrs.size());
    ptrs.insert(ptrs.end(), L.dsts.begin(), L.dsts.end());
    J.nv_items = 0;
  }
  std::vector<size_t> order(jobs.size());
  for (size_t i = 0; i < order.size(); ++i) order[i] = i;
  std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t c) {
    return jobs[a].tables != jobs[c].tables ? jobs[a].tables < jobs[c].tables : jobs[a].g0 < jobs[c].g0;
  });
  std::map<int, BatchClass> classes;  // key E * 8 + G, or 100 + K for byte-table classes; + 300 if shifted
  for (size_t i : order) {
    const LoweredJob& L = jobs[i];
    const int E = field_bytes(L.field);
    const bool fast = E == 1 && L.G == 1 && L.k >= 1 && L.k <= static_cast<size_t>(kFastMaxK);
    const int key = (fast ? 100 + static_cast<int>(L.k) : L.kara ? 200 + static_cast<int>(L.G)
                                                                  : E * 8 + static_cast<int>(L.G)) +
                    (L.shift ? 300 : 0);
    BatchClass& c = classes[key];
    c.shift = L.shift;
    c.kara = L.kara;
    c.E = E;
    c.G = static_cast<int>(L.G);
    c.K = fast ? static_cast<int>(L.k) : 0;
    c.jobs.push_back(static_cast<uint32_t>(i));
  }
  for (auto& kv : classes) {
    BatchClass& c = kv.second;
    c.uniform = c.K > 0;
    for (uint32_t i : c.jobs)
      c.uniform = c.uniform && jobs[i].tables == jobs[c.jobs[0]].tables && jobs[i].g0 == jobs[c.jobs[0]].g0;
    if (c.uniform) continue;
    // Columns per item: the class's tile (tune.cpp: tile_cols; 8 per
    // thread built in) for nibble classes, 8 per thread for byte-table
    // classes, fewer when the class is too small to give every SM a few
    // items (a small class runs beside the others on its own stream, see
    // enqueue).
    const uint64_t threads = c.K ? kFastThreads : kThreads;
    const uint64_t tile = c.K ? kFastVecPerItem : threads * static_cast<uint64_t>(tile_cols(c.E, c.G));
    if (!c.K) b->last_classes.emplace_back(c.E, c.G);
    uint64_t total = 0;
    for (uint32_t i : c.jobs) total += jobs[i].nvec;
    const uint64_t want = (total + 4 * static_cast<uint64_t>(sm_count()) - 1) / (4 * static_cast<uint64_t>(sm_count()));
    const uint64_t per_vec = std::min<uint64_t>(tile, std::max<uint64_t>(threads, (want + threads - 1) / threads * threads));
    const uint64_t per_grp = c.K ? kFastGroupsPerItem : kGroupsPerItem;
    for (uint32_t i : c.jobs) {
      const LoweredJob& L = jobs[i];
      const uint64_t nv_items = (L.nvec + per_vec - 1) / per_vec;
      const uint64_t tail = L.len - L.head - 16 * L.nvec;
      const uint64_t ngroups = (L.head + 3) / 4 + (tail + 3) / 4;
      const uint64_t ns_items = (ngroups + per_grp - 1) / per_grp;
      dj[i].nv_items = static_cast<uint32_t>(nv_items);
      if (c.K > 0) {
        // vectors: the segmented launch; scalar heads and tails: work items
        if (L.nvec) {
          if (c.seg_prefix.empty()) c.seg_prefix.push_back(0);
          c.seg_jobs.push_back(i);
          c.seg_prefix.push_back(c.seg_prefix.back() + L.nvec);
        }
        for (uint64_t p = nv_items; p < nv_items + ns_items; ++p)
          c.items.push_back(make_uint2(i, static_cast<unsigned>(p)));
      } else {
        for (uint64_t p = 0; p < nv_items + ns_items; ++p)
          c.items.push_back(make_uint2(i, static_cast<unsigned>(p)));
      }
    }
  }

  // ---- blob: jobs | ptrs | per work-list class: items, counter
  size_t off = 0;
  const size_t off_jobs = off;
  off = align16(off + dj.size() * sizeof(BatchJob));
  const size_t off_ptrs = off;
  off = align16(off + ptrs.size() * sizeof(uint64_t));
  std::vector<std::pair<size_t, size_t>> cb;  // (items, counter) offsets
  std::vector<std::pair<size_t, size_t>> sb;  // (segment jobs, segment prefix) offsets
  for (auto& kv : classes) {
    std::pair<size_t, size_t> x{0, 0}, y{0, 0};
    if (!kv.second.uniform) {
      x.first = off;
      off = align16(off + kv.second.items.size() * sizeof(uint2));
      x.second = off;
      off = align16(off + 64);
      if (!kv.second.seg_jobs.empty()) {
        y.first = off;
        off = align16(off + kv.second.seg_jobs.size() * sizeof(uint32_t));
        y.second = off;
        off = align16(off + kv.second.seg_prefix.size() * sizeof(uint64_t));
      }
    }
    cb.push_back(x);
    sb.push_back(y);
  }
  // tensor-core bodies: one launch per plan (bit matrix), its stripes'
  // pointers and first blocks in the blob
  struct TcGroup {
    std::vector<size_t> idx;
    size_t off_ptrs = 0, off_prefix = 0;
    uint64_t nblk = 0;
  };
  std::vector<TcGroup> tcg;
  {
    std::map<std::tuple<uint64_t, int, size_t, size_t, bool>, size_t> gi;
    for (size_t i = 0; i < tc.size(); ++i) {
      const Gf2Job& J = tc[i];
      const auto key = std::make_tuple(J.bits_key, J.field, J.k, J.m, J.ovr);
      auto it = gi.find(key);
      if (it == gi.end()) {
        it = gi.emplace(key, tcg.size()).first;
        tcg.emplace_back();
      }
      TcGroup& G = tcg[it->second];
      G.idx.push_back(i);
      G.nblk += J.nblk;
    }
    for (TcGroup& G : tcg) {
      const Gf2Job& J0 = tc[G.idx[0]];
      G.off_ptrs = off;
      off = align16(off + G.idx.size() * (J0.k + J0.m) * sizeof(uint64_t));
      G.off_prefix = off;
      off = align16(off + (G.idx.size() + 1) * sizeof(uint64_t));
    }
  }
  const size_t bytes = off;

  BatchSlot& s = b->slot[b->next];
  b->next = (b->next + 1) % kBatchSlots;
  cudaError_t e = cudaSuccess;
  if (s.done) {
    e = cudaEventSynchronize(s.done);  // the previous submission out of this slot finished
    if (e != cudaSuccess) return e;
  }
  e = ensure_slot(s, bytes);
  if (e != cudaSuccess) return e;
  std::memcpy(s.host + off_jobs, dj.data(), dj.size() * sizeof(BatchJob));
  std::memcpy(s.host + off_ptrs, ptrs.data(), ptrs.size() * sizeof(uint64_t));
  {
    size_t ci = 0;
    for (auto& kv : classes) {
      const auto& y = sb[ci];
      const auto& x = cb[ci++];
      if (kv.second.uniform) continue;
      std::memcpy(s.host + x.first, kv.second.items.data(), kv.second.items.size() * sizeof(uint2));
      std::memset(s.host + x.second, 0, 64);
      if (!kv.second.seg_jobs.empty()) {
        std::memcpy(s.host + y.first, kv.second.seg_jobs.data(), kv.second.seg_jobs.size() * sizeof(uint32_t));
        std::memcpy(s.host + y.second, kv.second.seg_prefix.data(), kv.second.seg_prefix.size() * sizeof(uint64_t));
      }
    }
    for (const TcGroup& G : tcg) {
      uint64_t* hp = reinterpret_cast<uint64_t*>(s.host + G.off_ptrs);
      uint64_t* pre = reinterpret_cast<uint64_t*>(s.host + G.off_prefix);
      uint64_t acc = 0;
      size_t n = 0;
      for (size_t i : G.idx) {
        const Gf2Job& J = tc[i];
        std::memcpy(hp, J.ptrs.data(), J.ptrs.size() * sizeof(uint64_t));
        hp += J.ptrs.size();
        pre[n++] = acc;
        acc += J.nblk;
      }
      pre[n] = acc;
    }
  }

  // ---- launches (their structure is the graph key)
  struct Launch {
    KernelFn fn = nullptr;
    UniformFn ufn = nullptr;
    unsigned grid = 0, threads = 0;
    uint32_t smem = 0;
    const uint2* items = nullptr;
    uint32_t n = 0;
    uint32_t* counter = nullptr;
    size_t uparam = 0;
    int tc_group = -1;  // >= 0: a tensor-core launch over that group's stripes
    SegmentFn sfn = nullptr;  // segmented launch over the class's vectors
    const uint32_t* seg_jobs = nullptr;
    const uint64_t* seg_prefix = nullptr;
  };
  std::vector<Launch> launches;
  std::vector<UniformParams>& uparams = b->uparams;
  uparams.clear();
  std::string key = std::to_string(reinterpret_cast<uintptr_t>(s.dev)) + ":" + std::to_string(bytes);
  const int sms = sm_count();
  size_t ci = 0;
  for (auto& kv : classes) {
    const BatchClass& c = kv.second;
    const auto& y = sb[ci];
    const auto& x = cb[ci++];
    const bool fast = c.K > 0;
    Launch L;
    const int akey = kv.first + (c.uniform ? 100 : 0);
    if (c.uniform) {
      L.ufn = uniform_kernel_for(c.K, c.shift);
    } else {
      L.fn = fast ? fast_kernel_for(c.K, c.shift) : c.kara ? kernel_for_k16(c.G, c.shift) : kernel_for(c.E, c.G, c.shift);
    }
    if (!L.fn && !L.ufn) return cudaErrorInvalidValue;
    L.smem = fast ? fast_smem(c.K) : static_cast<uint32_t>(kBatchSmem);
    L.threads = fast ? static_cast<unsigned>(kFastThreads) : static_cast<unsigned>(kThreads);
    e = ensure_smem_attr(L.ufn ? reinterpret_cast<const void*>(L.ufn) : reinterpret_cast<const void*>(L.fn),
                         static_cast<int>(L.smem));
    if (e != cudaSuccess) return e;
    if (c.uniform) {
      // one launch per block of kUniformJobs stripes
      for (size_t q0 = 0; q0 < c.jobs.size(); q0 += kUniformJobs) {
        const size_t nq = std::min<size_t>(kUniformJobs, c.jobs.size() - q0);
        uparams.emplace_back();
        UniformParams& P = uparams.back();
        std::memset(&P, 0, sizeof P);
        const BatchJob& J0 = dj[c.jobs[q0]];
        P.tables = J0.tables;
        P.gstride = J0.gstride;
        P.g0 = J0.g0;
        P.njobs = static_cast<uint32_t>(nq);
        for (size_t q = 0; q < nq; ++q) {
          const LoweredJob& LJ = jobs[c.jobs[q0 + q]];
          UJob& U = P.jobs[q];
          for (size_t t = 0; t < LJ.k; ++t) U.src[t] = reinterpret_cast<const uint8_t*>(LJ.srcs[t]);
          for (size_t rr = 0; rr < 4; ++rr) U.dst[rr] = reinterpret_cast<uint8_t*>(LJ.dsts[rr < LJ.nrows ? rr : 0]);
          U.len = LJ.len;
          U.head = LJ.head;
          U.nvec = LJ.nvec;
          U.nrows = static_cast<uint32_t>(LJ.nrows);
          U.ovr = LJ.ovr ? 1u : 0u;
          const uint64_t tail = LJ.len - LJ.head - 16 * LJ.nvec;
          P.vprefix[q + 1] = P.vprefix[q] + LJ.nvec;
          P.gprefix[q + 1] = P.gprefix[q] + (LJ.head + 3) / 4 + (tail + 3) / 4;
        }
        Launch U = L;
        const uint64_t want = (std::max(P.vprefix[nq], P.gprefix[nq]) + L.threads - 1) / L.threads;
        U.grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(want, sms)));
        U.uparam = uparams.size() - 1;
        // the parameter block is baked into a captured graph: hash it into the key
        uint64_t h = 1469598103934665603ull;
        const uint8_t* pb = reinterpret_cast<const uint8_t*>(&P);
        for (size_t i = 0; i < sizeof P; ++i) h = (h ^ pb[i]) * 1099511628211ull;
        key += "|u" + std::to_string(akey) + "," + std::to_string(h) + "," + std::to_string(U.grid);
        launches.push_back(U);
      }
      b->last_items += c.jobs.size();
    } else {
      if (!c.seg_jobs.empty()) {
        Launch S = L;
        S.fn = nullptr;
        S.sfn = segment_kernel_for(c.K, c.shift);
        if (!S.sfn) return cudaErrorInvalidValue;
        e = ensure_smem_attr(reinterpret_cast<const void*>(S.sfn), static_cast<int>(S.smem));
        if (e != cudaSuccess) return e;
        S.n = static_cast<uint32_t>(c.seg_jobs.size());
        S.seg_jobs = reinterpret_cast<const uint32_t*>(s.dev + y.first);
        S.seg_prefix = reinterpret_cast<const uint64_t*>(s.dev + y.second);
        const uint64_t rows = (c.seg_prefix.back() + S.threads - 1) / S.threads;
        S.grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(rows, sms)));
        b->last_items += c.seg_jobs.size();
        key += "|s" + std::to_string(akey) + "," + std::to_string(S.n) + "," + std::to_string(S.grid);
        launches.push_back(S);
      }
      if (!c.items.empty()) {
        L.n = static_cast<uint32_t>(c.items.size());
        L.grid = static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>((L.n + kClaim - 1) / kClaim, sms)));
        L.items = reinterpret_cast<const uint2*>(s.dev + x.first);
        L.counter = reinterpret_cast<uint32_t*>(s.dev + x.second);
        b->last_items += c.items.size();
        key += "|" + std::to_string(akey) + "," + std::to_string(L.n) + "," + std::to_string(L.grid);
        launches.push_back(L);
      }
    }
  }
  for (size_t g = 0; g < tcg.size(); ++g) {
    const Gf2Job& J0 = tc[tcg[g].idx[0]];
    e = gf2mma_prepare(field_bytes(J0.field));  // before any capture records the launch
    if (e != cudaSuccess) return e;
    Launch L;
    L.tc_group = static_cast<int>(g);
    b->last_items += tcg[g].idx.size();
    key += "|g" + std::to_string(J0.bits_key) + "," + std::to_string(J0.field) + "," + std::to_string(J0.k) + "," +
           std::to_string(J0.m) + "," + std::to_string(J0.ovr) + "," + std::to_string(tcg[g].idx.size()) + "," +
           std::to_string(tcg[g].nblk);
    launches.push_back(L);
  }
  const BatchJob* djobs = reinterpret_cast<const BatchJob*>(s.dev + off_jobs);
  const uint64_t* dptrs = reinterpret_cast<const uint64_t*>(s.dev + off_ptrs);

  const int nside = launches.size() > 1 ? static_cast<int>(std::min<size_t>(launches.size(), kSideStreams)) : 0;
  for (int i = 0; i < nside; ++i) {
    if (!b->side[i]) {
      e = cudaStreamCreateWithFlags(&b->side[i], cudaStreamNonBlocking);
      if (e == cudaSuccess) e = cudaEventCreateWithFlags(&b->join[i], cudaEventDisableTiming);
      if (e != cudaSuccess) return e;
    }
  }
  if (nside && !b->fork) {
    e = cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming);
    if (e != cudaSuccess) return e;
  }
  // blob copy on the caller's stream; with several classes, fork to the side
  // streams (class i on stream i % kSideStreams) and join back
  auto enqueue = [&](cudaStream_t st) -> cudaError_t {
    cudaError_t err = cudaMemcpyAsync(s.dev, s.host, bytes, cudaMemcpyHostToDevice, st);
    if (err != cudaSuccess) return err;
    if (nside) {
      err = cudaEventRecord(b->fork, st);
      for (int i = 0; i < nside && err == cudaSuccess; ++i) err = cudaStreamWaitEvent(b->side[i], b->fork, 0);
      if (err != cudaSuccess) return err;
    }
    for (size_t li = 0; li < launches.size(); ++li) {
      const Launch& L = launches[li];
      cudaStream_t ls = nside ? b->side[li % nside] : st;
      if (L.tc_group >= 0) {
        const TcGroup& G = tcg[L.tc_group];
        const Gf2Job& J0 = tc[G.idx[0]];
        err = gf2mma_launch_multi(J0.field, J0.k, J0.m, J0.bits, reinterpret_cast<const uint64_t*>(s.dev + G.off_ptrs),
                                  reinterpret_cast<const uint64_t*>(s.dev + G.off_prefix),
                                  static_cast<uint32_t>(G.idx.size()), G.nblk, J0.ovr, ls);
      } else if (L.ufn) {
        L.ufn<<<L.grid, L.threads, L.smem, ls>>>(uparams[L.uparam]);
        err = cudaGetLastError();
      } else if (L.sfn) {
        L.sfn<<<L.grid, L.threads, L.smem, ls>>>(djobs, dptrs, L.seg_jobs, L.seg_prefix, L.n);
        err = cudaGetLastError();
      } else {
        L.fn<<<L.grid, L.threads, L.smem, ls>>>(djobs, dptrs, L.items, L.n, L.counter);
        err = cudaGetLastError();
      }
      if (err != cudaSuccess) return err;
    }
    for (int i = 0; i < nside && err == cudaSuccess; ++i) {
      err = cudaEventRecord(b->join[i], b->side[i]);
      if (err == cudaSuccess) err = cudaStreamWaitEvent(st, b->join[i], 0);
    }
    return err;
  };

  b->last_launches = launches.size();
  if (b->graphs) {
    if (!(s.graph && s.key == key)) {
      if (s.graph) {
        cudaGraphExecDestroy(s.graph);
        s.graph = nullptr;
      }
      if (!b->capture) {
        e = cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking);
        if (e != cudaSuccess) return e;
      }
      cudaGraph_t g = nullptr;
      e = cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return e;
      const cudaError_t ee = enqueue(b->capture);
      e = cudaStreamEndCapture(b->capture, &g);
      if (ee != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return ee;
      }
      if (e != cudaSuccess) return e;
      e = cudaGraphInstantiate(&s.graph, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) {
        s.graph = nullptr;
        return e;
      }
      s.key = key;
    } else {
      b->last_replayed = 1;
    }
    e = cudaGraphLaunch(s.graph, stream);
  } else {
    e = enqueue(stream);
  }
  if (e != cudaSuccess) return e;
  return cudaEventRecord(s.done, stream);
}

// ---------------------------------------------------------------- without allocation
//
// fgfc_batch_run_noalloc: the work-list kernels above, with every byte of
// scratch they need (descriptors, pointers, work items, the claim counters and
// the stripes' compact product tables) placed in this fixed device array
// instead of device memory allocated for the call. The host side builds the
// whole blob in a fixed host array of the same size and copies it in with one
// stream-ordered copy, so nothing is allocated on either side.
//
// The host array is pageable, so the runtime stages the copy before the call
// returns: the call may block the host until the stream reaches the copy, and
// that is also what makes it safe to refill the host array on the next call.
// (Pinning the array would make the copy truly asynchronous, but then every
// call would first have to wait on an event recorded after the previous copy.)
//
// Stripes are grouped in classes as in fgfc_batch_run: Gf8 stripes of at most
// 4 rows and at most 14 sources run the byte-table kernel for their source
// count; the rest run the split-nibble kernel for their own number of table
// groups, so a wide stripe does not widen the others. One launch per class,
// in order, on the caller's stream.

static __device__ __align__(256) uint8_t g_noalloc_scratch[FGFC_NOALLOC_SCRATCH_BYTES];
alignas(256) static uint8_t g_noalloc_host[FGFC_NOALLOC_SCRATCH_BYTES];
static std::mutex g_noalloc_mu;
constexpr int kNoallocMaxDevices = 64;
static uint8_t* g_noalloc_dev[kNoallocMaxDevices];  // device address of the array, per device

namespace {

// Class of a stripe in fgfc_batch_run_noalloc: 1..14 = byte-table kernel
// with that many sources, 100 + G = nibble kernel with G table groups.
int noalloc_class(int E, size_t nsrcs, size_t nrows) {
  const int R = 4 / E;
  const size_t G = (nrows + R - 1) / R;
  if (E == 1 && G == 1 && nsrcs >= 1 && nsrcs <= static_cast<size_t>(kFastMaxK)) return static_cast<int>(nsrcs);
  return 100 + static_cast<int>(G);
}

}  // namespace

// Returns 0, or an fgfc_status-style code with `msg` filled in.
int noalloc_run(int field, const fgfc_noalloc_job* jobs, size_t njobs, cudaStream_t stream, char* msg,
                size_t msglen) {
  // A graph recorded from this call would replay whatever the shared host
  // and device arrays hold at replay time, not this call's descriptors.
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(stream, &cap);
  if (e != cudaSuccess) {
    snprintf(msg, msglen, "batch_run_noalloc: %s", cudaGetErrorString(e));
    return FGFC_ERR_CUDA;
  }
  if (cap != cudaStreamCaptureStatusNone) {
    snprintf(msg, msglen, "batch_run_noalloc: the stream is being captured; this call cannot be recorded");
    return FGFC_ERR_ARG;
  }
  std::lock_guard<std::mutex> lk(g_noalloc_mu);
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess || dev < 0 || dev >= kNoallocMaxDevices) {
    snprintf(msg, msglen, "batch_run_noalloc: no usable current device");
    return FGFC_ERR_CUDA;
  }
  if (!g_noalloc_dev[dev]) {
    // The array's name is only a host-side stand-in; the kernels need its
    // device address on this device.
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
      snprintf(msg, msglen, "batch_run_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
      return FGFC_ERR_CUDA;
    }
    g_noalloc_dev[dev] = static_cast<uint8_t*>(p);
  }
  uint8_t* const dbase = g_noalloc_dev[dev];
  const int E = field_bytes(field);
  const int R = 4 / E;

  // ---- sizes: per class its items; every stripe's tables at its own G
  constexpr int kClasses = 105;  // byte-table 1..14, nibble 101..104
  size_t nptr = 0, ntab = 0, nlive = 0;
  size_t class_items[kClasses] = {0};
  for (size_t i = 0; i < njobs; ++i) {
    const fgfc_noalloc_job& J = jobs[i];
    if (J.nrows == 0 || J.row_len == 0 || J.nsrcs == 0) continue;
    if (J.nrows > static_cast<size_t>(4 * R) || J.nsrcs > static_cast<size_t>(kMaxSrc)) {
      snprintf(msg, msglen, "batch_run_noalloc: job %zu has %zu rows and %zu sources; at most %d rows and %d sources",
               i, J.nrows, J.nsrcs, 4 * R, kMaxSrc);
      return FGFC_ERR_LIMIT;
    }
    const size_t G = (J.nrows + R - 1) / R;
    const int cls = noalloc_class(E, J.nsrcs, J.nrows);
    const bool fast = cls < 100;
    ++nlive;
    nptr += J.nsrcs + J.nrows;
    ntab += J.nsrcs * E * G * kCompactWords;
    const uint64_t nvec = J.row_len / 16 + 1;  // upper bound before alignment is known
    const uint64_t per_vec = fast ? kFastVecPerItem : kVecPerItem;
    const uint64_t per_grp = fast ? kFastGroupsPerItem : kGroupsPerItem;
    class_items[cls] += (nvec + per_vec - 1) / per_vec + (J.row_len / 4 + 2 + per_grp - 1) / per_grp + 1;
  }
  const size_t off_jobs = 0;
  const size_t off_ptrs = align16(off_jobs + nlive * sizeof(BatchJob));
  const size_t off_tabs = align16(off_ptrs + nptr * sizeof(uint64_t));
  size_t class_off[kClasses] = {0};
  size_t off = align16(off_tabs + ntab * sizeof(uint32_t));
  for (int c = 0; c < kClasses; ++c) {
    if (!class_items[c]) continue;
    class_off[c] = off;  // items, then a 64-byte counter
    off = align16(off + class_items[c] * sizeof(uint2)) + 64;
  }
  const size_t bytes = off;
  if (bytes > FGFC_NOALLOC_SCRATCH_BYTES) {
    snprintf(msg, msglen, "batch_run_noalloc: submission needs %zu bytes of scratch, more than the %u available",
             bytes, static_cast<unsigned>(FGFC_NOALLOC_SCRATCH_BYTES));
    return FGFC_ERR_LIMIT;
  }

  // ---- blob in the host array
  BatchJob* hj = reinterpret_cast<BatchJob*>(g_noalloc_host + off_jobs);
  uint64_t* hp = reinterpret_cast<uint64_t*>(g_noalloc_host + off_ptrs);
  uint32_t* ht = reinterpret_cast<uint32_t*>(g_noalloc_host + off_tabs);
  size_t jn = 0, pn = 0, tn = 0;
  size_t class_n[kClasses] = {0};
  for (size_t i = 0; i < njobs; ++i) {
    const fgfc_noalloc_job& S = jobs[i];
    if (S.nrows == 0 || S.row_len == 0) continue;
    if (S.nsrcs == 0) {
      if (S.overwrite) {  // an empty sum overwrites with zero
        for (size_t j = 0; j < S.nrows; ++j) {
          e = cudaMemsetAsync(S.dst + (S.row_starts ? S.row_starts[j] : j * S.row_len), 0, S.row_len, stream);
          if (e != cudaSuccess) {
            snprintf(msg, msglen, "batch_run_noalloc: %s", cudaGetErrorString(e));
            return FGFC_ERR_CUDA;
          }
        }
      }
      continue;
    }
    const size_t G = (S.nrows + R - 1) / R;
    const int cls = noalloc_class(E, S.nsrcs, S.nrows);
    const bool fast = cls < 100;
    BatchJob& J = hj[jn];
    const uintptr_t al = reinterpret_cast<uintptr_t>(S.srcs[0].ptr) & 15;
    bool same = (al % E) == 0;
    J.src_idx = static_cast<uint32_t>(pn);
    for (size_t t = 0; t < S.nsrcs; ++t) {
      hp[pn] = reinterpret_cast<uint64_t>(S.srcs[t].ptr);
      same = same && (hp[pn] & 15) == al;
      ++pn;
    }
    J.dst_idx = static_cast<uint32_t>(pn);
    for (size_t j = 0; j < S.nrows; ++j) {
      hp[pn] = reinterpret_cast<uint64_t>(S.dst + (S.row_starts ? S.row_starts[j] : j * S.row_len));
      same = same && (hp[pn] & 15) == al;
      ++pn;
    }
    J.len = S.row_len;
    J.head = S.row_len;
    J.nvec = 0;
    if (same) {
      J.head = std::min<uint64_t>((16 - al) & 15, S.row_len);
      J.nvec = (S.row_len - J.head) / 16;
    }
    uint64_t cm[kMaxSrc * 16];  // coefficients reduced to the field's width, as Plan::matrix does
    for (size_t q = 0; q < S.nsrcs * S.nrows; ++q) cm[q] = S.coeffs[q] & field_mask(field);
    build_compact_tables(field, cm, S.nrows, 0, S.nsrcs, 0, G, ht + tn);
    J.tables = reinterpret_cast<const uint32_t*>(dbase + off_tabs) + tn;
    tn += S.nsrcs * E * G * kCompactWords;
    J.gstride = static_cast<uint32_t>(G);
    J.g0 = 0;
    J.k = static_cast<uint32_t>(S.nsrcs);
    J.nrows = static_cast<uint32_t>(S.nrows);
    J.ovr = S.overwrite ? 1u : 0u;
    const uint64_t per_vec = fast ? kFastVecPerItem : kVecPerItem;
    const uint64_t per_grp = fast ? kFastGroupsPerItem : kGroupsPerItem;
    const uint64_t nv_items = (J.nvec + per_vec - 1) / per_vec;
    const uint64_t tail = J.len - J.head - 16 * J.nvec;
    const uint64_t ns_items = ((J.head + 3) / 4 + (tail + 3) / 4 + per_grp - 1) / per_grp;
    J.nv_items = static_cast<uint32_t>(nv_items);
    uint2* hi = reinterpret_cast<uint2*>(g_noalloc_host + class_off[cls]);
    for (uint64_t q = 0; q < nv_items + ns_items; ++q)
      hi[class_n[cls]++] = make_uint2(static_cast<unsigned>(jn), static_cast<unsigned>(q));
    ++jn;
  }
  if (jn == 0) return 0;
  for (int c = 0; c < kClasses; ++c)  // every claim counter starts at zero on every call
    if (class_items[c]) std::memset(g_noalloc_host + align16(class_off[c] + class_items[c] * sizeof(uint2)), 0, 64);

  // ---- one copy, then one launch of the work-list kernel per class
  e = cudaMemcpyAsync(dbase, g_noalloc_host, bytes, cudaMemcpyHostToDevice, stream);
  for (int c = 0; c < kClasses && e == cudaSuccess; ++c) {
    if (!class_n[c]) continue;
    const bool fast = c < 100;
    // rows share the sources' alignment here (otherwise the whole stripe is scalar)
    KernelFn fn = fast ? fast_kernel_for(c, false) : kernel_for(E, c - 100, false);
    const int smem = fast ? static_cast<int>(fast_smem(c)) : static_cast<int>(kBatchSmem);
    const unsigned threads = fast ? static_cast<unsigned>(kFastThreads) : static_cast<unsigned>(kThreads);
    if (!fn) {
      e = cudaErrorInvalidValue;
      break;
    }
    e = ensure_smem_attr(reinterpret_cast<const void*>(fn), smem);
    if (e != cudaSuccess) break;
    const unsigned grid = static_cast<unsigned>(std::min<uint64_t>((class_n[c] + kClaim - 1) / kClaim, sm_count()));
    const size_t items_off = class_off[c];
    const size_t counter_off = align16(class_off[c] + class_items[c] * sizeof(uint2));
    fn<<<grid, threads, smem, stream>>>(reinterpret_cast<const BatchJob*>(dbase + off_jobs),
                                        reinterpret_cast<const uint64_t*>(dbase + off_ptrs),
                                        reinterpret_cast<const uint2*>(dbase + items_off),
                                        static_cast<uint32_t>(class_n[c]),
                                        reinterpret_cast<uint32_t*>(dbase + counter_off));
    e = cudaGetLastError();
  }
  if (e != cudaSuccess) {
    snprintf(msg, msglen, "batch_run_noalloc: CUDA error: %s", cudaGetErrorString(e));
    return FGFC_ERR_CUDA;
  }
  return 0;
}

}  // namespace fgfc
