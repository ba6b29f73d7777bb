// gf2mma.cu -- the matrix ops as a bit-sliced GF(2) contraction on the
// tensor cores (tcgen05, sm_100a).
//
// Multiplying a packed element by a fixed coefficient is linear over GF(2):
// the 8E output bits of c * x are XORs of the 8E input bits of x. So for one
// element column (one element position of every source and row) the whole
// op rows[j] (^)= XOR_t c[t][j] * src_t is one GF(2) matrix-vector product:
// out (8E * m bits) = A (8E*m x 8E*k) . in (8E*k bits). It is evaluated as an
// integer matrix product whose bit 7 is the parity:
//
//   D[n][col] = sum_kappa A[n][kappa] * B[kappa][col]     (tcgen05.mma kind::i8)
//
// with A the plan's bit matrix (M = 128 output bits, one TMEM lane each, rows
// past the 8E*m real ones zero; K = input bits) and B the input bits of 256
// element columns (N = 256). Putting the columns on N makes every product the
// largest the instruction takes (M = 128, N = 256, K = 32); its cost on this
// part hardly depends on N, so fewer, wider products are what the contraction
// needs. The input bit b of a byte enters B as the value 2^b (the byte masked
// with 0x01010101 << b, one LOP3 per 4 values) and A holds 2^(7-b) where the
// bit matrix has a 1, so every product is 0 or 128 and D = 128 * (number of 1
// products): its bit 7 is the GF(2) sum, bits 0..6 are zero. Sums stay below
// 2^23 (at most 512 products of 2^14), so the int32 accumulator is exact.
//
// Layout and flow of one CTA (one per SM, persistent over 512-column blocks,
// two 256-column tiles each):
//   * the producer warp stages the k source rows of a block (512 * E bytes
//     per source) into a 2..4-deep shared-memory ring with cp.async.bulk
//     (single GPU, no multicast), completion on an mbarrier;
//   * warps 0..7 (expanders; thread i owns column i of a tile): gather the
//     column's input bytes from the stage and write its expanded input bits
//     into a ring of B slots in shared memory (4 input groups, K = 128, per
//     slot), each slot handed to the issuer through an mbarrier;
//   * warp 17 (issuer): allocates TMEM (two D buffers of 256 columns),
//     issues the K/32 products of a tile from one lane, A and B
//     both from shared memory, commits each slot back to the expanders once
//     its products are done and the tile to the epilogue;
//   * warps 8..15 (epilogue, two per TMEM lane quarter = 4 output bytes,
//     one per half of the tile's columns): read D back 32 columns at a time
//     (tcgen05.ld), pack bit 7 of each lane's 32 accumulators into a word,
//     transpose the warp's 32 words (5 shuffle steps) so that lane c holds
//     column c's 4 output bytes, release D and store;
//   * warp 16 (producer): see above, every lane issuing copies.
// Every mbarrier wait is bounded: a wait that runs out sets the error word,
// stops the CTA's loops, waits (bounded) for its own copies and products in
// flight and frees TMEM before returning.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <vector>

#include "fast_core.cuh"
#include "internal.hpp"

namespace fgfc {

namespace {

constexpr int kExpandWarps = 8;                        // warps 0 .. 7: expand inputs into B slots
constexpr int kEpilogueWarps = 8;                      // warps 8 .. 15: read D back, two per lane quarter
constexpr int kProducerWarp = kExpandWarps + kEpilogueWarps;  // bulk copies of source blocks
constexpr int kIssuerWarp = kProducerWarp + 1;         // TMEM allocation and the products
constexpr int kMmaThreads = (kIssuerWarp + 1) * 32;    // 576
constexpr uint32_t kCols = 512;        // element columns per block (2 tiles of 256)
constexpr uint32_t kMaxInBits = 512;   // K
constexpr uint32_t kMaxOutBits = 128;  // M
constexpr uint32_t kTmemCols = 512;
constexpr int kMaxLaunchSmem = 227 * 1024;  // the opt-in every launch fits under
constexpr uint64_t kWaitNs = 2000000000ull;   // 2 s: a wait this long means the pipeline is stuck
constexpr uint64_t kDrainNs = 1000000000ull;  // 1 s per drain wait before the CTA exits

// Error word of this device's launches (0 = fine): a bounded wait that ran
// out records where. Read and cleared by gf2mma_error.
__device__ int g_gf2_err;

struct Gf2Launch {
  const uint8_t* src[kMaxSrc];  // kMaxSrc >= 64 sources
  uint8_t* dst[16];             // rows
  uint64_t nblk;                // 512-column blocks
  uint32_t k, m, E;
  uint32_t ngroups;             // K / 32: groups of 4 input bytes
  uint32_t nstages, nslots;     // source stages and B slots in shared memory
  uint32_t overwrite;
  // Several stripes sharing this plan (nstripes > 0): stripe s owns blocks
  // [prefix[s], prefix[s + 1]) and its k source and m row pointers are
  // ptrs[s * (k + m) ..]; with nstripes == 0 the single stripe is src / dst.
  const uint64_t* ptrs;
  const uint64_t* prefix;
  uint32_t nstripes;
  // bits[n][g]: bit (8r + b) set iff output bit n takes input byte 4g + r, bit b
  uint32_t bits[kMaxOutBits][kMaxInBits / 32];
};
static_assert(sizeof(Gf2Launch) <= 32000, "launch parameter block too large");

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(b)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Wait bounded in time (every wait of a correct run lasts microseconds);
// false when it ran out. With `honor_abort` it also gives up once another
// role has aborted (the drain waits before exit do not). Between tries the
// thread sleeps (16 ns, doubling up to `max_sleep_ns`): back-to-back
// try_wait polling by a dozen waiting warps takes so much of the shared
// memory pipe that the tensor cores' operand reads slow several-fold.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort, bool honor_abort = true,
                                          uint32_t max_sleep_ns = 256) {
  if (mbar_try(b, parity)) return true;
  const uint64_t t0 = global_ns();
  const uint64_t limit = honor_abort ? kWaitNs : kDrainNs;
  uint32_t sleep_ns = 16;
  for (uint32_t i = 1;; ++i) {
    __nanosleep(sleep_ns);
    if (mbar_try(b, parity)) return true;
    sleep_ns = min(2u * sleep_ns, max_sleep_ns);
    if ((i & 15u) == 0) {
      if (honor_abort && *abort) return false;
      if (global_ns() - t0 > limit) return false;
    }
  }
}

// The same wait by every lane of a warp, with a warp-uniform result (the
// tcgen05 .sync.aligned instructions that follow need the whole warp).
__device__ __forceinline__ bool warp_wait(uint64_t* b, uint32_t parity, volatile int* abort,
                                          uint32_t max_sleep_ns = 256) {
  const bool ok = mbar_wait(b, parity, abort, true, max_sleep_ns);
  return __all_sync(0xffffffffu, ok);
}

__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,%17,%18,"
      "%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]),
        "=r"(v[17]), "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]), "=r"(v[24]),
        "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]), "=r"(v[30]), "=r"(v[31])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of 8
// rows x 16 bytes (128 contiguous bytes); `lbo` = bytes between the two
// 16-byte K halves of a 32-byte K step, `sbo` = bytes between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_i8_ss(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
      "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
      : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// The stripe of a block. A CTA meets its blocks in increasing order, so the
// cursor only walks forward.
struct StripeCursor {
  uint32_t s = 0;
  // Address of column block `blk` of source t (t < k) or row t - k.
  template <int E>
  __device__ __forceinline__ uint8_t* at(const Gf2Launch& a, uint64_t blk, uint32_t t) {
    if (!a.nstripes) return (t < a.k ? const_cast<uint8_t*>(a.src[t]) : a.dst[t - a.k]) + blk * kCols * E;
    while (s + 1 < a.nstripes && a.prefix[s + 1] <= blk) ++s;
    return reinterpret_cast<uint8_t*>(a.ptrs[static_cast<uint64_t>(s) * (a.k + a.m) + t]) +
           (blk - a.prefix[s]) * kCols * E;
  }
};

// Shared memory of a CTA: [A image: the bit matrix, 4 KiB per input group]
// [B slots: kSlotGroups groups of expanded inputs each, 8 KiB per group]
// [source stages: one 512-column block of every source each] [Smem].
// TMEM holds two D buffers of 256 columns (one per tile in flight).
constexpr uint32_t kTileCols = 256;                  // N: element columns per product
constexpr uint32_t kSlotGroups = 4;                  // input groups (K = 128) per B slot
constexpr uint32_t kGroupBytes = kTileCols * 32u;    // one group of a tile: 256 columns x 32 K-bytes
constexpr uint32_t kSlotBytes = kSlotGroups * kGroupBytes;
constexpr uint32_t kABytesPerGroup = 128u * 32u;     // M = 128 output bits x 32 K-bytes
constexpr int kMaxStages = 4;
constexpr int kMaxSlots = 6;
constexpr uint32_t kDBufs = 2;  // the issuer and epilogue index D by t & 1
static_assert(kDBufs * kTileCols <= kTmemCols, "TMEM budget");

struct Smem {
  uint64_t full[kMaxStages], empty[kMaxStages], bfull[kMaxSlots], bempty[kMaxSlots], dfull[kDBufs], dempty[kDBufs];
  uint32_t tmem_base;
  int abort;
};

// Position in a ring of n barrier-guarded buffers: the buffer index and the
// phase parity of its current use; `reused` once a full turn has been made
// (from then on a buffer must be released before it is filled again). Kept
// incrementally: the loops that walk the rings do no division.
struct Ring {
  uint32_t n, i = 0, ph = 0;
  bool reused = false;
  __device__ __forceinline__ explicit Ring(uint32_t count) : n(count) {}
  __device__ __forceinline__ void next() {
    if (++i == n) {
      i = 0;
      ph ^= 1u;
      reused = true;
    }
  }
};

__device__ __forceinline__ void sts128(uint32_t addr, uint32_t x, uint32_t y, uint32_t z, uint32_t w) {
  asm volatile("st.shared.v4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "r"(x), "r"(y), "r"(z), "r"(w) : "memory");
}

// Input bytes 4g .. 4g + 3 of element column `col` of the staged block
// (input byte u = t * E + p: byte p of source t's element), byte r of the
// result = input byte 4g + r; bytes past the k * E input bytes are zero.
template <int E>
__device__ __forceinline__ uint32_t gather_group(const uint8_t* st, uint32_t g, uint32_t col, uint32_t k) {
  if (E == 1) {
    uint32_t v = 0;
#pragma unroll
    for (uint32_t r = 0; r < 4; ++r) {
      const uint32_t t = 4u * g + r;
      if (t < k) v |= static_cast<uint32_t>(st[t * kCols + col]) << (8 * r);
    }
    return v;
  } else if (E == 2) {
    const uint32_t t = 2u * g;
    const uint32_t lo = reinterpret_cast<const uint16_t*>(st + t * kCols * 2u)[col];
    const uint32_t hi = t + 1 < k ? reinterpret_cast<const uint16_t*>(st + (t + 1) * kCols * 2u)[col] : 0u;
    return lo | (hi << 16);
  } else {
    return reinterpret_cast<const uint32_t*>(st + g * kCols * 4u)[col];
  }
}

// Expander warps 0..7: thread i owns element column i of every tile. For each
// B slot of a tile it writes the slot's groups of its column: group g, bit b
// of input byte 4g + r becomes K-byte 4b + r of the group with the value 2^b
// (the 4 input bytes masked with 0x01010101 << b), K-bytes 0..15 and 16..31
// in the two 16-byte halves of the column's row (LBO apart).
template <int E>
__device__ __forceinline__ void expander_loop(const Gf2Launch& a, Smem& S, const uint8_t* stages, uint32_t stage_bytes,
                                              uint32_t nstages, uint32_t slots, uint32_t nslots, uint64_t nmine,
                                              volatile int* abort) {
  const uint32_t i = threadIdx.x, lane = i & 31u;
  const uint32_t nq = (a.ngroups + kSlotGroups - 1) / kSlotGroups;  // slots per tile
  bool ok = true;
  Ring st(nstages), sl(nslots);
  for (uint64_t it = 0; it < nmine && ok; ++it, st.next()) {
    if (!warp_wait(&S.full[st.i], st.ph, abort)) {
      ok = false;
      break;
    }
    const uint8_t* stp = stages + st.i * stage_bytes;
    for (uint32_t T = 0; T < kCols / kTileCols && ok; ++T) {
      const uint32_t col = T * kTileCols + i;
      for (uint32_t j = 0; j < nq; ++j, sl.next()) {
        if (sl.reused && !warp_wait(&S.bempty[sl.i], sl.ph ^ 1u, abort, 64)) {
          ok = false;
          break;
        }
        const uint32_t sbase = slots + sl.i * kSlotBytes + i * 16u;
#pragma unroll
        for (uint32_t gg = 0; gg < kSlotGroups; ++gg) {
          const uint32_t g = kSlotGroups * j + gg;
          if (g >= a.ngroups) break;  // uniform
          const uint32_t w = gather_group<E>(stp, g, col, a.k);
          const uint32_t base = sbase + gg * kGroupBytes;
          sts128(base, w & 0x01010101u, w & 0x02020202u, w & 0x04040404u, w & 0x08080808u);
          sts128(base + kGroupBytes / 2, w & 0x10101010u, w & 0x20202020u, w & 0x40404040u, w & 0x80808080u);
        }
        // generic-proxy writes become visible to the tensor cores' reads
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&S.bfull[sl.i]);
      }
    }
    __syncwarp();
    if (lane == 0) mbar_arrive(&S.empty[st.i]);  // both tiles read: the stage may be refilled
  }
  if (!ok) {
    atomicExch(&g_gf2_err, 3);
    *abort = 1;
  }
}

// Bits 7 of 8 accumulators as one byte (bit o = bit 7 of r[o]) in bits 24..31.
// Every accumulator is 128 * (number of 1 products), so byte 0 of each holds
// bit 7 alone: PRMT gathers the 8 low bytes into two words, and one
// multiply-add moves bit 7 of byte i to bit 24 + i (p03) or 28 + i (p47);
// the shifted copies never land on the same bit.
__device__ __forceinline__ uint32_t pack_byte(const uint32_t* r) {
  const uint32_t p03 = prmt(prmt(r[0], r[1], 0x0040u), prmt(r[2], r[3], 0x0040u), 0x5410u);
  const uint32_t p47 = prmt(prmt(r[4], r[5], 0x0040u), prmt(r[6], r[7], 0x0040u), 0x5410u);
  return (p03 >> 4) * 0x00204081u + p47 * 0x00204081u;
}

// 32 x 32 bit-matrix transpose across a warp: on entry bit c of lane l's word
// is M[l][c], on return bit c of lane l's word is M[c][l]. Five exchange
// steps swap the off-diagonal j x j blocks of every 2j x 2j block.
__device__ __forceinline__ uint32_t warp_transpose32(uint32_t x, uint32_t lane) {
#pragma unroll
  for (uint32_t j = 16; j >= 1; j >>= 1) {
    const uint32_t lo = j == 16 ? 0x0000FFFFu : j == 8 ? 0x00FF00FFu : j == 4 ? 0x0F0F0F0Fu : j == 2 ? 0x33333333u : 0x55555555u;
    const uint32_t y = __shfl_xor_sync(0xffffffffu, x, j);
    x = (lane & j) ? ((x & ~lo) | ((y >> j) & lo)) : ((x & lo) | ((y << j) & ~lo));
  }
  return x;
}

// Output words of 4 consecutive columns (w[x] = output bytes 4q .. 4q + 3 of
// column colb + x, byte i = output byte 4q + i) into the rows they belong to.
template <int E>
__device__ __forceinline__ void store_columns(const Gf2Launch& a, StripeCursor& cur, uint64_t blk, uint32_t colb,
                                              uint32_t q, const uint32_t (&w)[4]) {
  if (E == 4) {  // row q: 4 elements
    if (q >= a.m) return;
    uint4* p = reinterpret_cast<uint4*>(cur.at<E>(a, blk, a.k + q) + colb * 4u);
    uint4 v = make_uint4(w[0], w[1], w[2], w[3]);
    if (!a.overwrite) {
      const uint4 d = *p;
      v.x ^= d.x; v.y ^= d.y; v.z ^= d.z; v.w ^= d.w;
    }
    *p = v;
  } else if (E == 2) {  // rows 2q (low halves) and 2q + 1 (high halves)
#pragma unroll
    for (uint32_t h = 0; h < 2; ++h) {
      const uint32_t j = 2u * q + h;
      if (j >= a.m) break;
      const uint32_t sel = h ? 0x7632u : 0x5410u;
      uint2 v = make_uint2(prmt(w[0], w[1], sel), prmt(w[2], w[3], sel));
      uint2* p = reinterpret_cast<uint2*>(cur.at<E>(a, blk, a.k + j) + colb * 2u);
      if (!a.overwrite) {
        const uint2 d = *p;
        v.x ^= d.x;
        v.y ^= d.y;
      }
      *p = v;
    }
  } else {  // rows 4q + r: byte r of every word
#pragma unroll
    for (uint32_t r = 0; r < 4; ++r) {
      const uint32_t j = 4u * q + r;
      if (j >= a.m) break;
      const uint32_t sel = r | ((4u + r) << 4);
      uint32_t v = prmt(prmt(w[0], w[1], sel), prmt(w[2], w[3], sel), 0x5410u);
      uint32_t* p = reinterpret_cast<uint32_t*>(cur.at<E>(a, blk, a.k + j) + colb);
      if (!a.overwrite) v ^= *p;
      *p = v;
    }
  }
}

// Epilogue warps 8 .. 15: warp e reads TMEM lane quarter q = e % 4 (output
// bits 32q .. 32q + 31, i.e. output bytes 4q .. 4q + 3) for the half
// h = (e - 8) / 4 of the tile's columns (128 columns), 32 columns per load.
// Lane l packs bit 7 of its 32 accumulators (output bit 32q + l of 32
// columns) into one word; a warp transpose of those 32 words gives lane c the
// 4 output bytes of column c. D is released once the half is read; 16
// shuffles then hand lane l the 4 consecutive columns 4l .. 4l + 3 it stores.
template <int E>
__device__ __forceinline__ void epilogue_loop(const Gf2Launch& a, Smem& S, uint64_t ntiles, uint32_t d_base,
                                              volatile int* abort) {
  constexpr uint32_t kHalfCols = kTileCols / 2u;
  constexpr uint32_t kChunks = kHalfCols / 32u;
  static_assert(kChunks == 4, "the regroup below hands each lane 4 columns of one chunk");
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t q = warp & 3u, half = (warp - kExpandWarps) >> 2;
  const uint32_t lane_base = (32u * q) << 16;
  const bool active = 4u * q < a.m * E;  // warp-uniform: this quarter holds output bytes
  StripeCursor cur;
  bool ok = true;
  for (uint64_t t = 0; t < ntiles; ++t) {
    const uint32_t d = static_cast<uint32_t>(t & 1u);
    if (!warp_wait(&S.dfull[d], static_cast<uint32_t>((t >> 1) & 1u), abort, 128)) {
      ok = false;
      break;
    }
    tc_fence_after();
    uint32_t w[kChunks];
#pragma unroll
    for (uint32_t ch = 0; ch < kChunks; ++ch) w[ch] = 0;
    if (active) {
      const uint32_t col0 = d_base + kTileCols * d + kHalfCols * half;
#pragma unroll
      for (uint32_t ch = 0; ch < kChunks; ++ch) {
        uint32_t r[32];
        tmem_ld32(lane_base | (col0 + 32u * ch), r);
        tmem_wait_ld();
        const uint32_t b0 = pack_byte(r), b1 = pack_byte(r + 8), b2 = pack_byte(r + 16), b3 = pack_byte(r + 24);
        w[ch] = prmt(prmt(b0, b1, 0x0073u), prmt(b2, b3, 0x0073u), 0x5410u);  // bit c = column c
      }
    }
    tc_fence_before();
    __syncwarp();
    if (lane == 0) mbar_arrive(&S.dempty[d]);  // a later product may overwrite D
    if (active) {
      // lane c of chunk ch holds column 32 ch + c; regroup so that lane l
      // holds columns 4l .. 4l + 3 (chunk l / 8, lanes 4 (l % 8) + x)
      uint32_t o[4] = {0u, 0u, 0u, 0u};
#pragma unroll
      for (uint32_t ch = 0; ch < kChunks; ++ch) {
        const uint32_t tw = warp_transpose32(w[ch], lane);
#pragma unroll
        for (uint32_t x = 0; x < 4; ++x) {
          const uint32_t v = __shfl_sync(0xffffffffu, tw, 4u * (lane & 7u) + x);
          if ((lane >> 3) == ch) o[x] = v;
        }
      }
      const uint64_t blk = blockIdx.x + (t >> 1) * gridDim.x;
      store_columns<E>(a, cur, blk, static_cast<uint32_t>(t & 1u) * kTileCols + kHalfCols * half + 4u * lane, q, o);
    }
  }
  if (!ok) {
    atomicExch(&g_gf2_err, 4);
    *abort = 1;
  }
}

template <int E>
__global__ void __launch_bounds__(kMmaThreads, 1) gf2mma_kernel(const __grid_constant__ Gf2Launch a) {
  const uint32_t K = a.ngroups * 32u;
  const uint32_t a_bytes = a.ngroups * kABytesPerGroup;
  const uint32_t stage_bytes = (a.k * kCols * E + 127u) & ~127u;
  uint8_t* aimg = g_smem;
  uint8_t* slots = g_smem + a_bytes;
  uint8_t* stages = slots + a.nslots * kSlotBytes;
  Smem& S = *reinterpret_cast<Smem*>(stages + a.nstages * stage_bytes);
  volatile int* abort = &S.abort;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;

  // ---- A image: entry (n, kappa = 32 g + 4 b + r) = 2^(7 - b) where output
  // bit n takes bit b of input byte 4 g + r; core matrix (kappa / 16, n / 8) at
  // ((kappa / 16) * 16 + n / 8) * 128, row n % 8, byte kappa % 16 (M = 128
  // rows, the rows past the m * E * 8 output bits zero)
  for (uint32_t idx = threadIdx.x; idx < 128u * K / 16u; idx += blockDim.x) {
    const uint32_t core = idx >> 3, row = idx & 7u;
    const uint32_t kc = core >> 4, n = (core & 15u) * 8u + row;
    uint32_t w[4];
#pragma unroll
    for (int qd = 0; qd < 4; ++qd) {
      uint32_t v = 0;
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        const uint32_t kappa = kc * 16u + qd * 4u + x;
        const uint32_t g = kappa >> 5, b = (kappa >> 2) & 7u, r = kappa & 3u;
        const uint32_t bit = (a.bits[n][g] >> (8u * r + b)) & 1u;
        v |= (bit << (7u - b)) << (8 * x);
      }
      w[qd] = v;
    }
    *reinterpret_cast<uint4*>(aimg + static_cast<size_t>(idx) * 16u) = make_uint4(w[0], w[1], w[2], w[3]);
  }
  if (threadIdx.x == 0) {
    for (uint32_t s = 0; s < a.nstages; ++s) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], kExpandWarps);
    }
    for (uint32_t s = 0; s < a.nslots; ++s) {
      mbar_init(&S.bfull[s], kExpandWarps);
      mbar_init(&S.bempty[s], 1);
    }
    for (uint32_t d = 0; d < kDBufs; ++d) {
      mbar_init(&S.dfull[d], 1);
      mbar_init(&S.dempty[d], kEpilogueWarps);
    }
    S.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // generic-proxy writes of the A image become visible to the tensor cores
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (warp == kIssuerWarp) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&S.tmem_base)),
                 "r"(kTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t d_base = S.tmem_base;  // kDBufs buffers x 256 columns

  // blocks of this CTA: blockIdx.x, + gridDim.x, ...; two tiles each
  const uint64_t nmine = a.nblk > blockIdx.x ? (a.nblk - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  const uint64_t ntiles = nmine * (kCols / kTileCols);

  if (warp == kProducerWarp) {
    // ---- producer: lane 0 arms the stage's barrier, every lane issues copies
    const uint32_t row_bytes = kCols * E;
    StripeCursor cur;
    uint64_t issued = 0;
    Ring st(a.nstages);
    for (uint64_t i = 0; i < nmine; ++i, st.next()) {
      const uint32_t s = st.i;
      int go = 1;
      if (lane == 0) {
        go = !*abort;
        if (go && st.reused && !mbar_wait(&S.empty[s], st.ph ^ 1u, abort)) {
          atomicExch(&g_gf2_err, 1);
          *abort = 1;
          go = 0;
        }
        if (go) mbar_expect_tx(&S.full[s], a.k * row_bytes);
      }
      go = __shfl_sync(0xffffffffu, go, 0);
      if (!go) break;
      const uint64_t blk = blockIdx.x + i * gridDim.x;
      for (uint32_t t = lane; t < a.k; t += 32)
        bulk_g2s(stages + s * stage_bytes + t * row_bytes, cur.at<E>(a, blk, t), row_bytes, &S.full[s]);
      ++issued;
    }
    // copies still in flight must land before the CTA exits
    if (lane == 0)
      for (uint64_t i = issued > a.nstages ? issued - a.nstages : 0; i < issued; ++i)
        mbar_wait(&S.full[i % a.nstages], static_cast<uint32_t>((i / a.nstages) & 1u), abort, false);
  } else if (warp == kIssuerWarp) {
    // ---- issuer: the whole warp walks the schedule, lane 0 issues (and commits)
    const uint32_t idesc = (2u << 4) | ((kTileCols >> 3) << 17) | ((128u >> 4) << 24);  // s32 += u8*u8, M=128, N=256
    const uint64_t a_desc0 = smem_desc(smem_u32(aimg), kABytesPerGroup / 2u, 128u);
    const uint64_t b_desc0 = smem_desc(smem_u32(slots), kGroupBytes / 2u, 128u);
    const uint32_t nq = (a.ngroups + kSlotGroups - 1) / kSlotGroups;
    uint64_t t = 0;
    Ring sl(a.nslots);
    bool ok = true;
    for (; t < ntiles && ok; ++t) {
      const uint32_t d = static_cast<uint32_t>(t & 1u);
      if (t >= kDBufs && !warp_wait(&S.dempty[d], static_cast<uint32_t>(((t >> 1) - 1u) & 1u), abort, 32)) {
        ok = false;
        break;
      }
      const uint32_t dcol = d_base + kTileCols * d;
      uint64_t ad = a_desc0;  // advanced by lane 0, the lane that issues
      uint32_t acc = 0;       // the tile's first product overwrites D
      for (uint32_t j = 0; j < nq; ++j, sl.next()) {
        if (!warp_wait(&S.bfull[sl.i], sl.ph, abort, 32)) {
          ok = false;
          break;
        }
        tc_fence_after();
        if (lane == 0) {
          const uint32_t gn = min(kSlotGroups, a.ngroups - kSlotGroups * j);
          uint64_t bd = b_desc0 + sl.i * (kSlotBytes >> 4);
          for (uint32_t gg = 0; gg < gn; ++gg) {
            mma_i8_ss(dcol, ad, bd, idesc, acc);
            ad += kABytesPerGroup >> 4;
            bd += kGroupBytes >> 4;
            acc = 1;
          }
          mma_commit(&S.bempty[sl.i]);  // the slot may be refilled once its products are done
        }
        __syncwarp();
      }
      if (!ok) break;
      if (lane == 0) mma_commit(&S.dfull[d]);
      __syncwarp();
    }
    if (!ok) {
      if (lane == 0) atomicExch(&g_gf2_err, 2);
      *abort = 1;
    }
    // the last products must finish before TMEM is freed
    if (lane == 0)
      for (uint64_t u = t > kDBufs ? t - kDBufs : 0; u < t; ++u)
        mbar_wait(&S.dfull[u % kDBufs], static_cast<uint32_t>((u / kDBufs) & 1u), abort, false);
    __syncwarp();
  } else if (warp < kExpandWarps) {
    expander_loop<E>(a, S, stages, stage_bytes, a.nstages, smem_u32(slots), a.nslots, nmine, abort);
  } else {
    epilogue_loop<E>(a, S, ntiles, d_base, abort);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kIssuerWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(d_base), "r"(kTmemCols) : "memory");
}

}  // namespace

bool gf2mma_shape_ok(int field, size_t k, size_t m) {
  const int E = field_bytes(field);
  return E > 0 && E <= 4 && k >= 1 && m >= 1 && k * E <= kMaxInBits / 8 && m * E <= kMaxOutBits / 8;
}

// Bit matrix of a coefficient matrix (term-major, k x m): bits[n][g] bit
// (8r + b) = output bit n (byte n / 8 of the m*E output bytes, bit n % 8)
// depends on bit b of input byte 4g + r (input byte u = t * E + p).
void gf2mma_bits(int field, const uint64_t* coeffs, size_t k, size_t m, uint32_t* bits /* [128][16] */) {
  const int E = field_bytes(field);
  std::memset(bits, 0, kMaxOutBits * (kMaxInBits / 32) * sizeof(uint32_t));
  for (size_t t = 0; t < k; ++t)
    for (size_t j = 0; j < m; ++j) {
      uint64_t img[8][8];
      coeff_images(field, coeffs[t * m + j], img);
      for (int p = 0; p < E; ++p) {
        const size_t u = t * E + p;
        for (int b = 0; b < 8; ++b) {
          const uint64_t prod = img[p][b];  // c * (bit b of input byte p), E bytes
          for (int ob = 0; ob < 8 * E; ++ob)
            if ((prod >> ob) & 1u) {
              const size_t n = j * E * 8 + ob;
              bits[n * (kMaxInBits / 32) + u / 4] |= 1u << (8 * (u % 4) + b);
            }
        }
      }
    }
}

namespace {

cudaError_t launch_common(Gf2Launch& a, int field, size_t k, size_t m, const uint32_t* bits, uint64_t nblk,
                          bool overwrite, cudaStream_t stream) {
  const int E = field_bytes(field);
  a.nblk = nblk;
  a.k = static_cast<uint32_t>(k);
  a.m = static_cast<uint32_t>(m);
  a.E = static_cast<uint32_t>(E);
  a.ngroups = static_cast<uint32_t>((k * E + 3) / 4);
  a.overwrite = overwrite ? 1u : 0u;
  std::memcpy(a.bits, bits, sizeof a.bits);
  // shared memory: the A image, then at least 2 B slots and 2 source stages;
  // what is left buys a third slot, then up to kMaxStages stages, then up to
  // kMaxSlots slots
  const size_t a_bytes = static_cast<size_t>(a.ngroups) * kABytesPerGroup;
  const size_t stage_bytes = (static_cast<size_t>(k) * kCols * E + 127u) & ~static_cast<size_t>(127u);
  uint32_t nst = 2, nsl = 2;
  const auto total = [&](uint32_t st, uint32_t sl) { return a_bytes + sl * kSlotBytes + st * stage_bytes + sizeof(Smem); };
  if (nsl < 3 && total(nst, 3) <= kMaxLaunchSmem) nsl = 3;
  while (nst < kMaxStages && total(nst + 1, nsl) <= kMaxLaunchSmem) ++nst;
  while (nsl < kMaxSlots && total(nst, nsl + 1) <= kMaxLaunchSmem) ++nsl;
  if (total(nst, nsl) > kMaxLaunchSmem) return cudaErrorInvalidValue;
  a.nstages = nst;
  a.nslots = nsl;
  const int smem = static_cast<int>(total(nst, nsl));
  const void* fn = E == 1 ? reinterpret_cast<const void*>(gf2mma_kernel<1>)
                          : (E == 2 ? reinterpret_cast<const void*>(gf2mma_kernel<2>)
                                    : reinterpret_cast<const void*>(gf2mma_kernel<4>));
  // one CTA per SM: TMEM (512 columns) is allocated whole
  const int smem_launch = std::max(smem, 116 * 1024);
  cudaError_t e = ensure_smem_attr(fn, kMaxLaunchSmem);
  if (e != cudaSuccess) return e;
  const unsigned grid = static_cast<unsigned>(std::min<uint64_t>(nblk, static_cast<uint64_t>(sm_count())));
  if (E == 1)
    gf2mma_kernel<1><<<grid, kMmaThreads, smem_launch, stream>>>(a);
  else if (E == 2)
    gf2mma_kernel<2><<<grid, kMmaThreads, smem_launch, stream>>>(a);
  else
    gf2mma_kernel<4><<<grid, kMmaThreads, smem_launch, stream>>>(a);
  return cudaGetLastError();
}

}  // namespace

cudaError_t gf2mma_prepare(int E) {
  const void* fn = E == 1 ? reinterpret_cast<const void*>(gf2mma_kernel<1>)
                          : (E == 2 ? reinterpret_cast<const void*>(gf2mma_kernel<2>)
                                    : reinterpret_cast<const void*>(gf2mma_kernel<4>));
  return ensure_smem_attr(fn, kMaxLaunchSmem);
}

// Rows [0, nblk * 512 * E) of every source and row, all 16-byte aligned.
cudaError_t gf2mma_launch(int field, const uint8_t* const* srcs, size_t k, uint8_t* const* rows, size_t m,
                          const uint32_t* bits, uint64_t nblk, bool overwrite, cudaStream_t stream) {
  if (!nblk) return cudaSuccess;
  static thread_local Gf2Launch a;
  for (size_t t = 0; t < k; ++t) a.src[t] = srcs[t];
  for (size_t j = 0; j < m; ++j) a.dst[j] = rows[j];
  a.ptrs = a.prefix = nullptr;
  a.nstripes = 0;
  return launch_common(a, field, k, m, bits, nblk, overwrite, stream);
}

// Several stripes of one plan: ptrs / prefix are device arrays (see Gf2Launch).
cudaError_t gf2mma_launch_multi(int field, size_t k, size_t m, const uint32_t* bits, const uint64_t* ptrs,
                                const uint64_t* prefix, uint32_t nstripes, uint64_t nblk, bool overwrite,
                                cudaStream_t stream) {
  if (!nblk || !nstripes) return cudaSuccess;
  static thread_local Gf2Launch a;
  a.ptrs = ptrs;
  a.prefix = prefix;
  a.nstripes = nstripes;
  return launch_common(a, field, k, m, bits, nblk, overwrite, stream);
}

// Error word of the current device: nonzero when a bounded wait ran out.
int gf2mma_error(bool clear) {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_gf2_err, sizeof v) != cudaSuccess) return -1;
  if (clear && v) {
    const int zero = 0;
    if (cudaMemcpyToSymbol(g_gf2_err, &zero, sizeof zero) != cudaSuccess) return -1;
  }
  return v;
}

}  // namespace fgfc
