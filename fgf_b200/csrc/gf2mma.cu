// gf2mma.cu -- the matrix ops as a bit-sliced GF(2) contraction on the
// tensor cores (tcgen05, sm_100a).
//
// Multiplying a packed element by a fixed coefficient is linear over GF(2):
// the 8E output bits of c * x are XORs of the 8E input bits of x. So for one
// element column (one element position of every source and row) the whole
// op rows[j] (^)= XOR_t c[t][j] * src_t is one GF(2) matrix-vector product:
// out (8E * m bits) = B (8E*m x 8E*k) . in (8E*k bits). It is evaluated as an
// integer matrix product whose low bit is the parity:
//
//   D[col][n] = sum_kappa A[col][kappa] * B[kappa][n]     (tcgen05.mma kind::i8)
//
// with A the input bits of 128 element columns (M = 128, one TMEM lane per
// column) and B the plan's bit matrix (N = output bits, K = input bits). The
// input bit b of a byte enters A as the value 2^b (the byte masked with
// 0x01010101 << b, one LOP3 per 4 values) and B holds 2^(7-b) where the bit
// matrix has a 1, so every product is 0 or 128 and D = 128 * (number of 1
// products): its bit 7 is the GF(2) sum, bits 0..6 are zero. Sums stay below
// 2^23 (at most 512 products of 2^14), so the int32 accumulator is exact.
//
// Layout and flow of one CTA (one per SM, persistent over 512-column blocks):
//   * the producer warp stages the k source rows of a block (512 columns,
//     512 * E bytes per source) into a 4-deep shared-memory ring with
//     cp.async.bulk (single GPU, no multicast), completion on an mbarrier;
//   * warps 0..7 (expanders; thread i of a lane quarter owns TMEM lane i):
//     read the 4 consecutive columns 4i..4i+3 of their half of the sources
//     into registers, then for each of the block's 4 tiles (tile q = columns
//     4i + q) build their half of the A lane and write it with tcgen05.st;
//   * warps 8..15 (epilogue): when a tile's product is done, read their half
//     of D back (tcgen05.ld), release the buffer, gather bit 7 of every
//     accumulator into output bytes with PRMT and two multiply-adds, and
//     after the 4th tile store 4 consecutive columns of their rows;
//   * warp 16 (producer): see above, every lane issuing copies;
//   * warp 17 (issuer): allocates TMEM (A and D double-buffered, 512 columns),
//     issues K/32 tcgen05.mma per tile from one thread and commits each tile
//     to an mbarrier.
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

constexpr int kExpandWarps = 8;                        // warps 0 .. 7: write A lanes
constexpr int kWorkerWarps = 16;                       // + warps 8 .. 15: read D back
constexpr int kProducerWarp = kWorkerWarps;            // bulk copies of source blocks
constexpr int kIssuerWarp = kWorkerWarps + 1;          // TMEM allocation and the products
constexpr int kMmaThreads = (kWorkerWarps + 2) * 32;   // 576
constexpr int kStages = 4;
constexpr uint32_t kCols = 512;        // element columns per block (4 tiles of 128)
constexpr uint32_t kMaxInBits = 512;   // K
constexpr uint32_t kMaxOutBits = 128;  // N
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
  uint32_t npad;                // N: output bits padded to a multiple of 16
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
// role has aborted (the drain waits before exit do not).
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort, bool honor_abort = true) {
  if (mbar_try(b, parity)) return true;
  const uint64_t t0 = global_ns();
  const uint64_t limit = honor_abort ? kWaitNs : kDrainNs;
  for (uint32_t i = 1;; ++i) {
    if (mbar_try(b, parity)) return true;
    if ((i & 255u) == 0) {
      if (honor_abort && *abort) return false;
      if (global_ns() - t0 > limit) return false;
    }
  }
}

// The same wait by every lane of a warp, with a warp-uniform result (the
// tcgen05 .sync.aligned instructions that follow need the whole warp).
__device__ __forceinline__ bool warp_wait(uint64_t* b, uint32_t parity, volatile int* abort) {
  const bool ok = mbar_wait(b, parity, abort);
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

__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]), "r"(v[17]), "r"(v[18]),
      "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]), "r"(v[26]), "r"(v[27]),
      "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
      : "memory");
}

__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t* v) {
  asm volatile("tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8};" ::"r"(taddr), "r"(v[0]),
               "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7])
               : "memory");
}

__device__ __forceinline__ void tmem_st16(uint32_t taddr, const uint32_t* v) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};" ::"r"(
          taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
      : "memory");
}

__device__ __forceinline__ void tmem_ld32(uint32_t taddr, uint32_t (&v)[32]) {
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

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, uint32_t* v) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]), "=r"(v[8]),
        "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(taddr)
      : "memory");
}

__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Shared-memory matrix descriptor, K-major, no swizzle: core matrices of 8
// rows x 16 bytes (128 contiguous bytes); `lbo` = bytes between the two
// 16-byte K halves of a 32-byte K step, `sbo` = bytes between 8-row groups.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return static_cast<uint64_t>((addr >> 4) & 0x3FFFu) | (static_cast<uint64_t>((lbo >> 4) & 0x3FFFu) << 16) |
         (static_cast<uint64_t>((sbo >> 4) & 0x3FFFu) << 32) | (1ull << 46);
}

__device__ __forceinline__ void mma_i8(uint32_t d_tmem, uint32_t a_tmem, uint64_t b_desc, uint32_t idesc,
                                       uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b_desc), "r"(idesc), "r"(accumulate)
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

// Output byte from 8 accumulators (bit o of the byte = bit 7 of r[o]).
__device__ __forceinline__ uint32_t pack_byte(const uint32_t* r) {
  const uint32_t p03 = prmt(prmt(r[0], r[1], 0x0040u), prmt(r[2], r[3], 0x0040u), 0x5410u);
  const uint32_t p47 = prmt(prmt(r[4], r[5], 0x0040u), prmt(r[6], r[7], 0x0040u), 0x5410u);
  // bit 7 of byte i of p03 -> bit 24 + i; of p47 -> bit 28 + i (no carries:
  // every shifted copy lands on a distinct bit)
  return (p03 >> 4) * 0x00204081u + p47 * 0x00204081u;  // output byte in bits 24..31
}

// TMEM holds a ring of 8 A slots of 32 columns (4 input groups each, K = 128
// per slot) and 2 D buffers of 128 columns. The issuer runs a tile's products
// slot by slot (quarter j of the tile = input groups 4j .. 4j + 3) and
// commits each slot back to the expanders as soon as its products are done,
// so the expanders refill A up to two tiles ahead of the products; D is read
// back by the epilogue warps one tile behind.
constexpr uint32_t kSlots = 8;
constexpr uint32_t kSlotCols = 32;
constexpr uint32_t kDBufs = 2;
static_assert(kSlots * kSlotCols + kDBufs * 128u <= kTmemCols, "TMEM budget");

struct Smem {
  uint64_t full[kStages], empty[kStages], afull[kSlots], aempty[kSlots], dfull[kDBufs], dempty[kDBufs];
  uint32_t tmem_base;
  int abort;
};


// The 16 worker warps have two jobs. Expander warp e (0..7) and epilogue
// warp e (8..15) own TMEM lanes 32 (e % 4) .. + 31, the element columns of a
// tile, and half h = (e % 8) / 4 of their job: an expander writes input
// groups 4j + 2h and 4j + 2h + 1 of every quarter j (16 TMEM columns), an
// epilogue warp reads output bytes 8h .. 8h + 7 (D columns 64h .. 64h + 63).

// Half h's two groups of quarter j of the A lane of tile Q (column 4i + Q of
// the block) into the TMEM slot at a_col. Group g = input bytes 4g..4g+3 of
// the column (input byte u = t * E + p); TMEM column 8g + b holds bit b of
// those 4 bytes, each as the value 2^b. sw[8 c + x] is global word
// 16 c + 8 h + x (c = quarter), i.e. this thread's words of the half's
// groups.
template <int E, int Q>
__device__ __forceinline__ void expand_quarter(const Gf2Launch& a, const uint32_t (&sw)[32], uint32_t j,
                                               uint32_t a_col, uint32_t half, uint32_t lane_base) {
  const uint32_t g0 = 4u * j + 2u * half;
  if (g0 >= a.ngroups) return;  // warp-uniform
  const uint32_t nwords = a.k * E;
  uint32_t col[16];
#pragma unroll
  for (uint32_t gg = 0; gg < 2; ++gg) {
    const uint32_t gw = 4u * (g0 + gg);  // global word of the group's first input byte
    uint32_t x[4];
#pragma unroll
    for (uint32_t y = 0; y < 4; ++y) {
      // sw index of global word gw + y: quarter j, word 8h + 4gg + y within it
      uint32_t v = 0;
#pragma unroll
      for (uint32_t jj = 0; jj < 4; ++jj)
        if (jj == j) v = sw[8 * jj + 4 * gg + y];
      x[y] = gw + y < nwords ? v : 0u;
    }
    uint32_t wg;
    if (E == 1) {  // sources 4g..4g+3, byte Q of each
      constexpr uint32_t qs = Q | ((4u + Q) << 4);
      wg = prmt(prmt(x[0], x[1], qs), prmt(x[2], x[3], qs), 0x5410u);
    } else if (E == 2) {  // sources 2g, 2g+1: element Q is word Q / 2, bytes 2 (Q % 2) .. + 1
      wg = prmt(x[Q / 2], x[2 + Q / 2], (Q & 1) ? 0x7632u : 0x5410u);
    } else {  // source g, element Q
      wg = x[Q];
    }
#pragma unroll
    for (uint32_t bb = 0; bb < 8; ++bb) col[gg * 8 + bb] = wg & (0x01010101u << bb);
  }
  const uint32_t taddr = lane_base | (a_col + 8u * (2u * half));
  if (a.ngroups - g0 >= 2)
    tmem_st16(taddr, col);
  else
    tmem_st8(taddr, col);
  tmem_wait_st();
}

template <int E>
__device__ __forceinline__ void expander_loop(const Gf2Launch& a, Smem& S, const uint8_t* stages, uint32_t stage_bytes,
                                              uint64_t nmine, uint32_t a_base, volatile int* abort) {
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t half = warp >> 2, i = (warp & 3u) * 32u + lane;
  const uint32_t lane_base = ((warp & 3u) * 32u) << 16;
  const uint32_t nq = (a.ngroups + 3u) / 4u;  // quarters per tile
  uint32_t sw[32];  // sw[8 c + x] = global word 16 c + 8 h + x of this thread's 4 columns
#pragma unroll
  for (int x = 0; x < 32; ++x) sw[x] = 0;
  const uint32_t nwords = a.k * E;
  bool ok = true;
  uint64_t qi = 0;  // slots filled so far
  for (uint64_t it = 0; it < nmine && ok; ++it) {
    const uint32_t s = static_cast<uint32_t>(it % kStages);
    if (!warp_wait(&S.full[s], static_cast<uint32_t>((it / kStages) & 1u), abort)) {
      ok = false;
      break;
    }
    const uint8_t* st = stages + s * stage_bytes;
#pragma unroll
    for (uint32_t c = 0; c < 4; ++c)
#pragma unroll
      for (uint32_t x = 0; x < 8; x += E) {
        const uint32_t gw = 16u * c + 8u * half + x;
        if (gw >= nwords) break;
        const uint8_t* p = st + (gw / E) * kCols * E + i * 4u * E;
        if (E == 1) {
          sw[8 * c + x] = *reinterpret_cast<const uint32_t*>(p);
        } else if (E == 2) {
          const uint2 v = *reinterpret_cast<const uint2*>(p);
          sw[8 * c + x] = v.x;
          sw[8 * c + x + 1] = v.y;
        } else {
          const uint4 v = *reinterpret_cast<const uint4*>(p);
          sw[8 * c + x] = v.x;
          sw[8 * c + x + 1] = v.y;
          sw[8 * c + x + 2] = v.z;
          sw[8 * c + x + 3] = v.w;
        }
      }
    __syncwarp();
    if (lane == 0) mbar_arrive(&S.empty[s]);  // the stage may be refilled
#define FGFC_TILE(Q)                                                                                \
    for (uint32_t j = 0; j < nq && ok; ++j, ++qi) {                                                 \
      const uint32_t slot = static_cast<uint32_t>(qi % kSlots);                                     \
      if (qi >= kSlots)                                                                             \
        ok = warp_wait(&S.aempty[slot], static_cast<uint32_t>((qi / kSlots - 1) & 1u), abort);      \
      if (!ok) break;                                                                               \
      tc_fence_after();                                                                             \
      expand_quarter<E, Q>(a, sw, j, a_base + kSlotCols * slot, half, lane_base);                   \
      tc_fence_before();                                                                            \
      __syncwarp();                                                                                 \
      if (lane == 0) mbar_arrive(&S.afull[slot]);                                                   \
    }
    FGFC_TILE(0)
    FGFC_TILE(1)
    FGFC_TILE(2)
    FGFC_TILE(3)
#undef FGFC_TILE
  }
  if (!ok) {
    atomicExch(&g_gf2_err, 3);
    *abort = 1;
  }
}

// Epilogue of tile tt (columns 4i + Q of its block, D buffer tt % 3): read
// this half's accumulators and release the buffer, fold bit 7 of each into
// output byte 8h + v of column Q (byte Q of out[v]); after the 4th tile
// store 4 columns of this half's rows.
template <int E, int Q>
__device__ __forceinline__ bool epilogue(const Gf2Launch& a, Smem& S, uint32_t d_base, uint64_t tt,
                                         uint32_t (&out)[8], volatile int* abort, StripeCursor& cur) {
  constexpr uint32_t qsel = (0x3210u & ~(0xFu << (4 * Q))) | (7u << (4 * Q));  // byte Q <- byte 3 of the pack
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
  const uint32_t half = (warp >> 2) & 1u, i = (warp & 3u) * 32u + lane;
  const uint32_t lane_base = ((warp & 3u) * 32u) << 16;
  const uint32_t d = static_cast<uint32_t>(tt % kDBufs);
  if (!warp_wait(&S.dfull[d], static_cast<uint32_t>((tt / kDBufs) & 1u), abort)) return false;
  tc_fence_after();
  const uint32_t d_col = d_base + 128u * d;
  const uint32_t c0 = 64u * half;
  const uint32_t nout = a.m * E;
  // two 32-column loads, one at a time (registers), then the buffer is released
#pragma unroll
  for (uint32_t c = 0; c < 2; ++c) {
    const uint32_t cc = c0 + 32u * c;
    if (cc < a.npad) {  // warp-uniform
      uint32_t r[32];
      if (a.npad - cc >= 32) {
        tmem_ld32(lane_base | (d_col + cc), r);
      } else {
        tmem_ld16(lane_base | (d_col + cc), r);
#pragma unroll
        for (int x = 16; x < 32; ++x) r[x] = 0;
      }
      tmem_wait_ld();
#pragma unroll
      for (uint32_t v = 0; v < 4; ++v)
        if (8 * half + 4 * c + v < nout) out[4 * c + v] = prmt(out[4 * c + v], pack_byte(&r[8 * v]), qsel);
    }
  }
  tc_fence_before();
  __syncwarp();
  if (lane == 0) mbar_arrive(&S.dempty[d]);  // a later product may overwrite D
  if (c0 >= a.npad) return true;
  if (Q == 3) {
    const uint64_t blk = blockIdx.x + (tt >> 2) * gridDim.x;
    const uint64_t off = static_cast<uint64_t>(i) * 4u * E;
    if (E == 1) {  // rows 8h .. 8h + 7
#pragma unroll
      for (uint32_t jj = 0; jj < 8; ++jj) {
        const uint32_t j = 8 * half + jj;
        if (j >= a.m) break;
        uint32_t* p = reinterpret_cast<uint32_t*>(cur.at<E>(a, blk, a.k + j) + off);
        *p = a.overwrite ? out[jj] : (out[jj] ^ *p);
      }
    } else if (E == 2) {  // rows 4h .. 4h + 3: bytes 0 and 1 of 4 elements, interleaved
#pragma unroll
      for (uint32_t jj = 0; jj < 4; ++jj) {
        const uint32_t j = 4 * half + jj;
        if (j >= a.m) break;
        uint2* p = reinterpret_cast<uint2*>(cur.at<E>(a, blk, a.k + j) + off);
        uint2 v = make_uint2(prmt(out[2 * jj], out[2 * jj + 1], 0x5140u), prmt(out[2 * jj], out[2 * jj + 1], 0x7362u));
        if (!a.overwrite) {
          const uint2 dd = *p;
          v.x ^= dd.x;
          v.y ^= dd.y;
        }
        *p = v;
      }
    } else {  // rows 2h, 2h + 1: 4 bytes of 4 elements, transposed
#pragma unroll
      for (uint32_t jj = 0; jj < 2; ++jj) {
        const uint32_t j = 2 * half + jj;
        if (j >= a.m) break;
        uint4* p = reinterpret_cast<uint4*>(cur.at<E>(a, blk, a.k + j) + off);
        const uint32_t* o = &out[4 * jj];
        uint4 v = make_uint4(row_word4(o, 0), row_word4(o, 1), row_word4(o, 2), row_word4(o, 3));
        if (!a.overwrite) {
          const uint4 dd = *p;
          v.x ^= dd.x;
          v.y ^= dd.y;
          v.z ^= dd.z;
          v.w ^= dd.w;
        }
        *p = v;
      }
    }
  }
  return true;
}

template <int E>
__device__ __forceinline__ void epilogue_loop(const Gf2Launch& a, Smem& S, uint64_t ntiles, uint32_t d_base,
                                              volatile int* abort) {
  uint32_t out[8];  // output bytes 8h .. 8h + 7 of this thread's 4 columns
#pragma unroll
  for (int x = 0; x < 8; ++x) out[x] = 0;
  StripeCursor cur;
  bool ok = true;
  for (uint64_t t = 0; t < ntiles && ok; t += 4) {
    ok = epilogue<E, 0>(a, S, d_base, t, out, abort, cur);
    if (ok) ok = epilogue<E, 1>(a, S, d_base, t + 1, out, abort, cur);
    if (ok) ok = epilogue<E, 2>(a, S, d_base, t + 2, out, abort, cur);
    if (ok) ok = epilogue<E, 3>(a, S, d_base, t + 3, out, abort, cur);
  }
  if (!ok) {
    atomicExch(&g_gf2_err, 4);
    *abort = 1;
  }
}

template <int E>
__global__ void __launch_bounds__(kMmaThreads, 1) gf2mma_kernel(const __grid_constant__ Gf2Launch a) {
  // dynamic shared memory: [B image (npad x K bytes)] [stages] [Smem]
  const uint32_t K = a.ngroups * 32u;
  const uint32_t b_bytes = (a.npad * K + 1023u) & ~1023u;
  const uint32_t stage_bytes = (a.k * kCols * E + 127u) & ~127u;
  uint8_t* bimg = g_smem;
  uint8_t* stages = g_smem + b_bytes;
  Smem& S = *reinterpret_cast<Smem*>(stages + kStages * stage_bytes);
  volatile int* abort = &S.abort;
  const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;

  // ---- B image: entry (n, kappa = 32 g + 4 b + r) = 2^(7 - b) where output
  // bit n takes bit b of input byte 4 g + r; core matrix (kappa / 16, n / 8) at
  // ((kappa / 16) * (npad / 8) + n / 8) * 128, row n % 8, byte kappa % 16
  for (uint32_t i = threadIdx.x; i < a.npad * K / 16u; i += blockDim.x) {
    const uint32_t core = i >> 3, row = i & 7u;
    const uint32_t kc = core / (a.npad / 8u), n = (core % (a.npad / 8u)) * 8u + row;
    uint32_t w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      uint32_t v = 0;
#pragma unroll
      for (int x = 0; x < 4; ++x) {
        const uint32_t kappa = kc * 16u + q * 4u + x;
        const uint32_t g = kappa >> 5, b = (kappa >> 2) & 7u, r = kappa & 3u;
        const uint32_t bit = (n < kMaxOutBits && g < kMaxInBits / 32u) ? (a.bits[n][g] >> (8u * r + b)) & 1u : 0u;
        v |= (bit << (7u - b)) << (8 * x);
      }
      w[q] = v;
    }
    *reinterpret_cast<uint4*>(bimg + static_cast<size_t>(i) * 16u) = make_uint4(w[0], w[1], w[2], w[3]);
  }
  if (threadIdx.x == 0) {
    for (int s = 0; s < kStages; ++s) {
      mbar_init(&S.full[s], 1);
      mbar_init(&S.empty[s], kExpandWarps);
    }
    for (uint32_t s = 0; s < kSlots; ++s) {
      mbar_init(&S.afull[s], kExpandWarps);
      mbar_init(&S.aempty[s], 1);
    }
    for (uint32_t d = 0; d < kDBufs; ++d) {
      mbar_init(&S.dfull[d], 1);
      mbar_init(&S.dempty[d], kWorkerWarps - kExpandWarps);
    }
    S.abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  // generic-proxy writes of the B image become visible to the tensor cores
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
  const uint32_t tbase = S.tmem_base;
  const uint32_t a_base = tbase;                        // kSlots slots x 32 columns
  const uint32_t d_base = tbase + kSlots * kSlotCols;   // kDBufs buffers x 128 columns

  // blocks of this CTA: blockIdx.x, + gridDim.x, ...
  const uint64_t nmine = a.nblk > blockIdx.x ? (a.nblk - blockIdx.x + gridDim.x - 1) / gridDim.x : 0;
  const uint64_t ntiles = nmine * 4u;

  if (warp == kProducerWarp) {
    // ---- producer: lane 0 arms the stage's barrier, every lane issues copies
    const uint32_t row_bytes = kCols * E;
    StripeCursor cur;
    uint64_t issued = 0;
    for (uint64_t i = 0; i < nmine; ++i) {
      const uint32_t s = static_cast<uint32_t>(i % kStages);
      int go = 1;
      if (lane == 0) {
        go = !*abort;
        if (go && i >= kStages && !mbar_wait(&S.empty[s], static_cast<uint32_t>((i / kStages - 1) & 1u), abort)) {
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
      for (uint64_t i = issued > kStages ? issued - kStages : 0; i < issued; ++i)
        mbar_wait(&S.full[i % kStages], static_cast<uint32_t>((i / kStages) & 1u), abort, false);
  } else if (warp == kIssuerWarp) {
    // ---- issuer: one thread issues every product, slot by slot
    if (lane == 0) {
      const uint32_t idesc = (2u << 4) | ((a.npad >> 3) << 17) | ((128u >> 4) << 24);  // s32 += u8 * u8, M = 128
      const uint32_t bsm = smem_u32(bimg);
      const uint32_t lbo = a.npad * 16u, sbo = 128u;
      const uint32_t nq = (a.ngroups + 3u) / 4u;
      uint64_t t = 0, qi = 0;
      bool ok = true;
      for (; t < ntiles && ok; ++t) {
        const uint32_t d = static_cast<uint32_t>(t % kDBufs);
        if (t >= kDBufs && !mbar_wait(&S.dempty[d], static_cast<uint32_t>((t / kDBufs - 1) & 1u), abort)) {
          ok = false;
          break;
        }
        for (uint32_t j = 0; j < nq; ++j, ++qi) {
          const uint32_t slot = static_cast<uint32_t>(qi % kSlots);
          if (!mbar_wait(&S.afull[slot], static_cast<uint32_t>((qi / kSlots) & 1u), abort)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t gend = min(a.ngroups, 4u * j + 4u);
          for (uint32_t g = 4u * j; g < gend; ++g)
            mma_i8(d_base + 128u * d, a_base + kSlotCols * slot + 8u * (g - 4u * j),
                   smem_desc(bsm + g * 2u * a.npad * 16u, lbo, sbo), idesc, g > 0);
          mma_commit(&S.aempty[slot]);  // this slot may be refilled once its products are done
        }
        if (!ok) break;
        mma_commit(&S.dfull[d]);
      }
      if (!ok) {
        atomicExch(&g_gf2_err, 2);
        *abort = 1;
      }
      // the last products must finish before TMEM is freed
      for (uint64_t u = t > kDBufs ? t - kDBufs : 0; u < t; ++u)
        mbar_wait(&S.dfull[u % kDBufs], static_cast<uint32_t>((u / kDBufs) & 1u), abort, false);
    }
  } else if (warp < kExpandWarps) {
    expander_loop<E>(a, S, stages, stage_bytes, nmine, a_base, abort);
  } else {
    epilogue_loop<E>(a, S, ntiles, d_base, abort);
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  if (warp == kIssuerWarp)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tbase), "r"(kTmemCols) : "memory");
}

}  // namespace

bool gf2mma_shape_ok(int field, size_t k, size_t m) {
  const int E = field_bytes(field);
  return E > 0 && k >= 1 && m >= 1 && k * E <= kMaxInBits / 8 && m * E <= kMaxOutBits / 8;
}

// Bit matrix of a coefficient matrix (term-major, k x m): bits[n][g] bit
// (8r + b) = output bit n (byte n / 8 of the m*E output bytes, bit n % 8)
// depends on bit b of input byte 4g + r (input byte u = t * E + p).
void gf2mma_bits(int field, const uint32_t* coeffs, size_t k, size_t m, uint32_t* bits /* [128][16] */) {
  const int E = field_bytes(field);
  std::memset(bits, 0, kMaxOutBits * (kMaxInBits / 32) * sizeof(uint32_t));
  for (size_t t = 0; t < k; ++t)
    for (size_t j = 0; j < m; ++j) {
      uint8_t M[4][4];
      coeff_byte_matrix(field, coeffs[t * m + j] & field_mask(field), M);
      for (int o = 0; o < E; ++o)
        for (int p = 0; p < E; ++p) {
          if (!M[o][p]) continue;
          const size_t u = t * E + p;
          for (int b = 0; b < 8; ++b) {
            const uint8_t prod = byte_mul(field, M[o][p], static_cast<uint8_t>(1u << b));
            for (int ob = 0; ob < 8; ++ob)
              if ((prod >> ob) & 1u) {
                const size_t n = (j * E + o) * 8 + ob;
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
  a.npad = static_cast<uint32_t>((m * E * 8 + 15) / 16 * 16);
  a.overwrite = overwrite ? 1u : 0u;
  std::memcpy(a.bits, bits, sizeof a.bits);
  const uint32_t K = a.ngroups * 32u;
  const uint32_t b_bytes = (a.npad * K + 1023u) & ~1023u;
  const uint32_t stage_bytes = (a.k * kCols * E + 127u) & ~127u;
  const int smem = static_cast<int>(b_bytes + kStages * stage_bytes + sizeof(Smem));
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
