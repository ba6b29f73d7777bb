// internal.hpp -- shared declarations between the C ABI layer (api.cpp) and
// the device code (kernels.cu) of libfgfcuda.so.
#pragma once
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <vector>

#include "../../include/fgf_cuda.h"
#include "gf_host.hpp"

namespace fgfc {

// Limits of one kernel launch. Calls with more sources or rows are split
// into several launches by the host (exact: rows are independent, and
// sources split into an overwrite launch followed by accumulate launches).
constexpr int kMaxSrc = 64;
constexpr int kMaxRows = 64;
// One nibble table slot: 16 rows x 256 bytes. Each row holds 32 lane copies
// of the lo-nibble word (bytes 0..127) and of the hi-nibble word (128..255),
// so a warp's 32 lookups hit 32 distinct banks.
constexpr int kSlotBytes = 4096;
constexpr int kMaxSlots = 54;            // 216 KiB of tables (+ 6.75 KiB staging) per CTA
constexpr int kInlineSlots = 48;         // tables carried in launch parameters
constexpr int kCompactWords = 32;        // 16 lo + 16 hi words per slot

// A compact table slot for (source t, source byte-plane p, row group g):
// word[n] (n < 16) = products of the lo nibble value n, word[16 + n] =
// products of (n << 4); byte q of each word is output byte (q % E) of row
// (g * R + q / E), R = 4 / E rows per group.

struct MatrixLaunch {
  uint64_t len;            // bytes per row processed by this launch
  uint64_t head;           // bytes handled by the scalar path before the vector body
  uint64_t nvec;           // 16-byte vectors in the body
  uint32_t k;              // sources
  uint32_t nrows;          // rows written by this launch (<= groups * R)
  uint32_t gstride;        // groups per (source, plane) in the compact table array
  uint32_t g0;             // first group of this launch within that array
  uint32_t shift;          // 1: some row is not at the sources' offset within 16 bytes
  const uint32_t* tables;  // device compact tables, or nullptr for `inline_tab`
  const uint8_t* src[kMaxSrc];
  uint8_t* dst[kMaxRows];
  uint32_t inline_tab[kInlineSlots * kCompactWords];
};

// Build compact tables for sources [t0, t0+k) and groups [g0, g0+G) of a
// coefficient matrix (term-major: coeffs[t * m + j]). Output layout
// [(t * E + p) * G + g][32].
void build_compact_tables(int field, const uint64_t* coeffs, size_t m, size_t t0, size_t k,
                          size_t g0, size_t G, uint32_t* out);

// The 8-byte fields multiply a constant c = c0 + c1 w by x = x0 + x1 w
// (halves over the 4-byte base field: Gf32 for GF(2^64), FP32 for Fan-Paar
// GF(2^64)) as three half-products A = c0 x0, B = c1 x1, C = (c0 + c1)(x0 + x1)
// and a fix-up of the sums (Karatsuba): GF(2^64) gives lo = A + beta B,
// hi = A + C; Fan-Paar gives lo = A + B, hi = A + C + (1 + alpha) B. Tables
// for sources [t0, t0+k) and rows [j0, j0+M), layout
// [((t * 3 + P) * 4 + p) * M + j][32]: product P (A, B, C), input byte p of
// the 4-byte half, 16 words for its low nibble and 16 for its high nibble.
constexpr size_t kWideSlotsPerSrcRow = 12;
// The same split for Gf16 = Gf8B[u]/(u^2 + u + 0x20): lo = A + 0x20 B,
// hi = A + C over byte half-products. Tables for the batched work lists:
// [(t * 3 + P) * Gq + q][32], nibble tables whose word holds the byte
// half-product P of rows 4q .. 4q + 3 (zero past m); Gq = ceil(m / 4).
void build_kara16_tables(const uint64_t* coeffs, size_t m, size_t k, size_t Gq, uint32_t* out);
void build_wide_tables(int field, const uint64_t* coeffs, size_t m, size_t t0, size_t k, size_t j0, size_t M,
                       uint32_t* out);
// The fix-up map of an 8-byte field as [4 input bytes][32] nibble tables:
// v -> beta v (GF(2^64)) or v -> (1 + alpha) v (Fan-Paar GF(2^64)).
void build_wide_fixup(int field, uint32_t* out /* [128] */);

// Kernel entry (kernels.cu). `groups` = G for this launch; `overwrite`
// selects dot-product (overwrite) or mul_add (accumulate) semantics.
// `byte_tables`: run the byte-table kernel (Gf8, one group, <= 14 sources)
// for the vector body instead of the split-nibble kernel.
cudaError_t launch_matrix(int field, int groups, bool overwrite, const MatrixLaunch& a,
                          cudaStream_t s, bool byte_tables);
// Fill `n` rows of `len` bytes with zero.
cudaError_t launch_zero_rows(uint8_t* const* rows, int n, uint64_t len, cudaStream_t s);
// dst ^= src over `len` bytes.
cudaError_t launch_xor(uint8_t* dst, const uint8_t* src, uint64_t len, cudaStream_t s);
// Elementwise product dst[i] = a[i] * b[i].
cudaError_t launch_elementwise(int field, uint8_t* dst, const uint8_t* a, const uint8_t* b,
                               uint64_t len, cudaStream_t s);

int sm_count();

// Kernel families (fgfc_kernel values) and the choice per shape (tune.cpp).
constexpr size_t kFastMaxSources = 14;  // byte-table kernels: sources per launch
bool kernel_usable(int kernel, int field, size_t k, size_t m);
int choose_kernel(int field, size_t k, size_t m, size_t len);
// Tile shape of the batched nibble work lists (tune.cpp): element-vector
// columns per thread per work item for the class of element width E and G
// table groups; set_tile_cols(E, G, 0) restores the built-in value.
constexpr int kTileColsDefault = 8;
int tile_cols(int E, int G);
void set_tile_cols(int E, int G, int cols, double us);
// Shapes the bit-sliced tensor-core contraction covers in one launch
// (gf2mma.cu): at most 512 input bits and 128 output bits per element column.
bool gf2mma_shape_ok(int field, size_t k, size_t m);
// Compact GF(2) bit matrix of a term-major k x m coefficient matrix:
// kGf2BitWords words, [output bit][input word group].
constexpr size_t kGf2BitWords = 128 * 16;
void gf2mma_bits(int field, const uint64_t* coeffs, size_t k, size_t m, uint32_t* bits);
// Columns [0, nblk * 512 * E) of k sources and m rows, all 16-byte aligned.
cudaError_t gf2mma_launch(int field, const uint8_t* const* srcs, size_t k, uint8_t* const* rows, size_t m,
                          const uint32_t* bits, uint64_t nblk, bool overwrite, cudaStream_t stream);
// Several stripes of one plan in one launch: ptrs (device) holds k source and
// m row pointers per stripe, prefix (device) the first block of each stripe.
cudaError_t gf2mma_launch_multi(int field, size_t k, size_t m, const uint32_t* bits, const uint64_t* ptrs,
                                const uint64_t* prefix, uint32_t nstripes, uint64_t nblk, bool overwrite,
                                cudaStream_t stream);
// Opt the tensor-core kernel of element width E in to its shared memory on
// the current device (done before a graph capture records a launch).
cudaError_t gf2mma_prepare(int E);
// Error word of the current device's tensor-core kernels (0 = fine);
// synchronises with the device.
int gf2mma_error(bool clear);
// Opt `fn` in to `bytes` of dynamic shared memory on the current device, once
// per (device, kernel); thread-safe.
cudaError_t ensure_smem_attr(const void* fn, int bytes);

// One lowered sub-job of a batched submission: all sources of a stripe and
// the rows of at most 4 table groups, with its alignment split resolved.
struct LoweredJob {
  int field;
  const uint32_t* tables;  // plan compact tables, matrix orientation
  size_t gstride;          // plan groups per (source, plane)
  size_t g0;               // first group of this sub-job
  size_t G;                // groups in this sub-job (1..4)
  uint64_t len, head, nvec;
  size_t k, nrows;
  bool ovr;
  bool shift;              // some row is not at the sources' offset within 16 bytes
  bool kara = false;       // Gf16 by byte half-products (tables: build_kara16_tables; G = row quads)
  std::vector<uint64_t> srcs, dsts;
};

// One stripe's 16-byte-aligned body for the tensor-core kernel in a batch:
// its k sources and m rows already offset to the body start, nblk blocks of
// 512 element columns.
struct Gf2Job {
  int field;
  const uint32_t* bits;  // the plan's GF(2) bit matrix (host copy)
  uint64_t bits_key;     // hash of the bit matrix: stripes with equal keys share a launch
  size_t k, m;
  bool ovr;
  uint64_t nblk;
  std::vector<uint64_t> ptrs;  // k sources, then m rows
};

void* batch_state_create();
void batch_state_destroy(void* state);
void batch_state_graphs(void* state, bool on);
// The nibble work-list classes (element width, table groups) of the state's
// last submission.
std::vector<std::pair<int, int>> batch_state_classes(const void* state);
void batch_state_stats(const void* state, size_t* launches, size_t* items, int* replayed);
cudaError_t batch_run(void* state, const std::vector<LoweredJob>& jobs, const std::vector<Gf2Job>& tc,
                      cudaStream_t stream);
// One stripe of a plan (api.cpp) as sub-jobs for batch_run: the tensor-core
// body (when the tuner picks that kernel for the shape and every pointer
// shares one offset within 16 bytes) plus table sub-jobs for the rest.
void lower_matrix_job(const fgfc_plan* plan, const std::vector<uint64_t>& srcs, const std::vector<uint64_t>& dsts,
                      size_t row_len, bool overwrite, std::vector<LoweredJob>& out, std::vector<Gf2Job>& tc);

// The matrix ops for 8-byte fields (wide.cu): coefficients either as raw
// host values (term-major k x m, tables built into the launch parameters) or
// as a plan's device tables in the compact layout with `gstride` groups per
// (source, byte plane).
// Matrix ops of the 8-byte fields (wide.cu): dev_tables in the
// build_wide_tables layout with `gstride` rows, or nullptr (tables built
// per launch from host_coeffs).
cudaError_t wide_launch(int field, const uint8_t* const* srcs, size_t k, uint8_t* const* rows, size_t m,
                        const uint64_t* host_coeffs, const uint32_t* dev_tables, size_t gstride, size_t len,
                        bool overwrite, cudaStream_t stream);

// Error text of the calling thread (api.cpp), for entry points defined in
// other files.
fgfc_status set_error(fgfc_status st, const char* msg);
fgfc_status clear_error();
const char* last_error_text();
fgfc_status validate_matrix_call(int field, const char* name, size_t dst_len, size_t row_len,
                                 const size_t* row_starts, size_t nrows, const fgfc_slice* srcs, size_t nsrcs,
                                 const uint32_t* coeffs, int overwrite);

// Decode rows of the code [I_k ; parity] for a survivor set and erased shards,
// term-major k x nerased (decode.cpp).
fgfc_status decode_matrix(int field, const uint32_t* parity, size_t k, size_t m, const size_t* survivors,
                          const size_t* erased, size_t nerased, uint32_t* out);

// fgfc_batch_run_noalloc's work (batch.cu): jobs already validated against
// the ops' rules; returns 0 or an fgfc_status with `msg` set.
int noalloc_run(int field, const fgfc_noalloc_job* jobs, size_t njobs, cudaStream_t stream, char* msg,
                size_t msglen);

}  // namespace fgfc
