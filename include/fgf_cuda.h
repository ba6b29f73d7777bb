/*
 * fgf_cuda.h -- C ABI of libfgfcuda.so, the sm_100a implementation of the
 * packed-vector `ops` AXPY family of the fgf crate (nanithefkuc/fgf 0.4.0).
 *
 * Every entry point here mirrors one public function of `fgf::ops`
 * (src/ops.rs) with the same name, argument order and argument meaning, but
 * over DEVICE buffers and stream-ordered: the call validates on the host
 * exactly what the reference validates, then enqueues the kernels on
 * `stream` and returns. Buffers are packed little-endian elements, as in the
 * reference (src/ops.rs:1-39). Rust slices become (pointer, byte length)
 * pairs; `&[(&[F::Elem], &[u8])]` terms become `fgfc_term` arrays; field
 * elements travel as uint32_t values (the low 8/16/32 bits are used).
 *
 * Errors: the reference panics with an operation-named message
 * (src/ops.rs:300-316 and each op's asserts). Here the same condition returns
 * a nonzero `fgfc_status` and `fgfc_last_error()` returns the reference's
 * message text for this thread. Nothing unwinds across the ABI.
 *
 * Aliasing: as in the reference (src/ops.rs:37-39) destinations must not
 * alias sources; the scattered op checks its rows for overlap on the host
 * (src/ops.rs:909-921).
 *
 * Allocation: entry points allocate no device memory per call. Plans own the
 * device copy of their coefficients and prepared tables (allocated once in
 * fgfc_plan_create); raw-coefficient calls carry their coefficients in the
 * kernel launch parameters.
 */
#ifndef FGF_CUDA_H
#define FGF_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Opaque CUDA stream handle (a cudaStream_t); NULL is the legacy default stream. */
typedef struct CUstream_st *fgfc_stream;

/* The fields of the hot path: src/field/gf8b.rs:57, src/field/gf8d.rs:40,
 * src/field/gf16.rs:54-60, src/field/gf32.rs:36-42. */
typedef enum fgfc_field {
  FGFC_GF8B = 0, /* GF(2^8) mod 0x11B, 1 byte */
  FGFC_GF8D = 1, /* GF(2^8) mod 0x11D, 1 byte */
  FGFC_GF16 = 2, /* (GF(2^8)/0x11B)[u]/(u^2+u+0x20), 2 bytes LE */
  FGFC_GF32 = 3, /* GF(2^16)[v]/(v^2+v+0x2000), 4 bytes LE */
  /* The canonical Fan-Paar binary tower (src/field/fan_paar.rs:1-150): the
     2h-bit level is h-bit[X]/(X^2 + alpha X + 1), alpha the h-bit level's
     top generator; elements lo + hi*X, little-endian. */
  FGFC_FP8 = 4,  /* Fan-Paar GF(2^8), 1 byte  (fan_paar::fp8, FanPaar8) */
  FGFC_FP16 = 5, /* Fan-Paar GF(2^16), 2 bytes (fan_paar::fp16, FanPaar16) */
  FGFC_FP32 = 6, /* Fan-Paar GF(2^32), 4 bytes (fan_paar::fp32, FanPaar32) */
  /* 8-byte fields. Their coefficients are 64-bit: make plans with
     fgfc_plan_create_u64 / fgfc_coeff_create_u64 and use the _with entry
     points; a raw entry point's uint32_t coefficient is the element whose
     high 32 bits are zero. */
  FGFC_GF64 = 7, /* GF(2^32)[w]/(w^2+w+0x20000000), 8 bytes LE (src/field/gf64.rs:1-11) */
  FGFC_FP64 = 8  /* Fan-Paar GF(2^64), 8 bytes (fan_paar::fp64, FanPaar64) */
} fgfc_field;

typedef enum fgfc_status {
  FGFC_OK = 0,
  FGFC_ERR_WIDTH = 1,       /* "not a whole number of <F> elements"      ops.rs:301-307 */
  FGFC_ERR_LENGTH = 2,      /* paired buffers differ in length            ops.rs:310-316 */
  FGFC_ERR_ROWS = 3,        /* "rows is N bytes but ... need M"           ops.rs:472-477 */
  FGFC_ERR_COEFFS = 4,      /* coefficient count does not match           ops.rs:535-541,690-696 */
  FGFC_ERR_SOURCE = 5,      /* a source has the wrong length              ops.rs:542-550 */
  FGFC_ERR_PLAN_DIMS = 6,   /* "plan dimensions do not match"             ops.rs:736-740 */
  FGFC_ERR_OVERLAP = 7,     /* scattered rows overlap                     ops.rs:913-921 */
  FGFC_ERR_BOUNDS = 8,      /* scattered row past the end of dst          ops.rs:898-902 */
  FGFC_ERR_ALIGN = 9,       /* scattered row offset not element-aligned   ops.rs:903-907 */
  FGFC_ERR_OVERFLOW = 10,   /* geometry overflows                         ops.rs:468-471 */
  FGFC_ERR_ARG = 11,        /* NULL pointer / unknown field / bad handle */
  FGFC_ERR_LIMIT = 12,      /* beyond a device limit (see fgfc_limits) */
  FGFC_ERR_CUDA = 13,       /* a CUDA runtime call failed */
  FGFC_ERR_NOMEM = 14       /* plan allocation failed */
} fgfc_status;

/* One `(coeffs, src)` term of the many-to-many ops (ops.rs:675-680). */
typedef struct fgfc_term {
  const uint32_t *coeffs; /* host array of `ncoeffs` field elements */
  size_t ncoeffs;
  const uint8_t *src;     /* device pointer */
  size_t src_len;         /* bytes */
} fgfc_term;

/* A device source slice `&[u8]` for the `_with` forms. */
typedef struct fgfc_slice {
  const uint8_t *ptr; /* device pointer */
  size_t len;         /* bytes */
} fgfc_slice;

/* A prepared coefficient vector or row-major matrix: `ops::Plan<F>`
 * (ops.rs:158-276). `ops::Coeff<F>` (ops.rs:44-73) is a 1x1 plan. */
typedef struct fgfc_plan fgfc_plan;

/* Thread-local text of the last error, formatted like the reference's panic
 * message (e.g. "mul_add: dst is 8 bytes but src is 4 bytes"). */
const char *fgfc_last_error(void);
const char *fgfc_version(void);

/* Device limits of this build: maximum sources and rows per call. */
void fgfc_limits(size_t *max_sources, size_t *max_rows);

/* Element width in bytes (F::BYTES), or 0 for an unknown field. */
size_t fgfc_field_bytes(fgfc_field field);

/* ---------------------------------------------------------------- plans */

/* Plan::matrix(rows, cols, coeffs) (ops.rs:198-212); Plan::new(coeffs) is
 * rows = 1 (ops.rs:176-190). Coefficients are copied and prepared (device
 * tables built and uploaded) once, here. */
fgfc_status fgfc_plan_create(fgfc_field field, size_t rows, size_t cols, const uint32_t *coeffs,
                             fgfc_plan **out);
/* Coeff::new(coeff) (ops.rs:61-65): a 1x1 plan. */
fgfc_status fgfc_coeff_create(fgfc_field field, uint32_t coeff, fgfc_plan **out);
/* The same with 64-bit coefficients, for every field (the 8-byte fields need
 * them; values are reduced to the field's width as above). */
fgfc_status fgfc_plan_create_u64(fgfc_field field, size_t rows, size_t cols, const uint64_t *coeffs,
                                 fgfc_plan **out);
fgfc_status fgfc_coeff_create_u64(fgfc_field field, uint64_t coeff, fgfc_plan **out);
void fgfc_plan_destroy(fgfc_plan *plan);
/* Plan::dimensions (ops.rs:231-233), Plan::len (ops.rs:217-219). */
fgfc_status fgfc_plan_dimensions(const fgfc_plan *plan, size_t *rows, size_t *cols);
size_t fgfc_plan_len(const fgfc_plan *plan);
fgfc_field fgfc_plan_field(const fgfc_plan *plan);
/* Plan::values (ops.rs:273-275): copies plan_len values into `out`. */
fgfc_status fgfc_plan_values(const fgfc_plan *plan, uint32_t *out);
/* Plan::get_at(row, col).value() (ops.rs:247-251); ERR_ARG when out of bounds. */
fgfc_status fgfc_plan_get_at(const fgfc_plan *plan, size_t row, size_t col, uint32_t *out);
/* Plan::values / Plan::get_at with 64-bit values (the 32-bit forms return
 * the low halves of an 8-byte field's coefficients). */
fgfc_status fgfc_plan_values_u64(const fgfc_plan *plan, uint64_t *out);
fgfc_status fgfc_plan_get_at_u64(const fgfc_plan *plan, size_t row, size_t col, uint64_t *out);

/* ---------------------------------------------------------------- single row */

/* add_assign / sub_assign: dst ^= src (ops.rs:323-335). */
fgfc_status fgfc_add_assign(fgfc_field field, uint8_t *dst, size_t dst_len, const uint8_t *src,
                            size_t src_len, fgfc_stream stream);
/* mul_add: dst ^= coeff * src (ops.rs:342-352). */
fgfc_status fgfc_mul_add(fgfc_field field, uint8_t *dst, size_t dst_len, uint32_t coeff,
                         const uint8_t *src, size_t src_len, fgfc_stream stream);
/* mul_add_with (ops.rs:359-374); `coeff` is a Coeff or any 1-entry plan. */
fgfc_status fgfc_mul_add_with(uint8_t *dst, size_t dst_len, const fgfc_plan *coeff,
                              const uint8_t *src, size_t src_len, fgfc_stream stream);
/* mul_into: dst = coeff * src (ops.rs:381-392) and its prepared form (ops.rs:399-415). */
fgfc_status fgfc_mul_into(fgfc_field field, uint8_t *dst, size_t dst_len, uint32_t coeff,
                          const uint8_t *src, size_t src_len, fgfc_stream stream);
fgfc_status fgfc_mul_into_with(uint8_t *dst, size_t dst_len, const fgfc_plan *coeff,
                               const uint8_t *src, size_t src_len, fgfc_stream stream);
/* mul_assign: dst *= coeff (ops.rs:422-432) and its prepared form (ops.rs:439-450). */
fgfc_status fgfc_mul_assign(fgfc_field field, uint8_t *dst, size_t dst_len, uint32_t coeff,
                            fgfc_stream stream);
fgfc_status fgfc_mul_assign_with(uint8_t *dst, size_t dst_len, const fgfc_plan *coeff,
                                 fgfc_stream stream);
/* mul_elementwise: dst[i] = a[i] * b[i] (ops.rs:953-957). */
fgfc_status fgfc_mul_elementwise(fgfc_field field, uint8_t *dst, size_t dst_len, const uint8_t *a,
                                 size_t a_len, const uint8_t *b, size_t b_len, fgfc_stream stream);

/* ---------------------------------------------------------------- one-to-many / many-to-one */

/* mul_add_scatter: rows[j] ^= coeffs[j] * src (ops.rs:461-482). */
fgfc_status fgfc_mul_add_scatter(fgfc_field field, uint8_t *rows, size_t rows_len, size_t row_len,
                                 const uint32_t *coeffs, size_t ncoeffs, const uint8_t *src,
                                 size_t src_len, fgfc_stream stream);
/* mul_add_scatter_with (ops.rs:493-520). */
fgfc_status fgfc_mul_add_scatter_with(uint8_t *rows, size_t rows_len, size_t row_len,
                                      const fgfc_plan *plan, const uint8_t *src, size_t src_len,
                                      fgfc_stream stream);
/* mul_add_gather: dst ^= sum coeffs[i] * srcs[i] (ops.rs:533-555). */
fgfc_status fgfc_mul_add_gather(fgfc_field field, uint8_t *dst, size_t dst_len,
                                const uint32_t *coeffs, size_t ncoeffs, const fgfc_slice *srcs,
                                size_t nsrcs, fgfc_stream stream);
/* mul_add_gather_with (ops.rs:563-585). */
fgfc_status fgfc_mul_add_gather_with(uint8_t *dst, size_t dst_len, const fgfc_plan *plan,
                                     const fgfc_slice *srcs, size_t nsrcs, fgfc_stream stream);
/* dot_product: dst = sum coeffs[i] * srcs[i] (ops.rs:597-624). */
fgfc_status fgfc_dot_product(fgfc_field field, uint8_t *dst, size_t dst_len,
                             const uint32_t *coeffs, size_t ncoeffs, const fgfc_slice *srcs,
                             size_t nsrcs, fgfc_stream stream);
/* dot_product_with (ops.rs:632-660). */
fgfc_status fgfc_dot_product_with(uint8_t *dst, size_t dst_len, const fgfc_plan *plan,
                                  const fgfc_slice *srcs, size_t nsrcs, fgfc_stream stream);

/* ---------------------------------------------------------------- many-to-many */

/* mul_add_matrix: rows[j] ^= sum_t terms[t].coeffs[j] * terms[t].src (ops.rs:675-708). */
fgfc_status fgfc_mul_add_matrix(fgfc_field field, uint8_t *rows, size_t rows_len, size_t row_len,
                                size_t nrows, const fgfc_term *terms, size_t nterms,
                                fgfc_stream stream);
/* mul_add_matrix_with: plan dimensions (nsrcs, nrows) (ops.rs:720-760). */
fgfc_status fgfc_mul_add_matrix_with(uint8_t *rows, size_t rows_len, size_t row_len, size_t nrows,
                                     const fgfc_plan *plan, const fgfc_slice *srcs, size_t nsrcs,
                                     fgfc_stream stream);
/* dot_product_matrix: overwrite form (ops.rs:773-810). */
fgfc_status fgfc_dot_product_matrix(fgfc_field field, uint8_t *rows, size_t rows_len,
                                    size_t row_len, size_t nrows, const fgfc_term *terms,
                                    size_t nterms, fgfc_stream stream);
/* dot_product_matrix_with (ops.rs:823-867): the RS encode entry point. */
fgfc_status fgfc_dot_product_matrix_with(uint8_t *rows, size_t rows_len, size_t row_len,
                                         size_t nrows, const fgfc_plan *plan,
                                         const fgfc_slice *srcs, size_t nsrcs,
                                         fgfc_stream stream);
/* mul_add_matrix_scattered: row j at dst + row_starts[j] (ops.rs:887-941). */
fgfc_status fgfc_mul_add_matrix_scattered(fgfc_field field, uint8_t *dst, size_t dst_len,
                                          size_t row_len, const size_t *row_starts,
                                          size_t nrows, const fgfc_term *terms, size_t nterms,
                                          fgfc_stream stream);
/* Extension with no reference counterpart (the reference has no prepared
 * form of the scattered op, README.md:113): the same op driven by a plan of
 * dimensions (nsrcs, nrows), as the reconstruct path uses a cached decode plan. */
fgfc_status fgfc_mul_add_matrix_scattered_with(uint8_t *dst, size_t dst_len, size_t row_len,
                                               const size_t *row_starts, size_t nrows,
                                               const fgfc_plan *plan, const fgfc_slice *srcs,
                                               size_t nsrcs, fgfc_stream stream);
/* Extension with no reference counterpart: the overwrite form of the
 * scattered op, rows[j] at dst + row_starts[j] = sum_t plan(t, j) * srcs[t].
 * It gives exactly what zeroing the rows and then calling
 * mul_add_matrix_scattered(_with) gives (the recipe a caller of the reference
 * uses to rebuild erased shards in place), in one pass that never reads the
 * rows' prior contents. Same validation as the accumulate form. */
fgfc_status fgfc_dot_product_matrix_scattered_with(uint8_t *dst, size_t dst_len, size_t row_len,
                                                   const size_t *row_starts, size_t nrows,
                                                   const fgfc_plan *plan, const fgfc_slice *srcs,
                                                   size_t nsrcs, fgfc_stream stream);

/* ---------------------------------------------------------------- coding and decode matrices */

/* No counterpart in the crate, which leaves coding-matrix construction to its
 * callers (src/lib.rs:115-116); the recipes of its round-trip test
 * (tests/ops.rs:897-950) with its inv(0) = 0 convention (src/field/mod.rs:38-41).
 * Host computation; no device work. */

/* Cauchy parity matrix, row-major m x k: out[i * k + j] = inv(x_i + y_j),
 * x_i = x0 + i, y_j = j. FGFC_ERR_ARG if some x_i + y_j is zero or a value
 * does not fit the field. */
fgfc_status fgfc_cauchy_matrix(fgfc_field field, size_t m, size_t k, uint32_t x0, uint32_t *out);
/* Decode rows of the systematic code [I_k ; C] (`parity` = C, row-major
 * m x k): with k distinct surviving shard indices (0..k-1 data, k..k+m-1
 * parity) and `nerased` shard indices to rebuild, out (k x nerased,
 * term-major: out[t * nerased + e]) satisfies
 * shard[erased[e]] = sum_t out[t * nerased + e] * shard[survivors[t]], the
 * layout Plan::matrix(k, nerased) takes. The survivor submatrix is inverted
 * by Gauss-Jordan elimination over the field; FGFC_ERR_ARG if it is
 * singular or an index is out of range or repeated. */
fgfc_status fgfc_decode_matrix(fgfc_field field, const uint32_t *parity, size_t k, size_t m,
                               const size_t *survivors, const size_t *erased, size_t nerased,
                               uint32_t *out);
/* The same decode rows as a prepared plan of dimensions (k, nerased), ready
 * for mul_add_matrix_scattered_with / dot_product_matrix_scattered_with. */
fgfc_status fgfc_decode_plan_create(fgfc_field field, const uint32_t *parity, size_t k, size_t m,
                                    const size_t *survivors, const size_t *erased, size_t nerased,
                                    fgfc_plan **out);

/* ---------------------------------------------------------------- batches */

/* One stripe of a batched submission: the arguments of one
 * dot_product_matrix_with (overwrite = 1, row_starts = NULL),
 * mul_add_matrix_with (overwrite = 0, row_starts = NULL),
 * mul_add_matrix_scattered_with (overwrite = 0, row_starts set) or
 * dot_product_matrix_scattered_with (overwrite = 1, row_starts set) call
 * (src/ops.rs:720-867, 887-941). Each job is validated exactly as that call
 * would be. */
typedef struct fgfc_matrix_job {
  const fgfc_plan *plan;    /* dimensions (nsrcs, nrows) */
  const fgfc_slice *srcs;   /* host array of nsrcs device slices */
  size_t nsrcs;
  uint8_t *dst;             /* device destination base */
  size_t dst_len;
  const size_t *row_starts; /* host array of nrows offsets into dst, or NULL for rows j * row_len */
  size_t nrows;
  size_t row_len;
  int overwrite;
} fgfc_matrix_job;

/* A reusable batch runner. No reference counterpart: the reference is a
 * single-threaded CPU library that serves one call at a time. The runner
 * owns its device work-list and pinned staging (grown on demand, reused
 * afterwards) and lowers every submission to one persistent launch per
 * (element width, row-group) class. */
typedef struct fgfc_batch fgfc_batch;

fgfc_status fgfc_batch_create(fgfc_batch **out);
void fgfc_batch_destroy(fgfc_batch *batch);
/* Replay submissions whose launch structure repeats as a captured CUDA graph
 * (default on). */
fgfc_status fgfc_batch_set_graphs(fgfc_batch *batch, int enable);
/* Enqueue all jobs on `stream`. Jobs must not write memory another job of the
 * same submission reads or writes. */
fgfc_status fgfc_batch_run(fgfc_batch *batch, const fgfc_matrix_job *jobs, size_t njobs,
                           fgfc_stream stream);
/* Statistics of the last submission: kernel launches issued, work items,
 * whether it replayed a graph. */
fgfc_status fgfc_batch_stats(const fgfc_batch *batch, size_t *launches, size_t *items,
                             int *graph_replayed);
/* The same jobs as fgfc_batch_run, each issued as its own call of the
 * per-call entry point it stands for (dot_product_matrix_with,
 * mul_add_matrix_with or mul_add_matrix_scattered_with), in order, from a
 * native loop: the one-call-per-stripe way a caller of the reference's ops
 * would do it, kept for comparison with the batched launch. Stops at the
 * first failing job and returns its status. */
fgfc_status fgfc_run_jobs_serial(const fgfc_matrix_job *jobs, size_t njobs, fgfc_stream stream);

/* ---------------------------------------------------------------- without allocation */

/* One stripe for fgfc_batch_run_noalloc: like fgfc_matrix_job, but with the
 * raw coefficient matrix instead of a plan (nsrcs x nrows, term-major: the
 * order of Plan::matrix(nsrcs, nrows, ..)). */
typedef struct fgfc_noalloc_job {
  const uint32_t *coeffs;   /* host, nsrcs * nrows: coeffs[t * nrows + j] multiplies source t into row j */
  const fgfc_slice *srcs;   /* host array of nsrcs device slices */
  size_t nsrcs;
  uint8_t *dst;             /* device destination base */
  size_t dst_len;
  const size_t *row_starts; /* host array of nrows offsets into dst, or NULL for rows j * row_len */
  size_t nrows;
  size_t row_len;
  int overwrite;            /* 1 = dot product (overwrite), 0 = accumulate */
} fgfc_noalloc_job;

/* No counterpart in the reference (a CPU library, which never allocates
 * device memory at all). The same work as fgfc_batch_run for stripes of one
 * field, but it allocates nothing: not on the device (no cudaMalloc, no
 * plan) and not on the host. It is meant for callers that may not allocate
 * while they run, such as an I/O path that must not take the implicit device
 * synchronisation and unbounded latency of cudaMalloc, or a process whose
 * device memory is fully handed to a pool it does not own.
 *
 * Its scratch (stripe descriptors, pointers, work items, the claim counter
 * and every stripe's product tables) lives in one fixed device array of
 * FGFC_NOALLOC_SCRATCH_BYTES that every GPU loading the library keeps until
 * process exit. A submission needing more returns FGFC_ERR_LIMIT; so does a
 * stripe with more than FGFC_NOALLOC_MAX_ROWS_GF8 rows (Gf8; 8 for Gf16, 4
 * for Gf32) or more than 64 sources.
 *
 * The first call on a device looks up the array's device address (once per
 * device, with that device current); make that first call before any stream
 * capture. A call made while `stream` is being captured returns FGFC_ERR_ARG
 * and enqueues nothing. Every call reuses the same array and leaves its
 * contents behind: calls whose work overlaps on the GPU (different streams,
 * or different threads without ordering) race on it; calls on one stream are
 * ordered. Host threads are serialised by a lock around the call itself.
 *
 * The descriptors are built in a fixed, pageable host array and copied in
 * with one cudaMemcpyAsync, which CUDA stages before returning: the call may
 * block the host until `stream` has reached that copy. Stripes are grouped as
 * in fgfc_batch_run (Gf8 stripes of at most 4 rows and 14 sources on the
 * byte-table kernel, the rest by their number of 4-byte row groups), one
 * launch per group. */
#define FGFC_NOALLOC_SCRATCH_BYTES (8u << 20)
#define FGFC_NOALLOC_MAX_ROWS_GF8 16
fgfc_status fgfc_batch_run_noalloc(fgfc_field field, const fgfc_noalloc_job *jobs, size_t njobs,
                                   fgfc_stream stream);

/* ---------------------------------------------------------------- kernel choice and tuning */

/* No reference counterpart as such: the reference picks its CPU backend once
 * (src/kernel/mod.rs:147-184) and routes each call between blocked and AXPY
 * paths by shape (src/kernel/gf16.rs:419-460). Here a matrix call runs one of
 * three kernel families, chosen per (field, sources, rows, row-length bucket)
 * by, in order: a process-wide override (fgfc_tune_force, or the environment
 * variable FGFC_KERNEL = nibble | byte | gf2mma, read once), the table of
 * measured winners (fgfc_tune_shape; fgfc_tune_save / fgfc_tune_load persist
 * it as JSON), and built-in rules. A family is only ever used for shapes it
 * can run; every family gives the same bytes. */
typedef enum fgfc_kernel {
  FGFC_KERNEL_AUTO = 0,   /* the tuned or built-in choice */
  FGFC_KERNEL_NIBBLE = 1, /* split-nibble product tables in shared memory (every shape) */
  FGFC_KERNEL_BYTE = 2,   /* 256-entry byte tables: Gf8, at most 4 rows and 14 sources */
  FGFC_KERNEL_GF2MMA = 3  /* bit-sliced GF(2) contraction on the tensor cores (tcgen05) */
} fgfc_kernel;

fgfc_status fgfc_tune_force(fgfc_kernel kernel);
/* The family a matrix call of this shape runs now. */
fgfc_kernel fgfc_tune_choice(fgfc_field field, size_t nsrcs, size_t nrows, size_t row_len);
/* 1 if `kernel` can run this shape. */
int fgfc_tune_usable(fgfc_kernel kernel, fgfc_field field, size_t nsrcs, size_t nrows);
/* Times every usable family on a dot_product_matrix_with call of this shape
 * on the current device (allocates and frees its own buffers) and records the
 * fastest for the shape's row-length bucket; the winner goes to *out. */
fgfc_status fgfc_tune_shape(fgfc_field field, size_t nsrcs, size_t nrows, size_t row_len, fgfc_kernel *out);
/* Error word of the current device's tensor-core kernels, whose waits are
 * bounded: FGFC_ERR_CUDA if one gave up (its call's results are then not
 * valid), else FGFC_OK. Synchronises with the device; `clear` resets it. */
fgfc_status fgfc_device_check(int clear);
/* Tile shape of the batched work lists (fgfc_batch_run and the serving
 * loop): the 16-byte element vectors each thread takes per work item, for a
 * split-nibble work-list class (element bytes 1, 2 or 4; table groups 1..4 =
 * rows per 4-byte group times groups). cols is 1, 2, 4, 8 or 16; 0 restores
 * the built-in 8. The environment variable FGFC_TILE_COLS (read once)
 * overrides every class for A/B runs. Tiles change only how work is split,
 * never the bytes produced. */
fgfc_status fgfc_tune_set_tile(size_t elem_bytes, size_t groups, unsigned cols);
unsigned fgfc_tune_tile(size_t elem_bytes, size_t groups);
/* Measures tile shapes on one submission (run on `stream`, repeatedly: its
 * jobs must be safe to run again, e.g. overwrite forms): for each
 * split-nibble class it uses, every tile shape with the other classes fixed,
 * keeping a shape that is at least 2 % faster; *us_before and *us_after
 * receive the submission's device time with the starting and the chosen
 * tiles (either may be NULL). fgfc_tune_save / fgfc_tune_load persist the
 * tiles with the family table. */
fgfc_status fgfc_tune_batch_tiles(fgfc_batch *batch, const fgfc_matrix_job *jobs, size_t njobs, fgfc_stream stream,
                                  double *us_before, double *us_after);
fgfc_status fgfc_tune_save(const char *path);
fgfc_status fgfc_tune_load(const char *path);
/* Forgets measured families and tiles. */
void fgfc_tune_clear(void);

/* ---------------------------------------------------------------- serving loop */

/* A request loop over host or device buffers. No counterpart in the reference (whose
 * callers run one `ops` call per stripe on the CPU); each request is exactly
 * one such call -- dot_product_matrix (overwrite), mul_add_matrix
 * (accumulate) or mul_add_matrix_scattered (row_starts != NULL) -- with the
 * same validation and the same bytes in the destination afterwards.
 *
 * A worker thread per server admits requests in arrival order while device
 * memory (hbm_budget) and staging allow, and issues each admitted group as
 * one launch of the batch work-list kernel; requests that arrive while
 * earlier launches run are admitted into the next one (continuous batching),
 * so host-to-device copies, kernels and device-to-host copies of successive
 * launches overlap on three streams. Coefficient matrices are turned into
 * device plans once and cached, keyed by a hash of (field, dimensions,
 * coefficients). Request buffers in page-locked host memory with rows of at
 * least 256 KiB are copied directly; other host buffers go through the
 * server's page-locked staging buffers, filled and emptied by a small pool of
 * host copy threads. A request whose buffers are all
 * device memory of the server's device runs in place, without copies (a
 * request mixing host and device buffers is rejected with FGFC_ERR_ARG). */
typedef struct fgfc_server fgfc_server;

typedef struct fgfc_server_config {
  size_t hbm_budget;    /* device bytes for admitted requests (0: 64 GiB) */
  size_t staging_bytes; /* page-locked host staging (0: 1 GiB) */
  size_t max_batch;     /* requests per launch (0: 1024) */
  size_t max_inflight;  /* launches issued and not yet retired (0: 4) */
  size_t plan_cache;    /* device plans kept (0: 64); least recently used unreferenced ones go first */
  size_t max_launch_bytes; /* device bytes per launch (0: 256 MiB), so that a burst is split into
                              launches whose copies and kernels overlap; a larger request runs alone */
  int plain;            /* 1: one request at a time through the per-call entry points, synchronously
                           (the one-call-per-stripe comparison); 0: continuous batching */
  int device;           /* CUDA device; -1: the device current at creation */
} fgfc_server_config;

typedef struct fgfc_request {
  fgfc_field field;
  const uint32_t *coeffs;   /* nsrcs * nrows, coeffs[t * nrows + j] multiplies source t into row j */
  const fgfc_slice *srcs;   /* host source shards, row_len bytes each */
  size_t nsrcs;
  uint8_t *dst;             /* host destination */
  size_t dst_len;
  const size_t *row_starts; /* NULL: rows j * row_len; else scattered rows */
  size_t nrows;
  size_t row_len;
  int overwrite;            /* 1: dot_product_matrix (scattered: its overwrite extension); 0: accumulate */
} fgfc_request;

typedef struct fgfc_server_stats {
  uint64_t completed;    /* requests finished (results in host memory) */
  uint64_t failed;
  uint64_t launches;     /* kernel submissions (batches, or calls in plain mode) */
  uint64_t plan_hits, plan_misses;
  uint64_t source_bytes; /* nsrcs * row_len summed over completed requests */
  uint64_t peak_device_bytes;
  uint64_t max_batch_seen;
  double p50_us, p99_us, mean_us, max_us; /* submit -> result in host memory */
  double busy_s;         /* first submit -> last completion since the last reset */
  double queue_us;       /* mean submit -> issue (waiting for admission) */
  double launch_us;      /* mean issue -> retire of a launch (copies, kernels, completion) */
} fgfc_server_stats;

fgfc_status fgfc_server_create(const fgfc_server_config *cfg, fgfc_server **out);
/* Validates and enqueues; coefficient, source-slice and row_starts arrays are
 * copied, the host shards and dst must stay valid and untouched until the
 * request completes. FGFC_ERR_LIMIT if it can never fit the budgets. */
fgfc_status fgfc_server_submit(fgfc_server *server, const fgfc_request *req, uint64_t *ticket);
/* A rebuild by erasure pattern: `srcs` hold the k survivor shards
 * `survivors` (indices into the code [I_k ; parity], parity row-major m x k)
 * and shard erased[e] is written over dst + row_starts[e] (row_starts NULL:
 * e * row_len). The server computes the decode rows itself
 * (fgfc_decode_matrix), caches them by pattern, and runs the request as the
 * overwrite form of mul_add_matrix_scattered. Same buffer rules as
 * fgfc_server_submit. */
typedef struct fgfc_rebuild_request {
  fgfc_field field;
  const uint32_t *parity;   /* m x k, row-major */
  size_t k, m;
  const size_t *survivors;  /* k shard indices, in the order of srcs */
  const fgfc_slice *srcs;   /* k survivor shards, row_len bytes each */
  const size_t *erased;     /* nerased shard indices to rebuild */
  size_t nerased;
  uint8_t *dst;
  size_t dst_len;
  const size_t *row_starts; /* nerased offsets into dst, or NULL */
  size_t row_len;
} fgfc_rebuild_request;
fgfc_status fgfc_server_submit_rebuild(fgfc_server *server, const fgfc_rebuild_request *req,
                                       uint64_t *ticket);
/* Blocks until the request is done and returns its status (its message via
 * fgfc_last_error); a ticket can be waited for once. */
fgfc_status fgfc_server_wait(fgfc_server *server, uint64_t ticket);
/* *done = 1 when the request finished; then behaves as fgfc_server_wait. */
fgfc_status fgfc_server_poll(fgfc_server *server, uint64_t ticket, int *done);
/* Blocks until every submitted request has finished. */
fgfc_status fgfc_server_drain(fgfc_server *server);
fgfc_status fgfc_server_get_stats(fgfc_server *server, fgfc_server_stats *out, int reset);
void fgfc_server_destroy(fgfc_server *server);

#ifdef __cplusplus
}
#endif
#endif /* FGF_CUDA_H */
