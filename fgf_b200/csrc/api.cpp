// api.cpp -- the C ABI of libfgfcuda.so (include/fgf_cuda.h).
//
// Each entry point validates its arguments in the same order, and with the
// same message text, as the matching `fgf::ops` function (src/ops.rs), applies
// the same zero/one shortcuts, and then lowers the call to launches of the
// matrix kernel: rows[j] (^)= XOR_t c[t][j] * src_t.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/fgf_cuda.h"
#include "internal.hpp"

using namespace fgfc;

namespace {

thread_local std::string t_err;

fgfc_status fail(fgfc_status st, const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  std::vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  t_err = buf;
  return st;
}

fgfc_status ok() {
  t_err.clear();
  return FGFC_OK;
}

fgfc_status cuda_fail(cudaError_t e, const char* what) {
  return fail(FGFC_ERR_CUDA, "%s: CUDA error: %s", what, cudaGetErrorString(e));
}

bool valid_field(int f) { return f >= 0 && f <= 8; }

size_t zu(size_t v) { return v; }

// ops.rs:300-307
bool check_width(int f, const char* name, size_t len, fgfc_status* st) {
  if (len % field_bytes(f) != 0) {
    *st = fail(FGFC_ERR_WIDTH, "%s: buffer of %zu bytes is not a whole number of %s elements", name,
               len, field_name(f));
    return false;
  }
  return true;
}

// ops.rs:309-316
bool check_pair(int f, const char* name, const char* ln, size_t l, const char* rn, size_t r,
                fgfc_status* st) {
  if (l != r) {
    *st = fail(FGFC_ERR_LENGTH, "%s: %s is %zu bytes but %s is %zu bytes", name, ln, l, rn, r);
    return false;
  }
  return check_width(f, name, l, st);
}

bool mul_overflows(size_t a, size_t b, size_t* out) {
  if (a && b > SIZE_MAX / a) return true;
  *out = a * b;
  return false;
}

}  // namespace

// ---------------------------------------------------------------- plans

struct fgfc_plan {
  int field;
  size_t rows, cols;
  std::vector<uint64_t> values;  // coefficients, any field width
  // GF(2) bit matrices for the tensor-core kernel, per orientation (matrix:
  // rows x cols; scatter: 1 x len; gather: len x 1), empty where the shape
  // is outside that kernel's range
  std::vector<uint32_t> bits_mat, bits_scat, bits_gath;
  uint64_t bits_key = 0;  // hash of bits_mat
  int device;
  uint32_t* dev;        // device tables, three orientations back to back
  size_t mat_groups;    // groups per source in the matrix orientation
  size_t off_mat, off_scat, off_gath;  // word offsets into `dev`
  size_t scat_groups, gath_groups;
  size_t off_k16 = 0, k16_groups = 0;  // Gf16: byte half-product tables of the matrix orientation (batches)
};

namespace {

// Coefficient source for a lowered matrix call: either raw host values
// (term-major, k x m) or device tables of a plan.
struct CoeffSrc {
  const uint64_t* host = nullptr;  // term-major k x m
  const uint32_t* dev = nullptr;   // compact tables [(t*E+p)*gstride + g][32]
  size_t gstride = 0;
  const uint32_t* bits = nullptr;  // GF(2) bit matrix (plans), or built from `host` when needed
};

std::mutex g_launch_mu;

fgfc_status run_matrix(int field, const uint8_t* const* srcs, size_t k, uint8_t* const* rows,
                       size_t m, const CoeffSrc& cs, size_t len, bool overwrite,
                       cudaStream_t stream, const char* name, bool allow_mma = true);

// The tensor-core contraction for the 16-byte-aligned body of a call whose
// sources and rows all share one offset within 16 bytes; the columns before
// and after the body go to the table kernels. Returns false (nothing
// enqueued) when the call does not qualify.
bool run_gf2mma(int field, const uint8_t* const* srcs, size_t k, uint8_t* const* rows, size_t m,
                const CoeffSrc& cs, size_t len, bool overwrite, cudaStream_t stream, const char* name,
                fgfc_status* st) {
  const int E = field_bytes(field);
  const uintptr_t al = reinterpret_cast<uintptr_t>(srcs[0]) & 15;
  if (al % E) return false;
  for (size_t t = 0; t < k; ++t)
    if ((reinterpret_cast<uintptr_t>(srcs[t]) & 15) != al) return false;
  for (size_t j = 0; j < m; ++j)
    if ((reinterpret_cast<uintptr_t>(rows[j]) & 15) != al) return false;
  const size_t head = std::min<size_t>((16 - al) & 15, len);
  const size_t blk_bytes = 512 * static_cast<size_t>(E);
  const uint64_t nblk = (len - head) / blk_bytes;
  if (!nblk) return false;
  std::vector<uint32_t> tmp;
  const uint32_t* bits = cs.bits;
  if (!bits) {
    tmp.resize(kGf2BitWords);
    gf2mma_bits(field, cs.host, k, m, tmp.data());
    bits = tmp.data();
  }
  std::vector<const uint8_t*> sp(k);
  std::vector<uint8_t*> rp(m);
  for (size_t t = 0; t < k; ++t) sp[t] = srcs[t] + head;
  for (size_t j = 0; j < m; ++j) rp[j] = rows[j] + head;
  cudaError_t e = gf2mma_launch(field, sp.data(), k, rp.data(), m, bits, nblk, overwrite, stream);
  if (e != cudaSuccess) {
    *st = cuda_fail(e, name);
    return true;
  }
  const size_t body_end = head + nblk * blk_bytes;
  if (head) {
    *st = run_matrix(field, srcs, k, rows, m, cs, head, overwrite, stream, name, false);
    if (*st != FGFC_OK) return true;
  }
  if (body_end < len) {
    for (size_t t = 0; t < k; ++t) sp[t] = srcs[t] + body_end;
    for (size_t j = 0; j < m; ++j) rp[j] = rows[j] + body_end;
    *st = run_matrix(field, sp.data(), k, rp.data(), m, cs, len - body_end, overwrite, stream, name, false);
    if (*st != FGFC_OK) return true;
  }
  *st = ok();
  return true;
}

fgfc_status run_matrix(int field, const uint8_t* const* srcs, size_t k, uint8_t* const* rows,
                       size_t m, const CoeffSrc& cs, size_t len, bool overwrite,
                       cudaStream_t stream, const char* name, bool allow_mma) {
  if (m == 0 || len == 0) return ok();
  if (allow_mma && k > 0 && (cs.bits || cs.host) && choose_kernel(field, k, m, len) == FGFC_KERNEL_GF2MMA) {
    fgfc_status st;
    if (run_gf2mma(field, srcs, k, rows, m, cs, len, overwrite, stream, name, &st)) return st;
  }
  if (k == 0) {
    if (overwrite) {
      cudaError_t e = launch_zero_rows(rows, static_cast<int>(m), len, stream);
      if (e != cudaSuccess) return cuda_fail(e, name);
    }
    return ok();
  }
  const int E = field_bytes(field);
  if (E == 8) {
    cudaError_t e = wide_launch(field, srcs, k, rows, m, cs.host, cs.dev, cs.gstride, len, overwrite, stream);
    return e == cudaSuccess ? ok() : cuda_fail(e, name);
  }
  const int R = 4 / E;
  const size_t gtot = (m + R - 1) / R;
  const bool inl = cs.dev == nullptr;
  const size_t slot_cap = inl ? kInlineSlots : kMaxSlots;
  size_t gp = std::min<size_t>(gtot, 4);
  while (gp > 1 && static_cast<size_t>(E) * gp > slot_cap) --gp;
  size_t kc = std::min<size_t>(k, slot_cap / (E * gp));
  kc = std::min<size_t>(kc, kMaxSrc);
  if (kc == 0) return fail(FGFC_ERR_LIMIT, "%s: internal tiling failed", name);

  // Alignment class shared by every source; the kernels store rows at any
  // offset (columns are spliced in registers when a row's offset differs).
  uintptr_t al = reinterpret_cast<uintptr_t>(srcs[0]) & 15;
  bool same = true;
  for (size_t t = 0; t < k; ++t) same &= (reinterpret_cast<uintptr_t>(srcs[t]) & 15) == al;
  same &= (al % E) == 0;
  uint64_t head = len, nvec = 0;
  bool shift = false;
  if (same) {
    head = std::min<uint64_t>((16 - al) & 15, len);
    nvec = (len - head) / 16;
    for (size_t j = 0; j < m; ++j) shift |= (reinterpret_cast<uintptr_t>(rows[j]) & 15) != al;
  }

  const bool byte_tables = choose_kernel(field, k, m, len) == FGFC_KERNEL_BYTE;
  static thread_local MatrixLaunch a;  // large (inline tables): keep off the stack
  for (size_t g0 = 0; g0 < gtot; g0 += gp) {
    const size_t G = std::min(gp, gtot - g0);
    const size_t r0 = g0 * R;
    const size_t nr = std::min(m - r0, G * R);
    for (size_t t0 = 0; t0 < k; t0 += kc) {
      const size_t kk = std::min(kc, k - t0);
      a.len = len;
      a.head = head;
      a.nvec = nvec;
      a.shift = 0;
      for (size_t j = 0; j < nr; ++j) a.shift |= (reinterpret_cast<uintptr_t>(rows[r0 + j]) & 15) != al;
      a.shift &= shift ? 1u : 0u;
      a.k = static_cast<uint32_t>(kk);
      a.nrows = static_cast<uint32_t>(nr);
      for (size_t t = 0; t < kk; ++t) a.src[t] = srcs[t0 + t];
      for (size_t j = 0; j < nr; ++j) a.dst[j] = rows[r0 + j];
      if (inl) {
        build_compact_tables(field, cs.host, m, t0, kk, g0, G, a.inline_tab);
        a.tables = nullptr;
        a.gstride = static_cast<uint32_t>(G);
        a.g0 = 0;
      } else {
        a.tables = cs.dev + t0 * E * cs.gstride * kCompactWords;
        a.gstride = static_cast<uint32_t>(cs.gstride);
        a.g0 = static_cast<uint32_t>(g0);
      }
      cudaError_t e;
      {
        std::lock_guard<std::mutex> lk(g_launch_mu);
        e = launch_matrix(field, static_cast<int>(G), overwrite && t0 == 0, a, stream, byte_tables);
      }
      if (e != cudaSuccess) return cuda_fail(e, name);
    }
  }
  return ok();
}

bool all_zero(const uint64_t* c, size_t n, uint64_t mask) {
  for (size_t i = 0; i < n; ++i)
    if (c[i] & mask) return false;
  return true;
}

fgfc_status upload_plan_tables(fgfc_plan* p) {
  const int E = field_bytes(p->field);
  const size_t len = p->values.size();
  // 4-byte output groups covering n rows of E-byte elements
  // Per source: E input bytes x (groups) slots of compact tables; the
  // 8-byte fields keep their half-product tables instead (build_wide_tables:
  // 12 slots per source and row, "groups" counting rows).
  const bool wide = E == 8;
  const auto groups = [E, wide](size_t n) { return wide ? n : (n * E + 3) / 4; };
  const size_t slots_per_src = wide ? kWideSlotsPerSrcRow : static_cast<size_t>(E);
  const auto build = [&](const uint64_t* c, size_t m, size_t k, size_t G, uint32_t* out) {
    if (wide)
      build_wide_tables(p->field, c, m, 0, k, 0, G, out);
    else
      build_compact_tables(p->field, c, m, 0, k, 0, G, out);
  };
  // matrix orientation: rows = sources, cols = destination rows
  p->mat_groups = groups(p->cols);
  const size_t n_mat = p->rows * slots_per_src * p->mat_groups * kCompactWords;
  p->scat_groups = groups(len);
  const size_t n_scat = slots_per_src * p->scat_groups * kCompactWords;
  p->gath_groups = groups(1);
  const size_t n_gath = len * slots_per_src * p->gath_groups * kCompactWords;
  // Gf16 batches also run the matrix orientation by byte half-products
  p->k16_groups = E == 2 ? (p->cols + 3) / 4 : 0;
  const size_t n_k16 = p->rows * 3 * p->k16_groups * kCompactWords;
  std::vector<uint32_t> host(n_mat + n_scat + n_gath + n_k16 + 1, 0);
  p->off_mat = 0;
  p->off_scat = n_mat;
  p->off_gath = n_mat + n_scat;
  p->off_k16 = n_mat + n_scat + n_gath;
  if (n_k16) build_kara16_tables(p->values.data(), p->cols, p->rows, p->k16_groups, host.data() + p->off_k16);
  if (n_mat) build(p->values.data(), p->cols, p->rows, p->mat_groups, host.data() + p->off_mat);
  if (n_scat) build(p->values.data(), len, 1, p->scat_groups, host.data() + p->off_scat);
  // gather orientation: source i has the single coefficient values[i]
  if (n_gath) build(p->values.data(), 1, len, p->gath_groups, host.data() + p->off_gath);
  if (n_mat && gf2mma_shape_ok(p->field, p->rows, p->cols)) {
    p->bits_mat.resize(kGf2BitWords);
    gf2mma_bits(p->field, p->values.data(), p->rows, p->cols, p->bits_mat.data());
    uint64_t h = 1469598103934665603ull ^ (static_cast<uint64_t>(p->field) << 56);
    for (uint32_t w : p->bits_mat) h = (h ^ w) * 1099511628211ull;
    p->bits_key = h;
  }
  if (len && gf2mma_shape_ok(p->field, 1, len)) {
    p->bits_scat.resize(kGf2BitWords);
    gf2mma_bits(p->field, p->values.data(), 1, len, p->bits_scat.data());
  }
  if (len && gf2mma_shape_ok(p->field, len, 1)) {
    p->bits_gath.resize(kGf2BitWords);
    gf2mma_bits(p->field, p->values.data(), len, 1, p->bits_gath.data());
  }
  cudaError_t e = cudaGetDevice(&p->device);
  if (e != cudaSuccess) return cuda_fail(e, "Plan::matrix");
  e = cudaMalloc(&p->dev, host.size() * sizeof(uint32_t));
  if (e != cudaSuccess) return fail(FGFC_ERR_NOMEM, "Plan::matrix: device allocation failed: %s",
                                    cudaGetErrorString(e));
  e = cudaMemcpy(p->dev, host.data(), host.size() * sizeof(uint32_t), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return cuda_fail(e, "Plan::matrix");
  return ok();
}

CoeffSrc plan_mat(const fgfc_plan* p) {
  CoeffSrc c;
  c.dev = p->dev + p->off_mat;
  c.gstride = p->mat_groups;
  c.bits = p->bits_mat.empty() ? nullptr : p->bits_mat.data();
  return c;
}
CoeffSrc plan_scat(const fgfc_plan* p) {
  CoeffSrc c;
  c.dev = p->dev + p->off_scat;
  c.gstride = p->scat_groups;
  c.bits = p->bits_scat.empty() ? nullptr : p->bits_scat.data();
  return c;
}
CoeffSrc plan_gath(const fgfc_plan* p) {
  CoeffSrc c;
  c.dev = p->dev + p->off_gath;
  c.gstride = p->gath_groups;
  c.bits = p->bits_gath.empty() ? nullptr : p->bits_gath.data();
  return c;
}

}  // namespace

template <typename C>
static fgfc_status plan_create(fgfc_field field, size_t rows, size_t cols, const C* coeffs, fgfc_plan** out) {
  if (!out || !valid_field(field)) return fail(FGFC_ERR_ARG, "Plan::matrix: invalid argument");
  *out = nullptr;
  size_t n;
  if (mul_overflows(rows, cols, &n)) return fail(FGFC_ERR_OVERFLOW, "Plan::matrix: dimensions overflow");
  if (n && !coeffs) return fail(FGFC_ERR_ARG, "Plan::matrix: null coefficients");
  fgfc_plan* p = new fgfc_plan();
  p->field = field;
  p->rows = rows;
  p->cols = cols;
  p->values.assign(coeffs, coeffs + n);
  for (auto& v : p->values) v &= field_mask(field);
  p->dev = nullptr;
  fgfc_status st = upload_plan_tables(p);
  if (st != FGFC_OK) {
    fgfc_plan_destroy(p);
    return st;
  }
  *out = p;
  return ok();
}

extern "C" {

const char* fgfc_last_error(void) { return t_err.c_str(); }

fgfc_status fgfc_device_check(int clear) {
  const int w = gf2mma_error(clear != 0);
  if (w < 0) return fail(FGFC_ERR_CUDA, "device_check: cannot read the device error word");
  if (w) return fail(FGFC_ERR_CUDA, "device_check: a tensor-core kernel gave up waiting (code %d)", w);
  return ok();
}
const char* fgfc_version(void) { return "fgf-cuda 0.1.0 (sm_100a; mirrors fgf 0.4.0 ops)"; }

void fgfc_limits(size_t* max_sources, size_t* max_rows) {
  if (max_sources) *max_sources = SIZE_MAX;
  if (max_rows) *max_rows = SIZE_MAX;
}

size_t fgfc_field_bytes(fgfc_field field) { return valid_field(field) ? field_bytes(field) : 0; }

fgfc_status fgfc_plan_create(fgfc_field field, size_t rows, size_t cols, const uint32_t* coeffs,
                             fgfc_plan** out) {
  return plan_create(field, rows, cols, coeffs, out);
}

fgfc_status fgfc_plan_create_u64(fgfc_field field, size_t rows, size_t cols, const uint64_t* coeffs,
                                 fgfc_plan** out) {
  return plan_create(field, rows, cols, coeffs, out);
}

fgfc_status fgfc_coeff_create(fgfc_field field, uint32_t coeff, fgfc_plan** out) {
  return plan_create(field, 1, 1, &coeff, out);
}

fgfc_status fgfc_coeff_create_u64(fgfc_field field, uint64_t coeff, fgfc_plan** out) {
  return plan_create(field, 1, 1, &coeff, out);
}

void fgfc_plan_destroy(fgfc_plan* plan) {
  if (!plan) return;
  if (plan->dev) {
    int cur = 0;
    cudaGetDevice(&cur);
    if (cur != plan->device) cudaSetDevice(plan->device);
    cudaFree(plan->dev);
    if (cur != plan->device) cudaSetDevice(cur);
  }
  delete plan;
}

fgfc_status fgfc_plan_dimensions(const fgfc_plan* plan, size_t* rows, size_t* cols) {
  if (!plan) return fail(FGFC_ERR_ARG, "Plan: null plan");
  if (rows) *rows = plan->rows;
  if (cols) *cols = plan->cols;
  return ok();
}

size_t fgfc_plan_len(const fgfc_plan* plan) { return plan ? plan->values.size() : 0; }

fgfc_field fgfc_plan_field(const fgfc_plan* plan) {
  return plan ? static_cast<fgfc_field>(plan->field) : FGFC_GF8B;
}

fgfc_status fgfc_plan_values(const fgfc_plan* plan, uint32_t* out) {
  if (!plan || (!out && !plan->values.empty())) return fail(FGFC_ERR_ARG, "Plan: null argument");
  for (size_t i = 0; i < plan->values.size(); ++i) out[i] = static_cast<uint32_t>(plan->values[i]);
  return ok();
}

fgfc_status fgfc_plan_values_u64(const fgfc_plan* plan, uint64_t* out) {
  if (!plan || (!out && !plan->values.empty())) return fail(FGFC_ERR_ARG, "Plan: null argument");
  std::copy(plan->values.begin(), plan->values.end(), out);
  return ok();
}

fgfc_status fgfc_plan_get_at_u64(const fgfc_plan* plan, size_t row, size_t col, uint64_t* out) {
  if (!plan || !out) return fail(FGFC_ERR_ARG, "Plan: null argument");
  if (row >= plan->rows || col >= plan->cols) return fail(FGFC_ERR_ARG, "Plan::get_at: out of bounds");
  *out = plan->values[row * plan->cols + col];
  return ok();
}

fgfc_status fgfc_plan_get_at(const fgfc_plan* plan, size_t row, size_t col, uint32_t* out) {
  if (!plan || !out) return fail(FGFC_ERR_ARG, "Plan: null argument");
  if (row >= plan->rows || col >= plan->cols) return fail(FGFC_ERR_ARG, "Plan::get_at: out of bounds");
  *out = static_cast<uint32_t>(plan->values[row * plan->cols + col]);
  return ok();
}

// ---------------------------------------------------------------- single row

fgfc_status fgfc_add_assign(fgfc_field field, uint8_t* dst, size_t dst_len, const uint8_t* src,
                            size_t src_len, fgfc_stream stream) {
  fgfc_status st;
  if (!valid_field(field)) return fail(FGFC_ERR_ARG, "add_assign: unknown field");
  if (!check_pair(field, "add_assign", "dst", dst_len, "src", src_len, &st)) return st;
  cudaError_t e = launch_xor(dst, src, dst_len, stream);
  return e == cudaSuccess ? ok() : cuda_fail(e, "add_assign");
}

static fgfc_status mul_add_impl(int field, const char* name, uint8_t* dst, size_t dst_len,
                                uint64_t coeff, const fgfc_plan* plan, const uint8_t* src,
                                size_t src_len, cudaStream_t stream) {
  fgfc_status st;
  if (!check_pair(field, name, "dst", dst_len, "src", src_len, &st)) return st;
  coeff &= field_mask(field);
  if (coeff == 0) return ok();
  if (coeff == 1) {
    cudaError_t e = launch_xor(dst, src, dst_len, stream);
    return e == cudaSuccess ? ok() : cuda_fail(e, name);
  }
  uint8_t* rows[1] = {dst};
  const uint8_t* srcs[1] = {src};
  CoeffSrc cs;
  if (plan) {
    cs = plan_mat(plan);
  } else {
    cs.host = &coeff;
  }
  return run_matrix(field, srcs, 1, rows, 1, cs, dst_len, false, stream, name);
}

fgfc_status fgfc_mul_add(fgfc_field field, uint8_t* dst, size_t dst_len, uint32_t coeff,
                         const uint8_t* src, size_t src_len, fgfc_stream stream) {
  if (!valid_field(field)) return fail(FGFC_ERR_ARG, "mul_add: unknown field");
  return mul_add_impl(field, "mul_add", dst, dst_len, coeff, nullptr, src, src_len, stream);
}

static bool single_coeff(const fgfc_plan* p, const char* name, fgfc_status* st) {
  if (!p) {
    *st = fail(FGFC_ERR_ARG, "%s: null coefficient", name);
    return false;
  }
  if (p->values.size() != 1) {
    *st = fail(FGFC_ERR_ARG, "%s: a prepared coefficient holds exactly one value, this plan holds %zu",
               name, p->values.size());
    return false;
  }
  return true;
}

fgfc_status fgfc_mul_add_with(uint8_t* dst, size_t dst_len, const fgfc_plan* coeff,
                              const uint8_t* src, size_t src_len, fgfc_stream stream) {
  fgfc_status st;
  if (!single_coeff(coeff, "mul_add_with", &st)) return st;
  return mul_add_impl(coeff->field, "mul_add_with", dst, dst_len, coeff->values[0], coeff, src,
                      src_len, stream);
}

static fgfc_status mul_into_impl(int field, const char* name, uint8_t* dst, size_t dst_len,
                                 uint64_t coeff, const fgfc_plan* plan, const uint8_t* src,
                                 size_t src_len, cudaStream_t stream) {
  fgfc_status st;
  if (!check_pair(field, name, "dst", dst_len, "src", src_len, &st)) return st;
  coeff &= field_mask(field);
  if (dst_len == 0) return ok();
  if (coeff == 0) {
    cudaError_t e = cudaMemsetAsync(dst, 0, dst_len, stream);
    return e == cudaSuccess ? ok() : cuda_fail(e, name);
  }
  if (coeff == 1) {
    cudaError_t e = cudaMemcpyAsync(dst, src, dst_len, cudaMemcpyDeviceToDevice, stream);
    return e == cudaSuccess ? ok() : cuda_fail(e, name);
  }
  uint8_t* rows[1] = {dst};
  const uint8_t* srcs[1] = {src};
  CoeffSrc cs;
  if (plan) {
    cs = plan_mat(plan);
  } else {
    cs.host = &coeff;
  }
  return run_matrix(field, srcs, 1, rows, 1, cs, dst_len, true, stream, name);
}

fgfc_status fgfc_mul_into(fgfc_field field, uint8_t* dst, size_t dst_len, uint32_t coeff,
                          const uint8_t* src, size_t src_len, fgfc_stream stream) {
  if (!valid_field(field)) return fail(FGFC_ERR_ARG, "mul_into: unknown field");
  return mul_into_impl(field, "mul_into", dst, dst_len, coeff, nullptr, src, src_len, stream);
}

fgfc_status fgfc_mul_into_with(uint8_t* dst, size_t dst_len, const fgfc_plan* coeff,
                               const uint8_t* src, size_t src_len, fgfc_stream stream) {
  fgfc_status st;
  if (!single_coeff(coeff, "mul_into_with", &st)) return st;
  return mul_into_impl(coeff->field, "mul_into_with", dst, dst_len, coeff->values[0], coeff, src,
                       src_len, stream);
}

static fgfc_status mul_assign_impl(int field, const char* name, uint8_t* dst, size_t dst_len,
                                   uint64_t coeff, const fgfc_plan* plan, cudaStream_t stream) {
  fgfc_status st;
  if (!check_width(field, name, dst_len, &st)) return st;
  coeff &= field_mask(field);
  if (coeff == 1 || dst_len == 0) return ok();
  if (coeff == 0) {
    cudaError_t e = cudaMemsetAsync(dst, 0, dst_len, stream);
    return e == cudaSuccess ? ok() : cuda_fail(e, name);
  }
  uint8_t* rows[1] = {dst};
  const uint8_t* srcs[1] = {dst};  // in place: every byte is read before it is written, by one thread
  CoeffSrc cs;
  if (plan) {
    cs = plan_mat(plan);
  } else {
    cs.host = &coeff;
  }
  return run_matrix(field, srcs, 1, rows, 1, cs, dst_len, true, stream, name);
}

fgfc_status fgfc_mul_assign(fgfc_field field, uint8_t* dst, size_t dst_len, uint32_t coeff,
                            fgfc_stream stream) {
  if (!valid_field(field)) return fail(FGFC_ERR_ARG, "mul_assign: unknown field");
  return mul_assign_impl(field, "mul_assign", dst, dst_len, coeff, nullptr, stream);
}

fgfc_status fgfc_mul_assign_with(uint8_t* dst, size_t dst_len, const fgfc_plan* coeff,
                                 fgfc_stream stream) {
  fgfc_status st;
  if (!single_coeff(coeff, "mul_assign_with", &st)) return st;
  return mul_assign_impl(coeff->field, "mul_assign_with", dst, dst_len, coeff->values[0], coeff,
                         stream);
}

fgfc_status fgfc_mul_elementwise(fgfc_field field, uint8_t* dst, size_t dst_len, const uint8_t* a,
                                 size_t a_len, const uint8_t* b, size_t b_len, fgfc_stream stream) {
  fgfc_status st;
  if (!valid_field(field)) return fail(FGFC_ERR_ARG, "mul_elementwise: unknown field");
  if (!check_pair(field, "mul_elementwise", "dst", dst_len, "a", a_len, &st)) return st;
  if (!check_pair(field, "mul_elementwise", "dst", dst_len, "b", b_len, &st)) return st;
  cudaError_t e = launch_elementwise(field, dst, a, b, dst_len, stream);
  return e == cudaSuccess ? ok() : cuda_fail(e, "mul_elementwise");
}

// ---------------------------------------------------------------- scatter / gather

static fgfc_status scatter_impl(int field, const char* name, const char* count_word, uint8_t* rows,
                                size_t rows_len, size_t row_len, const uint64_t* coeffs, size_t n,
                                const fgfc_plan* plan, const uint8_t* src, size_t src_len,
                                cudaStream_t stream) {
  fgfc_status st;
  if (!check_pair(field, name, "row_len", row_len, "src", src_len, &st)) return st;
  size_t used;
  if (mul_overflows(n, row_len, &used)) return fail(FGFC_ERR_OVERFLOW, "%s: row geometry overflows", name);
  if (rows_len < used)
    return fail(FGFC_ERR_ROWS, "%s: rows is %zu bytes but %zu rows of %zu bytes need %zu", name,
                rows_len, n, row_len, used);
  (void)count_word;
  if (all_zero(coeffs, n, field_mask(field))) return ok();
  std::vector<uint8_t*> rp(n);
  for (size_t j = 0; j < n; ++j) rp[j] = rows + j * row_len;
  const uint8_t* srcs[1] = {src};
  CoeffSrc cs;
  if (plan) {
    cs = plan_scat(plan);
  } else {
    cs.host = coeffs;
  }
  return run_matrix(field, srcs, 1, rp.data(), n, cs, row_len, false, stream, name);
}

fgfc_status fgfc_mul_add_scatter(fgfc_field field, uint8_t* rows, size_t rows_len, size_t row_len,
                                 const uint32_t* coeffs, size_t ncoeffs, const uint8_t* src,
                                 size_t src_len, fgfc_stream stream) {
  if (!valid_field(field)) return fail(FGFC_ERR_ARG, "mul_add_scatter: unknown field");
  std::vector<uint64_t> c(coeffs, coeffs + ncoeffs);
  for (auto& v : c) v &= field_mask(field);
  return scatter_impl(field, "mul_add_scatter", "coefficients", rows, rows_len, row_len, c.data(),
                      ncoeffs, nullptr, src, src_len, stream);
}

fgfc_status fgfc_mul_add_scatter_with(uint8_t* rows, size_t rows_len, size_t row_len,
                                      const fgfc_plan* plan, const uint8_t* src, size_t src_len,
                                      fgfc_stream stream) {
  if (!plan) return fail(FGFC_ERR_ARG, "mul_add_scatter_with: null plan");
  return scatter_impl(plan->field, "mul_add_scatter_with", "plan", rows, rows_len, row_len,
                      plan->values.data(), plan->values.size(), plan, src, src_len, stream);
}

// Shared validation of gather / dot_product (raw and prepared forms).
static bool check_sources(int field, const char* name, bool with_plan, size_t dst_len, size_t ncoeffs,
                          const fgfc_slice* srcs, size_t nsrcs, fgfc_status* st) {
  if (!check_width(field, name, dst_len, st)) return false;
  if (ncoeffs != nsrcs) {
    if (with_plan)
      *st = fail(FGFC_ERR_COEFFS, "%s: plan has %zu coefficients but there are %zu sources", name,
                 ncoeffs, nsrcs);
    else
      *st = fail(FGFC_ERR_COEFFS, "%s: %zu coefficients for %zu sources", name, ncoeffs, nsrcs);
    return false;
  }
  if (nsrcs && !srcs) {
    *st = fail(FGFC_ERR_ARG, "%s: null sources", name);
    return false;
  }
  for (size_t i = 0; i < nsrcs; ++i) {
    if (srcs[i].len != dst_len) {
      // mul_add_gather (raw) names no index: ops.rs:542-550
      if (!with_plan && std::strcmp(name, "mul_add_gather") == 0)
        *st = fail(FGFC_ERR_SOURCE, "%s: source is %zu bytes, expected %zu", name, srcs[i].len, dst_len);
      else
        *st = fail(FGFC_ERR_SOURCE, "%s: source %zu is %zu bytes, expected %zu", name, i, srcs[i].len,
                   dst_len);
      return false;
    }
  }
  return true;
}

static fgfc_status gather_impl(int field, const char* name, bool with_plan, uint8_t* dst,
                               size_t dst_len, const uint64_t* coeffs, size_t ncoeffs,
                               const fgfc_plan* plan, const fgfc_slice* srcs, size_t nsrcs,
                               bool overwrite, cudaStream_t stream) {
  fgfc_status st;
  if (!check_sources(field, name, with_plan, dst_len, ncoeffs, srcs, nsrcs, &st)) return st;
  const bool zero = nsrcs == 0 || all_zero(coeffs, ncoeffs, field_mask(field));
  if (zero) {
    if (overwrite && dst_len) {
      cudaError_t e = cudaMemsetAsync(dst, 0, dst_len, stream);
      if (e != cudaSuccess) return cuda_fail(e, name);
    }
    return ok();
  }
  if (overwrite && nsrcs == 1)  // ops.rs:619-622 / 654-658: one source is mul_into
    return mul_into_impl(field, with_plan ? "mul_into_with" : "mul_into", dst, dst_len, coeffs[0],
                         plan, srcs[0].ptr, srcs[0].len, stream);
  std::vector<const uint8_t*> sp(nsrcs);
  for (size_t i = 0; i < nsrcs; ++i) sp[i] = srcs[i].ptr;
  uint8_t* rows[1] = {dst};
  CoeffSrc cs;
  if (plan) {
    cs = plan_gath(plan);
  } else {
    cs.host = coeffs;  // k x 1, term-major
  }
  return run_matrix(field, sp.data(), nsrcs, rows, 1, cs, dst_len, overwrite, stream, name);
}

fgfc_status fgfc_mul_add_gather(fgfc_field field, uint8_t* dst, size_t dst_len,
                                const uint32_t* coeffs, size_t ncoeffs, const fgfc_slice* srcs,
                                size_t nsrcs, fgfc_stream stream) {
  if (!valid_field(field)) return fail(FGFC_ERR_ARG, "mul_add_gather: unknown field");
  std::vector<uint64_t> c(coeffs, coeffs + ncoeffs);
  for (auto& v : c) v &= field_mask(field);
  return gather_impl(field, "mul_add_gather", false, dst, dst_len, c.data(), ncoeffs, nullptr, srcs,
                     nsrcs, false, stream);
}

fgfc_status fgfc_mul_add_gather_with(uint8_t* dst, size_t dst_len, const fgfc_plan* plan,
                                     const fgfc_slice* srcs, size_t nsrcs, fgfc_stream stream) {
  if (!plan) return fail(FGFC_ERR_ARG, "mul_add_gather_with: null plan");
  return gather_impl(plan->field, "mul_add_gather_with", true, dst, dst_len, plan->values.data(),
                     plan->values.size(), plan, srcs, nsrcs, false, stream);
}

fgfc_status fgfc_dot_product(fgfc_field field, uint8_t* dst, size_t dst_len,
                             const uint32_t* coeffs, size_t ncoeffs, const fgfc_slice* srcs,
                             size_t nsrcs, fgfc_stream stream) {
  if (!valid_field(field)) return fail(FGFC_ERR_ARG, "dot_product: unknown field");
  std::vector<uint64_t> c(coeffs, coeffs + ncoeffs);
  for (auto& v : c) v &= field_mask(field);
  return gather_impl(field, "dot_product", false, dst, dst_len, c.data(), ncoeffs, nullptr, srcs, nsrcs,
                     true, stream);
}

fgfc_status fgfc_dot_product_with(uint8_t* dst, size_t dst_len, const fgfc_plan* plan,
                                  const fgfc_slice* srcs, size_t nsrcs, fgfc_stream stream) {
  if (!plan) return fail(FGFC_ERR_ARG, "dot_product_with: null plan");
  // A single-source prepared dot product is mul_into_with on plan entry 0,
  // whose device tables are the gather orientation's first slot.
  return gather_impl(plan->field, "dot_product_with", true, dst, dst_len, plan->values.data(),
                     plan->values.size(), plan, srcs, nsrcs, true, stream);
}

// ---------------------------------------------------------------- matrices

static fgfc_status matrix_terms_impl(int field, const char* name, bool overwrite, uint8_t* rows,
                                     size_t rows_len, size_t row_len, size_t nrows,
                                     const fgfc_term* terms, size_t nterms, cudaStream_t stream) {
  fgfc_status st;
  if (!check_width(field, name, row_len, &st)) return st;
  size_t used;
  if (mul_overflows(nrows, row_len, &used)) return fail(FGFC_ERR_OVERFLOW, "%s: row geometry overflows", name);
  if (rows_len < used)
    return fail(FGFC_ERR_ROWS, "%s: rows is %zu bytes but %zu rows of %zu bytes need %zu", name,
                rows_len, nrows, row_len, used);
  if (nterms && !terms) return fail(FGFC_ERR_ARG, "%s: null terms", name);
  for (size_t t = 0; t < nterms; ++t) {
    if (terms[t].ncoeffs != nrows)
      return fail(FGFC_ERR_COEFFS, "%s: term supplies %zu coefficients for %zu rows", name,
                  terms[t].ncoeffs, nrows);
    if (terms[t].src_len != row_len)
      return fail(FGFC_ERR_SOURCE, "%s: source is %zu bytes, expected %zu", name, terms[t].src_len,
                  row_len);
  }
  if (nrows == 0) return ok();
  if (nterms == 0) {
    if (overwrite && used) {
      cudaError_t e = cudaMemsetAsync(rows, 0, used, stream);
      if (e != cudaSuccess) return cuda_fail(e, name);
    }
    return ok();
  }
  std::vector<uint64_t> coeffs(nterms * nrows);
  std::vector<const uint8_t*> sp(nterms);
  for (size_t t = 0; t < nterms; ++t) {
    sp[t] = terms[t].src;
    for (size_t j = 0; j < nrows; ++j) coeffs[t * nrows + j] = terms[t].coeffs[j] & field_mask(field);
  }
  std::vector<uint8_t*> rp(nrows);
  for (size_t j = 0; j < nrows; ++j) rp[j] = rows + j * row_len;
  CoeffSrc cs;
  cs.host = coeffs.data();
  return run_matrix(field, sp.data(), nterms, rp.data(), nrows, cs, row_len, overwrite, stream, name);
}

fgfc_status fgfc_mul_add_matrix(fgfc_field field, uint8_t* rows, size_t rows_len, size_t row_len,
                                size_t nrows, const fgfc_term* terms, size_t nterms,
                                fgfc_stream stream) {
  if (!valid_field(field)) return fail(FGFC_ERR_ARG, "mul_add_matrix: unknown field");
  return matrix_terms_impl(field, "mul_add_matrix", false, rows, rows_len, row_len, nrows, terms,
                           nterms, stream);
}

fgfc_status fgfc_dot_product_matrix(fgfc_field field, uint8_t* rows, size_t rows_len,
                                    size_t row_len, size_t nrows, const fgfc_term* terms,
                                    size_t nterms, fgfc_stream stream) {
  if (!valid_field(field)) return fail(FGFC_ERR_ARG, "dot_product_matrix: unknown field");
  return matrix_terms_impl(field, "dot_product_matrix", true, rows, rows_len, row_len, nrows, terms,
                           nterms, stream);
}

static fgfc_status matrix_plan_impl(const char* name, bool overwrite, uint8_t* rows, size_t rows_len,
                                    size_t row_len, size_t nrows, const fgfc_plan* plan,
                                    const fgfc_slice* srcs, size_t nsrcs, cudaStream_t stream) {
  fgfc_status st;
  if (!plan) return fail(FGFC_ERR_ARG, "%s: null plan", name);
  const int field = plan->field;
  if (!check_width(field, name, row_len, &st)) return st;
  size_t used;
  if (mul_overflows(nrows, row_len, &used)) return fail(FGFC_ERR_OVERFLOW, "%s: row geometry overflows", name);
  if (rows_len < used)
    return fail(FGFC_ERR_ROWS, "%s: rows is %zu bytes but %zu rows of %zu bytes need %zu", name,
                rows_len, nrows, row_len, used);
  if (plan->rows != nsrcs || plan->cols != nrows)
    return fail(FGFC_ERR_PLAN_DIMS, "%s: plan dimensions do not match (sources, rows)", name);
  if (nsrcs && !srcs) return fail(FGFC_ERR_ARG, "%s: null sources", name);
  for (size_t i = 0; i < nsrcs; ++i)
    if (srcs[i].len != row_len)
      return fail(FGFC_ERR_SOURCE, "%s: source %zu is %zu bytes, expected %zu", name, i, srcs[i].len,
                  row_len);
  if (nrows == 0) return ok();
  if (nsrcs == 0) {
    if (overwrite && used) {
      cudaError_t e = cudaMemsetAsync(rows, 0, used, stream);
      if (e != cudaSuccess) return cuda_fail(e, name);
    }
    return ok();
  }
  std::vector<const uint8_t*> sp(nsrcs);
  for (size_t i = 0; i < nsrcs; ++i) sp[i] = srcs[i].ptr;
  std::vector<uint8_t*> rp(nrows);
  for (size_t j = 0; j < nrows; ++j) rp[j] = rows + j * row_len;
  return run_matrix(field, sp.data(), nsrcs, rp.data(), nrows, plan_mat(plan), row_len, overwrite,
                    stream, name);
}

fgfc_status fgfc_mul_add_matrix_with(uint8_t* rows, size_t rows_len, size_t row_len, size_t nrows,
                                     const fgfc_plan* plan, const fgfc_slice* srcs, size_t nsrcs,
                                     fgfc_stream stream) {
  return matrix_plan_impl("mul_add_matrix_with", false, rows, rows_len, row_len, nrows, plan, srcs,
                          nsrcs, stream);
}

fgfc_status fgfc_dot_product_matrix_with(uint8_t* rows, size_t rows_len, size_t row_len,
                                         size_t nrows, const fgfc_plan* plan,
                                         const fgfc_slice* srcs, size_t nsrcs,
                                         fgfc_stream stream) {
  return matrix_plan_impl("dot_product_matrix_with", true, rows, rows_len, row_len, nrows, plan, srcs,
                          nsrcs, stream);
}

// ops.rs:887-941
static bool check_scattered_rows(int field, const char* name, size_t dst_len, size_t row_len,
                                 const size_t* row_starts, size_t nrows, fgfc_status* st) {
  if (!check_width(field, name, row_len, st)) return false;
  if (nrows && !row_starts) {
    *st = fail(FGFC_ERR_ARG, "%s: null row_starts", name);
    return false;
  }
  for (size_t j = 0; j < nrows; ++j) {
    const size_t start = row_starts[j];
    if (start > SIZE_MAX - row_len) {
      *st = fail(FGFC_ERR_OVERFLOW, "%s: row offset + length overflows", name);
      return false;
    }
    const size_t end = start + row_len;
    if (end > dst_len) {
      *st = fail(FGFC_ERR_BOUNDS, "%s: row %zu spans %zu..%zu but dst is %zu bytes", name, j, start, end,
                 dst_len);
      return false;
    }
    if (start % field_bytes(field) != 0) {
      *st = fail(FGFC_ERR_ALIGN, "%s: row %zu offset %zu is not a whole number of %s elements", name, j,
                 start, field_name(field));
      return false;
    }
  }
  for (size_t a = 0; a < nrows; ++a)
    for (size_t b = a + 1; b < nrows; ++b) {
      const size_t sa = row_starts[a], sb = row_starts[b];
      const size_t lo = std::min(sa, sb), hi = std::max(sa, sb);
      if (hi - lo < row_len) {
        *st = fail(FGFC_ERR_OVERLAP, "%s: rows at %zu and %zu overlap for %zu-byte rows", name, sa, sb,
                   row_len);
        return false;
      }
    }
  return true;
}

fgfc_status fgfc_mul_add_matrix_scattered(fgfc_field field, uint8_t* dst, size_t dst_len,
                                          size_t row_len, const size_t* row_starts, size_t nrows,
                                          const fgfc_term* terms, size_t nterms,
                                          fgfc_stream stream) {
  const char* name = "mul_add_matrix_scattered";
  fgfc_status st;
  if (!valid_field(field)) return fail(FGFC_ERR_ARG, "%s: unknown field", name);
  if (!check_scattered_rows(field, name, dst_len, row_len, row_starts, nrows, &st)) return st;
  if (nterms && !terms) return fail(FGFC_ERR_ARG, "%s: null terms", name);
  for (size_t t = 0; t < nterms; ++t) {
    if (terms[t].ncoeffs != nrows)
      return fail(FGFC_ERR_COEFFS, "%s: term supplies %zu coefficients for %zu rows", name,
                  terms[t].ncoeffs, nrows);
    if (terms[t].src_len != row_len)
      return fail(FGFC_ERR_SOURCE, "%s: source is %zu bytes, expected %zu", name, terms[t].src_len,
                  row_len);
  }
  if (nrows == 0 || nterms == 0) return ok();
  std::vector<uint64_t> coeffs(nterms * nrows);
  std::vector<const uint8_t*> sp(nterms);
  for (size_t t = 0; t < nterms; ++t) {
    sp[t] = terms[t].src;
    for (size_t j = 0; j < nrows; ++j) coeffs[t * nrows + j] = terms[t].coeffs[j] & field_mask(field);
  }
  std::vector<uint8_t*> rp(nrows);
  for (size_t j = 0; j < nrows; ++j) rp[j] = dst + row_starts[j];
  CoeffSrc cs;
  cs.host = coeffs.data();
  return run_matrix(field, sp.data(), nterms, rp.data(), nrows, cs, row_len, false, stream, name);
}

static fgfc_status scattered_plan_impl(const char* name, bool overwrite, uint8_t* dst, size_t dst_len,
                                       size_t row_len, const size_t* row_starts, size_t nrows,
                                       const fgfc_plan* plan, const fgfc_slice* srcs, size_t nsrcs,
                                       fgfc_stream stream) {
  fgfc_status st;
  if (!plan) return fail(FGFC_ERR_ARG, "%s: null plan", name);
  if (!check_scattered_rows(plan->field, name, dst_len, row_len, row_starts, nrows, &st)) return st;
  if (plan->rows != nsrcs || plan->cols != nrows)
    return fail(FGFC_ERR_PLAN_DIMS, "%s: plan dimensions do not match (sources, rows)", name);
  if (nsrcs && !srcs) return fail(FGFC_ERR_ARG, "%s: null sources", name);
  for (size_t i = 0; i < nsrcs; ++i)
    if (srcs[i].len != row_len)
      return fail(FGFC_ERR_SOURCE, "%s: source %zu is %zu bytes, expected %zu", name, i, srcs[i].len,
                  row_len);
  if (nrows == 0 || (nsrcs == 0 && !overwrite)) return ok();
  std::vector<const uint8_t*> sp(nsrcs);
  for (size_t i = 0; i < nsrcs; ++i) sp[i] = srcs[i].ptr;
  std::vector<uint8_t*> rp(nrows);
  for (size_t j = 0; j < nrows; ++j) rp[j] = dst + row_starts[j];
  return run_matrix(plan->field, sp.data(), nsrcs, rp.data(), nrows, plan_mat(plan), row_len, overwrite,
                    stream, name);
}

fgfc_status fgfc_mul_add_matrix_scattered_with(uint8_t* dst, size_t dst_len, size_t row_len,
                                               const size_t* row_starts, size_t nrows,
                                               const fgfc_plan* plan, const fgfc_slice* srcs,
                                               size_t nsrcs, fgfc_stream stream) {
  return scattered_plan_impl("mul_add_matrix_scattered_with", false, dst, dst_len, row_len, row_starts, nrows,
                             plan, srcs, nsrcs, stream);
}

fgfc_status fgfc_dot_product_matrix_scattered_with(uint8_t* dst, size_t dst_len, size_t row_len,
                                                   const size_t* row_starts, size_t nrows,
                                                   const fgfc_plan* plan, const fgfc_slice* srcs,
                                                   size_t nsrcs, fgfc_stream stream) {
  return scattered_plan_impl("dot_product_matrix_scattered_with", true, dst, dst_len, row_len, row_starts,
                             nrows, plan, srcs, nsrcs, stream);
}

}  // extern "C"

// ---------------------------------------------------------------- batches

struct fgfc_batch {
  void* state;
};

namespace fgfc {

namespace {

// One stripe (all sources of a plan, rows at the given device addresses) as
// table sub-jobs of at most 4 groups. The vector body is used when every
// source has the same offset within 16 bytes (a multiple of the element
// size), whatever the rows' offsets; otherwise the whole stripe takes the
// 4-byte-group path.
void lower_tables(const fgfc_plan* plan, const std::vector<uint64_t>& srcs, const std::vector<uint64_t>& dsts,
                  size_t row_len, bool overwrite, std::vector<LoweredJob>& out) {
  const int field = plan->field;
  const int E = field_bytes(field);
  const int R = 4 / E;
  const size_t nrows = dsts.size();
  const uintptr_t al = srcs.empty() ? 0 : (srcs[0] & 15);
  bool same = (al % E) == 0;
  for (uint64_t p : srcs) same = same && (p & 15) == al;
  uint64_t head = row_len, nvec = 0;
  if (same) {
    head = std::min<uint64_t>((16 - al) & 15, row_len);
    nvec = (row_len - head) / 16;
  }
  const size_t gtot = (nrows + R - 1) / R;
  for (size_t g0 = 0; g0 < gtot; g0 += 4) {
    const size_t nr = std::min<size_t>(nrows - g0 * R, 4 * R);
    // FGFC_GF16_HALF=0 in the environment (read once) keeps every Gf16
    // sub-job on the Gf16 tables, for A/B runs
    static const bool half_on = [] {
      const char* v = std::getenv("FGFC_GF16_HALF");
      return !(v && v[0] == '0');
    }();
    if (half_on && E == 2 && plan->k16_groups && (nr % 4 == 0 || nr % 4 == 3)) {
      // 3, 4, 7 or 8 rows: byte half-products take 6 lookups per element and
      // 4 rows where the Gf16 tables take 8 (1 or 2 rows: more; 5 or 6: the same)
      LoweredJob L;
      L.field = field;
      L.kara = true;
      L.tables = plan->dev + plan->off_k16;
      L.gstride = plan->k16_groups;
      L.g0 = g0 * R / 4;
      L.G = (nr + 3) / 4;
      L.len = row_len;
      L.head = head;
      L.nvec = nvec;
      L.k = srcs.size();
      L.nrows = nr;
      L.ovr = overwrite;
      L.srcs = srcs;
      L.dsts.assign(dsts.begin() + g0 * R, dsts.begin() + g0 * R + nr);
      L.shift = false;
      if (same && nvec)
        for (uint64_t d : L.dsts) L.shift = L.shift || (d & 15) != al;
      out.push_back(std::move(L));
      continue;
    }
    LoweredJob L;
    L.field = field;
    L.tables = plan->dev + plan->off_mat;
    L.gstride = plan->mat_groups;
    L.g0 = g0;
    L.G = std::min<size_t>(4, gtot - g0);
    L.len = row_len;
    L.head = head;
    L.nvec = nvec;
    L.k = srcs.size();
    L.nrows = std::min(nrows - g0 * R, L.G * R);
    L.ovr = overwrite;
    L.srcs = srcs;
    L.dsts.assign(dsts.begin() + g0 * R, dsts.begin() + g0 * R + L.nrows);
    L.shift = false;
    if (same && nvec)
      for (uint64_t d : L.dsts) L.shift = L.shift || (d & 15) != al;
    out.push_back(std::move(L));
  }
}

std::vector<uint64_t> offset_by(const std::vector<uint64_t>& p, uint64_t off) {
  std::vector<uint64_t> out(p);
  for (auto& x : out) x += off;
  return out;
}

}  // namespace

void lower_matrix_job(const fgfc_plan* plan, const std::vector<uint64_t>& srcs, const std::vector<uint64_t>& dsts,
                      size_t row_len, bool overwrite, std::vector<LoweredJob>& out, std::vector<Gf2Job>& tc) {
  const int field = plan->field;
  const int E = field_bytes(field);
  const size_t k = srcs.size(), m = dsts.size();
  const size_t blk_bytes = 512 * static_cast<size_t>(E);
  if (k && m && !plan->bits_mat.empty() && choose_kernel(field, k, m, row_len) == FGFC_KERNEL_GF2MMA) {
    const uint64_t al = srcs[0] & 15;
    bool same = al % E == 0;
    for (uint64_t p : srcs) same = same && (p & 15) == al;
    for (uint64_t p : dsts) same = same && (p & 15) == al;
    const uint64_t head = std::min<uint64_t>((16 - al) & 15, row_len);
    const uint64_t nblk = same ? (row_len - head) / blk_bytes : 0;
    if (nblk) {
      Gf2Job J;
      J.field = field;
      J.bits = plan->bits_mat.data();
      J.bits_key = plan->bits_key;
      J.k = k;
      J.m = m;
      J.ovr = overwrite;
      J.nblk = nblk;
      J.ptrs = offset_by(srcs, head);
      const std::vector<uint64_t> d = offset_by(dsts, head);
      J.ptrs.insert(J.ptrs.end(), d.begin(), d.end());
      tc.push_back(std::move(J));
      if (head) lower_tables(plan, srcs, dsts, head, overwrite, out);
      const uint64_t end = head + nblk * blk_bytes;
      if (end < row_len) lower_tables(plan, offset_by(srcs, end), offset_by(dsts, end), row_len - end, overwrite, out);
      return;
    }
  }
  lower_tables(plan, srcs, dsts, row_len, overwrite, out);
}

}  // namespace fgfc

extern "C" {

fgfc_status fgfc_batch_create(fgfc_batch** out) {
  if (!out) return fail(FGFC_ERR_ARG, "batch: null argument");
  *out = new fgfc_batch{batch_state_create()};
  return ok();
}

void fgfc_batch_destroy(fgfc_batch* batch) {
  if (!batch) return;
  batch_state_destroy(batch->state);
  delete batch;
}

fgfc_status fgfc_batch_set_graphs(fgfc_batch* batch, int enable) {
  if (!batch) return fail(FGFC_ERR_ARG, "batch: null batch");
  batch_state_graphs(batch->state, enable != 0);
  return ok();
}

fgfc_status fgfc_batch_stats(const fgfc_batch* batch, size_t* launches, size_t* items,
                             int* graph_replayed) {
  if (!batch) return fail(FGFC_ERR_ARG, "batch: null batch");
  batch_state_stats(batch->state, launches, items, graph_replayed);
  return ok();
}

// Every job is validated exactly as the single call it stands for
// (src/ops.rs:720-867 contiguous, 887-941 scattered), then lowered to
// sub-jobs of at most 4 table groups.
fgfc_status fgfc_batch_run(fgfc_batch* batch, const fgfc_matrix_job* jobs, size_t njobs,
                           fgfc_stream stream) {
  if (!batch || (njobs && !jobs)) return fail(FGFC_ERR_ARG, "batch: null argument");
  std::vector<LoweredJob> low;
  std::vector<Gf2Job> tc;
  low.reserve(njobs);
  for (size_t i = 0; i < njobs; ++i) {
    const fgfc_matrix_job& J = jobs[i];
    const char* name = J.row_starts ? (J.overwrite ? "dot_product_matrix_scattered_with"
                                                   : "mul_add_matrix_scattered_with")
                                    : (J.overwrite ? "dot_product_matrix_with" : "mul_add_matrix_with");
    fgfc_status st;
    const fgfc_plan* plan = J.plan;
    if (!plan) return fail(FGFC_ERR_ARG, "batch job %zu: %s: null plan", i, name);
    const int field = plan->field;
    if (J.row_starts) {
      if (!check_scattered_rows(field, name, J.dst_len, J.row_len, J.row_starts, J.nrows, &st)) {
        t_err = "batch job " + std::to_string(i) + ": " + t_err;
        return st;
      }
    } else {
      if (!check_width(field, name, J.row_len, &st)) {
        t_err = "batch job " + std::to_string(i) + ": " + t_err;
        return st;
      }
      size_t used;
      if (mul_overflows(J.nrows, J.row_len, &used))
        return fail(FGFC_ERR_OVERFLOW, "batch job %zu: %s: row geometry overflows", i, name);
      if (J.dst_len < used)
        return fail(FGFC_ERR_ROWS, "batch job %zu: %s: rows is %zu bytes but %zu rows of %zu bytes need %zu",
                    i, name, J.dst_len, J.nrows, J.row_len, used);
    }
    if (plan->rows != J.nsrcs || plan->cols != J.nrows)
      return fail(FGFC_ERR_PLAN_DIMS, "batch job %zu: %s: plan dimensions do not match (sources, rows)", i,
                  name);
    if (J.nsrcs && !J.srcs) return fail(FGFC_ERR_ARG, "batch job %zu: %s: null sources", i, name);
    for (size_t t = 0; t < J.nsrcs; ++t)
      if (J.srcs[t].len != J.row_len)
        return fail(FGFC_ERR_SOURCE, "batch job %zu: %s: source %zu is %zu bytes, expected %zu", i, name, t,
                    J.srcs[t].len, J.row_len);
    if (J.nrows == 0 || J.row_len == 0) continue;
    if (J.nsrcs == 0) {
      if (J.overwrite) {  // an empty sum overwrites with zero
        for (size_t j = 0; j < J.nrows; ++j) {
          cudaError_t e =
              cudaMemsetAsync(J.dst + (J.row_starts ? J.row_starts[j] : j * J.row_len), 0, J.row_len, stream);
          if (e != cudaSuccess) return cuda_fail(e, name);
        }
      }
      continue;
    }
    if (field_bytes(field) == 8) {  // 8-byte fields have their own kernel: one launch per stripe
      std::vector<uint8_t*> rp(J.nrows);
      for (size_t j = 0; j < J.nrows; ++j) rp[j] = J.dst + (J.row_starts ? J.row_starts[j] : j * J.row_len);
      std::vector<const uint8_t*> sp(J.nsrcs);
      for (size_t t = 0; t < J.nsrcs; ++t) sp[t] = J.srcs[t].ptr;
      st = run_matrix(field, sp.data(), J.nsrcs, rp.data(), J.nrows, plan_mat(plan), J.row_len, J.overwrite != 0,
                      stream, name);
      if (st != FGFC_OK) {
        t_err = "batch job " + std::to_string(i) + ": " + t_err;
        return st;
      }
      continue;
    }
    std::vector<uint64_t> dsts(J.nrows);
    for (size_t j = 0; j < J.nrows; ++j)
      dsts[j] = reinterpret_cast<uint64_t>(J.dst + (J.row_starts ? J.row_starts[j] : j * J.row_len));
    std::vector<uint64_t> srcs(J.nsrcs);
    for (size_t t = 0; t < J.nsrcs; ++t) srcs[t] = reinterpret_cast<uint64_t>(J.srcs[t].ptr);
    lower_matrix_job(plan, srcs, dsts, J.row_len, J.overwrite != 0, low, tc);
  }
  cudaError_t e = batch_run(batch->state, low, tc, stream);
  return e == cudaSuccess ? ok() : cuda_fail(e, "batch");
}

// Tile shapes measured on one submission. A timing is the minimum over 3
// reps of one submission, each enqueued right behind an untimed one, so the
// host's lowering of the timed submission overlaps the device's work and
// the events bracket device time only.
fgfc_status fgfc_tune_batch_tiles(fgfc_batch* batch, const fgfc_matrix_job* jobs, size_t njobs, fgfc_stream stream,
                                  double* us_before, double* us_after) {
  if (!batch || (njobs && !jobs)) return fail(FGFC_ERR_ARG, "tune_batch_tiles: null argument");
  fgfc_status st = fgfc_batch_run(batch, jobs, njobs, stream);  // validates; records the classes
  if (st != FGFC_OK) return st;
  const std::vector<std::pair<int, int>> classes = batch_state_classes(batch->state);
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  double best_total = 0;
  const auto time_us = [&](double* out) -> fgfc_status {
    double best = 1e300;
    for (int rep = 0; rep < 3; ++rep) {
      fgfc_status s2 = fgfc_batch_run(batch, jobs, njobs, stream);
      if (s2 == FGFC_OK && cudaEventRecord(e0, stream) != cudaSuccess) s2 = fail(FGFC_ERR_CUDA, "tune_batch_tiles: event");
      if (s2 == FGFC_OK) s2 = fgfc_batch_run(batch, jobs, njobs, stream);
      if (s2 == FGFC_OK && (cudaEventRecord(e1, stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess))
        s2 = fail(FGFC_ERR_CUDA, "tune_batch_tiles: event");
      if (s2 != FGFC_OK) return s2;
      float ms = 0;
      cudaEventElapsedTime(&ms, e0, e1);
      best = std::min(best, 1e3 * static_cast<double>(ms));
    }
    *out = best;
    return FGFC_OK;
  };
  if (e != cudaSuccess) st = cuda_fail(e, "tune_batch_tiles");
  if (st == FGFC_OK) st = time_us(&best_total);
  if (st == FGFC_OK && us_before) *us_before = best_total;
  // one class at a time, the others at their current tiles
  for (size_t ci = 0; ci < classes.size() && st == FGFC_OK; ++ci) {
    const int E = classes[ci].first, G = classes[ci].second;
    const int start = tile_cols(E, G);
    int best_cols = start;
    for (int cols : {1, 2, 4, 8, 16}) {
      if (cols == start) continue;
      set_tile_cols(E, G, cols, 0.0);
      double us = 0;
      st = time_us(&us);
      if (st != FGFC_OK) break;
      if (us < best_total * 0.98) {  // a clear win only
        best_total = us;
        best_cols = cols;
      }
    }
    set_tile_cols(E, G, best_cols, best_total);
  }
  if (st == FGFC_OK) st = time_us(&best_total);
  if (st == FGFC_OK && us_after) *us_after = best_total;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  return st == FGFC_OK ? ok() : st;
}

fgfc_status fgfc_run_jobs_serial(const fgfc_matrix_job* jobs, size_t njobs, fgfc_stream stream) {
  if (njobs && !jobs) return fail(FGFC_ERR_ARG, "batch: null argument");
  for (size_t i = 0; i < njobs; ++i) {
    const fgfc_matrix_job& J = jobs[i];
    fgfc_status st;
    if (J.row_starts) {
      st = J.overwrite ? fgfc_dot_product_matrix_scattered_with(J.dst, J.dst_len, J.row_len, J.row_starts,
                                                                J.nrows, J.plan, J.srcs, J.nsrcs, stream)
                       : fgfc_mul_add_matrix_scattered_with(J.dst, J.dst_len, J.row_len, J.row_starts, J.nrows,
                                                            J.plan, J.srcs, J.nsrcs, stream);
    } else if (J.overwrite) {
      st = fgfc_dot_product_matrix_with(J.dst, J.dst_len, J.row_len, J.nrows, J.plan, J.srcs, J.nsrcs, stream);
    } else {
      st = fgfc_mul_add_matrix_with(J.dst, J.dst_len, J.row_len, J.nrows, J.plan, J.srcs, J.nsrcs, stream);
    }
    if (st != FGFC_OK) {
      t_err = "batch job " + std::to_string(i) + ": " + t_err;
      return st;
    }
  }
  return ok();
}

// Same per-job rules as fgfc_batch_run, with the raw coefficient forms'
// names; the limits of the fixed scratch are checked by noalloc_run before
// anything is issued. Nothing is allocated on success.
fgfc_status fgfc_batch_run_noalloc(fgfc_field field, const fgfc_noalloc_job* jobs, size_t njobs,
                                   fgfc_stream stream) {
  if (!valid_field(field) || (njobs && !jobs)) return fail(FGFC_ERR_ARG, "batch_run_noalloc: invalid argument");
  if (field_bytes(field) > 4)
    return fail(FGFC_ERR_LIMIT, "batch_run_noalloc: %s has 8-byte elements; this entry point takes 1-, 2- and "
                "4-byte fields", field_name(field));
  for (size_t i = 0; i < njobs; ++i) {
    const fgfc_noalloc_job& J = jobs[i];
    const char* name =
        J.row_starts ? "mul_add_matrix_scattered" : (J.overwrite ? "dot_product_matrix" : "mul_add_matrix");
    fgfc_status st;
    if (J.row_starts) {
      if (J.overwrite)
        return fail(FGFC_ERR_ARG, "batch job %zu: scattered rows accumulate; overwrite is not defined", i);
      if (!check_scattered_rows(field, name, J.dst_len, J.row_len, J.row_starts, J.nrows, &st)) {
        t_err = "batch job " + std::to_string(i) + ": " + t_err;
        return st;
      }
    } else {
      if (!check_width(field, name, J.row_len, &st)) {
        t_err = "batch job " + std::to_string(i) + ": " + t_err;
        return st;
      }
      size_t used;
      if (mul_overflows(J.nrows, J.row_len, &used))
        return fail(FGFC_ERR_OVERFLOW, "batch job %zu: %s: row geometry overflows", i, name);
      if (J.dst_len < used)
        return fail(FGFC_ERR_ROWS, "batch job %zu: %s: rows is %zu bytes but %zu rows of %zu bytes need %zu",
                    i, name, J.dst_len, J.nrows, J.row_len, used);
    }
    if (J.nsrcs && !J.srcs) return fail(FGFC_ERR_ARG, "batch job %zu: %s: null sources", i, name);
    if (J.nsrcs && J.nrows && !J.coeffs) return fail(FGFC_ERR_ARG, "batch job %zu: %s: null coefficients", i, name);
    for (size_t t = 0; t < J.nsrcs; ++t)
      if (J.srcs[t].len != J.row_len)
        return fail(FGFC_ERR_SOURCE, "batch job %zu: %s: source %zu is %zu bytes, expected %zu", i, name, t,
                    J.srcs[t].len, J.row_len);
  }
  char msg[256];
  const int st = noalloc_run(field, jobs, njobs, stream, msg, sizeof msg);
  return st == 0 ? ok() : fail(static_cast<fgfc_status>(st), "%s", msg);
}

}  // extern "C"

// ---------------------------------------------------------------- shared with serve.cpp

namespace fgfc {

fgfc_status set_error(fgfc_status st, const char* msg) {
  t_err = msg;
  return st;
}

fgfc_status clear_error() { return ok(); }

const char* last_error_text() { return t_err.c_str(); }

// The checks fgfc_batch_run applies to one job, for a job whose buffers are
// host memory (the serving loop's requests): name is the ops function it
// stands for.
fgfc_status validate_matrix_call(int field, const char* name, size_t dst_len, size_t row_len,
                                 const size_t* row_starts, size_t nrows, const fgfc_slice* srcs, size_t nsrcs,
                                 const uint32_t* coeffs, int overwrite) {
  fgfc_status st;
  if (!valid_field(field)) return fail(FGFC_ERR_ARG, "%s: unknown field", name);
  if (row_starts) {
    if (!check_scattered_rows(field, name, dst_len, row_len, row_starts, nrows, &st)) return st;
  } else {
    if (!check_width(field, name, row_len, &st)) return st;
    size_t used;
    if (mul_overflows(nrows, row_len, &used)) return fail(FGFC_ERR_OVERFLOW, "%s: row geometry overflows", name);
    if (dst_len < used)
      return fail(FGFC_ERR_ROWS, "%s: rows is %zu bytes but %zu rows of %zu bytes need %zu", name, dst_len, nrows,
                  row_len, used);
  }
  if (nsrcs && !srcs) return fail(FGFC_ERR_ARG, "%s: null sources", name);
  if (nsrcs && nrows && !coeffs) return fail(FGFC_ERR_ARG, "%s: null coefficients", name);
  for (size_t t = 0; t < nsrcs; ++t)
    if (srcs[t].len != row_len)
      return fail(FGFC_ERR_SOURCE, "%s: source %zu is %zu bytes, expected %zu", name, t, srcs[t].len, row_len);
  return ok();
}

}  // namespace fgfc
