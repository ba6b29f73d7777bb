// tune.cpp -- which kernel family computes a matrix call.
//
// The reference routes each call by shape once its CPU backend is known
// (blocked vs AXPY paths, src/kernel/gf16.rs:419-460; backend detection,
// src/kernel/mod.rs:147-184). Here the families are the split-nibble table
// kernels (every shape), the byte-table kernels (Gf8, one 4-row group, at most
// 14 sources) and the bit-sliced GF(2) contraction on the tensor cores
// (gf2mma.cu). The choice for a (field, sources, rows, row-length bucket)
// comes from, in order: a process-wide override for A/B runs
// (fgfc_tune_force, or FGFC_KERNEL=nibble|byte|gf2mma in the environment,
// read once), a table of measured winners (fgfc_tune_shape, persisted with
// fgfc_tune_save / fgfc_tune_load as JSON), and built-in rules measured on
// B200. A family that cannot run a shape is never chosen for it.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "internal.hpp"

namespace fgfc {

namespace {

std::mutex g_mu;
int g_force = -1;  // -1: environment not read yet

struct TuneKey {
  int field;
  uint32_t k, m, lb;
  bool operator<(const TuneKey& o) const {
    return std::tie(field, k, m, lb) < std::tie(o.field, o.k, o.m, o.lb);
  }
};

struct TuneVal {
  int kernel;
  double us;
};

std::map<TuneKey, TuneVal> g_table;

// Tile shape of the batched nibble work lists: element-vector columns per
// thread per work item, by (element width, table groups); 0 = built-in.
// FGFC_TILE_COLS=n in the environment (read once) overrides every class.
struct TileVal {
  int cols;
  double us;
};
std::map<std::pair<int, int>, TileVal> g_tiles;
int g_tile_env = -1;  // -1: environment not read yet, 0: unset

bool tile_ok(int cols) { return cols == 1 || cols == 2 || cols == 4 || cols == 8 || cols == 16; }

int tile_env_locked() {
  if (g_tile_env < 0) {
    const char* v = std::getenv("FGFC_TILE_COLS");
    const int n = v ? std::atoi(v) : 0;
    g_tile_env = tile_ok(n) ? n : 0;
  }
  return g_tile_env;
}

uint32_t len_bucket(size_t len) {  // floor(log2(len)), 0 for 0
  uint32_t b = 0;
  while (len > 1) {
    len >>= 1;
    ++b;
  }
  return b;
}

const char* kernel_name(int k) {
  switch (k) {
    case FGFC_KERNEL_NIBBLE: return "nibble";
    case FGFC_KERNEL_BYTE: return "byte";
    case FGFC_KERNEL_GF2MMA: return "gf2mma";
    default: return "auto";
  }
}

int kernel_from_name(const char* s) {
  if (!s) return FGFC_KERNEL_AUTO;
  if (!std::strcmp(s, "nibble")) return FGFC_KERNEL_NIBBLE;
  if (!std::strcmp(s, "byte")) return FGFC_KERNEL_BYTE;
  if (!std::strcmp(s, "gf2mma")) return FGFC_KERNEL_GF2MMA;
  return FGFC_KERNEL_AUTO;
}

int forced_locked() {
  if (g_force < 0) g_force = kernel_from_name(std::getenv("FGFC_KERNEL"));
  return g_force;
}

// Built-in rules (B200 measurements of dot_product_matrix over 1 and 4 MiB
// rows, every field, k * E in {4 .. 64} bytes, m * E in {1 .. 16} bytes):
// byte tables reach the HBM roofline for their shapes once a row is long
// enough to amortise the 1.5 us table fill; the tensor-core contraction
// wins where a column carries the most output it takes (m * E = 16 bytes)
// from at least 32 input bytes (Gf8 RS(64,16), Gf16 RS(16..32,8), Gf32
// RS(8..16,4): 1.1 - 1.6x the split-nibble kernel, whose lookups per output
// bit cost the most there).
int builtin_choice(int field, size_t k, size_t m, size_t len) {
  const size_t E = static_cast<size_t>(field_bytes(field));
  if (kernel_usable(FGFC_KERNEL_BYTE, field, k, m) && len >= (4u << 20)) return FGFC_KERNEL_BYTE;
  if (kernel_usable(FGFC_KERNEL_GF2MMA, field, k, m) && len >= (1u << 20) && E * m >= 16 && E * k >= 32)
    return FGFC_KERNEL_GF2MMA;
  return FGFC_KERNEL_NIBBLE;
}

}  // namespace

bool kernel_usable(int kernel, int field, size_t k, size_t m) {
  const int E = field_bytes(field);
  switch (kernel) {
    case FGFC_KERNEL_NIBBLE: return E > 0;
    case FGFC_KERNEL_BYTE: return E == 1 && k >= 1 && k <= static_cast<size_t>(kFastMaxSources) && m >= 1 && m <= 4;
    case FGFC_KERNEL_GF2MMA: return gf2mma_shape_ok(field, k, m);
    default: return false;
  }
}

int choose_kernel(int field, size_t k, size_t m, size_t len) {
  std::lock_guard<std::mutex> lk(g_mu);
  const int f = forced_locked();
  if (f != FGFC_KERNEL_AUTO && kernel_usable(f, field, k, m)) return f;
  const auto it = g_table.find(TuneKey{field, static_cast<uint32_t>(k), static_cast<uint32_t>(m), len_bucket(len)});
  if (it != g_table.end() && kernel_usable(it->second.kernel, field, k, m)) return it->second.kernel;
  return builtin_choice(field, k, m, len);
}

int tile_cols(int E, int G) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (const int env = tile_env_locked()) return env;
  const auto it = g_tiles.find({E, G});
  return it != g_tiles.end() ? it->second.cols : kTileColsDefault;
}

void set_tile_cols(int E, int G, int cols, double us) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (cols == 0)
    g_tiles.erase({E, G});
  else
    g_tiles[{E, G}] = TileVal{cols, us};
}

}  // namespace fgfc

using namespace fgfc;

extern "C" {

fgfc_status fgfc_tune_force(fgfc_kernel kernel) {
  if (kernel < FGFC_KERNEL_AUTO || kernel > FGFC_KERNEL_GF2MMA)
    return set_error(FGFC_ERR_ARG, "tune_force: unknown kernel family");
  std::lock_guard<std::mutex> lk(g_mu);
  g_force = kernel;
  return clear_error();
}

fgfc_kernel fgfc_tune_choice(fgfc_field field, size_t nsrcs, size_t nrows, size_t row_len) {
  if (field_bytes(field) == 0) return FGFC_KERNEL_AUTO;
  return static_cast<fgfc_kernel>(choose_kernel(field, nsrcs, nrows, row_len));
}

int fgfc_tune_usable(fgfc_kernel kernel, fgfc_field field, size_t nsrcs, size_t nrows) {
  return kernel_usable(kernel, field, nsrcs, nrows) ? 1 : 0;
}

// Time every usable family on this shape (device buffers allocated here and
// freed before returning; row_len bytes per source and row), on the current
// device, and record the fastest for the shape's row-length bucket.
fgfc_status fgfc_tune_shape(fgfc_field field, size_t nsrcs, size_t nrows, size_t row_len, fgfc_kernel* out) {
  const int E = field_bytes(field);
  if (!E || !nsrcs || !nrows || !row_len || row_len % E)
    return set_error(FGFC_ERR_ARG, "tune_shape: invalid shape");
  std::vector<uint32_t> coeffs(nsrcs * nrows);
  uint32_t x = 0x9E3779B9u;
  for (auto& c : coeffs) {  // nonzero pseudo-random coefficients
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    c = (x & field_mask(field)) | 1u;
  }
  fgfc_plan* plan = nullptr;
  fgfc_status st = fgfc_plan_create(field, nsrcs, nrows, coeffs.data(), &plan);
  if (st != FGFC_OK) return st;
  uint8_t* buf = nullptr;
  cudaError_t e = cudaMalloc(&buf, (nsrcs + nrows) * row_len);
  if (e != cudaSuccess) {
    fgfc_plan_destroy(plan);
    return set_error(FGFC_ERR_NOMEM, "tune_shape: device allocation failed");
  }
  cudaMemset(buf, 0x5A, nsrcs * row_len);
  std::vector<fgfc_slice> srcs(nsrcs);
  for (size_t t = 0; t < nsrcs; ++t) srcs[t] = fgfc_slice{buf + t * row_len, row_len};
  uint8_t* rows = buf + nsrcs * row_len;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  int prev;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    prev = forced_locked();
  }
  int best = FGFC_KERNEL_NIBBLE;
  double best_us = 1e300;
  for (int kern : {FGFC_KERNEL_NIBBLE, FGFC_KERNEL_BYTE, FGFC_KERNEL_GF2MMA}) {
    if (!kernel_usable(kern, field, nsrcs, nrows)) continue;
    {
      std::lock_guard<std::mutex> lk(g_mu);
      g_force = kern;
    }
    const int reps = 5;
    fgfc_status rs = FGFC_OK;
    for (int i = 0; i < 2 && rs == FGFC_OK; ++i)
      rs = fgfc_dot_product_matrix_with(rows, nrows * row_len, row_len, nrows, plan, srcs.data(), nsrcs, s);
    cudaEventRecord(e0, s);
    for (int i = 0; i < reps && rs == FGFC_OK; ++i)
      rs = fgfc_dot_product_matrix_with(rows, nrows * row_len, row_len, nrows, plan, srcs.data(), nsrcs, s);
    cudaEventRecord(e1, s);
    cudaEventSynchronize(e1);
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    if (rs != FGFC_OK) continue;
    const double us = 1e3 * ms / reps;
    if (us < best_us) {
      best_us = us;
      best = kern;
    }
  }
  {
    std::lock_guard<std::mutex> lk(g_mu);
    g_force = prev;
    g_table[TuneKey{field, static_cast<uint32_t>(nsrcs), static_cast<uint32_t>(nrows), len_bucket(row_len)}] =
        TuneVal{best, best_us};
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  cudaStreamDestroy(s);
  cudaFree(buf);
  fgfc_plan_destroy(plan);
  if (out) *out = static_cast<fgfc_kernel>(best);
  return clear_error();
}

fgfc_status fgfc_tune_set_tile(size_t elem_bytes, size_t groups, unsigned cols) {
  if ((elem_bytes != 1 && elem_bytes != 2 && elem_bytes != 4) || groups < 1 || groups > 4 ||
      (cols != 0 && !tile_ok(static_cast<int>(cols))))
    return set_error(FGFC_ERR_ARG, "tune_set_tile: invalid class or tile (columns 1, 2, 4, 8, 16 or 0)");
  set_tile_cols(static_cast<int>(elem_bytes), static_cast<int>(groups), static_cast<int>(cols), 0.0);
  return clear_error();
}

unsigned fgfc_tune_tile(size_t elem_bytes, size_t groups) {
  return static_cast<unsigned>(tile_cols(static_cast<int>(elem_bytes), static_cast<int>(groups)));
}

fgfc_status fgfc_tune_save(const char* path) {
  if (!path) return set_error(FGFC_ERR_ARG, "tune_save: null path");
  std::lock_guard<std::mutex> lk(g_mu);
  FILE* f = std::fopen(path, "w");
  if (!f) return set_error(FGFC_ERR_ARG, "tune_save: cannot open file");
  std::fprintf(f, "{\"version\": 1, \"entries\": [");
  bool first = true;
  for (const auto& kv : g_table) {
    std::fprintf(f, "%s\n  {\"field\": %d, \"k\": %u, \"m\": %u, \"len_log2\": %u, \"kernel\": \"%s\", \"us\": %.3f}",
                 first ? "" : ",", kv.first.field, kv.first.k, kv.first.m, kv.first.lb, kernel_name(kv.second.kernel),
                 kv.second.us);
    first = false;
  }
  std::fprintf(f, "\n], \"tiles\": [");
  first = true;
  for (const auto& kv : g_tiles) {
    std::fprintf(f, "%s\n  {\"elem_bytes\": %d, \"groups\": %d, \"cols\": %d, \"us\": %.3f}", first ? "" : ",",
                 kv.first.first, kv.first.second, kv.second.cols, kv.second.us);
    first = false;
  }
  std::fprintf(f, "\n]}\n");
  std::fclose(f);
  return clear_error();
}

// Reads the format fgfc_tune_save writes: one entry object per line.
fgfc_status fgfc_tune_load(const char* path) {
  if (!path) return set_error(FGFC_ERR_ARG, "tune_load: null path");
  FILE* f = std::fopen(path, "r");
  if (!f) return set_error(FGFC_ERR_ARG, "tune_load: cannot open file");
  char line[512];
  std::map<TuneKey, TuneVal> got;
  std::map<std::pair<int, int>, TileVal> tiles;
  while (std::fgets(line, sizeof line, f)) {
    int field;
    unsigned k, m, lb;
    char kern[32];
    double us;
    const char* p = std::strchr(line, '{');
    if (!p || std::strstr(line, "\"version\"")) continue;
    int te, tg, tc;
    if (std::sscanf(p, " {\"elem_bytes\": %d, \"groups\": %d, \"cols\": %d, \"us\": %lf", &te, &tg, &tc, &us) == 4) {
      if ((te == 1 || te == 2 || te == 4) && tg >= 1 && tg <= 4 && tile_ok(tc)) tiles[{te, tg}] = TileVal{tc, us};
      continue;
    }
    if (std::sscanf(p, " {\"field\": %d, \"k\": %u, \"m\": %u, \"len_log2\": %u, \"kernel\": \"%31[a-z0-9]\", \"us\": %lf",
                    &field, &k, &m, &lb, kern, &us) == 6) {
      const int kk = kernel_from_name(kern);
      if (field_bytes(field) && kk != FGFC_KERNEL_AUTO) got[TuneKey{field, k, m, lb}] = TuneVal{kk, us};
    }
  }
  std::fclose(f);
  std::lock_guard<std::mutex> lk(g_mu);
  for (const auto& kv : got) g_table[kv.first] = kv.second;
  for (const auto& kv : tiles) g_tiles[kv.first] = kv.second;
  return clear_error();
}

void fgfc_tune_clear(void) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_table.clear();
  g_tiles.clear();
}

}  // extern "C"
