// serve.cpp -- the serving loop of libfgfcuda.so (fgfc_server_*).
//
// Requests are single matrix calls over host buffers. One worker thread per
// server owns three streams and runs this loop:
//   admit   -- take pending requests in arrival order while the launch's
//              device block and staging block still fit (the HBM budget is
//              one device arena, the staging area one page-locked arena);
//   issue   -- copy staged inputs into page-locked memory, send them with one
//              host-to-device copy (direct requests row by row), run every
//              admitted request as one submission of the batch work-list
//              kernel, and queue the device-to-host copy of all results;
//   retire  -- when a launch's last copy has landed (its event on the
//              copy-out stream, polled by the worker), move staged results
//              into the callers' buffers, free the blocks and complete the
//              requests.
// The loop admits new requests while earlier launches are still on the GPU,
// so their copies and kernels overlap (continuous batching). Requests whose
// buffers are all device memory skip the copies and run in place. Plain mode
// runs one request at a time through the per-call entry points instead, for
// comparison.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <list>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/fgf_cuda.h"
#include "internal.hpp"

using namespace fgfc;
using Clock = std::chrono::steady_clock;

namespace {

constexpr size_t kAlign = 256;
constexpr size_t kDirectMin = 256u << 10;  // rows at least this long skip staging when page-locked

size_t up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

// First-fit allocator over [0, size) with coalescing of neighbours.
class Arena {
 public:
  void reset(size_t size) {
    free_.clear();
    if (size) free_[0] = size;
    size_ = size;
    used_ = 0;
  }
  bool alloc(size_t n, size_t* off) {
    if (n == 0) {
      *off = 0;
      return true;
    }
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second < n) continue;
      *off = it->first;
      const size_t rest = it->second - n, o = it->first + n;
      free_.erase(it);
      if (rest) free_[o] = rest;
      used_ += n;
      return true;
    }
    return false;
  }
  void release(size_t off, size_t n) {
    if (n == 0) return;
    used_ -= n;
    auto it = free_.emplace(off, n).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }
  size_t size() const { return size_; }
  size_t used() const { return used_; }

 private:
  std::map<size_t, size_t> free_;
  size_t size_ = 0, used_ = 0;
};

// Page-locked staging copies split over a few host threads: one thread's
// memcpy reaches a fraction of host memory bandwidth, and the worker thread
// must not spend launch time copying.
class CopyPool {
 public:
  struct Copy {
    void* dst;
    const void* src;
    size_t n;
  };
  explicit CopyPool(int nthreads) {
    for (int i = 0; i < nthreads; ++i) th_.emplace_back([this] { loop(); });
  }
  ~CopyPool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  // Runs every copy (split in pieces of at most kPiece bytes) and returns
  // when all are done; the calling thread copies too.
  void run(const std::vector<Copy>& copies) {
    size_t total = 0;
    for (const Copy& c : copies) total += c.n;
    if (total < kParallelMin || th_.empty()) {
      for (const Copy& c : copies) std::memcpy(c.dst, c.src, c.n);
      return;
    }
    std::unique_lock<std::mutex> lk(mu_);
    for (const Copy& c : copies)
      for (size_t o = 0; o < c.n; o += kPiece)
        work_.push_back(Copy{static_cast<uint8_t*>(c.dst) + o, static_cast<const uint8_t*>(c.src) + o,
                             std::min(kPiece, c.n - o)});
    pending_ += work_.size();
    cv_.notify_all();
    while (!work_.empty()) {
      const Copy c = work_.front();
      work_.pop_front();
      lk.unlock();
      std::memcpy(c.dst, c.src, c.n);
      lk.lock();
      --pending_;
    }
    done_cv_.wait(lk, [&] { return pending_ == 0; });
  }

 private:
  static constexpr size_t kPiece = 1u << 20;
  static constexpr size_t kParallelMin = 1u << 20;
  void loop() {
    std::unique_lock<std::mutex> lk(mu_);
    for (;;) {
      cv_.wait(lk, [&] { return stop_ || !work_.empty(); });
      if (stop_ && work_.empty()) return;
      const Copy c = work_.front();
      work_.pop_front();
      lk.unlock();
      std::memcpy(c.dst, c.src, c.n);
      lk.lock();
      if (--pending_ == 0) done_cv_.notify_all();
    }
  }
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, done_cv_;
  std::deque<Copy> work_;
  size_t pending_ = 0;
  bool stop_ = false;
};

struct PlanEntry {
  fgfc_plan* plan = nullptr;
  int field = 0;
  size_t k = 0, m = 0;
  std::vector<uint32_t> coeffs;
  uint64_t key = 0;
  int refs = 0;
  std::list<PlanEntry*>::iterator idle_pos;  // position in the idle list while refs == 0
};

uint64_t fnv1a(uint64_t h, const void* p, size_t n) {
  const uint8_t* b = static_cast<const uint8_t*>(p);
  for (size_t i = 0; i < n; ++i) {
    h ^= b[i];
    h *= 0x100000001b3ull;
  }
  return h;
}

struct Req {
  uint64_t ticket = 0;
  int field = 0;
  size_t k = 0, m = 0, L = 0, Ls = 0;  // sources, rows, row length, device row stride
  bool ovr = false;
  bool direct = false;                 // page-locked buffers with long rows: no staging
  bool on_device = false;              // every buffer is device memory: used in place, no copies
  bool scattered = false;              // row_starts given (mul_add_matrix_scattered)
  size_t dst_len = 0;
  std::vector<uint32_t> coeffs;        // term-major, masked to the field
  std::vector<const uint8_t*> src;
  std::vector<size_t> starts;          // host row offsets into dst
  uint8_t* dst = nullptr;
  uint64_t key = 0;
  PlanEntry* plan = nullptr;
  size_t d_src = 0, d_rows = 0;        // offsets inside the launch's device block
  Clock::time_point t0, t_issue;
  fgfc_status status = FGFC_OK;
  std::string err;
  bool done = false;

  size_t dev_bytes() const { return on_device ? 0 : (k + m) * Ls; }
  size_t stg_bytes() const { return direct || on_device ? 0 : k * Ls + (ovr ? m * Ls : 2 * m * Ls); }
};

struct Launch {
  std::vector<Req*> reqs;
  size_t dev_off = 0, dev_len = 0;  // device arena block
  size_t stg_off = 0, stg_len = 0;  // staging arena block
  size_t in_len = 0;                // staged input image: device [0, in_len) of the block
  size_t out0 = 0, out_len = 0;     // staged results: device [out0, out0 + out_len), staging [in_len, ...)
  cudaEvent_t ev_in = nullptr, ev_done = nullptr, ev_out = nullptr;  // ev_out: the last copy has landed
  bool failed = false;               // issuing stopped early; everything queued has been waited for
  Clock::time_point t_issue;
  cudaError_t err = cudaSuccess;
};

// cudaMemoryTypeHost (page-locked), cudaMemoryTypeDevice (with its device)
// or cudaMemoryTypeUnregistered (pageable).
cudaMemoryType where(const void* p, int* device) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return cudaMemoryTypeUnregistered;
  }
  *device = a.device;
  return a.type;
}

bool host_locked(const void* p) {
  int d = 0;
  return where(p, &d) == cudaMemoryTypeHost;
}

}  // namespace

struct fgfc_server {
  fgfc_server_config cfg{};
  int device = 0;
  cudaStream_t s_in = nullptr, s_run = nullptr, s_out = nullptr;
  uint8_t* dev = nullptr;
  uint8_t* stg = nullptr;
  Arena dev_arena, stg_arena;
  void* batch = nullptr;

  std::mutex mu;
  std::condition_variable cv;       // worker: new work or a landed launch
  std::condition_variable done_cv;  // waiters
  std::deque<Req*> pending;
  std::deque<std::unique_ptr<Launch>> inflight;
  std::unordered_map<uint64_t, std::unique_ptr<Req>> reqs;  // by ticket, until waited for
  uint64_t next_ticket = 1;
  size_t outstanding = 0;  // submitted, not yet completed
  bool stop = false;
  std::thread worker;

  // plan cache (worker thread only): unreferenced plans wait in `idle`,
  // least recently used first, and are evicted from its front
  std::list<PlanEntry> plans;
  std::list<PlanEntry*> idle;
  std::unordered_multimap<uint64_t, PlanEntry*> plan_index;
  std::unique_ptr<CopyPool> copies;
  std::unordered_map<uint64_t, std::vector<uint32_t>> decode_cache;  // rebuild requests (under mu)

  // statistics (under mu)
  std::vector<double> lat_us;
  double queue_sum = 0, launch_sum = 0;
  uint64_t launch_n = 0;
  uint64_t completed = 0, failed = 0, launches = 0, hits = 0, misses = 0, src_bytes = 0, peak_dev = 0,
           max_batch_seen = 0;
  Clock::time_point first_submit, last_done;
  bool have_first = false;

  void run();
  void run_plain(Req* r);
  bool acquire_plan(Req* r);
  void release_plan(Req* r);
  void issue(Launch* L);
  void retire(Launch* L);
  void finish(Req* r, fgfc_status st, const std::string& err);
};

bool fgfc_server::acquire_plan(Req* r) {
  auto range = plan_index.equal_range(r->key);
  for (auto it = range.first; it != range.second; ++it) {
    PlanEntry* e = it->second;
    if (e->field == r->field && e->k == r->k && e->m == r->m && e->coeffs == r->coeffs) {
      if (e->refs++ == 0) idle.erase(e->idle_pos);
      r->plan = e;
      std::lock_guard<std::mutex> lk(mu);
      hits++;
      return true;
    }
  }
  // miss: evict least recently used unreferenced plans beyond the cache size
  while (plans.size() >= cfg.plan_cache && !idle.empty()) {
    PlanEntry* victim = idle.front();
    idle.pop_front();
    auto range2 = plan_index.equal_range(victim->key);
    for (auto it = range2.first; it != range2.second; ++it)
      if (it->second == victim) {
        plan_index.erase(it);
        break;
      }
    fgfc_plan_destroy(victim->plan);
    for (auto it = plans.begin(); it != plans.end(); ++it)
      if (&*it == victim) {
        plans.erase(it);
        break;
      }
  }
  fgfc_plan* p = nullptr;
  if (fgfc_plan_create(static_cast<fgfc_field>(r->field), r->k, r->m, r->coeffs.data(), &p) != FGFC_OK) {
    r->err = last_error_text();
    return false;
  }
  plans.emplace_back();
  PlanEntry& e = plans.back();
  e.plan = p;
  e.field = r->field;
  e.k = r->k;
  e.m = r->m;
  e.coeffs = r->coeffs;
  e.key = r->key;
  e.refs = 1;
  plan_index.emplace(e.key, &e);
  r->plan = &e;
  std::lock_guard<std::mutex> lk(mu);
  misses++;
  return true;
}

void fgfc_server::release_plan(Req* r) {
  PlanEntry* e = r->plan;
  if (e && --e->refs == 0) e->idle_pos = idle.insert(idle.end(), e);
  r->plan = nullptr;
}

// Under mu.
void fgfc_server::finish(Req* r, fgfc_status st, const std::string& err) {
  r->status = st;
  r->err = err;
  r->done = true;
  const auto now = Clock::now();
  if (st == FGFC_OK) {
    completed++;
    src_bytes += r->k * r->L;
    lat_us.push_back(std::chrono::duration<double, std::micro>(now - r->t0).count());
    if (r->t_issue > r->t0) queue_sum += std::chrono::duration<double, std::micro>(r->t_issue - r->t0).count();
  } else {
    failed++;
  }
  last_done = now;
  outstanding--;
  done_cv.notify_all();
}

// Lays out the admitted requests in one device block and one staging block,
// stages inputs, and queues copy-in, kernel and copy-out.
void fgfc_server::issue(Launch* L) {
  // device layout: [staged sources | staged accumulate rows | staged overwrite rows | direct requests]
  auto staged = [](const Req* r) { return !r->direct && !r->on_device; };
  size_t off = 0;
  for (Req* r : L->reqs)
    if (staged(r)) {
      r->d_src = off;
      off += r->k * r->Ls;
    }
  const size_t acc0 = off;
  for (Req* r : L->reqs)
    if (staged(r) && !r->ovr) {
      r->d_rows = off;
      off += r->m * r->Ls;
    }
  for (Req* r : L->reqs)
    if (staged(r) && r->ovr) {
      r->d_rows = off;
      off += r->m * r->Ls;
    }
  const size_t out_end = off;
  for (Req* r : L->reqs)
    if (r->direct) {
      r->d_src = off;
      off += r->k * r->Ls;
      r->d_rows = off;
      off += r->m * r->Ls;
    }
  L->in_len = acc0;
  // accumulate rows are inputs too: the staged input image is device [0, first overwrite row)
  size_t in_end = acc0;
  for (Req* r : L->reqs)
    if (staged(r) && !r->ovr) in_end = std::max(in_end, r->d_rows + r->m * r->Ls);
  L->in_len = in_end;
  L->out0 = acc0;
  L->out_len = out_end - acc0;
  uint8_t* dbase = dev + L->dev_off;
  uint8_t* sbase = stg + L->stg_off;
  uint8_t* sout = sbase + L->in_len;  // staged results: mirror of device [out0, out0 + out_len)

  cudaError_t e = cudaSuccess;
  // stage inputs (CPU copies into page-locked memory, split over the copy
  // threads), then one copy in
  {
    std::vector<CopyPool::Copy> cp;
    for (Req* r : L->reqs) {
      if (!staged(r)) continue;
      for (size_t t = 0; t < r->k; ++t) cp.push_back({sbase + r->d_src + t * r->Ls, r->src[t], r->L});
      if (!r->ovr)
        for (size_t j = 0; j < r->m; ++j) cp.push_back({sbase + r->d_rows + j * r->Ls, r->dst + r->starts[j], r->L});
    }
    copies->run(cp);
  }
  if (L->in_len) e = cudaMemcpyAsync(dbase, sbase, L->in_len, cudaMemcpyHostToDevice, s_in);
  for (Req* r : L->reqs) {
    if (!r->direct || e != cudaSuccess) continue;
    for (size_t t = 0; t < r->k && e == cudaSuccess; ++t)
      e = cudaMemcpyAsync(dbase + r->d_src + t * r->Ls, r->src[t], r->L, cudaMemcpyHostToDevice, s_in);
    if (!r->ovr)
      for (size_t j = 0; j < r->m && e == cudaSuccess; ++j)
        e = cudaMemcpyAsync(dbase + r->d_rows + j * r->Ls, r->dst + r->starts[j], r->L, cudaMemcpyHostToDevice,
                            s_in);
  }
  if (e == cudaSuccess) e = cudaEventRecord(L->ev_in, s_in);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s_run, L->ev_in, 0);

  // one submission of the work-list kernel for every request
  if (e == cudaSuccess) {
    std::vector<LoweredJob> low;
    std::vector<Gf2Job> tc;
    std::vector<uint64_t> sp, dp;
    for (Req* r : L->reqs) {
      sp.resize(r->k);
      dp.resize(r->m);
      for (size_t t = 0; t < r->k; ++t)
        sp[t] = reinterpret_cast<uint64_t>(r->on_device ? r->src[t] : dbase + r->d_src + t * r->Ls);
      for (size_t j = 0; j < r->m; ++j)
        dp[j] = reinterpret_cast<uint64_t>(r->on_device ? r->dst + r->starts[j] : dbase + r->d_rows + j * r->Ls);
      lower_matrix_job(r->plan->plan, sp, dp, r->L, r->ovr, low, tc);
    }
    e = batch_run(batch, low, tc, s_run);
  }
  if (e == cudaSuccess) e = cudaEventRecord(L->ev_done, s_run);
  if (e == cudaSuccess) e = cudaStreamWaitEvent(s_out, L->ev_done, 0);

  // results out: staged ones in one copy, direct ones row by row
  if (e == cudaSuccess && L->out_len)
    e = cudaMemcpyAsync(sout, dbase + L->out0, L->out_len, cudaMemcpyDeviceToHost, s_out);
  for (Req* r : L->reqs) {
    if (!r->direct || e != cudaSuccess) continue;
    for (size_t j = 0; j < r->m && e == cudaSuccess; ++j)
      e = cudaMemcpyAsync(r->dst + r->starts[j], dbase + r->d_rows + j * r->Ls, r->L, cudaMemcpyDeviceToHost, s_out);
  }
  if (e == cudaSuccess) e = cudaEventRecord(L->ev_out, s_out);
  if (e != cudaSuccess) {
    // nothing further was queued for this launch; wait for what was, then fail it
    cudaStreamSynchronize(s_in);
    cudaStreamSynchronize(s_run);
    cudaStreamSynchronize(s_out);
    L->err = e;
    L->failed = true;
  }
}

void fgfc_server::retire(Launch* L) {
  const uint8_t* sout = stg + L->stg_off + L->in_len;
  if (L->err == cudaSuccess) {
    std::vector<CopyPool::Copy> cp;
    for (Req* r : L->reqs) {
      if (r->direct || r->on_device) continue;
      for (size_t j = 0; j < r->m; ++j) cp.push_back({r->dst + r->starts[j], sout + (r->d_rows - L->out0) + j * r->Ls, r->L});
    }
    copies->run(cp);
  }
  for (Req* r : L->reqs) release_plan(r);
  std::lock_guard<std::mutex> lk(mu);
  launch_sum += std::chrono::duration<double, std::micro>(Clock::now() - L->t_issue).count();
  launch_n++;
  dev_arena.release(L->dev_off, L->dev_len);
  stg_arena.release(L->stg_off, L->stg_len);
  const std::string msg =
      L->err == cudaSuccess ? std::string() : std::string("server: CUDA error: ") + cudaGetErrorString(L->err);
  for (Req* r : L->reqs) finish(r, L->err == cudaSuccess ? FGFC_OK : FGFC_ERR_CUDA, msg);
  cudaEventDestroy(L->ev_in);
  cudaEventDestroy(L->ev_done);
  cudaEventDestroy(L->ev_out);
}

// Plain mode: one request, one call of the per-call entry point, synchronously.
void fgfc_server::run_plain(Req* r) {
  cudaError_t e = cudaSuccess;
  fgfc_status st = FGFC_OK;
  std::string err;
  if (r->on_device) {
    // in place: exactly the call the request stands for
    std::vector<fgfc_slice> sl(r->k);
    for (size_t t = 0; t < r->k; ++t) sl[t] = fgfc_slice{r->src[t], r->L};
    if (r->scattered && r->ovr)
      st = fgfc_dot_product_matrix_scattered_with(r->dst, r->dst_len, r->L, r->starts.data(), r->m, r->plan->plan,
                                                  sl.data(), r->k, s_run);
    else if (r->scattered)
      st = fgfc_mul_add_matrix_scattered_with(r->dst, r->dst_len, r->L, r->starts.data(), r->m, r->plan->plan,
                                              sl.data(), r->k, s_run);
    else if (r->ovr)
      st = fgfc_dot_product_matrix_with(r->dst, r->dst_len, r->L, r->m, r->plan->plan, sl.data(), r->k, s_run);
    else
      st = fgfc_mul_add_matrix_with(r->dst, r->dst_len, r->L, r->m, r->plan->plan, sl.data(), r->k, s_run);
    if (st != FGFC_OK) err = last_error_text();
    e = cudaStreamSynchronize(s_run);
    if (e != cudaSuccess) {
      st = FGFC_ERR_CUDA;
      err = std::string("server: CUDA error: ") + cudaGetErrorString(e);
    }
    release_plan(r);
    std::lock_guard<std::mutex> lk(mu);
    launches++;
    max_batch_seen = std::max<uint64_t>(max_batch_seen, 1);
    finish(r, st, err);
    return;
  }
  uint8_t* d = dev;  // the whole arena serves one request at a time
  uint8_t* s = stg;
  const size_t src_bytes_ = r->k * r->Ls;
  for (size_t t = 0; t < r->k && e == cudaSuccess; ++t) {
    if (r->direct) {
      e = cudaMemcpyAsync(d + t * r->Ls, r->src[t], r->L, cudaMemcpyHostToDevice, s_run);
    } else {
      std::memcpy(s + t * r->Ls, r->src[t], r->L);
    }
  }
  if (!r->ovr)
    for (size_t j = 0; j < r->m && e == cudaSuccess; ++j) {
      if (r->direct)
        e = cudaMemcpyAsync(d + src_bytes_ + j * r->Ls, r->dst + r->starts[j], r->L, cudaMemcpyHostToDevice, s_run);
      else
        std::memcpy(s + src_bytes_ + j * r->Ls, r->dst + r->starts[j], r->L);
    }
  if (!r->direct && e == cudaSuccess)
    e = cudaMemcpyAsync(d, s, src_bytes_ + (r->ovr ? 0 : r->m * r->Ls), cudaMemcpyHostToDevice, s_run);
  if (e == cudaSuccess) {
    std::vector<fgfc_slice> sl(r->k);
    for (size_t t = 0; t < r->k; ++t) sl[t] = fgfc_slice{d + t * r->Ls, r->L};
    std::vector<size_t> rs(r->m);
    for (size_t j = 0; j < r->m; ++j) rs[j] = src_bytes_ + j * r->Ls;
    if (r->ovr && r->Ls == r->L) {
      st = fgfc_dot_product_matrix_with(d + src_bytes_, r->m * r->L, r->L, r->m, r->plan->plan, sl.data(), r->k,
                                        s_run);
    } else if (r->ovr) {
      // rows at a padded stride: clear them, then accumulate
      e = cudaMemsetAsync(d + src_bytes_, 0, r->m * r->Ls, s_run);
      if (e == cudaSuccess)
        st = fgfc_mul_add_matrix_scattered_with(d, src_bytes_ + r->m * r->Ls, r->L, rs.data(), r->m, r->plan->plan,
                                                sl.data(), r->k, s_run);
    } else {
      st = fgfc_mul_add_matrix_scattered_with(d, src_bytes_ + r->m * r->Ls, r->L, rs.data(), r->m, r->plan->plan,
                                              sl.data(), r->k, s_run);
    }
    if (st != FGFC_OK) err = last_error_text();
  }
  if (e == cudaSuccess && st == FGFC_OK) {
    for (size_t j = 0; j < r->m && e == cudaSuccess; ++j) {
      if (r->direct)
        e = cudaMemcpyAsync(r->dst + r->starts[j], d + src_bytes_ + j * r->Ls, r->L, cudaMemcpyDeviceToHost, s_run);
    }
    if (!r->direct && e == cudaSuccess)
      e = cudaMemcpyAsync(s, d + src_bytes_, r->m * r->Ls, cudaMemcpyDeviceToHost, s_run);
  }
  cudaError_t e2 = cudaStreamSynchronize(s_run);
  if (e == cudaSuccess) e = e2;
  if (e == cudaSuccess && st == FGFC_OK && !r->direct)
    for (size_t j = 0; j < r->m; ++j) std::memcpy(r->dst + r->starts[j], s + j * r->Ls, r->L);
  if (e != cudaSuccess) {
    st = FGFC_ERR_CUDA;
    err = std::string("server: CUDA error: ") + cudaGetErrorString(e);
  }
  release_plan(r);
  std::lock_guard<std::mutex> lk(mu);
  launches++;
  max_batch_seen = std::max<uint64_t>(max_batch_seen, 1);
  peak_dev = std::max<uint64_t>(peak_dev, r->dev_bytes());
  finish(r, st, err);
}

void fgfc_server::run() {
  cudaSetDevice(device);
  std::unique_lock<std::mutex> lk(mu);
  Clock::time_point idle_since = Clock::now();
  for (;;) {
    bool progressed = false;
    // retire launches whose last copy has landed, oldest first
    while (!inflight.empty()) {
      Launch* F = inflight.front().get();
      if (!F->failed) {
        const cudaError_t q = cudaEventQuery(F->ev_out);
        if (q == cudaErrorNotReady) break;
        if (q != cudaSuccess) F->err = q;
      }
      std::unique_ptr<Launch> L = std::move(inflight.front());
      inflight.pop_front();
      lk.unlock();
      retire(L.get());
      lk.lock();
      progressed = true;
    }
    if (cfg.plain) {
      if (!pending.empty()) {
        Req* r = pending.front();
        pending.pop_front();
        r->t_issue = Clock::now();
        lk.unlock();
        if (acquire_plan(r)) {
          run_plain(r);
        } else {
          std::lock_guard<std::mutex> g(mu);
          finish(r, FGFC_ERR_CUDA, r->err);
        }
        lk.lock();
        continue;
      }
    } else if (!pending.empty() && inflight.size() < cfg.max_inflight) {
      // admit in arrival order while the blocks still fit
      auto L = std::make_unique<Launch>();
      size_t dbytes = 0, sbytes = 0;
      while (!pending.empty() && L->reqs.size() < cfg.max_batch) {
        Req* r = pending.front();
        const size_t nd = dbytes + r->dev_bytes(), ns = sbytes + r->stg_bytes();
        if (!L->reqs.empty() && nd > cfg.max_launch_bytes) break;  // keep launches small enough to pipeline
        size_t o1, o2;
        if (!dev_arena.alloc(nd, &o1)) break;
        if (!stg_arena.alloc(ns, &o2)) {
          dev_arena.release(o1, nd);
          break;
        }
        dev_arena.release(o1, nd);
        stg_arena.release(o2, ns);
        dbytes = nd;
        sbytes = ns;
        L->reqs.push_back(r);
        pending.pop_front();
      }
      if (!L->reqs.empty()) {
        dev_arena.alloc(dbytes, &L->dev_off);
        stg_arena.alloc(sbytes, &L->stg_off);
        L->dev_len = dbytes;
        L->stg_len = sbytes;
        peak_dev = std::max<uint64_t>(peak_dev, dev_arena.used());
        max_batch_seen = std::max<uint64_t>(max_batch_seen, L->reqs.size());
        launches++;
        Launch* raw = L.get();
        raw->t_issue = Clock::now();
        for (Req* r : raw->reqs) r->t_issue = raw->t_issue;
        inflight.push_back(std::move(L));
        lk.unlock();
        // plans (a miss uploads tables), events, then the launch itself
        std::vector<Req*> bad;
        for (Req* r : raw->reqs)
          if (!acquire_plan(r)) bad.push_back(r);
        if (!bad.empty()) {
          raw->reqs.erase(std::remove_if(raw->reqs.begin(), raw->reqs.end(),
                                         [&](Req* r) { return std::find(bad.begin(), bad.end(), r) != bad.end(); }),
                          raw->reqs.end());
          std::lock_guard<std::mutex> g(mu);
          for (Req* r : bad) finish(r, FGFC_ERR_CUDA, r->err);
        }
        cudaError_t e = cudaEventCreateWithFlags(&raw->ev_in, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&raw->ev_done, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&raw->ev_out, cudaEventDisableTiming);
        if (e != cudaSuccess) {
          raw->err = e;
          raw->failed = true;
        } else {
          issue(raw);
        }
        lk.lock();
        progressed = true;
      }
    }
    if (progressed) {
      idle_since = Clock::now();
      continue;
    }
    if (stop && pending.empty() && inflight.empty()) break;
    if (inflight.empty()) {
      cv.wait(lk, [&] { return stop || !pending.empty(); });  // nothing on the GPU: sleep until a submission
    } else if (Clock::now() - idle_since < std::chrono::microseconds(500)) {
      lk.unlock();  // launches in flight: poll their events, briefly yielding
      std::this_thread::yield();
      lk.lock();
    } else {
      cv.wait_for(lk, std::chrono::microseconds(50));  // long kernels: poll less often
    }
  }
}

extern "C" {

fgfc_status fgfc_server_create(const fgfc_server_config* cfg, fgfc_server** out) {
  if (!out) return set_error(FGFC_ERR_ARG, "server: null argument");
  *out = nullptr;
  auto s = std::make_unique<fgfc_server>();
  if (cfg) s->cfg = *cfg;
  if (!s->cfg.hbm_budget) s->cfg.hbm_budget = size_t(64) << 30;
  if (!s->cfg.staging_bytes) s->cfg.staging_bytes = size_t(1) << 30;
  if (!s->cfg.max_batch) s->cfg.max_batch = 1024;
  if (!s->cfg.max_inflight) s->cfg.max_inflight = 4;
  if (!s->cfg.plan_cache) s->cfg.plan_cache = 64;
  if (!s->cfg.max_launch_bytes) s->cfg.max_launch_bytes = size_t(256) << 20;
  if (!cfg) s->cfg.device = -1;
  cudaError_t e = cudaSuccess;
  if (s->cfg.device >= 0) {
    s->device = s->cfg.device;
    e = cudaSetDevice(s->device);
  } else {
    e = cudaGetDevice(&s->device);
  }
  if (e == cudaSuccess) e = cudaMalloc(&s->dev, s->cfg.hbm_budget);
  if (e == cudaSuccess) e = cudaHostAlloc(&s->stg, s->cfg.staging_bytes, cudaHostAllocDefault);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->s_in, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->s_run, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->s_out, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    std::string msg = std::string("server: CUDA error: ") + cudaGetErrorString(e);
    if (s->dev) cudaFree(s->dev);
    if (s->stg) cudaFreeHost(s->stg);
    if (s->s_in) cudaStreamDestroy(s->s_in);
    if (s->s_run) cudaStreamDestroy(s->s_run);
    if (s->s_out) cudaStreamDestroy(s->s_out);
    return set_error(FGFC_ERR_CUDA, msg.c_str());
  }
  s->dev_arena.reset(s->cfg.hbm_budget);
  s->stg_arena.reset(s->cfg.staging_bytes);
  s->batch = batch_state_create();
  batch_state_graphs(s->batch, false);  // every launch has a new structure
  s->copies = std::make_unique<CopyPool>(s->cfg.plain ? 0 : 7);
  s->worker = std::thread([p = s.get()] { p->run(); });
  *out = s.release();
  return clear_error();
}

fgfc_status fgfc_server_submit(fgfc_server* s, const fgfc_request* q, uint64_t* ticket) {
  if (!s || !q || !ticket) return set_error(FGFC_ERR_ARG, "server: null argument");
  const char* name =
      q->row_starts ? "mul_add_matrix_scattered" : (q->overwrite ? "dot_product_matrix" : "mul_add_matrix");
  fgfc_status st = validate_matrix_call(q->field, name, q->dst_len, q->row_len, q->row_starts, q->nrows, q->srcs,
                                        q->nsrcs, q->coeffs, q->overwrite);
  if (st != FGFC_OK) return st;
  if (field_bytes(q->field) > 4)
    return set_error(FGFC_ERR_ARG, "server: 8-byte fields are not served (their coefficients do not fit the "
                                   "request's 32-bit coefficient array)");
  auto r = std::make_unique<Req>();
  r->field = q->field;
  r->k = q->nsrcs;
  r->m = q->nrows;
  r->L = q->row_len;
  r->Ls = up(q->row_len);
  r->ovr = q->overwrite != 0;
  r->dst = q->dst;
  r->t0 = Clock::now();
  const uint32_t mask = field_mask(q->field);
  r->coeffs.resize(r->k * r->m);
  for (size_t i = 0; i < r->coeffs.size(); ++i) r->coeffs[i] = q->coeffs[i] & mask;
  r->src.resize(r->k);
  for (size_t t = 0; t < r->k; ++t) r->src[t] = q->srcs[t].ptr;
  r->starts.resize(r->m);
  for (size_t j = 0; j < r->m; ++j) r->starts[j] = q->row_starts ? q->row_starts[j] : j * q->row_len;
  uint64_t h = 0xcbf29ce484222325ull;
  h = fnv1a(h, &r->field, sizeof r->field);
  h = fnv1a(h, &r->k, sizeof r->k);
  h = fnv1a(h, &r->m, sizeof r->m);
  h = fnv1a(h, r->coeffs.data(), r->coeffs.size() * 4);
  r->key = h;
  r->scattered = q->row_starts != nullptr;
  r->dst_len = q->dst_len;
  const bool trivial = r->m == 0 || r->L == 0 || r->k == 0;
  if (!trivial) {
    // all device memory of this server's device (used in place), or all host
    // memory; one attribute lookup per buffer (its first byte), plus the last
    // byte of page-locked buffers long enough to be copied without staging
    int dev = -1, ndev = 0, nbuf = 0;
    bool locked = r->L >= kDirectMin;
    auto look = [&](const void* p, size_t n) {
      ++nbuf;
      const cudaMemoryType t = where(p, &dev);
      if (t == cudaMemoryTypeDevice && dev == s->device) ++ndev;
      if (locked) locked = t == cudaMemoryTypeHost && host_locked(static_cast<const uint8_t*>(p) + n - 1);
    };
    look(r->dst, q->dst_len);
    for (size_t t = 0; t < r->k; ++t) look(r->src[t], r->L);
    if (ndev && ndev != nbuf)
      return set_error(FGFC_ERR_ARG, "server: a request's buffers must all be host memory or all device memory");
    r->on_device = ndev == nbuf;
    r->direct = !r->on_device && locked;
  }
  if (!trivial && (r->dev_bytes() > s->cfg.hbm_budget || r->stg_bytes() > s->cfg.staging_bytes))
    return set_error(FGFC_ERR_LIMIT, "server: request needs more device or staging memory than the server has");
  std::lock_guard<std::mutex> lk(s->mu);
  r->ticket = s->next_ticket++;
  *ticket = r->ticket;
  if (!s->have_first) {
    s->first_submit = r->t0;
    s->have_first = true;
  }
  Req* raw = r.get();
  s->reqs.emplace(raw->ticket, std::move(r));
  s->outstanding++;
  if (trivial) {
    // no sources: an overwrite clears the rows; everything else is a no-op
    if (raw->ovr && raw->L && raw->m) {
      int dev = -1;
      if (where(raw->dst, &dev) == cudaMemoryTypeDevice) {
        // device rows: cleared in stream order on the request stream
        for (size_t j = 0; j < raw->m; ++j) cudaMemsetAsync(raw->dst + raw->starts[j], 0, raw->L, s->s_run);
        cudaStreamSynchronize(s->s_run);
      } else {
        for (size_t j = 0; j < raw->m; ++j) std::memset(raw->dst + raw->starts[j], 0, raw->L);
      }
    }
    s->finish(raw, FGFC_OK, std::string());
    return clear_error();
  }
  s->pending.push_back(raw);
  s->cv.notify_all();
  return clear_error();
}

// A rebuild by erasure pattern: the decode rows of the pattern (host
// Gauss-Jordan, decode.cpp; kept in a small cache keyed by a hash of the
// code and the pattern) become the coefficients of an ordinary request that
// overwrites the rebuilt shards.
fgfc_status fgfc_server_submit_rebuild(fgfc_server* s, const fgfc_rebuild_request* q, uint64_t* ticket) {
  if (!s || !q || !ticket) return set_error(FGFC_ERR_ARG, "server: null argument");
  if (field_bytes(q->field) == 0) return set_error(FGFC_ERR_ARG, "server: unknown field");
  if (field_bytes(q->field) > 4)
    return set_error(FGFC_ERR_ARG, "server: 8-byte fields are not served (their coefficients do not fit the "
                                   "request's 32-bit coefficient arrays)");
  if (!q->k || !q->survivors || !q->parity || (q->nerased && !q->erased))
    return set_error(FGFC_ERR_ARG, "server: rebuild request without code or pattern");
  uint64_t h = 0xcbf29ce484222325ull;
  h = fnv1a(h, &q->field, sizeof q->field);
  h = fnv1a(h, &q->k, sizeof q->k);
  h = fnv1a(h, &q->m, sizeof q->m);
  h = fnv1a(h, q->parity, q->m * q->k * sizeof(uint32_t));
  h = fnv1a(h, q->survivors, q->k * sizeof(size_t));
  h = fnv1a(h, q->erased, q->nerased * sizeof(size_t));
  std::vector<uint32_t> d;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    auto it = s->decode_cache.find(h);
    if (it != s->decode_cache.end()) d = it->second;
  }
  if (d.empty()) {
    d.resize(q->k * q->nerased + 1);
    const fgfc_status st =
        decode_matrix(q->field, q->parity, q->k, q->m, q->survivors, q->erased, q->nerased, d.data());
    if (st != FGFC_OK) return st;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->decode_cache.size() >= 4096) s->decode_cache.clear();
    s->decode_cache.emplace(h, d);
  }
  fgfc_request r;
  r.field = q->field;
  r.coeffs = d.data();
  r.srcs = q->srcs;
  r.nsrcs = q->k;
  r.dst = q->dst;
  r.dst_len = q->dst_len;
  r.row_starts = q->row_starts;
  r.nrows = q->nerased;
  r.row_len = q->row_len;
  r.overwrite = 1;
  return fgfc_server_submit(s, &r, ticket);
}

fgfc_status fgfc_server_poll(fgfc_server* s, uint64_t ticket, int* done) {
  if (!s || !done) return set_error(FGFC_ERR_ARG, "server: null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return set_error(FGFC_ERR_ARG, "server: unknown ticket");
  *done = it->second->done ? 1 : 0;
  if (!*done) return clear_error();
  const fgfc_status st = it->second->status;
  const std::string err = it->second->err;
  s->reqs.erase(it);
  lk.unlock();
  return st == FGFC_OK ? clear_error() : set_error(st, err.c_str());
}

fgfc_status fgfc_server_wait(fgfc_server* s, uint64_t ticket) {
  if (!s) return set_error(FGFC_ERR_ARG, "server: null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->reqs.find(ticket);
  if (it == s->reqs.end()) return set_error(FGFC_ERR_ARG, "server: unknown ticket");
  Req* r = it->second.get();
  s->done_cv.wait(lk, [&] { return r->done; });
  const fgfc_status st = r->status;
  const std::string err = r->err;
  s->reqs.erase(ticket);
  lk.unlock();
  return st == FGFC_OK ? clear_error() : set_error(st, err.c_str());
}

fgfc_status fgfc_server_drain(fgfc_server* s) {
  if (!s) return set_error(FGFC_ERR_ARG, "server: null argument");
  std::unique_lock<std::mutex> lk(s->mu);
  s->done_cv.wait(lk, [&] { return s->outstanding == 0; });
  return clear_error();
}

fgfc_status fgfc_server_get_stats(fgfc_server* s, fgfc_server_stats* out, int reset) {
  if (!s || !out) return set_error(FGFC_ERR_ARG, "server: null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  std::memset(out, 0, sizeof *out);
  out->completed = s->completed;
  out->failed = s->failed;
  out->launches = s->launches;
  out->plan_hits = s->hits;
  out->plan_misses = s->misses;
  out->source_bytes = s->src_bytes;
  out->peak_device_bytes = s->peak_dev;
  out->max_batch_seen = s->max_batch_seen;
  if (!s->lat_us.empty()) {
    std::vector<double> v = s->lat_us;
    std::sort(v.begin(), v.end());
    auto pct = [&](double p) {
      const size_t i = static_cast<size_t>(p * static_cast<double>(v.size() - 1) + 0.5);
      return v[std::min(i, v.size() - 1)];
    };
    out->p50_us = pct(0.50);
    out->p99_us = pct(0.99);
    out->max_us = v.back();
    double sum = 0;
    for (double x : v) sum += x;
    out->mean_us = sum / static_cast<double>(v.size());
  }
  if (s->have_first && s->completed + s->failed)
    out->busy_s = std::chrono::duration<double>(s->last_done - s->first_submit).count();
  if (s->completed) out->queue_us = s->queue_sum / static_cast<double>(s->completed);
  if (s->launch_n) out->launch_us = s->launch_sum / static_cast<double>(s->launch_n);
  if (reset) {
    s->lat_us.clear();
    s->queue_sum = s->launch_sum = 0;
    s->launch_n = 0;
    s->completed = s->failed = s->launches = s->hits = s->misses = s->src_bytes = s->peak_dev =
        s->max_batch_seen = 0;
    s->have_first = false;
  }
  return clear_error();
}

void fgfc_server_destroy(fgfc_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
    s->cv.notify_all();
  }
  if (s->worker.joinable()) s->worker.join();
  cudaSetDevice(s->device);
  cudaStreamSynchronize(s->s_in);
  cudaStreamSynchronize(s->s_run);
  cudaStreamSynchronize(s->s_out);
  for (auto& e : s->plans) fgfc_plan_destroy(e.plan);
  batch_state_destroy(s->batch);
  cudaFree(s->dev);
  cudaFreeHost(s->stg);
  cudaStreamDestroy(s->s_in);
  cudaStreamDestroy(s->s_run);
  cudaStreamDestroy(s->s_out);
  delete s;
}

}  // extern "C"
