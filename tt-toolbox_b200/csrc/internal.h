// Internal declarations of libttgpu (not part of the C-ABI).
//
// One context = one device, one stream, one cuSOLVER handle and one caching
// device allocator.  All kernels of a context run on its stream.  Host code
// reports failures by throwing ttg::Error; every extern "C" entry point
// catches and converts to a status code + message (include/ttgpu.h).
#pragma once

#include <cuda_runtime.h>
#include <cusolverDn.h>

#include <atomic>
#include <cstdint>
#include <cstdio>
#include <functional>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "../../include/ttgpu.h"

namespace ttg {

struct Error {
  int code;
  std::string msg;
};

[[noreturn]] void fail(int code, const char* fmt, ...);

#define TTG_CUDA(call)                                                              \
  do {                                                                              \
    cudaError_t e_ = (call);                                                        \
    if (e_ != cudaSuccess) {                                                        \
      cudaGetLastError(); /* a refused call must not fail the next check */         \
      ::ttg::fail(TTG_ERR_CUDA, "%s:%d: %s: %s", __FILE__, __LINE__, #call,         \
                  cudaGetErrorString(e_));                                          \
    }                                                                               \
  } while (0)

#define TTG_SOLVER(call)                                                            \
  do {                                                                              \
    cusolverStatus_t s_ = (call);                                                   \
    if (s_ != CUSOLVER_STATUS_SUCCESS)                                              \
      ::ttg::fail(TTG_ERR_SOLVER, "%s:%d: %s: cusolver status %d", __FILE__,        \
                  __LINE__, #call, (int)s_);                                        \
  } while (0)

#define TTG_CHECK_LAUNCH() TTG_CUDA(cudaGetLastError())

#define TTG_REQUIRE(cond, ...)                                                      \
  do {                                                                              \
    if (!(cond)) ::ttg::fail(TTG_ERR_INVALID, __VA_ARGS__);                         \
  } while (0)

// Number of per-tile arrival counters a context holds for split-K GEMMs.
constexpr int64_t GEMM_TILE_COUNTERS = int64_t(1) << 16;

// Caching device allocator: blocks are rounded up to a size class and kept
// on per-class free lists, so a solve that reaches steady state performs no
// cudaMalloc.  get/put are serialised by a mutex: the batched solve draws its
// result handles from the owning context's allocator on worker threads.  A
// block put back is reused in stream order only on the stream of the thread
// that takes it, so blocks shared across streams are handed over only at
// points where both streams have been synchronised.
class Allocator {
 public:
  explicit Allocator(int device) : device_(device) {}
  ~Allocator();
  void* get(size_t bytes);
  void put(void* p);
  size_t bytes_in_use() const { return in_use_; }
  uint64_t gets() const { return n_get_; }
  uint64_t mallocs() const { return n_malloc_; }
  double ms_get() const { return double(ns_get_.load()) * 1e-6; }
  size_t bytes_cached() const { return cached_; }
  static size_t size_class(size_t bytes);

 private:
  int device_;
  std::mutex mu_;
  static constexpr size_t SLAB_CLASS_MAX = size_t(4) << 20;
  struct Carve {
    char* next = nullptr;
    size_t left = 0;
  };
  void* carve(size_t cls);  // mu_ held
  std::map<size_t, std::vector<void*>> free_;
  std::map<void*, size_t> live_;
  std::map<size_t, Carve> carve_;
  std::vector<void*> slabs_;
  size_t in_use_ = 0, cached_ = 0;
  uint64_t n_get_ = 0, n_malloc_ = 0;
  std::atomic<uint64_t> ns_get_{0};
};

struct Context;

// Grouped batch (group.cu).  A context whose `rec` is set belongs to one
// solve of a grouped batch: its stream work is recorded in order instead of
// issued, and the batch executor issues the records of all solves together,
// merging launches of the same kernel into grouped launches, whenever every
// solve waits for the device (a host read or a synchronisation).
struct Recorder;
using StreamOp = std::function<void(cudaStream_t, cusolverDnHandle_t)>;
// Record a stream operation (issued by the executor in the solve's order).
void rec_op(Recorder* r, StreamOp op);
// Block until the executor has issued and completed everything recorded.
void rec_wait(Recorder* r);
// Takes back the FLOPs of recorded tensor-core GEMMs that the solve found
// skipped on the device (Krylov steps queued past convergence).
void rec_retract_flop(Recorder* r, double flop, int64_t records);
class Allocator;
// Device blocks of a recording context: each solve keeps the blocks it frees
// for its own later allocations (its records are issued in its own order,
// so a block is reused only after the records that used it); blocks go back
// to the shared allocator when the batch ends.
void* rec_alloc(Recorder* r, Allocator* shared, size_t bytes);
void rec_free(Recorder* r, void* p, size_t bytes);
struct Context;
// Recorded memset and device-to-host read (into the context's pinned,
// device-mapped scalar buffer at byte offset `off`) as grouped kernels.
void rec_memset(Context* c, void* p, int value, size_t bytes);
void rec_read(Context* c, size_t off, const void* src, size_t bytes);

// RAII device buffer drawn from a context's allocator.
template <typename T>
class DBuf {
 public:
  DBuf() = default;
  DBuf(Context* c, size_t n);
  DBuf(const DBuf&) = delete;
  DBuf& operator=(const DBuf&) = delete;
  DBuf(DBuf&& o) noexcept { swap(o); }
  DBuf& operator=(DBuf&& o) noexcept {
    release();
    swap(o);
    return *this;
  }
  ~DBuf() { release(); }
  void reset(Context* c, size_t n);  // reallocate if capacity too small
  T* p() const { return p_; }
  size_t size() const { return n_; }
  void release();

 private:
  void swap(DBuf& o) {
    std::swap(c_, o.c_);
    std::swap(p_, o.p_);
    std::swap(n_, o.n_);
  }
  Context* c_ = nullptr;
  T* p_ = nullptr;
  size_t n_ = 0;
};

struct Context {
  int device = 0;
  int num_sms = 0;
  cudaStream_t stream = nullptr;
  cusolverDnHandle_t solver = nullptr;
  Allocator* alloc = nullptr;
  // Small pinned host buffer for scalar read-back (a grouped batch's
  // contexts: mapped, h_scal_dev its device address).
  double* h_scal = nullptr;
  double* h_scal_dev = nullptr;
  // Device int slots: 0-7 error flags of bounded waits and factorizations
  // (cleared per solve), 63 the arrival counter of the one-launch reductions.
  int* d_err = nullptr;
  // Sweep limit of the one-sided Jacobi SVDs (ttg_context_set_option).
  int jacobi_max_sweeps = 40;
  // SM count the solves of a grouped batch size their grids with (0: share).
  int group_sms = 0;
  // Per-output-tile arrival counters of split-K GEMMs (GEMM_TILE_COUNTERS,
  // zero between launches: the last slice of a tile resets its counter).
  unsigned* d_tile_cnt = nullptr;
  // Counters (reset by the caller through ttg_stats).
  int64_t launches = 0;
  int64_t matvecs = 0;
  int64_t matvec_flops = 0;
  // Per-kind local-matvec counters: [0] FP64 (DMMA), [1] BF16 (tcgen05).
  int64_t mv_count[2] = {0, 0};
  // Mixed local solves that finished in FP64 (see local_solve_mixed).
  int64_t mixed_fallbacks = 0;
  // Krylov steps of the last restart of the previous low-precision inner
  // solve: sizes the first chunk of queued steps of the next one.
  int krylov_hint = 0;
  double mv_flops[2] = {0.0, 0.0};
  // Algorithmic DRAM bytes of the BF16 local matvecs: the BF16 operand X,
  // the three BF16 operators and the FP32 result, once each.
  double mv_bytes_lp = 0.0;
  // Optional CUDA-event timing of every local matvec on the context stream.
  bool time_matvec = false;
  // Launch the library's stream-ordered kernels as programmatic dependent
  // launches (see launch()); off for contexts on a caller's stream.
  bool pdl = false;
  struct EvPair {
    cudaEvent_t a, b;
    int kind;       // -1: voided (a speculatively queued matvec that was skipped)
    uint64_t seq;   // running number of the pair on this context
  };
  std::vector<EvPair> ev_pool;
  size_t ev_used = 0;
  uint64_t ev_seq = 0;
  double mv_ms[2] = {0.0, 0.0};
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // While non-null, GEMM and matvec kernels launched on this context return
  // immediately when *skip != 0 (speculatively queued Krylov steps after
  // convergence).
  const int* skip = nullptr;
  // Non-null: the context records its stream work for a grouped batch.
  Recorder* rec = nullptr;

  int ev_begin(int kind) {
    if (ev_used == ev_pool.size()) {
      EvPair p{};
      cudaEventCreate(&p.a);
      cudaEventCreate(&p.b);
      ev_pool.push_back(p);
    }
    ev_pool[ev_used].kind = kind;
    ev_pool[ev_used].seq = ev_seq++;
    cudaEventRecord(ev_pool[ev_used].a, stream);
    return int(ev_used++);
  }
  void ev_end(int i) { cudaEventRecord(ev_pool[i].b, stream); }
  // Drop the pairs numbered [from, to) that are not collected yet.
  void ev_void(uint64_t from, uint64_t to) {
    for (size_t i = 0; i < ev_used; ++i)
      if (ev_pool[i].seq >= from && ev_pool[i].seq < to) ev_pool[i].kind = -1;
  }
  // Accumulate the elapsed time of all recorded pairs into mv_ms (syncs).
  void ev_collect() {
    if (rec) {  // no event timing in a grouped batch
      ev_used = 0;
      return;
    }
    cudaStreamSynchronize(stream);
    for (size_t i = 0; i < ev_used; ++i) {
      if (ev_pool[i].kind < 0) continue;
      float ms = 0.f;
      cudaEventElapsedTime(&ms, ev_pool[i].a, ev_pool[i].b);
      mv_ms[ev_pool[i].kind] += ms;
    }
    ev_used = 0;
  }
};

// Sets Context::skip for a scope (cleared on every exit path).
struct SkipGuard {
  Context* c;
  SkipGuard(Context* cc, const int* flag) : c(cc) { c->skip = flag; }
  void release() { c->skip = nullptr; }
  ~SkipGuard() { c->skip = nullptr; }
};

// Scope guard: records an event pair around a local matvec when timing is on.
struct MvTiming {
  Context* c;
  int idx = -1;
  MvTiming(Context* cc, int kind) : c(cc) {
    if (c->time_matvec) {
      if (c->ev_used >= 4096) c->ev_collect();
      idx = c->ev_begin(kind);
    }
  }
  ~MvTiming() {
    if (idx >= 0) c->ev_end(idx);
  }
};

template <typename T>
DBuf<T>::DBuf(Context* c, size_t n) {
  reset(c, n);
}
template <typename T>
void DBuf<T>::reset(Context* c, size_t n) {
  if (c_ == c && n <= n_ && p_) return;
  release();
  c_ = c;
  n_ = n;
  p_ = n ? static_cast<T*>(c->rec ? rec_alloc(c->rec, c->alloc, n * sizeof(T))
                                 : c->alloc->get(n * sizeof(T)))
         : nullptr;
}
template <typename T>
void DBuf<T>::release() {
  if (p_ && c_) {
    if (c_->rec)
      rec_free(c_->rec, p_, n_ * sizeof(T));
    else
      c_->alloc->put(p_);
  }
  p_ = nullptr;
  n_ = 0;
}

void set_last_error(const char* msg);

// Programmatic dependent launch.  A kernel launched by launch() may be
// scheduled while its predecessor on the stream is still running: the
// predecessor lets it start with pdl_trigger() once all of its own CTAs
// run, and the kernel itself must call pdl_wait() before its first access
// to global memory (pdl_wait returns when the predecessor grid has
// completed and its writes are visible; it is a no-op for a kernel launched
// without the attribute).  Every kernel launched through launch() therefore
// starts with pdl_begin(): it waits, then lets its own successor be
// scheduled.  This hides the kernel-to-kernel launch latency of the long
// chains of short kernels in a sweep.
#ifdef __CUDACC__
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}
#endif

template <typename... KArgs, typename... Args>
void launch(Context* c, void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem,
            Args&&... args) {
  if (c->rec) {  // grouped batch: one recorded launch of its own
    std::tuple<std::decay_t<KArgs>...> t(std::forward<Args>(args)...);
    const bool pdl = c->pdl;
    rec_op(c->rec, [kernel, grid, block, smem, t, pdl](cudaStream_t s, cusolverDnHandle_t) {
      std::apply(
          [&](const auto&... a) {
            cudaLaunchConfig_t cfg = {};
            cfg.gridDim = grid;
            cfg.blockDim = block;
            cfg.dynamicSmemBytes = smem;
            cfg.stream = s;
            cudaLaunchAttribute attr[1];
            attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
            attr[0].val.programmaticStreamSerializationAllowed = 1;
            cfg.attrs = attr;
            cfg.numAttrs = pdl ? 1 : 0;
            TTG_CUDA(cudaLaunchKernelEx(&cfg, kernel, a...));
          },
          t);
    });
    c->launches += 1;
    return;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = c->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = c->pdl ? 1 : 0;
  TTG_CUDA(cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...));
  c->launches += 1;
}

#define TTG_API_BEGIN try {
#define TTG_API_END                                    \
  }                                                    \
  catch (const ::ttg::Error& e) {                      \
    ::ttg::set_last_error(e.msg.c_str());              \
    return e.code;                                     \
  }                                                    \
  catch (const std::exception& e) {                    \
    ::ttg::set_last_error(e.what());                   \
    return TTG_ERR_INVALID;                            \
  }                                                    \
  ::ttg::set_last_error("");                           \
  return TTG_OK;

// Copy a device scalar (or a few) to the host; synchronises the stream.
void read_scalars(Context* c, const double* d, double* h, int count);
// Copy `bytes` (at most 32 KiB) of device memory to the host; synchronises.
void read_device(Context* c, void* h, const void* d, size_t bytes);
void sync(Context* c);
// Stream-ordered memset / device-to-device copy on the context's stream.
void memset_async(Context* c, void* p, int value, size_t bytes);
void copy_async(Context* c, void* dst, const void* src, size_t bytes);
// A cuSOLVER call on the context's stream and handle.
void solver_call(Context* c, const StreamOp& op);
// Stream, solver handle, allocator, pinned scalars and error slots of a
// context on `device` (the current device must be `device`).
void context_init(Context& c, int device);
void context_release(Context& c);
// Raise a kernel's dynamic shared-memory limit to `bytes` on `device`, once
// per (kernel, device); thread-safe (contexts on several host threads).
void ensure_smem_attr(const void* func, int device, int bytes);
// cudaOccupancyMaxActiveBlocksPerMultiprocessor, remembered per (kernel,
// block size, shared memory); thread-safe.
int max_active_blocks(const void* func, int threads, size_t smem);

}  // namespace ttg

// TT handle: cores stay resident on the device of the owning context.
struct ttg_tt_s {
  ttg::Context* ctx;
  int64_t d;
  bool is_matrix;
  std::vector<int64_t> n, m, r, ps;  // ps: 0-based offsets (d+1)
  double* core;                      // device, numel doubles
  int64_t numel;
};

struct ttg_context_s {
  ttg::Context c;
  // Worker contexts of the batched solve (created on first use, each with
  // its own stream), guarded by mu.
  std::mutex mu;
  std::vector<std::unique_ptr<ttg::Context>> workers;
};
