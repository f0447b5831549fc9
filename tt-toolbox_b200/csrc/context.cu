// Context, caching allocator, error reporting and TT handles of libttgpu.
#include <atomic>
#include <chrono>
#include <cstdlib>
#include <cstdarg>
#include <cstring>
#include <mutex>
#include <tuple>

#include "internal.h"

namespace {
thread_local std::string g_last_error;
}

namespace ttg {

void fail(int code, const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  throw Error{code, std::string(buf)};
}

Allocator::~Allocator() {
  int prev = 0;
  cudaGetDevice(&prev);
  cudaSetDevice(device_);
  for (void* p : slabs_) cudaFree(p);
  for (auto& kv : free_)
    for (void* p : kv.second)
      if (kv.first > SLAB_CLASS_MAX) cudaFree(p);
  for (auto& kv : live_)
    if (kv.second > SLAB_CLASS_MAX) cudaFree(kv.first);
  cudaSetDevice(prev);
}

size_t Allocator::size_class(size_t bytes) {
  // 256-byte granularity up to 4 KiB, then four classes per octave (at most
  // 25% over the request): few distinct sizes, so blocks freed by one solve
  // serve the next even when the shapes of the local problems vary.
  if (bytes < 256) return 256;
  if (bytes <= 4096) return (bytes + 255) & ~size_t(255);
  size_t p = 1;
  while (p < bytes) p <<= 1;
  size_t step = p >> 3;  // classes 5p/8, 6p/8, 7p/8, p of the octave (p/2, p]
  return ((bytes + step - 1) / step) * step;
}

// Blocks of at most SLAB_CLASS_MAX bytes are carved from slabs of 32 blocks
// (2 MiB to 64 MiB), one cudaMalloc per slab: a batch of solves that grows
// its pool by tens of thousands of blocks makes a few hundred driver calls.
// Larger blocks are allocated one by one.
void* Allocator::carve(size_t cls) {
  auto& c = carve_[cls];
  if (c.left < cls) {
    const size_t slab = std::min<size_t>(std::max<size_t>(32 * cls, size_t(2) << 20),
                                         size_t(64) << 20) / cls * cls;
    void* base = nullptr;
    ++n_malloc_;
    if (cudaMalloc(&base, slab) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    slabs_.push_back(base);
    c.next = static_cast<char*>(base);
    c.left = slab;
  }
  void* p = c.next;
  c.next += cls;
  c.left -= cls;
  return p;
}

void* Allocator::get(size_t bytes) {
  const auto t0 = std::chrono::steady_clock::now();
  struct Clock {  // time spent here, lock wait included
    std::atomic<uint64_t>& ns;
    std::chrono::steady_clock::time_point t0;
    ~Clock() {
      ns += uint64_t(std::chrono::duration_cast<std::chrono::nanoseconds>(
                         std::chrono::steady_clock::now() - t0).count());
    }
  } clock{ns_get_, t0};
  std::lock_guard<std::mutex> lock(mu_);
  size_t cls = size_class(bytes);
  ++n_get_;
  auto it = free_.find(cls);
  void* p = nullptr;
  if (it != free_.end() && !it->second.empty()) {
    p = it->second.back();
    it->second.pop_back();
    cached_ -= cls;
  } else {
    for (int attempt = 0; attempt < 2 && !p; ++attempt) {
      if (cls <= SLAB_CLASS_MAX) {
        p = carve(cls);
      } else {
        ++n_malloc_;
        if (cudaMalloc(&p, cls) != cudaSuccess) {
          cudaGetLastError();
          p = nullptr;
        }
      }
      if (!p && attempt == 0) {
        // Give the cached large blocks back and retry once.
        for (auto& kv : free_) {
          if (kv.first <= SLAB_CLASS_MAX) continue;
          for (void* q : kv.second) cudaFree(q);
          cached_ -= kv.first * kv.second.size();
          kv.second.clear();
        }
      }
    }
    if (!p) fail(TTG_ERR_ALLOC, "device allocation of %zu bytes failed", cls);
  }
  live_[p] = cls;
  in_use_ += cls;
  return p;
}

void Allocator::put(void* p) {
  std::lock_guard<std::mutex> lock(mu_);
  auto it = live_.find(p);
  if (it == live_.end()) return;
  size_t cls = it->second;
  live_.erase(it);
  in_use_ -= cls;
  free_[cls].push_back(p);
  cached_ += cls;
}

void set_last_error(const char* msg) { g_last_error = msg; }

void sync(Context* c) {
  if (c->rec) {
    rec_wait(c->rec);
    return;
  }
  TTG_CUDA(cudaStreamSynchronize(c->stream));
}

void context_init(Context& c, int device) {
  c.device = device;
  TTG_CUDA(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, device));
  TTG_CUDA(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
  TTG_SOLVER(cusolverDnCreate(&c.solver));
  TTG_SOLVER(cusolverDnSetStream(c.solver, c.stream));
  c.alloc = new Allocator(device);
  TTG_CUDA(cudaMallocHost(&c.h_scal, 4096 * sizeof(double)));
  TTG_CUDA(cudaMalloc(&c.d_err, 64 * sizeof(int)));
  TTG_CUDA(cudaMemset(c.d_err, 0, 64 * sizeof(int)));
  TTG_CUDA(cudaMalloc(&c.d_tile_cnt, GEMM_TILE_COUNTERS * sizeof(unsigned)));
  TTG_CUDA(cudaMemset(c.d_tile_cnt, 0, GEMM_TILE_COUNTERS * sizeof(unsigned)));
  TTG_CUDA(cudaEventCreate(&c.ev0));
  TTG_CUDA(cudaEventCreate(&c.ev1));
  const char* pdl = getenv("TTG_PDL");  // TTG_PDL=0: plain stream-ordered launches
  c.pdl = !(pdl && pdl[0] == '0');
}

void context_release(Context& c) {
  if (c.stream) cudaStreamSynchronize(c.stream);
  delete c.alloc;
  c.alloc = nullptr;
  if (c.solver) cusolverDnDestroy(c.solver);
  if (c.h_scal) cudaFreeHost(c.h_scal);
  if (c.d_err) cudaFree(c.d_err);
  if (c.d_tile_cnt) cudaFree(c.d_tile_cnt);
  if (c.ev0) cudaEventDestroy(c.ev0);
  if (c.ev1) cudaEventDestroy(c.ev1);
  for (auto& e : c.ev_pool) {
    cudaEventDestroy(e.a);
    cudaEventDestroy(e.b);
  }
  c.ev_pool.clear();
  if (c.stream) cudaStreamDestroy(c.stream);
  c.solver = nullptr;
  c.h_scal = nullptr;
  c.d_err = nullptr;
  c.d_tile_cnt = nullptr;
  c.ev0 = c.ev1 = nullptr;
  c.stream = nullptr;
}

void ensure_smem_attr(const void* func, int device, int bytes) {
  // Per-thread memo in front of the shared one: the grouped batch calls this
  // from many fibers on a few threads.
  thread_local std::map<std::pair<const void*, int>, int> seen;
  auto it = seen.find({func, device});
  if (it != seen.end() && it->second >= bytes) return;
  {
    static std::mutex mu;
    static std::map<std::pair<const void*, int>, int> done;
    std::lock_guard<std::mutex> lock(mu);
    auto d = done.find({func, device});
    if (d == done.end() || d->second < bytes) {
      TTG_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
      done[{func, device}] = bytes;
    }
  }
  seen[{func, device}] = bytes;
}

int max_active_blocks(const void* func, int threads, size_t smem) {
  using Key = std::tuple<const void*, int, size_t>;
  thread_local std::map<Key, int> seen;
  const Key k{func, threads, smem};
  auto it = seen.find(k);
  if (it != seen.end()) return it->second;
  int occ = 0;
  TTG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, func, threads, smem));
  seen[k] = occ;
  return occ;
}

void read_device(Context* c, void* h, const void* d, size_t bytes) {
  TTG_REQUIRE(bytes <= 4096 * sizeof(double), "read_device: %zu bytes", bytes);
  double* stage = c->h_scal;
  if (c->rec) {
    rec_read(c, 0, d, bytes);
    rec_wait(c->rec);
  } else {
    TTG_CUDA(cudaMemcpyAsync(stage, d, bytes, cudaMemcpyDeviceToHost, c->stream));
    TTG_CUDA(cudaStreamSynchronize(c->stream));
  }
  memcpy(h, stage, bytes);
}

void read_scalars(Context* c, const double* d, double* h, int count) {
  read_device(c, h, d, sizeof(double) * count);
}

void memset_async(Context* c, void* p, int value, size_t bytes) {
  if (c->rec) {
    rec_memset(c, p, value, bytes);
    return;
  }
  TTG_CUDA(cudaMemsetAsync(p, value, bytes, c->stream));
}

void copy_async(Context* c, void* dst, const void* src, size_t bytes) {
  if (c->rec) {
    rec_op(c->rec, [dst, src, bytes](cudaStream_t s, cusolverDnHandle_t) {
      TTG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, s));
    });
    return;
  }
  TTG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToDevice, c->stream));
}

void solver_call(Context* c, const StreamOp& op) {
  if (c->rec) {
    rec_op(c->rec, op);
    return;
  }
  op(c->stream, c->solver);
}

}  // namespace ttg

using namespace ttg;

// ---------------------------------------------------------------------------
// C ABI: library, context, memory
// ---------------------------------------------------------------------------

extern "C" {

const char* ttg_last_error(void) { return g_last_error.c_str(); }

int ttg_version(void) { return 10000; }

int ttg_context_create(int device, ttg_context* out) {
  TTG_API_BEGIN
  TTG_REQUIRE(out != nullptr, "out is NULL");
  int ndev = 0;
  TTG_CUDA(cudaGetDeviceCount(&ndev));
  TTG_REQUIRE(device >= 0 && device < ndev, "device %d out of range (%d devices)", device, ndev);
  TTG_CUDA(cudaSetDevice(device));
  std::unique_ptr<ttg_context_s> h(new ttg_context_s());
  try {
    context_init(h->c, device);
  } catch (...) {
    context_release(h->c);
    throw;
  }
  *out = h.release();
  TTG_API_END
}

int ttg_context_destroy(ttg_context ctx) {
  TTG_API_BEGIN
  if (!ctx) return TTG_OK;
  cudaSetDevice(ctx->c.device);
  {
    std::lock_guard<std::mutex> lock(ctx->mu);
    for (auto& w : ctx->workers) context_release(*w);
    ctx->workers.clear();
  }
  context_release(ctx->c);
  delete ctx;
  TTG_API_END
}

int ttg_context_sync(ttg_context ctx) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx, "ctx is NULL");
  TTG_CUDA(cudaSetDevice(ctx->c.device));
  sync(&ctx->c);
  TTG_API_END
}

int ttg_malloc(ttg_context ctx, size_t bytes, void** out) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx && out, "NULL argument");
  TTG_CUDA(cudaSetDevice(ctx->c.device));
  *out = nullptr;
  if (bytes) {
    cudaError_t e = cudaMalloc(out, bytes);
    if (e != cudaSuccess) {
      cudaGetLastError();
      fail(TTG_ERR_ALLOC, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
    }
  }
  TTG_API_END
}

int ttg_free(ttg_context ctx, void* p) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx, "ctx is NULL");
  TTG_CUDA(cudaSetDevice(ctx->c.device));
  if (p) {
    sync(&ctx->c);
    TTG_CUDA(cudaFree(p));
  }
  TTG_API_END
}

int ttg_memcpy_h2d(ttg_context ctx, void* dst, const void* src, size_t bytes) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx, "ctx is NULL");
  TTG_REQUIRE(bytes == 0 || (dst && src), "NULL pointer");
  TTG_CUDA(cudaSetDevice(ctx->c.device));
  if (bytes) {
    TTG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, ctx->c.stream));
    sync(&ctx->c);
  }
  TTG_API_END
}

int ttg_memcpy_d2h(ttg_context ctx, void* dst, const void* src, size_t bytes) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx, "ctx is NULL");
  TTG_REQUIRE(bytes == 0 || (dst && src), "NULL pointer");
  TTG_CUDA(cudaSetDevice(ctx->c.device));
  if (bytes) {
    TTG_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, ctx->c.stream));
    sync(&ctx->c);
  }
  TTG_API_END
}

int ttg_memset(ttg_context ctx, void* dst, int value, size_t bytes) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx, "ctx is NULL");
  TTG_REQUIRE(bytes == 0 || dst, "NULL pointer");
  TTG_CUDA(cudaSetDevice(ctx->c.device));
  if (bytes) {
    TTG_CUDA(cudaMemsetAsync(dst, value, bytes, ctx->c.stream));
    sync(&ctx->c);
  }
  TTG_API_END
}

int ttg_launch_count(ttg_context ctx, int64_t* out) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx && out, "NULL argument");
  *out = ctx->c.launches;
  TTG_API_END
}

// ---------------------------------------------------------------------------
// C ABI: TT handles
// ---------------------------------------------------------------------------

int ttg_tt_upload(ttg_context ctx, int64_t d, const int64_t* n, const int64_t* m,
                  const int64_t* r, const double* core, ttg_tt* out) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx && n && r && core && out, "NULL argument");
  TTG_REQUIRE(d >= 1 && d <= 4096, "d = %lld out of range", (long long)d);
  Context* c = &ctx->c;
  TTG_CUDA(cudaSetDevice(c->device));
  auto* t = new ttg_tt_s();
  t->ctx = c;
  t->d = d;
  t->is_matrix = (m != nullptr);
  t->n.assign(n, n + d);
  if (m) t->m.assign(m, m + d);
  t->r.assign(r, r + d + 1);
  t->ps.assign(d + 1, 0);
  for (int64_t k = 0; k < d; ++k) {
    if (n[k] < 1 || (m && m[k] < 1) || r[k] < 1 || r[k + 1] < 1) {
      delete t;
      fail(TTG_ERR_INVALID, "non-positive size at core %lld", (long long)k);
    }
    int64_t sz = r[k] * n[k] * (m ? m[k] : 1) * r[k + 1];
    t->ps[k + 1] = t->ps[k] + sz;
  }
  t->numel = t->ps[d];
  t->core = static_cast<double*>(c->alloc->get(sizeof(double) * t->numel));
  TTG_CUDA(cudaMemcpyAsync(t->core, core, sizeof(double) * t->numel, cudaMemcpyHostToDevice,
                           c->stream));
  sync(c);
  *out = t;
  TTG_API_END
}

int ttg_tt_shape(ttg_tt t, int64_t* d, int64_t* n, int64_t* m, int64_t* r, int64_t* numel) {
  TTG_API_BEGIN
  TTG_REQUIRE(t, "NULL handle");
  if (d) *d = t->d;
  if (n) memcpy(n, t->n.data(), sizeof(int64_t) * t->d);
  if (m) {
    if (t->is_matrix)
      memcpy(m, t->m.data(), sizeof(int64_t) * t->d);
    else
      memcpy(m, t->n.data(), sizeof(int64_t) * t->d);
  }
  if (r) memcpy(r, t->r.data(), sizeof(int64_t) * (t->d + 1));
  if (numel) *numel = t->numel;
  TTG_API_END
}

int ttg_tt_download(ttg_tt t, double* core) {
  TTG_API_BEGIN
  TTG_REQUIRE(t && core, "NULL argument");
  TTG_CUDA(cudaSetDevice(t->ctx->device));
  TTG_CUDA(cudaMemcpyAsync(core, t->core, sizeof(double) * t->numel, cudaMemcpyDeviceToHost,
                           t->ctx->stream));
  sync(t->ctx);
  TTG_API_END
}

int ttg_tt_free(ttg_tt t) {
  TTG_API_BEGIN
  if (!t) return TTG_OK;
  cudaSetDevice(t->ctx->device);
  cudaStreamSynchronize(t->ctx->stream);
  t->ctx->alloc->put(t->core);
  delete t;
  TTG_API_END
}

}  // extern "C"
