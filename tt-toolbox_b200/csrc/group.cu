// Executor of grouped batches: many independent solves advance together on
// one stream, and launches of the same kernel are merged into one launch.
//
// Each solve runs the ordinary host code on a fiber of its own (a few host
// worker threads resume the fibers in turn) with a recording context
// (Context::rec): launches, memsets, copies and library
// calls are appended to the solve's record instead of being issued, and
// device blocks it frees are kept for its own later allocations (reused in
// its own record order), going back to the allocator when the batch ends.  A solve that needs a device result (a host
// read or a synchronisation) blocks.  Once every running solve is blocked,
// the executor "flushes": it merges the records of all solves, issues them
// on the stream and waits for the device, then wakes the solves, which go on
// recording from where they stopped.
//
// Merging keeps each solve's own order.  The executor repeatedly looks at
// the first unissued record of every solve: stream operations are issued
// one by one; among the launches of TTG_KERNEL kernels it picks the kernel
// (and block shape) at the head of the most solves and issues one grouped
// launch over all of them (group.cuh).  Records of different solves touch
// disjoint memory, so any interleaving that keeps every solve's order gives
// each solve the results of its own sequential run.  The argument packs,
// launch headers and CTA maps of a flush are written to one pinned staging
// buffer and copied to the device with a single copy before the launches.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <tuple>
#include <vector>

#include <sys/mman.h>
#include <ucontext.h>
#include <unistd.h>

#include "group.cuh"

namespace ttg {

namespace {

struct RecOp {
  const GroupInfo* info;  // null: a stream operation (Recorder::closures[closure])
  dim3 grid, block;
  uint32_t smem;
  uint32_t pack_off;      // argument pack in Recorder::arena
  uint32_t closure;
  double flop;            // > 0: a tensor-core GEMM of that many FLOPs
};

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

struct Member {  // one recorded launch of a grouped step
  Recorder* r;
  uint32_t op;
};
struct Step {
  bool group;       // false: a stream operation (r, op)
  Recorder* r;
  uint32_t op;
  size_t first, n;  // grouped step: members[first, first + n)
};
struct Launch {  // one grouped launch (a cooperative step may need several)
  size_t lane, step;
  size_t first, n;
  uint32_t ctas, smem;
  size_t map_off, hdr_off, pack_off;
  uint32_t stride;
};

// TTG_GROUP=0 issues every recorded launch on its own (plain kernels, in the
// merged order): the grouped launches can then be compared with it.
// TTG_GROUP_COOP=0 does so for the cooperative kernels only.
bool env_on(const char* name) {
  const char* e = getenv(name);
  return !(e && e[0] == '0');
}

}  // namespace

// Stream operations of a recording context, as grouped kernels: a memset,
// and a read of device bytes into the context's mapped pinned buffer (the
// host sees the bytes once the flush has synchronised the stream).
TTG_BODY(k_fill_bytes)(TTG_BLOCK, unsigned char* p, int value, int64_t bytes) {
  pdl_begin();
  const int64_t stride = int64_t(gridDim.x) * blockDim.x;
  const int64_t t0 = int64_t(blockIdx.x) * blockDim.x + threadIdx.x;
  if ((reinterpret_cast<uintptr_t>(p) & 15) == 0) {
    const unsigned char b = static_cast<unsigned char>(value);
    const unsigned w = b * 0x01010101u;
    const uint4 v = make_uint4(w, w, w, w);
    const int64_t n16 = bytes / 16;
    for (int64_t i = t0; i < n16; i += stride) reinterpret_cast<uint4*>(p)[i] = v;
    for (int64_t i = n16 * 16 + t0; i < bytes; i += stride) p[i] = b;
  } else {
    for (int64_t i = t0; i < bytes; i += stride) p[i] = static_cast<unsigned char>(value);
  }
}
TTG_KERNEL(k_fill_bytes, 0);

TTG_BODY(k_read_host)(TTG_BLOCK, const unsigned char* src, unsigned char* dst, int64_t bytes) {
  pdl_begin();
  for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < bytes;
       i += int64_t(gridDim.x) * blockDim.x)
    dst[i] = src[i];
  __threadfence_system();
}
TTG_KERNEL(k_read_host, 0);

class Executor;

// A solve of a grouped batch runs on a fiber: its own stack and machine
// context, resumed by one host worker thread until it waits for the device
// (then it switches back to the worker) or its solves are done.  Many
// fibers share a worker, so a flush wakes a few threads, not one per solve.
struct Fiber {
  ucontext_t ctx;
  char* stack = nullptr;
  size_t stack_size = 0;
  Executor* ex = nullptr;
  int worker = 0;
  int slot = 0;  // recorder and context of this fiber
  bool done = false;
};

struct Recorder {
  Executor* ex = nullptr;
  Fiber* fiber = nullptr;
  std::vector<RecOp> ops;
  std::vector<StreamOp> closures;
  std::vector<char> arena;
  // Device blocks this solve freed, by size class, for its own reuse.
  std::unordered_map<size_t, std::vector<void*>> cache;
  // Tensor-core GEMMs recorded (less those the solve later found skipped).
  double tc_flop = 0.0;
  int64_t tc_records = 0;
};

// Plan of one lane: the lane's records in issue order.  Stream operations at
// the head of a solve go first, one by one; then the kernel (and block
// shape) at the head of the most solves becomes one grouped step over all
// of them; repeat.
namespace {

void plan_lane(const std::vector<Recorder*>& R, std::vector<Step>& steps,
               std::vector<Member>& members) {
  size_t remaining = 0;
  for (Recorder* r : R) remaining += r->ops.size();
  std::vector<size_t> head(R.size(), 0);
  struct Key {
    const GroupInfo* info;
    dim3 block;
    int count;
  };
  auto same = [](const RecOp& o, const GroupInfo* info, dim3 block) {
    return o.info == info && o.block.x == block.x && o.block.y == block.y &&
           o.block.z == block.z;
  };
  std::vector<Key> keys;
  while (remaining) {
    for (size_t q = 0; q < R.size(); ++q) {
      auto& ops = R[q]->ops;
      while (head[q] < ops.size() && !ops[head[q]].info) {
        steps.push_back(Step{false, R[q], uint32_t(head[q]), 0, 0});
        ++head[q];
        --remaining;
      }
    }
    if (!remaining) break;
    keys.clear();
    for (size_t q = 0; q < R.size(); ++q) {
      if (head[q] >= R[q]->ops.size()) continue;
      const RecOp& o = R[q]->ops[head[q]];
      bool found = false;
      for (auto& k : keys)
        if (same(o, k.info, k.block)) {
          ++k.count;
          found = true;
          break;
        }
      if (!found) keys.push_back(Key{o.info, o.block, 1});
    }
    const Key* best = &keys[0];
    for (auto& k : keys)
      if (k.count > best->count) best = &k;
    const Key kb = *best;
    Step g{true, nullptr, 0, members.size(), 0};
    for (size_t q = 0; q < R.size(); ++q) {
      if (head[q] >= R[q]->ops.size()) continue;
      if (same(R[q]->ops[head[q]], kb.info, kb.block)) {
        members.push_back(Member{R[q], uint32_t(head[q])});
        ++head[q];
        --remaining;
      }
    }
    g.n = members.size() - g.first;
    steps.push_back(g);
  }
}

// Lanes: solves whose records are the same sequence of kernels (the same
// phase of the sweep) share a lane, so that their launches merge step by
// step; the largest clusters get lanes of their own, the others are dealt
// round-robin.  Each lane is issued on its own stream.
std::vector<std::vector<Recorder*>> make_lanes(const std::vector<Recorder*>& R, size_t max_lanes) {
  std::map<uint64_t, std::vector<Recorder*>> clusters;
  for (Recorder* r : R) {
    uint64_t h = 1469598103934665603ull;
    for (const RecOp& o : r->ops) {
      h = (h ^ uint64_t(reinterpret_cast<uintptr_t>(o.info))) * 1099511628211ull;
      h = (h ^ uint64_t(o.block.x)) * 1099511628211ull;
    }
    clusters[h].push_back(r);
  }
  std::vector<std::vector<Recorder*>*> cl;
  for (auto& kv : clusters) cl.push_back(&kv.second);
  std::stable_sort(cl.begin(), cl.end(),
                   [](const std::vector<Recorder*>* a, const std::vector<Recorder*>* b) {
                     return a->size() > b->size();
                   });
  const size_t nl = std::max<size_t>(1, std::min(max_lanes, cl.size()));
  std::vector<std::vector<Recorder*>> lanes(nl);
  for (size_t c = 0; c < cl.size(); ++c)
    lanes[c % nl].insert(lanes[c % nl].end(), cl[c]->begin(), cl[c]->end());
  return lanes;
}

// Host threads that issue the lanes of a flush in parallel (each lane on its
// own stream, so their launches need no order between them).
class IssuePool {
 public:
  IssuePool(int nthreads, int device) : device_(device) {
    for (int t = 0; t < nthreads; ++t) th_.emplace_back(&IssuePool::loop, this);
  }
  ~IssuePool() {
    {
      std::lock_guard<std::mutex> lk(mu_);
      stop_ = true;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  // fn(j) for every j < jobs, on the pool and the calling thread; returns
  // the first error message ("" when none).
  std::string run(size_t jobs, const std::function<void(size_t)>& fn) {
    {
      std::lock_guard<std::mutex> lk(mu_);
      fn_ = &fn;
      jobs_ = jobs;
      next_ = 0;
      active_ = int(th_.size());
      err_.clear();
      ++gen_;
    }
    cv_.notify_all();
    work();
    std::unique_lock<std::mutex> lk(mu_);
    cv_done_.wait(lk, [&] { return active_ == 0; });
    return err_;
  }

 private:
  void work() {
    for (;;) {
      const size_t j = next_.fetch_add(1);
      if (j >= jobs_) return;
      try {
        (*fn_)(j);
      } catch (const Error& e) {
        std::lock_guard<std::mutex> lk(mu_);
        if (err_.empty()) err_ = e.msg;
      }
    }
  }
  void loop() {
    cudaSetDevice(device_);
    uint64_t seen = 0;
    for (;;) {
      {
        std::unique_lock<std::mutex> lk(mu_);
        cv_.wait(lk, [&] { return gen_ != seen || stop_; });
        if (stop_) return;
        seen = gen_;
      }
      work();
      std::lock_guard<std::mutex> lk(mu_);
      if (--active_ == 0) cv_done_.notify_one();
    }
  }
  int device_;
  std::vector<std::thread> th_;
  std::mutex mu_;
  std::condition_variable cv_, cv_done_;
  const std::function<void(size_t)>* fn_ = nullptr;
  size_t jobs_ = 0;
  std::atomic<size_t> next_{0};
  int active_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
  std::string err_;
};

}  // namespace

class Executor {
 public:
  Executor(Context* owner, int width);
  ~Executor();
  void run(int64_t count, const std::function<void(int64_t, Context*)>& body);
  void wait(Recorder* r);
  void fiber_main(Fiber* f);
  // Device blocks of the fibers of one worker thread (no lock: touched by
  // that thread while recording and by the executor while the workers wait).
  std::unordered_map<size_t, std::vector<void*>>& pool(int w) { return pools_[w]; }
  ttg_group_stats st{};

 private:
  void worker_loop(int w);
  void flush();
  int coop_capacity(const GroupInfo* info, dim3 block, size_t smem);
  void ensure_stage(size_t bytes);

  Context* owner_;
  int width_;
  std::vector<std::unique_ptr<Recorder>> recs_;
  std::vector<std::unique_ptr<Context>> ctxs_;
  double* h_slab_ = nullptr;
  int* d_err_slab_ = nullptr;
  unsigned* d_tile_slab_ = nullptr;
  char* h_stage_ = nullptr;
  char* d_stage_ = nullptr;
  // Streams of the lanes (lanes_[0] is the owner's stream) and the event that
  // orders every lane after the copy of the argument packs.
  std::vector<cudaStream_t> lanes_;
  cudaEvent_t stage_ev_ = nullptr;
  std::unique_ptr<IssuePool> pool_;
  std::mutex closure_mu_;  // stream operations (library calls share one handle)
  size_t stage_cap_ = 0;
  std::map<std::tuple<const void*, unsigned, size_t>, int> occ_;
  const bool group_on_ = env_on("TTG_GROUP");
  // TTG_GROUP_TIME=1: CUDA events around every tensor-core GEMM launch.
  const bool time_tc_ = [] {
    const char* e = getenv("TTG_GROUP_TIME");
    return e && e[0] == '1';
  }();
  std::vector<std::vector<cudaEvent_t>> tc_ev_;  // per lane: pairs, reused
  const bool group_coop_ = env_on("TTG_GROUP_COOP");
  std::string group_skip_ = getenv("TTG_GROUP_SKIP") ? getenv("TTG_GROUP_SKIP") : "";
  std::map<const GroupInfo*, bool> groupable_;
  bool groupable(const GroupInfo* info) {
    if (!group_on_ || (info->coop && !group_coop_)) return false;
    if (group_skip_.empty()) return true;
    auto it = groupable_.find(info);
    if (it != groupable_.end()) return it->second;
    const char* name = "";
    cudaFuncGetName(&name, info->plain);
    bool ok = true;
    size_t b = 0;
    while (b <= group_skip_.size()) {
      size_t e = group_skip_.find(',', b);
      if (e == std::string::npos) e = group_skip_.size();
      const std::string tok = group_skip_.substr(b, e - b);
      if (!tok.empty() && name && strstr(name, tok.c_str())) ok = false;
      b = e + 1;
    }
    groupable_[info] = ok;
    return ok;
  }

  // Fibers, the worker threads' own contexts, and the batch being run.
  std::vector<std::unique_ptr<Fiber>> fibers_;
  std::vector<std::unique_ptr<ucontext_t>> worker_ctx_;
  std::vector<std::unordered_map<size_t, std::vector<void*>>> pools_;
  int nworkers_ = 0;
  std::atomic<int64_t> next_{0};
  int64_t count_ = 0;
  uint64_t gets0_ = 0, mallocs0_ = 0;
  double ms_get0_ = 0.0;
  const std::function<void(int64_t, Context*)>* body_ = nullptr;

  std::mutex mu_;
  std::condition_variable cv_main_, cv_sys_;
  int idle_ = 0;      // workers whose fibers are all waiting or done
  bool stop_ = false;
  uint64_t epoch_ = 0;
  bool failed_ = false;
  int fail_code_ = TTG_OK;
  std::string fail_msg_;
};

Executor::Executor(Context* owner, int width) : owner_(owner), width_(width) {
  TTG_CUDA(cudaHostAlloc(&h_slab_, sizeof(double) * 4096 * size_t(width), cudaHostAllocMapped));
  double* h_slab_dev = nullptr;
  TTG_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void**>(&h_slab_dev), h_slab_, 0));
  TTG_CUDA(cudaMalloc(&d_err_slab_, sizeof(int) * 64 * size_t(width)));
  TTG_CUDA(cudaMemset(d_err_slab_, 0, sizeof(int) * 64 * size_t(width)));
  TTG_CUDA(cudaMalloc(&d_tile_slab_, sizeof(unsigned) * GEMM_TILE_COUNTERS * size_t(width)));
  TTG_CUDA(cudaMemset(d_tile_slab_, 0, sizeof(unsigned) * GEMM_TILE_COUNTERS * size_t(width)));
  TTG_CUDA(cudaDeviceSynchronize());
  // TTG_GROUP_LANES (default 16): streams the phase clusters are issued on.
  int nlanes = 16;
  if (const char* e = getenv("TTG_GROUP_LANES")) nlanes = std::max(1, std::min(64, atoi(e)));
  lanes_.push_back(owner->stream);
  for (int l = 1; l < nlanes; ++l) {
    cudaStream_t st = nullptr;
    TTG_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    lanes_.push_back(st);
  }
  TTG_CUDA(cudaEventCreateWithFlags(&stage_ev_, cudaEventDisableTiming));
  {
    const int hw = std::max(2, int(std::thread::hardware_concurrency()));
    pool_.reset(new IssuePool(std::min(nlanes - 1, std::min(7, hw / 2 - 1)), owner->device));
  }
  for (int k = 0; k < width; ++k) {
    recs_.emplace_back(new Recorder());
    recs_.back()->ex = this;
    std::unique_ptr<Context> c(new Context());
    c->device = owner->device;
    c->num_sms = owner->num_sms;
    c->stream = owner->stream;
    c->solver = nullptr;
    c->alloc = owner->alloc;
    c->h_scal = h_slab_ + size_t(k) * 4096;
    c->h_scal_dev = h_slab_dev + size_t(k) * 4096;
    c->d_err = d_err_slab_ + size_t(k) * 64;
    c->d_tile_cnt = d_tile_slab_ + size_t(k) * GEMM_TILE_COUNTERS;
    c->pdl = owner->pdl;
    c->jacobi_max_sweeps = owner->jacobi_max_sweeps;
    c->rec = recs_.back().get();
    ctxs_.push_back(std::move(c));
  }
}

Executor::~Executor() {
  for (cudaStream_t st : lanes_) cudaStreamSynchronize(st);
  for (auto& v : tc_ev_)
    for (cudaEvent_t e : v) cudaEventDestroy(e);
  for (size_t l = 1; l < lanes_.size(); ++l) cudaStreamDestroy(lanes_[l]);
  if (stage_ev_) cudaEventDestroy(stage_ev_);
  if (h_slab_) cudaFreeHost(h_slab_);
  if (d_err_slab_) cudaFree(d_err_slab_);
  if (d_tile_slab_) cudaFree(d_tile_slab_);
  if (h_stage_) cudaFreeHost(h_stage_);
  if (d_stage_) cudaFree(d_stage_);
}

void Executor::ensure_stage(size_t bytes) {
  if (bytes <= stage_cap_) return;
  size_t cap = std::max<size_t>(bytes + bytes / 2, size_t(8) << 20);
  // Called at the start of a flush: the stream is idle.
  if (h_stage_) cudaFreeHost(h_stage_);
  if (d_stage_) cudaFree(d_stage_);
  h_stage_ = nullptr;
  d_stage_ = nullptr;
  stage_cap_ = 0;
  TTG_CUDA(cudaMallocHost(&h_stage_, cap));
  TTG_CUDA(cudaMalloc(&d_stage_, cap));
  stage_cap_ = cap;
}

int Executor::coop_capacity(const GroupInfo* info, dim3 block, size_t smem) {
  const auto key = std::make_tuple(info->group, block.x * block.y * block.z, smem);
  auto it = occ_.find(key);
  if (it != occ_.end()) return it->second;
  int occ = 0;
  TTG_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(
      &occ, info->group, int(block.x * block.y * block.z), smem));
  const int cap = std::max(0, occ) * owner_->num_sms;
  occ_[key] = cap;
  return cap;
}

void Executor::wait(Recorder* r) {
  Fiber* f = r->fiber;
  // Back to the worker; resumed after the flush that issued this record.
  swapcontext(&f->ctx, worker_ctx_[f->worker].get());
  if (failed_) throw Error{fail_code_, fail_msg_};
}

namespace {
// makecontext passes int arguments: the fiber's address in two halves.
void fiber_entry(unsigned lo, unsigned hi) {
  Fiber* f = reinterpret_cast<Fiber*>((uintptr_t(hi) << 32) | uintptr_t(lo));
  f->ex->fiber_main(f);
}
}  // namespace

void Executor::fiber_main(Fiber* f) {
  Context* c = ctxs_[f->slot].get();
  for (;;) {
    const int64_t i = next_.fetch_add(1);
    if (i >= count_) break;
    try {
      (*body_)(i, c);
    } catch (...) {  // the body reports its own failures
    }
  }
  f->done = true;
  // A fiber never returns (its context has no successor): the worker does
  // not resume a finished fiber.
  swapcontext(&f->ctx, worker_ctx_[f->worker].get());
}

void Executor::worker_loop(int w) {
  cudaSetDevice(owner_->device);
  uint64_t seen = 0;
  for (;;) {
    for (auto& f : fibers_)
      if (f->worker == w && !f->done) swapcontext(worker_ctx_[w].get(), &f->ctx);
    std::unique_lock<std::mutex> lk(mu_);
    if (++idle_ == nworkers_) cv_main_.notify_one();
    cv_sys_.wait(lk, [&] { return epoch_ != seen || stop_; });
    seen = epoch_;
    if (stop_) return;
  }
}

void Executor::run(int64_t count, const std::function<void(int64_t, Context*)>& body) {
  const int nfib = int(std::min<int64_t>(width_, count));
  const int hw = std::max(1, int(std::thread::hardware_concurrency()));
  nworkers_ = std::max(1, std::min(nfib, hw));
  count_ = count;
  body_ = &body;
  gets0_ = owner_->alloc->gets();
  mallocs0_ = owner_->alloc->mallocs();
  ms_get0_ = owner_->alloc->ms_get();
  next_ = 0;
  const size_t page = size_t(sysconf(_SC_PAGESIZE));
  const size_t stack_size = size_t(2) << 20;
  for (int k = 0; k < nfib; ++k) {
    std::unique_ptr<Fiber> f(new Fiber());
    void* mem = mmap(nullptr, stack_size, PROT_READ | PROT_WRITE,
                     MAP_PRIVATE | MAP_ANONYMOUS | MAP_NORESERVE | MAP_STACK, -1, 0);
    if (mem == MAP_FAILED) fail(TTG_ERR_ALLOC, "grouped batch: no memory for a fiber stack");
    mprotect(mem, page, PROT_NONE);  // guard page below the stack
    f->stack = static_cast<char*>(mem);
    f->stack_size = stack_size;
    f->ex = this;
    f->slot = k;
    f->worker = k % nworkers_;
    getcontext(&f->ctx);
    f->ctx.uc_stack.ss_sp = f->stack + page;
    f->ctx.uc_stack.ss_size = stack_size - page;
    f->ctx.uc_link = nullptr;
    const uintptr_t a = reinterpret_cast<uintptr_t>(f.get());
    makecontext(&f->ctx, reinterpret_cast<void (*)()>(fiber_entry), 2, unsigned(a & 0xffffffffu),
                unsigned(a >> 32));
    recs_[k]->fiber = f.get();
    fibers_.push_back(std::move(f));
  }
  for (int w = 0; w < nworkers_; ++w) worker_ctx_.emplace_back(new ucontext_t());
  pools_.resize(nworkers_);
  {
    const int share = owner_->group_sms > 0
                          ? std::min(owner_->group_sms, owner_->num_sms)
                          : std::max(1, 2 * owner_->num_sms / std::max(1, nfib));
    for (auto& c : ctxs_) c->num_sms = share;
  }
  std::vector<std::thread> th;
  th.reserve(nworkers_);
  for (int w = 0; w < nworkers_; ++w) th.emplace_back(&Executor::worker_loop, this, w);
  {
    std::unique_lock<std::mutex> lk(mu_);
    auto t_wake = std::chrono::steady_clock::now();
    for (;;) {
      cv_main_.wait(lk, [&] { return idle_ == nworkers_; });
      st.ms_record += std::chrono::duration<double, std::milli>(
                          std::chrono::steady_clock::now() - t_wake).count();
      int live = 0;
      for (auto& f : fibers_) live += f->done ? 0 : 1;
      // Per-solve share of the SMs for the grids the solves size themselves
      // (cooperative Krylov grids, split-K slices, grid-stride loops): the
      // grouped launches fill the device across solves.
      const int share =
          owner_->group_sms > 0
              ? std::min(owner_->group_sms, owner_->num_sms)
              : std::max(1, std::min(owner_->num_sms, 2 * owner_->num_sms / std::max(1, live)));
      for (auto& c : ctxs_) c->num_sms = share;
      lk.unlock();
      try {
        flush();
      } catch (const Error& e) {
        for (auto& r : recs_) {  // nothing recorded so far is issued again
          r->ops.clear();
          r->closures.clear();
          r->arena.clear();
        }
        lk.lock();
        if (!failed_) {
          failed_ = true;
          fail_code_ = e.code;
          fail_msg_ = e.msg;
        }
        lk.unlock();
      }
      lk.lock();
      idle_ = 0;
      ++epoch_;
      t_wake = std::chrono::steady_clock::now();
      if (live == 0) stop_ = true;
      cv_sys_.notify_all();
      if (live == 0) break;
    }
  }
  for (auto& t : th) t.join();
  for (auto& f : fibers_) munmap(f->stack, f->stack_size);
  for (auto& r : recs_) {
    st.tc_gflop += r->tc_flop * 1e-9;
    st.tc_records += r->tc_records;
  }
  st.allocs = int64_t(owner_->alloc->gets() - gets0_);
  st.device_mallocs = int64_t(owner_->alloc->mallocs() - mallocs0_);
  st.ms_alloc = owner_->alloc->ms_get() - ms_get0_;
  for (auto& r : recs_) {  // every record is issued and complete
    for (auto& kv : r->cache)
      for (void* p : kv.second) owner_->alloc->put(p);
    r->cache.clear();
  }
  for (auto& pl : pools_)
    for (auto& kv : pl)
      for (void* p : kv.second) owner_->alloc->put(p);
  pools_.clear();
  if (failed_) fail(fail_code_, "grouped batch: %s", fail_msg_.c_str());
}

void Executor::flush() {
  const auto t0 = std::chrono::steady_clock::now();
  st.flushes += 1;
  std::vector<Recorder*> R;
  for (auto& r : recs_)
    if (!r->ops.empty()) {
      R.push_back(r.get());
      st.records += int64_t(r->ops.size());
    }
  const std::vector<std::vector<Recorder*>> laneR = make_lanes(R, lanes_.size());
  const size_t nl = laneR.size();
  std::vector<std::vector<Step>> steps(nl);
  std::vector<Member> members;
  for (size_t l = 0; l < nl; ++l) plan_lane(laneR[l], steps[l], members);

  // ---- launches: split cooperative groups by residency, lay out staging
  std::vector<Launch> launches;
  std::vector<std::vector<size_t>> launch_of_step(nl);
  std::vector<std::vector<char>> grouped(nl);  // step issued as grouped launches
  size_t bytes = 0;
  auto ctas_of = [](const RecOp& o) -> uint64_t {
    return uint64_t(o.grid.x) * o.grid.y * o.grid.z;
  };
  for (size_t l = 0; l < nl; ++l) {
    launch_of_step[l].assign(steps[l].size(), SIZE_MAX);
    grouped[l].assign(steps[l].size(), 0);
    for (size_t si = 0; si < steps[l].size(); ++si) {
      const Step& sp = steps[l][si];
      if (!sp.group) continue;
      const RecOp& o0 = members[sp.first].r->ops[members[sp.first].op];
      if (sp.n == 1 || !groupable(o0.info)) continue;  // plain launches
      grouped[l][si] = 1;
      uint32_t smem = 0;
      for (size_t m = sp.first; m < sp.first + sp.n; ++m)
        smem = std::max(smem, members[m].r->ops[members[m].op].smem);
      uint64_t cap = UINT32_MAX / 2;
      // Cooperative grids of all lanes may run at once: each lane keeps to
      // its share of the resident CTAs.
      if (o0.info->coop)
        cap = uint64_t(std::max<int64_t>(1, coop_capacity(o0.info, o0.block, smem) / int64_t(nl)));
      const uint32_t stride =
          uint32_t(align_up(o0.info->pack_size, std::max<uint32_t>(16, o0.info->pack_align)));
      size_t m = sp.first;
      launch_of_step[l][si] = launches.size();
      while (m < sp.first + sp.n) {
        Launch L{l, si, m, 0, 0, smem, 0, 0, 0, stride};
        uint64_t ctas = 0;
        while (m < sp.first + sp.n) {
          const uint64_t k = ctas_of(members[m].r->ops[members[m].op]);
          if (L.n > 0 && ctas + k > cap) break;
          ctas += k;
          ++L.n;
          ++m;
        }
        L.ctas = uint32_t(ctas);
        bytes = align_up(bytes, 256);
        L.map_off = bytes;
        bytes += sizeof(uint32_t) * ctas;
        bytes = align_up(bytes, 256);
        L.hdr_off = bytes;
        bytes += sizeof(uint4) * L.n;
        bytes = align_up(bytes, 256);
        L.pack_off = bytes;
        bytes += size_t(stride) * L.n;
        launches.push_back(L);
      }
    }
  }
  ensure_stage(bytes + 256);
  for (auto& L : launches) {
    uint32_t* map = reinterpret_cast<uint32_t*>(h_stage_ + L.map_off);
    uint4* hdr = reinterpret_cast<uint4*>(h_stage_ + L.hdr_off);
    char* packs = h_stage_ + L.pack_off;
    uint32_t cta = 0;
    for (size_t j = 0; j < L.n; ++j) {
      const Member& mb = members[L.first + j];
      const RecOp& o = mb.r->ops[mb.op];
      const uint32_t k = uint32_t(ctas_of(o));
      hdr[j] = make_uint4(cta, o.grid.x, o.grid.y, o.grid.z);
      for (uint32_t b = 0; b < k; ++b) map[cta + b] = uint32_t(j);
      cta += k;
      memcpy(packs + size_t(L.stride) * j, mb.r->arena.data() + o.pack_off, o.info->pack_size);
    }
  }
  const auto t1 = std::chrono::steady_clock::now();
  st.ms_plan += std::chrono::duration<double, std::milli>(t1 - t0).count();

  // ---- issue: one copy of the packs, then the lanes' steps interleaved
  // across their streams (each lane in its own order).
  cudaStream_t s0 = lanes_[0];
  if (bytes) TTG_CUDA(cudaMemcpyAsync(d_stage_, h_stage_, bytes, cudaMemcpyHostToDevice, s0));
  TTG_CUDA(cudaEventRecord(stage_ev_, s0));
  for (size_t l = 1; l < nl; ++l) TTG_CUDA(cudaStreamWaitEvent(lanes_[l], stage_ev_, 0));
  std::vector<int64_t> lane_launches(nl, 0), lane_grouped(nl, 0), lane_tc(nl, 0);
  if (time_tc_ && tc_ev_.size() < nl) tc_ev_.resize(nl);
  // tc_begin / tc_end bracket a tensor-core GEMM launch on lane l (events
  // only when timing is on; lane_tc counts the pairs used this flush).
  auto tc_begin = [&](size_t l, cudaStream_t s) {
    if (!time_tc_) return;
    auto& v = tc_ev_[l];
    const size_t k = size_t(lane_tc[l]) * 2;
    while (v.size() < k + 2) {
      cudaEvent_t e = nullptr;
      TTG_CUDA(cudaEventCreate(&e));
      v.push_back(e);
    }
    TTG_CUDA(cudaEventRecord(v[k], s));
  };
  auto tc_end = [&](size_t l, cudaStream_t s) {
    if (time_tc_) TTG_CUDA(cudaEventRecord(tc_ev_[l][size_t(lane_tc[l]) * 2 + 1], s));
    lane_tc[l] += 1;
  };
  auto issue_step = [&](size_t l, size_t si) {
    cudaStream_t s = lanes_[l];
    const Step& sp = steps[l][si];
    if (!sp.group) {  // library calls go on the lane's stream
      std::lock_guard<std::mutex> lk(closure_mu_);
      if (owner_->solver) TTG_SOLVER(cusolverDnSetStream(owner_->solver, s));
      sp.r->closures[sp.r->ops[sp.op].closure](s, owner_->solver);
      if (owner_->solver) TTG_SOLVER(cusolverDnSetStream(owner_->solver, owner_->stream));
      lane_launches[l] += 1;
      return;
    }
    const RecOp& o0 = members[sp.first].r->ops[members[sp.first].op];
    const GroupInfo* info = o0.info;
    auto plain_one = [&](const Member& mb) {
      const RecOp& o = mb.r->ops[mb.op];
      if (o.flop > 0) tc_begin(l, s);
      info->issue(mb.r->arena.data() + o.pack_off, o.grid, o.block, o.smem, s, owner_->pdl);
      if (o.flop > 0) tc_end(l, s);
      lane_launches[l] += 1;
    };
    if (!grouped[l][si]) {
      for (size_t m = sp.first; m < sp.first + sp.n; ++m) plain_one(members[m]);
      return;
    }
    lane_grouped[l] += int64_t(sp.n);
    for (size_t li = launch_of_step[l][si];
         li < launches.size() && launches[li].lane == l && launches[li].step == si; ++li) {
      const Launch& L = launches[li];
      if (L.n == 1) {  // one launch alone (a cooperative grid at its residency share)
        plain_one(members[L.first]);
        continue;
      }
      // The limit without opt-in is 48 KB of static plus dynamic shared
      // memory: a body with static arrays needs the attribute below 48 KB
      // of dynamic memory already (memoised, so set once per size).
      if (L.smem > 0) ensure_smem_attr(info->group, owner_->device, int(L.smem));
      GroupArgs ga{reinterpret_cast<const uint32_t*>(d_stage_ + L.map_off),
                   reinterpret_cast<const uint4*>(d_stage_ + L.hdr_off), d_stage_ + L.pack_off,
                   L.stride};
      void* kargs[] = {&ga};
      const bool tc = o0.flop > 0;
      if (tc) tc_begin(l, s);
      if (info->coop) {
        TTG_CUDA(cudaLaunchCooperativeKernel(info->group, dim3(L.ctas), o0.block, kargs, L.smem,
                                             s));
      } else {
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(L.ctas);
        cfg.blockDim = o0.block;
        cfg.dynamicSmemBytes = L.smem;
        cfg.stream = s;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
        attr[0].val.programmaticStreamSerializationAllowed = 1;
        cfg.attrs = attr;
        cfg.numAttrs = owner_->pdl ? 1 : 0;
        const cudaError_t le = cudaLaunchKernelExC(&cfg, info->group, kargs);
        if (le != cudaSuccess) {
          const char* name = "?";
          cudaFuncGetName(&name, info->plain);
          fail(TTG_ERR_CUDA, "grouped launch of %s (%zu launches, %u CTAs of %u threads, "
               "%u B dynamic shared memory): %s", name ? name : "?", L.n, L.ctas,
               o0.block.x * o0.block.y * o0.block.z, L.smem, cudaGetErrorString(le));
        }
      }
      if (tc) tc_end(l, s);
      lane_launches[l] += 1;
    }
  };
  // Lanes are issued by several host threads at once, each lane in order.
  cudaError_t e = cudaSuccess;
  const std::string issue_err = pool_->run(nl, [&](size_t l) {
    for (size_t si = 0; si < steps[l].size(); ++si) issue_step(l, si);
  });
  for (size_t l = 0; l < nl; ++l) {
    st.launches += lane_launches[l];
    st.grouped_records += lane_grouped[l];
    st.tc_launches += lane_tc[l];
  }
  const auto t_issued = std::chrono::steady_clock::now();
  st.ms_issue += std::chrono::duration<double, std::milli>(t_issued - t1).count();
  for (size_t l = 0; l < nl; ++l) {
    const cudaError_t el = cudaStreamSynchronize(lanes_[l]);
    if (e == cudaSuccess) e = el;
  }
  st.lanes_max = std::max<int64_t>(st.lanes_max, int64_t(nl));
  if (time_tc_ && e == cudaSuccess && issue_err.empty()) {
    for (size_t l = 0; l < nl; ++l)
      for (int64_t k = 0; k < lane_tc[l]; ++k) {
        float ms = 0.0f;
        TTG_CUDA(cudaEventElapsedTime(&ms, tc_ev_[l][2 * k], tc_ev_[l][2 * k + 1]));
        st.tc_ms += ms;
      }
  }
  const auto t2 = std::chrono::steady_clock::now();
  st.ms_issue_wait += std::chrono::duration<double, std::milli>(t2 - t1).count();
  for (Recorder* r : R) {
    r->ops.clear();
    r->closures.clear();
    r->arena.clear();
  }
  // Blocks the solves freed during this flush's segments may now serve any
  // solve of the same worker: everything recorded so far is complete.
  for (Recorder* r : R) {
    auto& pl = pools_[r->fiber->worker];
    for (auto& kv : r->cache) {
      auto& dst = pl[kv.first];
      dst.insert(dst.end(), kv.second.begin(), kv.second.end());
    }
    r->cache.clear();
  }
  if (!issue_err.empty()) fail(TTG_ERR_CUDA, "grouped launch: %s", issue_err.c_str());
  if (e != cudaSuccess) fail(TTG_ERR_CUDA, "grouped launch: %s", cudaGetErrorString(e));
}

void rec_op(Recorder* r, StreamOp op) {
  RecOp o{};
  o.info = nullptr;
  o.closure = uint32_t(r->closures.size());
  r->closures.push_back(std::move(op));
  r->ops.push_back(o);
}

void rec_group(Recorder* r, const GroupInfo* info, dim3 grid, dim3 block, size_t smem,
               const void* pack) {
  const size_t off = align_up(r->arena.size(), 16);
  r->arena.resize(off + info->pack_size);
  memcpy(r->arena.data() + off, pack, info->pack_size);
  RecOp o{};
  o.info = info;
  o.grid = grid;
  o.block = block;
  o.smem = uint32_t(smem);
  o.pack_off = uint32_t(off);
  r->ops.push_back(o);
}

void rec_note_flop(Recorder* r, double flop) {
  r->ops.back().flop = flop;
  r->tc_flop += flop;
  r->tc_records += 1;
}

void rec_retract_flop(Recorder* r, double flop, int64_t records) {
  r->tc_flop -= flop;
  r->tc_records -= records;
}

void rec_wait(Recorder* r) { r->ex->wait(r); }

void rec_memset(Context* c, void* p, int value, size_t bytes) {
  if (bytes == 0) return;
  const int64_t blocks = std::max<int64_t>(
      1, std::min<int64_t>((int64_t(bytes) / 16 + 255) / 256, int64_t(c->num_sms) * 4));
  launch(c, k_fill_bytes, unsigned(blocks), 256, 0, static_cast<unsigned char*>(p), value,
         int64_t(bytes));
}

void rec_read(Context* c, size_t off, const void* src, size_t bytes) {
  TTG_REQUIRE(off + bytes <= 4096 * sizeof(double), "rec_read: %zu bytes at %zu", bytes, off);
  launch(c, k_read_host, 1, 256, 0, static_cast<const unsigned char*>(src),
         reinterpret_cast<unsigned char*>(c->h_scal_dev) + off, int64_t(bytes));
}

void* rec_alloc(Recorder* r, Allocator* shared, size_t bytes) {
  const size_t cls = Allocator::size_class(bytes);
  auto it = r->cache.find(cls);
  if (it != r->cache.end() && !it->second.empty()) {
    void* p = it->second.back();
    it->second.pop_back();
    return p;
  }
  auto& pl = r->ex->pool(r->fiber->worker);
  auto jt = pl.find(cls);
  if (jt != pl.end() && !jt->second.empty()) {
    void* p = jt->second.back();
    jt->second.pop_back();
    return p;
  }
  return shared->get(bytes);
}

void rec_free(Recorder* r, void* p, size_t bytes) {
  r->cache[Allocator::size_class(bytes)].push_back(p);
}

void run_grouped(Context* owner, int width, int64_t count,
                 const std::function<void(int64_t, Context*)>& body, ttg_group_stats* gs) {
  const auto t0 = std::chrono::steady_clock::now();
  sync(owner);
  Executor ex(owner, width);
  ex.run(count, body);
  if (gs) {
    *gs = ex.st;
    gs->ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
  }
}

}  // namespace ttg
