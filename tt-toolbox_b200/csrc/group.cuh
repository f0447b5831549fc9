// Grouped launches: one launch of a kernel over the problems of many
// independent solves.
//
// A kernel written with TTG_KERNEL has its body in a __device__ function
// whose first two parameters are named blockIdx and gridDim: they shadow the
// built-in variables, so the body reads its block coordinates from them and
// stays the code of a plain kernel.  Two __global__ entries are instantiated
// from the body:
//   * the plain kernel (k_plain) passes the real blockIdx/gridDim;
//   * the grouped kernel (k_group) runs the CTAs of many launches of the
//     same body (each with its own grid and arguments) as one grid: CTA b
//     finds its launch in a CTA-to-launch map, rebuilds that launch's block
//     coordinates and grid from the launch header and calls the body with
//     the launch's argument pack.
// Helpers that read blockIdx/gridDim take them as parameters in the same way.
// Cooperative bodies (bounded grid barriers on a per-launch counter) are
// grouped into cooperative launches whose CTAs are all resident, so every
// launch's barrier completes as in its own grid.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <tuple>
#include <type_traits>
#include <utility>

#include "internal.h"

namespace ttg {

// Argument pack with one layout on host and device.
template <class... A>
struct Pack;
template <>
struct Pack<> {};
template <class H, class... T>
struct Pack<H, T...> {
  H h;
  Pack<T...> t;
};

template <size_t I, class P>
__host__ __device__ __forceinline__ auto& pk(P& p) {
  if constexpr (I == 0)
    return p.h;
  else
    return pk<I - 1>(p.t);
}

// Device arguments of a grouped launch.
struct GroupArgs {
  const uint32_t* map;  // launch index of each CTA
  const uint4* hdr;     // per launch: first CTA, grid x, grid y, grid z
  const char* packs;    // per launch argument pack, `stride` bytes apart
  uint32_t stride;
};

#ifdef __CUDACC__
// Launch index of this CTA in a grouped launch, with its block coordinates
// and grid in that launch (after the wait on the preceding grid: the map and
// headers come from the copy issued before the launches).
__device__ __forceinline__ uint32_t group_locate(const GroupArgs& g, uint3& b, dim3& gd) {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  const uint32_t r = g.map[blockIdx.x];
  const uint4 h = g.hdr[r];
  const uint32_t l = blockIdx.x - h.x;
  b.x = l % h.y;
  b.y = (l / h.y) % h.z;
  b.z = l / (h.y * h.z);
  gd = dim3(h.y, h.z, h.w);
  return r;
}

template <auto Body, class... A, size_t... I>
__device__ __forceinline__ void group_call(const GroupArgs& g, std::index_sequence<I...>) {
  uint3 b;
  dim3 gd;
  const uint32_t r = group_locate(g, b, gd);
  const Pack<A...>& p = *reinterpret_cast<const Pack<A...>*>(g.packs + size_t(r) * g.stride);
  Body(b, gd, pk<I>(const_cast<Pack<A...>&>(p))...);
}

template <auto Body, int LB, class... A>
__global__ void __launch_bounds__(LB) k_plain_lb(A... a) {
  Body(blockIdx, gridDim, a...);
}
template <auto Body, class... A>
__global__ void k_plain_nolb(A... a) {
  Body(blockIdx, gridDim, a...);
}
template <auto Body, int LB, class... A>
__global__ void __launch_bounds__(LB) k_group_lb(GroupArgs g) {
  group_call<Body, A...>(g, std::index_sequence_for<A...>{});
}
template <auto Body, class... A>
__global__ void k_group_nolb(GroupArgs g) {
  group_call<Body, A...>(g, std::index_sequence_for<A...>{});
}
#endif

// What the executor of grouped launches needs to know about a kernel.
struct GroupInfo {
  const void* plain;   // the plain __global__ entry
  const void* group;   // the grouped __global__ entry
  bool coop;           // body waits on grid barriers: all CTAs must be resident
  uint32_t pack_size;
  uint32_t pack_align;
  // One launch of the plain entry with a recorded argument pack.
  void (*issue)(const void* pack, dim3 grid, dim3 block, size_t smem, cudaStream_t s, bool pdl);
};

template <class... A, size_t... I>
void pack_pointers(Pack<A...>& p, void** out, std::index_sequence<I...>);

template <bool COOP, class... A>
void issue_plain(const void* fn, const void* pack, dim3 grid, dim3 block, size_t smem,
                 cudaStream_t s, bool pdl) {
  Pack<A...> p;
  memcpy(static_cast<void*>(&p), pack, sizeof(p));
  void* kargs[sizeof...(A) + 1];
  pack_pointers(p, kargs, std::index_sequence_for<A...>{});
  if constexpr (COOP) {
    TTG_CUDA(cudaLaunchCooperativeKernel(fn, grid, block, kargs, smem, s));
  } else {
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
    TTG_CUDA(cudaLaunchKernelExC(&cfg, fn, kargs));
  }
}

struct Recorder;
// Record one launch of a grouped kernel (argument pack copied).
void rec_group(Recorder* r, const GroupInfo* info, dim3 grid, dim3 block, size_t smem,
               const void* pack);
// Marks the launch recorded last as a tensor-core GEMM of `flop` algorithmic
// FLOPs (counted, and timed on request, by the executor).
void rec_note_flop(Recorder* r, double flop);

template <auto Body, int LB, bool COOP, class... A>
struct Kern {
  using plain_t = void (*)(A...);
  using pack_t = Pack<A...>;
#ifdef __CUDACC__
  static plain_t plain() {
    if constexpr (LB > 0)
      return &k_plain_lb<Body, LB, A...>;
    else
      return &k_plain_nolb<Body, A...>;
  }
  static const void* group() {
    if constexpr (LB > 0)
      return reinterpret_cast<const void*>(&k_group_lb<Body, LB, A...>);
    else
      return reinterpret_cast<const void*>(&k_group_nolb<Body, A...>);
  }
  static void issue(const void* pack, dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                    bool pdl) {
    issue_plain<COOP, A...>(reinterpret_cast<const void*>(plain()), pack, grid, block, smem, s,
                            pdl);
  }
  static const GroupInfo* info() {
    static const GroupInfo gi{reinterpret_cast<const void*>(plain()), group(), COOP,
                              uint32_t(sizeof(pack_t)), uint32_t(alignof(pack_t)), &issue};
    return &gi;
  }
  const void* fn() const { return reinterpret_cast<const void*>(plain()); }
  operator plain_t() const { return plain(); }
#endif
};

template <auto Body, int LB, bool COOP, class F>
struct KernOfT;
template <auto Body, int LB, bool COOP, class... A>
struct KernOfT<Body, LB, COOP, void (*)(uint3, dim3, A...)> {
  using type = Kern<Body, LB, COOP, A...>;
};

// Declares the body of kernel `name` (parameters follow the macro):
//   TTG_BODY(k_copy)(TTG_BLOCK, int64_t n, const double* x, double* y) { ... }
//   TTG_KERNEL(k_copy, 0);   // 0: no __launch_bounds__
#define TTG_BLOCK const uint3 blockIdx, const dim3 gridDim
#define TTG_BODY(name) __device__ __forceinline__ void name##_body
#define TTG_KERNEL(name, LB)                                                          \
  constexpr typename ::ttg::KernOfT<name##_body, LB, false, decltype(&name##_body)>::type \
      name {}
#define TTG_COOP_KERNEL(name, LB)                                                    \
  constexpr typename ::ttg::KernOfT<name##_body, LB, true, decltype(&name##_body)>::type \
      name {}
#define TTG_KERNEL_T(name, LB, ...)                                                   \
  constexpr typename ::ttg::KernOfT<name##_body<__VA_ARGS__>, LB, false,             \
                                    decltype(&name##_body<__VA_ARGS__>)>::type name {}

template <class... A, class... Args, size_t... I>
void fill_pack(Pack<A...>& p, std::index_sequence<I...>, Args&&... args) {
  ((pk<I>(p) = static_cast<std::tuple_element_t<I, std::tuple<A...>>>(std::forward<Args>(args))),
   ...);
}

template <class... A, size_t... I>
void pack_pointers(Pack<A...>& p, void** out, std::index_sequence<I...>) {
  ((out[I] = static_cast<void*>(&pk<I>(p))), ...);
}

// Runs body(i, context) for i in [0, count) as a grouped batch of `width`
// solves in flight (group.cu); the contexts record for the executor.
void run_grouped(Context* owner, int width, int64_t count,
                 const std::function<void(int64_t, Context*)>& body, ttg_group_stats* gs);

#ifdef __CUDACC__
// Launch of a TTG_KERNEL on the context's stream, or its record when the
// context belongs to a grouped batch.
template <auto Body, int LB, bool COOP, class... A, class... Args>
void launch(Context* c, Kern<Body, LB, COOP, A...> k, dim3 grid, dim3 block, size_t smem,
            Args&&... args) {
  static_assert(sizeof...(A) == sizeof...(Args), "argument count");
  c->launches += 1;
  if (c->rec) {
    Pack<A...> p{};
    fill_pack(p, std::index_sequence_for<A...>{}, std::forward<Args>(args)...);
    rec_group(c->rec, k.info(), grid, block, smem, &p);
    return;
  }
  if constexpr (COOP) {
    Pack<A...> p{};
    fill_pack(p, std::index_sequence_for<A...>{}, std::forward<Args>(args)...);
    void* kargs[sizeof...(A) + 1];
    pack_pointers(p, kargs, std::index_sequence_for<A...>{});
    TTG_CUDA(cudaLaunchCooperativeKernel(k.fn(), grid, block, kargs, smem, c->stream));
  } else {
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
    TTG_CUDA(cudaLaunchKernelEx(&cfg, k.plain(), std::forward<Args>(args)...));
  }
}
#endif

}  // namespace ttg
