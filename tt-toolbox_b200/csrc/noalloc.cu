// Local matvec for callers that must not allocate device memory.
//
// ttg_local_matvec draws its two contraction intermediates from the context's
// caching allocator, which calls cudaMalloc the first time it sees a size.
// Some callers cannot allow that: code that runs while another component owns
// the whole device memory budget (a host application with its own pool), code
// that must never trigger the implicit device synchronisation and the
// possible out-of-memory failure of cudaMalloc in the middle of a time-critical
// loop, or plugin hosts (such as a MATLAB MEX gateway) whose memory manager
// forbids allocations it does not track.  ttg_local_matvec_noalloc serves
// them: the caller passes inputs and outputs only, and the intermediates live
// in a fixed array inside this library on every GPU that loads it.
#include <mutex>

#include "local_ops.h"

namespace {

// 64 MiB of FP64 scratch per GPU, held from module load until process exit.
// It covers the local matvecs of the benchmark workloads (ranks up to 132 at
// n = 64 and operator rank 3 need 6.7 Mi doubles).
constexpr size_t kNoallocScratchDoubles = size_t(8) << 20;
static __device__ __align__(256) double g_noalloc_scratch[kNoallocScratchDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_scratch_ptr[kMaxDevices] = {};

// The host-side name g_noalloc_scratch is only a stand-in for the device
// array; the kernels need its device address, fetched once per device with
// that device current.
double* scratch_for_current_device(int dev) {
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    TTG_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_scratch_ptr[dev] = static_cast<double*>(p);
  }
  return g_scratch_ptr[dev];
}

}  // namespace

using namespace ttg;

extern "C" int ttg_local_matvec_noalloc(void* stream, int64_t rx1, int64_t n, int64_t rx2,
                                        int64_t ra1, int64_t ra2, const double* Phi1,
                                        const double* A, const double* Phi2, const double* x,
                                        double* y) {
  TTG_API_BEGIN
  TTG_REQUIRE(Phi1 && A && Phi2 && x && y, "NULL argument");
  TTG_REQUIRE(rx1 >= 1 && n >= 1 && rx2 >= 1 && ra1 >= 1 && ra2 >= 1, "sizes must be >= 1");
  MvDims d{rx1, rx1, ra1, n, n, rx2, ra2, rx2};
  // In double from the start: int64 products of large sizes could wrap.
  const double need = double(rx1) * double(n) * double(ra2) * double(rx2) +
                      double(rx1) * double(ra1) * double(n) * double(rx2);
  TTG_REQUIRE(need <= double(kNoallocScratchDoubles),
              "ttg_local_matvec_noalloc: the intermediates need %.0f doubles, more than the "
              "built-in scratch of %zu doubles (64 MiB); use ttg_local_matvec",
              need, kNoallocScratchDoubles);
  int dev = 0;
  TTG_CUDA(cudaGetDevice(&dev));
  TTG_REQUIRE(dev >= 0 && dev < kMaxDevices, "device %d out of range", dev);
  double* scratch = scratch_for_current_device(dev);
  // A context on the stack: stream and SM count only, no allocator.
  Context c;
  c.device = dev;
  c.stream = static_cast<cudaStream_t>(stream);
  TTG_CUDA(cudaDeviceGetAttribute(&c.num_sms, cudaDevAttrMultiProcessorCount, dev));
  local_matvec_f64(&c, d, Phi1, A, Phi2, x, y, scratch, scratch + d.t1_size());
  TTG_CUDA(cudaStreamSynchronize(c.stream));
  TTG_API_END
}
