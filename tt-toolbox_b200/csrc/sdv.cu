// SDV TT file format (TT-Toolbox fmex/tt_read.c:13-100, fmex/tt_write.c:21-80):
//
//   header   128 bytes: char txt[8] ("TT" + blanks), int32 ver[2] (1, 0),
//            int32 inf[4] (inf[0] = 128 header bytes, inf[1] = data type:
//            0 double, 1 complex double, 2 float, 3 complex float),
//            char comment[64], int32 i[8] (i[0] = 1, i[2] = d as written)
//   int32 l, m           core index range, d = m - l + 1
//   int32 n[d], r[d+1]   mode sizes and ranks
//   core                 sum_k r_k n_k r_{k+1} values of the data type,
//                        the flat column-major core vector
//
// Little-endian 32-bit ints, as the reference writes them on x86.  TT
// matrices are stored as tensors with mode sizes n_k m_k (the tt field of a
// tt_matrix).  Complex files are rejected (the library's path is real).
#include <cstdio>
#include <cstring>
#include <vector>

#include "internal.h"

using namespace ttg;

namespace {

struct SdvHead {
  char txt[8];
  int32_t ver[2];
  int32_t inf[4];
  char comment[64];
  int32_t i[8];
};
static_assert(sizeof(SdvHead) == 128, "SDV header is 128 bytes");

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

}  // namespace

extern "C" {

int ttg_tt_read_sdv(ttg_context ctx, const char* path, ttg_tt* out) {
  TTG_API_BEGIN
  TTG_REQUIRE(ctx && path && out, "NULL argument");
  *out = nullptr;
  File fh;
  fh.f = fopen(path, "rb");
  TTG_REQUIRE(fh.f, "the file %s can not be opened", path);
  SdvHead hd;
  TTG_REQUIRE(fread(&hd, sizeof(hd), 1, fh.f) == 1, "%s: short header", path);
  TTG_REQUIRE(strncmp(hd.txt, "TT", 2) == 0, "not a SDV TT file: %s", path);   // tt_read.c:37-40
  TTG_REQUIRE(hd.ver[0] == 1, "wrong version of SDV TT file (current is 1), received %d",
              hd.ver[0]);                                                    // :42-45
  const int dtype = hd.inf[1];
  TTG_REQUIRE(dtype >= 0 && dtype <= 3, "wrong datatype %d", dtype);         // :90-93
  if (dtype == 1 || dtype == 3) fail(TTG_ERR_UNSUPPORTED, "%s: complex SDV data", path);
  int32_t lm[2];
  TTG_REQUIRE(fread(lm, sizeof(lm), 1, fh.f) == 1, "%s: short file", path);
  const int64_t d = int64_t(lm[1]) - lm[0] + 1;                              // :50
  TTG_REQUIRE(d >= 1 && d <= (1 << 20), "%s: core range [%d, %d]", path, lm[0], lm[1]);
  std::vector<int32_t> n32(d), r32(d + 1);
  TTG_REQUIRE(fread(n32.data(), sizeof(int32_t), d, fh.f) == size_t(d), "%s: short file", path);
  TTG_REQUIRE(fread(r32.data(), sizeof(int32_t), d + 1, fh.f) == size_t(d + 1),
              "%s: short file", path);
  std::vector<int64_t> n(d), r(d + 1);
  int64_t numel = 0;
  for (int64_t k = 0; k <= d; ++k) {
    TTG_REQUIRE(r32[k] >= 1, "%s: rank %d at %lld", path, r32[k], (long long)k);
    r[k] = r32[k];
  }
  for (int64_t k = 0; k < d; ++k) {
    TTG_REQUIRE(n32[k] >= 1, "%s: mode size %d at %lld", path, n32[k], (long long)k);
    n[k] = n32[k];
    // Each factor is below 2^31, so the product is formed in double first:
    // an int64 product of three such values could overflow.
    const double core_numel = double(r[k]) * double(n[k]) * double(r[k + 1]);
    TTG_REQUIRE(core_numel + double(numel) < double(int64_t(1) << 40), "%s: core too large",
                path);
    numel += r[k] * n[k] * r[k + 1];
  }
  std::vector<double> core(numel);
  if (dtype == 0) {
    TTG_REQUIRE(fread(core.data(), sizeof(double), numel, fh.f) == size_t(numel),
                "%s: short core", path);
  } else {
    std::vector<float> cf(numel);
    TTG_REQUIRE(fread(cf.data(), sizeof(float), numel, fh.f) == size_t(numel),
                "%s: short core", path);
    for (int64_t e = 0; e < numel; ++e) core[e] = cf[e];
  }
  int st = ttg_tt_upload(ctx, d, n.data(), nullptr, r.data(), core.data(), out);
  if (st != TTG_OK) return st;
  TTG_API_END
}

int ttg_tt_write_sdv(ttg_tt tt, const char* path, int32_t precision) {
  TTG_API_BEGIN
  TTG_REQUIRE(tt && path, "NULL argument");
  TTG_REQUIRE(precision == 0 || precision == 1, "precision must be 0 (double) or 1 (float)");
  TTG_REQUIRE(tt->d <= 0x7fffffff, "too many cores");
  SdvHead hd;                                                              // tt_write.c:104-110
  memset(&hd, 0, sizeof(hd));
  memcpy(hd.txt, "TT      ", 8);
  hd.ver[0] = 1;
  hd.inf[0] = 128;
  hd.inf[1] = precision == 0 ? 0 : 2;
  hd.i[0] = 1;
  hd.i[2] = int32_t(tt->d);
  std::vector<int32_t> n32(tt->d), r32(tt->d + 1);
  for (int64_t k = 0; k < tt->d; ++k) {
    const int64_t nk = tt->is_matrix ? tt->n[k] * tt->m[k] : tt->n[k];
    TTG_REQUIRE(nk <= 0x7fffffff, "mode size too large for SDV");
    n32[k] = int32_t(nk);
  }
  for (int64_t k = 0; k <= tt->d; ++k) {
    TTG_REQUIRE(tt->r[k] <= 0x7fffffff, "rank too large for SDV");
    r32[k] = int32_t(tt->r[k]);
  }
  std::vector<double> core(tt->numel);
  TTG_CUDA(cudaSetDevice(tt->ctx->device));
  if (tt->numel)
    TTG_CUDA(cudaMemcpyAsync(core.data(), tt->core, sizeof(double) * tt->numel,
                             cudaMemcpyDeviceToHost, tt->ctx->stream));
  sync(tt->ctx);
  File fh;
  fh.f = fopen(path, "wb");
  TTG_REQUIRE(fh.f, "the file %s can not be opened", path);
  const int32_t lm[2] = {1, int32_t(tt->d)};                                // :38
  bool ok = fwrite(&hd, sizeof(hd), 1, fh.f) == 1 && fwrite(lm, sizeof(lm), 1, fh.f) == 1 &&
            fwrite(n32.data(), sizeof(int32_t), n32.size(), fh.f) == n32.size() &&
            fwrite(r32.data(), sizeof(int32_t), r32.size(), fh.f) == r32.size();
  if (ok && precision == 0) {
    ok = fwrite(core.data(), sizeof(double), core.size(), fh.f) == core.size();
  } else if (ok) {
    std::vector<float> cf(core.begin(), core.end());
    ok = fwrite(cf.data(), sizeof(float), cf.size(), fh.f) == cf.size();
  }
  TTG_REQUIRE(ok, "write to %s failed", path);
  TTG_REQUIRE(fclose(fh.f) == 0, "closing %s failed", path);
  fh.f = nullptr;
  TTG_API_END
}

}  // extern "C"
