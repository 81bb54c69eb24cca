// Export / import of a built H-matrix (no counterpart in the reference, which
// lists JLD2 in REQUIRE but never uses it): one binary file holding the
// parameters, the cluster tree, the block tree and leaf list, the geometry and
// the factor pools, so that an expensive construction (n = 2^20 and more) is
// paid once.  Factorised handles are refused: the H-LU state is rebuilt by
// calling lu! again.
//
// Layout (little-endian, no padding between items):
//   "HMB2SAVE" | u32 version | u32 sizeof(hm_params) | u32 sizeof(Node) |
//   u32 sizeof(Leaf) | u32 sizeof(KernelDesc) | i64 user_bytes | user bytes |
//   hm_params | i64 n | i32 dim | i32 storage | i64 depth | KernelDesc |
//   i64 ncl | 4 x ncl i64 (s, e, left, right) | i64 nnodes | nodes |
//   i64 nleaves | leaves | n*dim f64 geometry | u64 rk_bytes | u64 dense_bytes |
//   rk pool | dense pool | "HMB2END\0"
// The pools are the device bytes as laid out by construction; the loader lays
// the pools out again from the leaf list and refuses the file if the sizes
// differ.
#include "hm_internal.h"

#include <cstdio>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

namespace hm {

namespace {

constexpr char kMagic[8] = {'H', 'M', 'B', '2', 'S', 'A', 'V', 'E'};
constexpr char kEnd[8] = {'H', 'M', 'B', '2', 'E', 'N', 'D', '\0'};
constexpr uint32_t kVersion = 1;
constexpr size_t kChunk = (size_t)64 << 20;     // host staging of the pools

struct File {
  FILE* f = nullptr;
  ~File() { if (f) fclose(f); }
};

int wr(FILE* f, const void* p, size_t bytes) {
  if (bytes && fwrite(p, 1, bytes, f) != bytes) return fail(HM_ERR_IO, "write failed (disk full?)");
  return HM_OK;
}
int rd(FILE* f, void* p, size_t bytes) {
  if (bytes && fread(p, 1, bytes, f) != bytes) return fail(HM_ERR_IO, "file truncated or unreadable");
  return HM_OK;
}
template <typename T> int wr1(FILE* f, const T& v) { return wr(f, &v, sizeof(T)); }
template <typename T> int rd1(FILE* f, T& v) { return rd(f, &v, sizeof(T)); }

template <typename T> int wrv(FILE* f, const std::vector<T>& v) { return wr(f, v.data(), sizeof(T) * v.size()); }
// bytes from the current position to the end of the file
int64_t remaining(FILE* f) {
  const long pos = std::ftell(f);
  if (pos < 0 || std::fseek(f, 0, SEEK_END) != 0) return -1;
  const long end = std::ftell(f);
  if (std::fseek(f, pos, SEEK_SET) != 0) return -1;
  return end - pos;
}

template <typename T> int rdv(FILE* f, std::vector<T>& v, int64_t count, int64_t limit) {
  if (count < 0 || count > limit || (int64_t)sizeof(T) * count > remaining(f))
    return fail(HM_ERR_ARG, "file: implausible array length");
  v.resize((size_t)count);
  return rd(f, v.data(), sizeof(T) * v.size());
}

// device <-> file through a pinned staging buffer
int dev_to_file(FILE* f, const void* d, size_t bytes, cudaStream_t st, char* stage) {
  for (size_t o = 0; o < bytes; o += kChunk) {
    const size_t b = std::min(kChunk, bytes - o);
    HM_CUDA_TRY(cudaMemcpyAsync(stage, (const char*)d + o, b, cudaMemcpyDeviceToHost, st));
    HM_CUDA_TRY(cudaStreamSynchronize(st));
    HM_TRY(wr(f, stage, b));
  }
  return HM_OK;
}
int file_to_dev(FILE* f, void* d, size_t bytes, cudaStream_t st, char* stage) {
  for (size_t o = 0; o < bytes; o += kChunk) {
    const size_t b = std::min(kChunk, bytes - o);
    HM_TRY(rd(f, stage, b));
    HM_CUDA_TRY(cudaMemcpyAsync((char*)d + o, stage, b, cudaMemcpyHostToDevice, st));
    HM_CUDA_TRY(cudaStreamSynchronize(st));
  }
  return HM_OK;
}

struct Pinned {
  char* p = nullptr;
  ~Pinned() { if (p) cudaFreeHost(p); }
};

// header up to and including the user bytes; returns the user byte count
int read_header(FILE* f, int64_t* user_bytes) {
  char magic[8];
  uint32_t ver, sp, sn, sl, sk;
  HM_TRY(rd(f, magic, 8));
  if (std::memcmp(magic, kMagic, 8) != 0) return fail(HM_ERR_ARG, "not an H-matrix file (bad magic)");
  HM_TRY(rd1(f, ver));
  HM_TRY(rd1(f, sp));
  HM_TRY(rd1(f, sn));
  HM_TRY(rd1(f, sl));
  HM_TRY(rd1(f, sk));
  if (ver != kVersion) return fail(HM_ERR_ARG, "H-matrix file version " + std::to_string(ver) + " is not supported");
  if (sp != sizeof(hm_params) || sn != sizeof(Node) || sl != sizeof(Leaf) || sk != sizeof(KernelDesc))
    return fail(HM_ERR_ARG, "H-matrix file written by an incompatible build");
  HM_TRY(rd1(f, *user_bytes));
  if (*user_bytes < 0 || *user_bytes > ((int64_t)1 << 40)) return fail(HM_ERR_ARG, "file: implausible user block");
  return HM_OK;
}

}  // namespace

int save_handle(const hm_handle* h, const char* path, const void* user, int64_t user_bytes) {
  if (h->factorized || h->lu) return fail(HM_ERR_STATE, "save: the handle is factorised (save before lu!)");
  if (user_bytes < 0 || (user_bytes > 0 && !user)) return fail(HM_ERR_ARG, "save: invalid user block");
  File F;
  F.f = std::fopen(path, "wb");
  if (!F.f) return fail(HM_ERR_IO, std::string("save: cannot open ") + path);
  FILE* f = F.f;
  const uint32_t hdr[5] = {kVersion, (uint32_t)sizeof(hm_params), (uint32_t)sizeof(Node), (uint32_t)sizeof(Leaf),
                           (uint32_t)sizeof(KernelDesc)};
  HM_TRY(wr(f, kMagic, 8));
  HM_TRY(wr(f, hdr, sizeof(hdr)));
  HM_TRY(wr1(f, user_bytes));
  HM_TRY(wr(f, user, (size_t)user_bytes));
  HM_TRY(wr1(f, h->prm));
  HM_TRY(wr1(f, h->n));
  HM_TRY(wr1(f, (int32_t)h->dim));
  HM_TRY(wr1(f, (int32_t)h->storage));
  HM_TRY(wr1(f, h->depth));
  HM_TRY(wr1(f, h->kd));
  HM_TRY(wr1(f, (int64_t)h->cl_s.size()));
  HM_TRY(wrv(f, h->cl_s));
  HM_TRY(wrv(f, h->cl_e));
  HM_TRY(wrv(f, h->cl_left));
  HM_TRY(wrv(f, h->cl_right));
  HM_TRY(wr1(f, (int64_t)h->nodes.size()));
  HM_TRY(wrv(f, h->nodes));
  HM_TRY(wr1(f, (int64_t)h->leaves.size()));
  HM_TRY(wrv(f, h->leaves));
  Pinned stage;
  HM_CUDA_TRY(cudaMallocHost((void**)&stage.p, kChunk));
  HM_TRY(dev_to_file(f, h->d_geom, sizeof(double) * h->n * h->dim, h->stream, stage.p));
  HM_TRY(wr1(f, (uint64_t)h->rk_bytes));
  HM_TRY(wr1(f, (uint64_t)h->dense_bytes));
  HM_TRY(dev_to_file(f, h->d_rk, h->rk_bytes, h->stream, stage.p));
  HM_TRY(dev_to_file(f, h->d_dense, h->dense_bytes, h->stream, stage.p));
  HM_TRY(wr(f, kEnd, 8));
  if (std::fflush(f) != 0) return fail(HM_ERR_IO, "save: flush failed");
  return HM_OK;
}

int load_user(const char* path, void* user, int64_t cap, int64_t* user_bytes) {
  File F;
  F.f = std::fopen(path, "rb");
  if (!F.f) return fail(HM_ERR_IO, std::string("load: cannot open ") + path);
  int64_t ub = 0;
  HM_TRY(read_header(F.f, &ub));
  if (ub > remaining(F.f)) return fail(HM_ERR_IO, "file truncated");
  if (user_bytes) *user_bytes = ub;
  if (user && cap > 0) HM_TRY(rd(F.f, user, (size_t)std::min(cap, ub)));
  return HM_OK;
}

int load_handle(const char* path, int device, int (*validate)(const hm_params*), hm_handle** out) {
  File F;
  F.f = std::fopen(path, "rb");
  if (!F.f) return fail(HM_ERR_IO, std::string("load: cannot open ") + path);
  FILE* f = F.f;
  int64_t ub = 0;
  HM_TRY(read_header(f, &ub));
  if (ub > remaining(f) || std::fseek(f, (long)ub, SEEK_CUR) != 0) return fail(HM_ERR_IO, "file truncated");
  std::unique_ptr<hm_handle> h(new hm_handle());
  HM_TRY(rd1(f, h->prm));
  int32_t dim = 0, storage = 0;
  HM_TRY(rd1(f, h->n));
  HM_TRY(rd1(f, dim));
  HM_TRY(rd1(f, storage));
  HM_TRY(rd1(f, h->depth));
  HM_TRY(rd1(f, h->kd));
  h->prm.device = device;
  HM_TRY(validate(&h->prm));
  if (h->n < 1 || h->n > ((int64_t)1 << 40) || dim != h->prm.dim || storage != h->prm.storage ||
      h->kd.dim != dim || h->kd.kind != h->prm.kernel)
    return fail(HM_ERR_ARG, "file: header fields disagree");
  h->dim = dim;
  h->storage = storage;
  h->device = device;
  int64_t ncl = 0, nn = 0, nl = 0;
  const int64_t lim = 4 * h->n + 4;
  HM_TRY(rd1(f, ncl));
  HM_TRY(rdv(f, h->cl_s, ncl, lim));
  HM_TRY(rdv(f, h->cl_e, ncl, lim));
  HM_TRY(rdv(f, h->cl_left, ncl, lim));
  HM_TRY(rdv(f, h->cl_right, ncl, lim));
  HM_TRY(rd1(f, nn));
  HM_TRY(rdv(f, h->nodes, nn, ((int64_t)1 << 31)));
  HM_TRY(rd1(f, nl));
  HM_TRY(rdv(f, h->leaves, nl, nn));
  if (h->cl_s.empty() || h->cl_s[0] != 0 || h->cl_e[0] != h->n) return fail(HM_ERR_ARG, "file: root cluster");
  cudaError_t e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
  if (e != cudaSuccess) return fail(HM_ERR_CUDA, cudaGetErrorString(e));
  hm_handle* hp = h.get();
  auto drop = [&](int s) {      // the message of the failing step stays set
    free_handle_data(hp);
    cudaStreamDestroy(hp->stream);
    return s;
  };
  Pinned stage;
  uint64_t rkb = 0, dnb = 0;
  int s = HM_OK;
  if (cudaMallocHost((void**)&stage.p, kChunk) != cudaSuccess) s = fail(HM_ERR_OOM, "load: staging buffer");
  if (s == HM_OK && cudaMalloc((void**)&hp->d_geom, sizeof(double) * hp->n * hp->dim) != cudaSuccess)
    s = fail(HM_ERR_OOM, "load: geometry");
  if (s == HM_OK) s = file_to_dev(f, hp->d_geom, sizeof(double) * hp->n * hp->dim, hp->stream, stage.p);
  if (s == HM_OK) s = rd1(f, rkb);
  if (s == HM_OK) s = rd1(f, dnb);
  if (s == HM_OK) s = restore_structure(hp);
  if (s == HM_OK && (rkb != hp->rk_bytes || dnb != hp->dense_bytes))
    s = fail(HM_ERR_ARG, "file: pool sizes differ from the leaf list's layout");
  if (s == HM_OK) s = file_to_dev(f, hp->d_rk, hp->rk_bytes, hp->stream, stage.p);
  if (s == HM_OK) s = file_to_dev(f, hp->d_dense, hp->dense_bytes, hp->stream, stage.p);
  char end[8];
  if (s == HM_OK) s = rd(f, end, 8);
  if (s == HM_OK && std::memcmp(end, kEnd, 8) != 0) s = fail(HM_ERR_ARG, "file: missing end marker");
  if (s != HM_OK) return drop(s);
  *out = h.release();
  return HM_OK;
}

}  // namespace hm
