// Binary B2SR cache file: save a packed graph and load it back without
// reparsing the Matrix Market file or repacking.  The reference has no
// counterpart (its drivers read the .mtx and repack on every run,
// algorithm/bfs.cu:333-424); the packed arrays are the reference's B2SR
// layout, byte for byte.
//
// File layout (little-endian):
//   FileHeader (64 bytes)
//   bsrRowPtr int32[nbr + 1]
//   bsrColInd int32[nblk]
//   bsrVal    nblk * b words of word_bytes(b) bytes
//   outdeg    int32[ncols]      if kHasOutdeg
//   perm      int32[nrows]      if kHasPerm (degree-ordered graphs)
// The schedule, occupancy words and packed row words are derived data and are
// rebuilt on load.
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "bmv.cuh"

namespace gbo {
namespace {

constexpr char kMagic[8] = {'G', 'B', 'O', 'B', '2', 'S', 'R', '1'};
constexpr unsigned kHasOutdeg = 1u, kHasPerm = 2u, kSymmetric = 4u;

struct FileHeader {
  char magic[8];
  int nrows, ncols, b, layout;
  long long nblk, nnz;
  unsigned contents;
  int nbr;
  long long reserved[2];
};
static_assert(sizeof(FileHeader) == 64, "header layout");

constexpr size_t kChunk = 64u << 20;  // bytes per staged copy

struct File {
  FILE* f = nullptr;
  ~File() {
    if (f) fclose(f);
  }
};

struct Pinned {
  void* p = nullptr;
  ~Pinned() {
    if (p) cudaFreeHost(p);
  }
};

// Device array -> file through a pinned staging buffer.
int write_device(FILE* f, const void* d, size_t bytes, void* stage) {
  for (size_t off = 0; off < bytes; off += kChunk) {
    const size_t n = std::min(kChunk, bytes - off);
    GBO_CUDA_TRY(cudaMemcpy(stage, static_cast<const char*>(d) + off, n, cudaMemcpyDeviceToHost));
    if (fwrite(stage, 1, n, f) != n) return fail(GBO_ERR_IO, "graph file: write failed");
  }
  return GBO_OK;
}

// File -> device array through a pinned staging buffer.
int read_device(FILE* f, void* d, size_t bytes, void* stage) {
  for (size_t off = 0; off < bytes; off += kChunk) {
    const size_t n = std::min(kChunk, bytes - off);
    if (fread(stage, 1, n, f) != n) return fail(GBO_ERR_IO, "graph file: truncated");
    GBO_CUDA_TRY(cudaMemcpy(static_cast<char*>(d) + off, stage, n, cudaMemcpyHostToDevice));
  }
  return GBO_OK;
}

int read_host(FILE* f, void* h, size_t bytes) {
  if (bytes && fread(h, 1, bytes, f) != bytes) return fail(GBO_ERR_IO, "graph file: truncated");
  return GBO_OK;
}

}  // namespace
}  // namespace gbo

using namespace gbo;

extern "C" int gbo_graph_save(const gbo_graph* g, const char* path) {
  clear_error();
  if (!g || !path) return fail(GBO_ERR_INVALID, "NULL argument");
  GBO_CUDA_TRY(cudaDeviceSynchronize());
  File file;
  file.f = fopen(path, "wb");
  if (!file.f) return fail(GBO_ERR_IO, std::string("cannot create ") + path);
  FileHeader h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, kMagic, sizeof(kMagic));
  h.nrows = g->nrows;
  h.ncols = g->ncols;
  h.b = g->b;
  h.layout = g->layout;
  h.nblk = g->nblk;
  h.nnz = g->nnz;
  h.nbr = g->nbr;
  h.contents = (g->outdeg ? kHasOutdeg : 0u) | (g->perm ? kHasPerm : 0u) | (g->symmetric ? kSymmetric : 0u);
  if (fwrite(&h, sizeof(h), 1, file.f) != 1) return fail(GBO_ERR_IO, "graph file: write failed");
  Pinned stage;
  GBO_CUDA_TRY(cudaHostAlloc(&stage.p, kChunk, cudaHostAllocDefault));
  GBO_TRY(write_device(file.f, g->rowptr, sizeof(int) * ((size_t)g->nbr + 1), stage.p));
  GBO_TRY(write_device(file.f, g->colind, sizeof(int) * (size_t)g->nblk, stage.p));
  GBO_TRY(write_device(file.f, g->val, (size_t)g->nblk * g->b * word_bytes(g->b), stage.p));
  if (g->outdeg) GBO_TRY(write_device(file.f, g->outdeg, sizeof(int) * (size_t)g->ncols, stage.p));
  if (g->perm) GBO_TRY(write_device(file.f, g->perm, sizeof(int) * (size_t)g->nrows, stage.p));
  if (fflush(file.f) != 0) return fail(GBO_ERR_IO, "graph file: write failed");
  return GBO_OK;
}

extern "C" int gbo_graph_load(const char* path, int flags, gbo_stream_t stream, gbo_graph** out) {
  clear_error();
  if (!path || !out) return fail(GBO_ERR_INVALID, "NULL argument");
  *out = nullptr;
  File file;
  file.f = fopen(path, "rb");
  if (!file.f) return fail(GBO_ERR_IO, std::string("cannot open ") + path);
  FileHeader h;
  if (fread(&h, sizeof(h), 1, file.f) != 1 || memcmp(h.magic, kMagic, sizeof(kMagic)) != 0)
    return fail(GBO_ERR_IO, "graph file: not a B2SR graph file");
  if (!valid_tile_bits(h.b) || h.nrows < 0 || h.ncols < 0 || h.nblk < 0 ||
      (h.layout != GBO_LAYOUT_ROW && h.layout != GBO_LAYOUT_COL) ||
      h.nbr != (h.nrows + h.b - 1) / h.b || h.nblk > (long long)INT32_MAX)
    return fail(GBO_ERR_IO, "graph file: bad header");
  const int nbc = (h.ncols + h.b - 1) / h.b;
  if ((long long)h.nbr * nbc < h.nblk) return fail(GBO_ERR_IO, "graph file: bad header");
  // the block-row offsets and block-column indices are checked on the host
  std::vector<int> rp((size_t)h.nbr + 1), ci((size_t)h.nblk);
  GBO_TRY(read_host(file.f, rp.data(), sizeof(int) * rp.size()));
  GBO_TRY(read_host(file.f, ci.data(), sizeof(int) * ci.size()));
  if (rp[0] != 0 || rp[h.nbr] != h.nblk) return fail(GBO_ERR_IO, "graph file: bad block-row offsets");
  for (int R = 0; R < h.nbr; ++R) {
    if (rp[R + 1] < rp[R]) return fail(GBO_ERR_IO, "graph file: bad block-row offsets");
    for (int t = rp[R]; t < rp[R + 1]; ++t)
      if (ci[t] < 0 || ci[t] >= nbc || (t > rp[R] && ci[t] <= ci[t - 1]))
        return fail(GBO_ERR_IO, "graph file: block-column indices out of range or unsorted");
  }
  cudaStream_t s = as_stream(stream);
  gbo_graph* g = new gbo_graph();
  g->nrows = h.nrows;
  g->ncols = h.ncols;
  g->b = h.b;
  g->layout = h.layout;
  g->nbr = h.nbr;
  g->nbc = nbc;
  g->nblk = h.nblk;
  g->nnz = h.nnz;
  g->symmetric = (h.contents & kSymmetric) || (flags & GBO_FLAG_SYMMETRIC);
  g->tc_mma = flags & GBO_FLAG_TC_MMA;
  int st = GBO_OK;
  auto cu = [&](cudaError_t e, const char* what) {
    if (st == GBO_OK && e != cudaSuccess) st = fail_cuda(e, what);
  };
  const size_t vb = (size_t)h.nblk * h.b * word_bytes(h.b);
  cu(cudaMalloc(&g->rowptr, sizeof(int) * rp.size()), "rowptr");
  cu(cudaMalloc(&g->colind, sizeof(int) * (ci.empty() ? 1 : ci.size())), "colind");
  cu(cudaMalloc(&g->val, vb ? vb : 1), "tiles");
  g->device_bytes += (long long)(sizeof(int) * (rp.size() + ci.size()) + vb);
  cu(cudaMemcpy(g->rowptr, rp.data(), sizeof(int) * rp.size(), cudaMemcpyHostToDevice), "rowptr");
  if (!ci.empty()) cu(cudaMemcpy(g->colind, ci.data(), sizeof(int) * ci.size(), cudaMemcpyHostToDevice), "colind");
  Pinned stage;
  cu(cudaHostAlloc(&stage.p, kChunk, cudaHostAllocDefault), "staging buffer");
  if (st == GBO_OK) st = read_device(file.f, g->val, vb, stage.p);
  if (st == GBO_OK && (h.contents & kHasOutdeg)) {
    std::vector<int> deg((size_t)h.ncols);
    st = read_host(file.f, deg.data(), sizeof(int) * deg.size());
    if (st == GBO_OK) st = upload_outdeg(g, deg.data(), h.ncols, s);
    if (st == GBO_OK) cu(cudaStreamSynchronize(s), "out-degrees");
  }
  if (st == GBO_OK && (h.contents & kHasPerm)) {
    std::vector<int> perm((size_t)h.nrows);
    st = read_host(file.f, perm.data(), sizeof(int) * perm.size());
    cu(cudaMalloc(&g->perm, sizeof(int) * (perm.empty() ? 1 : perm.size())), "permutation");
    if (!perm.empty()) cu(cudaMemcpy(g->perm, perm.data(), sizeof(int) * perm.size(), cudaMemcpyHostToDevice), "permutation");
    g->device_bytes += 4LL * h.nrows;
  }
  if (st == GBO_OK) st = build_schedule(g, s);
  if (st == GBO_OK) st = build_rowmask(g, s);
  if (st == GBO_OK) st = build_rowwords(g, s);
  if (st == GBO_OK) st = ensure_workspace(g, bmv_scratch_bytes(g), s);
  if (st == GBO_OK) cu(cudaStreamSynchronize(s), "graph load sync");
  if (st != GBO_OK) {
    gbo_graph_free(g);
    return st;
  }
  *out = g;
  return GBO_OK;
}
