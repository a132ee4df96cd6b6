// Block-row sharded BFS: the level loop and its data plane.
//
// Each rank holds the block rows [bounds[rank], bounds[rank+1]) of the graph,
// every column, as its own B2SR graph.  A level is one pull step per shard
// against the whole frontier (gbo_bfs_shard_level), a sum of the ranks'
// new-vertex counts (the loop ends at zero) and an all-gather of the
// shards' next-frontier words (n/8 bytes in all) into every rank's frontier.
// The reference has no multi-GPU path; its single-GPU loop is
// algorithm/bfs.cu:508-564.
//
// The loop itself (gbo_bfs_shard_loop) is host logic over caller-supplied
// operations, so the same code drives the GPU shards over NCCL or a CPU
// restatement of the level step over any other transport.  A rank whose
// level step fails still takes part in the sum (with an error mark added),
// so every rank leaves the loop at the same level with the same status.
#include <dlfcn.h>

#include <mutex>
#include <vector>

#include <nccl.h>

#include "graph.cuh"

namespace gbo {
namespace {

// Error mark added to a rank's count when its level step failed: at most
// 255 failing ranks and 2^56 - 1 new vertices per level fit the sum.
constexpr uint64_t kFailMark = 1ull << 56;

// ------------------------------------------------------------- NCCL (dlopen)
// NCCL is loaded at run time so that the library has no link-time
// dependency on it; only the NCCL data plane needs it.
struct NcclApi {
  void* h = nullptr;
  ncclResult_t (*getUniqueId)(ncclUniqueId*) = nullptr;
  ncclResult_t (*commInitRank)(ncclComm_t*, int, ncclUniqueId, int) = nullptr;
  ncclResult_t (*commDestroy)(ncclComm_t) = nullptr;
  ncclResult_t (*allGather)(const void*, void*, size_t, ncclDataType_t, ncclComm_t, cudaStream_t) = nullptr;
  ncclResult_t (*allReduce)(const void*, void*, size_t, ncclDataType_t, ncclRedOp_t, ncclComm_t,
                            cudaStream_t) = nullptr;
  const char* (*errorString)(ncclResult_t) = nullptr;
};

int nccl_api(NcclApi** out) {
  static NcclApi api;
  static std::once_flag once;
  static int status = GBO_OK;
  static std::string why;
  std::call_once(once, [] {
    for (const char* name : {"libnccl.so.2", "libnccl.so"}) {
      api.h = dlopen(name, RTLD_NOW | RTLD_LOCAL);
      if (api.h) break;
    }
    if (!api.h) {
      status = GBO_ERR_UNSUPPORTED;
      why = "NCCL (libnccl.so.2) not found";
      return;
    }
    api.getUniqueId = reinterpret_cast<decltype(api.getUniqueId)>(dlsym(api.h, "ncclGetUniqueId"));
    api.commInitRank = reinterpret_cast<decltype(api.commInitRank)>(dlsym(api.h, "ncclCommInitRank"));
    api.commDestroy = reinterpret_cast<decltype(api.commDestroy)>(dlsym(api.h, "ncclCommDestroy"));
    api.allGather = reinterpret_cast<decltype(api.allGather)>(dlsym(api.h, "ncclAllGather"));
    api.allReduce = reinterpret_cast<decltype(api.allReduce)>(dlsym(api.h, "ncclAllReduce"));
    api.errorString = reinterpret_cast<decltype(api.errorString)>(dlsym(api.h, "ncclGetErrorString"));
    if (!api.getUniqueId || !api.commInitRank || !api.commDestroy || !api.allGather || !api.allReduce ||
        !api.errorString) {
      status = GBO_ERR_UNSUPPORTED;
      why = "NCCL library lacks an entry point";
    }
  });
  if (status != GBO_OK) return fail(status, why);
  *out = &api;
  return GBO_OK;
}

int nccl_fail(const NcclApi* api, ncclResult_t r, const char* what) {
  return fail(GBO_ERR_CUDA, std::string(what) + ": " + api->errorString(r));
}

// Caller-visible communicator: the gbo_shard_comm callbacks over an NCCL
// communicator, plus a device word for the count sum.
struct NcclComm {
  gbo_shard_comm pub;  // first member: a gbo_shard_comm* is a NcclComm*
  NcclApi* api = nullptr;
  ncclComm_t comm = nullptr;
  unsigned long long* d_count = nullptr;
  cudaStream_t st = nullptr;
};

int nccl_allreduce_u64(void* user, uint64_t* value) {
  NcclComm* c = static_cast<NcclComm*>(user);
  GBO_CUDA_TRY(cudaMemcpyAsync(c->d_count, value, sizeof(uint64_t), cudaMemcpyHostToDevice, c->st));
  const ncclResult_t r = c->api->allReduce(c->d_count, c->d_count, 1, ncclUint64, ncclSum, c->comm, c->st);
  if (r != ncclSuccess) return nccl_fail(c->api, r, "ncclAllReduce");
  GBO_CUDA_TRY(cudaMemcpyAsync(value, c->d_count, sizeof(uint64_t), cudaMemcpyDeviceToHost, c->st));
  GBO_CUDA_TRY(cudaStreamSynchronize(c->st));
  return GBO_OK;
}

int nccl_allgather(void* user, const void* d_send, void* d_recv, size_t bytes, gbo_stream_t stream) {
  NcclComm* c = static_cast<NcclComm*>(user);
  const ncclResult_t r = c->api->allGather(d_send, d_recv, bytes, ncclUint8, c->comm, as_stream(stream));
  if (r != ncclSuccess) return nccl_fail(c->api, r, "ncclAllGather");
  return GBO_OK;
}

// ------------------------------------------------------- GPU shard state
// Frontier placement: gathered part s (width words, the first
// wend[s] - wbeg[s] of them valid) goes to words [wbeg[s], wend[s]).
__global__ void k_place(const unsigned char* __restrict__ recv, unsigned char* __restrict__ front,
                        const int* __restrict__ wbound, int world, long long width_bytes, int word_bytes,
                        long long nbytes) {
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nbytes) return;
  const long long w = q / word_bytes;
  int lo = 0, hi = world;  // shard s with wbound[s] <= w < wbound[s + 1]
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (wbound[mid] <= w) lo = mid;
    else hi = mid;
  }
  front[q] = recv[(long long)lo * width_bytes + (w - wbound[lo]) * word_bytes + q % word_bytes];
}

// Level 0: the source bit in the frontier; in the owner's visited word and
// level.  One thread.
__global__ void k_shard_seed(unsigned char* front, unsigned char* visited, int* level, int src, int b,
                             int word_bytes, int r0, int r1) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  const long long w = src / b;
  const int bit = b - 1 - src % b;  // bit of the word, little-endian bytes
  front[w * word_bytes + bit / 8] |= (unsigned char)(1u << (bit % 8));
  if (src >= r0 && src < r1) {
    const long long lw = w - r0 / b;
    visited[lw * word_bytes + bit / 8] |= (unsigned char)(1u << (bit % 8));
    level[src - r0] = 0;
  }
}

struct GpuShard {
  gbo_graph* g;
  const gbo_shard_comm* comm;
  cudaStream_t s;
  int rank, world, b, wbytes;
  long long nbr_all, width;  // words of the whole frontier; widest shard's words
  void *front, *visited, *next, *send, *recv;
  int* wbound;
  int32_t* level;
  std::vector<int> h_wbound;
};

int gpu_level(void* user, int lvl, uint64_t* count) {
  GpuShard* S = static_cast<GpuShard*>(user);
  return gbo_bfs_shard_level(S->g, S->front, S->visited, S->level, lvl, S->next, count, S->s);
}

int gpu_allreduce(void* user, uint64_t* value) {
  GpuShard* S = static_cast<GpuShard*>(user);
  return S->comm->allreduce_sum_u64(S->comm->user, value);
}

int failed_level(void*, int, uint64_t*) { return GBO_ERR_CUDA; }

int gpu_exchange(void* user) {
  GpuShard* S = static_cast<GpuShard*>(user);
  const size_t wb = (size_t)S->width * S->wbytes;
  const long long mine = (long long)S->h_wbound[S->rank + 1] - S->h_wbound[S->rank];
  GBO_CUDA_TRY(cudaMemsetAsync(S->send, 0, wb, S->s));
  if (mine > 0) GBO_CUDA_TRY(cudaMemcpyAsync(S->send, S->next, (size_t)mine * S->wbytes, cudaMemcpyDeviceToDevice, S->s));
  GBO_TRY(S->comm->allgather(S->comm->user, S->send, S->recv, wb, S->s));
  const long long nbytes = S->nbr_all * S->wbytes;
  if (nbytes > 0)
    k_place<<<blocks_for(nbytes, 256), 256, 0, S->s>>>(static_cast<const unsigned char*>(S->recv),
                                                        static_cast<unsigned char*>(S->front), S->wbound, S->world,
                                                        (long long)wb, S->wbytes, nbytes);
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

}  // namespace
}  // namespace gbo

using namespace gbo;

extern "C" int gbo_bfs_shard_loop(const gbo_shard_ops* ops, int max_levels, int* h_depth) {
  clear_error();
  if (!ops || !ops->level || !ops->allreduce_sum_u64 || !ops->exchange || max_levels < 1)
    return fail(GBO_ERR_INVALID, "gbo_bfs_shard_loop: bad argument");
  for (int lvl = 0; lvl < max_levels; ++lvl) {
    uint64_t c = 0;
    const int st = ops->level(ops->user, lvl, &c);
    uint64_t v = st == GBO_OK ? c : kFailMark;
    const int sr = ops->allreduce_sum_u64(ops->user, &v);
    if (sr != GBO_OK) return sr;  // the transport itself failed: no agreement possible
    if (v >= kFailMark) return fail(st != GBO_OK ? st : GBO_ERR_CUDA, "a rank's level step failed at level " + std::to_string(lvl));
    if (v == 0) {
      if (h_depth) *h_depth = lvl + 1;
      return GBO_OK;
    }
    const int se = ops->exchange(ops->user);
    if (se != GBO_OK) return se;
  }
  return fail(GBO_ERR_TIMEOUT, "sharded BFS did not finish within max_levels");
}

extern "C" int gbo_bfs_sharded(const gbo_graph* shard, int rank, int world, const int* h_bounds, int src,
                               int32_t* d_level, int* h_depth, const gbo_shard_comm* comm,
                               gbo_stream_t stream) {
  clear_error();
  if (!shard || !h_bounds || !comm || !comm->allreduce_sum_u64 || !comm->allgather || world < 1 || rank < 0 ||
      rank >= world)
    return fail(GBO_ERR_INVALID, "gbo_bfs_sharded: bad argument");
  if (shard->layout != GBO_LAYOUT_ROW) return fail(GBO_ERR_UNSUPPORTED, "a BFS shard needs the ROW tile layout");
  const int b = shard->b;
  const int n = h_bounds[world];
  for (int s = 0; s < world; ++s)
    if (h_bounds[s] > h_bounds[s + 1] || (h_bounds[s + 1] < n && h_bounds[s + 1] % b) || h_bounds[0] != 0)
      return fail(GBO_ERR_INVALID, "row bounds must ascend from 0 on tile boundaries");
  if (shard->nrows != h_bounds[rank + 1] - h_bounds[rank] || shard->ncols != n)
    return fail(GBO_ERR_INVALID, "the shard holds rows [bounds[rank], bounds[rank+1]) and all n columns");
  if (src < 0 || src >= n) return fail(GBO_ERR_INVALID, "source out of range");
  if (shard->nrows > 0 && !d_level) return fail(GBO_ERR_INVALID, "d_level is NULL");
  GpuShard S{};
  S.g = const_cast<gbo_graph*>(shard);
  S.comm = comm;
  S.s = as_stream(stream);
  S.rank = rank;
  S.world = world;
  S.b = b;
  S.wbytes = word_bytes(b);
  S.nbr_all = (n + b - 1) / b;
  S.h_wbound.resize((size_t)world + 1);
  for (int s = 0; s <= world; ++s) S.h_wbound[(size_t)s] = h_bounds[s] < n ? h_bounds[s] / b : (int)S.nbr_all;
  S.width = 1;
  for (int s = 0; s < world; ++s) S.width = std::max<long long>(S.width, S.h_wbound[(size_t)s + 1] - S.h_wbound[(size_t)s]);
  const long long nbr = S.h_wbound[(size_t)rank + 1] - S.h_wbound[(size_t)rank];
  const size_t wb = (size_t)S.wbytes;
  // stream-ordered scratch for this call: frontier, shard state, exchange buffers
  void* mem[6] = {};
  const size_t sizes[6] = {wb * (size_t)std::max<long long>(S.nbr_all, 1) + 8, wb * (size_t)std::max<long long>(nbr, 1) + 8,
                           wb * (size_t)std::max<long long>(nbr, 1) + 8, wb * (size_t)S.width + 8,
                           wb * (size_t)S.width * (size_t)world + 8, sizeof(int) * ((size_t)world + 1)};
  int st = GBO_OK;
  for (int i = 0; i < 6 && st == GBO_OK; ++i) {
    const cudaError_t e = pool_malloc_async(&mem[i], sizes[i], S.s);
    if (e != cudaSuccess) st = fail_cuda(e, "gbo_bfs_sharded buffers");
  }
  if (st == GBO_OK) {
    S.front = mem[0];
    S.visited = mem[1];
    S.next = mem[2];
    S.send = mem[3];
    S.recv = mem[4];
    S.wbound = static_cast<int*>(mem[5]);
    S.level = d_level;
    cudaError_t e = cudaMemcpyAsync(S.wbound, S.h_wbound.data(), sizeof(int) * ((size_t)world + 1),
                                    cudaMemcpyHostToDevice, S.s);
    for (int i = 0; i < 3 && e == cudaSuccess; ++i) e = cudaMemsetAsync(mem[i], 0, sizes[i], S.s);
    if (e == cudaSuccess && shard->nrows > 0)
      e = cudaMemsetAsync(d_level, 0xff, sizeof(int32_t) * (size_t)shard->nrows, S.s);  // -1
    if (e == cudaSuccess) {
      k_shard_seed<<<1, 32, 0, S.s>>>(static_cast<unsigned char*>(S.front), static_cast<unsigned char*>(S.visited),
                                      d_level, src, b, S.wbytes, h_bounds[rank], h_bounds[rank + 1]);
      e = cudaGetLastError();
    }
    if (e != cudaSuccess) st = fail_cuda(e, "gbo_bfs_sharded set-up");
  }
  // every rank enters the loop, also after a failed set-up (its first level
  // step reports the failure through the count sum), so that no peer waits
  gbo_shard_ops ops;
  ops.user = &S;
  ops.level = st == GBO_OK ? gpu_level : failed_level;
  ops.allreduce_sum_u64 = gpu_allreduce;
  ops.exchange = gpu_exchange;
  const int ls = gbo_bfs_shard_loop(&ops, n + 1, h_depth);
  for (void* p : mem)
    if (p) cudaFreeAsync(p, S.s);
  if (st != GBO_OK) return st;
  if (ls != GBO_OK) return ls;
  GBO_CUDA_TRY(cudaStreamSynchronize(S.s));
  return GBO_OK;
}

extern "C" int gbo_nccl_unique_id(void* h_id) {
  clear_error();
  if (!h_id) return fail(GBO_ERR_INVALID, "NULL id buffer");
  NcclApi* api = nullptr;
  GBO_TRY(nccl_api(&api));
  ncclUniqueId id;
  const ncclResult_t r = api->getUniqueId(&id);
  if (r != ncclSuccess) return nccl_fail(api, r, "ncclGetUniqueId");
  memcpy(h_id, &id, sizeof(id));
  return GBO_OK;
}

extern "C" int gbo_nccl_comm_create(int world, int rank, const void* h_id, gbo_shard_comm** out) {
  clear_error();
  if (!h_id || !out || world < 1 || rank < 0 || rank >= world) return fail(GBO_ERR_INVALID, "bad argument");
  NcclApi* api = nullptr;
  GBO_TRY(nccl_api(&api));
  NcclComm* c = new NcclComm();
  c->api = api;
  ncclUniqueId id;
  memcpy(&id, h_id, sizeof(id));
  ncclResult_t r = api->commInitRank(&c->comm, world, id, rank);
  if (r != ncclSuccess) {
    delete c;
    return nccl_fail(api, r, "ncclCommInitRank");
  }
  cudaError_t e = cudaMalloc(&c->d_count, sizeof(unsigned long long));
  if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking);
  if (e != cudaSuccess) {
    api->commDestroy(c->comm);
    cudaFree(c->d_count);
    delete c;
    return fail_cuda(e, "NCCL communicator buffers");
  }
  c->pub.user = c;
  c->pub.allreduce_sum_u64 = nccl_allreduce_u64;
  c->pub.allgather = nccl_allgather;
  *out = &c->pub;
  return GBO_OK;
}

extern "C" int gbo_nccl_comm_destroy(gbo_shard_comm* comm) {
  clear_error();
  if (!comm) return GBO_OK;
  NcclComm* c = reinterpret_cast<NcclComm*>(comm);
  if (c->comm) c->api->commDestroy(c->comm);
  cudaFree(c->d_count);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
  return GBO_OK;
}
