// Batched traversals.
//
// Multi-source BFS: k sources at once.  The frontier is an n x k bit matrix
// (KW = k/32 words per vertex, vertex-major), so one level is the OR.AND
// product of the B2SR matrix with that bit matrix:
//   F'[i] = OR_{j : P[i][j]} F[j]  &  ~V[i],   V[i] |= F'[i].
// One warp per work item (b = 32).  For every tile whose block column holds a
// frontier row (one "any" byte per block row, written by the previous level),
// each set bit (r, c) of the tile ORs the KW-word row F[C*32+c] into the
// accumulator of tile row r, kept in shared memory.  With KW < 32 the warp
// handles 32/KW set bits at once (lane = slot x word) and OR-reduces the
// slots with shuffles.  The epilogue writes F', V, the levels of the new
// (vertex, source) pairs and the "any" byte of the block row.
//
// Multi-seed BFS (gbo_bfs_multi) reuses the single-frontier BFS loop of
// algo.cu with several level-0 vertices; on a block-diagonal union of graphs
// with one seed per graph it is every graph's own BFS in one traversal.
#include <vector>

#include "scan.cuh"

namespace gbo {

int bfs_seeded(gbo_graph* g, const int* h_seeds, int nseeds, int32_t* d_level, int* h_depth,
               cudaStream_t s);

namespace {

constexpr int kTPB = 256;
constexpr int kWarps = kTPB / 32;

__device__ __forceinline__ unsigned nth_set_bit(unsigned m, int nth) {
  return __fns(m, 0, nth);  // position of the nth (1-based) set bit from bit 0
}

// word mask of the sources [w*32, w*32+32) that exist (k not a multiple of 32)
__device__ __forceinline__ unsigned src_mask(int w, int k) {
  const int lo = w * 32;
  if (k >= lo + 32) return 0xffffffffu;
  if (k <= lo) return 0u;
  return (1u << (k - lo)) - 1u;
}

template <int KW>
__device__ __forceinline__ void ms_epilogue_row(int i, int w, uint32_t a, const GView& v,
                                                uint32_t* __restrict__ Fn,
                                                uint32_t* __restrict__ V,
                                                int* __restrict__ levels, int k, int lvl,
                                                unsigned long long& cnt, bool& any,
                                                uint32_t* __restrict__ slot_any) {
  if (i >= v.nrows) return;
  const size_t o = (size_t)i * KW + w;
  const uint32_t vo = V[o];
  const uint32_t nw = a & ~vo & src_mask(w, k);
  Fn[o] = nw;
  if (nw) {
    V[o] = vo | nw;
    any = true;
    if (slot_any) atomicOr(slot_any + w, nw);
    cnt += __popc(nw);
    uint32_t m = nw;
    while (m) {
      const int p = __ffs(m) - 1;
      m &= m - 1;
      levels[(size_t)i * k + w * 32 + p] = lvl + 1;
    }
  }
}

template <int KW>
__global__ void __launch_bounds__(kTPB) k_ms_step(GView v, uint32_t* __restrict__ Fbase,
                                                  size_t fstride, uint32_t* __restrict__ V,
                                                  uint8_t* __restrict__ anyb, int* __restrict__ levels,
                                                  int k, int* __restrict__ ctl,
                                                  uint32_t* __restrict__ scratch,
                                                  uint32_t* __restrict__ slot_any) {
  constexpr int S = 32 / KW;  // set bits processed at once
  __shared__ uint32_t acc_sh[kWarps][32 * KW];
  volatile int* c = ctl;
  if (c[1]) return;  // done
  const int lvl = c[0];
  const uint32_t* __restrict__ F = Fbase + (size_t)(lvl & 1) * fstride;
  uint32_t* __restrict__ Fn = Fbase + (size_t)((lvl + 1) & 1) * fstride;
  const uint8_t* __restrict__ fany = anyb + (size_t)(lvl & 1) * (v.nbr + 1);
  uint8_t* __restrict__ fany_n = anyb + (size_t)((lvl + 1) & 1) * (v.nbr + 1);
  const unsigned lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t* acc = acc_sh[wib];
  for (int q = lane; q < 32 * KW; q += 32) acc[q] = 0u;
  __syncwarp();
  const int w = lane % KW;
  const int s = lane / KW;
  unsigned long long cnt = 0;
  if (item < v.nitems) {
    const gbo_item it = v.items[item];
    const uint32_t* __restrict__ val = reinterpret_cast<const uint32_t*>(v.val);
    for (int b0 = it.t0; b0 < it.t1; b0 += 32) {
      const int t = b0 + (int)lane;
      int cb = 0;
      bool live = false;
      if (t < it.t1) {
        cb = v.colind[t];
        live = fany[cb] != 0;
      }
      unsigned tiles = __ballot_sync(0xffffffffu, live);
      while (tiles) {
        const int jt = __ffs(tiles) - 1;
        tiles &= tiles - 1;
        const int C = __shfl_sync(0xffffffffu, cb, jt);
        const uint32_t wr = val[(size_t)(b0 + jt) * 32 + lane];  // lane r: tile row r
        unsigned rows = __ballot_sync(0xffffffffu, wr != 0);
        while (rows) {
          const int r = __ffs(rows) - 1;
          rows &= rows - 1;
          unsigned bits = __shfl_sync(0xffffffffu, wr, r);
          uint32_t racc = 0;
          while (bits) {
            const unsigned pos = nth_set_bit(bits, s + 1);
            uint32_t f = 0;
            if (pos != 0xffffffffu) {
              const int col = 31 - (int)pos;  // column c sits at bit 31-c
              f = F[((size_t)C * 32 + col) * KW + w];
            }
#pragma unroll
            for (int o = KW; o < 32; o <<= 1) f |= __shfl_xor_sync(0xffffffffu, f, o);
            racc |= f;
            const unsigned last = nth_set_bit(bits, S);
            bits = last == 0xffffffffu ? 0u : (bits & ~(0xffffffffu >> (31 - last)));
          }
          if (s == 0) acc[r * KW + w] |= racc;
        }
      }
    }
    __syncwarp();
    if (it.slot >= 0) {
      uint32_t* dst = scratch + (size_t)it.slot * 32 * KW;
      for (int q = lane; q < 32 * KW; q += 32) dst[q] = acc[q];
    } else {
      bool any = false;
      for (int rr = 0; rr < 32; rr += S) {
        const int r = rr + s;
        ms_epilogue_row<KW>(it.row * 32 + r, w, acc[r * KW + w], v, Fn, V, levels, k, lvl, cnt, any,
                            slot_any);
      }
      const bool a = __any_sync(0xffffffffu, any);
      if (lane == 0) fany_n[it.row] = a ? 1 : 0;
    }
  }
  // block-level count
  __shared__ unsigned long long sh;
  if (threadIdx.x == 0) sh = 0;
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane == 0 && cnt) atomicAdd(&sh, cnt);
  __syncthreads();
  if (threadIdx.x == 0 && sh) atomicAdd(reinterpret_cast<unsigned long long*>(ctl + 4), sh);
}

// Split block rows: OR the slot accumulators, run the epilogue; the last
// block closes the level (ticket, no waiting).
template <int KW>
__global__ void __launch_bounds__(kTPB) k_ms_finish(GView v, uint32_t* __restrict__ Fbase,
                                                    size_t fstride, uint32_t* __restrict__ V,
                                                    uint8_t* __restrict__ anyb,
                                                    int* __restrict__ levels, int k,
                                                    int* __restrict__ ctl,
                                                    const uint32_t* __restrict__ scratch,
                                                    uint32_t* __restrict__ slot_any) {
  constexpr int S = 32 / KW;
  volatile int* c = ctl;
  if (c[1]) return;
  const int lvl = c[0];
  uint32_t* __restrict__ Fn = Fbase + (size_t)((lvl + 1) & 1) * fstride;
  uint8_t* __restrict__ fany_n = anyb + (size_t)((lvl + 1) & 1) * (v.nbr + 1);
  const unsigned lane = threadIdx.x & 31;
  const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int w = lane % KW;
  const int s = lane / KW;
  unsigned long long cnt = 0;
  if (wid < v.nsplit) {
    const gbo_split sp = v.splits[wid];
    bool any = false;
    for (int rr = 0; rr < 32; rr += S) {
      const int r = rr + s;
      uint32_t a = 0;
      for (int q = 0; q < sp.nslots; ++q) a |= scratch[(size_t)(sp.slot0 + q) * 32 * KW + r * KW + w];
      ms_epilogue_row<KW>(sp.row * 32 + r, w, a, v, Fn, V, levels, k, lvl, cnt, any, slot_any);
    }
    const bool a = __any_sync(0xffffffffu, any);
    if (lane == 0) fany_n[sp.row] = a ? 1 : 0;
  }
  __shared__ unsigned long long sh;
  __shared__ bool last;
  if (threadIdx.x == 0) sh = 0;
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane == 0 && cnt) atomicAdd(&sh, cnt);
  __syncthreads();
  unsigned long long* count = reinterpret_cast<unsigned long long*>(ctl + 4);
  if (threadIdx.x == 0) {
    if (sh) atomicAdd(count, sh);
    __threadfence();
    last = atomicAdd(reinterpret_cast<unsigned*>(ctl + 2), 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    volatile unsigned long long* vc = count;
    const int it = c[0] + 1;
    const bool stop = *vc == 0ull || it >= c[3];
    c[0] = it;
    *vc = 0ull;
    ctl[2] = 0;
    if (stop) c[1] = 1;
    __threadfence();
  }
}

__global__ void k_ms_init(uint32_t* F, size_t fstride, uint32_t* V, uint8_t* anyb, int nbr,
                          int* levels, long long nk, int kw_alloc, int n, int* ctl, int max_iter) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long q = i; q < nk; q += stride) levels[q] = -1;
  for (long long q = i; q < (long long)n * kw_alloc; q += stride) {
    F[q] = 0u;
    F[fstride + q] = 0u;
    V[q] = 0u;
  }
  for (long long q = i; q < 2LL * (nbr + 1); q += stride) anyb[q] = 0;
  if (i == 0) {
    ctl[0] = 0;
    ctl[1] = 0;
    ctl[2] = 0;
    ctl[3] = max_iter;
    reinterpret_cast<unsigned long long*>(ctl + 4)[0] = 0ull;
  }
}

__global__ void k_ms_seed(const int* __restrict__ srcs, int k, int kw, uint32_t* F, uint32_t* V,
                          uint8_t* anyb, int* levels, int n) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int s = 0; s < k; ++s) {
    const int v0 = srcs[s];
    if (v0 < 0 || v0 >= n) continue;
    F[(size_t)v0 * kw + s / 32] |= 1u << (s % 32);
    V[(size_t)v0 * kw + s / 32] |= 1u << (s % 32);
    levels[(size_t)v0 * k + s] = 0;
    anyb[v0 / 32] = 1;
  }
}

struct MsState {
  uint32_t* F = nullptr;  // 2 * n * kw
  uint32_t* V = nullptr;  // n * kw
  uint8_t* anyb = nullptr;
  uint32_t* scratch = nullptr;
  int* srcs = nullptr;
  int* ctl = nullptr;  // iter, done, ticket, max_iter, count(u64)
  int* h_ctl = nullptr;
  int kw = 0;
  int ksrc = 0;
  cudaStream_t cap = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void* key_levels = nullptr;
  int key_k = -1;
  int launches_per_replay = 0;
  std::vector<float> step_ms;
  cudaEvent_t ev[16] = {};
};

}  // namespace
}  // namespace gbo

// Per-graph batched-traversal state (freed with the graph).
struct MsHolder {
  gbo::MsState st;
};

namespace gbo {

void free_ms_state(gbo_graph* g) {
  MsHolder* h = reinterpret_cast<MsHolder*>(g->ms);
  if (!h) return;
  MsState& m = h->st;
  if (m.exec) cudaGraphExecDestroy(m.exec);
  for (auto& e : m.ev)
    if (e) cudaEventDestroy(e);
  cudaFree(m.F);
  cudaFree(m.V);
  cudaFree(m.anyb);
  cudaFree(m.scratch);
  cudaFree(m.srcs);
  cudaFree(m.ctl);
  cudaFreeHost(m.h_ctl);
  if (m.cap) cudaStreamDestroy(m.cap);
  delete h;
  g->ms = nullptr;
}

namespace {

template <int KW>
int ms_capture(gbo_graph* g, MsState& m, int32_t* d_levels, int k) {
  GView v = view_of(g);
  const size_t fstride = (size_t)g->nrows * m.kw;
  const unsigned gi = blocks_for_warps(g->nitems, kWarps);
  const unsigned gs = blocks_for_warps(g->nsplit > 0 ? g->nsplit : 1, kWarps);
  cudaGraph_t graph = nullptr;
  GBO_CUDA_TRY(cudaStreamBeginCapture(m.cap, cudaStreamCaptureModeThreadLocal));
  for (int q = 0; q < 8; ++q) {
    cudaEventRecordWithFlags(m.ev[2 * q], m.cap, cudaEventRecordExternal);
    if (g->nitems > 0)
      k_ms_step<KW><<<gi, kTPB, 0, m.cap>>>(v, m.F, fstride, m.V, m.anyb, d_levels, k, m.ctl, m.scratch,
                                            nullptr);
    cudaEventRecordWithFlags(m.ev[2 * q + 1], m.cap, cudaEventRecordExternal);
    k_ms_finish<KW><<<gs, kTPB, 0, m.cap>>>(v, m.F, fstride, m.V, m.anyb, d_levels, k, m.ctl, m.scratch,
                                              nullptr);
  }
  cudaError_t e = cudaStreamEndCapture(m.cap, &graph);
  if (e != cudaSuccess) return fail_cuda(e, "msbfs capture");
  if (m.exec) cudaGraphExecDestroy(m.exec);
  m.exec = nullptr;
  e = cudaGraphInstantiate(&m.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail_cuda(e, "msbfs instantiate");
  m.launches_per_replay = 8 * ((g->nitems > 0) + 1);
  return GBO_OK;
}

int msbfs_impl(gbo_graph* g, const int* h_srcs, int k, int32_t* d_levels, int* h_depth,
               cudaStream_t s) {
  if (!g->ms) g->ms = new MsHolder();
  MsState& m = reinterpret_cast<MsHolder*>(g->ms)->st;
  int kw = 1;
  while (kw * 32 < k) kw <<= 1;
  const int n = g->nrows;
  if (!m.cap) {
    GBO_CUDA_TRY(cudaStreamCreateWithFlags(&m.cap, cudaStreamNonBlocking));
    GBO_CUDA_TRY(cudaMalloc(&m.ctl, 64));
    GBO_CUDA_TRY(cudaHostAlloc(&m.h_ctl, 64, cudaHostAllocDefault));
    GBO_CUDA_TRY(cudaMalloc(&m.anyb, 2 * (size_t)(g->nbr + 1)));
    for (auto& e : m.ev) GBO_CUDA_TRY(cudaEventCreate(&e));
  }
  if (kw > m.kw) {
    cudaFree(m.F);
    cudaFree(m.V);
    cudaFree(m.scratch);
    m.F = m.V = m.scratch = nullptr;
    GBO_CUDA_TRY(cudaMalloc(&m.F, sizeof(uint32_t) * 2 * (size_t)n * kw + 16));
    GBO_CUDA_TRY(cudaMalloc(&m.V, sizeof(uint32_t) * (size_t)n * kw + 16));
    GBO_CUDA_TRY(cudaMalloc(&m.scratch, sizeof(uint32_t) * (size_t)(g->nslots > 0 ? g->nslots : 1) * 32 * kw));
    m.kw = kw;
    if (m.exec) cudaGraphExecDestroy(m.exec);
    m.exec = nullptr;
  }
  if (k > m.ksrc) {
    cudaFree(m.srcs);
    m.srcs = nullptr;
    GBO_CUDA_TRY(cudaMalloc(&m.srcs, sizeof(int) * (size_t)k));
    m.ksrc = k;
  }
  GBO_CUDA_TRY(cudaMemcpyAsync(m.srcs, h_srcs, sizeof(int) * (size_t)k, cudaMemcpyHostToDevice, s));
  if (!m.exec || m.key_levels != d_levels || m.key_k != k) {
    int st = GBO_OK;
    switch (kw) {
      case 1: st = ms_capture<1>(g, m, d_levels, k); break;
      case 2: st = ms_capture<2>(g, m, d_levels, k); break;
      case 4: st = ms_capture<4>(g, m, d_levels, k); break;
      case 8: st = ms_capture<8>(g, m, d_levels, k); break;
      case 16: st = ms_capture<16>(g, m, d_levels, k); break;
      default: st = ms_capture<32>(g, m, d_levels, k); break;
    }
    GBO_TRY(st);
    m.key_levels = d_levels;
    m.key_k = k;
  }
  const size_t fstride = (size_t)n * m.kw;
  const int max_iter = n + 1;
  unsigned gv = blocks_for((long long)n * k, 256);
  if (gv > (unsigned)num_sms() * 16u) gv = (unsigned)num_sms() * 16u;
  k_ms_init<<<gv, 256, 0, s>>>(m.F, fstride, m.V, m.anyb, g->nbr, d_levels, (long long)n * k, m.kw, n,
                               m.ctl, max_iter);
  k_ms_seed<<<1, 32, 0, s>>>(m.srcs, k, m.kw, m.F, m.V, m.anyb, d_levels, n);
  GBO_CUDA_TRY(cudaGetLastError());
  m.step_ms.clear();
  int it0 = 0;
  const long long max_launch = (long long)max_iter / 8 + 2;
  bool done = false;
  for (long long q = 0; q < max_launch; ++q) {
    GBO_CUDA_TRY(cudaGraphLaunch(m.exec, s));
    GBO_CUDA_TRY(cudaMemcpyAsync(m.h_ctl, m.ctl, 64, cudaMemcpyDeviceToHost, s));
    GBO_CUDA_TRY(cudaStreamSynchronize(s));
    const int it1 = m.h_ctl[0];
    for (int z = 0; z < it1 - it0 && z < 8; ++z) {
      float ms = 0.f;
      if (cudaEventElapsedTime(&ms, m.ev[2 * z], m.ev[2 * z + 1]) != cudaSuccess) {
        ms = -1.f;
        (void)cudaGetLastError();
      }
      m.step_ms.push_back(ms);
    }
    it0 = it1;
    if (m.h_ctl[1]) {
      done = true;
      break;
    }
  }
  if (!done) return fail(GBO_ERR_TIMEOUT, "multi-source BFS did not terminate");
  if (h_depth) *h_depth = m.h_ctl[0];
  return GBO_OK;
}

}  // namespace
}  // namespace gbo

using namespace gbo;

extern "C" int gbo_msbfs(const gbo_graph* gc, const int* h_srcs, int k, int32_t* d_levels,
                         int* h_depth, gbo_stream_t stream) {
  clear_error();
  if (!gc) return fail(GBO_ERR_INVALID, "graph is NULL");
  gbo_graph* g = const_cast<gbo_graph*>(gc);
  if (g->layout != GBO_LAYOUT_ROW || g->nrows != g->ncols)
    return fail(GBO_ERR_INVALID, "multi-source BFS needs a square ROW-layout graph");
  if (g->b != 32) return fail(GBO_ERR_UNSUPPORTED, "multi-source BFS is provided for 32x32 tiles");
  if (k < 1 || k > 1024) return fail(GBO_ERR_INVALID, "k must be in [1, 1024]");
  if (!h_srcs || !d_levels) return fail(GBO_ERR_INVALID, "NULL argument");
  for (int s = 0; s < k; ++s)
    if (h_srcs[s] < 0 || h_srcs[s] >= g->nrows) return fail(GBO_ERR_INVALID, "source out of range");
  return msbfs_impl(g, h_srcs, k, d_levels, h_depth, as_stream(stream));
}

extern "C" int gbo_bfs_multi(const gbo_graph* gc, const int* h_seeds, int nseeds, int32_t* d_level,
                             int* h_depth, gbo_stream_t stream) {
  clear_error();
  if (!gc) return fail(GBO_ERR_INVALID, "graph is NULL");
  gbo_graph* g = const_cast<gbo_graph*>(gc);
  if (g->layout != GBO_LAYOUT_ROW || g->nrows != g->ncols)
    return fail(GBO_ERR_INVALID, "BFS needs a square ROW-layout graph");
  if (nseeds < 1 || !h_seeds || !d_level) return fail(GBO_ERR_INVALID, "bad argument");
  for (int s = 0; s < nseeds; ++s)
    if (h_seeds[s] < 0 || h_seeds[s] >= g->nrows) return fail(GBO_ERR_INVALID, "seed out of range");
  return bfs_seeded(g, h_seeds, nseeds, d_level, h_depth, as_stream(stream));
}
