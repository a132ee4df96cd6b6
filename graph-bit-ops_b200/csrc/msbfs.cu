// Batched traversals: the multi-source BFS API (kernels in ms_kernels.cuh)
// and the multi-seed BFS.
//
// Multi-source BFS: k sources at once; the frontier is an n x k bit matrix,
// so every level is one B2SR x bit-matrix product (OR.AND).  K levels are
// captured once into a CUDA graph, replayed until the device says done.
//
// Multi-seed BFS (gbo_bfs_multi) reuses the single-frontier BFS loop of
// algo.cu with several level-0 vertices; on a block-diagonal union of graphs
// with one seed per graph it is every graph's own BFS in one traversal.
#include <vector>

#include "ms_kernels.cuh"

namespace gbo {

int bfs_seeded(gbo_graph* g, const int* h_seeds, int nseeds, int32_t* d_level, int* h_depth,
               cudaStream_t s);

namespace {

constexpr int kLevelsPerGraph = 8;

struct MsState {
  uint32_t* F = nullptr;  // 2 * n * kw
  uint32_t* V = nullptr;  // n * kw
  uint32_t* fbits = nullptr;
  uint32_t* vfull = nullptr;
  uint32_t* split_acc = nullptr;
  int* slot_split = nullptr;
  uint32_t* push_acc = nullptr;  // nbr * 32 * kw (push levels; k <= 64 on symmetric graphs)
  uint32_t* long_acc = nullptr;  // rws_nlong * 2 (slice steps, k <= 64)
  uint32_t* active = nullptr;    // 32 words: source columns still traversing
  uint32_t* slot_any = nullptr;  // 32 words: columns with a new vertex in the level
  int* srcs = nullptr;
  int* ctl = nullptr;
  int* h_ctl = nullptr;
  const uint32_t* live = nullptr;  // owned by the graph's algorithm state
  int kw = 0;
  int ksrc = 0;
  cudaStream_t cap = nullptr;
  cudaGraphExec_t exec = nullptr;
  const void* key_levels = nullptr;
  int key_k = -1;
  int key_group = -1;
  long long key_push = -1;  // push threshold the graph was captured with (0: pull only)
  std::vector<float> step_ms;
  long long launches = 0;
  int launches_per_replay = 0;
  int fixed_launches = 3;  // launches of a run outside its graph replays
  cudaEvent_t ev[2 * kLevelsPerGraph] = {};
  cudaEvent_t ev0[2] = {};  // level 0 when it runs as a seed push
};

// Levels with fewer new (vertex, source) pairs than this run as pushes: on
// symmetric graphs with k <= 64 when the caller set a positive BFS push
// threshold (gbo_graph_set_bfs_direction); otherwise (0) every level pulls.
long long ms_push_threshold(const gbo_graph* g, int kw) {
  if (!g->symmetric || g->bfs_push_thr <= 0) return 0;
  if (kw > 2 && !g->rws_head) return 0;  // wide frontier rows push over the slices only
  return g->bfs_push_thr;
}

// level_group 0: the API's vertex-major levels[v * k + s]; 32: the query
// server's layout (32-source planes, ms::level_index)
ms::Args make_args(gbo_graph* g, MsState& m, int32_t* d_levels, int k, int level_group) {
  ms::Args a;
  a.v = view_of(g);
  a.F = m.F;
  a.fstride = (size_t)g->nrows * m.kw;
  a.V = m.V;
  a.fbits = m.fbits;
  a.vfull = m.vfull;
  a.levels = d_levels;
  a.k = k;
  a.ctl = m.ctl;
  a.split_acc = m.split_acc;
  a.slot_split = m.slot_split;
  a.slot_any = m.slot_any;
  a.active = m.active;
  a.retire = 1;  // columns whose traversal ended stop keeping rows open
  a.live = m.live;
  a.level_group = level_group;
  a.push_thr = ms_push_threshold(g, m.kw);
  a.dir = a.push_thr > 0 ? 1 : 0;
  a.push_acc = m.push_acc;
  a.long_acc = m.long_acc;
  return a;
}

template <int KW>
int ms_capture(gbo_graph* g, MsState& m, int32_t* d_levels, int k, int level_group) {
  const ms::Args a = make_args(g, m, d_levels, k, level_group);
  // k <= 64 on a graph with row-word slices: the pull step walks rows
  // (k_step_rws, whole block rows: no split partials for the finish kernel);
  // wider frontier rows go through the tiles (k_step), which measured 2x
  // faster than walking the slices at k = 256 and 1024 on R-MAT 21
  const bool rws = KW <= 2 && g->rws_head != nullptr;
  ms::Args af = a;
  if (rws) af.v.nsplit = 0;
  const unsigned gi = rws ? blocks_for_warps(g->nbr > 0 ? g->nbr : 1, ms::kWarps)
                          : blocks_for_warps(g->nitems, ms::kWarps);
  const unsigned gs = blocks_for_warps(af.v.nsplit > 0 ? af.v.nsplit : 1, ms::kWarps);
  cudaGraph_t graph = nullptr;
  // with push levels a slot is push, push-finish, pull, finish (each
  // level runs in one of the two halves) and its events bracket all four
  const unsigned gr = blocks_for_warps(g->nbr > 0 ? g->nbr : 1, ms::kWarps);
  GBO_CUDA_TRY(cudaStreamBeginCapture(m.cap, cudaStreamCaptureModeThreadLocal));
  for (int q = 0; q < kLevelsPerGraph; ++q) {
    cudaEventRecordWithFlags(m.ev[2 * q], m.cap, cudaEventRecordExternal);
    if (a.dir) {
      if (g->rws_head) {  // push over the frontier vertices' own slice entries
        if (g->nitems > 0) ms::k_push_rows<KW><<<gr, ms::kTPB, 0, m.cap>>>(a);
        if (g->rws_nchunk > 0)
          ms::k_push_chunks<KW><<<std::min(blocks_for_warps(g->rws_nchunk, ms::kWarps), (unsigned)num_sms() * 8u),
                                  ms::kTPB, 0, m.cap>>>(a);
      } else if constexpr (KW <= 2) {
        // a warp per work item over the tiles
        if (g->nitems > 0) ms::k_push<KW><<<blocks_for_warps(g->nitems, ms::kWarps), ms::kTPB, 0, m.cap>>>(a);
      }
      ms::k_push_fin<KW><<<gr, ms::kTPB, 0, m.cap>>>(a);
    }
    if (g->nitems > 0) {
      if constexpr (KW <= 2) {
        if (rws && g->rws_nchunk > 0)
          ms::k_long_chunks<KW><<<std::min(blocks_for_warps(g->rws_nchunk, ms::kWarps), (unsigned)num_sms() * 8u),
                                  ms::kTPB, 0, m.cap>>>(a);
        if (rws) ms::k_step_rws<KW><<<gi, ms::kTPB, 0, m.cap>>>(a);
        else ms::k_step<KW><<<gi, ms::kTPB, 0, m.cap>>>(a);
        if (rws && g->rws_nchunk > 0)
          cudaMemsetAsync(m.long_acc, 0, sizeof(uint32_t) * (size_t)g->rws_nlong * KW, m.cap);
      } else {
        ms::k_step<KW><<<gi, ms::kTPB, 0, m.cap>>>(a);
      }
    }
    if (a.dir) ms::k_finish<KW><<<gs, ms::kTPB, 0, m.cap>>>(af);
    cudaEventRecordWithFlags(m.ev[2 * q + 1], m.cap, cudaEventRecordExternal);
    if (!a.dir) ms::k_finish<KW><<<gs, ms::kTPB, 0, m.cap>>>(af);
  }
  cudaError_t e = cudaStreamEndCapture(m.cap, &graph);
  if (e != cudaSuccess) return fail_cuda(e, "multi-source BFS capture");
  if (m.exec) cudaGraphExecDestroy(m.exec);
  m.exec = nullptr;
  e = cudaGraphInstantiate(&m.exec, graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail_cuda(e, "multi-source BFS instantiate");
  m.launches_per_replay = kLevelsPerGraph * ((g->nitems > 0) * (a.dir ? 2 : 1) + 1 + (a.dir ? 1 : 0));
  return GBO_OK;
}

// One multi-source BFS with state m.  Levels are written as lvl0 + hops in
// the layout level_group selects; sources < 0 are empty columns.
int msbfs_impl(gbo_graph* g, MsState& m, const int* h_srcs, int k, int32_t* d_levels, int level_group, int lvl0,
               int* h_depth, cudaStream_t s) {
  int kw = 1;
  while (kw * 32 < k) kw <<= 1;
  const int n = g->nrows;
  if (!m.cap) {
    GBO_CUDA_TRY(cudaStreamCreateWithFlags(&m.cap, cudaStreamNonBlocking));
    GBO_CUDA_TRY(cudaMalloc(&m.ctl, 64));
    GBO_CUDA_TRY(cudaHostAlloc(&m.h_ctl, 64, cudaHostAllocDefault));
    GBO_CUDA_TRY(cudaMalloc(&m.fbits, sizeof(uint32_t) * 2 * (size_t)(g->nbr + 1)));
    GBO_CUDA_TRY(cudaMalloc(&m.vfull, sizeof(uint32_t) * (size_t)(g->nbr + 1)));
    for (auto& e : m.ev) GBO_CUDA_TRY(cudaEventCreate(&e));
    for (auto& e : m.ev0) GBO_CUDA_TRY(cudaEventCreate(&e));
  }
  if (!m.live) {
    const void* lv = nullptr;
    GBO_TRY(live_rows(g, s, &lv));
    m.live = static_cast<const uint32_t*>(lv);
  }
  GBO_TRY(build_rws(g, s));
  if (!m.active) {
    GBO_CUDA_TRY(cudaMalloc(&m.active, sizeof(uint32_t) * 64));
    m.slot_any = m.active + 32;
  }
  if (!m.long_acc && g->rws_head) {  // slice steps: frontier rows of up to 2 words
    const size_t lw = (size_t)(g->rws_nlong > 0 ? g->rws_nlong : 1) * 2;
    GBO_CUDA_TRY(cudaMalloc(&m.long_acc, sizeof(uint32_t) * lw));
    GBO_CUDA_TRY(cudaMemsetAsync(m.long_acc, 0, sizeof(uint32_t) * lw, s));
  }
  if (kw != m.kw) {  // state sized for exactly kw words per vertex
    if (m.exec) cudaGraphExecDestroy(m.exec);
    m.exec = nullptr;
    cudaFree(m.F);
    cudaFree(m.V);
    cudaFree(m.split_acc);
    cudaFree(m.slot_split);
    cudaFree(m.push_acc);
    m.F = m.V = m.split_acc = m.push_acc = nullptr;
    m.slot_split = nullptr;
    m.kw = 0;
    GBO_CUDA_TRY(cudaMalloc(&m.F, sizeof(uint32_t) * 2 * (size_t)n * kw + 16));
    GBO_CUDA_TRY(cudaMalloc(&m.V, sizeof(uint32_t) * (size_t)n * kw + 16));
    GBO_TRY(ms::split_state(g, kw, &m.split_acc, &m.slot_split, s));
    if (kw <= 2 || (g->symmetric && g->rws_head)) {  // push levels' accumulator, zero between levels
      const size_t pw = (size_t)(g->nbr > 0 ? g->nbr : 1) * 32 * (size_t)kw;
      GBO_CUDA_TRY(cudaMalloc(&m.push_acc, sizeof(uint32_t) * pw));
      GBO_CUDA_TRY(cudaMemsetAsync(m.push_acc, 0, sizeof(uint32_t) * pw, s));
    }
    m.kw = kw;
  }
  if (k > m.ksrc) {
    cudaFree(m.srcs);
    m.srcs = nullptr;
    GBO_CUDA_TRY(cudaMalloc(&m.srcs, sizeof(int) * (size_t)k));
    m.ksrc = k;
  }
  GBO_CUDA_TRY(cudaMemcpyAsync(m.srcs, h_srcs, sizeof(int) * (size_t)k, cudaMemcpyHostToDevice, s));
  const long long push_thr = ms_push_threshold(g, kw);
  if (!m.exec || m.key_levels != d_levels || m.key_k != k || m.key_push != push_thr ||
      m.key_group != level_group) {
    int st = GBO_OK;
    switch (kw) {
      case 1: st = ms_capture<1>(g, m, d_levels, k, level_group); break;
      case 2: st = ms_capture<2>(g, m, d_levels, k, level_group); break;
      case 4: st = ms_capture<4>(g, m, d_levels, k, level_group); break;
      case 8: st = ms_capture<8>(g, m, d_levels, k, level_group); break;
      case 16: st = ms_capture<16>(g, m, d_levels, k, level_group); break;
      default: st = ms_capture<32>(g, m, d_levels, k, level_group); break;
    }
    GBO_TRY(st);
    m.key_levels = d_levels;
    m.key_k = k;
    m.key_push = push_thr;
    m.key_group = level_group;
  }
  const ms::Args a = make_args(g, m, d_levels, k, level_group);
  const int max_iter = lvl0 + n + 1;
  unsigned gv = blocks_for((long long)n * k, 256);
  if (gv > (unsigned)num_sms() * 16u) gv = (unsigned)num_sms() * 16u;
  ms::k_init<<<gv, 256, 0, s>>>(a, kw, max_iter, lvl0);
  ms::seed_sources(a, m.srcs, nullptr, k, kw, lvl0, s);
  GBO_CUDA_TRY(cudaGetLastError());
  m.step_ms.clear();
  m.launches = 3;
  // symmetric slice graphs whose levels all pull: level 0 pushes from the k
  // sources instead (k_seed_push, then the push epilogue) -- a pull would
  // walk every row of the graph for a frontier of k vertices
  const bool seed_push = g->symmetric && g->rws_head && !a.dir && g->nitems > 0 && m.push_acc;
  if (seed_push) {
    constexpr int kPieces = 64;  // warps per source: hubs' tails are split
    GBO_CUDA_TRY(cudaEventRecord(m.ev0[0], s));
    switch (kw) {
      case 1: ms::k_seed_push<1><<<blocks_for_warps((long long)k * kPieces, ms::kWarps), ms::kTPB, 0, s>>>(a, m.srcs, k, kPieces); break;
      case 2: ms::k_seed_push<2><<<blocks_for_warps((long long)k * kPieces, ms::kWarps), ms::kTPB, 0, s>>>(a, m.srcs, k, kPieces); break;
      case 4: ms::k_seed_push<4><<<blocks_for_warps((long long)k * kPieces, ms::kWarps), ms::kTPB, 0, s>>>(a, m.srcs, k, kPieces); break;
      case 8: ms::k_seed_push<8><<<blocks_for_warps((long long)k * kPieces, ms::kWarps), ms::kTPB, 0, s>>>(a, m.srcs, k, kPieces); break;
      case 16: ms::k_seed_push<16><<<blocks_for_warps((long long)k * kPieces, ms::kWarps), ms::kTPB, 0, s>>>(a, m.srcs, k, kPieces); break;
      default: ms::k_seed_push<32><<<blocks_for_warps((long long)k * kPieces, ms::kWarps), ms::kTPB, 0, s>>>(a, m.srcs, k, kPieces); break;
    }
    const unsigned gr = blocks_for_warps(g->nbr > 0 ? g->nbr : 1, ms::kWarps);
    switch (kw) {
      case 1: ms::k_push_fin<1><<<gr, ms::kTPB, 0, s>>>(a); break;
      case 2: ms::k_push_fin<2><<<gr, ms::kTPB, 0, s>>>(a); break;
      case 4: ms::k_push_fin<4><<<gr, ms::kTPB, 0, s>>>(a); break;
      case 8: ms::k_push_fin<8><<<gr, ms::kTPB, 0, s>>>(a); break;
      case 16: ms::k_push_fin<16><<<gr, ms::kTPB, 0, s>>>(a); break;
      default: ms::k_push_fin<32><<<gr, ms::kTPB, 0, s>>>(a); break;
    }
    GBO_CUDA_TRY(cudaGetLastError());
    GBO_CUDA_TRY(cudaEventRecord(m.ev0[1], s));
    m.launches += 2;
  }
  m.fixed_launches = (int)m.launches;
  int it0 = lvl0 + (seed_push ? 1 : 0);
  if (seed_push) {  // level 0's time (read once the loop has synchronised)
    m.step_ms.push_back(-1.f);
  }
  long long max_launch = (long long)max_iter / kLevelsPerGraph + 2;
  const long long cap = inject_replay_cap();
  if (cap > 0 && cap < max_launch) max_launch = cap;
  bool done = false;
  for (long long q = 0; q < max_launch; ++q) {
    GBO_CUDA_TRY(cudaGraphLaunch(m.exec, s));
    GBO_CUDA_TRY(cudaMemcpyAsync(m.h_ctl, m.ctl, 64, cudaMemcpyDeviceToHost, s));
    GBO_CUDA_TRY(cudaStreamSynchronize(s));
    m.launches += m.launches_per_replay;
    const int it1 = m.h_ctl[0];
    for (int z = 0; z < it1 - it0 && z < kLevelsPerGraph; ++z) {
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
  if (seed_push && cudaEventElapsedTime(&m.step_ms[0], m.ev0[0], m.ev0[1]) != cudaSuccess) {
    m.step_ms[0] = -1.f;
    (void)cudaGetLastError();
  }
  if (h_depth) *h_depth = m.h_ctl[0] - lvl0;
  return GBO_OK;
}

void destroy_ms(MsState* m) {
  if (!m) return;
  if (m->exec) cudaGraphExecDestroy(m->exec);
  for (auto& e : m->ev)
    if (e) cudaEventDestroy(e);
  cudaFree(m->F);
  cudaFree(m->V);
  cudaFree(m->fbits);
  cudaFree(m->vfull);
  cudaFree(m->split_acc);
  cudaFree(m->slot_split);
  cudaFree(m->push_acc);
  for (auto& e : m->ev0)
    if (e) cudaEventDestroy(e);
  cudaFree(m->long_acc);
  cudaFree(m->active);
  cudaFree(m->srcs);
  cudaFree(m->ctl);
  cudaFreeHost(m->h_ctl);
  if (m->cap) cudaStreamDestroy(m->cap);
  delete m;
}

}  // namespace

int ms_last_run(const gbo_graph* g, gbo_run_stats* st) {
  const MsState* m = reinterpret_cast<const MsState*>(g->ms);
  if (!m) return GBO_OK;
  st->iterations = m->h_ctl ? m->h_ctl[0] : 0;
  st->graph_replays =
      (int)((m->launches - m->fixed_launches) / (m->launches_per_replay > 0 ? m->launches_per_replay : 1));
  st->kernel_launches = m->launches;
  const int n = (int)m->step_ms.size();
  st->nsteps = n < GBO_MAX_STEP_TIMES ? n : GBO_MAX_STEP_TIMES;
  for (int i = 0; i < st->nsteps; ++i) st->step_ms[i] = m->step_ms[(size_t)i];
  return GBO_OK;
}

namespace ms {
namespace {
__global__ void k_slot_split(const gbo_split* __restrict__ splits, int nsplit, int* __restrict__ map) {
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; w < nsplit; w += nwarps) {
    const gbo_split sp = splits[w];
    for (int q = (int)lane; q < sp.nslots; q += 32) map[sp.slot0 + q] = (int)w;
  }
}
}  // namespace

int split_state(const gbo_graph* g, int kw, uint32_t** acc, int** slot_split, cudaStream_t s) {
  const size_t accw = (size_t)(g->nsplit > 0 ? g->nsplit : 1) * 32 * (size_t)kw;
  GBO_CUDA_TRY(cudaMalloc(acc, sizeof(uint32_t) * accw));
  GBO_CUDA_TRY(cudaMemsetAsync(*acc, 0, sizeof(uint32_t) * accw, s));
  GBO_CUDA_TRY(cudaMalloc(slot_split, sizeof(int) * (size_t)(g->nslots > 0 ? g->nslots : 1)));
  if (g->nsplit > 0) {
    const unsigned grid = (unsigned)std::min<long long>(((long long)g->nsplit + 7) / 8, 4096);
    k_slot_split<<<grid, 256, 0, s>>>(g->splits, g->nsplit, *slot_split);
    GBO_CUDA_TRY(cudaGetLastError());
  }
  return GBO_OK;
}
}  // namespace ms

void free_ms_state(gbo_graph* g) {
  destroy_ms(reinterpret_cast<MsState*>(g->ms));
  g->ms = nullptr;
}

// A multi-source BFS state of the caller's own (the query server's batch
// engine), apart from the graph's, so that the server's worker thread and
// the graph's own calls never share one.  live: the graph's rows with an
// entry (live_rows), read by the init kernel.
void* ms_batch_create(const uint32_t* live) {
  MsState* m = new MsState();
  m->live = live;
  return m;
}

void ms_batch_destroy(void* state) { destroy_ms(static_cast<MsState*>(state)); }

int ms_batch_run(gbo_graph* g, void* state, const int* h_srcs, int k, int32_t* d_levels, int level_group, int lvl0,
                 int* h_depth, long long* launches, cudaStream_t s) {
  MsState& m = *static_cast<MsState*>(state);
  const int st = msbfs_impl(g, m, h_srcs, k, d_levels, level_group, lvl0, h_depth, s);
  *launches = m.launches;
  return st;
}

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
  if (!g->ms) g->ms = new MsState();
  const int st = msbfs_impl(g, *reinterpret_cast<MsState*>(g->ms), h_srcs, k, d_levels, 0, 0, h_depth,
                            as_stream(stream));
  if (st == GBO_OK) g->last_run_ms = 1;
  return st;
}

extern "C" int gbo_bfs_multi(const gbo_graph* gc, const int* h_seeds, int nseeds, int32_t* d_level,
                             int* h_depth, gbo_stream_t stream) {
  clear_error();
  if (!gc) return fail(GBO_ERR_INVALID, "graph is NULL");
  gbo_graph* g = const_cast<gbo_graph*>(gc);
  if (g->nrows != g->ncols) return fail(GBO_ERR_INVALID, "BFS needs a square graph");
  if (nseeds < 1 || !h_seeds || !d_level) return fail(GBO_ERR_INVALID, "bad argument");
  for (int s = 0; s < nseeds; ++s)
    if (h_seeds[s] < 0 || h_seeds[s] >= g->nrows) return fail(GBO_ERR_INVALID, "seed out of range");
  return bfs_seeded(g, h_seeds, nseeds, d_level, h_depth, as_stream(stream));
}
