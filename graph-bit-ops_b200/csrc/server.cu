// Query server with continuous batching over a resident graph.
//
// BFS queries occupy columns ("slots") of the multi-source BFS state (bit
// frontier matrix, ms_kernels.cuh); PPR queries occupy columns of a 32-wide
// fp32 value matrix.  One worker thread drives the GPU in rounds: it admits
// waiting queries into free slots (a BFS query joins at the next level
// boundary, a PPR query at the next iteration boundary), runs one BFS level
// and/or one PPR iteration for every occupied slot, retires the slots that
// finished (BFS: no new vertex this level; PPR: L1 change <= tol or the
// iteration cap), copies their results into pinned host buffers and frees the
// slots for the next queries.  A query's result does not depend on the other
// queries in flight: every column is computed independently and in the same
// order (BFS bit-exact; PPR identical arithmetic per column).
//
// Batch mode (gbo_server_set_admission with 1): BFS queries enter only an
// idle engine, and each batch runs as one multi-source BFS (msbfs.cu: level
// 0 pushed from the sources, finished columns retired) in the server's level
// store; the batch's queries all finish in that call and retire as above.
#include <string.h>

#include <chrono>
#include <condition_variable>
#include <algorithm>
#include <cmath>
#include <atomic>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "ms_kernels.cuh"

namespace gbo {

// msbfs.cu: a multi-source BFS state of the server's own
void* ms_batch_create(const uint32_t* live);
void ms_batch_destroy(void* state);
int ms_batch_run(gbo_graph* g, void* state, const int* h_srcs, int k, int32_t* d_levels, int level_group, int lvl0,
                 int* h_depth, long long* launches, cudaStream_t s);

namespace {

constexpr int kPprSlots = 32;
constexpr int kPprTPB = 128;
constexpr int kPprWarps = kPprTPB / 32;

// Wait for the work queued on st with a blocking-sync event: the calling
// thread sleeps instead of spinning, so client threads, the two workers and
// the caller's own threads do not starve each other of host cores.
cudaError_t wait_stream(cudaStream_t st, cudaEvent_t ev) {
  cudaError_t e = cudaEventRecord(ev, st);
  if (e == cudaSuccess) e = cudaEventSynchronize(ev);
  return e;
}

double now_ms() {
  using namespace std::chrono;
  return duration<double, std::milli>(steady_clock::now().time_since_epoch()).count();
}

// ------------------------------------------------------------ PPR kernels
struct PprArgs {
  GView v;
  const float* inv;
  float* X;       // 2 * n * 32, vertex-major
  size_t xstride;
  const float* P;  // (1 - alpha) * personalization, n * 32
  float alpha;
  int parity;      // X half holding the current iterate
  uint32_t active; // slots still iterating; the others keep their column
  double* err;     // 32 slot L1 changes
  double* scratch; // split slots: 32 rows x 32 slots doubles each
};

// One iteration for all 32 slots: X'[i][s] = alpha * sum_{j: P[i][j]} X[j][s]
// inv[j] + P[i][s]; lane = slot; fp64 accumulators in shared memory.
// A warp deals its item's non-empty row words out to the lanes (below); each
// set bit (row r, column j) goes to a per-warp list in shared memory, which
// is then consumed with lane = slot, kP X-row gathers in flight.  The list
// order depends on the graph only, so every column's sum has a fixed order
// whatever the other slots hold.
constexpr int kPprList = 256;

__global__ void __launch_bounds__(kPprTPB) k_ppr_step(PprArgs a) {
  __shared__ double acc_sh[kPprWarps][32 * kPprSlots];
  __shared__ int lj_sh[kPprWarps][kPprList];
  __shared__ unsigned char lr_sh[kPprWarps][kPprList];
  const GView& v = a.v;
  const unsigned lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  double* acc = acc_sh[wib];
  int* lj = lj_sh[wib];
  unsigned char* lr = lr_sh[wib];
  const float* __restrict__ X = a.X + (size_t)a.parity * a.xstride;
  float* __restrict__ Xn = a.X + (size_t)(a.parity ^ 1) * a.xstride;
  double e = 0.0;
  if (item < v.nitems) {
    for (int q = lane; q < 32 * kPprSlots; q += 32) acc[q] = 0.0;
    __syncwarp();
    const gbo_item it = v.items[item];
    const uint32_t* __restrict__ val = reinterpret_cast<const uint32_t*>(v.val);
    const bool lane_active = (a.active >> lane) & 1u;
    constexpr int kP = 8;  // X-row gathers in flight
    int nl = 0;  // list length (warp-uniform)
    auto flush = [&]() {
      for (int q0 = 0; q0 < nl; q0 += kP) {
        int rq[kP];
        float xv[kP], iv[kP];
#pragma unroll
        for (int q = 0; q < kP; ++q) {
          rq[q] = q0 + q < nl ? (int)lr[q0 + q] : -1;
          if (rq[q] >= 0 && lane_active) {
            const size_t jj = (size_t)lj[q0 + q];
            xv[q] = X[jj * kPprSlots + lane];
            iv[q] = a.inv[jj];
          }
        }
#pragma unroll
        for (int q = 0; q < kP; ++q)
          if (rq[q] >= 0 && lane_active) acc[rq[q] * kPprSlots + lane] += (double)(xv[q] * iv[q]);
      }
      nl = 0;
      __syncwarp();
    };
    // Per batch of 32 tiles (lane j: tile j) the non-empty row words -- all
    // 32 rows of every tile without occupancy words -- are dealt out to the
    // lanes in (tile, row) order, 32 per round: lane p takes word p (its
    // tile by a binary search over the prefix counts; with packed row words
    // word p of the batch is simply the next packed word).  Each word's set
    // bits go to the list at positions from a warp prefix sum, at most
    // kPprList / 32 per lane per pass, so the list order -- and with it every
    // sum's order -- depends on the graph only.
    const unsigned* __restrict__ rm = v.rowmask;
    const unsigned* __restrict__ words = v.rowword;
    long long wb = words ? v.item_wbase[item] : 0ll;
    constexpr int kPerPass = kPprList / 32;
    for (int b0 = it.t0; b0 < it.t1; b0 += 32) {
      const int t = b0 + (int)lane;
      const int cb = t < it.t1 ? v.colind[t] : 0;
      const unsigned mw = t < it.t1 ? (rm ? rm[t] : ~0u) : 0u;
      const int mc = __popc(mw);
      const int mi = warp_incl_sum(mc, lane);
      const int mex = mi - mc;
      const int total = __shfl_sync(0xffffffffu, mi, 31);
      const long long wbat = wb;
      wb += total;
      for (int pb = 0; pb < total; pb += 32) {
        const int p = pb + (int)lane;
        int j = 0;
#pragma unroll
        for (int st = 16; st > 0; st >>= 1) {
          const int q = __shfl_sync(0xffffffffu, mi, j + st - 1);
          if (q <= p) j += st;
        }
        const int ej = __shfl_sync(0xffffffffu, mex, j);
        const unsigned mj = __shfl_sync(0xffffffffu, mw, j);
        const int C = __shfl_sync(0xffffffffu, cb, j);
        int r = 0;
        unsigned w = 0u;
        if (p < total) {
          r = (int)__fns(mj, 0, p - ej + 1);
          w = words ? words[wbat + p] : val[(size_t)(b0 + j) * 32 + r];
        }
        while (__any_sync(0xffffffffu, w != 0u)) {
          const int c = min(__popc(w), kPerPass);
          const int ic = warp_incl_sum(c, lane);
          const int tc = __shfl_sync(0xffffffffu, ic, 31);
          if (nl + tc > kPprList) flush();
          int pos = nl + ic - c;
          for (int q = 0; q < c; ++q) {
            const int col = __clz(w);
            w &= ~(0x80000000u >> col);
            lj[pos] = C * 32 + col;
            lr[pos] = (unsigned char)r;
            ++pos;
          }
          nl += tc;
          __syncwarp();
        }
      }
    }
    flush();
    if (it.slot >= 0) {
      double* dst = a.scratch + (size_t)it.slot * 32 * kPprSlots;
      for (int q = lane; q < 32 * kPprSlots; q += 32) dst[q] = acc[q];
    } else {
      for (int r = 0; r < 32; ++r) {
        const long long i = (long long)it.row * 32 + r;
        if (i >= v.nrows) break;
        const size_t o = (size_t)i * kPprSlots + lane;
        if (!((a.active >> lane) & 1u)) {
          Xn[o] = X[o];
          continue;
        }
        const float y = (float)((double)a.alpha * acc[r * kPprSlots + lane] + (double)a.P[o]);
        e += fabs((double)y - (double)X[o]);
        Xn[o] = y;
      }
    }
  }
  __shared__ double es[kPprWarps][32];
  es[wib][lane] = e;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = 0.0;
    for (int q = 0; q < kPprWarps; ++q) t += es[q][threadIdx.x];
    if (t != 0.0) atomicAdd(a.err + threadIdx.x, t);
  }
}

__global__ void __launch_bounds__(kPprTPB) k_ppr_finish(PprArgs a) {
  const GView& v = a.v;
  const unsigned lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const float* __restrict__ X = a.X + (size_t)a.parity * a.xstride;
  float* __restrict__ Xn = a.X + (size_t)(a.parity ^ 1) * a.xstride;
  double e = 0.0;
  if (wid < v.nsplit) {
    const gbo_split sp = v.splits[wid];
    for (int r = 0; r < 32; ++r) {
      const long long i = (long long)sp.row * 32 + r;
      if (i >= v.nrows) break;
      double s = 0.0;
      for (int q = 0; q < sp.nslots; ++q) s += a.scratch[((size_t)(sp.slot0 + q) * 32 + r) * kPprSlots + lane];
      const size_t o = (size_t)i * kPprSlots + lane;
      if (!((a.active >> lane) & 1u)) {
        Xn[o] = X[o];
        continue;
      }
      const float y = (float)((double)a.alpha * s + (double)a.P[o]);
      e += fabs((double)y - (double)X[o]);
      Xn[o] = y;
    }
  }
  __shared__ double es[kPprWarps][32];
  es[wib][lane] = e;
  __syncthreads();
  if (threadIdx.x < 32) {
    double t = 0.0;
    for (int q = 0; q < kPprWarps; ++q) t += es[q][threadIdx.x];
    if (t != 0.0) atomicAdd(a.err + threadIdx.x, t);
  }
}

// Admit PPR queries: column s of P = (1-alpha) v, X (current half) = P.
__global__ void k_ppr_admit(float* X, size_t xstride, int parity, float* P, int n,
                            const int* __restrict__ slots, int nslots_adm,
                            const int* __restrict__ verts, const float* __restrict__ wts,
                            const int* __restrict__ off, float one_minus_alpha) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  float* Xc = X + (size_t)parity * xstride;
  // clear the admitted columns
  for (long long q = i; q < (long long)n * nslots_adm; q += stride) {
    const int a = (int)(q % nslots_adm);
    const long long v0 = q / nslots_adm;
    const size_t o = (size_t)v0 * kPprSlots + slots[a];
    P[o] = 0.f;
    Xc[o] = 0.f;
  }
}

__global__ void k_ppr_admit_set(float* X, size_t xstride, int parity, float* P, int n,
                                const int* __restrict__ slots, int nslots_adm,
                                const int* __restrict__ verts, const float* __restrict__ wts,
                                const int* __restrict__ off, float one_minus_alpha) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  float* Xc = X + (size_t)parity * xstride;
  for (int a = 0; a < nslots_adm; ++a)
    for (int q = off[a]; q < off[a + 1]; ++q) {
      const int v0 = verts[q];
      if (v0 < 0 || v0 >= n) continue;
      const size_t o = (size_t)v0 * kPprSlots + slots[a];
      P[o] += one_minus_alpha * wts[q];
      Xc[o] = P[o];
    }
}

// ------------------------------------------------------------- retirement
// Up to kRetire finished slots of an engine leave per round.  A transposing
// kernel reads their values row by row and writes each result contiguously
// into its own buffer of a device result pool; the result stays there until
// a client takes it (wait/poll copy it to the host), so the engines never
// wait on host copies or on the order in which clients collect.
constexpr int kRetire = 128;
constexpr int kRetRows = 32;  // rows per block of the transposing kernels

// The BFS level store: 32 slots per plane, levels[((s / 32) * n + i) * 32 +
// s % 32] (ms::Args::level_group 32), so that the 32 lanes of a level write
// cover 128 contiguous bytes.  Sector of 8-slot group gid (slots 8 gid ..
// 8 gid + 7) in vertex i's plane row.
__device__ __forceinline__ const int* level_sector(const int* levels, int n, int gid, long long i) {
  return levels + ((size_t)(gid >> 2) * n + i) * 32 + (gid & 3) * 8;
}

struct RetireList {
  int count;
  int slot[kRetire];    // ascending, so the slots of one level group are adjacent
  int start[kRetire];
  uint32_t clr[32];     // visited bits to clear, per source word
  void* out[kRetire];   // destination buffer of each retired slot
  // BFS: the 8-slot groups (one 32-byte sector of a vertex's level row
  // within its 32-slot plane) holding retired slots:
  // group id, index of its first retired slot, which of its 8 slots retire
  int ngroups;
  int group[kRetire];
  short fbeg[kRetire];
  unsigned char mask8[kRetire];
};

// BFS: out[f][i] = level of (i, slot f) relative to its start level, -1 if
// unreachable, and the slot's visited bits become 0.  Levels are absolute
// (the server's level counter), so a slot's column never needs clearing: a
// value older than the query's start level was left by an earlier query of
// the slot and reads as unreachable.  Each thread loads the 32-byte sector of
// one (row, 8-slot group) and keeps the group's retiring slots; results go
// out through shared memory row-contiguous.  When every retired query is
// shallower than 255 levels (u8), a result is one byte per vertex (255 =
// unreachable), a quarter of the bytes the client copies.
__global__ void __launch_bounds__(256) k_bfs_retire(const int* __restrict__ levels, uint32_t* V, int n,
                                                    int kw, RetireList rl, int u8) {
  __shared__ int sm[kRetire][kRetRows + 1];
  const long long i0 = (long long)blockIdx.x * kRetRows;
  for (int q = threadIdx.x; q < kRetRows * rl.ngroups; q += blockDim.x) {
    const int gi = q / kRetRows, ii = q % kRetRows;
    const long long i = i0 + ii;
    if (i >= n) continue;
    const int4* p = reinterpret_cast<const int4*>(level_sector(levels, n, rl.group[gi], i));
    const int4 a = p[0], b = p[1];
    const int lv[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    const unsigned m = rl.mask8[gi];
    int f = rl.fbeg[gi];
#pragma unroll
    for (int w = 0; w < 8; ++w)
      if ((m >> w) & 1u) {
        sm[f][ii] = lv[w] >= rl.start[f] ? lv[w] - rl.start[f] : -1;
        ++f;
      }
  }
  for (int q = threadIdx.x; q < kRetRows * kw; q += blockDim.x) {
    const int ii = q / kw, w = q % kw;
    const long long i = i0 + ii;
    if (i < n && rl.clr[w]) V[(size_t)i * kw + w] &= ~rl.clr[w];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < kRetRows * rl.count; q += blockDim.x) {
    const int f = q / kRetRows, ii = q % kRetRows;
    const long long i = i0 + ii;
    if (i >= n) continue;
    if (u8)
      static_cast<uint8_t*>(rl.out[f])[i] = sm[f][ii] < 0 ? (uint8_t)255 : (uint8_t)sm[f][ii];
    else
      static_cast<int*>(rl.out[f])[i] = sm[f][ii];
  }
}

// Batch mode retirement.  A batch's levels sit vertex-major in their own
// store (blevels[i * k + c], k = the batch's width, the multi-source BFS's
// own layout, whose level writes cover whole 4 KB rows at k = 1,024).  A
// block takes 32 rows and columns c0 .. c0 + ncols - 1: its threads read the
// rows contiguously (16 bytes each), keep the values relative to `start` in
// shared memory as [row][column], and each column's 32 values then go out to
// its buffer as one run (32 bytes as u8, 255 = unreachable; 128 bytes as
// int32, -1).  bufidx[c]: column c's buffer in the pool, -1 for none.  T is
// uint8_t (MAXC 1,024 columns per launch) or int (256).
constexpr int kBatchCols = 1024;
template <typename T, int MAXC>
__global__ void __launch_bounds__(256) k_bfs_retire_batch(const int* __restrict__ levels, int n, int k, int c0,
                                                          int ncols, int start, const int* __restrict__ bufidx,
                                                          char* __restrict__ pool, size_t stride) {
  __shared__ __align__(16) T sm[kRetRows][MAXC];
  const long long i0 = (long long)blockIdx.x * kRetRows;
  const int nq = ncols / 4;
  for (int q = threadIdx.x; q < kRetRows * nq; q += blockDim.x) {
    const int ii = q / nq, c4 = q % nq;
    const long long i = i0 + ii;
    if (i >= n) continue;
    const int4 v = *reinterpret_cast<const int4*>(levels + (size_t)i * k + c0 + 4 * c4);
    const int lv[4] = {v.x, v.y, v.z, v.w};
    T o[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) o[j] = lv[j] >= start ? (T)(lv[j] - start) : (T)(sizeof(T) == 1 ? 255 : -1);
    if constexpr (sizeof(T) == 1) {
      *reinterpret_cast<uint32_t*>(&sm[ii][4 * c4]) =
          (uint32_t)o[0] | (uint32_t)o[1] << 8 | (uint32_t)o[2] << 16 | (uint32_t)o[3] << 24;
    } else {
      *reinterpret_cast<int4*>(&sm[ii][4 * c4]) = make_int4(o[0], o[1], o[2], o[3]);
    }
  }
  __syncthreads();
  for (int c = threadIdx.x; c < ncols; c += blockDim.x) {
    const int b = bufidx[c0 + c];
    if (b < 0) continue;
    T* dst = reinterpret_cast<T*>(pool + (size_t)b * stride) + i0;
    if constexpr (sizeof(T) == 1) {
      uint32_t w[8];
#pragma unroll
      for (int r = 0; r < 8; ++r)
        w[r] = (uint32_t)sm[4 * r][c] | (uint32_t)sm[4 * r + 1][c] << 8 | (uint32_t)sm[4 * r + 2][c] << 16 |
               (uint32_t)sm[4 * r + 3][c] << 24;
      reinterpret_cast<uint4*>(dst)[0] = make_uint4(w[0], w[1], w[2], w[3]);
      reinterpret_cast<uint4*>(dst)[1] = make_uint4(w[4], w[5], w[6], w[7]);
    } else {
#pragma unroll
      for (int r = 0; r < kRetRows; r += 4)
        reinterpret_cast<int4*>(dst)[r / 4] = make_int4(sm[r][c], sm[r + 1][c], sm[r + 2][c], sm[r + 3][c]);
    }
  }
}

// PPR: out[f][i] = X[i][slot f] of the current iterate.
__global__ void __launch_bounds__(256) k_ppr_retire(const float* X, int n, RetireList rl) {
  __shared__ float sm[kRetire][kRetRows + 1];
  const long long i0 = (long long)blockIdx.x * kRetRows;
  const int R = rl.count;
  for (int q = threadIdx.x; q < kRetRows * R; q += blockDim.x) {
    const int ii = q / R, f = q % R;
    const long long i = i0 + ii;
    if (i < n) sm[f][ii] = X[(size_t)i * kPprSlots + rl.slot[f]];
  }
  __syncthreads();
  for (int q = threadIdx.x; q < kRetRows * R; q += blockDim.x) {
    const int f = q / kRetRows, ii = q % kRetRows;
    const long long i = i0 + ii;
    if (i < n) static_cast<float*>(rl.out[f])[i] = sm[f][ii];
  }
}

// After visited columns were cleared no row is "all sources visited" any
// more: keep only the padding rows marked.
__global__ void k_vfull_reset(uint32_t* vfull, const uint32_t* __restrict__ live, int nbr, int n) {
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q <= nbr;
       q += (long long)gridDim.x * blockDim.x) {
    const long long lo = q * 32;
    uint32_t pad = 0;
    for (int r = 0; r < 32; ++r)
      if (lo + r >= n) pad |= 1u << (31 - r);
    if (q < nbr) pad |= ~live[q];  // rows without entries stay closed
    vfull[q] = pad;
  }
}

struct Query {
  long long ticket;
  int kind;  // 0 BFS, 1 PPR
  int src;
  std::vector<int> verts;
  std::vector<float> wts;
  double t_submit;
};

struct Result {
  int kind;
  int pool;         // 0: byte pool (BFS levels < 255), 1: word pool (PPR, deep BFS)
  int buf;          // buffer index in that pool (-1: moved to host memory)
  int u8;           // BFS levels stored one byte per vertex (255 = unreachable)
  cudaEvent_t ev;   // the result is in its buffer once this event completes
  double t_submit, t_done;
  int iters;
  bool moving = false;             // being copied to host memory by a worker
  std::vector<unsigned char> host;  // the result once moved out of the pool
};

}  // namespace
}  // namespace gbo

struct gbo_server {
  gbo_graph* g = nullptr;
  int n = 0, nbr = 0;
  long long max_pending = 0;  // per engine; 0 = unbounded (gbo_server_set_queue_limit)
  float bfs_admit_free = 0.5f;  // gbo_server_set_admission
  uint32_t* long_acc = nullptr;  // up to 64 slots: long-row tail gathers (ms::Args::long_acc)
  // batch mode's multi-source BFS states, one per frontier width (1..32
  // words per vertex, created on first use): a batch of m queries runs
  // with the narrowest width that holds m columns
  void* msb[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  float alpha = 0.85f, tol = 1e-7f;
  int ppr_max_iter = 1000;
  // one worker thread per engine (0 BFS, 1 PPR), each with its own stream,
  // so the engines overlap on the GPU
  cudaStream_t s[2] = {nullptr, nullptr};
  cudaEvent_t sync_ev[2] = {nullptr, nullptr};  // blocking-sync events of the workers
  int dev = 0;
  // BFS engine (levels in 32-slot planes, level_sector)
  int kb = 0, kw = 0;
  uint32_t *F = nullptr, *V = nullptr, *fbits = nullptr, *vfull = nullptr, *split_acc = nullptr;
  int* slot_split = nullptr;
  int* levels = nullptr;
  int* ctl = nullptr;
  uint32_t* slot_any = nullptr;
  uint32_t* h_slot_any = nullptr;
  uint32_t* d_active = nullptr;  // columns still traversing (kw words)
  std::vector<uint32_t> h_active;
  bool reopen = false;           // active set grew: rows marked finished reopen
  const uint32_t* live = nullptr;  // rows of P with an entry (owned by the graph)
  int *d_adm_src = nullptr, *d_adm_slot = nullptr;
  int* d_bufidx = nullptr;  // batch retirement: pool buffer of each slot column
  // batch mode: the level store of the last batch (vertex-major, n x width;
  // created on first use), and that batch while its results retire
  int* blevels = nullptr;
  bool bpend = false;
  int blvl0 = 0, bdepth = 0, bwidth = 0;
  int level = 0;
  // the round-by-round engine reads the frontier buffer of parity level & 1,
  // written by the round before; after a batch of odd depth the next round
  // moves one level further, so that it reads the buffer its last round left
  // empty
  bool parity_fix = false;
  std::vector<long long> bslot_ticket;
  std::vector<char> bslot_batch;  // the slot's query ran in a batch (its visited bits were never set)
  std::vector<int> bslot_start;
  std::vector<char> bslot_finished;
  // PPR engine
  float *X = nullptr, *P = nullptr;
  double* err = nullptr;
  double* h_err = nullptr;
  double* pscratch = nullptr;
  int *d_pslots = nullptr, *d_pverts = nullptr, *d_poff = nullptr;
  float* d_pwts = nullptr;
  int parity = 0;
  std::vector<long long> pslot_ticket;
  std::vector<int> pslot_iters;
  std::vector<char> pslot_finished;
  // results wait on the device: pool 0 holds n-byte buffers (BFS levels),
  // pool 1 n-word buffers (PPR values, BFS levels of deep queries)
  char* dpool[2] = {nullptr, nullptr};
  size_t dbytes[2] = {0, 0};       // bytes per buffer
  std::vector<int> pool_free[2];
  std::vector<cudaEvent_t> pool_ev[2];
  // host side
  std::mutex mu;
  std::condition_variable cv_work, cv_done;
  std::deque<gbo::Query> pending[2];
  std::map<long long, gbo::Result> results;
  std::map<long long, double> submit_time;
  long long next_ticket = 1;
  bool stop = false;
  int worker_status = GBO_OK;
  std::string worker_error;
  std::thread worker[2];
  // statistics
  std::atomic<long long> rounds{0}, launches{0};
  long long bfs_done = 0, ppr_done = 0;
  double phase_ms[4] = {0, 0, 0, 0};  // BFS round, PPR round, retire, client copies (under mu)
  double copy_parts[3] = {0, 0, 0};   // client copies: event wait, device-to-host, widening
};

namespace gbo {
namespace {

ms::Args bfs_args(gbo_server* S) {
  ms::Args a;
  a.v = view_of(S->g);
  a.F = S->F;
  a.fstride = (size_t)S->n * S->kw;
  a.V = S->V;
  a.fbits = S->fbits;
  a.vfull = S->vfull;
  a.levels = S->levels;
  a.k = S->kb;
  a.ctl = S->ctl;
  a.split_acc = S->split_acc;
  a.slot_split = S->slot_split;
  a.slot_any = S->slot_any;
  a.live = S->live;
  a.active = S->d_active;
  a.level_group = 32;
  a.long_acc = S->long_acc;
  return a;
}

template <int KW>
int bfs_round(gbo_server* S, std::vector<std::pair<int, gbo::Query>>& adm) {
  if (S->parity_fix) {
    S->level += 1;
    S->parity_fix = false;
    for (auto& q : adm) S->bslot_start[(size_t)q.first] = S->level;
  }
  const ms::Args a = bfs_args(S);
  cudaStream_t st = S->s[0];
  // columns still traversing; rows marked finished for the old set reopen
  // when the set grows
  for (int w = 0; w < S->kw; ++w) S->h_active[(size_t)w] = 0u;
  for (int q = 0; q < S->kb; ++q)
    if (S->bslot_ticket[(size_t)q] > 0 && !S->bslot_finished[(size_t)q]) S->h_active[(size_t)(q / 32)] |= 1u << (q % 32);
  GBO_CUDA_TRY(cudaMemcpyAsync(S->d_active, S->h_active.data(), sizeof(uint32_t) * S->kw, cudaMemcpyHostToDevice, st));
  if (!adm.empty()) {
    k_vfull_reset<<<blocks_for(S->nbr + 1, 256), 256, 0, st>>>(S->vfull, S->live, S->nbr, S->n);
    S->launches++;
  }
  if (!adm.empty()) {
    std::vector<int> src, slot;
    for (auto& q : adm) {
      slot.push_back(q.first);
      src.push_back(q.second.src);
    }
    GBO_CUDA_TRY(cudaMemcpyAsync(S->d_adm_src, src.data(), sizeof(int) * src.size(), cudaMemcpyHostToDevice, st));
    GBO_CUDA_TRY(cudaMemcpyAsync(S->d_adm_slot, slot.data(), sizeof(int) * slot.size(), cudaMemcpyHostToDevice, st));
    ms::seed_sources(a, S->d_adm_src, S->d_adm_slot, (int)src.size(), S->kw, S->level, st);
    S->launches += 2;
  }
  int h[4] = {S->level, 0, 0, 0x7fffffff};  // level, not done, ticket 0, no iteration cap
  GBO_CUDA_TRY(cudaMemcpyAsync(S->ctl, h, sizeof(h), cudaMemcpyHostToDevice, st));
  GBO_CUDA_TRY(cudaMemsetAsync(S->ctl + 4, 0, 8, st));
  GBO_CUDA_TRY(cudaMemsetAsync(S->slot_any, 0, sizeof(uint32_t) * S->kw, st));
  // up to 64 slots with row-word slices: the row-walking step (whole block
  // rows, so no split partials for the finish kernel)
  const bool rws = KW <= 2 && S->g->rws_head != nullptr;
  ms::Args af = a;
  if (rws) af.v.nsplit = 0;
  const unsigned gi = rws ? blocks_for_warps(S->nbr > 0 ? S->nbr : 1, ms::kWarps)
                          : blocks_for_warps(S->g->nitems, ms::kWarps);
  const unsigned gs = blocks_for_warps(af.v.nsplit > 0 ? af.v.nsplit : 1, ms::kWarps);
  if (S->g->nitems > 0) {
    if constexpr (KW <= 2) {
      if (rws && S->g->rws_nchunk > 0) {
        ms::k_long_chunks<KW><<<std::min(blocks_for_warps(S->g->rws_nchunk, ms::kWarps), (unsigned)num_sms() * 8u),
                                ms::kTPB, 0, st>>>(a);
        S->launches++;
      }
      if (rws) ms::k_step_rws<KW><<<gi, ms::kTPB, 0, st>>>(a);
      else ms::k_step<KW><<<gi, ms::kTPB, 0, st>>>(a);
      if (rws && S->g->rws_nchunk > 0)
        GBO_CUDA_TRY(cudaMemsetAsync(S->long_acc, 0, sizeof(uint32_t) * (size_t)S->g->rws_nlong * KW, st));
    } else {
      ms::k_step<KW><<<gi, ms::kTPB, 0, st>>>(a);
    }
  }
  ms::k_finish<KW><<<gs, ms::kTPB, 0, st>>>(af);
  S->launches += 2;
  GBO_CUDA_TRY(cudaGetLastError());
  GBO_CUDA_TRY(cudaMemcpyAsync(S->h_slot_any, S->slot_any, sizeof(uint32_t) * S->kw, cudaMemcpyDeviceToHost, st));
  GBO_CUDA_TRY(wait_stream(st, S->sync_ev[0]));
  S->level += 1;
  std::lock_guard<std::mutex> lk(S->mu);  // finished flags are read by the other worker
  for (int q = 0; q < S->kb; ++q)
    if (S->bslot_ticket[q] > 0 && !S->bslot_finished[q] && !((S->h_slot_any[q / 32] >> (q % 32)) & 1u))
      S->bslot_finished[q] = 1;
  return GBO_OK;
}

// Pool of a finished BFS slot's result: bytes when the query is shallower
// than 255 levels (a batch query: the batch's depth).
int bfs_slot_pool(const gbo_server* S, int q) {
  const int depth = S->bslot_batch[(size_t)q] ? S->bdepth : S->level - S->bslot_start[(size_t)q];
  return depth < 255 ? 0 : 1;
}

// Batch mode: the finished queries of the last batch into their pool, as
// many as have a free buffer (the rest wait, like round-by-round results,
// for clients or the move to host memory), with one launch for byte results
// and one per 256 columns for int32 ones.
int retire_batch(gbo_server* S) {
  if (!S->bpend) return GBO_OK;
  const int p = S->bdepth < 255 ? 0 : 1;
  const int width = S->bwidth;
  std::vector<int> idx((size_t)width, -1);
  std::vector<std::pair<int, int>> took;  // slot, buffer
  bool left = false;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    for (int q = 0; q < width; ++q) {
      if (!S->bslot_batch[(size_t)q] || S->bslot_ticket[(size_t)q] <= 0 || !S->bslot_finished[(size_t)q]) continue;
      if (S->pool_free[p].empty()) {
        left = true;
        break;
      }
      const int b = S->pool_free[p].back();
      S->pool_free[p].pop_back();
      idx[(size_t)q] = b;
      took.emplace_back(q, b);
    }
  }
  if (!left) S->bpend = false;
  if (took.empty()) return GBO_OK;
  cudaStream_t st = S->s[0];
  GBO_CUDA_TRY(cudaMemcpyAsync(S->d_bufidx, idx.data(), sizeof(int) * (size_t)width, cudaMemcpyHostToDevice, st));
  const unsigned grid = blocks_for(S->n, kRetRows);
  if (p == 0) {
    k_bfs_retire_batch<uint8_t, kBatchCols><<<grid, 256, 0, st>>>(S->blevels, S->n, width, 0, width, S->blvl0,
                                                                  S->d_bufidx, S->dpool[0], S->dbytes[0]);
    S->launches++;
  } else {
    for (int c0 = 0; c0 < width; c0 += 256) {
      k_bfs_retire_batch<int, 256><<<grid, 256, 0, st>>>(S->blevels, S->n, width, c0, std::min(256, width - c0),
                                                         S->blvl0, S->d_bufidx, S->dpool[1], S->dbytes[1]);
      S->launches++;
    }
  }
  GBO_CUDA_TRY(cudaGetLastError());
  for (auto& t : took) GBO_CUDA_TRY(cudaEventRecord(S->pool_ev[p][(size_t)t.second], st));
  const double t_now = now_ms();
  std::lock_guard<std::mutex> lk(S->mu);
  for (auto& t : took) {
    const int q = t.first;
    const long long tk = S->bslot_ticket[(size_t)q];
    Result r;
    r.kind = 0;
    r.pool = p;
    r.buf = t.second;
    r.u8 = p == 0;
    r.ev = S->pool_ev[p][(size_t)t.second];
    r.t_submit = S->submit_time[tk];
    r.t_done = t_now;
    r.iters = S->bdepth;
    S->results[tk] = r;
    S->bslot_ticket[(size_t)q] = 0;
    S->bslot_finished[(size_t)q] = 0;
    S->bfs_done++;
  }
  S->cv_done.notify_all();
  return GBO_OK;
}

// Batch mode: the admitted queries (the engine was idle, so admission took
// the lowest slots) as one multi-source BFS of the narrowest width that holds
// them, empty columns with no source, into the batch level store (vertex-
// major, apart from the round-by-round engine's).  Every query finishes
// here; the level counter moves past the batch (with the frontier parity
// kept for the round-by-round engine).
int bfs_batch(gbo_server* S, std::vector<std::pair<int, gbo::Query>>& adm) {
  int top = 0;
  for (auto& q : adm) top = std::max(top, q.first + 1);
  int w = 1, wi = 0;
  while (w * 32 < top) w <<= 1, ++wi;
  if (!S->blevels) GBO_CUDA_TRY(cudaMalloc(&S->blevels, sizeof(int) * (size_t)S->n * S->kb + 16));
  if (!S->msb[wi]) S->msb[wi] = ms_batch_create(S->live);
  std::vector<int> src((size_t)w * 32, -1);
  for (auto& q : adm) {
    src[(size_t)q.first] = q.second.src;
    S->bslot_batch[(size_t)q.first] = 1;
  }
  const int lvl0 = S->level;
  int depth = 0;
  long long nl = 0;
  GBO_TRY(ms_batch_run(S->g, S->msb[wi], src.data(), w * 32, S->blevels, 0, lvl0, &depth, &nl, S->s[0]));
  S->launches += nl;
  S->level = lvl0 + depth;
  S->parity_fix = (S->parity_fix != ((depth & 1) != 0));
  {
    std::lock_guard<std::mutex> lk(S->mu);
    for (auto& q : adm) S->bslot_finished[(size_t)q.first] = 1;
    S->bpend = true;
    S->blvl0 = lvl0;
    S->bdepth = depth;
    S->bwidth = w * 32;
  }
  return retire_batch(S);
}

int ppr_round(gbo_server* S, std::vector<std::pair<int, gbo::Query>>& adm) {
  cudaStream_t st = S->s[1];
  const size_t xstride = (size_t)S->n * kPprSlots;
  if (!adm.empty()) {
    std::vector<int> slots, verts, off(1, 0);
    std::vector<float> wts;
    for (auto& q : adm) {
      slots.push_back(q.first);
      for (size_t k = 0; k < q.second.verts.size(); ++k) {
        verts.push_back(q.second.verts[k]);
        wts.push_back(q.second.wts[k]);
      }
      off.push_back((int)verts.size());
    }
    GBO_CUDA_TRY(cudaMemcpyAsync(S->d_pslots, slots.data(), sizeof(int) * slots.size(), cudaMemcpyHostToDevice, st));
    GBO_CUDA_TRY(cudaMemcpyAsync(S->d_pverts, verts.data(), sizeof(int) * verts.size(), cudaMemcpyHostToDevice, st));
    GBO_CUDA_TRY(cudaMemcpyAsync(S->d_pwts, wts.data(), sizeof(float) * wts.size(), cudaMemcpyHostToDevice, st));
    GBO_CUDA_TRY(cudaMemcpyAsync(S->d_poff, off.data(), sizeof(int) * off.size(), cudaMemcpyHostToDevice, st));
    unsigned gv = blocks_for((long long)S->n * (long long)slots.size(), 256);
    if (gv > 4096u) gv = 4096u;
    k_ppr_admit<<<gv, 256, 0, st>>>(S->X, xstride, S->parity, S->P, S->n, S->d_pslots, (int)slots.size(),
                                    S->d_pverts, S->d_pwts, S->d_poff, 1.f - S->alpha);
    k_ppr_admit_set<<<1, 32, 0, st>>>(S->X, xstride, S->parity, S->P, S->n, S->d_pslots,
                                      (int)slots.size(), S->d_pverts, S->d_pwts, S->d_poff,
                                      1.f - S->alpha);
    S->launches += 2;
  }
  PprArgs a;
  a.v = view_of(S->g);
  a.inv = S->g->invdeg;
  a.X = S->X;
  a.xstride = xstride;
  a.P = S->P;
  a.alpha = S->alpha;
  a.parity = S->parity;
  a.active = 0u;
  for (int q = 0; q < kPprSlots; ++q)
    if (S->pslot_ticket[(size_t)q] > 0 && !S->pslot_finished[(size_t)q]) a.active |= 1u << q;
  a.err = S->err;
  a.scratch = S->pscratch;
  GBO_CUDA_TRY(cudaMemsetAsync(S->err, 0, sizeof(double) * kPprSlots, st));
  const unsigned gi = blocks_for_warps(S->g->nitems, kPprWarps);
  if (S->g->nitems > 0) k_ppr_step<<<gi, kPprTPB, 0, st>>>(a);
  if (S->g->nsplit > 0) k_ppr_finish<<<blocks_for_warps(S->g->nsplit, kPprWarps), kPprTPB, 0, st>>>(a);
  S->launches += 2;
  GBO_CUDA_TRY(cudaGetLastError());
  GBO_CUDA_TRY(cudaMemcpyAsync(S->h_err, S->err, sizeof(double) * kPprSlots, cudaMemcpyDeviceToHost, st));
  GBO_CUDA_TRY(wait_stream(st, S->sync_ev[1]));
  S->parity ^= 1;
  std::lock_guard<std::mutex> lk(S->mu);  // finished flags are read by the other worker
  for (int q = 0; q < kPprSlots; ++q) {
    if (S->pslot_ticket[q] <= 0 || S->pslot_finished[q]) continue;
    S->pslot_iters[q] += 1;
    if ((S->tol >= 0 && S->h_err[q] <= (double)S->tol) || S->pslot_iters[q] >= S->ppr_max_iter)
      S->pslot_finished[q] = 1;
  }
  return GBO_OK;
}

// Retire finished slots of one engine (kind 0 BFS, 1 PPR) into free device
// result buffers.  Called without the lock.
int retire(gbo_server* S, int kind) {
  std::vector<long long>& tick = kind == 0 ? S->bslot_ticket : S->pslot_ticket;
  std::vector<char>& fin = kind == 0 ? S->bslot_finished : S->pslot_finished;
  // BFS results of queries shallower than 255 levels go to the byte pool,
  // the others to the word pool; one launch per pool
  RetireList rl[2];
  std::vector<int> bufs[2];
  for (int p = 0; p < 2; ++p) memset(&rl[p], 0, sizeof(RetireList));
  {
    std::lock_guard<std::mutex> lk(S->mu);
    for (size_t q = 0; q < tick.size(); ++q) {
      if (tick[q] <= 0 || !fin[q] || (kind == 0 && S->bslot_batch[q])) continue;  // batches: retire_batch
      const int p = kind == 0 ? bfs_slot_pool(S, (int)q) : 1;
      if (rl[p].count >= kRetire || S->pool_free[p].empty()) continue;
      const int b = S->pool_free[p].back();
      S->pool_free[p].pop_back();
      RetireList& r = rl[p];
      r.slot[r.count] = (int)q;
      r.start[r.count] = kind == 0 ? S->bslot_start[q] : 0;
      r.out[r.count] = S->dpool[p] + (size_t)b * S->dbytes[p];
      if (kind == 0 && !S->bslot_batch[q]) r.clr[q / 32] |= 1u << (q % 32);
      bufs[p].push_back(b);
      r.count++;
    }
  }
  cudaStream_t st = S->s[kind];
  const unsigned grid = blocks_for(S->n, kRetRows);
  const double t_now = now_ms();
  for (int p = 0; p < 2; ++p) {
    if (rl[p].count == 0) continue;
    RetireList& r = rl[p];
    r.ngroups = 0;
    for (int f = 0; f < r.count; ++f) {  // slots ascend: a group's slots are adjacent
      const int gid = r.slot[f] / 8;
      if (r.ngroups == 0 || r.group[r.ngroups - 1] != gid) {
        r.group[r.ngroups] = gid;
        r.fbeg[r.ngroups] = (short)f;
        r.mask8[r.ngroups] = 0;
        r.ngroups++;
      }
      r.mask8[r.ngroups - 1] |= (unsigned char)(1u << (r.slot[f] % 8));
    }
    // retired columns were already out of the active set: rows marked
    // finished stay finished
    if (kind == 0) k_bfs_retire<<<grid, 256, 0, st>>>(S->levels, S->V, S->n, S->kw, rl[p], p == 0);
    else k_ppr_retire<<<grid, 256, 0, st>>>(S->X + (size_t)S->parity * S->n * kPprSlots, S->n, rl[p]);
    S->launches += 1;
    GBO_CUDA_TRY(cudaGetLastError());
    for (int b : bufs[p]) GBO_CUDA_TRY(cudaEventRecord(S->pool_ev[p][(size_t)b], st));
    std::lock_guard<std::mutex> lk(S->mu);
    for (int f = 0; f < rl[p].count; ++f) {
      const int q = rl[p].slot[f];
      const long long t = tick[(size_t)q];
      Result r;
      r.kind = kind;
      r.pool = p;
      r.buf = bufs[p][(size_t)f];
      r.u8 = kind == 0 && p == 0;
      r.ev = S->pool_ev[p][(size_t)r.buf];
      r.t_submit = S->submit_time[t];
      r.t_done = t_now;
      r.iters = kind == 0 ? S->level - S->bslot_start[(size_t)q] : S->pslot_iters[(size_t)q];
      S->results[t] = r;
      tick[(size_t)q] = 0;
      fin[(size_t)q] = 0;
      if (kind == 0) S->bfs_done++;
      else S->ppr_done++;
    }
    S->cv_done.notify_all();
  }
  return GBO_OK;
}

// Pool that finished slots of this engine wait for while it has no free
// buffer, or -1 (caller holds the lock).
int blocked_pool(gbo_server* S, int kind) {
  const std::vector<long long>& tab = kind == 0 ? S->bslot_ticket : S->pslot_ticket;
  const std::vector<char>& fin = kind == 0 ? S->bslot_finished : S->pslot_finished;
  for (size_t q = 0; q < tab.size(); ++q) {
    if (tab[q] <= 0 || !fin[q]) continue;
    const int p = kind == 0 ? bfs_slot_pool(S, (int)q) : 1;
    if (S->pool_free[p].empty()) return p;
  }
  return -1;
}

// Clients may collect in any order, so uncollected results can hold every
// buffer of a pool while finished queries wait for one: then the oldest
// results of that pool move to host memory (the copies run without the
// lock; clients wait until a result has moved).  Called and returns with lk
// held.
bool move_results_to_host(gbo_server* S, int p, std::unique_lock<std::mutex>& lk) {
  std::vector<std::pair<long long, Result*>> jobs;
  for (auto& kv : S->results) {
    Result& r = kv.second;
    if (r.pool != p || r.buf < 0 || r.moving) continue;
    r.moving = true;
    jobs.emplace_back(kv.first, &r);  // map nodes stay put while others change
    if ((int)jobs.size() == kRetire) break;
  }
  if (jobs.empty()) return false;
  lk.unlock();
  cudaError_t e = cudaSuccess;
  for (auto& j : jobs) {
    Result& r = *j.second;
    r.host.resize(r.u8 ? (size_t)S->n : sizeof(int) * (size_t)S->n);
    if (e == cudaSuccess) e = cudaEventSynchronize(r.ev);
    if (e == cudaSuccess)
      e = cudaMemcpy(r.host.data(), S->dpool[p] + (size_t)r.buf * S->dbytes[p], r.host.size(),
                     cudaMemcpyDeviceToHost);
  }
  lk.lock();
  for (auto& j : jobs) {
    Result& r = *j.second;
    S->pool_free[p].push_back(r.buf);
    r.buf = -1;
    r.moving = false;
  }
  S->cv_done.notify_all();
  if (e != cudaSuccess) {
    S->worker_status = fail_cuda(e, "server result move");
    S->worker_error = gbo_last_error();
  }
  return true;
}

void worker_main(gbo_server* S, int kind) {
  cudaSetDevice(S->dev);
  auto failw = [&](int st) {
    std::lock_guard<std::mutex> lk(S->mu);
    S->worker_status = st;
    S->worker_error = gbo_last_error();
    S->cv_done.notify_all();
  };
  std::vector<long long>& tab = kind == 0 ? S->bslot_ticket : S->pslot_ticket;
  std::vector<char>& fin = kind == 0 ? S->bslot_finished : S->pslot_finished;
  auto occupied = [&]() {
    for (long long t : tab)
      if (t > 0) return true;
    return false;
  };
  auto unfinished = [&]() {
    for (size_t q = 0; q < tab.size(); ++q)
      if (tab[q] > 0 && !fin[q]) return true;
    return false;
  };
  // Every query in flight keeps one result buffer of its pool in reserve
  // (BFS: the byte pool, PPR: the word pool), so a finished query can always
  // retire and the engines never wait on clients mid-traversal; queries past
  // that budget stay pending.
  const int rpool = kind == 0 ? 0 : 1;
  auto budget = [&]() {
    long long inflight = 0;
    for (long long t : tab) inflight += t > 0;
    return (long long)S->pool_free[rpool].size() - inflight;
  };
  // BFS admission batching (gbo_server_set_admission): enough free slots,
  // or nothing left traversing; batch mode: every slot free and retired
  auto batch_ready = [&]() {
    if (S->bfs_admit_free >= 1.f) return !occupied();
    long long nfree = 0;
    for (long long t : tab) nfree += t == 0;
    const double need = std::ceil((double)S->bfs_admit_free * (double)tab.size());
    return (double)nfree >= std::max(need, 1.0) || !unfinished();
  };
  double stall_since = -1.0;
  while (true) {
    std::vector<std::pair<int, Query>> adm;
    bool batch = false;  // the admitted queries run as one multi-source BFS
    {
      std::unique_lock<std::mutex> lk(S->mu);
      for (;;) {
        if (S->stop || S->worker_status != GBO_OK) return;
        const int bp = blocked_pool(S, kind);
        if (bp >= 0) move_results_to_host(S, bp, lk);
        const bool can_admit = !S->pending[kind].empty() && budget() > 0 && !inject_server_hold() &&
                               (kind != 0 || batch_ready());
        const bool work = can_admit || unfinished() || (occupied() && blocked_pool(S, kind) < 0);
        if (work) {
          stall_since = -1.0;
          break;
        }
        if (!S->pending[kind].empty()) {
          // every buffer of the pool holds a result nobody has taken: wait a
          // little for clients, then move results to host memory (a client
          // may be waiting for a query that is still pending)
          const double now = now_ms();
          if (stall_since < 0) stall_since = now;
          if (now - stall_since > 100.0) {
            move_results_to_host(S, rpool, lk);
            stall_since = -1.0;
            continue;
          }
        }
        // submit, take and destroy notify; the timeout bounds a missed wake-up
        S->cv_work.wait_for(lk, std::chrono::milliseconds(20));
      }
      // admission into free slots, arrival order, within the buffer budget
      size_t nx = 0;
      std::deque<Query>& pend = S->pending[kind];
      // BFS admission waits for its batching condition here too: the worker
      // also gets here with queries still traversing
      long long room = inject_server_hold() || (kind == 0 && !batch_ready()) ? 0 : budget();
      while (!pend.empty() && room > 0) {
        while (nx < tab.size() && tab[nx] != 0) ++nx;
        if (nx >= tab.size()) break;
        Query q = std::move(pend.front());
        pend.pop_front();
        const int slot = (int)nx++;
        tab[(size_t)slot] = q.ticket;
        fin[(size_t)slot] = 0;
        if (kind == 0) {
          S->bslot_start[(size_t)slot] = S->level;
          S->bslot_batch[(size_t)slot] = 0;
        }
        else S->pslot_iters[(size_t)slot] = 0;
        adm.emplace_back(slot, std::move(q));
        --room;
      }
      batch = kind == 0 && !adm.empty() && S->bfs_admit_free >= 1.f;
    }
    int st = GBO_OK;
    const bool busy = !adm.empty() || unfinished();
    const double t0 = now_ms();
    if (busy) {
      if (batch) {
        st = bfs_batch(S, adm);
      } else if (kind == 0) {
        switch (S->kw) {
          case 1: st = bfs_round<1>(S, adm); break;
          case 2: st = bfs_round<2>(S, adm); break;
          case 4: st = bfs_round<4>(S, adm); break;
          case 8: st = bfs_round<8>(S, adm); break;
          case 16: st = bfs_round<16>(S, adm); break;
          default: st = bfs_round<32>(S, adm); break;
        }
      } else {
        st = ppr_round(S, adm);
      }
    }
    const double t1 = now_ms();
    if (st == GBO_OK) st = retire(S, kind);
    if (st == GBO_OK && kind == 0) st = retire_batch(S);
    const double t2 = now_ms();
    if (st != GBO_OK) {
      failw(st);
      return;
    }
    {
      std::lock_guard<std::mutex> lk(S->mu);
      S->phase_ms[kind] += t1 - t0;
      S->phase_ms[2] += t2 - t1;
    }
    S->rounds++;
  }
}

void destroy_server(gbo_server* S) {
  if (!S) return;
  {
    std::lock_guard<std::mutex> lk(S->mu);
    S->stop = true;
  }
  S->cv_work.notify_all();
  for (int e = 0; e < 2; ++e) {
    if (S->worker[e].joinable()) S->worker[e].join();
    if (S->s[e]) cudaStreamSynchronize(S->s[e]);
  }
  for (void* m : S->msb)
    if (m) ms_batch_destroy(m);
  cudaFree(S->F);
  cudaFree(S->V);
  cudaFree(S->fbits);
  cudaFree(S->vfull);
  cudaFree(S->split_acc);
  cudaFree(S->slot_split);
  cudaFree(S->levels);
  cudaFree(S->ctl);
  cudaFree(S->slot_any);
  cudaFree(S->long_acc);
  cudaFreeHost(S->h_slot_any);
  cudaFree(S->d_active);
  cudaFree(S->d_adm_src);
  cudaFree(S->d_adm_slot);
  cudaFree(S->d_bufidx);
  cudaFree(S->blevels);
  cudaFree(S->X);
  cudaFree(S->P);
  cudaFree(S->err);
  cudaFreeHost(S->h_err);
  cudaFree(S->pscratch);
  cudaFree(S->d_pslots);
  cudaFree(S->d_pverts);
  cudaFree(S->d_poff);
  cudaFree(S->d_pwts);
  for (int p = 0; p < 2; ++p) {
    cudaFree(S->dpool[p]);
    for (cudaEvent_t e : S->pool_ev[p]) cudaEventDestroy(e);
  }
  for (int e = 0; e < 2; ++e) {
    if (S->s[e]) cudaStreamDestroy(S->s[e]);
    if (S->sync_ev[e]) cudaEventDestroy(S->sync_ev[e]);
  }
  delete S;
}

}  // namespace
}  // namespace gbo

using namespace gbo;

extern "C" int gbo_server_create(const gbo_graph* gc, int bfs_slots, int ppr_slots, float alpha,
                                 float tol, int ppr_max_iter, gbo_server** out) {
  clear_error();
  if (!gc || !out) return fail(GBO_ERR_INVALID, "NULL argument");
  *out = nullptr;
  gbo_graph* g = const_cast<gbo_graph*>(gc);
  if (g->b != 32 || g->layout != GBO_LAYOUT_ROW || g->nrows != g->ncols)
    return fail(GBO_ERR_UNSUPPORTED, "the server needs a square ROW-layout graph with 32x32 tiles");
  if (bfs_slots < 0 || bfs_slots > 1024 || (ppr_slots != 0 && ppr_slots != kPprSlots))
    return fail(GBO_ERR_INVALID, "bfs_slots in [0,1024]; ppr_slots 0 or 32");
  if (bfs_slots == 0 && ppr_slots == 0) return fail(GBO_ERR_INVALID, "no slots");
  if (ppr_slots && !g->invdeg) return fail(GBO_ERR_INVALID, "PPR needs out-degrees");
  gbo_server* S = new gbo_server();
  cudaGetDevice(&S->dev);
  S->g = g;
  S->n = g->nrows;
  S->nbr = g->nbr;
  S->alpha = alpha;
  S->tol = tol;
  S->ppr_max_iter = ppr_max_iter > 0 ? ppr_max_iter : 1000;
  int kw = 1;
  while (kw * 32 < bfs_slots) kw <<= 1;
  S->kb = bfs_slots > 0 ? kw * 32 : 0;  // slots rounded up to whole words
  S->kw = kw;
  auto cu = [&](cudaError_t e, const char* w) {
    if (e != cudaSuccess) throw fail_cuda(e, w);
  };
  try {
    for (int e = 0; e < 2; ++e) {
      cu(cudaStreamCreateWithFlags(&S->s[e], cudaStreamNonBlocking), "stream");
      cu(cudaEventCreateWithFlags(&S->sync_ev[e], cudaEventBlockingSync | cudaEventDisableTiming), "event");
    }
    const size_t n = (size_t)S->n;
    if (S->kb) {
      cu(cudaMalloc(&S->F, sizeof(uint32_t) * 2 * n * kw + 16), "F");
      cu(cudaMalloc(&S->V, sizeof(uint32_t) * n * kw + 16), "V");
      cu(cudaMalloc(&S->fbits, sizeof(uint32_t) * 2 * (size_t)(g->nbr + 1)), "fbits");
      cu(cudaMalloc(&S->vfull, sizeof(uint32_t) * (size_t)(g->nbr + 1)), "vfull");
      {
        const int st = ms::split_state(g, kw, &S->split_acc, &S->slot_split, S->s[0]);
        if (st != GBO_OK) throw st;
      }
      cu(cudaMalloc(&S->levels, sizeof(int) * n * S->kb + 16), "levels");
      cu(cudaMalloc(&S->ctl, 64), "ctl");
      cu(cudaMalloc(&S->slot_any, sizeof(uint32_t) * kw), "slot_any");
      cu(cudaHostAlloc(&S->h_slot_any, sizeof(uint32_t) * kw, cudaHostAllocDefault), "h_slot_any");
      cu(cudaMalloc(&S->d_adm_src, sizeof(int) * S->kb), "adm");
      cu(cudaMalloc(&S->d_adm_slot, sizeof(int) * S->kb), "adm");
      cu(cudaMalloc(&S->d_bufidx, sizeof(int) * S->kb), "bufidx");
      {
        const void* lv = nullptr;
        const int st = live_rows(g, S->s[0], &lv);
        if (st != GBO_OK) throw st;
        S->live = static_cast<const uint32_t*>(lv);
      }
      {  // rounds of up to 64 slots walk the row-word slices
        const int st = build_rws(g, S->s[0]);
        if (st != GBO_OK) throw st;
        const size_t lw = (size_t)(g->rws_nlong > 0 ? g->rws_nlong : 1) * (size_t)std::min(kw, 2);
        cu(cudaMalloc(&S->long_acc, sizeof(uint32_t) * lw), "long_acc");
        cu(cudaMemsetAsync(S->long_acc, 0, sizeof(uint32_t) * lw, S->s[0]), "long_acc");
      }
      ms::Args a = bfs_args(S);
      unsigned gv = blocks_for((long long)n * S->kb, 256);
      if (gv > (unsigned)num_sms() * 16u) gv = (unsigned)num_sms() * 16u;
      cu(cudaMalloc(&S->d_active, sizeof(uint32_t) * kw), "active");
      cu(cudaMemsetAsync(S->d_active, 0, sizeof(uint32_t) * kw, S->s[0]), "active");
      S->h_active.assign((size_t)kw, 0u);
      a.active = S->d_active;
      ms::k_init<<<gv, 256, 0, S->s[0]>>>(a, kw, 0x7fffffff);
      cu(cudaGetLastError(), "init");
    }
    S->bslot_ticket.assign((size_t)S->kb, 0);
    S->bslot_start.assign((size_t)S->kb, 0);
    S->bslot_finished.assign((size_t)S->kb, 0);
    S->bslot_batch.assign((size_t)S->kb, 0);
    if (ppr_slots) {
      cu(cudaMalloc(&S->X, sizeof(float) * 2 * n * kPprSlots), "X");
      cu(cudaMemsetAsync(S->X, 0, sizeof(float) * 2 * n * kPprSlots, S->s[1]), "X");
      cu(cudaMalloc(&S->P, sizeof(float) * n * kPprSlots), "P");
      cu(cudaMemsetAsync(S->P, 0, sizeof(float) * n * kPprSlots, S->s[1]), "P");
      cu(cudaMalloc(&S->err, sizeof(double) * kPprSlots), "err");
      cu(cudaHostAlloc(&S->h_err, sizeof(double) * kPprSlots, cudaHostAllocDefault), "h_err");
      cu(cudaMalloc(&S->pscratch, sizeof(double) * (size_t)(g->nslots > 0 ? g->nslots : 1) * 32 * kPprSlots), "pscratch");
      cu(cudaMalloc(&S->d_pslots, sizeof(int) * kPprSlots), "pslots");
      cu(cudaMalloc(&S->d_pverts, sizeof(int) * 64 * kPprSlots), "pverts");
      cu(cudaMalloc(&S->d_pwts, sizeof(float) * 64 * kPprSlots), "pwts");
      cu(cudaMalloc(&S->d_poff, sizeof(int) * (kPprSlots + 1)), "poff");
    }
    S->pslot_ticket.assign(ppr_slots ? (size_t)kPprSlots : 0, 0);
    S->pslot_iters.assign((size_t)kPprSlots, 0);
    S->pslot_finished.assign((size_t)kPprSlots, 0);
    // device result pools: every slot can hold a finished result plus two
    // rounds of retirements waiting for their clients
    // (BFS: a whole batch's results can wait for their clients while the
    // next batch runs)
    const int nbuf[2] = {S->kb > 0 ? 2 * S->kb + 2 * kRetire : 0, (ppr_slots ? kPprSlots : 0) + 2 * kRetire};
    S->dbytes[0] = (n + 255) / 256 * 256;
    S->dbytes[1] = (sizeof(int) * n + 255) / 256 * 256;
    for (int p = 0; p < 2; ++p) {
      if (nbuf[p] == 0) continue;
      cu(cudaMalloc(&S->dpool[p], S->dbytes[p] * (size_t)nbuf[p]), "result pool");
      for (int b = 0; b < nbuf[p]; ++b) {
        cudaEvent_t e = nullptr;
        cu(cudaEventCreateWithFlags(&e, cudaEventBlockingSync | cudaEventDisableTiming), "event");
        S->pool_ev[p].push_back(e);
        S->pool_free[p].push_back(nbuf[p] - 1 - b);
      }
    }
    cu(cudaStreamSynchronize(S->s[0]), "sync");
    cu(cudaStreamSynchronize(S->s[1]), "sync");
  } catch (int st) {
    destroy_server(S);
    return st;
  }
  if (S->kb > 0) S->worker[0] = std::thread(worker_main, S, 0);
  if (ppr_slots) S->worker[1] = std::thread(worker_main, S, 1);
  *out = S;
  return GBO_OK;
}

static int submit(gbo_server* S, Query&& q, int64_t* ticket) {
  std::lock_guard<std::mutex> lk(S->mu);
  if (S->worker_status != GBO_OK) return fail(S->worker_status, S->worker_error);
  if (S->max_pending > 0 && (long long)S->pending[q.kind].size() >= S->max_pending)
    return fail(GBO_ERR_FULL, "admission queue full (" + std::to_string(S->max_pending) + " pending queries)");
  q.ticket = S->next_ticket++;
  q.t_submit = now_ms();
  S->submit_time[q.ticket] = q.t_submit;
  *ticket = q.ticket;
  const int kind = q.kind;
  S->pending[kind].push_back(std::move(q));
  S->cv_work.notify_all();
  return GBO_OK;
}

extern "C" int gbo_server_set_queue_limit(gbo_server* S, long long max_pending) {
  clear_error();
  if (!S || max_pending < 0) return fail(GBO_ERR_INVALID, "bad argument");
  std::lock_guard<std::mutex> lk(S->mu);
  S->max_pending = max_pending;
  return GBO_OK;
}

extern "C" int gbo_server_set_admission(gbo_server* S, float min_free_fraction) {
  clear_error();
  if (!S || !(min_free_fraction >= 0.f && min_free_fraction <= 1.f)) return fail(GBO_ERR_INVALID, "bad argument");
  std::lock_guard<std::mutex> lk(S->mu);
  S->bfs_admit_free = min_free_fraction;
  S->cv_work.notify_all();
  return GBO_OK;
}

extern "C" int gbo_server_submit_bfs(gbo_server* S, int src, int64_t* ticket) {
  clear_error();
  if (!S || !ticket) return fail(GBO_ERR_INVALID, "NULL argument");
  if (S->kb == 0) return fail(GBO_ERR_INVALID, "server has no BFS slots");
  if (src < 0 || src >= S->n) return fail(GBO_ERR_INVALID, "source out of range");
  Query q;
  q.kind = 0;
  q.src = src;
  return submit(S, std::move(q), ticket);
}

extern "C" int gbo_server_submit_ppr(gbo_server* S, const int* verts, const float* weights, int count,
                                     int64_t* ticket) {
  clear_error();
  if (!S || !ticket || !verts || !weights) return fail(GBO_ERR_INVALID, "NULL argument");
  if (S->pslot_ticket.empty()) return fail(GBO_ERR_INVALID, "server has no PPR slots");
  if (count < 1 || count > 64) return fail(GBO_ERR_INVALID, "a PPR set has 1..64 vertices");
  for (int k = 0; k < count; ++k)
    if (verts[k] < 0 || verts[k] >= S->n) return fail(GBO_ERR_INVALID, "vertex out of range");
  Query q;
  q.kind = 1;
  q.src = -1;
  q.verts.assign(verts, verts + count);
  q.wts.assign(weights, weights + count);
  return submit(S, std::move(q), ticket);
}

// Byte levels to int32, 255 (unreachable) to -1 (host_io.cpp).
namespace gbo {
void host_widen_levels(const unsigned char* b8, int* o, long long n);
}
static void widen_levels(const unsigned char* b8, int* o, int n) { gbo::host_widen_levels(b8, o, n); }

// Byte levels to int32 on the device (device delivery), 16 per thread.
__global__ void k_widen_levels(const unsigned char* __restrict__ b8, int* __restrict__ o, int n) {
  const long long i = ((long long)blockIdx.x * blockDim.x + threadIdx.x) * 16;
  if (i >= n) return;
  const bool vec = i + 16 <= n && ((reinterpret_cast<uintptr_t>(o) | reinterpret_cast<uintptr_t>(b8)) & 15) == 0;
  if (vec) {
    const uint4 v = *reinterpret_cast<const uint4*>(b8 + i);
    const unsigned w[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      int4 r;
      const unsigned a = w[q];
      r.x = (int)(a & 0xffu);
      r.y = (int)((a >> 8) & 0xffu);
      r.z = (int)((a >> 16) & 0xffu);
      r.w = (int)(a >> 24);
      r.x = r.x == 255 ? -1 : r.x;
      r.y = r.y == 255 ? -1 : r.y;
      r.z = r.z == 255 ? -1 : r.z;
      r.w = r.w == 255 ? -1 : r.w;
      reinterpret_cast<int4*>(o + i)[q] = r;
    }
  } else {
    for (long long k = i; k < i + 16 && k < n; ++k) o[k] = b8[k] == 255 ? -1 : (int)b8[k];
  }
}

// Per client thread: a pinned bounce buffer and a stream, so that result
// copies from many client threads run at full link speed side by side
// (copies into pageable memory would serialise on the driver's staging).
struct ClientCopy {
  void* pinned = nullptr;
  size_t bytes = 0;
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  ~ClientCopy() {
    if (pinned) cudaFreeHost(pinned);
    if (st) cudaStreamDestroy(st);
    if (done) cudaEventDestroy(done);
  }
  // Copy `bytes` from device memory into the bounce buffer; returns it.
  const void* fetch(const void* src, size_t n, cudaError_t* err) {
    if (!st) *err = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (*err == cudaSuccess && !done) *err = cudaEventCreateWithFlags(&done, cudaEventBlockingSync | cudaEventDisableTiming);
    if (*err == cudaSuccess && bytes < n) {
      if (pinned) cudaFreeHost(pinned);
      pinned = nullptr;
      bytes = 0;
      *err = cudaHostAlloc(&pinned, n, cudaHostAllocDefault);
      if (*err == cudaSuccess) bytes = n;
    }
    if (*err == cudaSuccess) *err = cudaMemcpyAsync(pinned, src, n, cudaMemcpyDeviceToHost, st);
    if (*err == cudaSuccess) *err = wait_stream(st, done);
    return pinned;
  }
  // Copy `n` bytes from device memory straight into pinned host memory.
  cudaError_t copy_into(void* dst, const void* src, size_t n) {
    cudaError_t e = cudaSuccess;
    if (!st) e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
    if (e == cudaSuccess && !done) e = cudaEventCreateWithFlags(&done, cudaEventBlockingSync | cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaMemcpyAsync(dst, src, n, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = wait_stream(st, done);
    return e;
  }
};

// Per client thread for device delivery: a stream (when the caller gives
// none) and a blocking-sync event that says when the result buffer has been
// read.
struct ClientDeviceCopy {
  cudaStream_t st = nullptr;
  cudaEvent_t done = nullptr;
  std::vector<int> widened;  // results already moved to host memory
  ~ClientDeviceCopy() {
    if (st) cudaStreamDestroy(st);
    if (done) cudaEventDestroy(done);
  }
};

// Copy result r into the caller's device buffer d_out on stream ds (0: the
// thread's own stream), widening byte levels to int32, and wait until the
// copy has read the result buffer.
static cudaError_t deliver_device(gbo_server* S, const Result& r, void* d_out, cudaStream_t ds) {
  thread_local ClientDeviceCopy cc;
  cudaError_t e = cudaSuccess;
  if (!ds) {
    // the thread's own stream at the highest priority, so that the copy's
    // blocks are scheduled ahead of the traversal kernels already queued
    if (!cc.st) {
      int least = 0, greatest = 0;
      e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
      if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&cc.st, cudaStreamNonBlocking, greatest);
    }
    ds = cc.st;
  }
  if (e == cudaSuccess && !cc.done)
    e = cudaEventCreateWithFlags(&cc.done, cudaEventBlockingSync | cudaEventDisableTiming);
  if (e != cudaSuccess) return e;
  const int n = S->n;
  if (r.buf < 0) {  // already in host memory
    const void* src = r.host.data();
    if (r.u8) {
      cc.widened.resize((size_t)n);
      widen_levels(r.host.data(), cc.widened.data(), n);
      src = cc.widened.data();
    }
    e = cudaMemcpyAsync(d_out, src, sizeof(int) * (size_t)n, cudaMemcpyHostToDevice, ds);
  } else {
    const char* src = S->dpool[r.pool] + (size_t)r.buf * S->dbytes[r.pool];
    e = cudaStreamWaitEvent(ds, r.ev, 0);
    if (e == cudaSuccess && r.u8) {
      const long long th = ((long long)n + 15) / 16;
      if (th > 0)
        k_widen_levels<<<(unsigned)((th + 255) / 256), 256, 0, ds>>>(
            reinterpret_cast<const unsigned char*>(src), static_cast<int*>(d_out), n);
      e = cudaGetLastError();
    } else if (e == cudaSuccess) {
      e = cudaMemcpyAsync(d_out, src, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, ds);
    }
  }
  if (e == cudaSuccess) e = wait_stream(ds, cc.done);
  return e;
}

// Hand a finished result to the caller: wait for its retirement kernel,
// copy it from the device buffer (widening byte levels to int32) outside the
// lock -- to host memory (h_out) or, with `device`, to the caller's device
// buffer d_out -- then give the buffer back to the pool.
// True when p is page-locked host memory the device can copy into directly.
static bool is_pinned(const void* p) {
  cudaPointerAttributes at;
  if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

// The result of `ticket` (present, not moving) into h_out (byte levels when
// bytes_out), then its buffer back to the pool.
static int take_result(gbo_server* S, std::unique_lock<std::mutex>& lk, int64_t ticket, void* h_out,
                       double* latency_ms, int* iterations, bool device = false,
                       cudaStream_t ds = nullptr, bool bytes_out = false) {
  auto it = S->results.find(ticket);
  const Result r = std::move(it->second);
  S->results.erase(it);
  S->submit_time.erase(ticket);
  lk.unlock();
  const double t0 = now_ms();
  double t1 = t0, t2 = t0;
  cudaError_t e = cudaSuccess;
  if (device) {
    if (h_out) e = deliver_device(S, r, h_out, ds);
    t2 = t1 = now_ms();
  } else if (bytes_out) {  // byte levels as stored
    if (r.buf < 0) {
      if (h_out) memcpy(h_out, r.host.data(), (size_t)S->n);
    } else {
      const char* src = S->dpool[r.pool] + (size_t)r.buf * S->dbytes[r.pool];
      e = cudaEventSynchronize(r.ev);
      t1 = now_ms();
      if (e == cudaSuccess && h_out) {
        thread_local ClientCopy cc;
        if (is_pinned(h_out)) {
          e = cc.copy_into(h_out, src, (size_t)S->n);
        } else {
          const void* h = cc.fetch(src, (size_t)S->n, &e);
          if (e == cudaSuccess) memcpy(h_out, h, (size_t)S->n);
        }
      }
      t2 = now_ms();
    }
  } else if (r.buf < 0) {  // already in host memory
    if (h_out && r.u8) {
      int* o = static_cast<int*>(h_out);
      widen_levels(r.host.data(), o, S->n);
    } else if (h_out) {
      memcpy(h_out, r.host.data(), sizeof(int) * (size_t)S->n);
    }
  } else {
    const char* src = S->dpool[r.pool] + (size_t)r.buf * S->dbytes[r.pool];
    e = cudaEventSynchronize(r.ev);
    t1 = now_ms();
    if (e == cudaSuccess && h_out) {
      thread_local ClientCopy cc;
      const size_t nb = (r.u8 ? 1 : sizeof(int)) * (size_t)S->n;
      const void* h = cc.fetch(src, nb, &e);
      t2 = now_ms();
      if (e == cudaSuccess && r.u8) {
        const unsigned char* b8 = static_cast<const unsigned char*>(h);
        int* o = static_cast<int*>(h_out);
        widen_levels(b8, o, S->n);
      } else if (e == cudaSuccess) {
        memcpy(h_out, h, nb);
      }
    }
  }
  const double t3 = now_ms();
  if (latency_ms) *latency_ms = t3 - r.t_submit;
  if (iterations) *iterations = r.iters;
  lk.lock();
  if (r.buf >= 0) S->pool_free[r.pool].push_back(r.buf);
  S->phase_ms[3] += t3 - t0;
  if (r.buf >= 0) {
    S->copy_parts[0] += t1 - t0;
    S->copy_parts[1] += t2 - t1;
    S->copy_parts[2] += t3 - t2;
  }
  S->cv_work.notify_all();
  if (e != cudaSuccess) return fail_cuda(e, "server result copy");
  return GBO_OK;
}

extern "C" int gbo_server_poll(gbo_server* S, int64_t ticket, void* h_out, double* latency_ms,
                               int* iterations) {
  clear_error();
  if (!S) return fail(GBO_ERR_INVALID, "NULL server");
  std::unique_lock<std::mutex> lk(S->mu);
  if (S->worker_status != GBO_OK) return fail(S->worker_status, S->worker_error);
  auto it = S->results.find(ticket);
  if (it == S->results.end() || it->second.moving) return GBO_ERR_NOTREADY;
  if (it->second.buf >= 0 && cudaEventQuery(it->second.ev) == cudaErrorNotReady) {
    (void)cudaGetLastError();
    return GBO_ERR_NOTREADY;
  }
  return take_result(S, lk, ticket, h_out, latency_ms, iterations);
}

extern "C" int gbo_server_wait(gbo_server* S, int64_t ticket, void* h_out, double* latency_ms,
                               int* iterations, double timeout_s) {
  clear_error();
  if (!S) return fail(GBO_ERR_INVALID, "NULL server");
  std::unique_lock<std::mutex> lk(S->mu);
  const bool ok = S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
    if (S->worker_status != GBO_OK) return true;
    auto it = S->results.find(ticket);
    return it != S->results.end() && !it->second.moving;
  });
  if (S->worker_status != GBO_OK) return fail(S->worker_status, S->worker_error);
  if (!ok) return fail(GBO_ERR_TIMEOUT, "query not finished within the timeout");
  return take_result(S, lk, ticket, h_out, latency_ms, iterations);
}

extern "C" int gbo_server_wait_u8(gbo_server* S, int64_t ticket, uint8_t* h_out, double* latency_ms,
                                  int* iterations, double timeout_s) {
  clear_error();
  if (!S) return fail(GBO_ERR_INVALID, "NULL server");
  std::unique_lock<std::mutex> lk(S->mu);
  const bool ok = S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
    if (S->worker_status != GBO_OK) return true;
    auto it = S->results.find(ticket);
    return it != S->results.end() && !it->second.moving;
  });
  if (S->worker_status != GBO_OK) return fail(S->worker_status, S->worker_error);
  if (!ok) return fail(GBO_ERR_TIMEOUT, "query not finished within the timeout");
  const Result& r = S->results.find(ticket)->second;
  if (r.kind != 0) return fail(GBO_ERR_INVALID, "gbo_server_wait_u8 takes BFS tickets");
  if (!r.u8) return fail(GBO_ERR_OVERFLOW, "levels past 254: collect this result with gbo_server_wait");
  return take_result(S, lk, ticket, h_out, latency_ms, iterations, false, nullptr, true);
}

extern "C" int gbo_server_wait_device(gbo_server* S, int64_t ticket, void* d_out,
                                      double* latency_ms, int* iterations, double timeout_s,
                                      gbo_stream_t stream) {
  clear_error();
  if (!S) return fail(GBO_ERR_INVALID, "NULL server");
  std::unique_lock<std::mutex> lk(S->mu);
  const bool ok = S->cv_done.wait_for(lk, std::chrono::duration<double>(timeout_s), [&] {
    if (S->worker_status != GBO_OK) return true;
    auto it = S->results.find(ticket);
    return it != S->results.end() && !it->second.moving;
  });
  if (S->worker_status != GBO_OK) return fail(S->worker_status, S->worker_error);
  if (!ok) return fail(GBO_ERR_TIMEOUT, "query not finished within the timeout");
  return take_result(S, lk, ticket, d_out, latency_ms, iterations, true, as_stream(stream));
}

extern "C" int gbo_server_get_stats(gbo_server* S, gbo_server_stats* st) {
  clear_error();
  if (!S || !st) return fail(GBO_ERR_INVALID, "NULL argument");
  std::lock_guard<std::mutex> lk(S->mu);
  st->rounds = S->rounds;
  st->bfs_completed = S->bfs_done;
  st->ppr_completed = S->ppr_done;
  st->kernel_launches = S->launches;
  st->pending = (long long)(S->pending[0].size() + S->pending[1].size());
  long long a = 0;
  for (long long t : S->bslot_ticket) a += t > 0;
  for (long long t : S->pslot_ticket) a += t > 0;
  st->in_flight = a;
  st->bfs_round_ms = S->phase_ms[0];
  st->ppr_round_ms = S->phase_ms[1];
  st->retire_ms = S->phase_ms[2];
  st->copy_ms = S->phase_ms[3];
  st->copy_wait_ms = S->copy_parts[0];
  st->copy_d2h_ms = S->copy_parts[1];
  st->copy_widen_ms = S->copy_parts[2];
  return GBO_OK;
}

extern "C" int gbo_server_destroy(gbo_server* S) {
  clear_error();
  destroy_server(S);
  return GBO_OK;
}
