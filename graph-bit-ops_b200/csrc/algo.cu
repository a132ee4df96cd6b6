// Graph algorithms on the B2SR primitives with all state on the device.
//
// The reference loops (algorithm/bfs.cu:508-564, sssp.cu:420-470,
// pr.cu:449-513, cc.cu:223-287) launch 5-9 kernels per iteration and copy a
// convergence scalar to the host every iteration.  Here each iteration is one
// fused step kernel plus a small kernel that finishes split block rows; the
// last block of that kernel (atomic ticket) decides termination on the
// device.  One iteration is captured once as the body of a conditional WHILE
// node of a CUDA graph, and the deciding block clears the node's condition
// when the loop stops: a whole traversal or solve is one graph launch with
// no host round trip and no idle iterations.
#include <string.h>

#include <algorithm>
#include <vector>

#include "scan.cuh"

namespace gbo {

// Loop control word in device memory.
struct Ctrl {
  int iter;       // iterations completed
  int done;       // 1 once the loop has terminated
  unsigned ticket;
  int max_iter;
  unsigned long long count;  // vertices changed in the current iteration
  double err;                // error accumulator of the current iteration
  double last_err;           // error of the last finished iteration
  float tol;
  float alpha;
  float add;      // constant added to each PageRank entry
  float add_scale;  // PPR: add_scale * v[i] added as well
  int norm;       // 1 = L1, 2 = L2 error
  int n;
  double ref;     // PPR adjoint: ||w||_1, the scale of its stopping test
  unsigned long long work;  // BFS pull step: warp work units handed out this iteration
  int row_scale;  // PR-type step: 0 = columns scaled (PageRank), 1 = rows (adjoint on P = P^T)
  int mode;       // BFS: 0 = pull (bottom-up) step, 1 = push (top-down) step
  int push_thr;   // BFS: push while the frontier has fewer vertices (0 = never)
  // the running loop's CUDA graph condition (cleared when the loop stops)
  // and its iteration end times (globaltimer ns; [0] = loop start)
  unsigned long long cond;
  unsigned long long* stamps;
  // cooperative BFS: grid barrier (arrival word, give-up flag) and the
  // new-vertex counts of three consecutive levels
  unsigned bar_arrive;
  unsigned bar_err;
  unsigned long long push_acc[3];  // push list: rows << 40 | tail entries
  // new-vertex counts of three consecutive levels, each spread over eight
  // counters on their own 128-byte lines (block b adds into counter b % 8)
  unsigned long long lvl_part[3][8][16];
};

// Iteration end times kept per loop run (more iterations run untimed).
constexpr int kStampCap = 4096;

}  // namespace gbo

// Per-graph algorithm state (global scope: gbo_graph::algo is ::AlgoState*).
struct AlgoState {
  cudaStream_t cap = nullptr;  // capture stream
  gbo::Ctrl* ctrl = nullptr;
  gbo::Ctrl* h_ctrl = nullptr;  // pinned mirror
  // BFS / SSSP
  void* front = nullptr;   // 2 * nbr words (8 bytes each max)
  void* visited = nullptr; // nbr words
  void* live = nullptr;    // nbr words: bit set where the row of P has an entry
  int* level = nullptr;    // n
  uint32_t* dist = nullptr;
  // PR / PPR / CC vectors
  float* pr = nullptr;     // 2 * n
  float* prs = nullptr;    // 2 * n: the iterate scaled by D^-1 (PageRank gathers it)
  const float* ppr_v = nullptr;
  int* f = nullptr;
  int* gf = nullptr;
  int* mngf = nullptr;
  int* seeds = nullptr;  // multi-seed BFS sources
  int nseeds_cap = 0;
  double* acc64 = nullptr;  // PPR adjoint scatter accumulator
  double* pr_part = nullptr;  // row-word slices: one partial sum per long-row chunk
  long long* push_list = nullptr;  // cooperative BFS: (start, tail offset) per listed long row
  void* scratch = nullptr;  // split partials (nslots * b * 8 bytes)
  cudaGraphExec_t exec[8] = {};
  const void* exec_key[8] = {};
  unsigned long long cond[8] = {};       // each loop graph's condition handle
  unsigned long long* stamps = nullptr;  // kStampCap + 1 iteration end times
  int launches_per_iter = 0;             // kernels of one loop iteration
  int fixed_launches = 2;                // kernels of a run outside its iterations
  bool coop_run = false;                 // the last run was a cooperative BFS
  bool stats_pending = false;            // step times not yet read back

  // statistics of the last algorithm run
  std::vector<float> step_ms;
  int replays = 0;
  long long launches = 0;
  int launches_per_replay = 0;
};

namespace gbo {

namespace {

constexpr int kTPB = 256;
// Iterations per unit of the injected loop cap (gbo_debug_inject).
constexpr int kStepsPerGraph = 8;
// GBO_BFS_LOOP_AUTO runs b = 32 ROW BFS as one cooperative launch of at
// most this many blocks per SM.
constexpr bool kCoopBfsDefault = true;
constexpr int kCoopBlocksPerSM = 4;

enum AlgoId { A_BFS = 0, A_SSSP = 1, A_PR = 2, A_CC = 3, A_PPR_F = 4, A_PPR_B = 5, A_PPR_BG = 6 };

template <int B>
__device__ __forceinline__ typename Word<B>::T full_word() {
  using WT = typename Word<B>::T;
  return (WT)((WT)~(WT)0 >> (sizeof(WT) * 8 - B));
}

template <int B>
__device__ __forceinline__ bool bit_of(typename Word<B>::T w, int r) {
  return (w >> (B - 1 - r)) & 1;
}

template <int B>
__device__ __forceinline__ typename Word<B>::T gather_bits(bool p0, bool p1, unsigned lane) {
  using L = Lay<B>;
  if (L::RPL == 2) {
    unsigned lo = __ballot_sync(0xffffffffu, p0);
    unsigned hi = __ballot_sync(0xffffffffu, p1);
    return (typename Word<B>::T)__brevll(((unsigned long long)hi << 32) | lo);
  } else {
    unsigned bal = __ballot_sync(0xffffffffu, p0);
    unsigned g = lane / L::W;
    unsigned seg = (bal >> (g * L::W)) & seg_mask<B>();
    return (typename Word<B>::T)(__brev(seg) >> (32 - (B < 32 ? B : 32)));
  }
}

template <int B, typename F>
__device__ __forceinline__ void for_each_col(typename Word<B>::T w, F&& f) {
  unsigned long long a = (unsigned long long)w << (64 - B);
  while (a) {
    int j = __clzll(a);
    f(j);
    a &= ~(0x8000000000000000ull >> j);
  }
}

__device__ __forceinline__ long long item_index(unsigned lane, int W, int G) {
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  return warp * G + lane / W;
}

// The iteration kernels visit work items in a warp-uniform grid-stride loop
// and run on a persistent grid (a few blocks per SM): an iteration with
// nothing to do (the loop has finished, or the other BFS direction is
// active) then costs microseconds instead of a launch over every item.
__device__ __forceinline__ long long warp_global() {
  return ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
}
__device__ __forceinline__ long long warps_total() { return ((long long)gridDim.x * blockDim.x) >> 5; }

// Block-wide sum of `v` added to *dst once per block.
__device__ __forceinline__ void block_add_u64(unsigned long long v, unsigned long long* dst) {
  __shared__ unsigned long long sh;
  if (threadIdx.x == 0) sh = 0;
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v) atomicAdd(&sh, v);
  __syncthreads();
  if (threadIdx.x == 0 && sh) atomicAdd(dst, sh);
}

__device__ __forceinline__ void block_add_f64(double v, double* dst) {
  __shared__ double sh;
  if (threadIdx.x == 0) sh = 0;
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0 && v != 0.0) atomicAdd(&sh, v);
  __syncthreads();
  if (threadIdx.x == 0 && sh != 0.0) atomicAdd(dst, sh);
}

// Called by every block of an iteration's last kernel after its work: the
// last block to arrive closes the iteration.  No waiting: the ticket only
// counts arrivals.
template <typename Decide>
__device__ __forceinline__ void close_iteration(Ctrl* ctrl, Decide decide) {
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    unsigned t = atomicAdd(&ctrl->ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    volatile Ctrl* c = ctrl;
    const int it = c->iter + 1;
    const bool stop = decide(c, it);
    c->iter = it;
    c->last_err = c->err;
    c->err = 0.0;
    c->count = 0ull;
    c->work = 0ull;
    c->ticket = 0u;
    if (c->stamps && it <= kStampCap) {
      unsigned long long t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      c->stamps[it] = t;
    }
    if (stop) {
      c->done = 1;
      cudaGraphSetConditional((cudaGraphConditionalHandle)c->cond, 0u);
    }
    __threadfence();
  }
}

// Before a loop graph runs: its condition handle and the start stamp; an
// injected cap (gbo_debug_inject) cuts the loop's iteration limit.
__global__ void k_loop_begin(Ctrl* ctrl, unsigned long long cond, unsigned long long* stamps, int cap_iters) {
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  ctrl->cond = cond;
  ctrl->stamps = stamps;
  if (cap_iters > 0 && cap_iters < ctrl->max_iter) ctrl->max_iter = cap_iters;
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  stamps[0] = t;
}

// ============================================================== BFS
// Frontier words rotate through three buffers of front_stride(nbr) words:
// level L reads buffer L % 3 and writes buffer (L + 1) % 3, and its active
// step kernel zeroes buffer (L + 2) % 3 -- read last at level L - 1 -- so
// that a push step at level L + 1 finds its output empty without a clearing
// launch.  The stride keeps every buffer on a 4-byte boundary, so the 32-bit
// atomics that OR narrow words never reach into a neighbouring buffer.
__host__ __device__ __forceinline__ size_t front_stride(int nbr) { return ((size_t)nbr + 4) & ~(size_t)3; }
template <typename WT>
__device__ __forceinline__ WT* front_buf(WT* front, int nbr, int lvl) {
  return front + (size_t)(lvl % 3) * front_stride(nbr);
}

template <int B>
__global__ void __launch_bounds__(kTPB) k_bfs_step(GView v, typename Word<B>::T* __restrict__ front,
                                                   typename Word<B>::T* __restrict__ visited,
                                                   int* __restrict__ level, Ctrl* __restrict__ ctrl,
                                                   typename Word<B>::T* __restrict__ scratch) {
  using WT = typename Word<B>::T;
  using L = Lay<B>;
  if (((volatile Ctrl*)ctrl)->done || ((volatile Ctrl*)ctrl)->mode) return;
  const int lvl = ((volatile Ctrl*)ctrl)->iter;
  const WT* __restrict__ x = front_buf(front, v.nbr, lvl);
  WT* __restrict__ out = front_buf(front, v.nbr, lvl + 1);
  WT* __restrict__ z = front_buf(front, v.nbr, lvl + 2);
  const unsigned lane = threadIdx.x & 31;
  const int r = lane % L::W;
  const WT full = full_word<B>();
  unsigned long long cnt = 0;
  // warps take work units (L::G items each) kGrab at a time from a counter:
  // rows that stop early and rows scanned to the end even out dynamically
  constexpr long long kGrab = 4;
  long long w = 0, wend = 0;
  for (;;) {
    if (w == wend) {
      unsigned long long g0 = 0;
      if (lane == 0) g0 = atomicAdd(&ctrl->work, (unsigned long long)kGrab);
      w = (long long)__shfl_sync(0xffffffffu, g0, 0);
      wend = w + kGrab;
    }
    if (w * L::G >= v.nitems) break;
    const long long item = w * L::G + lane / L::W;
    ++w;
    const bool active = item < v.nitems;
    gbo_item it = active ? v.items[item] : gbo_item{0, 0, 0, -2};
    const WT vis = active ? visited[it.row] : full;
    bool p0 = false, p1 = false;
    if (active && (vis & full) != full) {  // uniform inside the item's lane group
      const long long row0 = (long long)it.row * B + r;
      const bool need0 = !bit_of<B>(vis, r) && row0 < v.nrows;
      const bool need1 = L::RPL == 2 && !bit_of<B>(vis, r + 32) && row0 + 32 < v.nrows;
      pull_or_scan<B>(v, it.t0, it.t1, x, need0, need1, p0, p1, lane);
    }
    const WT word = gather_bits<B>(p0, p1, lane);
    if (active) {
      if (r == 0) z[it.row] = 0;
      if (it.slot >= 0) {
        if (r == 0) scratch[it.slot] = word;
      } else {
        const WT nw = (WT)(word & ~vis & full);
        const long long row0 = (long long)it.row * B + r;
        if (bit_of<B>(nw, r) && row0 < v.nrows) level[row0] = lvl + 1;
        if (L::RPL == 2 && bit_of<B>(nw, r + 32) && row0 + 32 < v.nrows) level[row0 + 32] = lvl + 1;
        if (r == 0) {
          out[it.row] = nw;
          if (nw) visited[it.row] = (WT)(vis | nw);
          cnt += popc_w(nw);
        }
      }
    }
  }
  block_add_u64(cnt, &ctrl->count);
}

// Pull step on the row-word slices of a b = 32 ROW graph.  A warp reads the
// visited words of its next 32 block rows (strided over the grid) in one
// round of loads and walks each open block row (a row still unvisited) with
// lane r on row r: entry k of every open row comes in one 256-byte load,
// the frontier word of its block column is gathered, four entries per
// round; a row leaves at its first entry that meets the
// frontier or when its entries run out (entries are in ascending block
// column, hubs of power-law graphs first), the block row when no row is
// left.  Rows still open after the head scan their tails: tails of up to
// kLongTail entries one lane per row with four entries in flight, longer
// ones by the whole warp 32 entries at a time.  Rows without entries start
// visited (k_live), so every open row has an entry.
constexpr int kLongTail = kRwsLongTail;

// The cooperative loop's level counts carry, above this bit, the number of
// new vertices with long tails (hubs).
constexpr int kLongShift = 40;
constexpr unsigned long long kLongMask = (1ull << kLongShift) - 1ull;

// Loads of the traversal state (frontier and visited words): through the
// read-only path when the state only changes between launches; as plain
// (weak, L1-cached) loads inside the cooperative BFS kernel, where other
// blocks rewrite it between levels -- the grid barrier's fences order those
// writes before the loads, which the read-only path does not promise.
template <bool COH>
__device__ __forceinline__ unsigned ld_state(const unsigned* p) {
  if constexpr (COH) return *p;
  else return __ldg(p);
}

// One pull level over the row-word slices (see k_bfs_pull_rws); returns the
// new vertices counted by this thread.
template <bool COH>
__device__ __forceinline__ unsigned long long pull_rws_level(const GView& v, unsigned* front, unsigned* visited,
                                                             int* level, int lvl) {
  const unsigned* x = front_buf(front, v.nbr, lvl);
  unsigned* out = front_buf(front, v.nbr, lvl + 1);
  unsigned* z = front_buf(front, v.nbr, lvl + 2);
  const unsigned lane = threadIdx.x & 31;
  const unsigned kFull = 0xffffffffu;
  const long long nwarps = warps_total();
  unsigned long long cnt = 0;
  // lane j reads the visited word of block row base + j * nwarps: one round
  // of loads finds the warp's open block rows among its next 32, and the
  // stride spreads neighbouring (similar) block rows over the warps
  for (long long base = warp_global(); base < v.nbr; base += 32 * nwarps) {
    const long long Rl = base + (long long)lane * nwarps;
    unsigned visl = kFull;
    if (Rl < v.nbr) {
      visl = visited[Rl];
      z[Rl] = 0u;
    }
    unsigned openb = __ballot_sync(kFull, visl != kFull);
    // with COH (the cooperative kernel, which has the registers) the first
    // four head entries of the next open block row are loaded while the
    // current one is walked
    uint2 pf[4];
    if (COH && openb) {
      const int j0 = __ffs(openb) - 1;
      const bool n0 = !((__shfl_sync(kFull, visl, j0) >> (31 - lane)) & 1u);
      const uint2* h0 = v.rws_head + (size_t)(base + (long long)j0 * nwarps) * (kRwsHead * 32) + lane;
#pragma unroll
      for (int q = 0; q < 4; ++q) pf[q] = n0 ? h0[(size_t)q * 32] : make_uint2(kRwsNone, 0u);
    }
    while (openb) {
      const int j = __ffs(openb) - 1;
      openb &= openb - 1;
      const long long R = base + (long long)j * nwarps;
      const unsigned vis = __shfl_sync(kFull, visl, j);
      bool need = !((vis >> (31 - lane)) & 1u);
      bool hit = false;
      const uint2* __restrict__ hp = v.rws_head + (size_t)R * (kRwsHead * 32) + lane;
      uint2 cur[4];
      if constexpr (COH) {
#pragma unroll
        for (int q = 0; q < 4; ++q) cur[q] = pf[q];
        if (openb) {
          const int jn = __ffs(openb) - 1;
          const bool nn = !((__shfl_sync(kFull, visl, jn) >> (31 - lane)) & 1u);
          const uint2* hn = v.rws_head + (size_t)(base + (long long)jn * nwarps) * (kRwsHead * 32) + lane;
#pragma unroll
          for (int q = 0; q < 4; ++q) pf[q] = nn ? hn[(size_t)q * 32] : make_uint2(kRwsNone, 0u);
        }
      }
      // four entries per round: most rows of a dense level are answered by
      // the first round, so its loads are issued together
#pragma unroll
      for (int k = 0; k < kRwsHead; k += 4) {
        if (!__any_sync(kFull, need)) break;
        uint2 e[4];
        if (COH && k == 0) {
#pragma unroll
          for (int q = 0; q < 4; ++q) e[q] = cur[q];
        } else {
#pragma unroll
          for (int q = 0; q < 4; ++q) e[q] = need ? hp[(size_t)(k + q) * 32] : make_uint2(kRwsNone, 0u);
        }
        unsigned a = 0u;
#pragma unroll
        for (int q = 0; q < 4; ++q) a |= e[q].x != kRwsNone ? (e[q].y & ld_state<COH>(x + e[q].x)) : 0u;
        hit = hit || (need && a != 0u);
        need = need && !hit && e[3].x != kRwsNone;
      }
      if (__any_sync(kFull, need)) {
        const long long row = R * 32 + lane;
        long long tb = 0, te = 0;
        if (need) {
          tb = v.rws_tail_ptr[row];
          te = v.rws_tail_ptr[row + 1];
        }
        need = need && te > tb;
        unsigned longm = __ballot_sync(kFull, need && te - tb > kLongTail);
        need = need && te - tb <= kLongTail;
        for (long long p = tb; __any_sync(kFull, need); p += 4) {
          if (need) {
            uint2 e[4];
#pragma unroll
            for (int q = 0; q < 4; ++q) e[q] = p + q < te ? v.rws_tail[p + q] : make_uint2(kRwsNone, 0u);
            unsigned a = 0u;
#pragma unroll
            for (int q = 0; q < 4; ++q) a |= e[q].x != kRwsNone ? (e[q].y & ld_state<COH>(x + e[q].x)) : 0u;
            hit = a != 0u;
            need = !hit && p + 4 < te;
          }
        }
        while (longm) {
          const int q = __ffs(longm) - 1;
          longm &= longm - 1;
          const long long qb = __shfl_sync(kFull, tb, q), qe = __shfl_sync(kFull, te, q);
          bool qhit = false;
          for (long long p = qb; p < qe && !qhit; p += 32) {
            bool h = false;
            if (p + lane < qe) {
              const uint2 e = v.rws_tail[p + lane];
              h = (e.y & ld_state<COH>(x + e.x)) != 0u;
            }
            qhit = __any_sync(kFull, h);
          }
          if ((int)lane == q && qhit) hit = true;
        }
      }
      const unsigned nw = __brev(__ballot_sync(kFull, hit)) & ~vis;
      if (nw) {
        if (lane == 0) {
          out[R] = nw;
          visited[R] = vis | nw;
          cnt += __popc(nw);
          // the cooperative loop also counts the new vertices with long
          // tails (a push level after this one skips its hub phase at none)
          if (COH) cnt += (unsigned long long)__popc(nw & v.rws_longbits[R]) << kLongShift;
        }
        if ((nw >> (31 - lane)) & 1u) level[R * 32 + lane] = lvl + 1;
      }
    }
  }
  return cnt;
}

__global__ void __launch_bounds__(kTPB, 6) k_bfs_pull_rws(GView v, unsigned* __restrict__ front,
                                                       unsigned* __restrict__ visited,
                                                       int* __restrict__ level, Ctrl* __restrict__ ctrl) {
  if (((volatile Ctrl*)ctrl)->done || ((volatile Ctrl*)ctrl)->mode) return;
  const int lvl = ((volatile Ctrl*)ctrl)->iter;
  const unsigned long long cnt = pull_rws_level<false>(v, front, visited, level, lvl);
  block_add_u64(cnt, &ctrl->count);
}

// OR `val` into word idx of a b-bit word array with a 32- or 64-bit atomic
// (words narrower than 32 bits are OR-ed inside their enclosing 32-bit word;
// the other bytes receive zero bits and do not change).
template <int B>
__device__ __forceinline__ void atomic_or_word(typename Word<B>::T* base, long long idx,
                                               typename Word<B>::T val) {
  if (B == 64) {
    atomicOr(reinterpret_cast<unsigned long long*>(base) + idx, (unsigned long long)val);
  } else if (B == 32) {
    atomicOr(reinterpret_cast<unsigned*>(base) + idx, (unsigned)val);
  } else {
    const uintptr_t p = reinterpret_cast<uintptr_t>(base) + (uintptr_t)idx * sizeof(typename Word<B>::T);
    unsigned* w = reinterpret_cast<unsigned*>(p & ~(uintptr_t)3);
    atomicOr(w, (unsigned)val << ((p & 3) * 8));
  }
}

// Rows of P with at least one entry (bit b-1-r of word R for row R*b+r).
// A row without entries can never be reached, so BFS and SSSP start with it
// marked visited: block rows whose other rows are done are then skipped
// instead of being scanned to the end for a parent that does not exist.
template <int B>
__global__ void __launch_bounds__(kTPB) k_live(GView v, typename Word<B>::T* __restrict__ live) {
  using WT = typename Word<B>::T;
  using L = Lay<B>;
  const unsigned lane = threadIdx.x & 31;
  const long long item = item_index(lane, L::W, L::G);
  const bool active = item < v.nitems;
  const int r = lane % L::W;
  const gbo_item it = active ? v.items[item] : gbo_item{0, 0, 0, -2};
  const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
  WT a0 = 0, a1 = 0;
  for (int t = it.t0; t < it.t1; ++t) {
    a0 = (WT)(a0 | val[(size_t)t * B + r]);
    if (L::RPL == 2) a1 = (WT)(a1 | val[(size_t)t * B + 32 + r]);
  }
  const WT word = gather_bits<B>(a0 != 0, a1 != 0, lane);
  if (active && r == 0 && word) atomic_or_word<B>(live, it.row, word);
}

// Top-down (push) step for symmetric P, used while the frontier is small:
// for every frontier row r of block row J and every tile (J, C), the row
// word (the neighbours of vertex J*b+r in block C) is OR-ed into the next
// frontier, minus vertices already visited.  One warp per work item, one
// lane per tile; k_bfs_finish then keeps the unvisited bits.
template <int B>
__device__ __forceinline__ void push_level(const GView& v, typename Word<B>::T* front,
                                           const typename Word<B>::T* visited, int lvl) {
  using WT = typename Word<B>::T;
  const WT* x = front_buf(front, v.nbr, lvl);
  WT* out = front_buf(front, v.nbr, lvl + 1);
  WT* z = front_buf(front, v.nbr, lvl + 2);
  const unsigned lane = threadIdx.x & 31;
  const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
  const long long nwarps = warps_total();
  // lane j reads item base + j * nwarps and its frontier word, so that one
  // round of loads finds the (few) items with frontier rows among the warp's
  // next 32; the stride keeps a hub's consecutive items on different warps
  for (long long base = warp_global(); base < v.nitems; base += nwarps * 32) {
    const long long mine = base + (long long)lane * nwarps;
    gbo_item itl = {0, 0, 0, -2};
    WT xl = 0;
    if (mine < v.nitems) {
      itl = v.items[mine];
      z[itl.row] = 0;
      xl = x[itl.row];
    }
    unsigned act = __ballot_sync(0xffffffffu, xl != 0);
    while (act) {
      const int jj = __ffs(act) - 1;
      act &= act - 1;
      const long long item = base + (long long)jj * nwarps;
      gbo_item it;
      it.row = __shfl_sync(0xffffffffu, itl.row, jj);
      it.t0 = __shfl_sync(0xffffffffu, itl.t0, jj);
      it.t1 = __shfl_sync(0xffffffffu, itl.t1, jj);
      const WT xs = shfl_word<WT>(0xffffffffu, xl, jj, 32);
      if constexpr (B == 32) {
        if (v.rowword) {
          // frontier rows with a non-empty word only (bit r = row r), read from
          // the packed row words; batches of 32 tiles give each tile's offset
          long long wb = v.item_wbase[item];
          const unsigned fr = __brev((unsigned)xs);
          for (int b0 = it.t0; b0 < it.t1; b0 += 32) {
            const int t = b0 + (int)lane;
            const unsigned m = t < it.t1 ? v.rowmask[t] : 0u;
            const int mc = __popc(m);
            const int mi = warp_incl_sum(mc, lane);
            const long long off = wb + (mi - mc);
            wb += __shfl_sync(0xffffffffu, mi, 31);
            unsigned sel = fr & m;
            if (!sel) continue;
            WT acc = 0;
            while (sel) {
              const int r = __ffs(sel) - 1;
              sel &= sel - 1;
              acc = (WT)(acc | v.rowword[rowword_index(off, m, r)]);
            }
            const int C = v.colind[t];
            const WT cand = (WT)(acc & ~visited[C]);
            if (cand) atomic_or_word<B>(out, C, cand);
          }
          continue;
        }
      }
      for (int t = it.t0 + (int)lane; t < it.t1; t += 32) {
        const int C = v.colind[t];
        WT acc = 0;
        for_each_col<B>(xs, [&](int r) { acc = (WT)(acc | val[(size_t)t * B + r]); });
        const WT cand = (WT)(acc & ~visited[C]);
        if (cand) atomic_or_word<B>(out, C, cand);
      }
    }
  }
}

template <int B>
__global__ void __launch_bounds__(kTPB) k_bfs_push(GView v, typename Word<B>::T* __restrict__ front,
                                                   const typename Word<B>::T* __restrict__ visited,
                                                   Ctrl* __restrict__ ctrl) {
  if (((volatile Ctrl*)ctrl)->done || !((volatile Ctrl*)ctrl)->mode) return;
  push_level<B>(v, front, visited, ((volatile Ctrl*)ctrl)->iter);
}

// ------------------------------------------------ COL tile layout (BFS)
// With column words (word c of a tile = column c, row r at bit b-1-r) a pull
// step needs, per tile, only the words of the columns whose frontier bit is
// set: rows(I) |= OR_{c in x[C]} word_c(I, C).  Sparse frontier segments then
// cost a word or two per tile instead of one word per unvisited row.

// OR of a word across the warp.
template <int B>
__device__ __forceinline__ typename Word<B>::T warp_or(typename Word<B>::T w) {
  if (B == 64) {
    const unsigned long long u = (unsigned long long)w;
    const unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)u);
    const unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(u >> 32));
    return (typename Word<B>::T)(((unsigned long long)hi << 32) | lo);
  }
  return (typename Word<B>::T)__reduce_or_sync(0xffffffffu, (unsigned)w);
}

// OR of the column words of tile t selected by the set bits of sel (bit
// b-1-c selects column c), four loads in flight.
template <int B>
__device__ __forceinline__ typename Word<B>::T or_selected_cols(const typename Word<B>::T* __restrict__ val,
                                                                long long t, typename Word<B>::T sel) {
  using WT = typename Word<B>::T;
  unsigned long long a = (unsigned long long)sel << (64 - B);
  WT acc = 0;
  while (a) {
    int c[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      c[q] = a ? __clzll((long long)a) : -1;
      if (a) a &= ~(0x8000000000000000ull >> c[q]);
    }
    WT w[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) w[q] = c[q] >= 0 ? val[(size_t)t * B + c[q]] : (WT)0;
#pragma unroll
    for (int q = 0; q < 4; ++q) acc = (WT)(acc | w[q]);
  }
  return acc;
}

// Rows with an entry, COL layout: OR of every column word of the block row.
template <int B>
__global__ void __launch_bounds__(kTPB) k_live_col(GView v, typename Word<B>::T* __restrict__ live) {
  using WT = typename Word<B>::T;
  const unsigned lane = threadIdx.x & 31;
  const long long item = warp_global();
  if (item >= v.nitems) return;
  const gbo_item it = v.items[item];
  const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
  WT acc = 0;
  for (long long q = (long long)it.t0 * B + lane; q < (long long)it.t1 * B; q += 32) acc = (WT)(acc | val[q]);
  acc = warp_or<B>(acc);
  if (lane == 0 && acc) atomic_or_word<B>(live, it.row, acc);
}

// Pull step on COL tiles: a warp per work item, a lane per tile, 32 tiles
// per batch; the block row leaves once its rows are all visited or found.
template <int B>
__global__ void __launch_bounds__(kTPB) k_bfs_step_col(GView v, typename Word<B>::T* __restrict__ front,
                                                       typename Word<B>::T* __restrict__ visited,
                                                       int* __restrict__ level, Ctrl* __restrict__ ctrl,
                                                       typename Word<B>::T* __restrict__ scratch) {
  using WT = typename Word<B>::T;
  if (((volatile Ctrl*)ctrl)->done || ((volatile Ctrl*)ctrl)->mode) return;
  const int lvl = ((volatile Ctrl*)ctrl)->iter;
  const WT* __restrict__ x = front_buf(front, v.nbr, lvl);
  WT* __restrict__ out = front_buf(front, v.nbr, lvl + 1);
  WT* __restrict__ z = front_buf(front, v.nbr, lvl + 2);
  const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
  const unsigned lane = threadIdx.x & 31;
  const WT full = full_word<B>();
  unsigned long long cnt = 0;
  constexpr long long kGrab = 16;
  long long w = 0, wend = 0;
  for (;;) {
    if (w == wend) {
      unsigned long long g0 = 0;
      if (lane == 0) g0 = atomicAdd(&ctrl->work, (unsigned long long)kGrab);
      w = (long long)__shfl_sync(0xffffffffu, g0, 0);
      wend = w + kGrab;
    }
    if (w >= v.nitems) break;
    const gbo_item it = v.items[w];
    ++w;
    const WT vis = visited[it.row];
    WT found = 0;
    if ((vis & full) != full) {
      // batch i's tiles are ORed while batch i+1's x words and batch i+2's
      // block-column indices load
      int c2 = (it.t0 + 32 + (int)lane < it.t1) ? v.colind[it.t0 + 32 + lane] : -1;
      const int c1 = (it.t0 + (int)lane < it.t1) ? v.colind[it.t0 + lane] : -1;
      WT x1 = c1 >= 0 ? x[c1] : (WT)0;
      for (int base = it.t0; base < it.t1; base += 32) {
        const WT xs = x1;
        x1 = c2 >= 0 ? x[c2] : (WT)0;
        c2 = (base + 64 + (int)lane < it.t1) ? v.colind[base + 64 + lane] : -1;
        const WT acc = xs ? or_selected_cols<B>(val, base + lane, xs) : (WT)0;
        found = (WT)(found | warp_or<B>(acc));
        if ((WT)((found | vis) & full) == full) break;
      }
    }
    if (lane == 0) z[it.row] = 0;
    if (it.slot >= 0) {
      if (lane == 0) scratch[it.slot] = found;
      continue;
    }
    const WT nw = (WT)(found & ~vis & full);
    if (nw) {
      for (int r = (int)lane; r < B; r += 32) {
        const long long row = (long long)it.row * B + r;
        if (bit_of<B>(nw, r) && row < v.nrows) level[row] = lvl + 1;
      }
      if (lane == 0) visited[it.row] = (WT)(vis | nw);
    }
    if (lane == 0) {
      out[it.row] = nw;
      cnt += popc_w(nw);
    }
  }
  block_add_u64(cnt, &ctrl->count);
}

// Push step on COL tiles of a symmetric P: the neighbours of frontier row r
// in block C are bit r of every column word of tile (J, C), so the lane of a
// tile reads all its words and keeps the columns that meet the frontier rows.
template <int B>
__global__ void __launch_bounds__(kTPB) k_bfs_push_col(GView v, typename Word<B>::T* __restrict__ front,
                                                       const typename Word<B>::T* __restrict__ visited,
                                                       Ctrl* __restrict__ ctrl) {
  using WT = typename Word<B>::T;
  if (((volatile Ctrl*)ctrl)->done || !((volatile Ctrl*)ctrl)->mode) return;
  const int lvl = ((volatile Ctrl*)ctrl)->iter;
  const WT* __restrict__ x = front_buf(front, v.nbr, lvl);
  WT* out = front_buf(front, v.nbr, lvl + 1);
  WT* __restrict__ z = front_buf(front, v.nbr, lvl + 2);
  const unsigned lane = threadIdx.x & 31;
  const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
  const long long nwarps = warps_total();
  for (long long item = warp_global(); item < v.nitems; item += nwarps) {
    const gbo_item it = v.items[item];
    if (lane == 0) z[it.row] = 0;
    const WT xs = x[it.row];
    if (!xs) continue;
    for (int t = it.t0 + (int)lane; t < it.t1; t += 32) {
      const int C = v.colind[t];
      WT cand = 0;
#pragma unroll 8
      for (int c = 0; c < B; ++c)
        if ((WT)(val[(size_t)t * B + c] & xs)) cand = (WT)(cand | ((WT)1 << (B - 1 - c)));
      cand = (WT)(cand & ~visited[C]);
      if (cand) atomic_or_word<B>(out, C, cand);
    }
  }
}

// After a push step: keep the unvisited bits of every next-frontier word,
// mark them visited and give their vertices level lvl + 1 (a thread per
// block row, grid-stride); returns the new vertices counted by this thread.
template <int B>
__device__ __forceinline__ unsigned long long finish_push_rows(const GView& v, typename Word<B>::T* front,
                                                               typename Word<B>::T* visited, int* level,
                                                               int lvl) {
  using WT = typename Word<B>::T;
  WT* out = front_buf(front, v.nbr, lvl + 1);
  const WT full = full_word<B>();
  unsigned long long cnt = 0;
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < v.nbr;
       i += (long long)gridDim.x * blockDim.x) {
    const WT o = out[i];
    if (!o) continue;
    const WT vis = visited[i];
    const WT nw = (WT)(o & ~vis & full);
    out[i] = nw;
    if (nw) {
      visited[i] = (WT)(vis | nw);
      for (int r = 0; r < B; ++r) {
        const long long row = i * B + r;
        if (bit_of<B>(nw, r) && row < v.nrows) level[row] = lvl + 1;
      }
      cnt += popc_w(nw);
    }
  }
  return cnt;
}

template <int B>
__global__ void k_bfs_finish(GView v, typename Word<B>::T* __restrict__ front,
                             typename Word<B>::T* __restrict__ visited, int* __restrict__ level,
                             Ctrl* __restrict__ ctrl, const typename Word<B>::T* __restrict__ scratch) {
  using WT = typename Word<B>::T;
  if (((volatile Ctrl*)ctrl)->done) return;
  const int lvl = ((volatile Ctrl*)ctrl)->iter;
  const int push = ((volatile Ctrl*)ctrl)->mode;
  WT* __restrict__ out = front_buf(front, v.nbr, lvl + 1);
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long cnt = 0;
  if (push) {
    cnt = finish_push_rows<B>(v, front, visited, level, lvl);
  } else if (i < v.nsplit) {
    const gbo_split sp = v.splits[i];
    const WT full = full_word<B>();
    const WT vis = visited[sp.row];
    WT w = 0;
    if ((vis & full) != full)
      for (int q = 0; q < sp.nslots; ++q) w |= scratch[sp.slot0 + q];
    const WT nw = (WT)(w & ~vis & full);
    out[sp.row] = nw;
    if (nw) {
      visited[sp.row] = (WT)(vis | nw);
      for (int r = 0; r < B; ++r) {
        long long row = (long long)sp.row * B + r;
        if (bit_of<B>(nw, r) && row < v.nrows) level[row] = lvl + 1;
      }
      cnt = popc_w(nw);
    }
  }
  block_add_u64(cnt, &ctrl->count);
  close_iteration(ctrl, [](volatile Ctrl* c, int it) {
    // direction of the next level: push while the new frontier is small
    const unsigned long long nf = c->count;
    c->mode = (c->push_thr > 0 && nf > 0ull && nf < (unsigned long long)c->push_thr) ? 1 : 0;
    return nf == 0ull || it >= c->max_iter;
  });
}

// Level-0 vertices of a multi-seed BFS (one thread: seeds may share words).
template <int B>
__global__ void k_bfs_seed(const int* __restrict__ seeds, int nseeds, typename Word<B>::T* front,
                           typename Word<B>::T* visited, int* level) {
  using WT = typename Word<B>::T;
  if (blockIdx.x != 0 || threadIdx.x != 0) return;
  for (int q = 0; q < nseeds; ++q) {
    const int v0 = seeds[q];
    const WT bit = (WT)((WT)1 << (B - 1 - v0 % B));
    front[v0 / B] = (WT)(front[v0 / B] | bit);
    visited[v0 / B] = (WT)(visited[v0 / B] | bit);
    level[v0] = 0;
  }
}

template <int B>
__global__ void k_bfs_init(typename Word<B>::T* front, typename Word<B>::T* visited, int* level,
                           const typename Word<B>::T* __restrict__ live, int nbr, int n, int src,
                           Ctrl* ctrl, int max_iter, int push_thr, int mode0,
                           unsigned long long* stamps = nullptr, int cap_iters = 0) {
  using WT = typename Word<B>::T;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = i; k < n; k += stride) level[k] = (k == src) ? 0 : -1;
  for (long long k = i; k < nbr; k += stride) {
    WT w = (src >= 0 && k == src / B) ? (WT)((WT)1 << (B - 1 - src % B)) : (WT)0;
    front[k] = w;
    front[front_stride(nbr) + k] = 0;
    front[2 * front_stride(nbr) + k] = 0;
    visited[k] = (WT)(w | (~live[k] & full_word<B>()));
  }
  if (i == 0) {
    ctrl->iter = 0;
    ctrl->done = 0;
    ctrl->ticket = 0;
    ctrl->max_iter = cap_iters > 0 && cap_iters < max_iter ? cap_iters : max_iter;
    if (stamps) {  // the cooperative loop's start
      ctrl->cond = 0ull;
      ctrl->stamps = stamps;
      unsigned long long t;
      asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
      stamps[0] = t;
    }
    ctrl->count = 0;
    ctrl->err = 0;
    ctrl->last_err = 0;
    ctrl->push_thr = push_thr;
    ctrl->mode = mode0;
    ctrl->work = 0ull;
    ctrl->bar_arrive = 0u;
    ctrl->bar_err = 0u;
    for (int q = 0; q < 3; ++q) ctrl->push_acc[q] = 0ull;
  }
  if (i < 3 * 8) ctrl->lvl_part[i / 8][i % 8][0] = 0ull;
}

// --------------------------------------------- cooperative BFS (b = 32)
// The whole level loop of a b = 32 ROW BFS in one cooperative launch (one
// grid of co-resident blocks).  Each level runs its step over the grid,
// sums the new vertices and meets the other blocks at a grid barrier, after
// which every block reads the same count and takes the same decision (stop,
// direction of the next level).  Per level this replaces the loop graph's
// kernel launches and conditional node with one barrier (pull levels) or
// two (push levels).  The frontier and visited words are read with plain
// loads (ld_state<true>): the barrier's fences make the other blocks' writes
// of the previous level visible to them.
//
// Push levels walk the row-word slices of the frontier rows only (not the
// tiles of their block rows): each entry (block column C, row word w) ORs
// w & ~visited[C] into next-frontier word C, and the bits that this atomic
// newly sets are vertices found here first, so the lane that set them marks
// them visited and writes their level -- no finishing pass.  Rows whose
// tails are long (hubs) are listed in phase A and their tails spread over
// the whole grid after the phase barrier (phase B).
//
// Three level counts (and push-list counters) rotate like the frontier
// buffers: level L adds into slot L % 3 and every block reads it after the
// barrier; block 0 then clears slot (L + 2) % 3, which every block read at
// level L - 1, before arriving at this level's barrier, and which level L + 2
// fills after the next barrier.

// A grid barrier gives up after this long (or this many polls).
constexpr unsigned long long kBarrierLimitNs = 5000000000ull;
constexpr long long kBarrierPollCap = 1ll << 28;
// Push list counter: listed rows in the high bits, tail entries in the low 40.
constexpr int kListShift = 40;
constexpr unsigned long long kListMask = (1ull << kListShift) - 1ull;

__device__ __forceinline__ unsigned long long global_ns() {
  unsigned long long t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Barrier over every block of a cooperative launch on one arrival word:
// block 0 adds 2^31 - (blocks - 1), every other block adds 1, so the sum of
// one barrier's arrivals flips the word's top bit and leaves the low bits
// as they were -- the block that arrives last completes the flip, with no
// reset or second atomic on the way out.  A block that waits past the limit,
// or sees that another block gave up, sets bar_err and returns false: the
// caller leaves the kernel, so every block ends within about one limit of
// the first failure.
__device__ __forceinline__ bool grid_barrier(Ctrl* c, unsigned long long limit_ns,
                                             const unsigned long long* sum_src = nullptr, int nsum = 0,
                                             int sum_stride = 1, unsigned long long* sum = nullptr) {
  __shared__ int ok;
  __shared__ unsigned long long sh_sum;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned inc = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1u) : 1u;
    volatile unsigned* word = &c->bar_arrive;
    volatile unsigned* err = &c->bar_err;
    __threadfence();
    const unsigned old = atomicAdd(&c->bar_arrive, inc);
    int res = 1;
    const unsigned long long t0 = global_ns();
    for (long long k = 0; ((old ^ *word) & 0x80000000u) == 0u; ++k) {
      if (*err || k >= kBarrierPollCap || global_ns() - t0 > limit_ns) {
        atomicExch(&c->bar_err, 1u);
        res = 0;
        break;
      }
    }
    __threadfence();
    ok = res;
    // one read of the counters per block, shared with its threads
    unsigned long long t = 0;
    for (int q = 0; q < nsum; ++q) t += __ldcg(sum_src + (size_t)q * sum_stride);
    sh_sum = t;
  }
  __syncthreads();
  if (sum) *sum = sh_sum;
  return ok != 0;
}

// Push one row word into next-frontier word C; the vertices this call finds
// first are marked visited and get level lvl + 1.  Returns their number.
// Returns their number plus, shifted by kLongShift, how many of them have
// long tails.
__device__ __forceinline__ unsigned long long push_word(const GView& v, unsigned* out, unsigned* visited,
                                                        int* level, int lvl, unsigned C, unsigned w) {
  const unsigned cand = w & ~visited[C];
  if (!cand) return 0ull;
  const unsigned nw = cand & ~atomicOr(out + C, cand);
  if (!nw) return 0ull;
  atomicOr(visited + C, nw);
  for (unsigned m = nw; m; m &= m - 1) level[(long long)C * 32 + (32 - __ffs(m))] = lvl + 1;
  return (unsigned long long)__popc(nw) + ((unsigned long long)__popc(nw & v.rws_longbits[C]) << kLongShift);
}

// Push phase A: block rows with frontier bits (a lane per block row picks
// them, strided over the grid like the pull step); the head entries and
// short tails of their frontier rows form one list per block row that the
// warp's lanes take 32 entries at a time.  Frontier rows with long tails go
// on the push list (start in the list's entry space, tail offset).
__device__ __forceinline__ unsigned long long push_rws_rows(const GView& v, unsigned* front, unsigned* visited,
                                                            int* level, int lvl, unsigned long long* list_acc,
                                                            long long* list) {
  const unsigned* x = front_buf(front, v.nbr, lvl);
  unsigned* out = front_buf(front, v.nbr, lvl + 1);
  unsigned* z = front_buf(front, v.nbr, lvl + 2);
  const unsigned lane = threadIdx.x & 31;
  const unsigned kFull = 0xffffffffu;
  const long long nwarps = warps_total();
  unsigned long long cnt = 0;
  for (long long base = warp_global(); base < v.nbr; base += 32 * nwarps) {
    const long long Rl = base + (long long)lane * nwarps;
    unsigned xl = 0u;
    if (Rl < v.nbr) {
      xl = x[Rl];
      z[Rl] = 0u;
    }
    unsigned act = __ballot_sync(kFull, xl != 0u);
    while (act) {
      const int j = __ffs(act) - 1;
      act &= act - 1;
      const long long R = base + (long long)j * nwarps;
      const unsigned fr = __shfl_sync(kFull, xl, j);
      const bool mine = (fr >> (31 - lane)) & 1u;
      long long tb = 0, tl = 0;
      if (mine) {
        tb = v.rws_tail_ptr[R * 32 + lane];
        tl = v.rws_tail_ptr[R * 32 + lane + 1] - tb;
      }
      const bool lng = tl > kRwsLongTail;
      if (lng) {
        const unsigned long long old = atomicAdd(list_acc, (1ull << kListShift) | (unsigned long long)tl);
        const long long q = (long long)(old >> kListShift);
        list[2 * q] = (long long)(old & kListMask);
        list[2 * q + 1] = tb;
      }
      const int len = mine ? kRwsHead + (lng ? 0 : (int)tl) : 0;
      const int incl = warp_incl_sum(len, lane);
      const int total = __shfl_sync(kFull, incl, 31);
      const uint2* hb = v.rws_head + (size_t)R * (kRwsHead * 32);
      for (int p = 0; p < total; p += 32) {
        const int q = p + (int)lane;
        // r = the first lane whose inclusive sum exceeds q (the entry's row)
        int r = 0;
#pragma unroll
        for (int st = 16; st > 0; st >>= 1)
          if (__shfl_sync(kFull, incl, r + st - 1) <= q) r += st;
        const int rin = __shfl_sync(kFull, incl, r);
        const int rlen = __shfl_sync(kFull, len, r);
        const long long rtb = __shfl_sync(kFull, tb, r);
        if (q < total) {
          const int slot = q - (rin - rlen);
          const uint2 e = slot < kRwsHead ? hb[(size_t)slot * 32 + r] : v.rws_tail[rtb + (slot - kRwsHead)];
          if (e.x != kRwsNone) cnt += push_word(v, out, visited, level, lvl, e.x, e.y);
        }
      }
    }
  }
  return cnt;
}

// Push phase B: the listed long tails as one entry space over every thread
// of the grid; a thread finds its entry's row by binary search over the
// list's starts.
__device__ __forceinline__ unsigned long long push_rws_long(const GView& v, unsigned* front, unsigned* visited,
                                                            int* level, int lvl, unsigned long long acc,
                                                            const long long* list) {
  unsigned* out = front_buf(front, v.nbr, lvl + 1);
  const long long nl = (long long)(acc >> kListShift);
  const long long total = (long long)(acc & kListMask);
  unsigned long long cnt = 0;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < total;
       q += (long long)gridDim.x * blockDim.x) {
    long long lo = 0, hi = nl - 1;
    while (lo < hi) {
      const long long mid = (lo + hi + 1) >> 1;
      if (list[2 * mid] <= q) lo = mid;
      else hi = mid - 1;
    }
    const uint2 e = v.rws_tail[list[2 * lo + 1] + (q - list[2 * lo])];
    cnt += push_word(v, out, visited, level, lvl, e.x, e.y);
  }
  return cnt;
}

// limit_ns bounds every barrier wait (kBarrierLimitNs; shorter in the
// failure-path test, which also names a block that leaves at once, before
// the first barrier: skip_block, -1 for none).
__global__ void __launch_bounds__(kTPB, kCoopBlocksPerSM) k_bfs_coop(GView v, unsigned* front, unsigned* visited,
                                                                  int* level, Ctrl* ctrl, long long* push_list,
                                                                  unsigned long long limit_ns, int skip_block) {
  if ((int)blockIdx.x == skip_block) return;
  // the loop's starting state: written before the launch and changed by
  // block 0 only after the first barrier, so plain (cached) loads -- one
  // L2 request per SM instead of one per warp
  volatile Ctrl* vc = ctrl;
  if (ctrl->done) return;
  int lvl = ctrl->iter;
  int mode = ctrl->mode;
  const int max_iter = ctrl->max_iter;
  const unsigned long long push_thr = ctrl->push_thr > 0 ? (unsigned long long)ctrl->push_thr : 0ull;
  unsigned long long* stamps = ctrl->stamps;
  bool hubs = true;  // the frontier may hold rows with long tails (unknown at the start)
  for (;;) {
    unsigned long long cnt;
    if (!mode) {
      cnt = pull_rws_level<true>(v, front, visited, level, lvl);
    } else {
      cnt = push_rws_rows(v, front, visited, level, lvl, &ctrl->push_acc[lvl % 3], push_list);
      if (hubs) {  // the listed long tails, after every block listed its rows
        unsigned long long acc = 0;
        if (!grid_barrier(ctrl, limit_ns, &ctrl->push_acc[lvl % 3], 1, 1, &acc)) return;
        if (acc) cnt += push_rws_long(v, front, visited, level, lvl, acc, push_list);
      }
    }
    block_add_u64(cnt, &ctrl->lvl_part[lvl % 3][blockIdx.x & 7][0]);
    unsigned long long tot = 0;
    if (!grid_barrier(ctrl, limit_ns, &ctrl->lvl_part[lvl % 3][0][0], 8, 16, &tot)) return;
    const unsigned long long nf = tot & kLongMask;
    hubs = (tot >> kLongShift) != 0ull;
    const int it = lvl + 1;
    const bool stop = nf == 0ull || it >= max_iter;
    mode = (nf > 0ull && nf < push_thr) ? 1 : 0;
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      for (int q = 0; q < 8; ++q) ctrl->lvl_part[(lvl + 2) % 3][q][0] = 0ull;
      ctrl->push_acc[(lvl + 2) % 3] = 0ull;
      vc->iter = it;
      vc->mode = mode;
      vc->count = nf;
      if (stop) vc->done = 1;
      if (stamps && it <= kStampCap) stamps[it] = global_ns();
      __threadfence();
    }
    if (stop) return;
    lvl = it;
  }
}

// ============================================================= SSSP
// Unit weights: every frontier vertex at iteration k has distance k, so the
// min-plus relaxation min_j (d[j] + 1) over a row's frontier neighbours is
// k + 1 as soon as one such neighbour exists.  The SSSP step is therefore
// the BFS step (pull with early exit, push on small frontiers of symmetric
// graphs); distances are the levels in uint32 with 2147483647 unreachable.
__global__ void k_level_to_dist(uint32_t* __restrict__ d, int n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const int lv = (int)d[i];
    d[i] = lv < 0 ? (uint32_t)kINF : (uint32_t)lv;
  }
}

// ============================================================ PageRank
// p'[i] = alpha * sum_{j: P[i][j]} p[j] * inv[j] + add + add_scale * v[i].
// New value of row i from its gathered sum a (fp64): PageRank / PPR forward
// y = alpha * a + add + add_scale * pv[i], with a = sum of x[j] / deg(j);
// adjoint on a symmetric P (row_scale) y = pv[i] + alpha * inv[i] * a with
// a = sum of u[j].  Writes y (and y * inv[i], the next gathered operand, for
// PageRank) and returns the |change| (or its square for the L2 norm).
__device__ __forceinline__ double pr_row_update(long long i, double a, const float* __restrict__ x,
                                                float* __restrict__ y, float* __restrict__ ys,
                                                const float* __restrict__ inv, const float* __restrict__ pv,
                                                double alpha, double add, double adds, int norm,
                                                int row_scale) {
  const double base = pv ? adds * (double)pv[i] : 0.0;
  const float yn = row_scale ? (float)(base + alpha * (double)inv[i] * a) : (float)(alpha * a + add + base);
  y[i] = yn;
  if (!row_scale) ys[i] = yn * inv[i];
  const double d = (double)yn - (double)x[i];
  return norm == 1 ? fabs(d) : d * d;
}

template <int B>
__global__ void __launch_bounds__(kTPB) k_pr_step(GView v, float* __restrict__ pr, float* __restrict__ prs,
                                                  const float* __restrict__ inv,
                                                  const float* __restrict__ pv,
                                                  Ctrl* __restrict__ ctrl, double* __restrict__ scratch) {
  using L = Lay<B>;
  if (((volatile Ctrl*)ctrl)->done) return;
  const int itn = ((volatile Ctrl*)ctrl)->iter;
  const double alpha = ctrl->alpha, add = ctrl->add, adds = ctrl->add_scale;
  const int norm = ctrl->norm, row_scale = ctrl->row_scale;
  const int n = v.nrows;
  const float* __restrict__ x = pr + (size_t)(itn & 1) * n;
  float* __restrict__ y = pr + (size_t)((itn + 1) & 1) * n;
  float* __restrict__ ys = prs + (size_t)((itn + 1) & 1) * n;
  // gathered operand: x / deg (kept up to date by the previous iteration) or x
  const float* __restrict__ xg = row_scale ? x : prs + (size_t)(itn & 1) * n;
  const unsigned lane = threadIdx.x & 31;
  double e = 0.0;
  const long long nwarps = warps_total();
  for (long long w = warp_global(); w * L::G < v.nitems; w += nwarps) {
    const long long item = w * L::G + lane / L::W;
    if (item < v.nitems) {
      const int r = lane % L::W;
      const gbo_item it = v.items[item];
      double a0 = 0.0, a1 = 0.0;
      fold_row_cols<B, 4>(v, it.t0, it.t1, v.item_wbase ? v.item_wbase[item] : 0ll, r, [&](long long j) { return (double)xg[j]; },
                          [](double& a, double b) { a += b; }, a0, a1);
      if (it.slot >= 0) {
        scratch[(size_t)it.slot * B + r] = a0;
        if (L::RPL == 2) scratch[(size_t)it.slot * B + 32 + r] = a1;
      } else {
        const long long row0 = (long long)it.row * B + r;
        if (row0 < n) e += pr_row_update(row0, a0, x, y, ys, inv, pv, alpha, add, adds, norm, row_scale);
        if (L::RPL == 2 && row0 + 32 < n)
          e += pr_row_update(row0 + 32, a1, x, y, ys, inv, pv, alpha, add, adds, norm, row_scale);
      }
    }
  }
  block_add_f64(e, &ctrl->err);
}

// The same iteration over the row-word slices of a b = 32 ROW graph: a warp
// per block row, lane r sums row r's columns entry by entry (the head's
// entry k of the 32 rows in one 256-byte load, two entries in flight), then
// its tail.  Rows with tails longer than kRwsLongTail (hubs) are left to
// k_pr_long_chunks / k_pr_long_rows, which spread them over many warps.
// Every row's sum has a fixed order (fp64), whatever the grid.
__device__ __forceinline__ double pr_word_sum(unsigned c, unsigned w, const float* __restrict__ xg) {
  double a = 0.0;
  const size_t base = (size_t)c * 32;
  while (w) {
    const int j = __clz(w);
    a += (double)__ldg(xg + base + j);
    w &= ~(0x80000000u >> j);
  }
  return a;
}

// Four entries at once: the gathered operand of one set column per entry
// per round, four gathers in flight; the adds follow a fixed order (round,
// then entry), so a row's sum depends on the graph only.
__device__ __forceinline__ double pr_entries4(const uint2 (&e)[4], const float* __restrict__ xg) {
  uint32_t m[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) m[u] = e[u].x != kRwsNone ? e[u].y : 0u;
  double a = 0.0;
  while (m[0] | m[1] | m[2] | m[3]) {
    float g[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      g[u] = 0.f;
      if (m[u]) {
        const int j = __clz(m[u]);
        m[u] &= ~(0x80000000u >> j);
        g[u] = __ldg(xg + (size_t)e[u].x * 32 + j);
      }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) a += (double)g[u];
  }
  return a;
}

// The whole head (eight entries) at once: PageRank reads every entry of a
// row, so the second half is not worth a round trip of its own.
__device__ __forceinline__ double pr_entries8(const uint2 (&e)[8], const float* __restrict__ xg) {
  uint32_t m[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) m[u] = e[u].x != kRwsNone ? e[u].y : 0u;
  double a = 0.0;
  while (m[0] | m[1] | m[2] | m[3] | m[4] | m[5] | m[6] | m[7]) {
    float g[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      g[u] = 0.f;
      if (m[u]) {
        const int j = __clz(m[u]);
        m[u] &= ~(0x80000000u >> j);
        g[u] = __ldg(xg + (size_t)e[u].x * 32 + j);
      }
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) a += (double)g[u];
  }
  return a;
}

struct PrIter {  // the iterate's buffers and coefficients of iteration itn
  const float* x;
  float* y;
  float* ys;
  const float* xg;
  double alpha, add, adds;
  int norm, row_scale;
};

__device__ __forceinline__ PrIter pr_iter(float* pr, float* prs, const Ctrl* ctrl, int n) {
  PrIter p;
  const int itn = ((volatile Ctrl*)ctrl)->iter;
  p.alpha = ctrl->alpha;
  p.add = ctrl->add;
  p.adds = ctrl->add_scale;
  p.norm = ctrl->norm;
  p.row_scale = ctrl->row_scale;
  p.x = pr + (size_t)(itn & 1) * n;
  p.y = pr + (size_t)((itn + 1) & 1) * n;
  p.ys = prs + (size_t)((itn + 1) & 1) * n;
  p.xg = p.row_scale ? p.x : prs + (size_t)(itn & 1) * n;
  return p;
}

// Five blocks per SM (48 registers, a few spilled): the step is bound by the
// latency of its gathers, and R-MAT 22 iterations took 1.05 ms at the 71
// registers (3 blocks per SM) the compiler chose unbounded, 0.97 ms at 4
// blocks and 0.90 ms at 5 to 8.
__global__ void __launch_bounds__(kTPB, 5) k_pr_step_rws(GView v, float* __restrict__ pr, float* __restrict__ prs,
                                                      const float* __restrict__ inv,
                                                      const float* __restrict__ pv, Ctrl* __restrict__ ctrl) {
  __shared__ double pr_tail_sh[kTPB / 32][32];
  if (((volatile Ctrl*)ctrl)->done) return;
  const int n = v.nrows;
  const PrIter P = pr_iter(pr, prs, ctrl, n);
  const unsigned lane = threadIdx.x & 31;
  const unsigned kFull = 0xffffffffu;
  double e = 0.0;
  const long long nwarps = warps_total();
  for (long long R = warp_global(); R < v.nbr; R += nwarps) {
    const long long row = R * 32 + lane;
    const uint2* __restrict__ hp = v.rws_head + (size_t)R * (kRwsHead * 32) + lane;
    // the head's eight entries and the tail offsets in one round of loads
    static_assert(kRwsHead == 8, "pr_entries8 takes the whole head");
    uint2 h8[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) h8[u] = hp[(size_t)u * 32];
    const long long tb = v.rws_tail_ptr[row], te = v.rws_tail_ptr[row + 1];
    double a = pr_entries8(h8, P.xg);
    const bool long_row = te - tb > kRwsLongTail;  // the chunk kernels own a long row
    // The block row's short tails as one list, 32 entries per round over the
    // warp's lanes (a lane per row would wait for the block row's longest
    // tail): lane q of a round finds its entry's row r by a binary search
    // over the tails' inclusive sums, and a segmented scan across the lanes
    // adds each row's entries of the round, in lane order, into tsum[r].
    const int len = long_row ? 0 : (int)(te - tb);
    const int incl = warp_incl_sum(len, lane);
    const int total = __shfl_sync(kFull, incl, 31);
    double* tsum = pr_tail_sh[threadIdx.x >> 5];
    tsum[lane] = 0.0;
    __syncwarp();
    for (int p0 = 0; p0 < total; p0 += 32) {
      const int q = p0 + (int)lane;
      int r = 0;
#pragma unroll
      for (int st = 16; st > 0; st >>= 1)
        if (__shfl_sync(kFull, incl, r + st - 1) <= q) r += st;
      const int rin = __shfl_sync(kFull, incl, r);
      const int rlen = __shfl_sync(kFull, len, r);
      const long long rtb = __shfl_sync(kFull, tb, r);
      double val = 0.0;
      if (q < total) {
        const uint2 t = v.rws_tail[rtb + (q - (rin - rlen))];
        for (uint32_t m = t.y; m;) {
          const int j = __clz(m);
          m &= ~(0x80000000u >> j);
          val += (double)__ldg(P.xg + (size_t)t.x * 32 + j);
        }
      }
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const double y = __shfl_up_sync(kFull, val, o);
        const int ry = __shfl_up_sync(kFull, r, o);
        if ((int)lane >= o && ry == r) val += y;
      }
      const int rn = __shfl_down_sync(kFull, r, 1);
      if (q < total && (lane == 31 || q + 1 == total || rn != r)) tsum[r] += val;
      __syncwarp();
    }
    a += tsum[lane];
    if (row < n && !long_row)
      e += pr_row_update(row, a, P.x, P.y, P.ys, inv, pv, P.alpha, P.add, P.adds, P.norm, P.row_scale);
  }
  block_add_f64(e, &ctrl->err);
}

// Long rows, part 1: a warp per chunk of a long row's tail sums its entries
// (lanes strided, partial sums combined by a fixed shuffle tree); the first
// chunk of a row also sums the row's head.  One fp64 partial per chunk.
__global__ void __launch_bounds__(kTPB) k_pr_long_chunks(GView v, float* __restrict__ pr,
                                                         float* __restrict__ prs, Ctrl* __restrict__ ctrl,
                                                         double* __restrict__ part) {
  if (((volatile Ctrl*)ctrl)->done) return;
  const PrIter P = pr_iter(pr, prs, ctrl, v.nrows);
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = warps_total();
  for (long long q = warp_global(); q < v.rws_nchunk; q += nwarps) {
    const long long row = v.rws_chunk_row[q];
    const long long b = v.rws_chunk_beg[q], e = v.rws_chunk_end[q];
    double a = 0.0;
    if (b == v.rws_tail_ptr[row] && lane < kRwsHead) {
      const uint2 h = v.rws_head[((size_t)(row >> 5) * kRwsHead + lane) * 32 + (row & 31)];
      a += pr_word_sum(h.x, h.y, P.xg);  // a long row fills its head
    }
    for (long long p = b + lane; p < e; p += 128) {
      uint2 t[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) t[u] = p + 32 * u < e ? v.rws_tail[p + 32 * u] : make_uint2(kRwsNone, 0u);
      a += pr_entries4(t, P.xg);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) a += __shfl_xor_sync(0xffffffffu, a, o);
    if (lane == 0) part[q] = a;
  }
}

// Long rows, part 2: a thread per long row adds its chunks' partials in
// chunk order and updates the row.
__global__ void k_pr_long_rows(GView v, float* __restrict__ pr, float* __restrict__ prs,
                               const float* __restrict__ inv, const float* __restrict__ pv,
                               Ctrl* __restrict__ ctrl, const double* __restrict__ part) {
  if (((volatile Ctrl*)ctrl)->done) return;
  const PrIter P = pr_iter(pr, prs, ctrl, v.nrows);
  const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (q < v.rws_nlong) {
    const long long row = v.rws_long_row[q];
    double a = 0.0;
    for (long long c = v.rws_long_chunk0[q]; c < v.rws_long_chunk0[q + 1]; ++c) a += part[c];
    if (row < v.nrows)
      e = pr_row_update(row, a, P.x, P.y, P.ys, inv, pv, P.alpha, P.add, P.adds, P.norm, P.row_scale);
  }
  block_add_f64(e, &ctrl->err);
}

template <int B>
__global__ void k_pr_finish(GView v, float* __restrict__ pr, float* __restrict__ prs,
                            const float* __restrict__ inv, const float* __restrict__ pv,
                            Ctrl* __restrict__ ctrl, const double* __restrict__ scratch) {
  if (((volatile Ctrl*)ctrl)->done) return;
  const int itn = ((volatile Ctrl*)ctrl)->iter;
  const double alpha = ctrl->alpha, add = ctrl->add, adds = ctrl->add_scale;
  const int norm = ctrl->norm, row_scale = ctrl->row_scale;
  const int n = v.nrows;
  const float* __restrict__ x = pr + (size_t)(itn & 1) * n;
  float* __restrict__ y = pr + (size_t)((itn + 1) & 1) * n;
  float* __restrict__ ys = prs + (size_t)((itn + 1) & 1) * n;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  double e = 0.0;
  if (gid < (long long)v.nsplit * B) {
    const gbo_split sp = v.splits[gid / B];
    const int r = (int)(gid % B);
    double a = 0.0;
    for (int q = 0; q < sp.nslots; ++q) a += scratch[(size_t)(sp.slot0 + q) * B + r];
    const long long row = (long long)sp.row * B + r;
    if (row < n) e += pr_row_update(row, a, x, y, ys, inv, pv, alpha, add, adds, norm, row_scale);
  }
  block_add_f64(e, &ctrl->err);
  close_iteration(ctrl, [](volatile Ctrl* c, int it) {
    const double m = c->norm == 2 ? sqrt(c->err) : c->err;
    const double ref = c->ref > 0.0 ? c->ref : 1.0;  // ||w||_1 for the adjoint, else 1
    return it >= c->max_iter || (c->tol >= 0.f && m <= (double)c->tol * ref);
  });
}

__global__ void k_pr_init(float* pr, float* prs, const float* inv, const float* pv, int n,
                          float init_const, float init_scale, Ctrl* ctrl, int max_iter, float tol,
                          float alpha, float add, float add_scale, int norm, int row_scale) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = i; k < n; k += stride) {
    const float x0 = init_const + (pv ? init_scale * pv[k] : 0.f);
    pr[k] = x0;
    pr[n + k] = 0.f;
    if (prs) {
      prs[k] = inv ? x0 * inv[k] : 0.f;
      prs[n + k] = 0.f;
    }
  }
  if (i == 0) {
    ctrl->iter = 0;
    ctrl->done = max_iter <= 0 ? 1 : 0;
    ctrl->ticket = 0;
    ctrl->max_iter = max_iter;
    ctrl->count = 0;
    ctrl->err = 0;
    ctrl->last_err = 0;
    ctrl->bar_err = 0u;
    ctrl->tol = tol;
    ctrl->alpha = alpha;
    ctrl->add = add;
    ctrl->add_scale = add_scale;
    ctrl->norm = norm;
    ctrl->n = n;
    ctrl->ref = 0.0;
    ctrl->row_scale = row_scale;
  }
}

// ===================================================== PPR adjoint step
// u'[j] = w[j] + alpha * inv[j] * sum_{i: P[i][j]} u[i]   (P^T by scatter)
__global__ void k_adj_prep(float* __restrict__ pr, const float* __restrict__ w, int n,
                           Ctrl* __restrict__ ctrl, double* __restrict__ acc) {
  if (((volatile Ctrl*)ctrl)->done) return;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = i; k < n; k += stride) acc[k] = 0.0;
}

template <int B>
__global__ void __launch_bounds__(kTPB) k_adj_scatter(GView v, const float* __restrict__ pr,
                                                      Ctrl* __restrict__ ctrl, double* __restrict__ acc) {
  using WT = typename Word<B>::T;
  using L = Lay<B>;
  if (((volatile Ctrl*)ctrl)->done) return;
  const int itn = ((volatile Ctrl*)ctrl)->iter;
  const int n = v.nrows;
  const float* __restrict__ u = pr + (size_t)(itn & 1) * n;
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = warps_total();
  for (long long w = warp_global(); w * L::G < v.nitems; w += nwarps) {
    const long long item = w * L::G + lane / L::W;
    if (item >= v.nitems) continue;
    const int r = lane % L::W;
    const gbo_item it = v.items[item];
    const long long row0 = (long long)it.row * B + r;
    const float u0 = row0 < n ? u[row0] : 0.f;
    const float u1 = (L::RPL == 2 && row0 + 32 < n) ? u[row0 + 32] : 0.f;
    if (u0 == 0.f && u1 == 0.f) continue;
    const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
    for (int t = it.t0; t < it.t1; ++t) {
      const long long base = (long long)v.colind[t] * B;
      if (u0 != 0.f)
        for_each_col<B>(val[(size_t)t * B + r], [&](int j) { atomicAdd(acc + base + j, (double)u0); });
      if (L::RPL == 2 && u1 != 0.f)
        for_each_col<B>(val[(size_t)t * B + 32 + r], [&](int j) { atomicAdd(acc + base + j, (double)u1); });
    }
  }
}

__global__ void k_adj_apply(float* __restrict__ pr, const float* __restrict__ w,
                            const float* __restrict__ inv, int n, Ctrl* __restrict__ ctrl,
                            const double* __restrict__ acc) {
  if (((volatile Ctrl*)ctrl)->done) return;
  const int itn = ((volatile Ctrl*)ctrl)->iter;
  const float alpha = ctrl->alpha;
  const float* __restrict__ x = pr + (size_t)(itn & 1) * n;
  float* __restrict__ y = pr + (size_t)((itn + 1) & 1) * n;
  double e = 0.0;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x) {
    float yn = (float)((double)w[k] + (double)alpha * (double)inv[k] * acc[k]);
    y[k] = yn;
    e += fabs((double)yn - (double)x[k]);
  }
  block_add_f64(e, &ctrl->err);
  close_iteration(ctrl, [](volatile Ctrl* c, int it) {
    // relative test: w is any real vector, not a distribution
    const double ref = c->ref > 0.0 ? c->ref : 1.0;
    return it >= c->max_iter || (c->tol >= 0.f && c->err <= (double)c->tol * ref);
  });
}

// ||w||_1 into ctrl->ref (after k_pr_init zeroed it).
__global__ void k_l1_ref(const float* __restrict__ w, int n, Ctrl* __restrict__ ctrl) {
  double e = 0.0;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    e += fabs((double)w[k]);
  block_add_f64(e, &ctrl->ref);
}

__global__ void k_scale_copy(const float* __restrict__ src, float* __restrict__ dst, int n, float s) {
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < n;
       k += (long long)gridDim.x * blockDim.x)
    dst[k] = s * src[k];
}

// ================================================================== CC
// FastSV (Zhang, Azad, Hu 2020): min-neighbour grandparent, stochastic and
// aggressive hooking, shortcutting, until the grandparents stop changing.
template <int B>
__global__ void __launch_bounds__(kTPB) k_cc_mngf(GView v, const int* __restrict__ gf,
                                                  int* __restrict__ mngf, Ctrl* __restrict__ ctrl,
                                                  int* __restrict__ scratch) {
  using WT = typename Word<B>::T;
  using L = Lay<B>;
  if (((volatile Ctrl*)ctrl)->done) return;
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = warps_total();
  for (long long w = warp_global(); w * L::G < v.nitems; w += nwarps) {
    const long long item = w * L::G + lane / L::W;
    if (item >= v.nitems) continue;
    const int r = lane % L::W;
    const gbo_item it = v.items[item];
    int a0 = kINF, a1 = kINF;
    fold_row_cols<B, 4>(v, it.t0, it.t1, v.item_wbase ? v.item_wbase[item] : 0ll, r, [&](long long j) { return gf[j]; },
                        [](int& a, int b) { a = min(a, b); }, a0, a1);
    if (it.slot >= 0) {
      scratch[(size_t)it.slot * B + r] = a0;
      if (L::RPL == 2) scratch[(size_t)it.slot * B + 32 + r] = a1;
      continue;
    }
    const long long row0 = (long long)it.row * B + r;
    if (row0 < v.nrows && a0 < mngf[row0]) mngf[row0] = a0;
    if (L::RPL == 2 && row0 + 32 < v.nrows && a1 < mngf[row0 + 32]) mngf[row0 + 32] = a1;
  }
}

// The same minimum over the row-word slices of a 32x32 ROW graph: a warp per
// block row, lane r over row r's entries (the whole head in one round, then
// tails of up to kRwsLongTail entries four at a time), the grandparent of
// every column of each entry gathered; longer tails are k_cc_mngf_chunks'.
__device__ __forceinline__ int cc_min_entries(const uint2* e, int ne, const int* __restrict__ gf, int a) {
  for (int u = 0; u < ne; ++u) {
    if (e[u].x == kRwsNone) continue;
    for (uint32_t m = e[u].y; m;) {
      const int j = __clz(m);
      m &= ~(0x80000000u >> j);
      a = min(a, __ldg(gf + (size_t)e[u].x * 32 + j));
    }
  }
  return a;
}

__global__ void __launch_bounds__(kTPB) k_cc_mngf_rws(GView v, const int* __restrict__ gf, int* __restrict__ mngf,
                                                      Ctrl* __restrict__ ctrl) {
  if (((volatile Ctrl*)ctrl)->done) return;
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = warps_total();
  for (long long R = warp_global(); R < v.nbr; R += nwarps) {
    const long long row = R * 32 + lane;
    const uint2* __restrict__ hp = v.rws_head + (size_t)R * (kRwsHead * 32) + lane;
    uint2 h8[kRwsHead];
#pragma unroll
    for (int u = 0; u < kRwsHead; ++u) h8[u] = hp[(size_t)u * 32];
    const long long tb = v.rws_tail_ptr[row], te = v.rws_tail_ptr[row + 1];
    int a = cc_min_entries(h8, kRwsHead, gf, kINF);
    if (te - tb <= kRwsLongTail) {
      for (long long p = tb; p < te; p += 4) {
        uint2 e[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) e[u] = p + u < te ? v.rws_tail[p + u] : make_uint2(kRwsNone, 0u);
        a = cc_min_entries(e, 4, gf, a);
      }
    }
    if (row < v.nrows && a < mngf[row]) mngf[row] = a;
  }
}

// Long tails: a warp per chunk, the chunk's minimum folded into its row with
// atomicMin (after k_cc_mngf_rws wrote the row's head and short part).
__global__ void __launch_bounds__(kTPB) k_cc_mngf_chunks(GView v, const int* __restrict__ gf,
                                                         int* __restrict__ mngf, Ctrl* __restrict__ ctrl) {
  if (((volatile Ctrl*)ctrl)->done) return;
  const unsigned lane = threadIdx.x & 31;
  const long long nwarps = warps_total();
  for (long long q = warp_global(); q < v.rws_nchunk; q += nwarps) {
    const long long e0 = v.rws_chunk_end[q];
    int a = kINF;
    for (long long p = v.rws_chunk_beg[q] + lane; p < e0; p += 32) {
      const uint2 e = v.rws_tail[p];
      a = cc_min_entries(&e, 1, gf, a);
    }
    a = __reduce_min_sync(0xffffffffu, a);
    const long long row = v.rws_chunk_row[q];
    if (lane == 0 && row < v.nrows && a < mngf[row]) atomicMin(mngf + row, a);
  }
}

template <int B>
__global__ void k_cc_mngf_finish(GView v, int* __restrict__ mngf, Ctrl* __restrict__ ctrl,
                                 const int* __restrict__ scratch) {
  if (((volatile Ctrl*)ctrl)->done) return;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)v.nsplit * B) return;
  const gbo_split sp = v.splits[gid / B];
  const int r = (int)(gid % B);
  int a = kINF;
  for (int q = 0; q < sp.nslots; ++q) a = min(a, scratch[(size_t)(sp.slot0 + q) * B + r]);
  const long long row = (long long)sp.row * B + r;
  if (row < v.nrows && a < mngf[row]) mngf[row] = a;
}

__global__ void k_cc_hook(int* __restrict__ f, const int* __restrict__ mngf, int n, Ctrl* ctrl) {
  if (((volatile Ctrl*)ctrl)->done) return;
  for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (long long)gridDim.x * blockDim.x) {
    const int m = mngf[u];
    const int fu = f[u];
    if (m < fu) atomicMin(f + fu, m);  // stochastic hooking f[f[u]] <- mngf[u]
  }
}

__global__ void k_cc_shortcut(int* __restrict__ f, const int* __restrict__ mngf,
                              const int* __restrict__ gf, int n, Ctrl* ctrl) {
  if (((volatile Ctrl*)ctrl)->done) return;
  for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (long long)gridDim.x * blockDim.x) {
    const int m = min(mngf[u], gf[u]);  // aggressive hooking + shortcutting
    if (m < f[u]) atomicMin(f + u, m);
  }
}

__global__ void k_cc_grand(const int* __restrict__ f, int* __restrict__ gf, int n, Ctrl* ctrl) {
  if (((volatile Ctrl*)ctrl)->done) return;
  unsigned long long changed = 0;
  for (long long u = (long long)blockIdx.x * blockDim.x + threadIdx.x; u < n;
       u += (long long)gridDim.x * blockDim.x) {
    const int g2 = f[f[u]];
    if (g2 != gf[u]) {
      gf[u] = g2;
      ++changed;
    }
  }
  block_add_u64(changed, &ctrl->count);
  close_iteration(ctrl, [](volatile Ctrl* c, int it) {
    return c->count == 0ull || it >= c->max_iter;
  });
}

__global__ void k_cc_init(int* f, int* gf, int* mngf, int n, Ctrl* ctrl, int max_iter) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  for (long long k = i; k < n; k += stride) {
    f[k] = (int)k;
    gf[k] = (int)k;
    mngf[k] = (int)k;
  }
  if (i == 0) {
    ctrl->iter = 0;
    ctrl->done = 0;
    ctrl->ticket = 0;
    ctrl->max_iter = max_iter;
    ctrl->count = 0;
    ctrl->err = 0;
    ctrl->last_err = 0;
    ctrl->bar_err = 0u;
  }
}

// ================================================================ host
unsigned grid_for_items(int nitems, int b) {
  const int G = b >= 32 ? 1 : 32 / b;
  long long warps = ((long long)nitems + G - 1) / G;
  return blocks_for_warps(warps, kTPB / 32);
}

// Persistent grid of an iteration kernel: enough warps for every item, and
// no more blocks than stay resident together (the kernels loop over items,
// so a second wave would only lengthen the tail).
template <typename K>
unsigned grid_persistent(K kernel, long long warps) {
  const unsigned g = blocks_for_warps(warps, kTPB / 32);
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTPB, 0) != cudaSuccess || per_sm < 1) {
    (void)cudaGetLastError();
    per_sm = 1;
  }
  const unsigned cap = (unsigned)num_sms() * (unsigned)per_sm;
  return g < cap ? g : cap;
}

// Same, for a kernel that gives each work item min(b, 32) lanes.
template <typename K>
unsigned grid_items_persistent(K kernel, int nitems, int b) {
  const int G = b >= 32 ? 1 : 32 / b;
  return grid_persistent(kernel, ((long long)nitems + G - 1) / G);
}

unsigned grid_vertex(long long n) {
  unsigned g = blocks_for(n, kTPB);
  unsigned cap = (unsigned)num_sms() * 8u;
  return g < cap ? g : cap;
}

int get_state(gbo_graph* g, AlgoState** out) {
  g->last_run_ms = 0;  // statistics now describe this algorithm's run
  if (!g->algo) {
    AlgoState* a = new AlgoState();
    g->algo = a;
    GBO_CUDA_TRY(cudaStreamCreateWithFlags(&a->cap, cudaStreamNonBlocking));
    GBO_CUDA_TRY(cudaMalloc(&a->ctrl, sizeof(Ctrl)));
    GBO_CUDA_TRY(cudaMemset(a->ctrl, 0, sizeof(Ctrl)));
    GBO_CUDA_TRY(cudaHostAlloc(&a->h_ctrl, sizeof(Ctrl), cudaHostAllocDefault));
    const size_t sb = (size_t)g->nslots * (size_t)g->b * 8 + 64;
    GBO_CUDA_TRY(cudaMalloc(&a->scratch, sb));
    g->device_bytes += (long long)sb + (long long)sizeof(Ctrl);
    GBO_CUDA_TRY(cudaMalloc(&a->stamps, sizeof(unsigned long long) * (kStampCap + 1)));
  }
  *out = g->algo;
  return GBO_OK;
}

int ensure_frontier(gbo_graph* g, AlgoState* a, cudaStream_t s) {
  if (!a->front) {
    const size_t wb = 8;  // widest word
    GBO_CUDA_TRY(cudaMalloc(&a->front, wb * 3 * front_stride(g->nbr)));
    GBO_CUDA_TRY(cudaMalloc(&a->visited, wb * (size_t)(g->nbr + 1)));
    GBO_CUDA_TRY(cudaMalloc(&a->live, wb * (size_t)(g->nbr + 1)));
    g->device_bytes += (long long)(wb * (3 * front_stride(g->nbr) + 2 * (g->nbr + 1)));
    GBO_CUDA_TRY(cudaMemsetAsync(a->live, 0, wb * (size_t)(g->nbr + 1), s));
    if (g->nitems > 0 && g->layout == GBO_LAYOUT_COL) {
      const GView v = view_of(g);
      const unsigned grid = blocks_for_warps(g->nitems, kTPB / 32);
      switch (g->b) {
        case 4: k_live_col<4><<<grid, kTPB, 0, s>>>(v, (Word<4>::T*)a->live); break;
        case 8: k_live_col<8><<<grid, kTPB, 0, s>>>(v, (Word<8>::T*)a->live); break;
        case 16: k_live_col<16><<<grid, kTPB, 0, s>>>(v, (Word<16>::T*)a->live); break;
        case 32: k_live_col<32><<<grid, kTPB, 0, s>>>(v, (Word<32>::T*)a->live); break;
        default: k_live_col<64><<<grid, kTPB, 0, s>>>(v, (Word<64>::T*)a->live); break;
      }
      GBO_CUDA_TRY(cudaGetLastError());
    } else if (g->nitems > 0) {
      const GView v = view_of(g);
      const unsigned grid = grid_for_items(g->nitems, g->b);
      switch (g->b) {
        case 4: k_live<4><<<grid, kTPB, 0, s>>>(v, (Word<4>::T*)a->live); break;
        case 8: k_live<8><<<grid, kTPB, 0, s>>>(v, (Word<8>::T*)a->live); break;
        case 16: k_live<16><<<grid, kTPB, 0, s>>>(v, (Word<16>::T*)a->live); break;
        case 32: k_live<32><<<grid, kTPB, 0, s>>>(v, (Word<32>::T*)a->live); break;
        default: k_live<64><<<grid, kTPB, 0, s>>>(v, (Word<64>::T*)a->live); break;
      }
      GBO_CUDA_TRY(cudaGetLastError());
    }
  }
  return GBO_OK;
}

}  // namespace

int live_rows(gbo_graph* g, cudaStream_t s, const void** out) {
  AlgoState* a = nullptr;
  GBO_TRY(get_state(g, &a));
  GBO_TRY(ensure_frontier(g, a, s));
  *out = a->live;
  return GBO_OK;
}

namespace {

int ensure_pr_vectors(gbo_graph* g, AlgoState* a) {
  const size_t n = (size_t)(g->nrows > 0 ? g->nrows : 1);
  if (!a->pr) {
    GBO_CUDA_TRY(cudaMalloc(&a->pr, sizeof(float) * 2 * n));
    g->device_bytes += 8LL * g->nrows;
  }
  if (!a->prs) {
    GBO_CUDA_TRY(cudaMalloc(&a->prs, sizeof(float) * 2 * n));
    g->device_bytes += 8LL * g->nrows;
  }
  return GBO_OK;
}

int ensure_pr_part(gbo_graph* g, AlgoState* a) {
  if (a->pr_part || g->rws_nchunk <= 0) return GBO_OK;
  GBO_CUDA_TRY(cudaMalloc(&a->pr_part, sizeof(double) * (size_t)g->rws_nchunk));
  g->device_bytes += 8LL * g->rws_nchunk;
  return GBO_OK;
}

int ensure_vec_i32(gbo_graph* g, int** p) {
  if (!*p) {
    GBO_CUDA_TRY(cudaMalloc(p, sizeof(int) * (size_t)(g->nrows > 0 ? g->nrows : 1)));
    g->device_bytes += 4LL * g->nrows;
  }
  return GBO_OK;
}

// One loop graph per (graph, algorithm): a conditional WHILE node whose
// body is one iteration of `body`, captured once.  The iteration's closing
// kernel clears the condition when the loop stops (close_iteration), so the
// whole loop runs on the device from one launch: no host round trip per
// iteration and no iterations past the last.
template <typename Body>
int get_exec(AlgoState* a, int id, const void* key, Body body) {
  if (a->exec[id] && a->exec_key[id] == key) return GBO_OK;
  if (a->exec[id]) {
    cudaGraphExecDestroy(a->exec[id]);
    a->exec[id] = nullptr;
  }
  cudaGraph_t graph = nullptr;
  GBO_CUDA_TRY(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle handle;
  cudaError_t e = cudaGraphConditionalHandleCreate(&handle, graph, 1, cudaGraphCondAssignDefault);
  cudaGraphNodeParams p = {};
  p.type = cudaGraphNodeTypeConditional;
  p.conditional.handle = handle;
  p.conditional.type = cudaGraphCondTypeWhile;
  p.conditional.size = 1;
  cudaGraphNode_t node;
  if (e == cudaSuccess) e = cudaGraphAddNode(&node, graph, nullptr, 0, &p);
  if (e == cudaSuccess)
    e = cudaStreamBeginCaptureToGraph(a->cap, p.conditional.phGraph_out[0], nullptr, nullptr, 0,
                                      cudaStreamCaptureModeThreadLocal);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return fail_cuda(e, "loop graph");
  }
  int launches = 0;
  const int st = body(a->cap, 0, &launches);
  cudaGraph_t body_graph = p.conditional.phGraph_out[0];
  e = cudaStreamEndCapture(a->cap, &body_graph);
  if (st != GBO_OK || e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return st != GBO_OK ? st : fail_cuda(e, "cudaStreamEndCapture");
  }
  e = cudaGraphInstantiate(&a->exec[id], graph, 0);
  cudaGraphDestroy(graph);
  if (e != cudaSuccess) return fail_cuda(e, "cudaGraphInstantiate");
  a->exec_key[id] = key;
  a->cond[id] = (unsigned long long)handle;
  a->launches_per_iter = launches;
  return GBO_OK;
}

// Run a loop graph on s (after the algorithm's init kernel).  With `iters`
// the call waits for the loop and returns its iteration count; otherwise it
// returns at once (stream-ordered).  An injected iteration cap that cuts the
// loop returns GBO_ERR_TIMEOUT.
int injected_cap_iters() {
  const long long cap = inject_replay_cap();
  return cap > 0 ? (int)std::min<long long>(cap * kStepsPerGraph, 1 << 30) : 0;
}

// After a loop run was queued: wait for it when the caller wants the
// iteration count or a cap or a barrier skip was injected, and check how it
// ended.
int finish_loop(AlgoState* a, cudaStream_t s, int max_iter, int cap_iters, int* iters, bool coop = false,
                bool must_wait = false) {
  a->replays = 1;
  a->stats_pending = true;
  if (!iters && cap_iters == 0 && !must_wait) return GBO_OK;
  GBO_CUDA_TRY(cudaMemcpyAsync(a->h_ctrl, a->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost, s));
  GBO_CUDA_TRY(cudaStreamSynchronize(s));
  if (coop && a->h_ctrl->bar_err) return fail(GBO_ERR_TIMEOUT, "cooperative BFS: a grid barrier gave up");
  if (!a->h_ctrl->done) return fail(GBO_ERR_TIMEOUT, "iteration loop did not terminate");
  if (cap_iters > 0 && cap_iters < max_iter && a->h_ctrl->iter >= cap_iters)
    return fail(GBO_ERR_TIMEOUT, "iteration loop cut off by the injected cap");
  if (iters) *iters = a->h_ctrl->iter;
  return GBO_OK;
}

int run_until_done(AlgoState* a, int id, cudaStream_t s, int max_iter, int* iters) {
  const int cap_iters = injected_cap_iters();
  k_loop_begin<<<1, 32, 0, s>>>(a->ctrl, a->cond[id], a->stamps, cap_iters);
  GBO_CUDA_TRY(cudaGetLastError());
  GBO_CUDA_TRY(cudaGraphLaunch(a->exec[id], s));
  a->fixed_launches = 2;  // init and loop start kernels
  a->coop_run = false;
  return finish_loop(a, s, max_iter, cap_iters, iters);
}

// Blocks of the cooperative BFS: every block resident at once (the grid
// barrier needs it) and at most kCoopBlocksPerSM per SM -- a barrier costs
// 2.4 us over 148 blocks and 4.0 us over 888 on B200, and R-MAT 22 BFS runs
// fastest at 4-5 blocks per SM -- and about one warp per 4 block rows or 32
// work items; or the caller's choice (gbo_graph_set_bfs_loop) within the
// resident limit.
int coop_grid(const gbo_graph* g, unsigned* grid) {
  int per_sm = 0, coop = 0, dev = 0;
  GBO_CUDA_TRY(cudaGetDevice(&dev));
  GBO_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
  if (!coop) return fail(GBO_ERR_UNSUPPORTED, "device has no cooperative launch");
  GBO_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_bfs_coop, kTPB, 0));
  if (per_sm < 1) return fail(GBO_ERR_UNSUPPORTED, "cooperative BFS kernel does not fit an SM");
  const unsigned cap = (unsigned)num_sms() * (unsigned)per_sm;
  const long long warps = std::max<long long>(((long long)g->nbr + 3) / 4, ((long long)g->nitems + 31) / 32);
  unsigned want = blocks_for_warps(std::max<long long>(warps, 1), kTPB / 32);
  want = std::min(want, (unsigned)num_sms() * (unsigned)kCoopBlocksPerSM);
  if (g->bfs_coop_blocks > 0) want = (unsigned)g->bfs_coop_blocks;
  *grid = want < cap ? want : cap;
  return GBO_OK;
}

// The BFS level loop as one cooperative launch (k_bfs_coop) on s.
int run_bfs_coop(gbo_graph* g, AlgoState* a, const GView& v, unsigned* front, unsigned* vis, int* level,
                 cudaStream_t s, int max_iter, int cap_iters, int* iters) {
  unsigned grid = 0;
  GBO_TRY(coop_grid(g, &grid));
  if (!a->push_list) {
    const size_t nb = sizeof(long long) * 2 * (size_t)std::max(g->rws_nlong, 1);
    GBO_CUDA_TRY(cudaMalloc(&a->push_list, nb));
    g->device_bytes += (long long)nb;
  }
  long long* list = a->push_list;
  GView va = v;
  Ctrl* ctrl = a->ctrl;
  // failure-path test (GBO_INJECT_BARRIER_SKIP): a block that never arrives
  // and a 100 ms limit, so that the others' bounded wait runs out
  const long long skip = take_inject_barrier_skip();
  unsigned long long limit_ns = skip > 0 ? 100000000ull : kBarrierLimitNs;
  int skip_block = skip > 0 ? (int)std::min<long long>(skip - 1, (long long)grid - 1) : -1;
  void* args[] = {&va, &front, &vis, &level, &ctrl, &list, &limit_ns, &skip_block};
  GBO_CUDA_TRY(cudaLaunchCooperativeKernel((const void*)k_bfs_coop, dim3(grid), dim3(kTPB), args, 0, s));
  a->fixed_launches = 2;  // init and the cooperative loop
  a->coop_run = true;
  a->launches_per_iter = 0;
  return finish_loop(a, s, max_iter, cap_iters, iters, true, skip > 0);
}

// Step times and counts of the last loop run, read back on first request.
int collect_stats(AlgoState* a) {
  if (!a->stats_pending) return GBO_OK;
  a->stats_pending = false;
  GBO_CUDA_TRY(cudaDeviceSynchronize());
  GBO_CUDA_TRY(cudaMemcpy(a->h_ctrl, a->ctrl, sizeof(Ctrl), cudaMemcpyDeviceToHost));
  // a stream-ordered cooperative BFS whose grid barrier gave up reports it here
  if (a->coop_run && a->h_ctrl->bar_err) return fail(GBO_ERR_TIMEOUT, "cooperative BFS: a grid barrier gave up");
  const int it = a->h_ctrl->iter;
  const int nst = std::min(it, kStampCap);
  std::vector<unsigned long long> t((size_t)nst + 1);
  GBO_CUDA_TRY(cudaMemcpy(t.data(), a->stamps, sizeof(unsigned long long) * t.size(), cudaMemcpyDeviceToHost));
  a->step_ms.clear();
  for (int q = 0; q < nst; ++q) a->step_ms.push_back((float)((double)(t[(size_t)q + 1] - t[(size_t)q]) * 1e-6));
  a->launches = a->fixed_launches + (long long)it * a->launches_per_iter;
  return GBO_OK;
}

#define ALGO_DISPATCH_B(b, CALL) \
  switch (b) {                  \
    case 4: { constexpr int B = 4; CALL; } break;   \
    case 8: { constexpr int B = 8; CALL; } break;   \
    case 16: { constexpr int B = 16; CALL; } break; \
    case 32: { constexpr int B = 32; CALL; } break; \
    default: { constexpr int B = 64; CALL; } break; \
  }

// src >= 0: one source passed by value; otherwise nseeds seeds from h_seeds.
template <int B>
int bfs_impl(gbo_graph* g, int src, const int* h_seeds, int nseeds, int32_t* d_level, int* h_depth,
             cudaStream_t s) {
  using WT = typename Word<B>::T;
  AlgoState* a = nullptr;
  GBO_TRY(get_state(g, &a));
  GBO_TRY(ensure_frontier(g, a, s));
  GBO_TRY(ensure_vec_i32(g, &a->level));
  GView v = view_of(g);
  WT* front = (WT*)a->front;
  WT* vis = (WT*)a->visited;
  Ctrl* ctrl = a->ctrl;
  WT* scratch = (WT*)a->scratch;
  // the COL tile layout has its own pull and push kernels (column words)
  const bool col = g->layout == GBO_LAYOUT_COL;
  // b = 32 ROW graphs pull over their row-word slices (built on first use)
  if (B == 32 && !col) GBO_TRY(build_rws(g, s));
  const bool rws = B == 32 && !col && g->rws_head != nullptr;
  if (rws) v = view_of(g);
  // the level loop in one cooperative launch (its push list counts rows in
  // 24 bits and tail entries in 40)
  const bool coop = rws && g->nitems > 0 && g->rws_nlong < (1 << 23) && g->rws_ntail < (1ll << 39) &&
                    (g->bfs_loop == GBO_BFS_LOOP_COOP || (g->bfs_loop == GBO_BFS_LOOP_AUTO && kCoopBfsDefault));
  if (g->bfs_loop == GBO_BFS_LOOP_COOP && !rws)
    return fail(GBO_ERR_UNSUPPORTED, "the cooperative BFS loop needs a b = 32 ROW graph");
  // the cooperative loop writes the caller's level array itself; the loop
  // graph (captured once) writes the graph's own and copies it out
  int* level = coop ? d_level : a->level;
  // cooperative loop: the init kernel also starts the step clock and
  // applies an injected iteration cap (no loop-start kernel)
  const int cap_iters = coop ? injected_cap_iters() : 0;
  // the slice pull step finishes every block row itself: no split partials
  GView vfin = v;
  if (rws) vfin.nsplit = 0;
  const unsigned gi = col ? grid_persistent(k_bfs_step_col<B>, g->nitems)
                          : rws ? grid_persistent(k_bfs_pull_rws, ((long long)g->nbr + 31) / 32)
                                : grid_items_persistent(k_bfs_step<B>, g->nitems, B);
  // push steps (symmetric graphs) finalise every block row in k_bfs_finish
  const bool push_ok = g->symmetric;
  const unsigned gs = blocks_for(std::max<long long>(g->nsplit, push_ok ? g->nbr : 0), kTPB);
  const unsigned gp = col ? grid_persistent(k_bfs_push_col<B>, g->nitems) : grid_persistent(k_bfs_push<B>, g->nitems);
  if (!coop) GBO_TRY(get_exec(a, A_BFS, nullptr, [&](cudaStream_t cs, int k, int* nl) -> int {
    if (g->nitems > 0) {
      if (col) k_bfs_step_col<B><<<gi, kTPB, 0, cs>>>(v, front, vis, level, ctrl, scratch);
      else if (rws)
        k_bfs_pull_rws<<<gi, kTPB, 0, cs>>>(v, reinterpret_cast<unsigned*>(front),
                                            reinterpret_cast<unsigned*>(vis), level, ctrl);
      else k_bfs_step<B><<<gi, kTPB, 0, cs>>>(v, front, vis, level, ctrl, scratch);
    }
    if (push_ok && g->nitems > 0) {
      if (col) k_bfs_push_col<B><<<gp, kTPB, 0, cs>>>(v, front, vis, ctrl);
      else k_bfs_push<B><<<gp, kTPB, 0, cs>>>(v, front, vis, ctrl);
    }
    k_bfs_finish<B><<<gs, kTPB, 0, cs>>>(vfin, front, vis, level, ctrl, scratch);
    *nl += (g->nitems > 0) + 1 + (push_ok ? (g->nitems > 0) : 0);
    GBO_CUDA_TRY(cudaGetLastError());
    return GBO_OK;
  }));
  const int max_iter = g->nrows + 1;
  // push while the frontier holds fewer than n/64 vertices (symmetric only)
  const int push_thr = !push_ok ? 0 : g->bfs_push_thr >= 0 ? g->bfs_push_thr : std::max(1, g->nrows / 64);
  const int nstart = src >= 0 ? 1 : nseeds;
  k_bfs_init<B><<<grid_vertex(std::max(g->nrows, g->nbr)), kTPB, 0, s>>>(
      front, vis, level, (const WT*)a->live, g->nbr, g->nrows, src, ctrl, max_iter, push_thr,
      push_ok && nstart < push_thr ? 1 : 0, coop ? a->stamps : nullptr, cap_iters);
  if (src < 0) {
    if (a->nseeds_cap < nseeds) {
      cudaFree(a->seeds);
      a->seeds = nullptr;
      GBO_CUDA_TRY(cudaMalloc(&a->seeds, sizeof(int) * (size_t)nseeds));
      a->nseeds_cap = nseeds;
    }
    GBO_CUDA_TRY(cudaMemcpyAsync(a->seeds, h_seeds, sizeof(int) * (size_t)nseeds,
                                 cudaMemcpyHostToDevice, s));
    k_bfs_seed<B><<<1, 32, 0, s>>>(a->seeds, nseeds, front, vis, level);
  }
  GBO_CUDA_TRY(cudaGetLastError());
  int iters = 0;
  // without h_depth the call is asynchronous: the loop and the level copy
  // are queued on s and the call returns
  if (coop) {
    if constexpr (B == 32)
      GBO_TRY(run_bfs_coop(g, a, v, reinterpret_cast<unsigned*>(front), reinterpret_cast<unsigned*>(vis), level,
                           s, max_iter, cap_iters, h_depth ? &iters : nullptr));
  } else {
    GBO_TRY(run_until_done(a, A_BFS, s, max_iter, h_depth ? &iters : nullptr));
    if (g->nrows > 0)
      GBO_CUDA_TRY(cudaMemcpyAsync(d_level, level, sizeof(int) * (size_t)g->nrows,
                                   cudaMemcpyDeviceToDevice, s));
  }
  if (h_depth) *h_depth = iters;
  return GBO_OK;
}

template <int B>
int sssp_impl(gbo_graph* g, int src, uint32_t* d_dist, int* h_iters, cudaStream_t s) {
  GBO_TRY(bfs_impl<B>(g, src, nullptr, 0, reinterpret_cast<int32_t*>(d_dist), h_iters, s));
  if (g->nrows > 0) k_level_to_dist<<<grid_vertex(g->nrows), kTPB, 0, s>>>(d_dist, g->nrows);
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

// Shared by PageRank (v = NULL) and the PPR forward pass.
template <int B>
int pr_impl(gbo_graph* g, const float* d_v, float alpha, int max_iter, float tol, float* d_p,
            int* h_iters, int norm, float init_const, float init_scale, float add, float add_scale,
            int id, cudaStream_t s) {
  AlgoState* a = nullptr;
  GBO_TRY(get_state(g, &a));
  GBO_TRY(ensure_pr_vectors(g, a));
  GView v = view_of(g);
  float* pr = a->pr;
  float* prs = a->prs;
  const float* inv = g->invdeg;
  Ctrl* ctrl = a->ctrl;
  double* scratch = (double*)a->scratch;
  // b = 32 ROW graphs iterate over their row-word slices (no split rows)
  if (B == 32 && g->layout == GBO_LAYOUT_ROW) GBO_TRY(build_rws(g, s));
  const bool rws = B == 32 && g->layout == GBO_LAYOUT_ROW && g->rws_head != nullptr;
  if (rws) v = view_of(g);
  GView vfin = v;
  if (rws) vfin.nsplit = 0;
  if (rws) GBO_TRY(ensure_pr_part(g, a));
  const unsigned gi = rws ? grid_persistent(k_pr_step_rws, g->nbr)
                          : grid_items_persistent(k_pr_step<B>, g->nitems, B);
  const unsigned gc = rws ? grid_persistent(k_pr_long_chunks, std::max<long long>(g->rws_nchunk, 1)) : 1;
  const unsigned gs = blocks_for((long long)vfin.nsplit * B, kTPB);
  GBO_TRY(get_exec(a, id, d_v, [&](cudaStream_t cs, int k, int* nl) -> int {
    if (g->nitems > 0) {
      if (rws) {
        k_pr_step_rws<<<gi, kTPB, 0, cs>>>(v, pr, prs, inv, d_v, ctrl);
        if (g->rws_nchunk > 0) {
          k_pr_long_chunks<<<gc, kTPB, 0, cs>>>(v, pr, prs, ctrl, a->pr_part);
          k_pr_long_rows<<<blocks_for(g->rws_nlong, kTPB), kTPB, 0, cs>>>(v, pr, prs, inv, d_v, ctrl, a->pr_part);
          *nl += 2;
        }
      } else {
        k_pr_step<B><<<gi, kTPB, 0, cs>>>(v, pr, prs, inv, d_v, ctrl, scratch);
      }
    }
    k_pr_finish<B><<<gs, kTPB, 0, cs>>>(vfin, pr, prs, inv, d_v, ctrl, scratch);
    *nl += (g->nitems > 0) + 1;
    GBO_CUDA_TRY(cudaGetLastError());
    return GBO_OK;
  }));
  k_pr_init<<<grid_vertex(g->nrows), kTPB, 0, s>>>(pr, prs, inv, d_v, g->nrows, init_const, init_scale,
                                                  ctrl, max_iter, tol, alpha, add, add_scale, norm, 0);
  GBO_CUDA_TRY(cudaGetLastError());
  int iters = 0;
  if (max_iter > 0) GBO_TRY(run_until_done(a, id, s, max_iter, &iters));
  if (g->nrows > 0)
    GBO_CUDA_TRY(cudaMemcpyAsync(d_p, pr + (size_t)(iters & 1) * g->nrows,
                                 sizeof(float) * (size_t)g->nrows, cudaMemcpyDeviceToDevice, s));
  if (h_iters) *h_iters = iters;
  return GBO_OK;
}

template <int B>
int ppr_backward_impl(gbo_graph* g, const float* d_w, float alpha, float tol, int max_iter,
                      float* d_grad, int* h_iters, cudaStream_t s) {
  AlgoState* a = nullptr;
  GBO_TRY(get_state(g, &a));
  GBO_TRY(ensure_pr_vectors(g, a));
  const int n = g->nrows;
  const unsigned gv = grid_vertex(n);
  int iters = 0;
  if (g->symmetric) {
    // P^T = P: u' = w + alpha * D^-1 P u is a gather over P's rows (the
    // PageRank step with the scale on rows), no scatter atomics
    float* pr = a->pr;
    float* prs = a->prs;
    const float* inv = g->invdeg;
    Ctrl* ctrl = a->ctrl;
    double* scratch = (double*)a->scratch;
    if (B == 32 && g->layout == GBO_LAYOUT_ROW) GBO_TRY(build_rws(g, s));
    const bool rws = B == 32 && g->layout == GBO_LAYOUT_ROW && g->rws_head != nullptr;
    GView v = view_of(g);
    GView vfin = v;
    if (rws) vfin.nsplit = 0;
    if (rws) GBO_TRY(ensure_pr_part(g, a));
    const unsigned gi = rws ? grid_persistent(k_pr_step_rws, g->nbr)
                            : grid_items_persistent(k_pr_step<B>, g->nitems, B);
    const unsigned gc = rws ? grid_persistent(k_pr_long_chunks, std::max<long long>(g->rws_nchunk, 1)) : 1;
    const unsigned gs = blocks_for((long long)vfin.nsplit * B, kTPB);
    GBO_TRY(get_exec(a, A_PPR_BG, d_w, [&](cudaStream_t cs, int k, int* nl) -> int {
      if (g->nitems > 0) {
        if (rws) {
          k_pr_step_rws<<<gi, kTPB, 0, cs>>>(v, pr, prs, inv, d_w, ctrl);
          if (g->rws_nchunk > 0) {
            k_pr_long_chunks<<<gc, kTPB, 0, cs>>>(v, pr, prs, ctrl, a->pr_part);
            k_pr_long_rows<<<blocks_for(g->rws_nlong, kTPB), kTPB, 0, cs>>>(v, pr, prs, inv, d_w, ctrl, a->pr_part);
            *nl += 2;
          }
        } else {
          k_pr_step<B><<<gi, kTPB, 0, cs>>>(v, pr, prs, inv, d_w, ctrl, scratch);
        }
      }
      k_pr_finish<B><<<gs, kTPB, 0, cs>>>(vfin, pr, prs, inv, d_w, ctrl, scratch);
      *nl += (g->nitems > 0) + 1;
      GBO_CUDA_TRY(cudaGetLastError());
      return GBO_OK;
    }));
    // u0 = w; y = w + alpha * inv * (P u)
    k_pr_init<<<gv, kTPB, 0, s>>>(pr, nullptr, nullptr, d_w, n, 0.f, 1.f, ctrl, max_iter, tol, alpha,
                                  0.f, 1.f, 1, 1);
    k_l1_ref<<<gv, kTPB, 0, s>>>(d_w, n, ctrl);
    GBO_CUDA_TRY(cudaGetLastError());
    if (max_iter > 0) GBO_TRY(run_until_done(a, A_PPR_BG, s, max_iter, &iters));
    if (n > 0) k_scale_copy<<<gv, kTPB, 0, s>>>(pr + (size_t)(iters & 1) * n, d_grad, n, 1.f - alpha);
    GBO_CUDA_TRY(cudaGetLastError());
    if (h_iters) *h_iters = iters;
    return GBO_OK;
  }
  if (!a->acc64) {
    GBO_CUDA_TRY(cudaMalloc(&a->acc64, sizeof(double) * (size_t)(g->nrows > 0 ? g->nrows : 1)));
    g->device_bytes += 8LL * g->nrows;
  }
  GView v = view_of(g);
  float* pr = a->pr;
  double* acc = a->acc64;
  const float* inv = g->invdeg;
  Ctrl* ctrl = a->ctrl;
  const unsigned gi = grid_items_persistent(k_adj_scatter<B>, g->nitems, B);
  GBO_TRY(get_exec(a, A_PPR_B, d_w, [&](cudaStream_t cs, int k, int* nl) -> int {
    k_adj_prep<<<gv, kTPB, 0, cs>>>(pr, d_w, n, ctrl, acc);
    if (g->nitems > 0) k_adj_scatter<B><<<gi, kTPB, 0, cs>>>(v, pr, ctrl, acc);
    k_adj_apply<<<gv, kTPB, 0, cs>>>(pr, d_w, inv, n, ctrl, acc);
    *nl += (g->nitems > 0) + 2;
    GBO_CUDA_TRY(cudaGetLastError());
    return GBO_OK;
  }));
  // u0 = w
  k_pr_init<<<gv, kTPB, 0, s>>>(pr, nullptr, nullptr, d_w, n, 0.f, 1.f, ctrl, max_iter, tol, alpha, 0.f,
                                0.f, 1, 0);
  k_l1_ref<<<gv, kTPB, 0, s>>>(d_w, n, ctrl);
  GBO_CUDA_TRY(cudaGetLastError());
  if (max_iter > 0) GBO_TRY(run_until_done(a, A_PPR_B, s, max_iter, &iters));
  if (n > 0) k_scale_copy<<<gv, kTPB, 0, s>>>(pr + (size_t)(iters & 1) * n, d_grad, n, 1.f - alpha);
  GBO_CUDA_TRY(cudaGetLastError());
  if (h_iters) *h_iters = iters;
  return GBO_OK;
}

template <int B>
int cc_impl(gbo_graph* g, int32_t* d_label, int* h_iters, cudaStream_t s) {
  AlgoState* a = nullptr;
  GBO_TRY(get_state(g, &a));
  GBO_TRY(ensure_vec_i32(g, &a->f));
  GBO_TRY(ensure_vec_i32(g, &a->gf));
  GBO_TRY(ensure_vec_i32(g, &a->mngf));
  GView v = view_of(g);
  int *f = a->f, *gf = a->gf, *mngf = a->mngf;
  Ctrl* ctrl = a->ctrl;
  int* scratch = (int*)a->scratch;
  const int n = g->nrows;
  // 32x32 ROW graphs take the neighbours' minimum over their row-word slices
  if (B == 32 && g->layout == GBO_LAYOUT_ROW) GBO_TRY(build_rws(g, s));
  const bool rws = B == 32 && g->layout == GBO_LAYOUT_ROW && g->rws_head != nullptr;
  if (rws) v = view_of(g);
  const unsigned gi = rws ? grid_persistent(k_cc_mngf_rws, g->nbr) : grid_items_persistent(k_cc_mngf<B>, g->nitems, B);
  const unsigned gc = rws && g->rws_nchunk > 0 ? grid_persistent(k_cc_mngf_chunks, g->rws_nchunk) : 0u;
  const unsigned gs = blocks_for((long long)g->nsplit * B, kTPB);
  const unsigned gv = grid_vertex(n);
  GBO_TRY(get_exec(a, A_CC, nullptr, [&](cudaStream_t cs, int k, int* nl) -> int {
    if (rws) {
      if (g->nitems > 0) k_cc_mngf_rws<<<gi, kTPB, 0, cs>>>(v, gf, mngf, ctrl);
      if (gc > 0) k_cc_mngf_chunks<<<gc, kTPB, 0, cs>>>(v, gf, mngf, ctrl);
      *nl += (g->nitems > 0) + (gc > 0) + 3;
    } else {
      if (g->nitems > 0) k_cc_mngf<B><<<gi, kTPB, 0, cs>>>(v, gf, mngf, ctrl, scratch);
      *nl += (g->nitems > 0) + (g->nsplit > 0) + 3;
      if (g->nsplit > 0) k_cc_mngf_finish<B><<<gs, kTPB, 0, cs>>>(v, mngf, ctrl, scratch);
    }
    k_cc_hook<<<gv, kTPB, 0, cs>>>(f, mngf, n, ctrl);
    k_cc_shortcut<<<gv, kTPB, 0, cs>>>(f, mngf, gf, n, ctrl);
    k_cc_grand<<<gv, kTPB, 0, cs>>>(f, gf, n, ctrl);
    GBO_CUDA_TRY(cudaGetLastError());
    return GBO_OK;
  }));
  const int max_iter = n + 2;
  k_cc_init<<<gv, kTPB, 0, s>>>(f, gf, mngf, n, ctrl, max_iter);
  GBO_CUDA_TRY(cudaGetLastError());
  GBO_TRY(run_until_done(a, A_CC, s, max_iter, h_iters));
  if (n > 0)
    GBO_CUDA_TRY(cudaMemcpyAsync(d_label, f, sizeof(int) * (size_t)n, cudaMemcpyDeviceToDevice, s));
  return GBO_OK;
}

// ------------------------------------------------ block-row shards (BFS)
// One pull level over a shard -- the block rows of some of the vertices,
// every column -- against the whole graph's frontier words x: the shard's
// next-frontier words, visited words and levels.  A work group per item;
// split rows leave their words in scratch slots for k_bfs_shard_finish.
template <int B>
__global__ void __launch_bounds__(kTPB) k_bfs_shard_step(GView v, const typename Word<B>::T* __restrict__ x,
                                                         typename Word<B>::T* __restrict__ visited,
                                                         int* __restrict__ level, int lvl,
                                                         typename Word<B>::T* __restrict__ out,
                                                         typename Word<B>::T* __restrict__ scratch,
                                                         unsigned long long* __restrict__ count) {
  using WT = typename Word<B>::T;
  using L = Lay<B>;
  const unsigned lane = threadIdx.x & 31;
  const int r = lane % L::W;
  const WT full = full_word<B>();
  const long long item = item_index(lane, L::W, L::G);
  const bool active = item < v.nitems;
  const gbo_item it = active ? v.items[item] : gbo_item{0, 0, 0, -2};
  const WT vis = active ? visited[it.row] : full;
  bool p0 = false, p1 = false;
  if (active && (vis & full) != full) {  // uniform inside the item's lane group
    const long long row0 = (long long)it.row * B + r;
    const bool need0 = !bit_of<B>(vis, r) && row0 < v.nrows;
    const bool need1 = L::RPL == 2 && !bit_of<B>(vis, r + 32) && row0 + 32 < v.nrows;
    pull_or_scan<B>(v, it.t0, it.t1, x, need0, need1, p0, p1, lane);
  }
  const WT word = gather_bits<B>(p0, p1, lane);
  unsigned long long cnt = 0;
  if (active) {
    if (it.slot >= 0) {
      if (r == 0) scratch[it.slot] = word;
    } else {
      const WT nw = (WT)(word & ~vis & full);
      const long long row0 = (long long)it.row * B + r;
      if (bit_of<B>(nw, r) && row0 < v.nrows) level[row0] = lvl + 1;
      if (L::RPL == 2 && bit_of<B>(nw, r + 32) && row0 + 32 < v.nrows) level[row0 + 32] = lvl + 1;
      if (r == 0) {
        out[it.row] = nw;
        if (nw) visited[it.row] = (WT)(vis | nw);
        cnt = popc_w(nw);
      }
    }
  }
  block_add_u64(cnt, count);
}

template <int B>
__global__ void k_bfs_shard_finish(GView v, typename Word<B>::T* __restrict__ visited, int* __restrict__ level,
                                   int lvl, typename Word<B>::T* __restrict__ out,
                                   const typename Word<B>::T* __restrict__ scratch,
                                   unsigned long long* __restrict__ count) {
  using WT = typename Word<B>::T;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  unsigned long long cnt = 0;
  if (i < v.nsplit) {
    const gbo_split sp = v.splits[i];
    const WT full = full_word<B>();
    const WT vis = visited[sp.row];
    WT w = 0;
    if ((vis & full) != full)
      for (int q = 0; q < sp.nslots; ++q) w |= scratch[sp.slot0 + q];
    const WT nw = (WT)(w & ~vis & full);
    out[sp.row] = nw;
    if (nw) {
      visited[sp.row] = (WT)(vis | nw);
      for (int rr = 0; rr < B; ++rr) {
        const long long row = (long long)sp.row * B + rr;
        if (bit_of<B>(nw, rr) && row < v.nrows) level[row] = lvl + 1;
      }
      cnt = popc_w(nw);
    }
  }
  block_add_u64(cnt, count);
}

template <int B>
int bfs_shard_level_impl(gbo_graph* g, const void* x, void* visited, int32_t* level, int lvl, void* out,
                         uint64_t* h_count, cudaStream_t s) {
  using WT = typename Word<B>::T;
  AlgoState* a = nullptr;
  GBO_TRY(get_state(g, &a));
  unsigned long long* cnt = &a->ctrl->count;
  GBO_CUDA_TRY(cudaMemsetAsync(cnt, 0, sizeof(unsigned long long), s));
  const GView v = view_of(g);
  auto* scratch = static_cast<WT*>(g->ws);  // split-row words (one per slot)
  if (g->nitems > 0)
    k_bfs_shard_step<B><<<blocks_for_warps((g->nitems + Lay<B>::G - 1) / Lay<B>::G, kTPB / 32), kTPB, 0, s>>>(
        v, static_cast<const WT*>(x), static_cast<WT*>(visited), level, lvl, static_cast<WT*>(out), scratch, cnt);
  if (g->nsplit > 0)
    k_bfs_shard_finish<B><<<blocks_for(g->nsplit, kTPB), kTPB, 0, s>>>(v, static_cast<WT*>(visited), level, lvl,
                                                                      static_cast<WT*>(out), scratch, cnt);
  GBO_CUDA_TRY(cudaGetLastError());
  if (h_count) {
    unsigned long long h = 0;
    GBO_CUDA_TRY(cudaMemcpyAsync(&h, cnt, sizeof(h), cudaMemcpyDeviceToHost, s));
    GBO_CUDA_TRY(cudaStreamSynchronize(s));
    *h_count = h;
  }
  return GBO_OK;
}

int check_algo_graph(const gbo_graph* g, bool col_ok = false) {
  if (!g) return fail(GBO_ERR_INVALID, "graph is NULL");
  if (g->layout != GBO_LAYOUT_ROW && !col_ok)
    return fail(GBO_ERR_UNSUPPORTED, "this algorithm needs the ROW tile layout (BFS and SSSP also take COL)");
  if (g->nrows != g->ncols) return fail(GBO_ERR_INVALID, "algorithms need a square matrix");
  return GBO_OK;
}

}  // namespace

void free_algo_state(gbo_graph* g) {
  AlgoState* a = g->algo;
  if (!a) return;
  for (auto& e : a->exec)
    if (e) cudaGraphExecDestroy(e);
  cudaFree(a->stamps);
  cudaFree(a->ctrl);
  cudaFreeHost(a->h_ctrl);
  cudaFree(a->front);
  cudaFree(a->visited);
  cudaFree(a->live);
  cudaFree(a->level);
  cudaFree(a->dist);
  cudaFree(a->pr);
  cudaFree(a->prs);
  cudaFree(a->f);
  cudaFree(a->gf);
  cudaFree(a->mngf);
  cudaFree(a->acc64);
  cudaFree(a->pr_part);
  cudaFree(a->push_list);
  cudaFree(a->seeds);
  cudaFree(a->scratch);
  if (a->cap) cudaStreamDestroy(a->cap);
  delete a;
  g->algo = nullptr;
}

}  // namespace gbo

using namespace gbo;

extern "C" int gbo_bfs(const gbo_graph* gc, int src, int32_t* d_level, int* h_depth,
                       gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_algo_graph(gc, true));
  gbo_graph* g = const_cast<gbo_graph*>(gc);
  if (src < 0 || src >= g->nrows) return fail(GBO_ERR_INVALID, "source vertex out of range");
  if (!d_level) return fail(GBO_ERR_INVALID, "level is NULL");
  int st = GBO_OK;
  ALGO_DISPATCH_B(g->b, st = bfs_impl<B>(g, src, nullptr, 0, d_level, h_depth, as_stream(stream)));
  return st;
}

namespace gbo {
int bfs_seeded(gbo_graph* g, const int* h_seeds, int nseeds, int32_t* d_level, int* h_depth,
               cudaStream_t s) {
  int st = GBO_OK;
  ALGO_DISPATCH_B(g->b, st = bfs_impl<B>(g, -1, h_seeds, nseeds, d_level, h_depth, s));
  return st;
}
}  // namespace gbo

extern "C" int gbo_sssp_unit(const gbo_graph* gc, int src, uint32_t* d_dist, int* h_iters,
                             gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_algo_graph(gc, true));
  gbo_graph* g = const_cast<gbo_graph*>(gc);
  if (src < 0 || src >= g->nrows) return fail(GBO_ERR_INVALID, "source vertex out of range");
  if (!d_dist) return fail(GBO_ERR_INVALID, "dist is NULL");
  int st = GBO_OK;
  ALGO_DISPATCH_B(g->b, st = sssp_impl<B>(g, src, d_dist, h_iters, as_stream(stream)));
  return st;
}

extern "C" int gbo_pagerank(const gbo_graph* gc, float alpha, int max_iter, float tol, float* d_p,
                            int* h_iters, gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_algo_graph(gc));
  gbo_graph* g = const_cast<gbo_graph*>(gc);
  if (!g->invdeg) return fail(GBO_ERR_INVALID, "graph has no out-degrees (wrapped without d_outdeg)");
  if (!d_p && g->nrows > 0) return fail(GBO_ERR_INVALID, "p is NULL");
  if (max_iter < 0) return fail(GBO_ERR_INVALID, "max_iter < 0");
  const float n = (float)(g->nrows > 0 ? g->nrows : 1);
  int st = GBO_OK;
  ALGO_DISPATCH_B(g->b, st = pr_impl<B>(g, nullptr, alpha, max_iter, tol, d_p, h_iters, 2, 1.0f / n,
                                         0.f, (1.0f - alpha) / n, 0.f, A_PR, as_stream(stream)));
  return st;
}

extern "C" int gbo_cc(const gbo_graph* gc, int32_t* d_label, int* h_iters, gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_algo_graph(gc));
  gbo_graph* g = const_cast<gbo_graph*>(gc);
  if (!d_label && g->nrows > 0) return fail(GBO_ERR_INVALID, "label is NULL");
  int st = GBO_OK;
  ALGO_DISPATCH_B(g->b, st = cc_impl<B>(g, d_label, h_iters, as_stream(stream)));
  return st;
}

extern "C" int gbo_ppr_forward(const gbo_graph* gc, const float* d_v, float alpha, float tol,
                               int max_iter, float* d_p, int* h_iters, gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_algo_graph(gc));
  gbo_graph* g = const_cast<gbo_graph*>(gc);
  if (!g->invdeg) return fail(GBO_ERR_INVALID, "graph has no out-degrees");
  if (g->nrows > 0 && (!d_v || !d_p)) return fail(GBO_ERR_INVALID, "NULL vector");
  if (max_iter < 0) return fail(GBO_ERR_INVALID, "max_iter < 0");
  int st = GBO_OK;
  // p0 = (1-alpha) v;  p' = alpha P D^-1 p + (1-alpha) v
  ALGO_DISPATCH_B(g->b, st = pr_impl<B>(g, d_v, alpha, max_iter, tol, d_p, h_iters, 1, 0.f,
                                         1.f - alpha, 0.f, 1.f - alpha, A_PPR_F, as_stream(stream)));
  return st;
}

extern "C" int gbo_ppr_backward(const gbo_graph* gc, const float* d_w, float alpha, float tol,
                                int max_iter, float* d_grad_v, int* h_iters, gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_algo_graph(gc));
  gbo_graph* g = const_cast<gbo_graph*>(gc);
  if (!g->invdeg) return fail(GBO_ERR_INVALID, "graph has no out-degrees");
  if (g->nrows > 0 && (!d_w || !d_grad_v)) return fail(GBO_ERR_INVALID, "NULL vector");
  if (max_iter < 0) return fail(GBO_ERR_INVALID, "max_iter < 0");
  int st = GBO_OK;
  ALGO_DISPATCH_B(g->b, st = ppr_backward_impl<B>(g, d_w, alpha, tol, max_iter, d_grad_v, h_iters,
                                                  as_stream(stream)));
  return st;
}

extern "C" int gbo_graph_last_run(const gbo_graph* g, gbo_run_stats* stats) {
  clear_error();
  if (!g || !stats) return fail(GBO_ERR_INVALID, "NULL argument");
  memset(stats, 0, sizeof(*stats));
  if (g->last_run_ms) return ms_last_run(g, stats);
  AlgoState* a = g->algo;
  if (!a) return GBO_OK;
  GBO_TRY(collect_stats(a));
  stats->iterations = a->h_ctrl ? a->h_ctrl->iter : 0;
  stats->graph_replays = a->replays;
  stats->kernel_launches = a->launches;
  const int n = (int)a->step_ms.size();
  stats->nsteps = n < GBO_MAX_STEP_TIMES ? n : GBO_MAX_STEP_TIMES;
  for (int i = 0; i < stats->nsteps; ++i) stats->step_ms[i] = a->step_ms[(size_t)i];
  return GBO_OK;
}

extern "C" int gbo_bfs_shard_level(const gbo_graph* shard, const void* d_front, void* d_visited,
                                   int32_t* d_level, int level, void* d_next, uint64_t* h_count,
                                   gbo_stream_t stream) {
  clear_error();
  if (!shard) return fail(GBO_ERR_INVALID, "graph is NULL");
  if (shard->layout != GBO_LAYOUT_ROW) return fail(GBO_ERR_UNSUPPORTED, "a BFS shard needs the ROW tile layout");
  if ((shard->nrows > 0 && (!d_visited || !d_level || !d_next)) || (shard->ncols > 0 && !d_front) || level < 0)
    return fail(GBO_ERR_INVALID, "gbo_bfs_shard_level: bad argument");
  gbo_graph* g = const_cast<gbo_graph*>(shard);
  cudaStream_t s = as_stream(stream);
  switch (g->b) {
    case 4: return bfs_shard_level_impl<4>(g, d_front, d_visited, d_level, level, d_next, h_count, s);
    case 8: return bfs_shard_level_impl<8>(g, d_front, d_visited, d_level, level, d_next, h_count, s);
    case 16: return bfs_shard_level_impl<16>(g, d_front, d_visited, d_level, level, d_next, h_count, s);
    case 32: return bfs_shard_level_impl<32>(g, d_front, d_visited, d_level, level, d_next, h_count, s);
    default: return bfs_shard_level_impl<64>(g, d_front, d_visited, d_level, level, d_next, h_count, s);
  }
}
