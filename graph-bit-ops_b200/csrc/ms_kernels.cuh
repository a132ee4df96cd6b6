// Device code of the multi-source (bit frontier matrix) BFS, shared by the
// batched API (msbfs.cu) and the query server (server.cu).
//
// State for k sources, KW = k/32 words per vertex (vertex-major):
//   F[2][n*KW]  frontier rows (double-buffered by level parity); a row is
//               valid only where its frontier bit (fbits) is set
//   V[n*KW]     visited rows
//   fbits[2][nbr+1]  per-vertex "frontier row non-empty" bits, b=32 word per
//               block row, row r at bit 31-r (the B2SR vector layout)
//   vfull[nbr]  per-vertex "all k sources visited" bits (padding rows set)
//   levels[n*k] hops per (vertex, source), -1 unreachable
// A level is the OR.AND product of the B2SR matrix with the frontier matrix.
// One warp per work item; only tiles whose block column has frontier rows,
// only set bits whose frontier row is non-empty, and only tile rows that are
// not fully visited are touched.  The epilogue writes new frontier rows,
// visited rows, levels and both bit vectors.
#pragma once

#include "scan.cuh"

namespace gbo {
namespace ms {

// Per-split-row accumulators (nsplit x 32 x kw words, zeroed) and the split
// index of every slot, for the step/finish kernels (msbfs.cu).
int split_state(const gbo_graph* g, int kw, uint32_t** acc, int** slot_split, cudaStream_t s);

constexpr int kTPB = 256;
constexpr int kWarps = kTPB / 32;

struct Args {
  GView v;
  uint32_t* F;
  size_t fstride;
  uint32_t* V;
  uint32_t* fbits;  // 2 * (nbr + 1)
  uint32_t* vfull;  // nbr + 1
  int* levels;
  int k;
  int* ctl;  // iter, done, ticket, max_iter, count (u64 at ctl + 4)
  uint32_t* split_acc;     // per split block row: 32 x KW words OR-ed by its items, zero
                           // between levels (the finish kernel reads and clears them)
  const int* slot_split;   // split index of every work item's slot
  uint32_t* slot_any;  // optional: OR of the new bits of every source word
  const uint32_t* live;  // optional: rows of P with an entry (others can never be reached)
  uint32_t* active;  // optional: source columns still traversing (kw words); a row
                     // counts as finished once every active column reached it
  // with retire set (and active, slot_any), the level close drops the
  // columns that found no new vertex in the level (active &= slot_any) and
  // clears slot_any: a source whose traversal ended (an isolated source, or
  // one whose component is exhausted) no longer keeps every row open
  int retire = 0;
  int level_group;     // 0: levels[i*k + s]; g > 0: levels[((s/g)*n + i)*g + s%g]
  // Direction-optimising levels (symmetric graphs): with dir set, a level
  // whose frontier holds fewer than push_thr (vertex, source) pairs runs as
  // a push (k_push scatters frontier rows into push_acc, nbr x 32 x KW words,
  // zero between levels; k_push_fin finalises every block row).  ctl[6] is
  // the current level's mode (1 push), ctl[7] is set once a push level has
  // closed in the current slot of the captured graph, so that the pull
  // kernels of the slot leave it alone.
  int dir = 0;
  long long push_thr = 0;
  uint32_t* push_acc = nullptr;
  // row-word slice steps: the frontier rows gathered from the tails of long
  // rows (rws_nlong x KW words, zero between levels; k_long_chunks ORs into
  // them, k_step_rws reads them, a memset after the step clears them)
  uint32_t* long_acc = nullptr;
};

// Address of the level of (vertex i, source s) in either layout.
__device__ __forceinline__ size_t level_index(const Args& a, long long i, int s) {
  if (a.level_group == 0) return (size_t)i * a.k + s;
  const int g = a.level_group;
  return ((size_t)(s / g) * a.v.nrows + i) * g + s % g;
}

// Bits of word w that are real sources (k need not be a multiple of 32).
__device__ __forceinline__ unsigned src_mask(int w, int k) {
  const int lo = w * 32;
  if (k >= lo + 32) return 0xffffffffu;
  if (k <= lo) return 0u;
  return (1u << (k - lo)) - 1u;
}

// Epilogue of one block row R: acc(r, w) is the OR of the frontier rows of
// row r's neighbours (word w), read through `get`.  Lane = (slot s, word w).
template <int KW, typename Get>
__device__ __forceinline__ void block_row_epilogue(const Args& a, int R, int lvl, uint32_t vrow,
                                                   unsigned lane, Get get,
                                                   unsigned long long& cnt) {
  constexpr int S = 32 / KW;
  const int w = lane % KW;
  const int s = lane / KW;
  const unsigned wmask = seg_mask<KW>();
  uint32_t* Fn = a.F + (size_t)((lvl + 1) & 1) * a.fstride;
  uint32_t fword = 0, vword = vrow, anyw = 0;
  const uint32_t need = src_mask(w, a.k) & (a.active ? a.active[w] : 0xffffffffu);
  for (int rr = 0; rr < 32; rr += S) {
    const int r = rr + s;
    const int i = R * 32 + r;
    const bool open = !((vrow >> (31 - r)) & 1u);  // padding rows are marked full
    uint32_t nw = 0, vn = 0;
    size_t o = 0;
    if (open) {
      o = (size_t)i * KW + w;
      const uint32_t vo = a.V[o];
      nw = get(r, w) & ~vo & src_mask(w, a.k);
      vn = vo | nw;
    }
    const unsigned bnew = __ballot_sync(0xffffffffu, nw != 0);
    const unsigned bfull = __ballot_sync(0xffffffffu, !open || (vn & need) == need);
    const bool rowany = ((bnew >> (s * KW)) & wmask) != 0;
    if (open && rowany) Fn[o] = nw;  // only rows marked in fbits are ever read
    if (nw) {
      a.V[o] = vn;
      cnt += __popc(nw);
      anyw |= nw;
    }
    // levels of the pass's new (vertex, source) pairs: in step t every lane
    // takes one bit of lane t's word (row rr + t / KW, word t % KW), so
    // consecutive lanes write consecutive sources of one vertex
    for (int t = 0; t < 32; ++t) {
      const uint32_t wt = __shfl_sync(0xffffffffu, nw, t);
      if (!wt) continue;
      if ((wt >> lane) & 1u)
        a.levels[level_index(a, (long long)R * 32 + rr + t / KW, (t % KW) * 32 + (int)lane)] = lvl + 1;
    }
#pragma unroll
    for (int q = 0; q < S; ++q) {
      const unsigned rowbit = 1u << (31 - (rr + q));
      if ((bnew >> (q * KW)) & wmask) fword |= rowbit;
      if (((bfull >> (q * KW)) & wmask) == wmask) vword |= rowbit;
    }
  }
  if (lane == 0) {
    a.fbits[(size_t)((lvl + 1) & 1) * (a.v.nbr + 1) + R] = fword;
    a.vfull[R] = vword;
  }
  if (a.slot_any) {
    // the block row's new bits per source word (lanes w, w + KW, ... hold
    // word w), added only where the word does not have them yet: most
    // columns are marked early in a level, so few atomics reach one address
#pragma unroll
    for (int o = KW; o < 32; o <<= 1) anyw |= __shfl_xor_sync(0xffffffffu, anyw, o);
    if (s == 0 && anyw) {
      const uint32_t cur = __ldcg(a.slot_any + w);
      if (anyw & ~cur) atomicOr(a.slot_any + w, anyw);
    }
  }
}

// Bit pairs (tile row r, frontier vertex j) queued per warp before their
// frontier rows are gathered: S pairs per round, U rounds in flight.
constexpr int kList = 192;

template <int KW>
__global__ void __launch_bounds__(kTPB, KW <= 2 ? 6 : 4) k_step(Args a) {
  constexpr int S = 32 / KW;
  constexpr int U = S >= 64 ? 1 : (64 / S > 8 ? 8 : 64 / S);  // gathers in flight: S*U pairs
  __shared__ uint32_t acc_sh[kWarps][32 * KW];
  __shared__ int2 list_sh[kWarps][kList];
  __shared__ unsigned long long cnt_sh;
  __shared__ int arrived_sh;
  volatile int* c = a.ctl;
  if (c[1]) return;  // done (the same for every block)
  if (a.dir && (c[7] || c[6] == 1)) return;  // this slot's level ran as a push
  if (threadIdx.x == 0) {
    cnt_sh = 0ull;
    arrived_sh = 0;
  }
  __syncthreads();
  const int lvl = c[0];
  const GView& v = a.v;
  const uint32_t* __restrict__ F = a.F + (size_t)(lvl & 1) * a.fstride;
  const uint32_t* __restrict__ fb = a.fbits + (size_t)(lvl & 1) * (v.nbr + 1);
  const unsigned lane = threadIdx.x & 31;
  const int wib = threadIdx.x >> 5;
  const long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  uint32_t* acc = acc_sh[wib];
  const int w = lane % KW;
  const int s = lane / KW;
  unsigned long long cnt = 0;
  if (item < v.nitems) {
    const gbo_item it = v.items[item];
    const uint32_t vrow = a.vfull[it.row];
    if (vrow != 0xffffffffu) {
      for (int q = lane; q < 32 * KW; q += 32) acc[q] = 0u;
      __syncwarp();
      const bool row_open = !((vrow >> (31 - lane)) & 1u);  // lane r: row r still open
      const uint32_t* __restrict__ val = reinterpret_cast<const uint32_t*>(v.val);
      int2* list = list_sh[wib];
      int nlist = 0;  // warp-uniform
      // gather the queued frontier rows, S pairs per round, U rounds in flight
      auto flush = [&]() {
        __syncwarp();
        for (int base = 0; base < nlist; base += S * U) {
          uint32_t f[U];
          int rr[U];
#pragma unroll
          for (int u = 0; u < U; ++u) {
            const int e = base + s + S * u;
            rr[u] = -1;
            f[u] = 0;
            if (e < nlist) {
              const int2 ent = list[e];
              rr[u] = ent.x;
              f[u] = F[(size_t)ent.y * KW + w];
            }
          }
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (rr[u] >= 0 && f[u]) atomicOr(acc + rr[u] * KW + w, f[u]);
        }
        nlist = 0;
        __syncwarp();
      };
      // Per batch of 32 tiles (lane j: tile j) the row words worth a load
      // are the pairs (tile j, row r) with frontier columns at j and row r
      // open and non-empty in tile j (all open rows without occupancy
      // words).  They are dealt out to the lanes, 32 per round: lane p takes
      // pair p (its tile by a binary search over the lanes' prefix counts,
      // its row as the k-th candidate bit), loads the word and ANDs it with
      // the tile's frontier columns.  Each set bit (row r, frontier vertex)
      // then goes to the list, at most kPerPass per lane per pass, at
      // positions from a warp prefix sum (the OR accumulation does not
      // depend on the order).
      constexpr int kPerPass = kList / 32;
      const unsigned* __restrict__ rm = v.rowmask;
      // packed non-empty row words (32x32 ROW graphs): the words a batch
      // loads sit together instead of one per 32-byte sector
      const unsigned* __restrict__ words = v.rowword;
      long long wb = words ? v.item_wbase[item] : 0ll;
      const unsigned openm = __ballot_sync(0xffffffffu, row_open);
      // one batch of 32 tiles from b0: lane j holds tile b0+j's block
      // column cb, occupancy word mw and frontier word fw
      auto batch = [&](int b0, int cb, uint32_t mw, uint32_t fw) {
        const unsigned cand = fw ? (mw & openm) : 0u;
        const int cnt = __popc(cand);
        const int total = (int)__reduce_add_sync(0xffffffffu, (unsigned)cnt);
        const long long wbat = wb;
        const int mc = words ? __popc(mw) : 0;
        if (words) wb += (long long)__reduce_add_sync(0xffffffffu, (unsigned)mc);
        if (total == 0) return;
        const int woff = words ? warp_incl_sum(mc, lane) - mc : 0;  // lane j: tile j's first word
        const int incl = warp_incl_sum(cnt, lane);
        const int excl = incl - cnt;
        for (int pb = 0; pb < total; pb += 32) {
          const int p = pb + (int)lane;
          int j = 0;
#pragma unroll
          for (int st = 16; st > 0; st >>= 1) {
            const int q = __shfl_sync(0xffffffffu, incl, j + st - 1);
            if (q <= p) j += st;
          }
          const int ej = __shfl_sync(0xffffffffu, excl, j);
          const unsigned cj = __shfl_sync(0xffffffffu, cand, j);
          const uint32_t fj = __shfl_sync(0xffffffffu, fw, j);
          const int vbase = __shfl_sync(0xffffffffu, cb, j) * 32;
          const unsigned mj = __shfl_sync(0xffffffffu, mw, j);
          const int oj = __shfl_sync(0xffffffffu, woff, j);
          int r = 0;
          uint32_t eff = 0u;
          if (p < total) {
            r = (int)__fns(cj, 0, p - ej + 1);
            eff = (words ? words[rowword_index(wbat + oj, mj, r)] : val[(size_t)(b0 + j) * 32 + r]) & fj;
          }
          if constexpr (KW <= 2) {
            // narrow frontier rows (k <= 64): every frontier vertex of the
            // lane's word lands in row r, so the lane ORs their rows in
            // registers, several loads in flight, and adds the result to
            // the accumulator once
            constexpr int kIn = 3;
            uint32_t o0 = 0u, o1 = 0u;
            while (eff) {
              uint2 f[kIn];
#pragma unroll
              for (int u = 0; u < kIn; ++u) {
                f[u] = make_uint2(0u, 0u);
                if (eff) {
                  const int col = __clz(eff);
                  eff &= ~(0x80000000u >> col);
                  const size_t fo = (size_t)(vbase + col) * KW;
                  if (KW == 1)
                    f[u].x = F[fo];
                  else
                    f[u] = *reinterpret_cast<const uint2*>(F + fo);
                }
              }
#pragma unroll
              for (int u = 0; u < kIn; ++u) {
                o0 |= f[u].x;
                o1 |= f[u].y;
              }
            }
            if (o0) atomicOr(acc + r * KW, o0);
            if (KW == 2 && o1) atomicOr(acc + r * KW + 1, o1);
          } else {
            while (__any_sync(0xffffffffu, eff != 0u)) {
              const int c = min(__popc(eff), kPerPass);
              const int ic = warp_incl_sum(c, lane);
              const int tc = __shfl_sync(0xffffffffu, ic, 31);
              if (nlist + tc > kList) flush();
              int pos = nlist + ic - c;
              for (int q = 0; q < c; ++q) {
                const int col = __clz(eff);
                eff &= ~(0x80000000u >> col);
                list[pos++] = make_int2(r, vbase + col);
              }
              nlist += tc;
              __syncwarp();
            }
          }
        }
      };
      // two batches per step: the loads of both (block column -> frontier
      // word, a dependent pair) are in flight together
      for (int b0 = it.t0; b0 < it.t1; b0 += 64) {
        const int ta = b0 + (int)lane, tb = ta + 32;
        int ca = 0, cbb = 0;
        uint32_t ma = rm ? 0u : ~0u, mb = ma, fa = 0u, fbb = 0u;
        if (ta < it.t1) {
          ca = v.colind[ta];
          if (rm) ma = rm[ta];
        }
        if (tb < it.t1) {
          cbb = v.colind[tb];
          if (rm) mb = rm[tb];
        }
        if (ta < it.t1) fa = fb[ca];
        if (tb < it.t1) fbb = fb[cbb];
        batch(b0, ca, ma, fa);
        if (b0 + 32 < it.t1) batch(b0 + 32, cbb, mb, fbb);
      }
      flush();
      if (it.slot >= 0) {
        // a piece of a split block row: OR its non-zero words into the row's
        // accumulator (pieces of one row OR in any order)
        uint32_t* dst = a.split_acc + (size_t)a.slot_split[it.slot] * 32 * KW;
        for (int q = lane; q < 32 * KW; q += 32)
          if (acc[q]) atomicOr(dst + q, acc[q]);
      } else {
        block_row_epilogue<KW>(a, it.row, lvl, vrow, lane,
                               [&](int r, int ww) { return acc[r * KW + ww]; }, cnt);
      }
    } else if (it.slot < 0 && lane == 0) {
      a.fbits[(size_t)((lvl + 1) & 1) * (v.nbr + 1) + it.row] = 0u;
    }
  }
  // block count without a closing barrier: warps add and leave; the last
  // warp of the block to arrive adds the block's count to the level total
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane == 0) {
    if (cnt) atomicAdd(&cnt_sh, cnt);
    __threadfence_block();
    if (atomicAdd(&arrived_sh, 1) == kWarps - 1) {
      __threadfence_block();
      const unsigned long long tot = atomicAdd(&cnt_sh, 0ull);
      if (tot) atomicAdd(reinterpret_cast<unsigned long long*>(a.ctl + 4), tot);
    }
  }
}

// Pull step over the row-word slices of a 32x32 ROW graph, k <= 64 (KW <= 2
// words per frontier row): a warp per block row and lane r on row r.  The
// lane walks the row's entries {block column, row word} in ascending block
// column (head entry-major, two per round, then the tail; the tails of
// rows longer than kMsLongTail come from k_long_chunks), keeps the
// bits of each word whose vertex has a non-empty frontier row (fbits) and
// ORs those frontier rows in registers; the row leaves once every active
// source has reached it (seen | gathered covers them) or its entries run
// out.  The gathered rows go through the same block-row epilogue as k_step.
constexpr int kMsLongTail = kRwsLongTail;  // the slices' long-row chunking

template <int KW>
__device__ __forceinline__ void or_rows(const uint32_t* __restrict__ F, unsigned col_base, uint32_t m,
                                        uint32_t& f0, uint32_t& f1) {
  while (m) {
    uint2 g[2];
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      g[u] = make_uint2(0u, 0u);
      if (m) {
        const int col = __clz(m);
        m &= ~(0x80000000u >> col);
        const size_t fo = (size_t)(col_base + col) * KW;
        if (KW == 1) g[u].x = __ldg(F + fo);
        else g[u] = __ldg(reinterpret_cast<const uint2*>(F + fo));
      }
    }
    f0 |= g[0].x | g[1].x;
    f1 |= g[0].y | g[1].y;
  }
}

// Four entries at once: their block columns' frontier bits gathered
// together, then their frontier rows one set bit per entry per round, the
// four gathers of a round in flight together.
template <int KW>
__device__ __forceinline__ void or_entries4(const uint32_t* __restrict__ F, const uint32_t* __restrict__ fb,
                                            const uint2 (&e)[4], uint32_t& f0, uint32_t& f1) {
  uint32_t m[4];
#pragma unroll
  for (int u = 0; u < 4; ++u) m[u] = e[u].x != kRwsNone ? e[u].y & __ldg(fb + e[u].x) : 0u;
  while (m[0] | m[1] | m[2] | m[3]) {
    uint2 g[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      g[u] = make_uint2(0u, 0u);
      if (m[u]) {
        const int col = __clz(m[u]);
        m[u] &= ~(0x80000000u >> col);
        const size_t fo = ((size_t)e[u].x * 32 + col) * KW;
        if (KW == 1) g[u].x = __ldg(F + fo);
        else g[u] = __ldg(reinterpret_cast<const uint2*>(F + fo));
      }
    }
    f0 |= g[0].x | g[1].x | g[2].x | g[3].x;
    f1 |= g[0].y | g[1].y | g[2].y | g[3].y;
  }
}

// Tails of long rows (more than kMsLongTail entries), a warp per chunk of
// kRwsChunk entries: the frontier rows of the chunk's frontier neighbours
// OR-ed into the row's long_acc words, the chunk left early once the row is
// covered.  Runs before k_step_rws in every pull level, on a resident grid
// (warps stride over the chunks).
template <int KW>
__global__ void __launch_bounds__(kTPB) k_long_chunks(Args a) {
  volatile int* c = a.ctl;
  if (c[1]) return;
  if (a.dir && (c[7] || c[6] == 1)) return;
  const int lvl = c[0];
  const GView& v = a.v;
  const uint32_t* __restrict__ F = a.F + (size_t)(lvl & 1) * a.fstride;
  const uint32_t* __restrict__ fb = a.fbits + (size_t)(lvl & 1) * (v.nbr + 1);
  const unsigned lane = threadIdx.x & 31;
  const unsigned kFull = 0xffffffffu;
  const uint32_t need0 = src_mask(0, a.k) & (a.active ? a.active[0] : kFull);
  const uint32_t need1 = KW == 2 ? src_mask(1, a.k) & (a.active ? a.active[1] : kFull) : 0u;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long q = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < v.rws_nchunk; q += nwarps) {
    const long long i = v.rws_chunk_row[q];
    if ((a.vfull[i >> 5] >> (31 - (i & 31))) & 1u) continue;  // row finished
    const uint32_t s0 = a.V[(size_t)i * KW], s1 = KW == 2 ? a.V[(size_t)i * KW + 1] : 0u;
    if ((s0 & need0) == need0 && (s1 & need1) == need1) continue;
    const long long b = v.rws_chunk_beg[q], e = v.rws_chunk_end[q];
    uint32_t g0 = 0u, g1 = 0u;
    for (long long p = b; p < e; p += 128) {
      uint2 t[4];
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const long long pp = p + lane + 32 * u;
        t[u] = pp < e ? v.rws_tail[pp] : make_uint2(kRwsNone, 0u);
      }
      or_entries4<KW>(F, fb, t, g0, g1);
      const uint32_t r0 = __reduce_or_sync(kFull, g0), r1 = __reduce_or_sync(kFull, g1);
      if (((s0 | r0) & need0) == need0 && ((s1 | r1) & need1) == need1) break;
    }
    g0 = __reduce_or_sync(kFull, g0);
    g1 = __reduce_or_sync(kFull, g1);
    if (lane == 0) {
      int lo = 0, hi = v.rws_nlong;  // the row's index among the long rows
      while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (v.rws_long_row[mid] <= i) lo = mid;
        else hi = mid;
      }
      if (g0) atomicOr(a.long_acc + (size_t)lo * KW, g0);
      if (KW == 2 && g1) atomicOr(a.long_acc + (size_t)lo * KW + 1, g1);
    }
  }
}

template <int KW>
__global__ void __launch_bounds__(kTPB, 6) k_step_rws(Args a) {
  static_assert(KW <= 2, "one lane per row holds the row's frontier words in registers");
  __shared__ uint32_t acc_sh[kWarps][32 * KW];
  __shared__ unsigned long long cnt_sh;
  __shared__ int arrived_sh;
  volatile int* c = a.ctl;
  if (c[1]) return;
  if (a.dir && (c[7] || c[6] == 1)) return;  // this slot's level ran as a push
  if (threadIdx.x == 0) {
    cnt_sh = 0ull;
    arrived_sh = 0;
  }
  __syncthreads();
  const int lvl = c[0];
  const GView& v = a.v;
  const uint32_t* __restrict__ F = a.F + (size_t)(lvl & 1) * a.fstride;
  const uint32_t* __restrict__ fb = a.fbits + (size_t)(lvl & 1) * (v.nbr + 1);
  const unsigned lane = threadIdx.x & 31;
  const unsigned kFull = 0xffffffffu;
  uint32_t* acc = acc_sh[threadIdx.x >> 5];
  const long long R = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  unsigned long long cnt = 0;
  if (R < v.nbr) {
    const uint32_t vrow = a.vfull[R];
    if (vrow != kFull) {
      const long long i = R * 32 + lane;
      const uint32_t need0 = src_mask(0, a.k) & (a.active ? a.active[0] : kFull);
      const uint32_t need1 = KW == 2 ? src_mask(1, a.k) & (a.active ? a.active[1] : kFull) : 0u;
      bool go = !((vrow >> (31 - lane)) & 1u);
      uint32_t s0 = 0u, s1 = 0u;  // seen (visited) words of the row
      if (go) {
        s0 = a.V[(size_t)i * KW];
        if (KW == 2) s1 = a.V[(size_t)i * KW + 1];
      }
      uint32_t f0 = 0u, f1 = 0u;  // OR of the neighbours' frontier rows
      auto covered = [&]() { return ((s0 | f0) & need0) == need0 && ((s1 | f1) & need1) == need1; };
      go = go && !covered();
      const uint2* __restrict__ hp = v.rws_head + (size_t)R * (kRwsHead * 32) + lane;
#pragma unroll
      for (int k = 0; k < kRwsHead; k += 4) {
        if (!__any_sync(kFull, go)) break;
        uint2 e[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) e[u] = go ? hp[(size_t)(k + u) * 32] : make_uint2(kRwsNone, 0u);
        or_entries4<KW>(F, fb, e, f0, f1);
        go = go && e[3].x != kRwsNone && !covered();
      }
      if (__any_sync(kFull, go)) {
        long long tb = 0, te = 0;
        if (go) {
          tb = v.rws_tail_ptr[i];
          te = v.rws_tail_ptr[i + 1];
        }
        go = go && te > tb;
        if (go && te - tb > kMsLongTail) {
          // a long row: k_long_chunks gathered its tail over many warps
          int lo = 0, hi = v.rws_nlong;  // its index among the long rows
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (v.rws_long_row[mid] <= i) lo = mid;
            else hi = mid;
          }
          const uint32_t* la = a.long_acc + (size_t)lo * KW;
          f0 |= la[0];
          if (KW == 2) f1 |= la[1];
          go = false;
        }
        for (long long p = tb; __any_sync(kFull, go); p += 4) {
          if (go) {
            uint2 e[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) e[u] = p + u < te ? v.rws_tail[p + u] : make_uint2(kRwsNone, 0u);
            or_entries4<KW>(F, fb, e, f0, f1);
            go = p + 4 < te && !covered();
          }
        }
      }
      acc[lane * KW] = f0;
      if (KW == 2) acc[lane * KW + 1] = f1;
      __syncwarp();
      block_row_epilogue<KW>(a, (int)R, lvl, vrow, lane, [&](int r, int ww) { return acc[r * KW + ww]; }, cnt);
    } else if (lane == 0) {
      a.fbits[(size_t)((lvl + 1) & 1) * (v.nbr + 1) + R] = 0u;
    }
  }
  // block count without a closing barrier (as k_step)
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane == 0) {
    if (cnt) atomicAdd(&cnt_sh, cnt);
    __threadfence_block();
    if (atomicAdd(&arrived_sh, 1) == kWarps - 1) {
      __threadfence_block();
      const unsigned long long tot = atomicAdd(&cnt_sh, 0ull);
      if (tot) atomicAdd(reinterpret_cast<unsigned long long*>(a.ctl + 4), tot);
    }
  }
}

// Block count of a level and its close: the last block to arrive (arrival
// ticket in ctl[2], no waiting) advances the level, stops at a zero count or
// the iteration cap and, with dir, picks the next level's mode; `pushed`
// marks a level that ran as a push, so that the slot's pull kernels skip.
__device__ __forceinline__ void close_level(const Args& a, unsigned long long cnt, bool pushed) {
  volatile int* c = a.ctl;
  const unsigned lane = threadIdx.x & 31;
  __shared__ unsigned long long sh;
  __shared__ bool last;
  if (threadIdx.x == 0) sh = 0;
  __syncthreads();
  for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
  if (lane == 0 && cnt) atomicAdd(&sh, cnt);
  __syncthreads();
  unsigned long long* count = reinterpret_cast<unsigned long long*>(a.ctl + 4);
  if (threadIdx.x == 0) {
    if (sh) atomicAdd(count, sh);
    __threadfence();
    last = atomicAdd(reinterpret_cast<unsigned*>(a.ctl + 2), 1u) == gridDim.x - 1;
  }
  __syncthreads();
  if (last && threadIdx.x == 0) {
    __threadfence();
    volatile unsigned long long* vc = count;
    const unsigned long long total = *vc;
    const int it = c[0] + 1;
    const bool stop = total == 0ull || it >= c[3];
    if (a.dir) {
      c[6] = (long long)total < a.push_thr ? 1 : 0;
      c[7] = pushed ? 1 : 0;
    }
    c[0] = it;
    *vc = 0ull;
    a.ctl[2] = 0;
    if (stop) c[1] = 1;
    if (a.retire && a.active && a.slot_any) {
      volatile uint32_t* any = a.slot_any;
      for (int w = 0; w < (a.k + 31) / 32; ++w) {
        a.active[w] &= any[w];
        any[w] = 0u;
      }
    }
    __threadfence();
  }
}

// Split block rows (one warp each): OR the slot accumulators and run the
// epilogue.  The last block closes the level (arrival ticket, no waiting).
template <int KW>
__global__ void __launch_bounds__(kTPB) k_finish(Args a) {
  volatile int* c = a.ctl;
  if (c[1]) return;
  if (a.dir && c[7]) {
    // the slot's level ran as a push: every block takes a ticket and the
    // last one clears the flag for the next slot (all blocks have read it)
    if (threadIdx.x == 0 &&
        atomicAdd(reinterpret_cast<unsigned*>(a.ctl + 2), 1u) == gridDim.x - 1) {
      a.ctl[2] = 0;
      c[7] = 0;
      __threadfence();
    }
    return;
  }
  const int lvl = c[0];
  const GView& v = a.v;
  const unsigned lane = threadIdx.x & 31;
  const long long wid = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  unsigned long long cnt = 0;
  if (wid < v.nsplit) {
    const gbo_split sp = v.splits[wid];
    const uint32_t vrow = a.vfull[sp.row];
    if (vrow != 0xffffffffu) {
      uint32_t* sacc = a.split_acc + (size_t)wid * 32 * KW;
      block_row_epilogue<KW>(a, sp.row, lvl, vrow, lane, [&](int r, int ww) { return sacc[r * KW + ww]; },
                             cnt);
      __syncwarp();
      for (int q = lane; q < 32 * KW; q += 32) sacc[q] = 0u;  // zero for the next level
    } else if (lane == 0) {
      a.fbits[(size_t)((lvl + 1) & 1) * (v.nbr + 1) + sp.row] = 0u;
    }
  }
  close_level(a, cnt, false);
}

// Push level, one warp per work item (a block row R, or a piece of a long
// one) with frontier vertices in R: the (tile, row) pairs with row r in the
// frontier and non-empty in the tile are dealt out to the lanes, and every
// column x of the row word gets the frontier row of vertex 32R + r OR-ed
// into push_acc[x].  On a symmetric graph push_acc[x]
// is then the OR of the frontier rows of x's neighbours, which is what the
// pull step accumulates for row x.  k <= 64 (KW <= 2): lane r holds vertex
// 32R + r's frontier row in registers.
template <int KW>
__global__ void __launch_bounds__(kTPB) k_push(Args a) {
  static_assert(KW <= 2, "push levels hold frontier rows in registers");
  volatile int* c = a.ctl;
  if (c[1] || c[7] || c[6] != 1) return;
  const int lvl = c[0];
  const GView& v = a.v;
  const unsigned lane = threadIdx.x & 31;
  const long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (item >= v.nitems) return;
  const gbo_item it = v.items[item];
  const long long R = it.row;
  const uint32_t fword = a.fbits[(size_t)(lvl & 1) * (v.nbr + 1) + R];
  if (fword == 0u) return;
  const uint32_t* __restrict__ F = a.F + (size_t)(lvl & 1) * a.fstride;
  uint32_t fr0 = 0u, fr1 = 0u;
  if ((fword >> (31 - lane)) & 1u) {  // only frontier rows are valid (and in bounds)
    const size_t o = ((size_t)R * 32 + lane) * KW;
    fr0 = F[o];
    if (KW == 2) fr1 = F[o + 1];
  }
  const unsigned frows = __brev(fword);  // bit r: vertex 32R + r in the frontier
  const uint32_t* __restrict__ val = reinterpret_cast<const uint32_t*>(v.val);
  const unsigned* __restrict__ rm = v.rowmask;
  uint32_t* __restrict__ acc = a.push_acc;
  const int t0 = it.t0, t1 = it.t1;
  for (int b0 = t0; b0 < t1; b0 += 32) {
    const int t = b0 + (int)lane;
    int cb = 0;
    unsigned cand = 0u;
    if (t < t1) {
      cb = v.colind[t];
      cand = (rm ? rm[t] : 0xffffffffu) & frows;
    }
    const int cnt = __popc(cand);
    const int incl = warp_incl_sum(cnt, lane);
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int excl = incl - cnt;
    for (int pb = 0; pb < total; pb += 32) {
      const int p = pb + (int)lane;
      int j = 0;
#pragma unroll
      for (int st = 16; st > 0; st >>= 1) {
        const int q = __shfl_sync(0xffffffffu, incl, j + st - 1);
        if (q <= p) j += st;
      }
      const int ej = __shfl_sync(0xffffffffu, excl, j);
      const unsigned cj = __shfl_sync(0xffffffffu, cand, j);
      const int xbase = __shfl_sync(0xffffffffu, cb, j) * 32;
      int r = 0;
      uint32_t word = 0u;
      if (p < total) {
        r = (int)__fns(cj, 0, p - ej + 1);
        word = val[(size_t)(b0 + j) * 32 + r];
      }
      const uint32_t f0 = __shfl_sync(0xffffffffu, fr0, r);
      const uint32_t f1 = __shfl_sync(0xffffffffu, fr1, r);
      if (!(f0 | f1)) word = 0u;
      while (word) {
        const int col = __clz(word);
        word &= ~(0x80000000u >> col);
        const size_t xo = (size_t)(xbase + col) * KW;
        if (f0) atomicOr(acc + xo, f0);
        if (KW == 2 && f1) atomicOr(acc + xo + 1, f1);
      }
    }
  }
}

// Push level over the row-word slices (symmetric graphs, any k): the
// frontier rows of the level's frontier vertices are OR-ed into push_acc of
// their neighbours, as k_push does from the tiles, but walking only the
// frontier vertices' own entries.  push_one ORs vertex u's non-zero
// frontier words (nz: which of its KW words) into neighbour word w's
// accumulators; the words are read through L1 (every lane the same).
template <int KW>
__device__ __forceinline__ void push_entry(const Args& a, const uint32_t* __restrict__ fu, uint32_t nz, uint2 e) {
  if (e.x == kRwsNone) return;
  for (uint32_t m = e.y; m;) {
    const int c = __clz(m);
    m &= ~(0x80000000u >> c);
    uint32_t* dst = a.push_acc + ((size_t)e.x * 32 + c) * KW;
    for (uint32_t jm = nz; jm; jm &= jm - 1) {
      const int j = __ffs(jm) - 1;
      atomicOr(dst + j, fu[j]);
    }
  }
}

// Part 1, a warp per block row with frontier vertices: for each of them the
// head (eight entries, one per lane) and a tail of up to kMsLongTail entries
// (32 per round); longer tails are k_push_chunks'.
template <int KW>
__global__ void __launch_bounds__(kTPB) k_push_rows(Args a) {
  volatile int* c = a.ctl;
  if (c[1] || c[7] || c[6] != 1) return;
  const int lvl = c[0];
  const GView& v = a.v;
  const unsigned lane = threadIdx.x & 31;
  const long long R = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (R >= v.nbr) return;
  const uint32_t fw = a.fbits[(size_t)(lvl & 1) * (v.nbr + 1) + R];
  if (!fw) return;
  const uint32_t* __restrict__ F = a.F + (size_t)(lvl & 1) * a.fstride;
  for (uint32_t rm = fw; rm;) {
    const int r = __clz(rm);  // bit 31 - r: row r
    rm &= ~(0x80000000u >> r);
    const long long u = R * 32 + r;
    const uint32_t* fu = F + (size_t)u * KW;
    const uint32_t nz = __ballot_sync(0xffffffffu, (int)lane < KW && fu[lane < KW ? lane : 0] != 0u);
    if (!nz) continue;
    if (lane < kRwsHead) push_entry<KW>(a, fu, nz, v.rws_head[((size_t)R * kRwsHead + lane) * 32 + r]);
    const long long tb = v.rws_tail_ptr[u], te = v.rws_tail_ptr[u + 1];
    if (te - tb > kMsLongTail) continue;  // k_push_chunks walks long tails
    for (long long p = tb + lane; p < te; p += 32) push_entry<KW>(a, fu, nz, v.rws_tail[p]);
  }
}

// Part 2, a warp per long-tail chunk whose row is a frontier vertex.
template <int KW>
__global__ void __launch_bounds__(kTPB) k_push_chunks(Args a) {
  volatile int* c = a.ctl;
  if (c[1] || c[7] || c[6] != 1) return;
  const int lvl = c[0];
  const GView& v = a.v;
  const unsigned lane = threadIdx.x & 31;
  const uint32_t* __restrict__ fb = a.fbits + (size_t)(lvl & 1) * (v.nbr + 1);
  const uint32_t* __restrict__ F = a.F + (size_t)(lvl & 1) * a.fstride;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  for (long long q = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5; q < v.rws_nchunk; q += nwarps) {
    const long long u = v.rws_chunk_row[q];
    if (!((fb[u >> 5] >> (31 - (u & 31))) & 1u)) continue;
    const uint32_t* fu = F + (size_t)u * KW;
    const uint32_t nz = __ballot_sync(0xffffffffu, (int)lane < KW && fu[lane < KW ? lane : 0] != 0u);
    if (!nz) continue;
    for (long long p = v.rws_chunk_beg[q] + lane; p < v.rws_chunk_end[q]; p += 32)
      push_entry<KW>(a, fu, nz, v.rws_tail[p]);
  }
}

// After k_push: the epilogue of every block row from push_acc (zeroed
// again), then the level close.  Block rows without new bits only clear
// their next-frontier word.
template <int KW>
__global__ void __launch_bounds__(kTPB) k_push_fin(Args a) {
  volatile int* c = a.ctl;
  if (c[1] || c[7] || c[6] != 1) return;
  const int lvl = c[0];
  const GView& v = a.v;
  const unsigned lane = threadIdx.x & 31;
  const long long R = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  unsigned long long cnt = 0;
  if (R < v.nbr) {
    uint32_t* na = a.push_acc + (size_t)R * 32 * KW;
    uint32_t any = 0u;
    for (int q = lane; q < 32 * KW; q += 32) any |= na[q];
    const uint32_t vrow = a.vfull[R];
    if (vrow != 0xffffffffu && __any_sync(0xffffffffu, any != 0u)) {
      block_row_epilogue<KW>(a, (int)R, lvl, vrow, lane, [&](int r, int ww) { return na[r * KW + ww]; },
                             cnt);
      __syncwarp();
    } else if (lane == 0) {
      a.fbits[(size_t)((lvl + 1) & 1) * (v.nbr + 1) + R] = 0u;
    }
    if (__any_sync(0xffffffffu, any != 0u))
      for (int q = lane; q < 32 * KW; q += 32) na[q] = 0u;
  }
  close_level(a, cnt, true);
}

// Level 0 of a multi-source BFS on a symmetric slice graph as a push: the
// sources' own entries (a warp per (source, piece of its tail); piece 0
// also takes the head) OR the source's bit into push_acc of every
// neighbour, which on P = P^T is what the level's pull step would gather
// for that neighbour -- but without walking every row of the graph for a
// frontier of k vertices.  k_push_fin then runs the block-row epilogue and
// closes the level; this kernel sets the level's mode so that it does.
template <int KW>
__global__ void __launch_bounds__(kTPB) k_seed_push(Args a, const int* __restrict__ srcs, int nsrc, int pieces) {
  const unsigned lane = threadIdx.x & 31;
  const long long w = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (w == 0 && lane == 0) a.ctl[6] = 1;
  if (w >= (long long)nsrc * pieces) return;
  const int q = (int)(w / pieces), piece = (int)(w % pieces);
  const int v0 = srcs[q];
  const GView& v = a.v;
  if (v0 < 0 || v0 >= v.nrows) return;
  const uint32_t bit = 1u << (q % 32);
  uint32_t* acc = a.push_acc + q / 32;
  auto push = [&](uint2 e) {
    for (uint32_t m = e.y; m;) {
      const int c = __clz(m);
      m &= ~(0x80000000u >> c);
      atomicOr(acc + ((size_t)e.x * 32 + c) * KW, bit);
    }
  };
  if (piece == 0 && lane < kRwsHead) {
    const uint2 e = v.rws_head[((size_t)(v0 / 32) * kRwsHead + lane) * 32 + v0 % 32];
    if (e.x != kRwsNone) push(e);
  }
  const long long tb = v.rws_tail_ptr[v0], te = v.rws_tail_ptr[v0 + 1];
  const long long per = (te - tb + pieces - 1) / pieces;
  const long long pb = tb + (long long)piece * per;
  const long long pe = pb + per < te ? pb + per : te;
  for (long long p = pb + lane; p < pe; p += 32) push(v.rws_tail[p]);
}

// Reset: levels -1, V 0, F[0] 0, frontier bits 0, padding rows and rows
// without entries marked full (no source can reach them).  A source in such
// a row reopens it in k_seed.  The level counter starts at lvl0 (levels are
// written as lvl0 + hops; the query server's batches keep its absolute
// level count) and the loop stops at max_iter.
static __global__ void k_init(Args a, int kw, int max_iter, int lvl0 = 0) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long stride = (long long)gridDim.x * blockDim.x;
  const int n = a.v.nrows, nbr = a.v.nbr;
  for (long long q = i; q < (long long)n * a.k; q += stride) a.levels[q] = -1;
  for (long long q = i; q < (long long)n * kw; q += stride) {
    a.F[q] = 0u;
    a.V[q] = 0u;
  }
  for (long long q = i; q < 2LL * (nbr + 1); q += stride) a.fbits[q] = 0u;
  for (long long q = i; q <= nbr; q += stride) {
    const long long lo = q * 32;
    uint32_t pad = 0;
    for (int r = 0; r < 32; ++r)
      if (lo + r >= n) pad |= 1u << (31 - r);
    if (a.live && q < nbr) pad |= ~a.live[q];
    a.vfull[q] = pad;
  }
  if (a.retire && i < kw) {
    a.active[i] = src_mask((int)i, a.k);
    a.slot_any[i] = 0u;
  }
  if (i == 0) {
    a.ctl[0] = lvl0;
    a.ctl[1] = 0;
    a.ctl[2] = 0;
    a.ctl[3] = max_iter;
    reinterpret_cast<unsigned long long*>(a.ctl + 4)[0] = 0ull;
    a.ctl[6] = a.dir ? 1 : 0;  // k sources: the first level pushes
    a.ctl[7] = 0;
  }
}

// Sources entering the frontier of level lvl, one thread per source (two
// kernels, so that every row is cleared before any source bit is set):
// a row that is not in the frontier yet has stale words, cleared first.
static __global__ void k_seed_clear(Args a, const int* __restrict__ srcs, int nsrc, int kw, int lvl) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsrc) return;
  const int v0 = srcs[q];
  if (v0 < 0 || v0 >= a.v.nrows) return;
  const uint32_t* fb = a.fbits + (size_t)(lvl & 1) * (a.v.nbr + 1);
  uint32_t* F = a.F + (size_t)(lvl & 1) * a.fstride;
  if (!((fb[v0 / 32] >> (31 - v0 % 32)) & 1u))
    for (int w = 0; w < kw; ++w) F[(size_t)v0 * kw + w] = 0u;
}

static __global__ void k_seed_set(Args a, const int* __restrict__ srcs, const int* __restrict__ slots,
                                  int nsrc, int kw, int lvl) {
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if (q >= nsrc) return;
  const int v0 = srcs[q];
  const int s = slots ? slots[q] : q;
  if (v0 < 0 || v0 >= a.v.nrows) return;
  uint32_t* F = a.F + (size_t)(lvl & 1) * a.fstride;
  uint32_t* fb = a.fbits + (size_t)(lvl & 1) * (a.v.nbr + 1);
  atomicOr(F + (size_t)v0 * kw + s / 32, 1u << (s % 32));
  atomicOr(a.V + (size_t)v0 * kw + s / 32, 1u << (s % 32));
  a.levels[level_index(a, v0, s)] = lvl;
  atomicOr(fb + v0 / 32, 1u << (31 - v0 % 32));
  atomicAnd(a.vfull + v0 / 32, ~(1u << (31 - v0 % 32)));
}

// Both seeding kernels on stream st.
static inline void seed_sources(const Args& a, const int* srcs, const int* slots, int nsrc, int kw, int lvl,
                                cudaStream_t st) {
  if (nsrc <= 0) return;
  const unsigned g = (unsigned)((nsrc + 255) / 256);
  k_seed_clear<<<g, 256, 0, st>>>(a, srcs, nsrc, kw, lvl);
  k_seed_set<<<g, 256, 0, st>>>(a, srcs, slots, nsrc, kw, lvl);
}

}  // namespace ms
}  // namespace gbo
