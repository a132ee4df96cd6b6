// Shared device building blocks of the pull kernels: the lane layout of a
// work item and the batched Boolean (OR.AND) scan of a block row.
#pragma once

#include <type_traits>

#include "bmv.cuh"

namespace gbo {

// Lane layout: W = min(b,32) lanes per work item, G items per warp, RPL rows
// per lane (b = 64: rows r and r+32).
template <int B>
struct Lay {
  static constexpr int W = B >= 32 ? 32 : B;
  static constexpr int G = 32 / W;
  static constexpr int RPL = B > 32 ? 2 : 1;
};

// Mask of the lanes that share this lane's work item.
template <int B>
__device__ __forceinline__ unsigned group_mask(unsigned lane) {
  constexpr int W = Lay<B>::W;
  if (W == 32) return 0xffffffffu;
  return seg_mask<W>() << ((lane / W) * W);
}

template <typename WT>
__device__ __forceinline__ WT shfl_word(unsigned mask, WT v, int src, int width) {
  if (sizeof(WT) == 8)
    return (WT)__shfl_sync(mask, (unsigned long long)v, src, width);
  return (WT)__shfl_sync(mask, (unsigned)v, src, width);
}

// Inclusive prefix sum over the lanes of a warp.
__device__ __forceinline__ int warp_incl_sum(int x, unsigned lane) {
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, x, o);
    if ((int)lane >= o) x += y;
  }
  return x;
}

// The b = 32 form of pull_or_scan (below) for tiles with occupancy words
// (v.rowmask).  Per batch of 32 tiles (lane j: tile j) the words that can
// answer a row are the pairs (tile j, row r) with a non-empty frontier
// segment at j and r both still open and non-empty in tile j: one or two per
// tile on sparse graphs.  Those pairs are dealt out to the lanes (lane p
// takes pair p of the batch: its tile by a binary search over the lanes'
// prefix counts, its row as the k-th set bit of the tile's candidate rows),
// so a batch costs a round of 32 independent word loads instead of a pass
// over every tile with one or two lanes active.  A word that hits the tile's
// frontier segment answers its row; the answers are OR-ed across the warp
// after each round, and rows answered meanwhile drop their remaining pairs.
// NB batches are dealt side by side so that their word loads are in flight
// together.
__device__ __forceinline__ void pull_or_scan_rowmask32(const GView& v, int t0, int t1,
                                                       const unsigned* __restrict__ x, bool need0,
                                                       bool& p0, unsigned lane) {
  constexpr int NB = 2;          // batches per step
  constexpr int SPAN = 32 * NB;  // tiles per step
  const unsigned* __restrict__ val = reinterpret_cast<const unsigned*>(v.val);
  const unsigned* __restrict__ rm = v.rowmask;
  // pipeline: step i+1's x words and occupancy words and step i+2's
  // block-column indices are in flight while step i's row words load
  int c2[NB];
  unsigned m1[NB], x1[NB];
#pragma unroll
  for (int q = 0; q < NB; ++q) {
    const int t = t0 + q * 32 + (int)lane;
    const int c1 = t < t1 ? v.colind[t] : -1;
    c2[q] = t + SPAN < t1 ? v.colind[t + SPAN] : -1;
    m1[q] = c1 >= 0 ? rm[t] : 0u;
    x1[q] = c1 >= 0 ? x[c1] : 0u;
  }
  unsigned needm = __ballot_sync(0xffffffffu, need0 && !p0);  // bit r: row r open
  for (int base = t0; base < t1 && needm; base += SPAN) {
    unsigned xs[NB], cand[NB];
    int incl[NB], excl[NB], total[NB];
    int most = 0;
#pragma unroll
    for (int q = 0; q < NB; ++q) {
      const int t = base + q * 32 + (int)lane;
      xs[q] = x1[q];
      cand[q] = xs[q] ? (m1[q] & needm) : 0u;  // this lane's tile: rows worth a load
      m1[q] = c2[q] >= 0 ? rm[t + SPAN] : 0u;
      x1[q] = c2[q] >= 0 ? x[c2[q]] : 0u;
      c2[q] = t + 2 * SPAN < t1 ? v.colind[t + 2 * SPAN] : -1;
      // pair positions, only for batches with pairs
      const int cnt = __popc(cand[q]);
      total[q] = (int)__reduce_add_sync(0xffffffffu, (unsigned)cnt);
      incl[q] = excl[q] = 0;
      if (total[q]) {
        incl[q] = warp_incl_sum(cnt, lane);
        excl[q] = incl[q] - cnt;
      }
      most = max(most, total[q]);
    }
    for (int pb = 0; pb < most; pb += 32) {
      unsigned hit = 0u;
#pragma unroll
      for (int q = 0; q < NB; ++q) {
        const int p = pb + (int)lane;
        // tile of pair p: the number of lanes whose inclusive count is <= p
        int j = 0;
#pragma unroll
        for (int st = 16; st > 0; st >>= 1) {
          const int c = __shfl_sync(0xffffffffu, incl[q], j + st - 1);
          if (c <= p) j += st;
        }
        const int ej = __shfl_sync(0xffffffffu, excl[q], j);
        const unsigned cj = __shfl_sync(0xffffffffu, cand[q], j);
        const unsigned xj = __shfl_sync(0xffffffffu, xs[q], j);
        if (p < total[q]) {
          const int r = (int)__fns(cj, 0, p - ej + 1);
          if ((needm >> r) & 1u) {
            if (val[(size_t)(base + q * 32 + j) * 32 + r] & xj) hit |= 1u << r;
          }
        }
      }
      const unsigned found = __reduce_or_sync(0xffffffffu, hit);
      needm &= ~found;
      if (!needm) break;
    }
  }
  p0 = p0 || (need0 && !((needm >> lane) & 1u));
}

// Boolean pull over tiles [t0, t1) of one block row for the rows this lane
// owns: p0 |= (row word & x[colind]) != 0 (p1 for row r+32 when b = 64).
// need0/need1 say whether the row still needs an answer; a row stops loading
// once it has one, and the group leaves the row as soon as all its rows are
// answered.  Block-column indices are read W at a time (one coalesced load),
// their x words gathered in parallel, and only tiles with a non-empty x
// segment are fetched, U tile words in flight per lane.
template <int B>
__device__ __forceinline__ void pull_or_scan(const GView& v, int t0, int t1,
                                             const typename Word<B>::T* __restrict__ x,
                                             bool need0, bool need1, bool& p0, bool& p1,
                                             unsigned lane) {
  using WT = typename Word<B>::T;
  using L = Lay<B>;
  if constexpr (B == 32) {
    if (v.rowmask) {
      pull_or_scan_rowmask32(v, t0, t1, reinterpret_cast<const unsigned*>(x), need0, p0, lane);
      return;
    }
  }
  constexpr int W = L::W;
  const unsigned gmask = group_mask<B>(lane);
  const int r = lane % W;
  const unsigned gshift = (lane / W) * W;
  const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
  constexpr int U = 8;  // tile words in flight per lane
  // Software pipeline over batches of W tiles: while batch i's tile words
  // load, batch i+1's x words and batch i+2's block-column indices are in
  // flight, so only the tile loads sit on the critical path.
  int c1 = (t0 + r < t1) ? v.colind[t0 + r] : -1;
  int c2 = (t0 + W + r < t1) ? v.colind[t0 + W + r] : -1;
  WT x1 = c1 >= 0 ? x[c1] : (WT)0;
  for (int base = t0; base < t1; base += W) {
    const WT xs = x1;
    x1 = c2 >= 0 ? x[c2] : (WT)0;
    c2 = (base + 2 * W + r < t1) ? v.colind[base + 2 * W + r] : -1;
    unsigned nz = (__ballot_sync(gmask, xs != 0) >> gshift) & seg_mask<W>();
    while (nz) {
      int j[U];
#pragma unroll
      for (int q = 0; q < U; ++q) {
        j[q] = nz ? __ffs(nz) - 1 : -1;
        nz &= nz - 1;
      }
      WT xv[U];
#pragma unroll
      for (int q = 0; q < U; ++q) xv[q] = shfl_word<WT>(gmask, xs, j[q] < 0 ? 0 : j[q], W);
      const bool l0 = need0 && !p0;
      const bool l1 = L::RPL == 2 && need1 && !p1;
      WT a[U], c[U];
#pragma unroll
      for (int q = 0; q < U; ++q) {
        a[q] = 0;
        c[q] = 0;
        if (j[q] >= 0) {
          const size_t off = (size_t)(base + j[q]) * B;
          if (l0) a[q] = val[off + r];
          if (L::RPL == 2 && l1) c[q] = val[off + 32 + r];
        }
      }
#pragma unroll
      for (int q = 0; q < U; ++q) {
        p0 |= (a[q] & xv[q]) != 0;
        if (L::RPL == 2) p1 |= (c[q] & xv[q]) != 0;
      }
    }
    const bool open = (need0 && !p0) || (L::RPL == 2 && need1 && !p1);
    if (!__any_sync(gmask, open)) break;
  }
}

// 32x32 bit transpose across a warp: lane j holds word m_j; lane r gets the
// word whose bit j is bit r of m_j (recursive swap of off-diagonal blocks).
__device__ __forceinline__ unsigned warp_transpose32(unsigned x, unsigned lane) {
  const unsigned lo_masks[5] = {0x0000FFFFu, 0x00FF00FFu, 0x0F0F0F0Fu, 0x33333333u, 0x55555555u};
#pragma unroll
  for (int s = 0; s < 5; ++s) {
    const int k = 16 >> s;
    const unsigned lo = lo_masks[s];
    const unsigned y = __shfl_xor_sync(0xffffffffu, x, k);
    x = (lane & k) ? ((x & ~lo) | ((y & ~lo) >> k)) : ((x & lo) | ((y & lo) << k));
  }
  return x;
}

// fold_row_cols (below) for b = 32 tiles with packed row words.  Per batch
// of 32 tiles the occupancy words are transposed (lane r: the tiles where
// row r is non-empty), and the batch's non-empty words are dealt out to the
// lanes in row-major order, 32 per round: lane p takes word p (its row by a
// binary search over the rows' prefix counts, its tile as the k-th tile of
// that row), folds the word's columns (first set column, then the others in
// order), and a segmented scan over the lanes of each row's run (the runs
// are contiguous) leaves the run's fold in its last lane, which the row's
// own lane folds into its accumulator.  Every lane does one word per round
// whatever the rows' lengths (two rounds at a time, so that their loads
// overlap), and the order of every fold is fixed by the graph alone.
template <int U, typename Acc, typename Term, typename Comb>
__device__ __forceinline__ void fold_row_cols_t32(const GView& v, int t0, int t1, long long wb,
                                                  unsigned lane, Term term, Comb comb, Acc& acc) {
  const unsigned* __restrict__ words = v.rowword;
  const unsigned* __restrict__ rm = v.rowmask;
  int cn = t0 + (int)lane < t1 ? v.colind[t0 + lane] : 0;
  unsigned mn = t0 + (int)lane < t1 ? rm[t0 + lane] : 0u;
  for (int b0 = t0; b0 < t1; b0 += 32) {
    const int cb = cn;
    const unsigned m = mn;
    if (b0 + 32 < t1) {
      const int t = b0 + 32 + (int)lane;
      cn = t < t1 ? v.colind[t] : 0;
      mn = t < t1 ? rm[t] : 0u;
    }
    const int mc = __popc(m);
    const int off = warp_incl_sum(mc, lane) - mc;  // lane j: tile j's first word, relative to wb
    const long long wbat = wb;
    const unsigned tl = warp_transpose32(m, lane);  // lane r: tiles of the batch where row r is non-empty
    const int rc = __popc(tl);
    const int rincl = warp_incl_sum(rc, lane);
    const int total = __shfl_sync(0xffffffffu, rincl, 31);
    wb += total;
    const int rexcl = rincl - rc;
    constexpr int H = 2;  // rounds dealt together (their loads overlap)
    for (int pb = 0; pb < total; pb += 32 * H) {
      Acc x[H];
      int key[H];
      unsigned w[H];
      long long base[H];
#pragma unroll
      for (int h = 0; h < H; ++h) {
        const int p = pb + 32 * h + (int)lane;
        // row of word p: the number of rows whose inclusive count is <= p
        int r = 0;
#pragma unroll
        for (int st = 16; st > 0; st >>= 1) {
          const int c = __shfl_sync(0xffffffffu, rincl, r + st - 1);
          if (c <= p) r += st;
        }
        const int er = __shfl_sync(0xffffffffu, rexcl, r);
        const unsigned tr = __shfl_sync(0xffffffffu, tl, r);
        const bool valid = p < total;
        const int j = valid ? (int)__fns(tr, 0, p - er + 1) : 0;
        const unsigned mj = __shfl_sync(0xffffffffu, m, j);
        const int oj = __shfl_sync(0xffffffffu, off, j);
        base[h] = (long long)__shfl_sync(0xffffffffu, cb, j) * 32;
        w[h] = valid ? words[wbat + oj + __popc(mj & ((1u << r) - 1u))] : 0u;
        key[h] = valid ? r : -1 - (int)lane;
      }
      // the first set column of each word gathered together, then the others
#pragma unroll
      for (int h = 0; h < H; ++h) {
        x[h] = Acc{};
        if (w[h]) {
          const int col = __clz((int)w[h]);
          w[h] &= ~(0x80000000u >> col);
          x[h] = term(base[h] + col);
        }
      }
#pragma unroll
      for (int h = 0; h < H; ++h) {
        while (w[h]) {
          const int col = __clz((int)w[h]);
          w[h] &= ~(0x80000000u >> col);
          comb(x[h], term(base[h] + col));
        }
      }
      // segmented inclusive scan over each row's run of lanes, per round
#pragma unroll
      for (int d = 1; d < 32; d <<= 1) {
#pragma unroll
        for (int h = 0; h < H; ++h) {
          const Acc y = __shfl_up_sync(0xffffffffu, x[h], d);
          const int ky = __shfl_up_sync(0xffffffffu, key[h], d);
          if ((int)lane >= d && ky == key[h]) {
            Acc z = y;
            comb(z, x[h]);
            x[h] = z;
          }
        }
      }
      // row `lane`: the last lane of its run in each round, rounds in order
#pragma unroll
      for (int h = 0; h < H; ++h) {
        const int rb = pb + 32 * h;
        const int lo = max(rexcl, rb), hi = min(rincl, rb + 32);
        const Acc seg = __shfl_sync(0xffffffffu, x[h], hi > lo ? hi - 1 - rb : 0);
        if (hi > lo) comb(acc, seg);
      }
    }
  }
}

// Fold term(column) over the set columns of this lane's row words in tiles
// [t0, t1) (row r, and r + 32 for b = 64), for semirings whose value comes
// from a gather at the column (x[j], dist[j], labels[j] ...).  wb is the
// packed-word index of tile t0's first word (b = 32 graphs with packed row
// words take fold_row_cols_t32 above).  U tiles per
// step: their block-column indices and row words are loaded together, then
// the first set column of every word is gathered together (U or 2U
// independent loads in flight); further set columns of a word (rare in
// sparse tiles) follow one at a time.  term(idx) returns the value at global
// column idx; comb(acc, value) folds it into acc.  Words are left-aligned
// in 32 bits for b <= 32 (64 for b = 64) so that column 0 is the top bit.
template <int B, int U, typename Acc, typename Term, typename Comb>
__device__ __forceinline__ void fold_row_cols(const GView& v, int t0, int t1, long long wb, int r,
                                              Term term, Comb comb, Acc& acc0, Acc& acc1) {
  using WT = typename Word<B>::T;
  using L = Lay<B>;
  using T = decltype(term(0ll));
  using AW = typename std::conditional<(B > 32), unsigned long long, unsigned>::type;
  if constexpr (B == 32) {
    if (v.rowword) {
      fold_row_cols_t32<U>(v, t0, t1, wb, (unsigned)r, term, comb, acc0);
      return;
    }
  }
  constexpr int kBits = sizeof(AW) * 8;
  constexpr AW kTop = (AW)1 << (kBits - 1);
  const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
  auto lead = [](AW a) -> int { return kBits == 64 ? __clzll((long long)a) : __clz((int)a); };
  auto rest = [&](AW a, long long base, Acc& acc) {
    while (a) {
      const int j = lead(a);
      a &= ~(kTop >> j);
      comb(acc, term(base + j));
    }
  };
  // software pipeline: batch i+1's column indices and row words load while
  // batch i's gathers run
  auto load = [&](int tb, unsigned (&base)[U], AW (&a0)[U], AW (&a1)[U]) {
#pragma unroll
    for (int k = 0; k < U; ++k) {
      base[k] = (unsigned)v.colind[tb + k] * (unsigned)B;  // < 2^32: ncols is an int
      a0[k] = (AW)val[(size_t)(tb + k) * B + r] << (kBits - B);
      a1[k] = L::RPL == 2 ? (AW)val[(size_t)(tb + k) * B + 32 + r] << (kBits - B) : (AW)0;
    }
  };
  int t = t0;
  unsigned base[U];
  AW a0[U], a1[U];
  bool have = t + U <= t1;
  if (have) load(t, base, a0, a1);
  while (have) {
    const int tn = t + U;
    const bool next = tn + U <= t1;
    unsigned nbase[U];
    AW n0[U], n1[U];
    if (next) load(tn, nbase, n0, n1);
    T g0[U], g1[U];
    bool h0[U], h1[U];
#pragma unroll
    for (int k = 0; k < U; ++k) {
      h0[k] = a0[k] != 0;
      h1[k] = L::RPL == 2 && a1[k] != 0;
      if (h0[k]) {
        const int j = lead(a0[k]);
        a0[k] &= ~(kTop >> j);
        g0[k] = term((long long)base[k] + j);
      }
      if (h1[k]) {
        const int j = lead(a1[k]);
        a1[k] &= ~(kTop >> j);
        g1[k] = term((long long)base[k] + j);
      }
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
      if (h0[k]) comb(acc0, g0[k]);
      if (h1[k]) comb(acc1, g1[k]);
    }
#pragma unroll
    for (int k = 0; k < U; ++k) {
      rest(a0[k], (long long)base[k], acc0);
      if (L::RPL == 2) rest(a1[k], (long long)base[k], acc1);
    }
    t = tn;
    have = next;
    if (next) {
#pragma unroll
      for (int k = 0; k < U; ++k) {
        base[k] = nbase[k];
        a0[k] = n0[k];
        a1[k] = n1[k];
      }
    }
  }
  for (; t < t1; ++t) {
    const long long base = (long long)v.colind[t] * B;
    rest((AW)val[(size_t)t * B + r] << (kBits - B), base, acc0);
    if (L::RPL == 2) rest((AW)val[(size_t)t * B + 32 + r] << (kBits - B), base, acc1);
  }
}

}  // namespace gbo
