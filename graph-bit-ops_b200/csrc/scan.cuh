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

// The b = 32 form of pull_or_scan (below) for tiles with occupancy words
// (v.rowmask).  Per batch of 32 tiles (lane j: tile j) the words that can
// answer a row are the pairs (tile j, row r) with a non-empty frontier
// segment at j and r both still open and non-empty in tile j: one or two per
// tile on sparse graphs.  Those pairs are dealt out to the lanes (lane p
// takes pair p of the batch: its tile by a binary search over the lanes'
// prefix counts, its row as the k-th set bit of the tile's candidate rows),
// so a batch costs a round or two of 32 independent word loads instead of a
// pass over every tile with one or two lanes active.  A word that hits the
// tile's frontier segment answers its row; the answers are OR-ed across the
// warp after each pair of rounds, and rows answered meanwhile drop their
// remaining pairs.
__device__ __forceinline__ void pull_or_scan_rowmask32(const GView& v, int t0, int t1,
                                                       const unsigned* __restrict__ x, bool need0,
                                                       bool& p0, unsigned lane) {
  const unsigned* __restrict__ val = reinterpret_cast<const unsigned*>(v.val);
  const unsigned* __restrict__ rm = v.rowmask;
  // pipeline: batch i+1's x words and occupancy words and batch i+2's
  // block-column indices are in flight while batch i's row words load
  int c1 = (t0 + (int)lane < t1) ? v.colind[t0 + lane] : -1;
  int c2 = (t0 + 32 + (int)lane < t1) ? v.colind[t0 + 32 + lane] : -1;
  unsigned m1 = c1 >= 0 ? rm[t0 + lane] : 0u;
  unsigned x1 = c1 >= 0 ? x[c1] : 0u;
  unsigned needm = __ballot_sync(0xffffffffu, need0 && !p0);  // bit r: row r open
  for (int base = t0; base < t1 && needm; base += 32) {
    const unsigned xs = x1, ms = m1;
    m1 = c2 >= 0 ? rm[base + 32 + lane] : 0u;
    x1 = c2 >= 0 ? x[c2] : 0u;
    c2 = (base + 64 + (int)lane < t1) ? v.colind[base + 64 + lane] : -1;
    const unsigned cand = xs ? (ms & needm) : 0u;  // this lane's tile: rows worth a load
    const int cnt = __popc(cand);
    int incl = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int y = __shfl_up_sync(0xffffffffu, incl, o);
      if ((int)lane >= o) incl += y;
    }
    const int total = __shfl_sync(0xffffffffu, incl, 31);
    const int excl = incl - cnt;
    for (int pb = 0; pb < total; pb += 64) {
      unsigned hit = 0u;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int p = pb + h * 32 + (int)lane;
        // tile of pair p: the number of lanes whose inclusive count is <= p
        int j = 0;
#pragma unroll
        for (int st = 16; st > 0; st >>= 1) {
          const int q = __shfl_sync(0xffffffffu, incl, j + st - 1);
          if (q <= p) j += st;
        }
        const int ej = __shfl_sync(0xffffffffu, excl, j);
        const unsigned cj = __shfl_sync(0xffffffffu, cand, j);
        const unsigned xj = __shfl_sync(0xffffffffu, xs, j);
        if (p < total) {
          const int r = (int)__fns(cj, 0, p - ej + 1);
          if ((needm >> r) & 1u) {
            if (val[(size_t)(base + j) * 32 + r] & xj) hit |= 1u << r;
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

// Fold term(column) over the set columns of this lane's row words in tiles
// [t0, t1) (row r, and r + 32 for b = 64), for semirings whose value comes
// from a gather at the column (x[j], dist[j], labels[j] ...).  U tiles per
// step: their block-column indices and row words are loaded together, then
// the first set column of every word is gathered together (U or 2U
// independent loads in flight); further set columns of a word (rare in
// sparse tiles) follow one at a time.  term(idx) returns the value at global
// column idx; comb(acc, value) folds it into acc.  Words are left-aligned
// in 32 bits for b <= 32 (64 for b = 64) so that column 0 is the top bit.
template <int B, int U, typename Acc, typename Term, typename Comb>
__device__ __forceinline__ void fold_row_cols(const GView& v, int t0, int t1, int r, Term term,
                                              Comb comb, Acc& acc0, Acc& acc1) {
  using WT = typename Word<B>::T;
  using L = Lay<B>;
  using T = decltype(term(0ll));
  using AW = typename std::conditional<(B > 32), unsigned long long, unsigned>::type;
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
  // b = 32 tiles with occupancy words: a lane loads its row word only where
  // it is non-empty (the others are zero and fold nothing), so a sparse
  // tile costs the sectors of its non-empty rows.  The occupancy words run
  // one batch ahead of the row words they predicate.
  const unsigned* __restrict__ rm = B == 32 ? v.rowmask : nullptr;
  auto masks = [&](int tb, unsigned (&m)[U]) {
#pragma unroll
    for (int k = 0; k < U; ++k) m[k] = rm ? rm[tb + k] : ~0u;
  };
  // software pipeline: batch i+1's column indices and row words load while
  // batch i's gathers run
  auto load = [&](int tb, unsigned (&base)[U], AW (&a0)[U], AW (&a1)[U], const unsigned (&m)[U]) {
#pragma unroll
    for (int k = 0; k < U; ++k) {
      base[k] = (unsigned)v.colind[tb + k] * (unsigned)B;  // < 2^32: ncols is an int
      a0[k] = (m[k] >> (r & 31)) & 1u ? (AW)val[(size_t)(tb + k) * B + r] << (kBits - B) : (AW)0;
      a1[k] = L::RPL == 2 ? (AW)val[(size_t)(tb + k) * B + 32 + r] << (kBits - B) : (AW)0;
    }
  };
  int t = t0;
  unsigned base[U], mk[U];
  AW a0[U], a1[U];
  bool have = t + U <= t1;
  if (have) {
    masks(t, mk);
    load(t, base, a0, a1, mk);
    if (t + 2 * U <= t1) masks(t + U, mk);
  }
  while (have) {
    const int tn = t + U;
    const bool next = tn + U <= t1;
    unsigned nbase[U];
    AW n0[U], n1[U];
    if (next) {
      load(tn, nbase, n0, n1, mk);
      if (tn + 2 * U <= t1) masks(tn + U, mk);
    }
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
