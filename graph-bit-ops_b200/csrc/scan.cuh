// Shared device building blocks of the pull kernels: the lane layout of a
// work item and the batched Boolean (OR.AND) scan of a block row.
#pragma once

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

// Boolean pull over tiles [t0, t1) of one block row for the rows this lane
// owns: p0 |= (row word & x[colind]) != 0 (p1 for row r+32 when b = 64).
// need0/need1 say whether the row still needs an answer; a row stops loading
// once it has one, and the group leaves the row as soon as all its rows are
// answered.  Block-column indices are read W at a time (one coalesced load),
// their x words gathered in parallel, and only tiles with a non-empty x
// segment are fetched, four tile words in flight per lane.
template <int B>
__device__ __forceinline__ void pull_or_scan(const GView& v, int t0, int t1,
                                             const typename Word<B>::T* __restrict__ x,
                                             bool need0, bool need1, bool& p0, bool& p1,
                                             unsigned lane) {
  using WT = typename Word<B>::T;
  using L = Lay<B>;
  constexpr int W = L::W;
  const unsigned gmask = group_mask<B>(lane);
  const int r = lane % W;
  const unsigned gshift = (lane / W) * W;
  const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
  constexpr int U = 8;  // tile words in flight per lane
  // the next batch's block-column indices are loaded while this batch runs
  int cnext = (t0 + r < t1) ? v.colind[t0 + r] : -1;
  for (int base = t0; base < t1; base += W) {
    const int cb = cnext;
    cnext = (base + W + r < t1) ? v.colind[base + W + r] : -1;
    const WT xs = cb >= 0 ? x[cb] : (WT)0;
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

}  // namespace gbo
