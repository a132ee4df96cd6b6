// Bit-packed BSR SpMV ("BMV") kernels over the balanced work-item schedule.
//
// Reference kernels replaced (algorithm/bsrbmv.cu):
//   count      bmv{4,8,16,32,64}_sparse 262-474, *_sparse_new 2434-3094
//   masked     bmv32_sparse_bin_masked_v4 740-783, bmv4_..._v4 637-697
//   min-plus   bmv{4,32}_sparse_full_minplus 989-1138
//   float      bmv{4,32}_sparse_full 1156-1286
//   min-select bmv{4,8,16,32}_sparse_full_cc* 1367-2099
//
// Mapping: a group of W = min(b,32) lanes handles one work item (a block row
// or a chunk of a long block row); lane r owns tile row r (and r+32 for
// b = 64).  For every tile the lane loads its b-bit row word (the group's
// loads of one tile are contiguous) and combines it with the x segment of
// the tile's block column.  Items that cover a chunk of a split row write
// partial results to scratch; k_reduce_* combines them in slot order.
#include "scan.cuh"

namespace gbo {

namespace {

constexpr int kTPB = 256;

// Left-align a b-bit word in 32 or 64 bits so that column 0 is the MSB.
template <int B>
__device__ __forceinline__ unsigned long long align_word(typename Word<B>::T w) {
  return (unsigned long long)w << (64 - B);
}

// Iterate the set columns of a b-bit word (column 0 = MSB).
template <int B, typename F>
__device__ __forceinline__ void for_each_col(typename Word<B>::T w, F&& f) {
  unsigned long long a = align_word<B>(w);
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

// ----------------------------------------------------------------- count
template <int B, bool OUTF>
__global__ void __launch_bounds__(kTPB) k_count(GView v, const typename Word<B>::T* __restrict__ x,
                                                void* __restrict__ yv, int accumulate,
                                                int* __restrict__ scratch) {
  using WT = typename Word<B>::T;
  using L = Lay<B>;
  const unsigned lane = threadIdx.x & 31;
  const long long item = item_index(lane, L::W, L::G);
  if (item >= v.nitems) return;
  const int r = lane % L::W;
  const gbo_item it = v.items[item];
  const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
  unsigned acc0 = 0, acc1 = 0;
  int t = it.t0;
  for (; t + 4 <= it.t1; t += 4) {
    int c[4];
    WT w[4], w2[4], xs[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) c[k] = v.colind[t + k];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      w[k] = val[(size_t)(t + k) * B + r];
      if (L::RPL == 2) w2[k] = val[(size_t)(t + k) * B + 32 + r];
      xs[k] = x[c[k]];
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      acc0 += popc_w((WT)(w[k] & xs[k]));
      if (L::RPL == 2) acc1 += popc_w((WT)(w2[k] & xs[k]));
    }
  }
  for (; t < it.t1; ++t) {
    const int c = v.colind[t];
    const WT xs = x[c];
    acc0 += popc_w((WT)(val[(size_t)t * B + r] & xs));
    if (L::RPL == 2) acc1 += popc_w((WT)(val[(size_t)t * B + 32 + r] & xs));
  }
  if (it.slot >= 0) {
    scratch[(size_t)it.slot * B + r] = (int)acc0;
    if (L::RPL == 2) scratch[(size_t)it.slot * B + 32 + r] = (int)acc1;
    return;
  }
  const long long row0 = (long long)it.row * B + r;
  if (OUTF) {
    float* y = reinterpret_cast<float*>(yv);
    if (row0 < v.nrows) y[row0] = (accumulate ? y[row0] : 0.f) + (float)acc0;
    if (L::RPL == 2 && row0 + 32 < v.nrows) y[row0 + 32] = (accumulate ? y[row0 + 32] : 0.f) + (float)acc1;
  } else {
    int* y = reinterpret_cast<int*>(yv);
    if (row0 < v.nrows) y[row0] = (accumulate ? y[row0] : 0) + (int)acc0;
    if (L::RPL == 2 && row0 + 32 < v.nrows) y[row0 + 32] = (accumulate ? y[row0 + 32] : 0) + (int)acc1;
  }
}

// Narrow tiles (b = 4, 8, 16: 4, 8 or 32 bytes per tile): a warp per work
// item and a lane per tile, so that a lane reads its whole tile with one
// 4-, 8- or two 16-byte loads (consecutive lanes, consecutive tiles: the
// warp's loads are one contiguous run) instead of b lanes reading one or two
// bytes each.  The lane adds popc(row word & x segment) into b counters; the
// item's counters are summed across the warp at the end.
template <int B>
__device__ __forceinline__ void tile_counts(const void* __restrict__ val, long long t, unsigned xs,
                                            unsigned (&c)[B]) {
  if constexpr (B == 4) {
    const unsigned w = reinterpret_cast<const unsigned*>(val)[t];  // row r = byte r (low nibble)
#pragma unroll
    for (int r = 0; r < 4; ++r) c[r] += __popc((w >> (8 * r)) & xs & 0xfu);
  } else if constexpr (B == 8) {
    const unsigned long long w = reinterpret_cast<const unsigned long long*>(val)[t];  // row r = byte r
    const unsigned long long xr = 0x0101010101010101ull * (xs & 0xffu);
    const unsigned long long a = w & xr;
#pragma unroll
    for (int r = 0; r < 8; ++r) c[r] += __popc((unsigned)(a >> (8 * r)) & 0xffu);
  } else {
    const uint4* q = reinterpret_cast<const uint4*>(val) + 2 * t;  // row r = halfword r
    const uint4 lo = q[0], hi = q[1];
    const unsigned xx = (xs & 0xffffu) * 0x10001u;
    const unsigned w[8] = {lo.x, lo.y, lo.z, lo.w, hi.x, hi.y, hi.z, hi.w};
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      const unsigned a = w[k] & xx;
      c[2 * k] += __popc(a & 0xffffu);
      c[2 * k + 1] += __popc(a >> 16);
    }
  }
}

template <int B, bool OUTF>
__global__ void __launch_bounds__(kTPB) k_count_narrow(GView v, const typename Word<B>::T* __restrict__ x,
                                                       void* __restrict__ yv, int accumulate,
                                                       int* __restrict__ scratch) {
  const unsigned lane = threadIdx.x & 31;
  const long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (item >= v.nitems) return;
  const gbo_item it = v.items[item];
  unsigned c[B];
#pragma unroll
  for (int r = 0; r < B; ++r) c[r] = 0u;
  int t = it.t0 + (int)lane;
  for (; t + 32 < it.t1; t += 64) {  // two tiles per lane in flight
    const int c0 = v.colind[t], c1 = v.colind[t + 32];
    const unsigned x0 = x[c0], x1 = x[c1];
    tile_counts<B>(v.val, t, x0, c);
    tile_counts<B>(v.val, t + 32, x1, c);
  }
  if (t < it.t1) tile_counts<B>(v.val, t, x[v.colind[t]], c);
  unsigned mine = 0u;
#pragma unroll
  for (int r = 0; r < B; ++r) {
    const unsigned s = __reduce_add_sync(0xffffffffu, c[r]);
    if ((int)lane == r) mine = s;
  }
  if ((int)lane >= B) return;
  const int r = (int)lane;
  if (it.slot >= 0) {
    scratch[(size_t)it.slot * B + r] = (int)mine;
    return;
  }
  const long long row = (long long)it.row * B + r;
  if (row >= v.nrows) return;
  if (OUTF) {
    float* y = reinterpret_cast<float*>(yv);
    y[row] = (accumulate ? y[row] : 0.f) + (float)mine;
  } else {
    int* y = reinterpret_cast<int*>(yv);
    y[row] = (accumulate ? y[row] : 0) + (int)mine;
  }
}

template <int B, bool OUTF>
__global__ void k_count_reduce(GView v, const int* __restrict__ scratch, void* __restrict__ yv,
                               int accumulate) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)v.nsplit * B) return;
  const gbo_split sp = v.splits[gid / B];
  const int r = (int)(gid % B);
  long long s = 0;
  for (int q = 0; q < sp.nslots; ++q) s += scratch[(size_t)(sp.slot0 + q) * B + r];
  const long long row = (long long)sp.row * B + r;
  if (row >= v.nrows) return;
  if (OUTF) {
    float* y = reinterpret_cast<float*>(yv);
    y[row] = (accumulate ? y[row] : 0.f) + (float)s;
  } else {
    int* y = reinterpret_cast<int*>(yv);
    y[row] = (accumulate ? y[row] : 0) + (int)s;
  }
}

// ---------------------------------------------------------------- masked
// Assemble the b-bit output word of an item from per-lane predicates.
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

template <int B>
__global__ void __launch_bounds__(kTPB) k_masked(GView v, const typename Word<B>::T* __restrict__ x,
                                                 const typename Word<B>::T* __restrict__ mask,
                                                 typename Word<B>::T* __restrict__ out,
                                                 typename Word<B>::T* __restrict__ scratch) {
  using WT = typename Word<B>::T;
  using L = Lay<B>;
  const unsigned lane = threadIdx.x & 31;
  const long long item = item_index(lane, L::W, L::G);
  const long long warp0 = item - lane / L::W;
  if (warp0 >= v.nitems) return;  // whole warp idle (uniform)
  const bool active = item < v.nitems;
  const int r = lane % L::W;
  gbo_item it = active ? v.items[item] : gbo_item{0, 0, 0, -2};
  const WT full = (WT)~(WT)0 >> (sizeof(WT) * 8 - B);
  WT mk = 0;
  if (active && mask) mk = mask[it.row];
  bool p0 = false, p1 = false;
  if (active && (mk & full) != full) {  // uniform inside the item's lane group
    // masked-out rows need no answer: their output bit is cleared anyway;
    // tiles whose x segment is empty contribute nothing and are not read
    const bool need0 = !((mk >> (B - 1 - r)) & 1);
    const bool need1 = L::RPL == 2 && !((mk >> (B - 1 - (r + 32) % B)) & 1);
    pull_or_scan<B>(v, it.t0, it.t1, x, need0, need1, p0, p1, lane);
  }
  const WT word = gather_bits<B>(p0, p1, lane);
  if (!active || r != 0) return;
  if (it.slot >= 0)
    scratch[it.slot] = word;
  else
    out[it.row] = (WT)(word & ~mk & full);
}

template <int B>
__global__ void k_masked_reduce(GView v, const typename Word<B>::T* __restrict__ mask,
                                typename Word<B>::T* __restrict__ out,
                                const typename Word<B>::T* __restrict__ scratch) {
  using WT = typename Word<B>::T;
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= v.nsplit) return;
  const gbo_split sp = v.splits[i];
  const WT full = (WT)~(WT)0 >> (sizeof(WT) * 8 - B);
  WT w = 0;
  const WT mk = mask ? mask[sp.row] : (WT)0;
  if ((mk & full) != full)
    for (int q = 0; q < sp.nslots; ++q) w |= scratch[sp.slot0 + q];
  out[sp.row] = (WT)(w & ~mk & full);
}

// -------------------------------------------------------- value semirings
enum Semiring { SR_MINPLUS = 0, SR_MINSEL = 1, SR_FLOAT = 2 };

// V = element type of x and y; A = accumulator (fp32 sums accumulate in fp64
// so that rows with 10^4+ terms keep ~1e-7 relative accuracy).
template <int SR> struct SRT;
template <> struct SRT<SR_MINPLUS> { using V = uint32_t; using A = uint32_t; };
template <> struct SRT<SR_MINSEL> { using V = int32_t; using A = int32_t; };
template <> struct SRT<SR_FLOAT> { using V = float; using A = double; };

template <int SR>
__device__ __forceinline__ typename SRT<SR>::A sr_identity() {
  if (SR == SR_FLOAT) return (typename SRT<SR>::A)0;
  return (typename SRT<SR>::A)kINF;
}

template <int SR>
__device__ __forceinline__ void sr_combine(typename SRT<SR>::A& a, typename SRT<SR>::A b) {
  if (SR == SR_FLOAT) a += b;
  else a = min(a, b);
}

// The contribution of x[j] to a row.
template <int SR>
__device__ __forceinline__ typename SRT<SR>::A sr_term(const typename SRT<SR>::V* __restrict__ x,
                                                       const float* __restrict__ scale, long long j) {
  if (SR == SR_MINPLUS) {
    uint32_t d = ((const uint32_t*)x)[j];
    return d >= (uint32_t)kINF ? (uint32_t)kINF : d + 1u;
  } else if (SR == SR_MINSEL) {
    return (typename SRT<SR>::A)x[j];
  } else {
    float f = ((const float*)x)[j];
    return (typename SRT<SR>::A)(scale ? f * scale[j] : f);
  }
}

struct SrParams {
  float alpha, add;
  const float* scale;
  const int* degptr;  // when set: x[j] / (degptr[j+1] - degptr[j]) (the reference's form)
};

// Float term with the per-column degree read from a CSR row pointer at every
// set bit, as bmv32_sparse_full does (algorithm/bsrbmv.cu:1277).
__device__ __forceinline__ double float_term_deg(const float* __restrict__ x,
                                                 const int* __restrict__ degptr, long long j) {
  const int d = degptr[j + 1] - degptr[j];
  return d > 0 ? (double)(x[j] / (float)d) : 0.0;
}

template <int SR>
__device__ __forceinline__ typename SRT<SR>::V sr_finish(typename SRT<SR>::A acc,
                                                         const typename SRT<SR>::V* __restrict__ x,
                                                         long long row, const SrParams& p) {
  if (SR == SR_MINPLUS) {
    uint32_t d = ((const uint32_t*)x)[row];  // the (P + I) diagonal term
    return (typename SRT<SR>::V)min((uint32_t)acc, d);
  } else if (SR == SR_FLOAT) {
    return (typename SRT<SR>::V)((double)p.alpha * (double)acc + (double)p.add);
  }
  return (typename SRT<SR>::V)acc;
}

template <int B, int SR>
__global__ void __launch_bounds__(kTPB) k_semiring(GView v, const typename SRT<SR>::V* __restrict__ x,
                                                   typename SRT<SR>::V* __restrict__ y, SrParams p,
                                                   typename SRT<SR>::A* __restrict__ scratch) {
  using WT = typename Word<B>::T;
  using A = typename SRT<SR>::A;
  using L = Lay<B>;
  const unsigned lane = threadIdx.x & 31;
  const long long item = item_index(lane, L::W, L::G);
  if (item >= v.nitems) return;
  const int r = lane % L::W;
  const gbo_item it = v.items[item];
  A acc0 = sr_identity<SR>(), acc1 = sr_identity<SR>();
  auto comb = [](A& a, A b) { sr_combine<SR>(a, b); };
  if (SR == SR_FLOAT && p.degptr)
    fold_row_cols<B, 4>(v, it.t0, it.t1, v.item_wbase ? v.item_wbase[item] : 0ll, r,
                        [&](long long j) { return (A)float_term_deg((const float*)x, p.degptr, j); },
                        comb, acc0, acc1);
  else
    fold_row_cols<B, 4>(v, it.t0, it.t1, v.item_wbase ? v.item_wbase[item] : 0ll, r, [&](long long j) { return sr_term<SR>(x, p.scale, j); },
                        comb, acc0, acc1);
  if (it.slot >= 0) {
    scratch[(size_t)it.slot * B + r] = acc0;
    if (L::RPL == 2) scratch[(size_t)it.slot * B + 32 + r] = acc1;
    return;
  }
  const long long row0 = (long long)it.row * B + r;
  if (row0 < v.nrows) y[row0] = sr_finish<SR>(acc0, x, row0, p);
  if (L::RPL == 2 && row0 + 32 < v.nrows) y[row0 + 32] = sr_finish<SR>(acc1, x, row0 + 32, p);
}

template <int B, int SR>
__global__ void k_semiring_reduce(GView v, const typename SRT<SR>::V* __restrict__ x,
                                  typename SRT<SR>::V* __restrict__ y, SrParams p,
                                  const typename SRT<SR>::A* __restrict__ scratch) {
  using A = typename SRT<SR>::A;
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)v.nsplit * B) return;
  const gbo_split sp = v.splits[gid / B];
  const int r = (int)(gid % B);
  A acc = sr_identity<SR>();
  for (int q = 0; q < sp.nslots; ++q) sr_combine<SR>(acc, scratch[(size_t)(sp.slot0 + q) * B + r]);
  const long long row = (long long)sp.row * B + r;
  if (row < v.nrows) y[row] = sr_finish<SR>(acc, x, row, p);
}

// ---------------------------------------------------- transposed float BMV
__global__ void k_fill_f32(float* __restrict__ y, long long n, float v) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    y[i] = v;
}

template <int B>
__global__ void __launch_bounds__(kTPB) k_float_t(GView v, const float* __restrict__ x,
                                                  const float* __restrict__ scale, float alpha,
                                                  float* __restrict__ y) {
  using WT = typename Word<B>::T;
  using L = Lay<B>;
  const unsigned lane = threadIdx.x & 31;
  const long long item = item_index(lane, L::W, L::G);
  if (item >= v.nitems) return;
  const int r = lane % L::W;
  const gbo_item it = v.items[item];
  const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
  const long long row0 = (long long)it.row * B + r;
  float xr0 = 0.f, xr1 = 0.f;
  if (row0 < v.nrows) xr0 = alpha * x[row0] * (scale ? scale[row0] : 1.f);
  if (L::RPL == 2 && row0 + 32 < v.nrows) xr1 = alpha * x[row0 + 32] * (scale ? scale[row0 + 32] : 1.f);
  if (xr0 == 0.f && xr1 == 0.f) return;
  for (int t = it.t0; t < it.t1; ++t) {
    const long long base = (long long)v.colind[t] * B;
    if (xr0 != 0.f) {
      const WT w0 = val[(size_t)t * B + r];
      for_each_col<B>(w0, [&](int j) { atomicAdd(y + base + j, xr0); });
    }
    if (L::RPL == 2 && xr1 != 0.f) {
      const WT w1 = val[(size_t)t * B + 32 + r];
      for_each_col<B>(w1, [&](int j) { atomicAdd(y + base + j, xr1); });
    }
  }
}

template <int B>
unsigned grid_items(const GView& v) {
  long long warps = ((long long)v.nitems + Lay<B>::G - 1) / Lay<B>::G;
  return blocks_for_warps(warps, kTPB / 32);
}

// ------------------------------------------------------------- launchers
template <int B>
int count_impl(const GView& v, const void* x, void* y, int out_type, int accumulate,
               int* scratch, cudaStream_t s) {
  using WT = typename Word<B>::T;
  if (v.nitems > 0) {
    // whole-tile loads need the tile array aligned to a tile (4, 8 or 16
    // bytes); a caller's wrapped B2SR may not be
    bool narrow = false;
    if constexpr (B <= 16) {
      constexpr uintptr_t kAlign = B == 4 ? 4 : B == 8 ? 8 : 16;
      narrow = (reinterpret_cast<uintptr_t>(v.val) % kAlign) == 0;
      if (narrow) {
        const unsigned grid = blocks_for_warps(v.nitems, kTPB / 32);
        if (out_type == GBO_OUT_F32)
          k_count_narrow<B, true><<<grid, kTPB, 0, s>>>(v, (const WT*)x, y, accumulate, scratch);
        else
          k_count_narrow<B, false><<<grid, kTPB, 0, s>>>(v, (const WT*)x, y, accumulate, scratch);
      }
    }
    if (!narrow) {
      if (out_type == GBO_OUT_F32)
        k_count<B, true><<<grid_items<B>(v), kTPB, 0, s>>>(v, (const WT*)x, y, accumulate, scratch);
      else
        k_count<B, false><<<grid_items<B>(v), kTPB, 0, s>>>(v, (const WT*)x, y, accumulate, scratch);
    }
  }
  if (v.nsplit > 0) {
    unsigned g = blocks_for((long long)v.nsplit * B, 256);
    if (out_type == GBO_OUT_F32)
      k_count_reduce<B, true><<<g, 256, 0, s>>>(v, scratch, y, accumulate);
    else
      k_count_reduce<B, false><<<g, 256, 0, s>>>(v, scratch, y, accumulate);
  }
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

template <int B>
int masked_impl(const GView& v, const void* x, const void* mask, void* out, void* scratch,
                cudaStream_t s) {
  using WT = typename Word<B>::T;
  if (v.nitems > 0)
    k_masked<B><<<grid_items<B>(v), kTPB, 0, s>>>(v, (const WT*)x, (const WT*)mask, (WT*)out,
                                                  (WT*)scratch);
  if (v.nsplit > 0)
    k_masked_reduce<B><<<blocks_for(v.nsplit, 256), 256, 0, s>>>(v, (const WT*)mask, (WT*)out,
                                                                 (const WT*)scratch);
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

template <int B, int SR>
int semiring_impl(const GView& v, const void* x, void* y, SrParams p, void* scratch,
                  cudaStream_t s) {
  using V = typename SRT<SR>::V;
  using A = typename SRT<SR>::A;
  if (v.nitems > 0)
    k_semiring<B, SR><<<grid_items<B>(v), kTPB, 0, s>>>(v, (const V*)x, (V*)y, p, (A*)scratch);
  if (v.nsplit > 0)
    k_semiring_reduce<B, SR><<<blocks_for((long long)v.nsplit * B, 256), 256, 0, s>>>(
        v, (const V*)x, (V*)y, p, (const A*)scratch);
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

template <int B>
int float_t_impl(const GView& v, const float* x, float* y, float alpha, const float* scale,
                 float add, cudaStream_t s) {
  if (v.ncols > 0) {
    unsigned g = blocks_for(v.ncols, 256);
    k_fill_f32<<<g > 4096u ? 4096u : g, 256, 0, s>>>(y, v.ncols, add);
  }
  if (v.nitems > 0) k_float_t<B><<<grid_items<B>(v), kTPB, 0, s>>>(v, x, scale, alpha, y);
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

}  // namespace

GView view_of(const gbo_graph* g) {
  GView v;
  v.nrows = g->nrows;
  v.ncols = g->ncols;
  v.nbr = g->nbr;
  v.nbc = g->nbc;
  v.rowptr = g->rowptr;
  v.colind = g->colind;
  v.val = g->val;
  v.items = g->items;
  v.nitems = g->nitems;
  v.splits = g->splits;
  v.nsplit = g->nsplit;
  v.rowmask = g->rowmask;
  v.rowword = g->rowword;
  v.item_wbase = g->item_wbase;
  v.rws_head = g->rws_head;
  v.rws_tail = g->rws_tail;
  v.rws_tail_ptr = g->rws_tail_ptr;
  v.rws_nlong = g->rws_nlong;
  v.rws_nchunk = g->rws_nchunk;
  v.rws_ntail = g->rws_ntail;
  v.rws_long_row = g->rws_long_row;
  v.rws_long_chunk0 = g->rws_long_chunk0;
  v.rws_chunk_row = g->rws_chunk_row;
  v.rws_chunk_beg = g->rws_chunk_beg;
  v.rws_chunk_end = g->rws_chunk_end;
  v.rws_longbits = g->rws_longbits;
  return v;
}

size_t bmv_scratch_bytes(const gbo_graph* g) {
  // count: int per slot row; semirings: up to 8-byte accumulators; masked:
  // one word per slot
  return (size_t)g->nslots * (size_t)g->b * 8 + 64;
}

#define GBO_DISPATCH_B(b, CALL) \
  switch (b) {                  \
    case 4: { constexpr int B = 4; CALL; } break;   \
    case 8: { constexpr int B = 8; CALL; } break;   \
    case 16: { constexpr int B = 16; CALL; } break; \
    case 32: { constexpr int B = 32; CALL; } break; \
    default: { constexpr int B = 64; CALL; } break; \
  }

int bmv_count(const gbo_graph* g, const void* x, void* y, int out_type, int accumulate,
              void* scratch, cudaStream_t s) {
  GView v = view_of(g);
  int st = GBO_OK;
  GBO_DISPATCH_B(g->b, st = count_impl<B>(v, x, y, out_type, accumulate, (int*)scratch, s));
  return st;
}

int bmv_masked(const gbo_graph* g, const void* x, const void* mask, void* out, void* scratch,
               cudaStream_t s) {
  GView v = view_of(g);
  int st = GBO_OK;
  GBO_DISPATCH_B(g->b, st = masked_impl<B>(v, x, mask, out, scratch, s));
  return st;
}

int bmv_minplus(const gbo_graph* g, const uint32_t* x, uint32_t* y, void* scratch, cudaStream_t s) {
  GView v = view_of(g);
  SrParams p{1.f, 0.f, nullptr, nullptr};
  int st = GBO_OK;
  GBO_DISPATCH_B(g->b, st = (semiring_impl<B, SR_MINPLUS>(v, x, y, p, scratch, s)));
  return st;
}

int bmv_minselect(const gbo_graph* g, const int32_t* x, int32_t* y, void* scratch, cudaStream_t s) {
  GView v = view_of(g);
  SrParams p{1.f, 0.f, nullptr, nullptr};
  int st = GBO_OK;
  GBO_DISPATCH_B(g->b, st = (semiring_impl<B, SR_MINSEL>(v, x, y, p, scratch, s)));
  return st;
}

int bmv_float(const gbo_graph* g, const float* x, float* y, float alpha, const float* scale,
              float add, void* scratch, cudaStream_t s, const int* degptr) {
  GView v = view_of(g);
  SrParams p{alpha, add, scale, degptr};
  int st = GBO_OK;
  GBO_DISPATCH_B(g->b, st = (semiring_impl<B, SR_FLOAT>(v, x, y, p, scratch, s)));
  return st;
}

int bmv_float_transposed(const gbo_graph* g, const float* x, float* y, float alpha,
                         const float* scale, float add, cudaStream_t s) {
  GView v = view_of(g);
  int st = GBO_OK;
  GBO_DISPATCH_B(g->b, st = float_t_impl<B>(v, x, y, alpha, scale, add, s));
  return st;
}

}  // namespace gbo
