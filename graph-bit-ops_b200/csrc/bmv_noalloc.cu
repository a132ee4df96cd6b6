// BMV count straight from caller-owned B2SR buffers, allocating nothing.
//
// gbo_bmv_count runs over a graph handle, whose creation allocates the
// balanced schedule and a split-row workspace.  Some callers cannot do that:
// a host framework that owns every device byte through its own pool (a
// hard budget, no allocations behind its back), or a latency-bound thread
// sharing the GPU with other streams, where cudaMalloc / cudaFree would
// synchronise the whole device.  This entry point takes the bare B2SR
// arrays (as the reference's bmv{b}_sparse launches do) and allocates no
// device or host memory at any call.
//
// Work split: the tile range [0, nblocks) is cut into chunks of `chunk`
// tiles, sized per call: enough chunks for every lane group the GPU holds
// at once (so that a graph of 10^5 tiles is not one warp per SM), between
// 64 and 32768 / b tiles; a group of W = min(b, 32) lanes takes one chunk (lane r
// owns tile row r, and r + 32 for b = 64).  A block row that lies wholly
// inside a chunk is written to y directly.  A block row that crosses a
// chunk boundary leaves one partial per chunk it touches in a file-scope
// __device__ array (the scratch below); a second kernel adds the partials
// of each such row in chunk order and writes y.  Per chunk there are two
// partial slots of b ints:
//   slot 0  the chunk's first row, when that row began in an earlier chunk
//   slot 1  the chunk's last row, when that row began in this chunk and
//           continues into the next one
// so a row split over chunks cs..ce reads slot 1 of cs and slot 0 of
// cs+1..ce.  Every slot the second kernel reads is written by the first
// kernel of the same call, so nothing in the scratch has to start at zero.
//
// Input: a well-formed B2SR (rowptr non-decreasing from 0 with rowptr[nbr]
// == nblocks, block columns below ceil(ncols / b)).  Block columns out of
// range read as an empty x segment; a malformed row pointer is not detected
// (that would need a device-to-host read) and leaves y undefined.
//
// Limits: the scratch holds kScratchInts ints (8 MiB), so a call accepts at
// most kScratchInts / (2 b) chunks, i.e. 2^35 / b^2 tiles (33,554,432 at
// b = 32; 8,388,608 at b = 64); larger graphs are rejected with
// GBO_ERR_UNSUPPORTED before anything is launched.  All calls in a process
// share the one array per device, so two calls whose kernels may overlap
// (different streams, or different host threads without ordering) race on
// it and can return wrong counts: order them on one stream.
#include "common.cuh"

#include <mutex>

namespace gbo {

namespace {

constexpr int kTPB = 256;
constexpr int kMaxDevices = 64;
constexpr long long kScratchInts = 2ll * 1024 * 1024;  // 8 MiB

__device__ __align__(256) int g_scratch[kScratchInts];

template <int B>
struct NL {  // lane layout: W lanes per chunk, G chunks per warp
  static constexpr int W = B >= 32 ? 32 : B;
  static constexpr int G = 32 / W;
  static constexpr int RPL = B > 32 ? 2 : 1;
};

// Tiles per chunk: at most 32768 / b (1024 tiles of 32 words at b = 32),
// which bounds a call's chunks by the scratch, and at least kMinChunk.
template <int B>
constexpr long long kChunk = 32768 / B;
constexpr long long kMinChunk = 64;

__device__ __forceinline__ int count_bits(unsigned long long w) { return __popcll(w); }

// Largest block row R with rowptr[R] <= t (t < rowptr[nbr]).
__device__ __forceinline__ int row_of(const int* __restrict__ rowptr, int nbr, long long t) {
  int lo = 0, hi = nbr;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (rowptr[mid] <= t) lo = mid;
    else hi = mid;
  }
  return lo;
}

template <int B, bool OUTF>
__device__ __forceinline__ void put(void* yv, long long row, long long nrows, long long add,
                                   int accumulate) {
  if (row >= nrows) return;
  if (OUTF) {
    float* y = reinterpret_cast<float*>(yv);
    y[row] = (accumulate ? y[row] : 0.f) + (float)add;
  } else {
    int* y = reinterpret_cast<int*>(yv);
    y[row] = (accumulate ? y[row] : 0) + (int)add;
  }
}

template <int B, bool OUTF>
__global__ void __launch_bounds__(kTPB) k_count_chunks(
    const int* __restrict__ rowptr, const int* __restrict__ colind,
    const typename Word<B>::T* __restrict__ val, const typename Word<B>::T* __restrict__ x,
    void* __restrict__ y, int nrows, int nbr, int nbc, long long nblk, long long nchunks, long long chunk,
    int accumulate, int* __restrict__ scratch) {
  using WT = typename Word<B>::T;
  using L = NL<B>;
  const unsigned lane = threadIdx.x & 31;
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long c = warp * L::G + lane / L::W;
  if (c >= nchunks) return;
  const int r = lane % L::W;
  const long long t0 = c * chunk;
  const long long t1 = t0 + chunk < nblk ? t0 + chunk : nblk;
  int R = row_of(rowptr, nbr, t0);
  long long t = t0;
  while (t < t1 && R < nbr) {
    const long long rs = rowptr[R], re = rowptr[R + 1];
    const long long e = re < t1 ? re : t1;
    unsigned acc0 = 0, acc1 = 0;
    for (; t + 4 <= e; t += 4) {
      WT w[4], w2[4], xs[4];
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        w[k] = val[(size_t)(t + k) * B + r];
        if (L::RPL == 2) w2[k] = val[(size_t)(t + k) * B + 32 + r];
        const int cc = colind[t + k];
        xs[k] = (unsigned)cc < (unsigned)nbc ? x[cc] : (WT)0;
      }
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        acc0 += count_bits((unsigned long long)(WT)(w[k] & xs[k]));
        if (L::RPL == 2) acc1 += count_bits((unsigned long long)(WT)(w2[k] & xs[k]));
      }
    }
    for (; t < e; ++t) {
      const int cc = colind[t];
      const WT xs = (unsigned)cc < (unsigned)nbc ? x[cc] : (WT)0;
      acc0 += count_bits((unsigned long long)(WT)(val[(size_t)t * B + r] & xs));
      if (L::RPL == 2) acc1 += count_bits((unsigned long long)(WT)(val[(size_t)t * B + 32 + r] & xs));
    }
    if (rs >= t0 && re <= t1) {  // whole row inside this chunk
      put<B, OUTF>(y, (long long)R * B + r, nrows, acc0, accumulate);
      if (L::RPL == 2) put<B, OUTF>(y, (long long)R * B + 32 + r, nrows, acc1, accumulate);
    } else {
      const long long slot = c * 2 + (rs < t0 ? 0 : 1);
      scratch[slot * B + r] = (int)acc0;
      if (L::RPL == 2) scratch[slot * B + 32 + r] = (int)acc1;
    }
    // next non-empty block row (empty rows are written by k_count_rows)
    ++R;
    while (R < nbr && rowptr[R + 1] <= t) ++R;
  }
}

// One thread per (block row, tile row): empty block rows get 0 (or keep y
// when accumulating); rows split over chunks get the sum of their partials.
template <int B, bool OUTF>
__global__ void k_count_rows(const int* __restrict__ rowptr, void* __restrict__ y, int nrows,
                             int nbr, long long nblk, long long chunk, int accumulate,
                             const int* __restrict__ scratch) {
  const long long gid = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (gid >= (long long)nbr * B) return;
  const int R = (int)(gid / B);
  const int r = (int)(gid % B);
  const long long rs = rowptr[R], re = rowptr[R + 1];
  if (rs < 0 || rs > re || re > nblk) return;  // not a valid B2SR row pointer
  if (rs == re) {
    put<B, OUTF>(y, (long long)R * B + r, nrows, 0, accumulate);
    return;
  }
  const long long cs = rs / chunk, ce = (re - 1) / chunk;
  if (cs == ce) return;  // written by k_count_chunks
  long long s = scratch[(cs * 2 + 1) * B + r];
  for (long long q = cs + 1; q <= ce; ++q) s += scratch[(q * 2) * B + r];
  put<B, OUTF>(y, (long long)R * B + r, nrows, s, accumulate);
}

template <int B>
int launch(int nrows, int nbr, int nbc, long long nblk, const int* rowptr, const int* colind, const void* val,
           const void* x, void* y, int out_type, int accumulate, int* scratch, cudaStream_t s) {
  using WT = typename Word<B>::T;
  using L = NL<B>;
  // enough chunks for every lane group resident on the GPU, within
  // [kMinChunk, kChunk<B>] tiles (the upper bound keeps 2 * nchunks * b
  // partial ints inside the scratch: nblk was checked against it)
  const long long groups = (long long)num_sms() * 64 * L::G;
  long long chunk = (nblk + groups - 1) / groups;
  chunk = chunk < kMinChunk ? kMinChunk : chunk > kChunk<B> ? kChunk<B> : chunk;
  const long long fit = (nblk * 2 * B + kScratchInts - 1) / kScratchInts;  // chunks must fit the scratch
  if (chunk < fit) chunk = fit;
  const long long nchunks = (nblk + chunk - 1) / chunk;
  if (nchunks > 0) {
    const long long warps = (nchunks + L::G - 1) / L::G;
    const unsigned grid = blocks_for_warps(warps, kTPB / 32);
    if (out_type == GBO_OUT_F32)
      k_count_chunks<B, true><<<grid, kTPB, 0, s>>>(rowptr, colind, (const WT*)val, (const WT*)x, y,
                                                    nrows, nbr, nbc, nblk, nchunks, chunk, accumulate, scratch);
    else
      k_count_chunks<B, false><<<grid, kTPB, 0, s>>>(rowptr, colind, (const WT*)val, (const WT*)x, y,
                                                     nrows, nbr, nbc, nblk, nchunks, chunk, accumulate, scratch);
  }
  if (nbr > 0) {
    const unsigned grid = blocks_for((long long)nbr * B, kTPB);
    if (out_type == GBO_OUT_F32)
      k_count_rows<B, true><<<grid, kTPB, 0, s>>>(rowptr, y, nrows, nbr, nblk, chunk, accumulate, scratch);
    else
      k_count_rows<B, false><<<grid, kTPB, 0, s>>>(rowptr, y, nrows, nbr, nblk, chunk, accumulate, scratch);
  }
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

// Device address of g_scratch, looked up once per device on first use.
std::mutex g_mu;
int* g_addr[kMaxDevices] = {};

int scratch_for_current_device(int** out) {
  int dev = -1;
  GBO_CUDA_TRY(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(GBO_ERR_UNSUPPORTED, "device ordinal above 63");
  std::lock_guard<std::mutex> lk(g_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGetSymbolAddress(bmv no-alloc scratch)");
    g_addr[dev] = static_cast<int*>(p);
  }
  *out = g_addr[dev];
  return GBO_OK;
}

}  // namespace

long long bmv_noalloc_max_tiles(int b) {
  const long long chunk = 32768 / b;
  return kScratchInts / (2ll * b) * chunk;
}

}  // namespace gbo

using namespace gbo;

extern "C" int gbo_bmv_count_noalloc(int nrows, int ncols, int tile_bits, int nblocks,
                                     const int* d_bsrRowPtr, const int* d_bsrColInd,
                                     const void* d_bsrVal, const void* d_x_bits, void* d_y,
                                     int out_type, int accumulate, gbo_stream_t stream) {
  clear_error();
  if (tile_bits != 4 && tile_bits != 8 && tile_bits != 16 && tile_bits != 32 && tile_bits != 64)
    return fail(GBO_ERR_INVALID, "tile_bits must be 4, 8, 16, 32 or 64");
  if (nrows < 0 || ncols < 0 || nblocks < 0) return fail(GBO_ERR_INVALID, "negative size");
  if (out_type != GBO_OUT_I32 && out_type != GBO_OUT_F32) return fail(GBO_ERR_INVALID, "bad out_type");
  const long long max_tiles = bmv_noalloc_max_tiles(tile_bits);
  if (nblocks > max_tiles)
    return fail(GBO_ERR_UNSUPPORTED,
                "gbo_bmv_count_noalloc: " + std::to_string(nblocks) + " tiles exceed the " +
                    std::to_string(max_tiles) + " that its fixed 8 MiB scratch covers at b=" +
                    std::to_string(tile_bits) + "; use gbo_bmv_count on a graph handle");
  // block counts in 64-bit: nrows + tile_bits - 1 overflows int near INT_MAX
  const int nbr = (int)(((long long)nrows + tile_bits - 1) / tile_bits);
  const int nbc = (int)(((long long)ncols + tile_bits - 1) / tile_bits);
  if (nbr == 0) return GBO_OK;
  if (!d_bsrRowPtr || !d_y || (nblocks > 0 && (!d_bsrColInd || !d_bsrVal || !d_x_bits)))
    return fail(GBO_ERR_INVALID, "NULL pointer");
  int* scratch = nullptr;
  GBO_TRY(scratch_for_current_device(&scratch));
  cudaStream_t s = as_stream(stream);
  const long long nblk = nblocks;
  switch (tile_bits) {
    case 4: return launch<4>(nrows, nbr, nbc, nblk, d_bsrRowPtr, d_bsrColInd, d_bsrVal, d_x_bits, d_y, out_type, accumulate, scratch, s);
    case 8: return launch<8>(nrows, nbr, nbc, nblk, d_bsrRowPtr, d_bsrColInd, d_bsrVal, d_x_bits, d_y, out_type, accumulate, scratch, s);
    case 16: return launch<16>(nrows, nbr, nbc, nblk, d_bsrRowPtr, d_bsrColInd, d_bsrVal, d_x_bits, d_y, out_type, accumulate, scratch, s);
    case 32: return launch<32>(nrows, nbr, nbc, nblk, d_bsrRowPtr, d_bsrColInd, d_bsrVal, d_x_bits, d_y, out_type, accumulate, scratch, s);
    default: return launch<64>(nrows, nbr, nbc, nblk, d_bsrRowPtr, d_bsrColInd, d_bsrVal, d_x_bits, d_y, out_type, accumulate, scratch, s);
  }
}
