// Triangle counting by masked binary SpGEMM on B2SR tiles.
//
// Reference: bmm32_sparse_masked_v5 (bsrbmm/bsrbmm.cu:1214-1265) computes
// sum over mask tiles (I,K) of L of sum_r sum_c M[r][c] * (L L^T)[I*b+r][K*b+c],
// looking up B = L^T tiles (col layout) by binary search, and reduces into an
// int32 (overflows past 2^31 triangles, bsrbmm/tc.cu:861-863).
//
// Here the L^T operand is never built: the col-layout tile (J,K) of L^T has
// the same words as the row-layout tile (K,J) of L, so the intersection of
// block rows I and K of L (restricted to block columns <= K) gives every
// contributing pair.  One warp per mask tile probes the shorter of the two
// sorted column lists into the longer with binary searches (32 probes per
// step), and for each hit computes
//   sum_r sum_{c in M_r} popc(A_(I,J)[r] & A_(K,J)[c])
// with the K-tile rows broadcast by warp shuffles.  The count is uint64.
#include "bmv.cuh"

namespace gbo {

namespace {

constexpr int kTPB = 256;

__device__ __forceinline__ int lower_bound_dev(const int* __restrict__ a, int lo, int hi, int key) {
  while (lo < hi) {
    int mid = (lo + hi) >> 1;
    if (a[mid] < key) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// Block row of every tile (computed once per graph, from the work items).
__global__ void k_tile_row(GView v, int* __restrict__ tile_row) {
  const long long item = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  if (item >= v.nitems) return;
  const gbo_item it = v.items[item];
  for (int t = it.t0 + (int)(threadIdx.x & 31); t < it.t1; t += 32) tile_row[t] = it.row;
}

// Mask tiles with at most kSparsePairs set bits take the lane-per-hit path:
// the (row, column) bits of the mask go to a per-warp list, and every lane
// with a hit sums popc(A[r] & B[c]) over the list for its own tile pair,
// loading just those rows -- hits of a probe round proceed side by side
// instead of one after another.  Denser masks broadcast the K-tile rows.
constexpr int kSparsePairs = 16;

template <int B>
__global__ void __launch_bounds__(kTPB) k_tc(GView v, long long nblk, const int* __restrict__ tile_row,
                                             int skip_dense, unsigned long long* __restrict__ count) {
  using WT = typename Word<B>::T;
  constexpr int RPL = B > 32 ? 2 : 1;
  __shared__ short pairs_sh[kTPB / 32][kSparsePairs];  // (r << 7) | c
  const unsigned lane = threadIdx.x & 31;
  short* pairs = pairs_sh[threadIdx.x >> 5];
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const WT* __restrict__ val = reinterpret_cast<const WT*>(v.val);
  unsigned long long acc = 0;
  // mask tiles strided over the warps (hub rows spread out)
  for (long long m = warp; m < nblk; m += nwarps) {
    const int I = tile_row[m];
    const int K = v.colind[m];
    // mask rows of tile (I,K)
    WT M0 = 0, M1 = 0;
    if (lane < (unsigned)(B < 32 ? B : 32)) M0 = val[(size_t)m * B + lane];
    if (RPL == 2) M1 = val[(size_t)m * B + 32 + lane];
    // union of the mask columns over the tile's rows
    unsigned long long U = (unsigned long long)M0 | (unsigned long long)M1;
    {
      unsigned lo = __reduce_or_sync(0xffffffffu, (unsigned)U);
      unsigned hi = __reduce_or_sync(0xffffffffu, (unsigned)(U >> 32));
      U = ((unsigned long long)hi << 32) | lo;
    }
    // mask bits as a list when the mask is sparse (lane order = row order)
    int npairs = -1;
    {
      const int c0 = popc_w(M0) + (RPL == 2 ? popc_w(M1) : 0);
      int incl = c0;
#pragma unroll
      for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, incl, o);
        if ((int)lane >= o) incl += y;
      }
      const int total = __shfl_sync(0xffffffffu, incl, 31);
      if (total <= kSparsePairs) {
        int pos = incl - c0;
        for (int h = 0; h < RPL; ++h) {
          const int r = (int)lane + 32 * h;
          unsigned long long w = (unsigned long long)(h ? M1 : M0) << (64 - B);
          while (w) {
            const int c = __clzll(w);
            w &= ~(0x8000000000000000ull >> c);
            pairs[pos++] = (short)((r << 7) | c);
          }
        }
        npairs = total;
      }
      __syncwarp();
    }
    if (npairs < 0 && skip_dense) continue;  // dense masks go to the tensor-core kernel
    // list A: row I, tiles with block column <= K  -> [rowptr[I], m]
    // list B: row K, all tiles (block columns <= K in a lower triangle)
    const int a0 = v.rowptr[I], a1 = (int)m + 1;
    const int b0 = v.rowptr[K], b1 = v.rowptr[K + 1];
    const bool probe_a = (a1 - a0) <= (b1 - b0);
    const int p0 = probe_a ? a0 : b0, p1 = probe_a ? a1 : b1;
    const int s0 = probe_a ? b0 : a0, s1 = probe_a ? b1 : a1;
    if constexpr (B == 32) {
      if (npairs < 0) {
        // dense 32x32 mask: lane r accumulates P[r][c] = sum over hits of
        // popc(A[r] & B[c]) for all 32 columns (B rows broadcast by 32
        // unrolled shuffles, no data-dependent loop), masked once at the end
        unsigned cm[32];
#pragma unroll
        for (int c = 0; c < 32; ++c) cm[c] = 0u;
        for (int base = p0; base < p1; base += 32) {
          const int p = base + (int)lane;
          int hit = -1;
          if (p < p1) {
            const int J = v.colind[p];
            const int q = lower_bound_dev(v.colind, s0, s1, J);
            if (q < s1 && v.colind[q] == J) hit = q;
          }
          unsigned found = __ballot_sync(0xffffffffu, hit >= 0);
          while (found) {
            const int src = __ffs(found) - 1;
            found &= found - 1;
            const int ph = __shfl_sync(0xffffffffu, p, src);
            const int qh = __shfl_sync(0xffffffffu, hit, src);
            const unsigned ar = (unsigned)val[(size_t)(probe_a ? ph : qh) * 32 + lane];
            const unsigned br = (unsigned)val[(size_t)(probe_a ? qh : ph) * 32 + lane];
#pragma unroll
            for (int c = 0; c < 32; ++c) cm[c] += __popc(ar & __shfl_sync(0xffffffffu, br, c));
          }
        }
        const unsigned mr = (unsigned)M0;
#pragma unroll
        for (int c = 0; c < 32; ++c) acc += ((mr >> (31 - c)) & 1u) ? cm[c] : 0u;
        continue;
      }
    }
    for (int base = p0; base < p1; base += 32) {
      const int p = base + (int)lane;
      int hit = -1;
      if (p < p1) {
        const int J = v.colind[p];
        const int q = lower_bound_dev(v.colind, s0, s1, J);
        if (q < s1 && v.colind[q] == J) hit = q;
      }
      unsigned found = __ballot_sync(0xffffffffu, hit >= 0);
      if (npairs >= 0) {  // sparse mask: each lane handles its own hit
        if (hit >= 0) {
          const int ia = probe_a ? p : hit;  // tile (I,J)
          const int ib = probe_a ? hit : p;  // tile (K,J)
          for (int k = 0; k < npairs; ++k) {
            const int pr = pairs[k];
            acc += popc_w((WT)(val[(size_t)ia * B + (pr >> 7)] & val[(size_t)ib * B + (pr & 127)]));
          }
        }
        continue;
      }
      while (found) {
        const int src = __ffs(found) - 1;
        found &= found - 1;
        const int ph = __shfl_sync(0xffffffffu, p, src);
        const int qh = __shfl_sync(0xffffffffu, hit, src);
        const int ia = probe_a ? ph : qh;  // tile (I,J)
        const int ib = probe_a ? qh : ph;  // tile (K,J)
        // only the rows that matter are loaded: A rows with mask bits, B
        // rows of the mask's columns (sparse tiles touch one or two sectors)
        WT A0 = 0, A1 = 0, Bw0 = 0, Bw1 = 0;
        if (lane < (unsigned)(B < 32 ? B : 32)) {
          if (M0) A0 = val[(size_t)ia * B + lane];
          if ((U >> (B - 1 - lane)) & 1ull) Bw0 = val[(size_t)ib * B + lane];
        }
        if (RPL == 2) {
          if (M1) A1 = val[(size_t)ia * B + 32 + lane];
          if ((U >> (31 - lane)) & 1ull) Bw1 = val[(size_t)ib * B + 32 + lane];
        }
        unsigned long long u = U << (64 - B);  // column c at bit 63-c
        while (u) {
          const int c = __clzll(u);
          u &= ~(0x8000000000000000ull >> c);
          WT bc;
          if (RPL == 2)
            bc = c < 32 ? (WT)__shfl_sync(0xffffffffu, (unsigned long long)Bw0, c)
                        : (WT)__shfl_sync(0xffffffffu, (unsigned long long)Bw1, c - 32);
          else
            bc = (WT)__shfl_sync(0xffffffffu, (unsigned)Bw0, c);
          if ((M0 >> (B - 1 - c)) & 1) acc += popc_w((WT)(A0 & bc));
          if (RPL == 2 && ((M1 >> (B - 1 - c)) & 1)) acc += popc_w((WT)(A1 & bc));
        }
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0 && acc) atomicAdd(count, acc);
}

// D += popc(A AND B) over 256-bit rows/columns: the 1-bit tensor-core MMA
// (m16n8k256, A row-major 16x256, B column-major 256x8, s32 accumulators).
// Fragments, with g = lane / 4 and q = lane % 4: a0 = A[g][32q..32q+31],
// a1 = A[g+8][same], a2 = A[g][128+32q..], a3 = A[g+8][128+32q..];
// b0 = B[32q..][g], b1 = B[128+32q..][g]; d0,d1 = D[g][2q, 2q+1],
// d2,d3 = D[g+8][2q, 2q+1].
__device__ __forceinline__ void mma_and_popc(int (&d)[4], unsigned a0, unsigned a1, unsigned a2,
                                             unsigned a3, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k256.row.col.s32.b1.b1.s32.and.popc "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+r"(d[0]), "+r"(d[1]), "+r"(d[2]), "+r"(d[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// Opt-in (GBO_FLAG_TC_MMA): on the configured graphs this path did not beat
// the CUDA-core one (king mesh b=32: 3.3 vs 3.6 ms but b=16 without it 2.1 ms;
// R-MAT 20 degree-ordered b=32: 25.8 vs 20.5 ms), so it is not the default.
// Dense 32x32 mask tiles (more than kSparsePairs bits) on the tensor cores:
// for a mask tile (I,K) the product P = sum_J A_IJ B_KJ^T over the hits J is
// a 32x32 AND-popc product with the hits' 32-bit rows laid side by side
// along k (8 hits per 256-bit step), then sum_{r,c} M[r][c] P[r][c].
__global__ void __launch_bounds__(kTPB) k_tc32_mma(GView v, long long nblk, const int* __restrict__ tile_row,
                                                   unsigned long long* __restrict__ count) {
  __shared__ int2 hits_sh[kTPB / 32][32];
  __shared__ uint32_t tiles_sh[kTPB / 32][2][8][32];  // A and B tiles of 8 hits
  const unsigned lane = threadIdx.x & 31;
  const int g = (int)(lane >> 2), q4 = (int)(lane & 3);
  int2* hits = hits_sh[threadIdx.x >> 5];
  uint32_t (*sA)[32] = tiles_sh[threadIdx.x >> 5][0];
  uint32_t (*sB)[32] = tiles_sh[threadIdx.x >> 5][1];
  const long long warp = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const long long nwarps = ((long long)gridDim.x * blockDim.x) >> 5;
  const uint32_t* __restrict__ val = reinterpret_cast<const uint32_t*>(v.val);
  unsigned long long acc = 0;
  for (long long m = warp; m < nblk; m += nwarps) {
    const uint32_t M0 = val[(size_t)m * 32 + lane];
    const int total = (int)__reduce_add_sync(0xffffffffu, (unsigned)__popc(M0));
    if (total <= kSparsePairs) continue;  // handled by k_tc
    const int I = tile_row[m];
    const int K = v.colind[m];
    const int a0i = v.rowptr[I], a1i = (int)m + 1;
    const int b0i = v.rowptr[K], b1i = v.rowptr[K + 1];
    const bool probe_a = (a1i - a0i) <= (b1i - b0i);
    const int p0 = probe_a ? a0i : b0i, p1 = probe_a ? a1i : b1i;
    const int s0 = probe_a ? b0i : a0i, s1 = probe_a ? b1i : a1i;
    int d[2][4][4];
#pragma unroll
    for (int mb = 0; mb < 2; ++mb)
#pragma unroll
      for (int nb = 0; nb < 4; ++nb)
#pragma unroll
        for (int e = 0; e < 4; ++e) d[mb][nb][e] = 0;
    for (int base = p0; base < p1; base += 32) {
      const int p = base + (int)lane;
      int hit = -1;
      if (p < p1) {
        const int J = v.colind[p];
        const int qq = lower_bound_dev(v.colind, s0, s1, J);
        if (qq < s1 && v.colind[qq] == J) hit = qq;
      }
      const unsigned found = __ballot_sync(0xffffffffu, hit >= 0);
      const int nh = __popc(found);
      if (hit >= 0)
        hits[__popc(found & ((1u << lane) - 1u))] = probe_a ? make_int2(p, hit) : make_int2(hit, p);
      __syncwarp();
      for (int c0 = 0; c0 < nh; c0 += 8) {
        // stage the 8 hits' A tiles (I,J) and B tiles (K,J), one coalesced
        // 128-byte load per tile, then build the fragments from shared memory
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          const int2 hh = c0 + h < nh ? hits[c0 + h] : make_int2(-1, -1);
          sA[h][lane] = hh.x >= 0 ? val[(size_t)hh.x * 32 + lane] : 0u;
          sB[h][lane] = hh.y >= 0 ? val[(size_t)hh.y * 32 + lane] : 0u;
        }
        __syncwarp();
        unsigned bq[4][2];
#pragma unroll
        for (int nb = 0; nb < 4; ++nb) {
          bq[nb][0] = sB[q4][8 * nb + g];
          bq[nb][1] = sB[q4 + 4][8 * nb + g];
        }
#pragma unroll
        for (int mb = 0; mb < 2; ++mb) {
          const unsigned a0 = sA[q4][16 * mb + g], a1 = sA[q4][16 * mb + g + 8];
          const unsigned a2 = sA[q4 + 4][16 * mb + g], a3 = sA[q4 + 4][16 * mb + g + 8];
#pragma unroll
          for (int nb = 0; nb < 4; ++nb) mma_and_popc(d[mb][nb], a0, a1, a2, a3, bq[nb][0], bq[nb][1]);
        }
        __syncwarp();
      }
      __syncwarp();
    }
    // sum of P over the mask's bits: row r, column c at bit 31-c of M[r]
#pragma unroll
    for (int mb = 0; mb < 2; ++mb) {
      const uint32_t mr0 = __shfl_sync(0xffffffffu, M0, 16 * mb + g);
      const uint32_t mr1 = __shfl_sync(0xffffffffu, M0, 16 * mb + g + 8);
#pragma unroll
      for (int nb = 0; nb < 4; ++nb) {
        const int col = 8 * nb + 2 * q4;
        if ((mr0 >> (31 - col)) & 1u) acc += (unsigned)d[mb][nb][0];
        if ((mr0 >> (30 - col)) & 1u) acc += (unsigned)d[mb][nb][1];
        if ((mr1 >> (31 - col)) & 1u) acc += (unsigned)d[mb][nb][2];
        if ((mr1 >> (30 - col)) & 1u) acc += (unsigned)d[mb][nb][3];
      }
    }
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0 && acc) atomicAdd(count, acc);
}

}  // namespace

int tc_launch(gbo_graph* g, unsigned long long* d_count, cudaStream_t s) {
  GBO_CUDA_TRY(cudaMemsetAsync(d_count, 0, sizeof(unsigned long long), s));
  if (g->nblk == 0) return GBO_OK;
  GView v = view_of(g);
  if (!g->tile_row) {  // block row of every tile, kept with the graph
    GBO_CUDA_TRY(cudaMalloc(&g->tile_row, sizeof(int) * (size_t)g->nblk));
    g->device_bytes += 4LL * g->nblk;
    k_tile_row<<<blocks_for_warps(g->nitems, kTPB / 32), kTPB, 0, s>>>(v, g->tile_row);
  }
  long long warps = g->nblk;
  long long cap = (long long)num_sms() * 64;  // 64 resident warps per SM
  if (warps > cap * 8) warps = cap * 8;
  const unsigned grid = blocks_for_warps(warps, kTPB / 32);
  switch (g->b) {
    case 4: k_tc<4><<<grid, kTPB, 0, s>>>(v, g->nblk, g->tile_row, 0, d_count); break;
    case 8: k_tc<8><<<grid, kTPB, 0, s>>>(v, g->nblk, g->tile_row, 0, d_count); break;
    case 16: k_tc<16><<<grid, kTPB, 0, s>>>(v, g->nblk, g->tile_row, 0, d_count); break;
    case 32: if (g->tc_mma) {
      k_tc<32><<<grid, kTPB, 0, s>>>(v, g->nblk, g->tile_row, 1, d_count);
      k_tc32_mma<<<grid, kTPB, 0, s>>>(v, g->nblk, g->tile_row, d_count);
    } else {
      k_tc<32><<<grid, kTPB, 0, s>>>(v, g->nblk, g->tile_row, 0, d_count);
    }; break;
    default: k_tc<64><<<grid, kTPB, 0, s>>>(v, g->nblk, g->tile_row, 0, d_count); break;
  }
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}

}  // namespace gbo

using namespace gbo;

static int check_tc_graph(const gbo_graph* g) {
  if (!g) return fail(GBO_ERR_INVALID, "graph is NULL");
  if (g->layout != GBO_LAYOUT_ROW) return fail(GBO_ERR_UNSUPPORTED, "TC needs the ROW tile layout");
  if (g->nrows != g->ncols) return fail(GBO_ERR_INVALID, "TC needs a square matrix");
  return GBO_OK;
}

extern "C" int gbo_tc_device(const gbo_graph* lower, unsigned long long* d_count,
                             gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_tc_graph(lower));
  if (!d_count) return fail(GBO_ERR_INVALID, "count is NULL");
  return tc_launch(const_cast<gbo_graph*>(lower), d_count, as_stream(stream));
}

extern "C" int gbo_tc(const gbo_graph* lower, uint64_t* h_count, gbo_stream_t stream) {
  clear_error();
  GBO_TRY(check_tc_graph(lower));
  if (!h_count) return fail(GBO_ERR_INVALID, "count is NULL");
  cudaStream_t s = as_stream(stream);
  unsigned long long* d = nullptr;
  GBO_CUDA_TRY(pool_malloc_async(&d, sizeof(unsigned long long), s));
  int st = tc_launch(const_cast<gbo_graph*>(lower), d, s);
  unsigned long long h = 0;
  if (st == GBO_OK) {
    cudaError_t e = cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) st = fail_cuda(e, "tc readback");
  }
  cudaFreeAsync(d, s);
  if (st == GBO_OK) *h_count = h;
  return st;
}
