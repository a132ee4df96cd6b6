// ORACLE (test infrastructure): C-ABI launchers for a subset of the
// reference's own BMV kernels, compiled from algorithm/bsrbmv.cu where it
// lies in the reference checkout (see oracle/Makefile, target _ref).  Used by
// tests to run the reference kernels on B2SR packed by libgbo, which pins the
// packing and the BMV semantics to the reference's code.
//
// Launch shapes follow the reference drivers (cube grids, algorithm/bfs.cu:
// 492-536, sssp.cu:447, pr.cu:482, bsrbmv/benchmark-bsrbmv.cu:1124).
// The reference kernels use int32 word offsets (row_start*b): callers keep
// nblocks*b below 2^31.  Value vectors and the CSR row pointer passed to the
// fp32 / min-plus kernels must be padded to nblockrows*b (+1) entries: those
// kernels read every column of a tile, set or not (bsrbmv.cu:1108,1274).
#include <math.h>

#include "bsrbmv.cu"

static dim3 cube(double units) {
  int g = (int)ceil(cbrt(units));
  if (g < 1) g = 1;
  return dim3(g, g, g);
}

extern "C" int ref_bmv4_sparse(const uchar* A, const uchar* B, float* C, const int* rowptr,
                               const int* colind, int nblockrows, int nblocks) {
  bmv4_sparse<int, float><<<cube(ceil(nblockrows / 8.0)), 32>>>(A, B, C, rowptr, colind, nblockrows,
                                                               nblocks);
  return (int)cudaGetLastError();
}

extern "C" int ref_bmv8_sparse(const uchar* A, const uchar* B, float* C, const int* rowptr,
                               const int* colind, int nblockrows, int nblocks) {
  bmv8_sparse<int, float><<<cube(ceil(nblockrows / 4.0)), 32>>>(A, B, C, rowptr, colind, nblockrows,
                                                               nblocks);
  return (int)cudaGetLastError();
}

extern "C" int ref_bmv16_sparse_new(const ushort* A, const ushort* B, float* C, const int* rowptr,
                                    const int* colind, int nblockrows, int nblocks) {
  bmv16_sparse_new<int, float><<<cube(ceil(nblockrows / 64.0)), 1024>>>(A, B, C, rowptr, colind,
                                                                       nblockrows, nblocks);
  return (int)cudaGetLastError();
}

extern "C" int ref_bmv32_sparse_new(const unsigned* A, const unsigned* B, float* C,
                                    const int* rowptr, const int* colind, int nblockrows,
                                    int nblocks) {
  bmv32_sparse_new<int, float><<<cube(ceil(nblockrows / 32.0)), 1024>>>(
      A, B, C, 0, 0, 0, rowptr, colind, nblockrows, nblocks);
  return (int)cudaGetLastError();
}

extern "C" int ref_bmv64_sparse_new(const ullong* A, const ullong* B, float* C, const int* rowptr,
                                    const int* colind, int nblockrows, int nblocks) {
  bmv64_sparse_new<int, float><<<cube(ceil(nblockrows / 32.0)), 1024>>>(
      A, B, C, 0, 0, 0, rowptr, colind, nblockrows, nblocks);
  return (int)cudaGetLastError();
}

extern "C" int ref_bmv32_sparse_bin_masked_v4(const unsigned* A, const unsigned* B, unsigned* C,
                                              const int* rowptr, const int* colind,
                                              int nblockrows, const unsigned* mask) {
  bmv32_sparse_bin_masked_v4<int, unsigned><<<cube(ceil(nblockrows / 32.0)), 1024>>>(
      A, B, C, rowptr, colind, nblockrows, mask);
  return (int)cudaGetLastError();
}

extern "C" int ref_bmv32_sparse_full_minplus(const unsigned* A, const unsigned* B, unsigned* C,
                                             const int* rowptr, const int* colind,
                                             int nblockrows) {
  bmv32_sparse_full_minplus<int, unsigned><<<cube(ceil(nblockrows / 16.0)), 512>>>(
      A, B, C, rowptr, colind, nblockrows);
  return (int)cudaGetLastError();
}

extern "C" int ref_bmv32_sparse_full(const unsigned* A, const float* B, float* C,
                                     const int* rowptr, const int* colind, int nblockrows,
                                     const int* csrrowptr, float alpha) {
  bmv32_sparse_full<int, float><<<cube(ceil(nblockrows / 16.0)), 512>>>(
      A, B, C, rowptr, colind, nblockrows, csrrowptr, alpha);
  return (int)cudaGetLastError();
}

extern "C" int ref_sync(void) { return (int)cudaDeviceSynchronize(); }

// The BFS loop of algorithm/bfs.cu:508-564 (main32, "solution 4") on the
// caller's B2SR (a symmetric graph, so the CSC packing the driver builds is
// the same B2SR): per iteration OR(visited, frontier1), the masked v4 BMV
// into frontier2, a device-to-device copy back into frontier1, fillZero,
// resetSuccptr + reduce and a blocking copy of succ to the host, until succ
// is 0 or max_iter iterations ran.  Launch shapes as in the driver.  The
// driver leaves `visited` uninitialised (bfs.cu:479); it is zeroed here.
// The per-iteration printf is left out.  succ of iteration i goes to
// h_succ[i]; returns the number of iterations (the driver's niter - 1 when
// it breaks on succ == 0), or -1 on a CUDA error; *ms is the loop's device
// time measured like the driver's GpuTimer (events around the loop).
extern "C" int ref_bfs32_masked_v4(const unsigned* A, const int* rowptr, const int* colind,
                                   int nblockrows, int src, int max_iter, int* h_succ, float* ms) {
  unsigned *f1 = nullptr, *f2 = nullptr, *vis = nullptr;
  int* succptr = nullptr;
  if (cudaMalloc(&f1, nblockrows * sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&f2, nblockrows * sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&vis, nblockrows * sizeof(unsigned)) != cudaSuccess ||
      cudaMalloc(&succptr, sizeof(int)) != cudaSuccess)
    return -1;
  cudaMemset(f1, 0, nblockrows * sizeof(unsigned));
  cudaMemset(f2, 0, nblockrows * sizeof(unsigned));
  cudaMemset(vis, 0, nblockrows * sizeof(unsigned));
  const unsigned bit = 1u << (31 - src % 32);
  cudaMemcpy(f1 + src / 32, &bit, sizeof(unsigned), cudaMemcpyHostToDevice);
  const dim3 grid_new = cube(nblockrows / 32.0);
  const int nb1024 = (int)ceil(nblockrows / 1024.0);
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaDeviceSynchronize();
  cudaEventRecord(e0);
  int i = 0, succ = 0;
  for (i = 0; i < max_iter; ++i) {
    OR<unsigned><<<nb1024, 1024>>>(vis, nblockrows, f1);
    bmv32_sparse_bin_masked_v4<int, unsigned><<<grid_new, 1024>>>(A, f1, f2, rowptr, colind, nblockrows,
                                                                  vis);
    cudaMemcpy(f1, f2, nblockrows * sizeof(unsigned), cudaMemcpyDeviceToDevice);
    fillZero<unsigned><<<nb1024, 1024>>>(f2, nblockrows);
    resetSuccptr<<<1, 1>>>(succptr);
    reduce<unsigned><<<nb1024, 1024>>>(f1, nblockrows, succptr);
    cudaMemcpy(&succ, succptr, sizeof(int), cudaMemcpyDeviceToHost);
    h_succ[i] = succ;
    if (succ == 0) break;
  }
  cudaEventRecord(e1);
  cudaEventSynchronize(e1);
  cudaEventElapsedTime(ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const int err = (int)cudaGetLastError();
  cudaFree(f1);
  cudaFree(f2);
  cudaFree(vis);
  cudaFree(succptr);
  return err ? -1 : (i < max_iter ? i + 1 : i);
}
