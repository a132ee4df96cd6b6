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
