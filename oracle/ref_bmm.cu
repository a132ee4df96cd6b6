// ORACLE (test infrastructure): C-ABI launcher for the reference's masked
// BMM (triangle counting), compiled from bsrbmm/bsrbmm.cu where it lies in
// the reference checkout (oracle/Makefile, target _ref).  The launch follows
// bsrbmm/tc.cu:948 (cube grid over block rows, one warp each).  A is the
// ROW-layout B2SR of L = tril(A), B the COL-layout B2SR of L^T; the int
// result accumulates like the reference's atomicAdd.  int32 word offsets:
// keep nblocks*32 below 2^31.
#include <math.h>

#include "bsrbmm.cu"

extern "C" int ref_bmm32_sparse_masked_v5(const unsigned* A, const unsigned* B, int* C,
                                          const int* A_rowptr, const int* A_colind,
                                          const int* B_rowptr, const int* B_colind,
                                          int nblockrows, int nblocks, int nrows) {
  int g = (int)ceil(cbrt((double)nblockrows));
  if (g < 1) g = 1;
  bmm32_sparse_masked_v5<int, int><<<dim3(g, g, g), 32>>>(A, B, C, A_rowptr, A_colind, B_rowptr,
                                                         B_colind, nblockrows, nblocks, nrows);
  return (int)cudaGetLastError();
}

extern "C" int ref_bmm_sync(void) { return (int)cudaDeviceSynchronize(); }
