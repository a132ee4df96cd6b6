// A reference-style driver ported onto gbo_compat.hpp: the control flow of
// algorithm/bfs.cu:main32 (read .mtx, CSC, csr2bsr_batch_32, ToBit32Row, a
// level loop of bmv32_sparse_bin_masked_v4 with the frontier count read back
// every level) followed by the same BFS through gbo_bfs and the triangle
// count through bmm32_sparse_masked_v5 (bsrbmm/tc.cu).
//
//   ./bfs_driver file.mtx directed
// prints "succ: <new vertices>" per level like the reference, then
// "gbo_bfs depth: D reached: R" and "ntris: T".
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <vector>

#include "gbo_compat.hpp"

using namespace gbo_compat;

#define CHECK(x)                                                            \
  do {                                                                      \
    int s_ = (x);                                                           \
    if (s_ != GBO_OK) {                                                     \
      fprintf(stderr, "%s failed: %s\n", #x, gbo_last_error());            \
      return 1;                                                             \
    }                                                                       \
  } while (0)

int main(int argc, char* argv[]) {
  if (argc < 3) {
    printf("./bfs_driver [xxx.mtx] [directed]\n");
    return 1;
  }
  std::vector<int> row_indices, col_indices;
  std::vector<float> values;
  int nrows = 0, ncols = 0, nnz = 0;
  CHECK(readMtx(argv[1], &row_indices, &col_indices, &values, &nrows, &ncols, &nnz, atoi(argv[2]), false));
  std::vector<int> h_csrRowPtr(nrows + 1), h_csrColInd(nnz);
  std::vector<float> h_csrVal(nnz);
  CHECK(coo2csr(h_csrRowPtr.data(), h_csrColInd.data(), h_csrVal.data(), row_indices, col_indices,
                values, nrows, ncols));
  printf("nrows: %d, ncols: %d, nnz: %d\n", nrows, ncols, nnz);

  // CSC of A so that the pull BMV follows A's edges (bfs.cu:398-423)
  std::vector<int> h_cscColPtr(ncols + 1), h_cscRowInd(nnz);
  std::vector<float> h_cscVal(nnz);
  CHECK(csr2csc(h_cscColPtr.data(), h_cscRowInd.data(), h_cscVal.data(), h_csrRowPtr.data(),
                h_csrColInd.data(), h_csrVal.data(), nrows, ncols));

  const int blocksize = 32;
  const int nblockrows = (nrows + blocksize - 1) / blocksize;
  int *d_ptr, *d_col, *bsrRowPtr, *bsrColInd;
  cudaMalloc(&d_ptr, sizeof(int) * (ncols + 1));
  cudaMalloc(&d_col, sizeof(int) * (nnz > 0 ? nnz : 1));
  cudaMemcpy(d_ptr, h_cscColPtr.data(), sizeof(int) * (ncols + 1), cudaMemcpyHostToDevice);
  cudaMemcpy(d_col, h_cscRowInd.data(), sizeof(int) * nnz, cudaMemcpyHostToDevice);
  cudaMalloc(&bsrRowPtr, sizeof(int) * (nblockrows + 1));
  int nblocks = 0;
  CHECK(csr2bsrNnz(d_ptr, d_col, ncols, nrows, nnz, blocksize, bsrRowPtr, &nblocks));
  printf("blocksize: %d, nblockrows: %d, nblocks: %d\n", blocksize, nblockrows, nblocks);
  unsigned* tA;
  cudaMalloc(&bsrColInd, sizeof(int) * (nblocks > 0 ? nblocks : 1));
  cudaMalloc(&tA, sizeof(unsigned) * blocksize * (nblocks > 0 ? nblocks : 1));
  CHECK(csr2bsr_batch_32(h_cscColPtr.data(), h_cscRowInd.data(), ncols, nrows, nnz, bsrRowPtr,
                         bsrColInd, tA, blocksize, nblockrows, nblocks));

  // source vertex 0 as a dense float vector packed to bits (bfs.cu:445-464)
  std::vector<float> B(nblockrows * blocksize, 0.f);
  B[0] = 1.f;
  float* fB;
  unsigned *frontier1, *frontier2, *visited;
  cudaMalloc(&fB, sizeof(float) * B.size());
  cudaMemcpy(fB, B.data(), sizeof(float) * B.size(), cudaMemcpyHostToDevice);
  cudaMalloc(&frontier1, sizeof(unsigned) * nblockrows);
  cudaMalloc(&frontier2, sizeof(unsigned) * nblockrows);
  cudaMalloc(&visited, sizeof(unsigned) * nblockrows);
  cudaMemset(visited, 0, sizeof(unsigned) * nblockrows);  // the reference leaves it unset
  CHECK(ToBit32Row(fB, frontier1, (int)B.size()));

  std::vector<unsigned> hv(nblockrows), hf(nblockrows);
  int niter = 0;
  for (int i = 0; i < nrows + 1; ++i) {
    // visited |= frontier1 (the reference's OR kernel), on the host here
    cudaMemcpy(hv.data(), visited, sizeof(unsigned) * nblockrows, cudaMemcpyDeviceToHost);
    cudaMemcpy(hf.data(), frontier1, sizeof(unsigned) * nblockrows, cudaMemcpyDeviceToHost);
    for (int k = 0; k < nblockrows; ++k) hv[k] |= hf[k];
    cudaMemcpy(visited, hv.data(), sizeof(unsigned) * nblockrows, cudaMemcpyHostToDevice);
    CHECK((bmv32_sparse_bin_masked_v4<int, unsigned>(tA, frontier1, frontier2, bsrRowPtr, bsrColInd,
                                                      nblockrows, visited)));
    cudaMemcpy(hf.data(), frontier2, sizeof(unsigned) * nblockrows, cudaMemcpyDeviceToHost);
    int succ = 0;
    for (int k = 0; k < nblockrows; ++k) succ += __builtin_popcount(hf[k]);
    cudaMemcpy(frontier1, frontier2, sizeof(unsigned) * nblockrows, cudaMemcpyDeviceToDevice);
    printf("succ: %d\n", succ);
    niter = i + 1;
    if (succ == 0) break;
  }
  printf("niter: %d\n", niter);

  // the same traversal through the device-resident loop
  gbo_graph* g = nullptr;
  CHECK(gbo_graph_from_csr(h_csrRowPtr.data(), h_csrColInd.data(), nrows, ncols, nnz, 32,
                           GBO_FLAG_TRANSPOSE, nullptr, &g));
  int* d_level;
  cudaMalloc(&d_level, sizeof(int) * nrows);
  int depth = 0;
  CHECK(gbo_bfs(g, 0, d_level, &depth, nullptr));
  std::vector<int> level(nrows);
  cudaMemcpy(level.data(), d_level, sizeof(int) * nrows, cudaMemcpyDeviceToHost);
  int reached = 0;
  for (int v : level) reached += v >= 0;
  printf("gbo_bfs depth: %d reached: %d\n", depth, reached);

  // triangle counting on L = tril(A) as in bsrbmm/tc.cu
  gbo_graph* low = nullptr;
  CHECK(gbo_graph_from_csr(h_csrRowPtr.data(), h_csrColInd.data(), nrows, ncols, nnz, 32,
                           GBO_FLAG_LOWER, nullptr, &low));
  const int *lptr, *lcol;
  const void* lval;
  CHECK(gbo_graph_b2sr(low, &lptr, &lcol, &lval));
  int* fC;
  cudaMalloc(&fC, sizeof(int));
  cudaMemset(fC, 0, sizeof(int));
  CHECK((bmm32_sparse_masked_v5<int, int>((const unsigned*)lval, nullptr, fC, lptr, lcol, nullptr,
                                          nullptr, nblockrows, 0, nrows)));
  int ntris = 0;
  cudaMemcpy(&ntris, fC, sizeof(int), cudaMemcpyDeviceToHost);
  uint64_t ntri64 = 0;
  CHECK(gbo_tc(low, &ntri64, nullptr));
  printf("ntris: %d (uint64 %llu)\n", ntris, (unsigned long long)ntri64);

  gbo_graph_free(g);
  gbo_graph_free(low);
  return 0;
}
