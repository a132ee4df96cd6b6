// Kernel-facing view of a graph and the BMV entry points used by the
// algorithm loops and the C ABI.
#pragma once

#include "graph.cuh"

namespace gbo {

// Plain-old-data copy of the fields the kernels read (passed by value).
struct GView {
  int nrows, ncols, nbr, nbc;
  const int* __restrict__ rowptr;
  const int* __restrict__ colind;
  const void* __restrict__ val;
  const gbo_item* __restrict__ items;
  int nitems;
  const gbo_split* __restrict__ splits;
  int nsplit;
  // b = 32 ROW tiles: bit r of rowmask[t] is set iff row word r of tile t is
  // non-zero (null for other widths and layouts)
  const unsigned* __restrict__ rowmask = nullptr;
  // with rowmask: the non-empty row words packed in tile order (row order
  // inside a tile) and the index of every work item's first word
  const unsigned* __restrict__ rowword = nullptr;
  const long long* __restrict__ item_wbase = nullptr;
  // row-word slices (b = 32 ROW, once built): see gbo_graph::rws_head
  const uint2* __restrict__ rws_head = nullptr;
  const uint2* __restrict__ rws_tail = nullptr;
  const long long* __restrict__ rws_tail_ptr = nullptr;
  int rws_nlong = 0;
  long long rws_nchunk = 0;
  long long rws_ntail = 0;
  const int* __restrict__ rws_long_row = nullptr;
  const long long* __restrict__ rws_long_chunk0 = nullptr;
  const int* __restrict__ rws_chunk_row = nullptr;
  const long long* __restrict__ rws_chunk_beg = nullptr;
  const long long* __restrict__ rws_chunk_end = nullptr;
  const unsigned* __restrict__ rws_longbits = nullptr;
};

// Index in rowword of row r's word of a tile with occupancy word m whose
// first word is at `off` (bit r of m must be set).
__device__ __forceinline__ long long rowword_index(long long off, unsigned m, int r) {
  return off + __popc(m & ((1u << r) - 1u));
}

GView view_of(const gbo_graph* g);

// Scratch bytes the split-row partials of one BMV launch need.
size_t bmv_scratch_bytes(const gbo_graph* g);

int bmv_count(const gbo_graph* g, const void* x, void* y, int out_type, int accumulate,
              void* scratch, cudaStream_t s);
int bmv_masked(const gbo_graph* g, const void* x, const void* mask, void* out, void* scratch,
               cudaStream_t s);
int bmv_minplus(const gbo_graph* g, const uint32_t* x, uint32_t* y, void* scratch, cudaStream_t s);
int bmv_minselect(const gbo_graph* g, const int32_t* x, int32_t* y, void* scratch, cudaStream_t s);
int bmv_float(const gbo_graph* g, const float* x, float* y, float alpha, const float* scale,
              float add, void* scratch, cudaStream_t s, const int* degptr = nullptr);
int bmv_float_transposed(const gbo_graph* g, const float* x, float* y, float alpha,
                         const float* scale, float add, cudaStream_t s);

}  // namespace gbo
