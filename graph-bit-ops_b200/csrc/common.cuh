// Internal helpers shared by the CUDA translation units of libgbo.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string>

#include "gbo.h"

namespace gbo {

// Records a failure message for gbo_last_error() on this host thread and
// returns the status, so call sites can write `return fail(...)`.
int fail(int status, const std::string& msg);
int fail_cuda(cudaError_t err, const char* what);
void clear_error();

#define GBO_CUDA_TRY(call)                                    \
  do {                                                        \
    cudaError_t e_ = (call);                                  \
    if (e_ != cudaSuccess) return ::gbo::fail_cuda(e_, #call); \
  } while (0)

#define GBO_TRY(call)               \
  do {                              \
    int s_ = (call);                \
    if (s_ != GBO_OK) return s_;    \
  } while (0)

inline cudaStream_t as_stream(gbo_stream_t s) { return reinterpret_cast<cudaStream_t>(s); }

inline bool valid_tile_bits(int b) { return b == 4 || b == 8 || b == 16 || b == 32 || b == 64; }

// Bytes of one tile row word (b=4 uses the low nibble of a byte).
inline int word_bytes(int b) { return b <= 8 ? 1 : b / 8; }

// Device-side error word bits (OR-ed by kernels, read by the host).
enum : unsigned {
  DERR_UNSORTED = 1u,
  DERR_COL_BOUNDS = 2u,
  DERR_ROWPTR = 4u,
  DERR_INDEX = 8u,
};

template <int B> struct Word;
template <> struct Word<4> { using T = uint8_t; };
template <> struct Word<8> { using T = uint8_t; };
template <> struct Word<16> { using T = uint16_t; };
template <> struct Word<32> { using T = uint32_t; };
template <> struct Word<64> { using T = unsigned long long; };

__device__ __forceinline__ int popc_w(unsigned long long v) { return __popcll(v); }
__device__ __forceinline__ int popc_w(uint32_t v) { return __popc(v); }
__device__ __forceinline__ int popc_w(uint16_t v) { return __popc((uint32_t)v); }
__device__ __forceinline__ int popc_w(uint8_t v) { return __popc((uint32_t)v); }

__device__ __forceinline__ unsigned lane_id() {
  unsigned l;
  asm volatile("mov.u32 %0, %%laneid;" : "=r"(l));
  return l;
}

// Mask of the low min(B,32) bits.
template <int B>
__host__ __device__ constexpr unsigned seg_mask() {
  return B >= 32 ? 0xffffffffu : ((1u << (B & 31)) - 1u);
}

constexpr int kWarp = 32;
constexpr int kINF = 2147483647;  // the reference's "infinity" (sssp.cu:140)

// Grid size for `n` independent warps with `wpb` warps per block.
inline unsigned blocks_for_warps(long long n, int wpb) {
  long long b = (n + wpb - 1) / wpb;
  return (unsigned)(b < 1 ? 1 : b);
}
inline unsigned blocks_for(long long n, int tpb) {
  long long b = (n + tpb - 1) / tpb;
  return (unsigned)(b < 1 ? 1 : b);
}

int num_sms();

// Stream-ordered temporaries come from a pool of the library's own (one per
// device, created on first use) that keeps up to kPoolKeepBytes of freed
// memory mapped: the default pool returns freed memory at every
// synchronisation, so calls that allocate and synchronise (packing, SpGEMM,
// the GPU reader) mapped fresh memory each time, at a cost that varied
// severalfold from run to run.  Free with cudaFreeAsync.
constexpr unsigned long long kPoolKeepBytes = 8ull << 30;
cudaError_t pool_malloc_async(void** p, size_t bytes, cudaStream_t s);
template <typename T>
inline cudaError_t pool_malloc_async(T** p, size_t bytes, cudaStream_t s) {
  return pool_malloc_async(reinterpret_cast<void**>(p), bytes, s);
}

// Host-side fault injection (gbo_debug_inject): true when this host CSR
// allocation is the one armed to fail; the replay cap of the iteration
// loops (0: none); whether server workers hold admission.
bool inject_host_alloc_fails();
long long inject_replay_cap();
bool inject_server_hold();
// Armed GBO_INJECT_BARRIER_SKIP value (0: none), disarmed by the read.
long long take_inject_barrier_skip();

// Exclusive scan of n int32 counts into out[0..n] (out[n] = total) with the
// total also returned through d_total (int64).  No spin waits: three kernels.
int exclusive_scan_i32(const int* d_in, int* d_out, long long n, long long* d_total,
                       cudaStream_t stream);
// The same with int64 outputs.
int exclusive_scan_i32_to_i64(const int* d_in, long long* d_out, long long n, long long* d_total,
                              cudaStream_t stream);

}  // namespace gbo
