// Error reporting, version and the device plumbing part of the C ABI.
#include <atomic>
#include <mutex>
#include <cstring>
#include <string>

#include "common.cuh"

namespace gbo {

namespace {
thread_local std::string g_last_error;

__global__ void k_flush(unsigned* p, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x)
    p[i] = (unsigned)i;
}
}  // namespace

int fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}

int fail_cuda(cudaError_t err, const char* what) {
  g_last_error = std::string(what) + ": " + cudaGetErrorString(err);
  if (err == cudaErrorMemoryAllocation) return GBO_ERR_NOMEM;
  return GBO_ERR_CUDA;
}

// Also drops a stale non-sticky CUDA error left by an earlier call, so that
// the cudaGetLastError() checks after our launches report our own launches.
void clear_error() {
  g_last_error.clear();
  (void)cudaGetLastError();
}

// Host-side fault injection state (gbo_debug_inject).
namespace {
std::atomic<long long> g_inject_alloc{0};
std::atomic<long long> g_inject_replay_cap{0};
std::atomic<int> g_inject_hold{0};
std::atomic<long long> g_inject_barrier{0};
}  // namespace

bool inject_host_alloc_fails() {
  long long v = g_inject_alloc.load();
  while (v > 0)
    if (g_inject_alloc.compare_exchange_weak(v, v - 1)) return v == 1;
  return false;
}
long long inject_replay_cap() { return g_inject_replay_cap.load(); }
bool inject_server_hold() { return g_inject_hold.load() != 0; }
long long take_inject_barrier_skip() { return g_inject_barrier.exchange(0); }

cudaError_t pool_malloc_async(void** p, size_t bytes, cudaStream_t s) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaMallocAsync(p, bytes, s);
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.handleTypes = cudaMemHandleTypeNone;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      e = cudaMemPoolCreate(&pools[dev], &props);
      if (e != cudaSuccess) {
        pools[dev] = nullptr;
        return e;
      }
      unsigned long long keep = kPoolKeepBytes;
      e = cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) return e;
    }
    pool = pools[dev];
  }
  return cudaMallocFromPoolAsync(p, bytes, pool, s);
}

int num_sms() {
  static thread_local int cached = 0;
  if (cached == 0) {
    int dev = 0, n = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0)
      n = 148;
    cached = n;
  }
  return cached;
}

}  // namespace gbo

using namespace gbo;

extern "C" const char* gbo_status_string(int status) {
  switch (status) {
    case GBO_OK: return "GBO_OK";
    case GBO_ERR_INVALID: return "GBO_ERR_INVALID";
    case GBO_ERR_CUDA: return "GBO_ERR_CUDA";
    case GBO_ERR_NOMEM: return "GBO_ERR_NOMEM";
    case GBO_ERR_UNSORTED: return "GBO_ERR_UNSORTED";
    case GBO_ERR_BOUNDS: return "GBO_ERR_BOUNDS";
    case GBO_ERR_TIMEOUT: return "GBO_ERR_TIMEOUT";
    case GBO_ERR_IO: return "GBO_ERR_IO";
    case GBO_ERR_UNSUPPORTED: return "GBO_ERR_UNSUPPORTED";
    case GBO_ERR_OVERFLOW: return "GBO_ERR_OVERFLOW";
    case GBO_ERR_NOTREADY: return "GBO_ERR_NOTREADY";
    case GBO_ERR_FULL: return "GBO_ERR_FULL";
  }
  return "GBO_ERR_UNKNOWN";
}

extern "C" const char* gbo_last_error(void) { return g_last_error.c_str(); }

extern "C" int gbo_debug_inject(int what, long long n) {
  clear_error();
  if (n < 0) return fail(GBO_ERR_INVALID, "injection count must be >= 0");
  switch (what) {
    case GBO_INJECT_HOST_ALLOC: g_inject_alloc.store(n); return GBO_OK;
    case GBO_INJECT_REPLAY_CAP: g_inject_replay_cap.store(n); return GBO_OK;
    case GBO_INJECT_SERVER_HOLD: g_inject_hold.store(n ? 1 : 0); return GBO_OK;
    case GBO_INJECT_BARRIER_SKIP: g_inject_barrier.store(n); return GBO_OK;
  }
  return fail(GBO_ERR_INVALID, "unknown injection");
}

extern "C" int gbo_version(void) { return 100; }

extern "C" int gbo_device_count(int* count) {
  clear_error();
  if (!count) return fail(GBO_ERR_INVALID, "count is NULL");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess) {
    *count = 0;
    return fail_cuda(e, "cudaGetDeviceCount");
  }
  *count = n;
  return GBO_OK;
}

extern "C" int gbo_set_device(int device) {
  clear_error();
  GBO_CUDA_TRY(cudaSetDevice(device));
  return GBO_OK;
}

extern "C" int gbo_malloc(void** d_ptr, size_t bytes) {
  clear_error();
  if (!d_ptr) return fail(GBO_ERR_INVALID, "d_ptr is NULL");
  *d_ptr = nullptr;
  GBO_CUDA_TRY(cudaMalloc(d_ptr, bytes ? bytes : 1));
  return GBO_OK;
}

extern "C" int gbo_free(void* d_ptr) {
  clear_error();
  if (d_ptr) GBO_CUDA_TRY(cudaFree(d_ptr));
  return GBO_OK;
}

extern "C" int gbo_host_alloc(void** h_ptr, size_t bytes) {
  clear_error();
  if (!h_ptr) return fail(GBO_ERR_INVALID, "h_ptr is NULL");
  *h_ptr = nullptr;
  GBO_CUDA_TRY(cudaHostAlloc(h_ptr, bytes ? bytes : 1, cudaHostAllocDefault));
  return GBO_OK;
}

extern "C" int gbo_host_free(void* h_ptr) {
  clear_error();
  if (h_ptr) GBO_CUDA_TRY(cudaFreeHost(h_ptr));
  return GBO_OK;
}

extern "C" int gbo_memset(void* d_ptr, int value, size_t bytes, gbo_stream_t stream) {
  clear_error();
  if (bytes) GBO_CUDA_TRY(cudaMemsetAsync(d_ptr, value, bytes, as_stream(stream)));
  return GBO_OK;
}

extern "C" int gbo_memcpy_h2d(void* d_dst, const void* h_src, size_t bytes, gbo_stream_t stream) {
  clear_error();
  if (bytes) GBO_CUDA_TRY(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, as_stream(stream)));
  return GBO_OK;
}

extern "C" int gbo_memcpy_d2h(void* h_dst, const void* d_src, size_t bytes, gbo_stream_t stream) {
  clear_error();
  if (bytes) GBO_CUDA_TRY(cudaMemcpyAsync(h_dst, d_src, bytes, cudaMemcpyDeviceToHost, as_stream(stream)));
  return GBO_OK;
}

extern "C" int gbo_memcpy_d2d(void* d_dst, const void* d_src, size_t bytes, gbo_stream_t stream) {
  clear_error();
  if (bytes) GBO_CUDA_TRY(cudaMemcpyAsync(d_dst, d_src, bytes, cudaMemcpyDeviceToDevice, as_stream(stream)));
  return GBO_OK;
}

extern "C" int gbo_stream_create(gbo_stream_t* stream) {
  clear_error();
  if (!stream) return fail(GBO_ERR_INVALID, "stream is NULL");
  cudaStream_t s = nullptr;
  GBO_CUDA_TRY(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
  *stream = reinterpret_cast<gbo_stream_t>(s);
  return GBO_OK;
}

extern "C" int gbo_stream_destroy(gbo_stream_t stream) {
  clear_error();
  if (stream) GBO_CUDA_TRY(cudaStreamDestroy(as_stream(stream)));
  return GBO_OK;
}

extern "C" int gbo_stream_sync(gbo_stream_t stream) {
  clear_error();
  GBO_CUDA_TRY(cudaStreamSynchronize(as_stream(stream)));
  return GBO_OK;
}

extern "C" int gbo_device_sync(void) {
  clear_error();
  GBO_CUDA_TRY(cudaDeviceSynchronize());
  return GBO_OK;
}

extern "C" int gbo_event_create(gbo_event_t* ev) {
  clear_error();
  if (!ev) return fail(GBO_ERR_INVALID, "ev is NULL");
  cudaEvent_t e = nullptr;
  GBO_CUDA_TRY(cudaEventCreate(&e));
  *ev = reinterpret_cast<gbo_event_t>(e);
  return GBO_OK;
}

extern "C" int gbo_event_destroy(gbo_event_t ev) {
  clear_error();
  if (ev) GBO_CUDA_TRY(cudaEventDestroy(reinterpret_cast<cudaEvent_t>(ev)));
  return GBO_OK;
}

extern "C" int gbo_event_record(gbo_event_t ev, gbo_stream_t stream) {
  clear_error();
  GBO_CUDA_TRY(cudaEventRecord(reinterpret_cast<cudaEvent_t>(ev), as_stream(stream)));
  return GBO_OK;
}

extern "C" int gbo_event_elapsed_ms(gbo_event_t start, gbo_event_t stop, float* ms) {
  clear_error();
  if (!ms) return fail(GBO_ERR_INVALID, "ms is NULL");
  GBO_CUDA_TRY(cudaEventSynchronize(reinterpret_cast<cudaEvent_t>(stop)));
  GBO_CUDA_TRY(cudaEventElapsedTime(ms, reinterpret_cast<cudaEvent_t>(start),
                                    reinterpret_cast<cudaEvent_t>(stop)));
  return GBO_OK;
}

extern "C" int gbo_flush_l2(gbo_stream_t stream) {
  clear_error();
  static thread_local unsigned* buf = nullptr;
  static thread_local long long n = 0;
  if (!buf) {
    int dev = 0, l2 = 0;
    GBO_CUDA_TRY(cudaGetDevice(&dev));
    GBO_CUDA_TRY(cudaDeviceGetAttribute(&l2, cudaDevAttrL2CacheSize, dev));
    n = (long long)(l2 > 0 ? l2 : (128 << 20)) / 4 * 2;  // 2x the L2 size
    GBO_CUDA_TRY(cudaMalloc(&buf, sizeof(unsigned) * (size_t)n));
  }
  k_flush<<<num_sms() * 4, 256, 0, as_stream(stream)>>>(buf, n);
  GBO_CUDA_TRY(cudaGetLastError());
  return GBO_OK;
}
