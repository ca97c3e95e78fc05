// Allocation-free variant of the convergence-norm kernel (field_change).
//
// Some callers cannot let a library allocate device memory: a host runtime
// whose GPU memory is owned by its own pool allocator (a Julia or Python
// array package) may forbid foreign cudaMalloc calls behind its back, a
// latency-critical loop must not stall on an allocation, and a process
// running under a fixed memory budget may have no headroom for one. For them
// hh_field_change_noalloc computes the same 95th-percentile change as
// hh_field_change, on caller-owned device buffers, with its only scratch (one
// 32-bit key per vector) in a fixed array compiled into this library.
//
// The array below lives in every GPU that loads the library until the
// process exits (HH_NOALLOC_MAX_VECTORS * 4 bytes = 4 MiB). Host code cannot
// use its name as a device address: the address is looked up once per
// device with cudaGetSymbolAddress, with that device current, on the first
// call made there, and cached.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <mutex>
#include <string>

#include "hammerhead_b200.h"

namespace {

constexpr int64_t kMaxVectors = HH_NOALLOC_MAX_VECTORS;
constexpr int kThreads = 1024;
constexpr int kMaxDevices = 64;

// Shared by every call on a device; the kernel rewrites the first n entries
// before reading them, so no clearing is needed between calls.
__device__ __align__(256) uint32_t g_noalloc_keys[kMaxVectors];

std::mutex g_setup_mutex;
uint32_t* g_keys_addr[kMaxDevices] = {};
thread_local std::string g_noalloc_err;

// k-th smallest key (0-based) among keys[0, n) by a 4 x 8-bit radix select.
__device__ uint32_t radix_select(const uint32_t* keys, int64_t n, int64_t kth, uint32_t* hist, uint32_t* s_bucket,
                                 int64_t* s_k) {
  uint32_t prefix = 0, pmask = 0;
  int64_t k = kth;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
      const uint32_t x = keys[i];
      if ((x & pmask) == prefix) atomicAdd(&hist[(x >> shift) & 255u], 1u);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
      int64_t acc = 0;
      uint32_t sel = 255;
      for (uint32_t b = 0; b < 256; ++b) {
        if (acc + hist[b] > k) {
          sel = b;
          break;
        }
        acc += hist[b];
      }
      *s_bucket = sel;
      *s_k = k - acc;
    }
    __syncthreads();
    prefix |= *s_bucket << shift;
    pmask |= 255u << shift;
    k = *s_k;
    __syncthreads();
  }
  return prefix;
}

// field_change (src/pipeline.jl:849-866): 95th percentile (type 7) of
// max(|du|, |dv|) over unmasked vectors, NaN transitions counted as +Inf.
__global__ void __launch_bounds__(kThreads) field_change_noalloc_kernel(const float* u, const float* v, const float* pu,
                                                                         const float* pv, const uint8_t* mask,
                                                                         int64_t n, uint32_t* keys, float* out) {
  __shared__ uint32_t hist[256];
  __shared__ uint32_t s_bucket;
  __shared__ int64_t s_k;
  __shared__ unsigned long long s_count;
  if (threadIdx.x == 0) s_count = 0;
  __syncthreads();
  unsigned long long local = 0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    uint32_t key = 0xFFFFFFFFu;  // excluded: orders after every real value
    if (!(mask && mask[i])) {
      const float du = fabsf(__fsub_rn(u[i], pu[i])), dv = fabsf(__fsub_rn(v[i], pv[i]));
      if (isnan(du) || isnan(dv)) {
        if (!(isnan(u[i]) == isnan(pu[i]) && isnan(v[i]) == isnan(pv[i]))) {
          key = 0x7F800000u;  // +Inf
          ++local;
        }
      } else {
        key = __float_as_uint(fmaxf(du, dv));
        ++local;
      }
    }
    keys[i] = key;
  }
  atomicAdd(&s_count, local);
  __syncthreads();
  const int64_t cnt = (int64_t)s_count;
  if (cnt == 0) {
    if (threadIdx.x == 0) *out = 0.f;
    return;
  }
  const double p = 0.95;
  const double aleph = fma((double)cnt, p, 1.0 - p);
  int64_t j = (int64_t)trunc(aleph);
  const int64_t hi = cnt - 1 > 1 ? cnt - 1 : 1;
  j = j < 1 ? 1 : (j > hi ? hi : j);
  double g = aleph - (double)j;
  g = g < 0 ? 0 : (g > 1 ? 1 : g);
  const uint32_t ka = radix_select(keys, n, cnt == 1 ? 0 : j - 1, hist, &s_bucket, &s_k);
  const uint32_t kb = cnt == 1 ? ka : radix_select(keys, n, j, hist, &s_bucket, &s_k);
  if (threadIdx.x == 0) {
    const float a = __uint_as_float(ka), b = __uint_as_float(kb);
    double q;
    if (isfinite(a) && isfinite(b)) q = __dadd_rn((double)a, __dmul_rn(g, (double)__fsub_rn(b, a)));
    else q = __dadd_rn(__dmul_rn(1.0 - g, (double)a), __dmul_rn(g, (double)b));
    *out = (float)q;
  }
}

hh_status fail(hh_status code, const std::string& msg) {
  g_noalloc_err = msg;
  return code;
}

}  // namespace

extern "C" const char* hh_noalloc_last_error(void) { return g_noalloc_err.c_str(); }

extern "C" hh_status hh_field_change_noalloc(const float* d_u, const float* d_v, const float* d_pu, const float* d_pv,
                                             const uint8_t* d_mask, int64_t n, float* d_change, void* stream) {
  g_noalloc_err.clear();  // the message describes this call's failure only
  if (n > kMaxVectors)
    return fail(HH_ERR_ARG, "hh_field_change_noalloc: " + std::to_string(n) + " vectors exceed the fixed scratch of " +
                                std::to_string(kMaxVectors) + " (HH_NOALLOC_MAX_VECTORS); use hh_field_change");
  if (n < 0 || !d_change || (n > 0 && (!d_u || !d_v || !d_pu || !d_pv)))
    return fail(HH_ERR_ARG, "hh_field_change_noalloc: invalid pointer or size argument");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail(HH_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail(HH_ERR_UNSUPPORTED, "device index beyond the scratch table");
  uint32_t* keys = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_keys_addr[dev]) {
      // once per device, with that device current (it is: cudaGetDevice above)
      void* addr = nullptr;
      e = cudaGetSymbolAddress(&addr, g_noalloc_keys);
      if (e != cudaSuccess || !addr)
        return fail(HH_ERR_CUDA, std::string("cudaGetSymbolAddress(g_noalloc_keys): ") + cudaGetErrorString(e));
      g_keys_addr[dev] = static_cast<uint32_t*>(addr);
    }
    keys = g_keys_addr[dev];
  }
  field_change_noalloc_kernel<<<1, kThreads, 0, static_cast<cudaStream_t>(stream)>>>(d_u, d_v, d_pu, d_pv, d_mask, n,
                                                                                     keys, d_change);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail(HH_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
  return HH_OK;
}
