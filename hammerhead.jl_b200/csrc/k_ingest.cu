// Frame ingestion (sm_100a): UInt16 camera counts to float32 on the device,
// so frames cross PCIe at 2 bytes per pixel. Normalised: value / 65535, the
// Float32 value of a Gray{N0f16} pixel as load_image returns it
// (src/io.jl:20-25); raw: the count itself. One correctly rounded IEEE
// operation per pixel; 8 pixels per thread with 16-byte loads when aligned.
#include <stdint.h>

#include "hh_internal.h"

namespace hh {

__global__ void u16_to_f32_kernel(const uint16_t* __restrict__ src, int64_t n, int32_t normalise,
                                  float* __restrict__ dst) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  const bool vec = ((reinterpret_cast<uintptr_t>(src) & 15) == 0) && ((reinterpret_cast<uintptr_t>(dst) & 15) == 0);
  const int64_t n8 = vec ? n / 8 : 0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n8; i += stride) {
    const uint4 raw = reinterpret_cast<const uint4*>(src)[i];
    const uint32_t w[4] = {raw.x, raw.y, raw.z, raw.w};
    float f[8];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const float lo = (float)(w[k] & 0xFFFFu), hi = (float)(w[k] >> 16);
      f[2 * k] = normalise ? __fdiv_rn(lo, 65535.0f) : lo;
      f[2 * k + 1] = normalise ? __fdiv_rn(hi, 65535.0f) : hi;
    }
    reinterpret_cast<float4*>(dst)[2 * i] = make_float4(f[0], f[1], f[2], f[3]);
    reinterpret_cast<float4*>(dst)[2 * i + 1] = make_float4(f[4], f[5], f[6], f[7]);
  }
  for (int64_t i = 8 * n8 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const float v = (float)src[i];
    dst[i] = normalise ? __fdiv_rn(v, 65535.0f) : v;
  }
}

cudaError_t launch_u16_to_f32(const uint16_t* src, int64_t n, int32_t normalise, float* dst, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  int64_t blocks = (n / 8 + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (blocks < 1) blocks = 1;
  u16_to_f32_kernel<<<(unsigned)blocks, 256, 0, s>>>(src, n, normalise, dst);
  return cudaGetLastError();
}

}  // namespace hh
