// Vector-grid kernels of a WIDIM sweep on one image pair (sm_100a):
// combine, validation, peak substitution, replacement, predictor
// smoothing, convergence norm. The per-cell logic lives in hh_grid.cuh.
#include <math.h>
#include <stdint.h>

#include "hh_grid.cuh"
#include "hh_internal.h"

namespace hh {

static inline int grid_blocks(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

#define GRID_STRIDE(k, n) for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (n); k += (int64_t)gridDim.x * blockDim.x)

// u = predictor + residual, alternatives + predictor, masked -> NaN
// (src/pipeline.jl:755-767), optional measured copy (:768-770).
__device__ __forceinline__ void combine_cell(float* u, float* v, const float* resu, const float* resv, float* ratio,
                                             float* moment, float* alt_u, float* alt_v, int nalt, bool masked,
                                             int64_t G, int64_t k, float* meas_u, float* meas_v) {
  const float pu = u[k], pv = v[k];
  for (int m = 0; m < nalt; ++m) {
    alt_u[k + m * G] = FADD(alt_u[k + m * G], pu);
    alt_v[k + m * G] = FADD(alt_v[k + m * G], pv);
  }
  float uu = FADD(pu, resu[k]), vv = FADD(pv, resv[k]);
  if (masked) {
    uu = vv = f_nan();
    ratio[k] = f_nan();
    moment[k] = f_nan();
  }
  u[k] = uu;
  v[k] = vv;
  if (meas_u) {
    meas_u[k] = uu;
    meas_v[k] = vv;
  }
}

__global__ void combine_kernel(float* u, float* v, const float* resu, const float* resv, float* ratio, float* moment,
                               float* alt_u, float* alt_v, int32_t nalt, const uint8_t* gmask, int64_t G,
                               float* meas_u, float* meas_v) {
  GRID_STRIDE(k, G)
  combine_cell(u, v, resu, resv, ratio, moment, alt_u, alt_v, nalt, gmask && gmask[k], G, k, meas_u, meas_v);
}

cudaError_t launch_combine(float* u, float* v, const float* resu, const float* resv, float* ratio, float* moment,
                           float* alt_u, float* alt_v, int32_t nalt, const uint8_t* gmask, int64_t G, float* meas_u,
                           float* meas_v, cudaStream_t s) {
  combine_kernel<<<grid_blocks(G), 256, 0, s>>>(u, v, resu, resv, ratio, moment, alt_u, alt_v, nalt, gmask, G, meas_u,
                                                meas_v);
  return cudaGetLastError();
}

__global__ void uod_kernel(const float* u, const float* v, int32_t ny, int32_t nx, double thr, int32_t nb, double eps,
                           const uint8_t* exclude, uint8_t* flags, int32_t or_into) {
  GRID_STRIDE(k, (int64_t)ny * nx) {
    const uint8_t f = uod_cell(u, v, ny, nx, (int)(k % ny), (int)(k / ny), thr, nb, eps, exclude);
    if (or_into) flags[k] |= f;
    else flags[k] = f;
  }
}

cudaError_t launch_uod(const float* u, const float* v, int32_t ny, int32_t nx, double thr, int32_t nb, double eps,
                       const uint8_t* exclude, uint8_t* flags, int32_t or_into, cudaStream_t s) {
  if (nb < 1 || (2 * nb + 1) * (2 * nb + 1) - 1 > UOD_MAXN) return cudaErrorInvalidValue;
  uod_kernel<<<grid_blocks((int64_t)ny * nx, 128), 128, 0, s>>>(u, v, ny, nx, thr, nb, eps, exclude, flags, or_into);
  return cudaGetLastError();
}

// apply_validator! for the local validators (src/quality.jl:466-486).
__global__ void flag_ratio_kernel(const float* ratio, int64_t G, double thr, uint8_t* flags) {
  GRID_STRIDE(k, G) if (!((double)ratio[k] >= thr)) flags[k] = 1;
}
__global__ void flag_moment_kernel(const float* m, int64_t G, double thr, uint8_t* flags) {
  GRID_STRIDE(k, G) if (!((double)m[k] <= thr)) flags[k] = 1;
}
__global__ void flag_velocity_kernel(const float* u, const float* v, int64_t G, double vmin, double vmax,
                                     uint8_t* flags) {
  GRID_STRIDE(k, G) {
    const double mag = (double)hypotf(u[k], v[k]);
    if (!(vmin <= mag && mag <= vmax)) flags[k] = 1;
  }
}
__global__ void mask_flags_kernel(uint8_t* flags, const uint8_t* gmask, int64_t G) {
  GRID_STRIDE(k, G) if (gmask[k]) flags[k] = 0;
}
cudaError_t launch_flag_ratio(const float* ratio, int64_t G, double thr, uint8_t* flags, cudaStream_t s) {
  flag_ratio_kernel<<<grid_blocks(G), 256, 0, s>>>(ratio, G, thr, flags);
  return cudaGetLastError();
}
cudaError_t launch_flag_moment(const float* moment, int64_t G, double thr, uint8_t* flags, cudaStream_t s) {
  flag_moment_kernel<<<grid_blocks(G), 256, 0, s>>>(moment, G, thr, flags);
  return cudaGetLastError();
}
cudaError_t launch_flag_velocity(const float* u, const float* v, int64_t G, double vmin, double vmax, uint8_t* flags,
                                 cudaStream_t s) {
  flag_velocity_kernel<<<grid_blocks(G), 256, 0, s>>>(u, v, G, vmin, vmax, flags);
  return cudaGetLastError();
}
cudaError_t launch_mask_flags(uint8_t* flags, const uint8_t* gmask, int64_t G, cudaStream_t s) {
  mask_flags_kernel<<<grid_blocks(G), 256, 0, s>>>(flags, gmask, G);
  return cudaGetLastError();
}

__global__ void substitute_kernel(float* u, float* v, const uint8_t* outl_in, uint8_t* outl_out, const uint8_t* gmask,
                                  const float* alt_u, const float* alt_v, int32_t nalt, int32_t ny, int32_t nx,
                                  int32_t er, double thr) {
  GRID_STRIDE(k, (int64_t)ny * nx)
  outl_out[k] = substitute_cell(u, v, outl_in, gmask, alt_u, alt_v, nalt, ny, nx, (int)(k % ny), (int)(k / ny), er, thr);
}

cudaError_t launch_substitute(float* u, float* v, const uint8_t* outl_in, uint8_t* outl_out, const uint8_t* gmask,
                              const float* alt_u, const float* alt_v, int32_t nalt, int32_t ny, int32_t nx, int32_t er,
                              double thr, cudaStream_t s) {
  if (er < 1 || (2 * er + 1) * (2 * er + 1) - 1 > UOD_MAXN) return cudaErrorInvalidValue;
  substitute_kernel<<<grid_blocks((int64_t)ny * nx, 128), 128, 0, s>>>(u, v, outl_in, outl_out, gmask, alt_u, alt_v,
                                                                       nalt, ny, nx, er, thr);
  return cudaGetLastError();
}

__global__ void replace_kernel(float* u, float* v, const uint8_t* flags, const uint8_t* gmask, int32_t ny, int32_t nx,
                               int32_t nan_mask) {
  GRID_STRIDE(k, (int64_t)ny * nx) {
    if (!repl_invalid(flags, gmask, k)) continue;
    float nu = u[k], nvv = v[k];
    replace_cell(u, v, flags, gmask, ny, nx, (int)(k % ny), (int)(k / ny), nu, nvv);
    if (nan_mask && gmask && gmask[k]) nu = nvv = f_nan();
    u[k] = nu;
    v[k] = nvv;
  }
}

cudaError_t launch_replace(float* u, float* v, const uint8_t* flags, const uint8_t* gmask, int32_t ny, int32_t nx,
                           int32_t nan_mask, cudaStream_t s) {
  replace_kernel<<<grid_blocks((int64_t)ny * nx, 128), 128, 0, s>>>(u, v, flags, gmask, ny, nx, nan_mask);
  return cudaGetLastError();
}

__global__ void smooth_kernel(const float* f, int32_t ny, int32_t nx, float* out) {
  GRID_STRIDE(k, (int64_t)ny * nx) out[k] = smooth_cell(f, ny, nx, (int)(k % ny), (int)(k / ny));
}
cudaError_t launch_smooth(const float* f, int32_t ny, int32_t nx, float* out, cudaStream_t s) {
  smooth_kernel<<<grid_blocks((int64_t)ny * nx), 256, 0, s>>>(f, ny, nx, out);
  return cudaGetLastError();
}

// field_change (src/pipeline.jl:849-866): one CTA, keys in scratch.
constexpr int FC_THREADS = 1024;

__global__ void __launch_bounds__(FC_THREADS) field_change_kernel(const float* u, const float* v, const float* pu,
                                                                  const float* pv, const uint8_t* gmask, int64_t G,
                                                                  uint32_t* keys, float* out) {
  __shared__ uint32_t hist[256];
  __shared__ uint32_t s_bucket;
  __shared__ int64_t s_k;
  __shared__ unsigned long long s_n;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  unsigned long long n_local = 0;
  for (int64_t i = threadIdx.x; i < G; i += blockDim.x) {
    bool counts;
    keys[i] = change_key(u[i], v[i], pu[i], pv[i], gmask && gmask[i], counts);
    n_local += counts;
  }
  atomicAdd(&s_n, n_local);
  __syncthreads();
  const int64_t n = (int64_t)s_n;
  if (n == 0) {
    if (threadIdx.x == 0) *out = 0.f;
    return;
  }
  int64_t ka, kb;
  double g;
  quantile95_index(n, ka, kb, g);
  const uint32_t a = cta_radix_select(keys, G, ka, hist, &s_bucket, &s_k);
  const uint32_t b = kb == ka ? a : cta_radix_select(keys, G, kb, hist, &s_bucket, &s_k);
  if (threadIdx.x == 0) *out = quantile95_value(a, b, g);
}

cudaError_t launch_field_change(const float* u, const float* v, const float* pu, const float* pv, const uint8_t* gmask,
                                int64_t G, float* scratch, float* out, cudaStream_t s) {
  field_change_kernel<<<1, FC_THREADS, 0, s>>>(u, v, pu, pv, gmask, G, reinterpret_cast<uint32_t*>(scratch), out);
  return cudaGetLastError();
}

__global__ void restore_measured_kernel(float* u, float* v, const float* mu, const float* mv, const uint8_t* outl,
                                        int64_t G) {
  GRID_STRIDE(k, G) if (outl[k]) {
    u[k] = mu[k];
    v[k] = mv[k];
  }
}
cudaError_t launch_restore_measured(float* u, float* v, const float* meas_u, const float* meas_v, const uint8_t* outl,
                                    int64_t G, cudaStream_t s) {
  restore_measured_kernel<<<grid_blocks(G), 256, 0, s>>>(u, v, meas_u, meas_v, outl, G);
  return cudaGetLastError();
}

__global__ void fill_kernel(float* p, float value, int64_t n) {
  GRID_STRIDE(k, n) p[k] = value;
}
cudaError_t launch_fill(float* p, float value, int64_t n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  fill_kernel<<<grid_blocks(n), 256, 0, s>>>(p, value, n);
  return cudaGetLastError();
}

}  // namespace hh
