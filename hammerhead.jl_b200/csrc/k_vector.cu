// Vector-grid kernels of a WIDIM sweep (sm_100a): combine, validation,
// peak substitution, replacement, predictor smoothing, convergence norm.
//
// The grid is column-major (ny, nx) like PIVResult fields. Every operation
// restates src/quality.jl / src/pipeline.jl with the reference's precision
// (Float32 fields, Float64 where Julia widens) and explicit round-to-nearest
// intrinsics, so flags and replaced values equal the CPU restatement bit for
// bit on identical inputs.
#include <math.h>
#include <stdint.h>

#include "hh_internal.h"

namespace hh {

#define FADD(a, b) __fadd_rn((a), (b))
#define FSUB(a, b) __fsub_rn((a), (b))
#define FMUL(a, b) __fmul_rn((a), (b))

static __device__ __forceinline__ float f_nan() { return __int_as_float(0x7fc00000); }

static inline int grid_blocks(int64_t n, int threads = 256) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return (int)b;
}

// ---------------------------------------------------------------------------
// u = predictor + residual, alternatives + predictor, masked -> NaN
// (src/pipeline.jl:755-767), optional measured copy (:768-770).
__global__ void combine_kernel(float* u, float* v, const float* resu, const float* resv, float* ratio, float* moment,
                               float* alt_u, float* alt_v, int32_t nalt, const uint8_t* gmask, int64_t G,
                               float* meas_u, float* meas_v) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < G; k += (int64_t)gridDim.x * blockDim.x) {
    const float pu = u[k], pv = v[k];
    for (int m = 0; m < nalt; ++m) {
      alt_u[k + m * G] = FADD(alt_u[k + m * G], pu);
      alt_v[k + m * G] = FADD(alt_v[k + m * G], pv);
    }
    float uu = FADD(pu, resu[k]), vv = FADD(pv, resv[k]);
    if (gmask && gmask[k]) {
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
}

cudaError_t launch_combine(float* u, float* v, const float* resu, const float* resv, float* ratio, float* moment,
                           float* alt_u, float* alt_v, int32_t nalt, const uint8_t* gmask, int64_t G, float* meas_u,
                           float* meas_v, cudaStream_t s) {
  combine_kernel<<<grid_blocks(G), 256, 0, s>>>(u, v, resu, resv, ratio, moment, alt_u, alt_v, nalt, gmask, G, meas_u,
                                                meas_v);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Statistics.median! on a small local array: NaN if any NaN; even n ->
// a/2 + b/2 of the two middle order statistics.
template <class T> __device__ __forceinline__ void isort(T* a, int n) {
  for (int i = 1; i < n; ++i) {
    T x = a[i];
    int j = i - 1;
    while (j >= 0 && a[j] > x) {
      a[j + 1] = a[j];
      --j;
    }
    a[j + 1] = x;
  }
}
__device__ __forceinline__ float median_f(float* a, int n) {
  for (int i = 0; i < n; ++i)
    if (isnan(a[i])) return f_nan();
  isort(a, n);
  if (n & 1) return a[n / 2];
  return FADD(a[n / 2 - 1] / 2.0f, a[n / 2] / 2.0f);
}
__device__ __forceinline__ double median_d(double* a, int n) {
  for (int i = 0; i < n; ++i)
    if (isnan(a[i])) return __longlong_as_double(0x7ff8000000000000LL);
  isort(a, n);
  if (n & 1) return a[n / 2];
  return __dadd_rn(a[n / 2 - 1] / 2.0, a[n / 2] / 2.0);
}

constexpr int UOD_MAXN = 80;  // neighbourhood <= 4 layers

// universal_outlier_detection (src/quality.jl:244-293).
__global__ void uod_kernel(const float* u, const float* v, int32_t ny, int32_t nx, double thr, int32_t nb, double eps,
                           const uint8_t* exclude, uint8_t* flags, int32_t or_into) {
  const int64_t G = (int64_t)ny * nx;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < G; k += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(k % ny), c = (int)(k / ny);
    uint8_t f = 0;
    if (!(exclude && exclude[k])) {
      float nu[UOD_MAXN], nv[UOD_MAXN], ru[UOD_MAXN], rv[UOD_MAXN];
      int n = 0;
      for (int c2 = max(0, c - nb); c2 <= min(nx - 1, c + nb); ++c2)
        for (int r2 = max(0, r - nb); r2 <= min(ny - 1, r + nb); ++r2) {
          if (r2 == r && c2 == c) continue;
          const int64_t q = r2 + (int64_t)c2 * ny;
          if (exclude && exclude[q]) continue;
          nu[n] = u[q];
          nv[n] = v[q];
          ++n;
        }
      if (n > 0) {
        for (int i = 0; i < n; ++i) {
          ru[i] = nu[i];
          rv[i] = nv[i];
        }
        const float um = median_f(ru, n), vm = median_f(rv, n);
        for (int i = 0; i < n; ++i) {
          ru[i] = fabsf(FSUB(nu[i], um));
          rv[i] = fabsf(FSUB(nv[i], vm));
        }
        const double un = (double)fabsf(FSUB(u[k], um)) / __dadd_rn((double)median_f(ru, n), eps);
        const double vn = (double)fabsf(FSUB(v[k], vm)) / __dadd_rn((double)median_f(rv, n), eps);
        if (un > thr || vn > thr) f = 1;
      }
    }
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
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < G; k += (int64_t)gridDim.x * blockDim.x)
    if (!((double)ratio[k] >= thr)) flags[k] = 1;
}
__global__ void flag_moment_kernel(const float* m, int64_t G, double thr, uint8_t* flags) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < G; k += (int64_t)gridDim.x * blockDim.x)
    if (!((double)m[k] <= thr)) flags[k] = 1;
}
__global__ void flag_velocity_kernel(const float* u, const float* v, int64_t G, double vmin, double vmax,
                                     uint8_t* flags) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < G; k += (int64_t)gridDim.x * blockDim.x) {
    const double mag = (double)hypotf(u[k], v[k]);
    if (!(vmin <= mag && mag <= vmax)) flags[k] = 1;
  }
}
__global__ void mask_flags_kernel(uint8_t* flags, const uint8_t* gmask, int64_t G) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < G; k += (int64_t)gridDim.x * blockDim.x)
    if (gmask[k]) flags[k] = 0;
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

// ---------------------------------------------------------------------------
// substitute_alternatives! (src/quality.jl:307-351). Judged against the
// snapshot outl_in; only flagged cells change, and they read valid cells
// only, so u/v are updated in place without races.
__global__ void substitute_kernel(float* u, float* v, const uint8_t* outl_in, uint8_t* outl_out, const uint8_t* gmask,
                                  const float* alt_u, const float* alt_v, int32_t nalt, int32_t ny, int32_t nx,
                                  int32_t er, double thr) {
  const int64_t G = (int64_t)ny * nx;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < G; k += (int64_t)gridDim.x * blockDim.x) {
    uint8_t o = outl_in[k];
    if (o && !(gmask && gmask[k])) {
      const int r = (int)(k % ny), c = (int)(k / ny);
      double bu[UOD_MAXN], bv[UOD_MAXN], tu[UOD_MAXN], tv[UOD_MAXN];
      int n = 0;
      for (int c2 = max(0, c - er); c2 <= min(nx - 1, c + er); ++c2)
        for (int r2 = max(0, r - er); r2 <= min(ny - 1, r + er); ++r2) {
          if (r2 == r && c2 == c) continue;
          const int64_t q = r2 + (int64_t)c2 * ny;
          if (outl_in[q] || (gmask && gmask[q])) continue;
          bu[n] = (double)u[q];
          bv[n] = (double)v[q];
          ++n;
        }
      if (n >= 3) {
        for (int i = 0; i < n; ++i) {
          tu[i] = bu[i];
          tv[i] = bv[i];
        }
        const double mu = median_d(tu, n), mv = median_d(tv, n);
        for (int i = 0; i < n; ++i) {
          tu[i] = fabs(__dsub_rn(bu[i], mu));
          tv[i] = fabs(__dsub_rn(bv[i], mv));
        }
        const double madu = median_d(tu, n), madv = median_d(tv, n);
        for (int m = 0; m < nalt; ++m) {
          const float au = alt_u[k + m * G], av = alt_v[k + m * G];
          if (!(isfinite(au) && isfinite(av))) break;
          if (fabs(__dsub_rn((double)au, mu)) / __dadd_rn(madu, 0.1) <= thr &&
              fabs(__dsub_rn((double)av, mv)) / __dadd_rn(madv, 0.1) <= thr) {
            u[k] = au;
            v[k] = av;
            o = 0;
            break;
          }
        }
      }
    }
    outl_out[k] = o;
  }
}

cudaError_t launch_substitute(float* u, float* v, const uint8_t* outl_in, uint8_t* outl_out, const uint8_t* gmask,
                              const float* alt_u, const float* alt_v, int32_t nalt, int32_t ny, int32_t nx, int32_t er,
                              double thr, cudaStream_t s) {
  if (er < 1 || (2 * er + 1) * (2 * er + 1) - 1 > UOD_MAXN) return cudaErrorInvalidValue;
  substitute_kernel<<<grid_blocks((int64_t)ny * nx, 128), 128, 0, s>>>(u, v, outl_in, outl_out, gmask, alt_u, alt_v,
                                                                       nalt, ny, nx, er, thr);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// replace_vectors! (src/quality.jl:85-114): growing square until >= 3 valid
// neighbours, component-wise Float64 median. Invalid cells are written,
// valid cells only read, so the update is in place.
constexpr int REPL_LOCAL = 64;

__device__ __forceinline__ bool repl_invalid(const uint8_t* flags, const uint8_t* gmask, int64_t q) {
  return (flags && flags[q]) || (gmask && gmask[q]);
}

// k-th smallest (0-based) of the valid values in a square, by counting;
// used only when a square holds more than REPL_LOCAL valid values.
__device__ double select_square(const float* f, const uint8_t* flags, const uint8_t* gmask, int ny, int r0, int r1,
                                int c0, int c1, int kth) {
  for (int cc = c0; cc <= c1; ++cc)
    for (int rr = r0; rr <= r1; ++rr) {
      const int64_t q = rr + (int64_t)cc * ny;
      if (repl_invalid(flags, gmask, q)) continue;
      const double x = (double)f[q];
      int less = 0, le = 0;
      for (int c2 = c0; c2 <= c1; ++c2)
        for (int r2 = r0; r2 <= r1; ++r2) {
          const int64_t q2 = r2 + (int64_t)c2 * ny;
          if (repl_invalid(flags, gmask, q2)) continue;
          const double y = (double)f[q2];
          less += y < x;
          le += y <= x;
        }
      if (less <= kth && kth < le) return x;
    }
  return __longlong_as_double(0x7ff8000000000000LL);
}

__device__ double median_square(const float* f, const uint8_t* flags, const uint8_t* gmask, int ny, int r0, int r1,
                                int c0, int c1, int n) {
  if (n <= REPL_LOCAL) {
    double buf[REPL_LOCAL];
    int m = 0;
    for (int cc = c0; cc <= c1; ++cc)
      for (int rr = r0; rr <= r1; ++rr) {
        const int64_t q = rr + (int64_t)cc * ny;
        if (repl_invalid(flags, gmask, q)) continue;
        buf[m++] = (double)f[q];
      }
    return median_d(buf, m);
  }
  for (int cc = c0; cc <= c1; ++cc)  // NaN anywhere -> NaN
    for (int rr = r0; rr <= r1; ++rr) {
      const int64_t q = rr + (int64_t)cc * ny;
      if (!repl_invalid(flags, gmask, q) && isnan(f[q])) return __longlong_as_double(0x7ff8000000000000LL);
    }
  if (n & 1) return select_square(f, flags, gmask, ny, r0, r1, c0, c1, n / 2);
  const double a = select_square(f, flags, gmask, ny, r0, r1, c0, c1, n / 2 - 1);
  const double b = select_square(f, flags, gmask, ny, r0, r1, c0, c1, n / 2);
  return __dadd_rn(a / 2.0, b / 2.0);
}

__global__ void replace_kernel(float* u, float* v, const uint8_t* flags, const uint8_t* gmask, int32_t ny, int32_t nx,
                               int32_t nan_mask) {
  const int64_t G = (int64_t)ny * nx;
  const int maxr = (ny > nx ? ny : nx) - 1;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < G; k += (int64_t)gridDim.x * blockDim.x) {
    if (!repl_invalid(flags, gmask, k)) continue;
    const int r = (int)(k % ny), c = (int)(k / ny);
    float nu = u[k], nvv = v[k];
    for (int rad = 1; rad <= maxr; ++rad) {
      const int r0 = max(0, r - rad), r1 = min(ny - 1, r + rad), c0 = max(0, c - rad), c1 = min(nx - 1, c + rad);
      int n = 0;
      for (int cc = c0; cc <= c1; ++cc)
        for (int rr = r0; rr <= r1; ++rr) n += !repl_invalid(flags, gmask, rr + (int64_t)cc * ny);
      if (n >= 3) {
        nu = (float)median_square(u, flags, gmask, ny, r0, r1, c0, c1, n);
        nvv = (float)median_square(v, flags, gmask, ny, r0, r1, c0, c1, n);
        break;
      }
    }
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

// smooth_field (src/quality.jl:123-136): separable [1 2 1]/4, replicated edges.
__device__ __forceinline__ float smooth_row(const float* f, int ny, int nx, int r, int c) {
  const float q = 0.25f;
  const int cl = c > 0 ? c - 1 : 0, cr = c < nx - 1 ? c + 1 : nx - 1;
  return FMUL(q, FADD(FADD(f[r + (int64_t)cl * ny], FMUL(2.0f, f[r + (int64_t)c * ny])), f[r + (int64_t)cr * ny]));
}
__global__ void smooth_kernel(const float* f, int32_t ny, int32_t nx, float* out) {
  const int64_t G = (int64_t)ny * nx;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < G; k += (int64_t)gridDim.x * blockDim.x) {
    const int r = (int)(k % ny), c = (int)(k / ny);
    const int rl = r > 0 ? r - 1 : 0, rr = r < ny - 1 ? r + 1 : ny - 1;
    const float tl = smooth_row(f, ny, nx, rl, c), t0 = smooth_row(f, ny, nx, r, c), tr = smooth_row(f, ny, nx, rr, c);
    out[k] = FMUL(0.25f, FADD(FADD(tl, FMUL(2.0f, t0)), tr));
  }
}
cudaError_t launch_smooth(const float* f, int32_t ny, int32_t nx, float* out, cudaStream_t s) {
  smooth_kernel<<<grid_blocks((int64_t)ny * nx), 256, 0, s>>>(f, ny, nx, out);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// field_change (src/pipeline.jl:849-866): 95th percentile (type 7) of
// max(|du|, |dv|) over unmasked cells; NaN transitions count as Inf.
// One CTA: the per-cell changes are all >= 0 (or +Inf), so their IEEE bit
// patterns order like the values and a 4 x 8-bit radix select finds the two
// order statistics the quantile interpolates between.
constexpr int FC_THREADS = 1024;

__device__ uint32_t fc_select(const uint32_t* keys, int64_t G, int64_t kth, uint32_t* hist) {
  uint32_t prefix = 0, pmask = 0;
  int64_t k = kth;
  for (int shift = 24; shift >= 0; shift -= 8) {
    for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    for (int64_t i = threadIdx.x; i < G; i += blockDim.x) {
      const uint32_t x = keys[i];
      if ((x & pmask) == prefix) atomicAdd(&hist[(x >> shift) & 255u], 1u);
    }
    __syncthreads();
    __shared__ uint32_t s_bucket;
    __shared__ int64_t s_k;
    if (threadIdx.x == 0) {
      int64_t acc = 0;
      uint32_t bsel = 255;
      for (uint32_t b = 0; b < 256; ++b) {
        if (acc + hist[b] > k) {
          bsel = b;
          break;
        }
        acc += hist[b];
      }
      s_bucket = bsel;
      s_k = k - acc;
    }
    __syncthreads();
    prefix |= s_bucket << shift;
    pmask |= 255u << shift;
    k = s_k;
    __syncthreads();
  }
  return prefix;
}

__global__ void __launch_bounds__(FC_THREADS) field_change_kernel(const float* u, const float* v, const float* pu,
                                                                  const float* pv, const uint8_t* gmask, int64_t G,
                                                                  uint32_t* keys, float* out) {
  __shared__ uint32_t hist[256];
  __shared__ unsigned long long s_n;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  unsigned long long n_local = 0;
  for (int64_t i = threadIdx.x; i < G; i += blockDim.x) {
    uint32_t key = 0xFFFFFFFFu;  // excluded entries sort after every real value
    if (!(gmask && gmask[i])) {
      const float du = fabsf(FSUB(u[i], pu[i])), dv = fabsf(FSUB(v[i], pv[i]));
      if (isnan(du) || isnan(dv)) {
        if (!(isnan(u[i]) == isnan(pu[i]) && isnan(v[i]) == isnan(pv[i]))) {
          key = 0x7F800000u;  // +Inf
          ++n_local;
        }
      } else {
        key = __float_as_uint(fmaxf(du, dv));
        ++n_local;
      }
    }
    keys[i] = key;
  }
  atomicAdd(&s_n, n_local);
  __syncthreads();
  const int64_t n = (int64_t)s_n;
  if (n == 0) {
    if (threadIdx.x == 0) *out = 0.f;
    return;
  }
  const double p = 0.95;
  const double aleph = fma((double)n, p, 1.0 - p);
  int64_t j = (int64_t)trunc(aleph);
  const int64_t hi = n - 1 > 1 ? n - 1 : 1;
  if (j < 1) j = 1;
  if (j > hi) j = hi;
  double g = aleph - (double)j;
  g = g < 0 ? 0 : (g > 1 ? 1 : g);
  const uint32_t ka = fc_select(keys, G, n == 1 ? 0 : j - 1, hist);
  const uint32_t kb = n == 1 ? ka : fc_select(keys, G, j, hist);
  if (threadIdx.x == 0) {
    const float a = __uint_as_float(ka), b = __uint_as_float(kb);
    double q;
    if (isfinite(a) && isfinite(b)) q = __dadd_rn((double)a, __dmul_rn(g, (double)FSUB(b, a)));
    else q = __dadd_rn(__dmul_rn(1.0 - g, (double)a), __dmul_rn(g, (double)b));
    *out = (float)q;
  }
}

cudaError_t launch_field_change(const float* u, const float* v, const float* pu, const float* pv, const uint8_t* gmask,
                                int64_t G, float* scratch, float* out, cudaStream_t s) {
  field_change_kernel<<<1, FC_THREADS, 0, s>>>(u, v, pu, pv, gmask, G, reinterpret_cast<uint32_t*>(scratch), out);
  return cudaGetLastError();
}

__global__ void restore_measured_kernel(float* u, float* v, const float* mu, const float* mv, const uint8_t* outl,
                                        int64_t G) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < G; k += (int64_t)gridDim.x * blockDim.x)
    if (outl[k]) {
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
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < n; k += (int64_t)gridDim.x * blockDim.x)
    p[k] = value;
}
cudaError_t launch_fill(float* p, float value, int64_t n, cudaStream_t s) {
  if (n <= 0) return cudaSuccess;
  fill_kernel<<<grid_blocks(n), 256, 0, s>>>(p, value, n);
  return cudaGetLastError();
}

}  // namespace hh
