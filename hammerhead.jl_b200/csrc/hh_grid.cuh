// Per-cell operations on a column-major (ny, nx) vector grid, shared by the
// single-pair kernels (k_vector.cu) and the batched ones (k_batch.cu). Each
// restates src/quality.jl / src/pipeline.jl in the reference's precision
// (Float32 fields, Float64 where Julia widens) with explicit round-to-nearest
// arithmetic, so flags and replaced values equal the CPU restatement bit for
// bit on identical inputs. Pointers address the grid of one image pair.
#pragma once
#include <math.h>
#include <stdint.h>

namespace hh {

#define FADD(a, b) __fadd_rn((a), (b))
#define FSUB(a, b) __fsub_rn((a), (b))
#define FMUL(a, b) __fmul_rn((a), (b))

static __device__ __forceinline__ float f_nan() { return __int_as_float(0x7fc00000); }

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


// Neighbourhoods of 1 and 2 layers in registers: the S = (2nb+1)^2 - 1
// neighbour slots hold +inf where a neighbour is missing (edge or excluded),
// so sorting the slots with a fixed comparator network puts the n present
// values first, in order, and no array needs dynamic indexing. The networks
// are Batcher's odd-even merge sort (19 comparators for 8 inputs; the
// 32-input network without the comparators that reach slots 24..31, which
// hold +inf throughout, for 24); both sort every 0/1 input (checked
// exhaustively), hence every input. The medians equal median_f's up to the
// sign of a zero, which only ever enters through |x - m|.
__device__ __forceinline__ void cas_f(float& a, float& b) {
  const float lo = fminf(a, b), hi = fmaxf(a, b);
  a = lo;
  b = hi;
}
template <int S> __device__ __forceinline__ void sort_net_f(float (&a)[S]);
template <> __device__ __forceinline__ void sort_net_f<8>(float (&a)[8]) {
  cas_f(a[0], a[1]); cas_f(a[2], a[3]); cas_f(a[4], a[5]); cas_f(a[6], a[7]); cas_f(a[0], a[2]); cas_f(a[1], a[3]);
  cas_f(a[4], a[6]); cas_f(a[5], a[7]); cas_f(a[1], a[2]); cas_f(a[5], a[6]); cas_f(a[0], a[4]); cas_f(a[3], a[7]);
  cas_f(a[1], a[5]); cas_f(a[2], a[6]); cas_f(a[1], a[4]); cas_f(a[3], a[6]); cas_f(a[2], a[4]); cas_f(a[3], a[5]);
  cas_f(a[3], a[4]);
}
template <> __device__ __forceinline__ void sort_net_f<24>(float (&a)[24]) {
  cas_f(a[0], a[1]); cas_f(a[2], a[3]); cas_f(a[0], a[2]); cas_f(a[1], a[3]); cas_f(a[1], a[2]); cas_f(a[4], a[5]);
  cas_f(a[6], a[7]); cas_f(a[4], a[6]); cas_f(a[5], a[7]); cas_f(a[5], a[6]); cas_f(a[0], a[4]); cas_f(a[2], a[6]);
  cas_f(a[2], a[4]); cas_f(a[1], a[5]); cas_f(a[3], a[7]); cas_f(a[3], a[5]); cas_f(a[1], a[2]); cas_f(a[3], a[4]);
  cas_f(a[5], a[6]); cas_f(a[8], a[9]); cas_f(a[10], a[11]); cas_f(a[8], a[10]); cas_f(a[9], a[11]); cas_f(a[9], a[10]);
  cas_f(a[12], a[13]); cas_f(a[14], a[15]); cas_f(a[12], a[14]); cas_f(a[13], a[15]); cas_f(a[13], a[14]); cas_f(a[8], a[12]);
  cas_f(a[10], a[14]); cas_f(a[10], a[12]); cas_f(a[9], a[13]); cas_f(a[11], a[15]); cas_f(a[11], a[13]); cas_f(a[9], a[10]);
  cas_f(a[11], a[12]); cas_f(a[13], a[14]); cas_f(a[0], a[8]); cas_f(a[4], a[12]); cas_f(a[4], a[8]); cas_f(a[2], a[10]);
  cas_f(a[6], a[14]); cas_f(a[6], a[10]); cas_f(a[2], a[4]); cas_f(a[6], a[8]); cas_f(a[10], a[12]); cas_f(a[1], a[9]);
  cas_f(a[5], a[13]); cas_f(a[5], a[9]); cas_f(a[3], a[11]); cas_f(a[7], a[15]); cas_f(a[7], a[11]); cas_f(a[3], a[5]);
  cas_f(a[7], a[9]); cas_f(a[11], a[13]); cas_f(a[1], a[2]); cas_f(a[3], a[4]); cas_f(a[5], a[6]); cas_f(a[7], a[8]);
  cas_f(a[9], a[10]); cas_f(a[11], a[12]); cas_f(a[13], a[14]); cas_f(a[16], a[17]); cas_f(a[18], a[19]); cas_f(a[16], a[18]);
  cas_f(a[17], a[19]); cas_f(a[17], a[18]); cas_f(a[20], a[21]); cas_f(a[22], a[23]); cas_f(a[20], a[22]); cas_f(a[21], a[23]);
  cas_f(a[21], a[22]); cas_f(a[16], a[20]); cas_f(a[18], a[22]); cas_f(a[18], a[20]); cas_f(a[17], a[21]); cas_f(a[19], a[23]);
  cas_f(a[19], a[21]); cas_f(a[17], a[18]); cas_f(a[19], a[20]); cas_f(a[21], a[22]); cas_f(a[18], a[20]); cas_f(a[19], a[21]);
  cas_f(a[17], a[18]); cas_f(a[19], a[20]); cas_f(a[21], a[22]); cas_f(a[0], a[16]); cas_f(a[8], a[16]); cas_f(a[4], a[20]);
  cas_f(a[12], a[20]); cas_f(a[4], a[8]); cas_f(a[12], a[16]); cas_f(a[2], a[18]); cas_f(a[10], a[18]); cas_f(a[6], a[22]);
  cas_f(a[14], a[22]); cas_f(a[6], a[10]); cas_f(a[14], a[18]); cas_f(a[2], a[4]); cas_f(a[6], a[8]); cas_f(a[10], a[12]);
  cas_f(a[14], a[16]); cas_f(a[18], a[20]); cas_f(a[1], a[17]); cas_f(a[9], a[17]); cas_f(a[5], a[21]); cas_f(a[13], a[21]);
  cas_f(a[5], a[9]); cas_f(a[13], a[17]); cas_f(a[3], a[19]); cas_f(a[11], a[19]); cas_f(a[7], a[23]); cas_f(a[15], a[23]);
  cas_f(a[7], a[11]); cas_f(a[15], a[19]); cas_f(a[3], a[5]); cas_f(a[7], a[9]); cas_f(a[11], a[13]); cas_f(a[15], a[17]);
  cas_f(a[19], a[21]); cas_f(a[1], a[2]); cas_f(a[3], a[4]); cas_f(a[5], a[6]); cas_f(a[7], a[8]); cas_f(a[9], a[10]);
  cas_f(a[11], a[12]); cas_f(a[13], a[14]); cas_f(a[15], a[16]); cas_f(a[17], a[18]); cas_f(a[19], a[20]); cas_f(a[21], a[22]);
}

// median of the n (1..S) present slots; NaN when one of them is NaN
template <int S> __device__ __forceinline__ float median_net_f(float (&a)[S], int n) {
  bool nan = false;
#pragma unroll
  for (int i = 0; i < S; ++i) nan |= isnan(a[i]);
  if (nan) return f_nan();
  sort_net_f<S>(a);
  const int h = n / 2;
  float lo = a[0], hi = a[0];  // a[h - 1], a[h]
#pragma unroll
  for (int i = 1; i < S; ++i) {
    if (i == h) hi = a[i];
    if (i == h - 1) lo = a[i];
  }
  if (n & 1) return hi;
  return FADD(lo / 2.0f, hi / 2.0f);
}

template <int NB>
__device__ __forceinline__ uint8_t uod_cell_net(const float* u, const float* v, int ny, int nx, int r, int c, double thr,
                                                double eps, const uint8_t* exclude) {
  constexpr int D = 2 * NB + 1, S = D * D - 1;
  const int64_t k = r + (int64_t)c * ny;
  const float INF = __int_as_float(0x7f800000);
  float nu[S], nv[S];
  uint32_t present = 0;
  int n = 0;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int d = s < S / 2 ? s : s + 1;  // skip the centre of the D x D block
    const int r2 = r + d % D - NB, c2 = c + d / D - NB;
    const int64_t q = r2 + (int64_t)c2 * ny;
    const bool ok = r2 >= 0 && r2 < ny && c2 >= 0 && c2 < nx && !(exclude && exclude[q]);
    nu[s] = ok ? u[q] : INF;
    nv[s] = ok ? v[q] : INF;
    present |= ok ? 1u << s : 0u;
    n += ok;
  }
  if (n == 0) return 0;
  float ru[S], rv[S];
#pragma unroll
  for (int s = 0; s < S; ++s) {
    ru[s] = nu[s];
    rv[s] = nv[s];
  }
  const float um = median_net_f<S>(ru, n), vm = median_net_f<S>(rv, n);
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const bool ok = (present >> s) & 1u;
    ru[s] = ok ? fabsf(FSUB(nu[s], um)) : INF;
    rv[s] = ok ? fabsf(FSUB(nv[s], vm)) : INF;
  }
  const double un = (double)fabsf(FSUB(u[k], um)) / __dadd_rn((double)median_net_f<S>(ru, n), eps);
  const double vn = (double)fabsf(FSUB(v[k], vm)) / __dadd_rn((double)median_net_f<S>(rv, n), eps);
  return (un > thr || vn > thr) ? 1 : 0;
}

// universal_outlier_detection (src/quality.jl:244-293) at cell (r, c).
__device__ __forceinline__ uint8_t uod_cell(const float* u, const float* v, int ny, int nx, int r, int c, double thr,
                                            int nb, double eps, const uint8_t* exclude) {
  const int64_t k = r + (int64_t)c * ny;
  if (exclude && exclude[k]) return 0;
  if (nb == 1) return uod_cell_net<1>(u, v, ny, nx, r, c, thr, eps, exclude);
  if (nb == 2) return uod_cell_net<2>(u, v, ny, nx, r, c, thr, eps, exclude);
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
  if (n == 0) return 0;
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
  return (un > thr || vn > thr) ? 1 : 0;
}

// substitute_alternatives! (src/quality.jl:307-351) at cell (r, c): judged
// against the snapshot outl_in; returns the new flag and may update u/v at
// the cell (it reads valid cells only, so in-place updates do not race).
// alt_u/alt_v hold nalt planes of G = ny*nx values.
__device__ __forceinline__ uint8_t substitute_cell(float* u, float* v, const uint8_t* outl_in, const uint8_t* gmask,
                                                   const float* alt_u, const float* alt_v, int nalt, int ny, int nx,
                                                   int r, int c, int er, double thr) {
  const int64_t G = (int64_t)ny * nx, k = r + (int64_t)c * ny;
  uint8_t o = outl_in[k];
  if (!o || (gmask && gmask[k])) return o;
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
  if (n < 3) return o;
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
      return 0;
    }
  }
  return o;
}

// replace_vectors! (src/quality.jl:85-114) support: growing square until >= 3
// valid neighbours, component-wise Float64 median.
constexpr int REPL_LOCAL = 64;

__device__ __forceinline__ bool repl_invalid(const uint8_t* flags, const uint8_t* gmask, int64_t q) {
  return (flags && flags[q]) || (gmask && gmask[q]);
}

// k-th smallest (0-based) of the valid values in a square, by counting;
// used only when a square holds more than REPL_LOCAL valid values.
static __device__ double select_square(const float* f, const uint8_t* flags, const uint8_t* gmask, int ny, int r0, int r1,
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

static __device__ double median_square(const float* f, const uint8_t* flags, const uint8_t* gmask, int ny, int r0, int r1,
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


// Replacement of one invalid cell (invalid = flags | gmask); writes the new
// values through nu/nv (unchanged when no square holds 3 valid cells).
__device__ __forceinline__ void replace_cell(const float* u, const float* v, const uint8_t* flags,
                                             const uint8_t* gmask, int ny, int nx, int r, int c, float& nu,
                                             float& nvv) {
  const int maxr = (ny > nx ? ny : nx) - 1;
  for (int rad = 1; rad <= maxr; ++rad) {
    const int r0 = max(0, r - rad), r1 = min(ny - 1, r + rad), c0 = max(0, c - rad), c1 = min(nx - 1, c + rad);
    int n = 0;
    for (int cc = c0; cc <= c1; ++cc)
      for (int rr = r0; rr <= r1; ++rr) n += !repl_invalid(flags, gmask, rr + (int64_t)cc * ny);
    if (n >= 3) {
      nu = (float)median_square(u, flags, gmask, ny, r0, r1, c0, c1, n);
      nvv = (float)median_square(v, flags, gmask, ny, r0, r1, c0, c1, n);
      return;
    }
  }
}

// smooth_field (src/quality.jl:123-136): separable [1 2 1]/4, replicated edges.
__device__ __forceinline__ float smooth_row(const float* f, int ny, int nx, int r, int c) {
  const float q = 0.25f;
  const int cl = c > 0 ? c - 1 : 0, cr = c < nx - 1 ? c + 1 : nx - 1;
  return FMUL(q, FADD(FADD(f[r + (int64_t)cl * ny], FMUL(2.0f, f[r + (int64_t)c * ny])), f[r + (int64_t)cr * ny]));
}
__device__ __forceinline__ float smooth_cell(const float* f, int ny, int nx, int r, int c) {
  const int rl = r > 0 ? r - 1 : 0, rr = r < ny - 1 ? r + 1 : ny - 1;
  const float tl = smooth_row(f, ny, nx, rl, c), t0 = smooth_row(f, ny, nx, r, c), tr = smooth_row(f, ny, nx, rr, c);
  return FMUL(0.25f, FADD(FADD(tl, FMUL(2.0f, t0)), tr));
}

// field_change key of one cell: max(|du|, |dv|) as its IEEE bits (all
// values are >= 0, so bits order like values), +Inf for a NaN transition,
// 0xFFFFFFFF (after every value) for cells that do not count.
__device__ __forceinline__ uint32_t change_key(float u, float v, float pu, float pv, bool masked, bool& counts) {
  counts = false;
  if (masked) return 0xFFFFFFFFu;
  const float du = fabsf(FSUB(u, pu)), dv = fabsf(FSUB(v, pv));
  if (isnan(du) || isnan(dv)) {
    if (isnan(u) == isnan(pu) && isnan(v) == isnan(pv)) return 0xFFFFFFFFu;
    counts = true;
    return 0x7F800000u;
  }
  counts = true;
  return __float_as_uint(fmaxf(du, dv));
}

// 95th percentile (Statistics.quantile! type 7) of n counted keys given the
// two order statistics it interpolates: index helper and final formula.
__device__ __forceinline__ void quantile95_index(int64_t n, int64_t& ka, int64_t& kb, double& g) {
  const double aleph = fma((double)n, 0.95, 0.05);
  int64_t j = (int64_t)trunc(aleph);
  const int64_t hi = n - 1 > 1 ? n - 1 : 1;
  j = j < 1 ? 1 : (j > hi ? hi : j);
  g = aleph - (double)j;
  g = g < 0 ? 0 : (g > 1 ? 1 : g);
  ka = n == 1 ? 0 : j - 1;
  kb = n == 1 ? 0 : j;
}
__device__ __forceinline__ float quantile95_value(uint32_t ka, uint32_t kb, double g) {
  const float a = __uint_as_float(ka), b = __uint_as_float(kb);
  double q;
  if (isfinite(a) && isfinite(b)) q = __dadd_rn((double)a, __dmul_rn(g, (double)FSUB(b, a)));
  else q = __dadd_rn(__dmul_rn(1.0 - g, (double)a), __dmul_rn(g, (double)b));
  return (float)q;
}

// k-th smallest (0-based) of keys[0, n) by a 4 x 8-bit radix select, run by
// one whole CTA (hist: 256 shared counters; s_bucket, s_k: shared scalars).
__device__ __forceinline__ uint32_t cta_radix_select(const uint32_t* keys, int64_t n, int64_t kth, uint32_t* hist,
                                                     uint32_t* s_bucket, int64_t* s_k) {
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

}  // namespace hh
