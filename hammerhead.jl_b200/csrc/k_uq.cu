// Wieneke (2015) correlation-statistics uncertainty (sm_100a).
//
// One CTA per interrogation window (grid-stride over jobs). It restates
// src/uncertainty.jl:51-179: the windows are mean-subtracted (column-major
// fold) and apodized exactly like load_windows!, the per-pixel correlation
// difference dC = a0*b1 - a1*b0 and its (1,2,1)/4 smoothing are formed in
// FP32, and the 2 x 44 statistics (C0, C+, C-, S00 and the 40 half-plane
// covariance sums of rings 1..4) are reduced in FP64. Each statistic is
// summed by one thread in the reference's loop order with explicit
// round-to-nearest FP64 arithmetic, so the sums equal the CPU restatement
// bit for bit; finalize_uncertainty (:162-179) then runs on the same thread.
#include <math.h>
#include <stdint.h>

#include "hh_internal.h"

namespace hh {

// covariance offsets (dr, dc) of one half-plane, ring 1..4 (UQ_OFFSETS,
// src/uncertainty.jl:16-35): dc in 0:4, dr in (dc == 0 ? 1:4 : -4:4), stably
// ordered by ring max(|dr|, |dc|).
struct UQOffsets {
  int8_t dr[40], dc[40];
  int8_t ring_start[5];
};
static UQOffsets make_offsets() {
  UQOffsets o{};
  int tmp[40][2], n = 0;
  for (int dc = 0; dc <= 4; ++dc)
    for (int dr = (dc == 0 ? 1 : -4); dr <= 4; ++dr) {
      tmp[n][0] = dr;
      tmp[n][1] = dc;
      ++n;
    }
  int k = 0;
  for (int ring = 1; ring <= 4; ++ring) {
    o.ring_start[ring - 1] = (int8_t)k;
    for (int q = 0; q < 40; ++q) {
      int a = tmp[q][0] < 0 ? -tmp[q][0] : tmp[q][0];
      int b = tmp[q][1];
      if ((a > b ? a : b) == ring) {
        o.dr[k] = (int8_t)tmp[q][0];
        o.dc[k] = (int8_t)tmp[q][1];
        ++k;
      }
    }
  }
  o.ring_start[4] = 40;
  return o;
}

__device__ __forceinline__ float uq_finalize(const double* s, const UQOffsets& o) {
  const double C0 = s[0], Cp = s[1], Cm = s[2], S00 = s[3];
  double s2 = S00;
  for (int ring = 0; ring < 4; ++ring) {
    double mx = -INFINITY;
    for (int k = o.ring_start[ring]; k < o.ring_start[ring + 1]; ++k) mx = fmax(mx, s[4 + k]);
    if (mx < __dmul_rn(0.05, S00)) break;
    for (int k = o.ring_start[ring]; k < o.ring_start[ring + 1]; ++k) s2 = __dadd_rn(s2, __dmul_rn(2.0, s[4 + k]));
  }
  const double sdc = sqrt(fmax(s2, 0.0));
  const double Cpm = __dadd_rn(Cp, Cm) / 2.0;
  const double lo = __dsub_rn(Cpm, sdc / 2.0), hi = __dadd_rn(Cpm, sdc / 2.0);
  if (!(C0 > 0 && lo > 0)) return __int_as_float(0x7fc00000);
  const double lhi = log(hi), llo = log(lo);
  const double denom = __dsub_rn(__dsub_rn(__dmul_rn(2.0, log(C0)), lhi), llo);
  if (!(denom > 0)) return __int_as_float(0x7fc00000);
  return (float)(__dsub_rn(lhi, llo) / __dmul_rn(2.0, denom));
}

// Statistic `si` (0..43) of one component over the smoothed field dCs
// (nr x m, column-major, leading dim nr) and windows wa/wb viewed through
// (str, stc) strides.
__device__ double uq_stat(int si, const float* wa, const float* wb, int str, int stc, int nr, int m,
                          const float* dCs, double mu, const UQOffsets& o) {
  double acc = 0.0;
  if (si < 3) {
    for (int c = 0; c < m; ++c)
      for (int r = 0; r < nr; ++r) {
        const float a0 = wa[r * str + c * stc], a1 = wa[r * str + (c + 1) * stc];
        const float b0 = wb[r * str + c * stc], b1 = wb[r * str + (c + 1) * stc];
        const float pr = si == 0 ? __fmul_rn(a0, b0) : (si == 1 ? __fmul_rn(a0, b1) : __fmul_rn(a1, b0));
        acc = __dadd_rn(acc, (double)pr);
      }
    return acc;
  }
  if (si == 3) {
    for (int c = 0; c < m; ++c)
      for (int r = 0; r < nr; ++r) {
        const double d = __dsub_rn((double)dCs[r + c * nr], mu);
        acc = __dadd_rn(acc, __dmul_rn(d, d));
      }
    return acc;
  }
  const int k = si - 4, dr = o.dr[k], dc = o.dc[k];
  const int c0 = 1 > 1 - dc ? 1 : 1 - dc, c1 = m < m - dc ? m : m - dc;
  const int r0 = 1 > 1 - dr ? 1 : 1 - dr, r1 = nr < nr - dr ? nr : nr - dr;
  for (int c = c0; c <= c1; ++c)
    for (int r = r0; r <= r1; ++r) {
      const double d1 = __dsub_rn((double)dCs[(r - 1) + (c - 1) * nr], mu);
      const double d2 = __dsub_rn((double)dCs[(r - 1 + dr) + (c - 1 + dc) * nr], mu);
      acc = __dadd_rn(acc, __dmul_rn(d1, d2));
    }
  return acc;
}

__global__ void __launch_bounds__(128) uq_kernel(const UQArgs a, const UQOffsets o) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = a.W, m = W - 1;
  float* wa = reinterpret_cast<float*>(smem_raw);  // W*W
  float* wb = wa + W * W;                           // W*W
  float* dC = wb + W * W;                           // 2 * W*m (u then v)
  float* dCs = dC + 2 * W * m;                      // 2 * W*m
  double* stats = reinterpret_cast<double*>(dCs + 2 * W * m + ((2 * W * m) & 1));  // 88
  __shared__ float s_mean[2];
  __shared__ double s_mu[2];
  __shared__ int s_any;
  const int tid = threadIdx.x;
  for (int64_t job = blockIdx.x; job < a.njobs; job += gridDim.x) {
    const int rs = a.jobs[4 * job + 2], cs = a.jobs[4 * job + 3];
    if (tid == 0) s_any = 0;
    __syncthreads();
    for (int k = tid; k < W * W; k += blockDim.x) {
      const int p = k % W, q = k / W;
      const int64_t off = (int64_t)(rs + p) + (int64_t)(cs + q) * a.ld;
      wa[k] = a.A[off];
      wb[k] = a.B[off];
      if (a.mask && a.mask[off]) s_any = 1;
    }
    __syncthreads();
    // means (load_uncertainty_windows!, :51-83)
    if (tid < 2) {
      const float* x = tid == 0 ? wa : wb;
      float s = 0.f;
      int n = 0;
      if (!s_any) {
        s = x[0];
        for (int k = 1; k < W * W; ++k) s = __fadd_rn(s, x[k]);
        n = W * W;
      } else {
        for (int k = 0; k < W * W; ++k) {
          const int p = k % W, q = k / W;
          if (a.mask[(int64_t)(rs + p) + (int64_t)(cs + q) * a.ld]) continue;
          s = __fadd_rn(s, x[k]);
          ++n;
        }
      }
      s_mean[tid] = n > 0 ? __fdiv_rn(s, (float)n) : 0.f;
    }
    __syncthreads();
    for (int k = tid; k < W * W; k += blockDim.x) {
      const int p = k % W, q = k / W;
      bool masked = s_any && a.mask[(int64_t)(rs + p) + (int64_t)(cs + q) * a.ld];
      const float ap = a.apod[k];
      wa[k] = masked ? 0.f : __fmul_rn(ap, __fsub_rn(wa[k], s_mean[0]));
      wb[k] = masked ? 0.f : __fmul_rn(ap, __fsub_rn(wb[k], s_mean[1]));
    }
    __syncthreads();
    // dC for both components: u views (r, c) = (p, q); v views (r, c) = (q, p)
    for (int k = tid; k < 2 * W * m; k += blockDim.x) {
      const int comp = k / (W * m), e = k % (W * m), r = e % W, c = e / W;
      const int str = comp == 0 ? 1 : W, stc = comp == 0 ? W : 1;
      const float a0 = wa[r * str + c * stc], a1 = wa[r * str + (c + 1) * stc];
      const float b0 = wb[r * str + c * stc], b1 = wb[r * str + (c + 1) * stc];
      dC[k] = __fsub_rn(__fmul_rn(a0, b1), __fmul_rn(a1, b0));
    }
    __syncthreads();
    for (int k = tid; k < 2 * W * m; k += blockDim.x) {
      const int comp = k / (W * m), e = k % (W * m), r = e % W, c = e / W;
      const float* d = dC + comp * W * m;
      const int cl = c > 0 ? c - 1 : 0, cr = c < m - 1 ? c + 1 : m - 1;
      dCs[k] = __fmul_rn(0.25f, __fadd_rn(__fadd_rn(d[r + cl * W], __fmul_rn(2.0f, d[r + c * W])), d[r + cr * W]));
    }
    __syncthreads();
    if (tid < 2) {
      const float* d = dCs + tid * W * m;
      double mu = 0.0;
      for (int c = 0; c < m; ++c)
        for (int r = 0; r < W; ++r) mu = __dadd_rn(mu, (double)d[r + c * W]);
      s_mu[tid] = mu / (double)(W * m);
    }
    __syncthreads();
    for (int it = tid; it < 88; it += blockDim.x) {
      const int comp = it / 44, si = it % 44;
      const int str = comp == 0 ? 1 : W, stc = comp == 0 ? W : 1;
      stats[it] = uq_stat(si, wa, wb, str, stc, W, m, dCs + comp * W * m, s_mu[comp], o);
    }
    __syncthreads();
    if (a.stats)
      for (int it = tid; it < 88; it += blockDim.x) a.stats[job * 88 + it] = stats[it];
    if (a.unc_u && tid < 2) {
      const int64_t gid = (int64_t)a.jobs[4 * job] + (int64_t)a.jobs[4 * job + 1] * a.ny;
      const float sg = uq_finalize(stats + 44 * tid, o);
      if (tid == 0) a.unc_u[gid] = sg;
      else a.unc_v[gid] = sg;
    }
    __syncthreads();
  }
}

cudaError_t launch_uq(const UQArgs& a, cudaStream_t s, int num_sms) {
  if (a.njobs <= 0) return cudaSuccess;
  static const UQOffsets offs = make_offsets();
  const int W = a.W, m = W - 1;
  const size_t sm = (size_t)(2 * W * W + 4 * W * m + 2) * sizeof(float) + 88 * sizeof(double) + 16;
  if (sm > 200 * 1024) return cudaErrorInvalidValue;
  cudaError_t e = cudaFuncSetAttribute(uq_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, uq_kernel, 128, sm);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * num_sms;
  if (grid > a.njobs) grid = a.njobs;
  uq_kernel<<<(unsigned)grid, 128, sm, s>>>(a, offs);
  return cudaGetLastError();
}

}  // namespace hh
