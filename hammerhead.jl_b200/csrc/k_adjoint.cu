// Adjoint of deformation + zero-lag correlation (sm_100a).
//
// Loss of a predictor field P = (u, v) on a uniform node grid:
//   L(P) = - sum over windows j of NCC0_j,
//   NCC0_j = sum (a - abar)(b - bbar) / sqrt(sum (a - abar)^2 sum (b - bbar)^2)
// over the W x W pixels of window j of the pair deformed by P exactly as a
// WIDIM sweep deforms it (bilinear predictor with flat extrapolation, cubic
// B-spline samples at -+ (u, v)/2; deform_columns!, src/pipeline.jl:957-965).
//
// Three launches, no atomics, no stored deformed image:
//   1. per window (one CTA): recompute the deformed window, FP64 moments,
//      and the window constants of the gradient;
//   2. per pixel: recompute the deformed samples and their B-spline
//      derivatives, sum dL/da, dL/db over the windows holding the pixel,
//      chain through -+ 1/2 to the pixel displacement gradient (gu, gv);
//   3. per node: the transpose of the bilinear predictor interpolation,
//      gathered over the node's support in FP64.
#include <math.h>
#include <stdint.h>

#include "hh_internal.h"

namespace hh {

namespace {

__device__ __forceinline__ void cubw_f(float d, float* w) {
  const float x3 = d * d * d, c = 1.f - d, c3 = c * c * c;
  w[0] = c3 / 6.f;
  w[1] = 2.f / 3.f - d * d + x3 / 2.f;
  w[2] = 2.f / 3.f - c * c + c3 / 2.f;
  w[3] = x3 / 6.f;
}
// d/dd of the cubic B-spline weights
__device__ __forceinline__ void cubw_df(float d, float* w) {
  const float c = 1.f - d;
  w[0] = -0.5f * c * c;
  w[1] = -2.f * d + 1.5f * d * d;
  w[2] = 2.f * c - 1.5f * c * c;
  w[3] = 0.5f * d * d;
}

// zero-extrapolated cubic B-spline sample at 1-based (yy, xx); with GRAD
// also its derivatives along rows (gy) and columns (gx)
template <bool GRAD>
__device__ __forceinline__ float bs_sample(const float* __restrict__ C, int64_t nr, int64_t nc, float yy, float xx,
                                           float& gy, float& gx) {
  gy = gx = 0.f;
  if (yy < 1.f || yy > (float)nr || xx < 1.f || xx > (float)nc) return 0.f;
  int64_t iy = (int64_t)floorf(yy);
  if (iy > nr - 1) iy = nr - 1;
  int64_t ix = (int64_t)floorf(xx);
  if (ix > nc - 1) ix = nc - 1;
  float wy[4], wx[4], dy[4], dx[4];
  cubw_f(yy - (float)iy, wy);
  cubw_f(xx - (float)ix, wx);
  if (GRAD) {
    cubw_df(yy - (float)iy, dy);
    cubw_df(xx - (float)ix, dx);
  }
  const int64_t ld = nr + 2;
  const float* base = C + (iy - 1) + (ix - 1) * ld;
  float s = 0.f, sy = 0.f, sx = 0.f;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    float t = 0.f, tx = 0.f;
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const float c = __ldg(base + a + b * ld);
      t += wx[b] * c;
      if (GRAD) tx += dx[b] * c;
    }
    s += wy[a] * t;
    if (GRAD) {
      sy += dy[a] * t;
      sx += wy[a] * tx;
    }
  }
  gy = sy;
  gx = sx;
  return s;
}

// Gridded(Linear()) + Flat() along one axis (as the deformation kernel)
__device__ __forceinline__ void lin_axis_f(float q, float q0, float step, int n, int& i, float& d) {
  if (n == 1) { i = 0; d = 0.f; return; }
  const float last = __fadd_rn(q0, __fmul_rn((float)(n - 1), step));
  if (q <= q0) { i = 0; d = 0.f; return; }
  if (q >= last) { i = n - 2; d = 1.f; return; }
  i = (int)floorf(__fdiv_rn(__fsub_rn(q, q0), step));
  if (i > n - 2) i = n - 2;
  const float k0 = __fadd_rn(q0, __fmul_rn((float)i, step)), k1 = __fadd_rn(q0, __fmul_rn((float)(i + 1), step));
  d = __fdiv_rn(__fsub_rn(q, k0), __fsub_rn(k1, k0));
}

__device__ __forceinline__ float bilin(const float* f, const NccArgs& a, float qy, float qx) {
  int iy, ix;
  float dy, dx;
  lin_axis_f(qy, a.y0, a.ysp, a.gny, iy, dy);
  lin_axis_f(qx, a.x0, a.xsp, a.gnx, ix, dx);
  const int iy2 = a.gny == 1 ? iy : iy + 1, ix2 = a.gnx == 1 ? ix : ix + 1;
  const float f00 = f[iy + ix * a.gny], f01 = f[iy + ix2 * a.gny], f10 = f[iy2 + ix * a.gny],
              f11 = f[iy2 + ix2 * a.gny];
  const float p = __fadd_rn(__fmul_rn(__fsub_rn(1.f, dx), f00), __fmul_rn(dx, f01));
  const float q = __fadd_rn(__fmul_rn(__fsub_rn(1.f, dx), f10), __fmul_rn(dx, f11));
  return __fadd_rn(__fmul_rn(__fsub_rn(1.f, dy), p), __fmul_rn(dy, q));
}

// deformed samples of pixel (r, c) (0-based) of both frames
template <bool GRAD>
__device__ __forceinline__ void deformed(const NccArgs& a, int64_t r, int64_t c, float& va, float& vb, float& ay,
                                         float& ax, float& by, float& bx) {
  const float R = (float)(r + 1), Cc = (float)(c + 1);
  const float u2 = __fdiv_rn(bilin(a.P, a, R, Cc), 2.f);
  const float v2 = __fdiv_rn(bilin(a.P + (int64_t)a.gny * a.gnx, a, R, Cc), 2.f);
  va = bs_sample<GRAD>(a.CA, a.nr, a.nc, __fsub_rn(R, v2), __fsub_rn(Cc, u2), ay, ax);
  vb = bs_sample<GRAD>(a.CB, a.nr, a.nc, __fadd_rn(R, v2), __fadd_rn(Cc, u2), by, bx);
}

constexpr int NCC_THREADS = 256;

__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  __syncthreads();
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < NCC_THREADS / 32; ++w) t += red[w];
  return t;
}

// 1. window constants: ncc, abar, bbar, inv = 1/sqrt(Saa Sbb), ca = ncc/Saa, cb = ncc/Sbb
template <int PPT>
__global__ void __launch_bounds__(NCC_THREADS) ncc_window_kernel(const NccArgs a) {
  __shared__ double red[NCC_THREADS / 32];
  const int W = a.W, n = W * W;
  const int64_t nwin = (int64_t)a.wy * a.wx;
  for (int64_t j = blockIdx.x; j < nwin; j += gridDim.x) {
    const int64_t rs = (j % a.wy) * a.step, cs = (j / a.wy) * a.step;
    float va[PPT], vb[PPT];
    double sa = 0.0, sb = 0.0;
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
      const int k = threadIdx.x + i * NCC_THREADS;
      va[i] = vb[i] = 0.f;
      if (k < n) {
        float d0, d1, d2, d3;
        deformed<false>(a, rs + k % W, cs + k / W, va[i], vb[i], d0, d1, d2, d3);
        sa += (double)va[i];
        sb += (double)vb[i];
      }
    }
    const double ma = block_sum(sa, red) / n, mb = block_sum(sb, red) / n;
    double saa = 0.0, sbb = 0.0, sab = 0.0;
#pragma unroll
    for (int i = 0; i < PPT; ++i) {
      const int k = threadIdx.x + i * NCC_THREADS;
      if (k < n) {
        const double da = (double)va[i] - ma, db = (double)vb[i] - mb;
        saa += da * da;
        sbb += db * db;
        sab += da * db;
      }
    }
    saa = block_sum(saa, red);
    sbb = block_sum(sbb, red);
    sab = block_sum(sab, red);
    if (threadIdx.x == 0) {
      double* o = a.wstat + 6 * j;
      if (saa > 0 && sbb > 0) {
        const double inv = 1.0 / sqrt(saa * sbb), ncc = sab * inv;
        o[0] = ncc;
        o[1] = ma;
        o[2] = mb;
        o[3] = inv;
        o[4] = ncc / saa;
        o[5] = ncc / sbb;
      } else {  // a flat window contributes nothing
        o[0] = o[1] = o[2] = o[3] = o[4] = o[5] = 0.0;
      }
    }
  }
}

// 2. pixel displacement gradient (gu, gv) = dL/d(u, v) at every pixel
__global__ void __launch_bounds__(256) ncc_pixel_kernel(const NccArgs a) {
  const int64_t P = a.nr * a.nc;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < P; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = k % a.nr, c = k / a.nr;
    // windows j = (jr, jc) with jr*step <= r < jr*step + W
    const int64_t jr0 = r - a.W + 1 <= 0 ? 0 : (r - a.W + 1 + a.step - 1) / a.step;
    const int64_t jr1 = min((int64_t)a.wy - 1, r / a.step);
    const int64_t jc0 = c - a.W + 1 <= 0 ? 0 : (c - a.W + 1 + a.step - 1) / a.step;
    const int64_t jc1 = min((int64_t)a.wx - 1, c / a.step);
    float gu = 0.f, gv = 0.f;
    if (jr0 <= jr1 && jc0 <= jc1) {
      float va, vb, ay, ax, by, bx;
      deformed<true>(a, r, c, va, vb, ay, ax, by, bx);
      double ga = 0.0, gb = 0.0;
      for (int64_t jc = jc0; jc <= jc1; ++jc)
        for (int64_t jr = jr0; jr <= jr1; ++jr) {
          const double* s = a.wstat + 6 * (jr + jc * a.wy);
          const double da = (double)va - s[1], db = (double)vb - s[2];
          ga += -db * s[3] + s[4] * da;
          gb += -da * s[3] + s[5] * db;
        }
      const float fa = (float)ga, fb = (float)gb;
      gu = fa * (-0.5f * ax) + fb * (0.5f * bx);
      gv = fa * (-0.5f * ay) + fb * (0.5f * by);
    }
    a.gpix[k] = gu;
    a.gpix[P + k] = gv;
  }
}

// bilinear weight of node g for query q (flat outside)
__device__ __forceinline__ float node_w(float q, float q0, float step, int n, int g) {
  int i;
  float d;
  lin_axis_f(q, q0, step, n, i, d);
  const int i2 = n == 1 ? i : i + 1;
  return (i == g ? 1.f - d : 0.f) + (i2 == g ? d : 0.f);
}

// 3. dL/dP at every node: the transpose of the bilinear interpolation
__global__ void __launch_bounds__(256) ncc_node_kernel(const NccArgs a) {
  const int64_t G = (int64_t)a.gny * a.gnx;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < 2 * G; k += (int64_t)gridDim.x * blockDim.x) {
    const int comp = (int)(k / G);
    const int64_t node = k % G;
    const int gy = (int)(node % a.gny), gx = (int)(node / a.gny);
    // 1-based pixel rows / columns whose stencil may reach the node
    const int64_t r_lo = gy == 0 ? 1 : max((int64_t)1, (int64_t)floorf(a.y0 + (gy - 1) * a.ysp));
    const int64_t r_hi = gy == a.gny - 1 ? a.nr : min(a.nr, (int64_t)ceilf(a.y0 + (gy + 1) * a.ysp));
    const int64_t c_lo = gx == 0 ? 1 : max((int64_t)1, (int64_t)floorf(a.x0 + (gx - 1) * a.xsp));
    const int64_t c_hi = gx == a.gnx - 1 ? a.nc : min(a.nc, (int64_t)ceilf(a.x0 + (gx + 1) * a.xsp));
    const float* g = a.gpix + comp * a.nr * a.nc;
    double acc = 0.0;
    for (int64_t C = c_lo; C <= c_hi; ++C) {
      const float wx = node_w((float)C, a.x0, a.xsp, a.gnx, gx);
      if (wx == 0.f) continue;
      double col = 0.0;
      for (int64_t R = r_lo; R <= r_hi; ++R) {
        const float wy = node_w((float)R, a.y0, a.ysp, a.gny, gy);
        if (wy != 0.f) col += (double)wy * (double)g[(R - 1) + (C - 1) * a.nr];
      }
      acc += (double)wx * col;
    }
    a.grad[k] = (float)acc;
  }
}

// loss = -sum of the window correlations, in window order (one CTA)
__global__ void __launch_bounds__(NCC_THREADS) ncc_loss_kernel(const NccArgs a) {
  __shared__ double red[NCC_THREADS / 32];
  const int64_t nwin = (int64_t)a.wy * a.wx;
  double s = 0.0;
  for (int64_t j = threadIdx.x; j < nwin; j += NCC_THREADS) s += a.wstat[6 * j];
  s = block_sum(s, red);
  if (threadIdx.x == 0) *a.loss = -s;
}

template <int PPT> static void launch_win(const NccArgs& a, int64_t nwin, cudaStream_t s) {
  const int64_t grid = nwin < 148 * 8 ? nwin : 148 * 8;
  ncc_window_kernel<PPT><<<(unsigned)grid, NCC_THREADS, 0, s>>>(a);
}

}  // namespace

cudaError_t launch_ncc_loss_grad(const NccArgs& a, cudaStream_t s) {
  const int64_t nwin = (int64_t)a.wy * a.wx;
  if (nwin <= 0 || a.W < 2) return cudaErrorInvalidValue;
  const int n = a.W * a.W;
  if (n <= NCC_THREADS) launch_win<1>(a, nwin, s);
  else if (n <= 4 * NCC_THREADS) launch_win<4>(a, nwin, s);
  else if (n <= 16 * NCC_THREADS) launch_win<16>(a, nwin, s);
  else return cudaErrorInvalidValue;
  ncc_loss_kernel<<<1, NCC_THREADS, 0, s>>>(a);
  if (a.grad) {
    const int64_t P = a.nr * a.nc, G2 = 2 * (int64_t)a.gny * a.gnx;
    int64_t b1 = (P + 255) / 256, b2 = (G2 + 255) / 256;
    if (b1 > 148 * 16) b1 = 148 * 16;
    if (b2 > 148 * 16) b2 = 148 * 16;
    ncc_pixel_kernel<<<(unsigned)b1, 256, 0, s>>>(a);
    ncc_node_kernel<<<(unsigned)(b2 < 1 ? 1 : b2), 256, 0, s>>>(a);
  }
  return cudaGetLastError();
}

}  // namespace hh
