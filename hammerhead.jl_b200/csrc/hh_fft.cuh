// Register-resident DFTs for the fused correlation kernel.
//
// RDFT<R, INV>::run(x, nz) transforms R complex values held in registers, in
// natural order in and out: forward X[k] = sum_n x[n] exp(-2 pi i nk/R), INV
// uses exp(+...). Inputs x[n] with n >= nz are known to be zero (the zero
// padding of `padding = true` windows); nz is a compile-time constant at every
// call site after unrolling, so the skipped terms cost nothing.
//
// Composite sizes use the four-step split R = A*B (n = B*n1 + n2,
// k = k1 + A*k2): A-point DFTs over n1, twiddle W_R^{n2 k1}, B-point DFTs
// over n2. Twiddles come from the 96-point table (every R used divides 96).
#pragma once
#include "hh_twiddle.cuh"

namespace hh {

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// multiply by -i (forward) or +i (inverse)
template <bool INV> __device__ __forceinline__ float2 mul_mi(float2 v) {
  return INV ? make_float2(-v.y, v.x) : make_float2(v.y, -v.x);
}
// v * exp(-+2 pi i j / 96), j a compile-time constant after unrolling
template <bool INV> __device__ __forceinline__ float2 tw96mul(float2 v, int j) {
  j = ((j % 96) + 96) % 96;
  if (j == 0) return v;
  if (j == 24) return mul_mi<INV>(v);
  if (j == 48) return make_float2(-v.x, -v.y);
  if (j == 72) return mul_mi<!INV>(v);
  const float c = (float)cos96(j);
  const float s = INV ? (float)sin96(j) : -(float)sin96(j);
  return make_float2(v.x * c - v.y * s, v.x * s + v.y * c);
}

template <int R, bool INV> struct RDFT;

template <bool INV> struct RDFT<1, INV> {
  static __device__ __forceinline__ void run(float2*, int = 1) {}
};

template <bool INV> struct RDFT<2, INV> {
  static __device__ __forceinline__ void run(float2* x, int nz = 2) {
    if (nz <= 0) return;
    if (nz == 1) { x[1] = x[0]; return; }
    float2 a = cadd(x[0], x[1]), b = csub(x[0], x[1]);
    x[0] = a;
    x[1] = b;
  }
};

template <bool INV> struct RDFT<3, INV> {
  static __device__ __forceinline__ void run(float2* x, int nz = 3) {
    if (nz <= 0) return;
    if (nz == 1) { x[1] = x[0]; x[2] = x[0]; return; }
    const float h = 0.86602540378443865f;  // sqrt(3)/2
    float2 x2 = nz >= 3 ? x[2] : make_float2(0.f, 0.f);
    float2 t = nz >= 3 ? cadd(x[1], x2) : x[1];
    float2 d = nz >= 3 ? csub(x[1], x2) : x[1];
    float2 X0 = cadd(x[0], t);
    float2 m = make_float2(x[0].x - 0.5f * t.x, x[0].y - 0.5f * t.y);
    float2 r = make_float2(h * d.x, h * d.y);
    // W x1 + W^2 x2 = -(x1+x2)/2 -+ i sqrt(3)/2 (x1-x2)
    float2 ir = mul_mi<INV>(r);  // -i r forward, +i r inverse
    x[0] = X0;
    x[1] = cadd(m, ir);
    x[2] = csub(m, ir);
  }
};

template <bool INV> struct RDFT<4, INV> {
  static __device__ __forceinline__ void run(float2* x, int nz = 4) {
    if (nz <= 0) return;
    if (nz == 1) { x[1] = x[2] = x[3] = x[0]; return; }
    float2 a0, a1, b0, b1;
    if (nz == 2) {
      a0 = a1 = x[0];
      b0 = b1 = x[1];
    } else {
      a0 = cadd(x[0], x[2]);
      a1 = csub(x[0], x[2]);
      if (nz == 3) {
        b0 = b1 = x[1];
      } else {
        b0 = cadd(x[1], x[3]);
        b1 = csub(x[1], x[3]);
      }
    }
    float2 jb = mul_mi<INV>(b1);
    x[0] = cadd(a0, b0);
    x[2] = csub(a0, b0);
    x[1] = cadd(a1, jb);
    x[3] = csub(a1, jb);
  }
};

template <int R, bool INV> struct RDFT {
  static constexpr int A = (R % 4 == 0) ? 4 : ((R % 2 == 0) ? 2 : 3);
  static constexpr int B = R / A;
  static_assert(A * B == R, "unsupported radix");
  static_assert(96 % R == 0, "radix must divide 96");
  static __device__ __forceinline__ void run(float2* x, int nz = R) {
    float2 y[R];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) {
      float2 s[A];
      // inputs x[B*n1 + n2], nonzero while B*n1 + n2 < nz
      const int nzA = (nz - n2 + B - 1) / B < 0 ? 0 : ((nz - n2 + B - 1) / B > A ? A : (nz - n2 + B - 1) / B);
#pragma unroll
      for (int n1 = 0; n1 < A; ++n1) s[n1] = (n1 < nzA) ? x[B * n1 + n2] : make_float2(0.f, 0.f);
      RDFT<A, INV>::run(s, nzA);
#pragma unroll
      for (int k1 = 0; k1 < A; ++k1)
        y[k1 * B + n2] = (nzA > 0) ? tw96mul<INV>(s[k1], (n2 * k1) * (96 / R)) : make_float2(0.f, 0.f);
    }
    const int nzB = nz < B ? nz : B;
#pragma unroll
    for (int k1 = 0; k1 < A; ++k1) {
      float2 t[B];
#pragma unroll
      for (int n2 = 0; n2 < B; ++n2) t[n2] = y[k1 * B + n2];
      RDFT<B, INV>::run(t, nzB);
#pragma unroll
      for (int k2 = 0; k2 < B; ++k2) x[k1 + A * k2] = t[k2];
    }
  }
};

// Split of an N-point axis into an in-register radix N1 and a second radix
// N2 applied after one exchange through shared memory (N = N1 * N2).
template <int N> struct AxisSplit;
template <> struct AxisSplit<16> { static constexpr int N1 = 16, N2 = 1; };
template <> struct AxisSplit<24> { static constexpr int N1 = 24, N2 = 1; };
template <> struct AxisSplit<32> { static constexpr int N1 = 32, N2 = 1; };
template <> struct AxisSplit<48> { static constexpr int N1 = 8, N2 = 6; };
template <> struct AxisSplit<64> { static constexpr int N1 = 16, N2 = 4; };
template <> struct AxisSplit<96> { static constexpr int N1 = 12, N2 = 8; };
template <> struct AxisSplit<128> { static constexpr int N1 = 16, N2 = 8; };

// The alternative split the autotuner times against AxisSplit: a shorter
// in-register radix and a longer second pass (one more exchange through
// shared memory for N <= 32, fewer live registers per item).
template <int N> struct AxisSplitAlt;
template <> struct AxisSplitAlt<16> { static constexpr int N1 = 4, N2 = 4; };
template <> struct AxisSplitAlt<24> { static constexpr int N1 = 6, N2 = 4; };
template <> struct AxisSplitAlt<32> { static constexpr int N1 = 8, N2 = 4; };
template <> struct AxisSplitAlt<48> { static constexpr int N1 = 12, N2 = 4; };
template <> struct AxisSplitAlt<64> { static constexpr int N1 = 8, N2 = 8; };
template <> struct AxisSplitAlt<96> { static constexpr int N1 = 8, N2 = 12; };
template <> struct AxisSplitAlt<128> { static constexpr int N1 = 8, N2 = 16; };

}  // namespace hh
