// Hammerhead planar-WIDIM CPU oracle.
//
// TEST INFRASTRUCTURE ONLY. This file is the checker for the sm_100a library:
// a plain CPU restatement of the reference (stillyslalom/Hammerhead.jl, Julia)
// planar WIDIM path, instantiated in float (the reference's Float32 pipeline)
// and double (the FP64 oracle). Only tests/, __graft_entry__.smoke() and the
// CPU-baseline legs of bench.py load it; the product library never links it.
//
// Parity status
//   * pinned: peak finding / tie rules, gauss3 / gauss9, moment, peak ratio,
//     UOD, substitution, replacement, smoothing, validators, pass grid,
//     multipass schedule identities -- against the reference's own
//     known-answer tests (test/runtests.jl, test/test_peaks.jl,
//     test/test_ka.jl, test/test_validation.jl, test/test_accuracy.jl),
//     restated as pytest cases in tests/test_oracle_golden.py.
//   * FFT: the reference calls FFTW (FFTW.jl compat 1.8, not vendored). The
//     DFT below is an own mixed-radix restatement of the published transform,
//     checked against numpy.fft in FP64. Bit-level FFT round-off is unpinned.
//   * Cubic B-spline prefilter: the reference calls Interpolations.jl
//     (compat 0.16, not vendored), BSpline(Cubic(Line(OnGrid()))). The system
//     solved here is the published one (interior rows [1 4 1]/6, "Line"
//     boundary rows c0 - 2c1 + c2 = 0 on the padded index set); boundary-row
//     round-off is unpinned.
//   * Statistics.median!/quantile! (type 7) are restated from their
//     definitions.
//
// Arithmetic follows the Julia code: T-typed (float) arithmetic where Julia
// uses T, Float64 islands where Julia widens. Build with -ffp-contract=off so
// no multiply-add is fused (Julia does not contract).

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <limits>
#include <thread>
#include <vector>

namespace orc {

using i64 = int64_t;

template <class T> struct cx {
  T re, im;
};
template <class T> static inline cx<T> cadd(cx<T> a, cx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <class T> static inline cx<T> csub(cx<T> a, cx<T> b) { return {a.re - b.re, a.im - b.im}; }
// Julia's Complex * Complex: (ar*br - ai*bi, ar*bi + ai*br)
template <class T> static inline cx<T> cmul(cx<T> a, cx<T> b) {
  return {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
template <class T> static inline T cabs_(cx<T> a) { return std::hypot(a.re, a.im); }

// ---------------------------------------------------------------------------
// Mixed-radix DFT (own restatement of the transform FFTW computes: forward
// unnormalised e^{-2 pi i jk/n}; inverse e^{+2 pi i jk/n}).
template <class T> struct FFT1 {
  int n = 0;
  std::vector<int> fac;
  std::vector<double> twr, twi;  // W_n^k, k = 0..n-1, in double
  std::vector<cx<T>> buf;
  explicit FFT1(int n_ = 1) { init(n_); }
  void init(int n_) {
    n = n_;
    fac.clear();
    int m = n;
    while (m % 4 == 0) { fac.push_back(4); m /= 4; }
    while (m % 2 == 0) { fac.push_back(2); m /= 2; }
    for (int p = 3; m > 1; p += 2)
      while (m % p == 0) { fac.push_back(p); m /= p; }
    twr.resize(n);
    twi.resize(n);
    for (int k = 0; k < n; ++k) {
      double a = -2.0 * M_PI * (double)k / (double)n;
      twr[k] = std::cos(a);
      twi[k] = std::sin(a);
    }
    buf.resize(n);
  }
  cx<T> w(int k, bool inv) const {  // W_n^k (conjugated for inverse)
    k %= n;
    if (k < 0) k += n;
    return {(T)twr[k], inv ? (T)(-twi[k]) : (T)twi[k]};
  }
  void rec(const cx<T>* in, int istride, cx<T>* out, int len, int fi, bool inv) {
    if (len == 1) { out[0] = in[0]; return; }
    int p = fac[fi], m = len / p;
    for (int q = 0; q < p; ++q) rec(in + (i64)q * istride, istride * p, out + q * m, m, fi + 1, inv);
    int step = n / len;  // W_len^j = W_n^{j*step}
    cx<T> t[64], y[64];
    for (int k = 0; k < m; ++k) {
      for (int q = 0; q < p; ++q) {
        cx<T> v = out[q * m + k];
        t[q] = (q == 0 || k == 0) ? v : cmul(v, w(q * k * step, inv));
      }
      if (p == 2) {
        y[0] = cadd(t[0], t[1]);
        y[1] = csub(t[0], t[1]);
      } else if (p == 4) {
        cx<T> a0 = cadd(t[0], t[2]), a1 = csub(t[0], t[2]);
        cx<T> b0 = cadd(t[1], t[3]), b1 = csub(t[1], t[3]);
        // -i*b1 forward, +i*b1 inverse
        cx<T> jb1 = inv ? cx<T>{-b1.im, b1.re} : cx<T>{b1.im, -b1.re};
        y[0] = cadd(a0, b0);
        y[2] = csub(a0, b0);
        y[1] = cadd(a1, jb1);
        y[3] = csub(a1, jb1);
      } else {
        int pstep = n / p;
        for (int r = 0; r < p; ++r) {
          cx<T> s = t[0];
          for (int q = 1; q < p; ++q) s = cadd(s, cmul(t[q], w(((q * r) % p) * pstep, inv)));
          y[r] = s;
        }
      }
      for (int r = 0; r < p; ++r) out[k + r * m] = y[r];
    }
  }
  // in-place transform of n elements spaced `stride` apart
  void exec(cx<T>* x, i64 stride, bool inv) {
    std::vector<cx<T>> in(n);
    for (int k = 0; k < n; ++k) in[k] = x[(i64)k * stride];
    rec(in.data(), 1, buf.data(), n, 0, inv);
    for (int k = 0; k < n; ++k) x[(i64)k * stride] = buf[k];
  }
};

// 2-D transform of a column-major n1 x n2 complex array (FFTW plan_fft! over
// both dims; the inverse plan is scaled by 1/(n1*n2) in T, as inv(plan) does).
template <class T> struct FFT2 {
  int n1, n2;
  FFT1<T> f1, f2;
  FFT2(int a, int b) : n1(a), n2(b), f1(a), f2(b) {}
  void forward(cx<T>* x) {
    for (int j = 0; j < n2; ++j) f1.exec(x + (i64)j * n1, 1, false);
    for (int i = 0; i < n1; ++i) f2.exec(x + i, n1, false);
  }
  void inverse(cx<T>* x) {
    for (int j = 0; j < n2; ++j) f1.exec(x + (i64)j * n1, 1, true);
    for (int i = 0; i < n1; ++i) f2.exec(x + i, n1, true);
    T scale = T(1) / (T)((i64)n1 * n2);
    for (i64 k = 0; k < (i64)n1 * n2; ++k) { x[k].re *= scale; x[k].im *= scale; }
  }
};

// ---------------------------------------------------------------------------
// Pass parameters: field-for-field mirror of PIVParameters (src/types.jl:212-291).
struct Validator {
  int32_t kind;          // 0 peak_ratio, 1 correlation_moment, 2 velocity_magnitude, 3 uod
  int32_t neighborhood;  // uod
  double threshold;      // peak_ratio / moment / uod threshold
  double vmin, vmax;     // velocity magnitude
  double epsilon;        // uod
};
struct Pass {
  int32_t window[2], search[2], overlap[2];
  int32_t method;    // 0 cross, 1 phase
  int32_t padding;   // bool
  int32_t apod;      // 0 none, 1 gauss
  int32_t subpixel;  // 0 gauss3, 1 gauss9, 2 gauss2d, 3 none
  int32_t n_peaks;
  int32_t finder;    // 0 regionalmax, 1 exclusion
  int32_t uncertainty, uod_enable;
  double uod_threshold;
  int32_t uod_neighborhood;
  int32_t replace_outliers;
  double min_peak_ratio;
  int32_t max_iterations;
  int32_t keep_planes;
  double convergence_tol;
  int32_t n_validators;
  int32_t _pad;
  Validator validators[8];
};

// ---------------------------------------------------------------------------
// Statistics.median! / median (even n: middle(a,b) = a/2 + b/2; NaN -> NaN)
template <class T> static T median_inplace(T* v, int n) {
  for (int i = 0; i < n; ++i)
    if (std::isnan(v[i])) return std::numeric_limits<T>::quiet_NaN();
  int mid = (n + 1) / 2 - 1;  // 0-based index of div(1+n, 2)
  if (n & 1) {
    std::nth_element(v, v + mid, v + n);
    return v[mid];
  }
  std::nth_element(v, v + mid, v + n);
  T a = v[mid];
  T b = *std::min_element(v + mid + 1, v + n);
  return a / 2 + b / 2;
}

// ---------------------------------------------------------------------------
// src/correlators.jl:18-25  apodization_window
template <class T> static void apodization_window(int wr, int wc, int apod, T* out) {
  if (apod == 0) {
    for (int k = 0; k < wr * wc; ++k) out[k] = T(1);
    return;
  }
  double cr = (wr + 1) / 2.0, cc = (wc + 1) / 2.0, sr = wr / 4.0, sc = wc / 4.0;
  for (int j = 1; j <= wc; ++j)
    for (int i = 1; i <= wr; ++i)
      out[(i - 1) + (j - 1) * wr] =
          (T)std::exp(-((i - cr) * (i - cr) / (2 * sr * sr) + (j - cc) * (j - cc) / (2 * sc * sc)));
}

// src/correlators.jl:282-289  fftshift_abs!
template <class T> static void fftshift_abs(T* R, const cx<T>* C, int nr, int nc) {
  int sr = nr / 2, sc = nc / 2;
  for (int j = 0; j < nc; ++j)
    for (int i = 0; i < nr; ++i) R[((i + sr) % nr) + ((j + sc) % nc) * nr] = cabs_(C[i + j * nr]);
}

// src/correlators.jl:170-181  overlap_gain!
template <class T> static void overlap_gain(int wr, int wc, const T* apod, int nr, int nc, T* gain) {
  std::vector<cx<T>> C((size_t)nr * nc, cx<T>{0, 0});
  for (int j = 0; j < wc; ++j)
    for (int i = 0; i < wr; ++i) C[i + j * nr] = {apod[i + j * wr], 0};
  FFT2<T> f(nr, nc);
  f.forward(C.data());
  for (auto& z : C) z = {z.re * z.re + z.im * z.im, 0};  // abs2
  f.inverse(C.data());
  std::vector<T> weight((size_t)nr * nc);
  fftshift_abs(weight.data(), C.data(), nr, nc);
  T wmax = weight[0];
  for (T w : weight) wmax = std::max(wmax, w);
  for (size_t k = 0; k < weight.size(); ++k) gain[k] = weight[k] >= wmax / 2 ? wmax / weight[k] : T(0);
}

// Correlator state: src/correlators.jl:42-129
template <class T> struct Correlator {
  int wr, wc, sr, sc, nr, nc;
  int method, padding;
  std::vector<T> apod, gain, W, R;
  std::vector<cx<T>> C1, C2;
  FFT2<T> fft;
  Correlator(const Pass& p)
      : wr(p.window[0]), wc(p.window[1]), sr(p.search[0]), sc(p.search[1]),
        nr(p.padding ? 2 * p.search[0] : p.search[0]), nc(p.padding ? 2 * p.search[1] : p.search[1]),
        method(p.method), padding(p.padding), fft(nr, nc) {
    apod.resize((size_t)wr * wc);
    apodization_window(wr, wc, p.apod, apod.data());
    C1.assign((size_t)nr * nc, cx<T>{0, 0});
    C2.assign((size_t)nr * nc, cx<T>{0, 0});
    R.assign((size_t)nr * nc, T(0));
    if (padding && sr == wr && sc == wc) {
      gain.resize((size_t)nr * nc);
      overlap_gain(wr, wc, apod.data(), nr, nc, gain.data());
    }
    if (method == 1) {
      double fs = std::min(nr, nc) / 8.0;
      W.resize((size_t)nr * nc);
      for (int j = 0; j < nc; ++j)
        for (int i = 0; i < nr; ++i) {
          double fi = i < (nr + 1) / 2 ? i : i - nr;  // fftfreq(n, n)
          double fj = j < (nc + 1) / 2 ? j : j - nc;
          W[i + j * nr] = (T)std::exp(-(fi * fi + fj * fj) / (2 * fs * fs));
        }
    }
  }
};

// src/correlators.jl:188-263  load_windows!  (A, B, masks passed as
// column-major sub-views with leading dimension ld)
template <class T>
static void load_windows(Correlator<T>& c, const T* A, const T* B, i64 ld, const uint8_t* mA,
                         const uint8_t* mB, i64 ldm) {
  const int wr = c.wr, wc = c.wc, sr = c.sr, sc = c.sc, nr = c.nr;
  if (c.nr != wr || c.nc != wc || sr != wr || sc != wc) {
    std::fill(c.C1.begin(), c.C1.end(), cx<T>{0, 0});
    std::fill(c.C2.begin(), c.C2.end(), cx<T>{0, 0});
  }
  if (sr == wr && sc == wc) {
    if (!mA) {
      T sA = A[0], sB = B[0];  // sequential column-major fold
      for (int k = 1; k < wr * wc; ++k) {
        int i = k % wr, j = k / wr;
        sA += A[i + j * ld];
        sB += B[i + j * ld];
      }
      T meanA = sA / (T)(wr * wc), meanB = sB / (T)(wr * wc);
      for (int j = 0; j < wc; ++j)
        for (int i = 0; i < wr; ++i) {
          c.C1[i + j * nr] = {c.apod[i + j * wr] * (A[i + j * ld] - meanA), 0};
          c.C2[i + j * nr] = {c.apod[i + j * wr] * (B[i + j * ld] - meanB), 0};
        }
    } else {
      T sA = 0, sB = 0;
      int n = 0;
      for (int j = 0; j < wc; ++j)
        for (int i = 0; i < wr; ++i) {
          if (mA[i + j * ldm]) continue;
          sA += A[i + j * ld];
          sB += B[i + j * ld];
          ++n;
        }
      T meanA = n > 0 ? sA / (T)n : T(0), meanB = n > 0 ? sB / (T)n : T(0);
      for (int j = 0; j < wc; ++j)
        for (int i = 0; i < wr; ++i) {
          if (mA[i + j * ldm]) {
            c.C1[i + j * nr] = {0, 0};
            c.C2[i + j * nr] = {0, 0};
          } else {
            c.C1[i + j * nr] = {c.apod[i + j * wr] * (A[i + j * ld] - meanA), 0};
            c.C2[i + j * nr] = {c.apod[i + j * wr] * (B[i + j * ld] - meanB), 0};
          }
        }
    }
    return;
  }
  // Enlarged search area: A is the centred window at offset (off_r, off_c)
  // inside the search area; B is the full search area (no apodization).
  int off_r = (sr - wr) / 2, off_c = (sc - wc) / 2;
  const T* Aw = A;  // caller passes A already at the window origin
  T meanA, meanB;
  if (!mA) {
    T s = Aw[0];
    for (int k = 1; k < wr * wc; ++k) s += Aw[(k % wr) + (k / wr) * ld];
    meanA = s / (T)(wr * wc);
  } else {
    T s = 0;
    int n = 0;
    for (int j = 0; j < wc; ++j)
      for (int i = 0; i < wr; ++i)
        if (!mA[i + j * ldm]) { s += Aw[i + j * ld]; ++n; }
    meanA = n > 0 ? s / (T)n : T(0);
  }
  if (!mB) {
    T s = B[0];
    for (int k = 1; k < sr * sc; ++k) s += B[(k % sr) + (k / sr) * ld];
    meanB = s / (T)(sr * sc);
  } else {
    T s = 0;
    int n = 0;
    for (int j = 0; j < sc; ++j)
      for (int i = 0; i < sr; ++i)
        if (!mB[i + j * ldm]) { s += B[i + j * ld]; ++n; }
    meanB = n > 0 ? s / (T)n : T(0);
  }
  for (int j = 0; j < wc; ++j)
    for (int i = 0; i < wr; ++i)
      c.C1[(off_r + i) + (off_c + j) * nr] =
          (mA && mA[i + j * ldm]) ? cx<T>{0, 0} : cx<T>{c.apod[i + j * wr] * (Aw[i + j * ld] - meanA), 0};
  for (int j = 0; j < sc; ++j)
    for (int i = 0; i < sr; ++i)
      c.C2[i + j * nr] = (mB && mB[i + j * ldm]) ? cx<T>{0, 0} : cx<T>{B[i + j * ld] - meanB, 0};
}

// src/correlators.jl:326-341 correlation_plane! (+ spectrum! :266-279,
// restrict_search_lags! :347-355)
template <class T>
static const T* correlation_plane(Correlator<T>& c, const T* A, const T* B, i64 ld, const uint8_t* mA,
                                  const uint8_t* mB, i64 ldm) {
  load_windows(c, A, B, ld, mA, mB, ldm);
  c.fft.forward(c.C1.data());
  c.fft.forward(c.C2.data());
  const size_t P = (size_t)c.nr * c.nc;
  if (c.method == 0) {
    for (size_t k = 0; k < P; ++k) {
      cx<T> a = {c.C1[k].re, -c.C1[k].im};
      c.C1[k] = cmul(a, c.C2[k]);
    }
  } else {
    const T eps = std::numeric_limits<T>::epsilon();
    for (size_t k = 0; k < P; ++k) {
      cx<T> a = {c.C1[k].re, -c.C1[k].im};
      cx<T> s = cmul(a, c.C2[k]);
      T den = cabs_(s) + eps;
      T wk = c.W[k];
      c.C1[k] = {(wk * s.re) / den, (wk * s.im) / den};
    }
  }
  c.fft.inverse(c.C1.data());
  fftshift_abs(c.R.data(), c.C1.data(), c.nr, c.nc);
  if (!c.gain.empty())
    for (size_t k = 0; k < P; ++k) c.R[k] *= c.gain[k];
  if (c.sr != c.wr || c.sc != c.wc) {
    int mr = (c.sr - c.wr) / 2, mc = (c.sc - c.wc) / 2;
    int cr = c.nr / 2 + 1, cc = c.nc / 2 + 1;
    for (int j = 1; j <= c.nc; ++j)
      for (int i = 1; i <= c.nr; ++i)
        if (!(std::abs(i - cr) <= mr && std::abs(j - cc) <= mc)) c.R[(i - 1) + (j - 1) * c.nr] = 0;
  }
  return c.R.data();
}

// ---------------------------------------------------------------------------
// src/localmax.jl:3-19
template <class T> static bool is_local_maximum(const T* A, int nr, int nc, int r, int c) {
  T I0 = A[(r - 1) + (i64)(c - 1) * nr];
  if (std::isnan(I0)) return false;
  i64 lin0 = r + (i64)(c - 1) * nr;
  for (int jj = std::max(1, c - 1); jj <= std::min(nc, c + 1); ++jj)
    for (int ii = std::max(1, r - 1); ii <= std::min(nr, r + 1); ++ii) {
      if (ii == r && jj == c) continue;
      T In = A[(ii - 1) + (i64)(jj - 1) * nr];
      if (ii + (i64)(jj - 1) * nr < lin0) {
        if (In > I0) return false;
      } else {
        if (In >= I0) return false;
      }
    }
  return true;
}

// src/correlators.jl:390-421  (locs are 1-based (row, col) pairs)
template <class T>
static int find_peaks_exclusion(T* vals, int* locs, const T* R, int nr, int nc, int k, int excl) {
  int found = 0;
  for (int it = 0; it < k; ++it) {
    T best = -std::numeric_limits<T>::infinity();
    int bi = 0, bj = 0;
    for (int j = 1; j <= nc; ++j)
      for (int i = 1; i <= nr; ++i) {
        bool excluded = false;
        for (int p = 0; p < found; ++p)
          if (std::abs(i - locs[2 * p]) <= excl && std::abs(j - locs[2 * p + 1]) <= excl) {
            excluded = true;
            break;
          }
        if (excluded) continue;
        T v = R[(i - 1) + (i64)(j - 1) * nr];
        if (v > best) { best = v; bi = i; bj = j; }
      }
    if (bi == 0) break;
    if (found > 0 && best <= 0) break;
    vals[found] = best;
    locs[2 * found] = bi;
    locs[2 * found + 1] = bj;
    ++found;
  }
  return found;
}

// src/correlators.jl:426-454
template <class T> static int find_peaks_regionalmax(T* vals, int* locs, const T* R, int nr, int nc, int k) {
  int nfound = 0;
  for (int j = 1; j <= nc; ++j)
    for (int i = 1; i <= nr; ++i) {
      if (!is_local_maximum(R, nr, nc, i, j)) continue;
      T val = R[(i - 1) + (i64)(j - 1) * nr];
      if (!(nfound < k || val > vals[nfound - 1])) continue;
      int pos = nfound;
      while (pos >= 1 && val > vals[pos - 1]) --pos;
      int ins = pos + 1;
      if (ins > k) continue;
      if (nfound < k) ++nfound;
      for (int m = nfound; m >= ins + 1; --m) {
        vals[m - 1] = vals[m - 2];
        locs[2 * (m - 1)] = locs[2 * (m - 2)];
        locs[2 * (m - 1) + 1] = locs[2 * (m - 2) + 1];
      }
      vals[ins - 1] = val;
      locs[2 * (ins - 1)] = i;
      locs[2 * (ins - 1) + 1] = j;
    }
  if (nfound == 0) return 0;
  int found = 1;
  while (found < nfound && vals[found] > 0) ++found;
  return found;
}

template <class T>
static int find_peaks(T* vals, int* locs, const T* R, int nr, int nc, int k, int finder, int excl) {
  return finder == 1 ? find_peaks_exclusion(vals, locs, R, nr, nc, k, excl)
                     : find_peaks_regionalmax(vals, locs, R, nr, nc, k);
}

// src/correlators.jl:499-520
template <class T> static void gauss3(const T* R, int nr, int nc, int i, int j, T* out) {
  T di = 0, dj = 0;
  T I0 = R[(i - 1) + (i64)(j - 1) * nr];
  if (1 < i && i < nr) {
    T Im = R[(i - 2) + (i64)(j - 1) * nr], Ip = R[i + (i64)(j - 1) * nr];
    if (Im > 0 && I0 > 0 && Ip > 0) {
      T denom = std::log(Im) - T(2) * std::log(I0) + std::log(Ip);
      di = denom != 0 ? (std::log(Im) - std::log(Ip)) / (T(2) * denom) : T(0);
    }
  }
  if (1 < j && j < nc) {
    T Im = R[(i - 1) + (i64)(j - 2) * nr], Ip = R[(i - 1) + (i64)j * nr];
    if (Im > 0 && I0 > 0 && Ip > 0) {
      T denom = std::log(Im) - T(2) * std::log(I0) + std::log(Ip);
      dj = denom != 0 ? (std::log(Im) - std::log(Ip)) / (T(2) * denom) : T(0);
    }
  }
  out[0] = (T)i + di;
  out[1] = (T)j + dj;
}

// src/correlators.jl:534-564
template <class T> static void gauss9(const T* R, int nr, int nc, int pr, int pc, T* out) {
  if (!(1 < pr && pr < nr && 1 < pc && pc < nc)) return gauss3(R, nr, nc, pr, pc, out);
  T sL = 0, sxL = 0, syL = 0, sxxL = 0, syyL = 0, sxyL = 0;
  for (int dj = -1; dj <= 1; ++dj)
    for (int di = -1; di <= 1; ++di) {
      T val = R[(pr + di - 1) + (i64)(pc + dj - 1) * nr];
      if (!(val > 0)) return gauss3(R, nr, nc, pr, pc, out);
      T L = std::log(val);
      sL += L;
      sxL += (T)dj * L;
      syL += (T)di * L;
      sxxL += (T)(dj * dj) * L;
      syyL += (T)(di * di) * L;
      sxyL += (T)(di * dj) * L;
    }
  T a1 = sxL / 6, a2 = syL / 6, a3 = sxxL / 2 - sL / 3, a4 = sxyL / 4, a5 = syyL / 2 - sL / 3;
  T D = 4 * a3 * a5 - a4 * a4;
  if (!(a3 < 0 && D > 0)) return gauss3(R, nr, nc, pr, pc, out);
  T dx = (a4 * a2 - 2 * a5 * a1) / D;
  T dy = (a4 * a1 - 2 * a3 * a2) / D;
  if (!(std::abs(dx) <= 1 && std::abs(dy) <= 1)) return gauss3(R, nr, nc, pr, pc, out);
  out[0] = (T)pr + dy;
  out[1] = (T)pc + dx;
}

template <class T> static void refine_peak(const T* R, int nr, int nc, int pr, int pc, int method, T* out) {
  if (method == 1) return gauss9(R, nr, nc, pr, pc, out);
  if (method == 3) { out[0] = (T)pr; out[1] = (T)pc; return; }
  return gauss3(R, nr, nc, pr, pc, out);  // gauss2d is rejected before it gets here
}

// src/quality.jl:49-74 (neighborhood_size = 3). Julia: (c - pc)^2 is in the
// precision of pc, then widened by the Float64 weight.
template <class T> static double correlation_moment(const T* R, int nr, int nc, T pr, T pc) {
  if (!(std::isfinite(pr) && std::isfinite(pc))) return NAN;
  int r0 = (int)std::nearbyint(pr), c0 = (int)std::nearbyint(pc);  // round: ties to even
  int rlo = std::max(1, r0 - 1), rhi = std::min(nr, r0 + 1);
  int clo = std::max(1, c0 - 1), chi = std::min(nc, c0 + 1);
  if (rlo > rhi || clo > chi) return NAN;
  double sumC = 0, sdx = 0, sdy = 0;
  for (int c = clo; c <= chi; ++c)
    for (int r = rlo; r <= rhi; ++r) {
      double w = std::max((double)R[(r - 1) + (i64)(c - 1) * nr], 0.0);
      T dx = (T)c - pc, dy = (T)r - pr;
      sumC += w;
      sdx += (double)(dx * dx) * w;
      sdy += (double)(dy * dy) * w;
    }
  if (sumC < 1e-9) return NAN;
  return std::sqrt((sdx + sdy) / sumC);
}

// src/quality.jl:11-36
template <class T> static T peak_ratio(const T* R, int nr, int nc, int pr, int pc, int excl, int finder) {
  T P1 = R[(pr - 1) + (i64)(pc - 1) * nr];
  T P2 = -std::numeric_limits<T>::infinity();
  for (int j = 1; j <= nc; ++j)
    for (int i = 1; i <= nr; ++i) {
      if (finder == 1) {
        if (std::abs(i - pr) <= excl && std::abs(j - pc) <= excl) continue;
      } else {
        if (i == pr && j == pc) continue;
        if (!is_local_maximum(R, nr, nc, i, j)) continue;
      }
      T v = R[(i - 1) + (i64)(j - 1) * nr];
      if (v > P2) P2 = v;
    }
  if (!(P2 > 0)) return P1 > 0 ? std::numeric_limits<T>::infinity() : std::numeric_limits<T>::quiet_NaN();
  return P1 / P2;
}

// Packed per-window result, the layout of src/ka_backend.jl:497-506:
// [du, dv, ratio, moment, found, alt du (K-1), alt dv (K-1)].
// analyze_plane! src/correlators.jl:459-468 + alternatives src/pipeline.jl:1009-1017
template <class T>
static void analyze_plane(const T* R, int nr, int nc, int npeaks, int finder, int subpixel, T* out, int* locs_out) {
  const int K = std::max(npeaks, 2);
  T vals[64];
  int locs[128];
  int found = find_peaks(vals, locs, R, nr, nc, K, finder, 2);
  const T NaN = std::numeric_limits<T>::quiet_NaN();
  for (int m = 0; m < 5 + 2 * (K - 1); ++m) out[m] = NaN;
  out[4] = (T)found;
  if (locs_out)
    for (int m = 0; m < 2 * K; ++m) locs_out[m] = m < 2 * found ? locs[m] : 0;
  if (found == 0) return;
  T ref[2];
  refine_peak(R, nr, nc, locs[0], locs[1], subpixel, ref);
  int cr = nr / 2 + 1, cc = nc / 2 + 1;
  out[0] = ref[1] - (T)cc;
  out[1] = ref[0] - (T)cr;
  out[2] = found >= 2 ? vals[0] / vals[1] : (vals[0] > 0 ? std::numeric_limits<T>::infinity() : NaN);
  out[3] = (T)correlation_moment(R, nr, nc, ref[0], ref[1]);
  for (int m = 2; m <= std::min(found, npeaks); ++m) {
    T a[2];
    gauss3(R, nr, nc, locs[2 * (m - 1)], locs[2 * (m - 1) + 1], a);
    out[5 + (m - 2)] = a[1] - (T)cc;
    out[5 + (K - 1) + (m - 2)] = a[0] - (T)cr;
  }
}

// ---------------------------------------------------------------------------
// Uncertainty: src/uncertainty.jl
static int UQ_OFF[40][2];
static int UQ_RING_START[5];
static bool uq_init_done = false;
static void uq_init() {
  if (uq_init_done) return;
  // offsets (dr, dc): dc in 0:4, dr in (dc==0 ? 1:4 : -4:4), stably sorted by ring
  int tmp[40][2], n = 0;
  for (int dc = 0; dc <= 4; ++dc)
    for (int dr = (dc == 0 ? 1 : -4); dr <= 4; ++dr) { tmp[n][0] = dr; tmp[n][1] = dc; ++n; }
  int k = 0;
  for (int ring = 1; ring <= 4; ++ring) {
    UQ_RING_START[ring - 1] = k;
    for (int q = 0; q < 40; ++q)
      if (std::max(std::abs(tmp[q][0]), std::abs(tmp[q][1])) == ring) {
        UQ_OFF[k][0] = tmp[q][0];
        UQ_OFF[k][1] = tmp[q][1];
        ++k;
      }
  }
  UQ_RING_START[4] = 40;
  uq_init_done = true;
}

// uq_component! src/uncertainty.jl:104-151. A, B accessed as A(r, c) through
// (stride_r, stride_c) so the v component can pass the transposed view.
template <class T>
static void uq_component(double* s, const T* A, const T* B, int nr, int ncol, i64 str, i64 stc, std::vector<T>& dC,
                         std::vector<T>& dCs) {
  const int m = ncol - 1;
  auto a = [&](const T* X, int r, int c) { return X[(i64)r * str + (i64)c * stc]; };
  double C0 = 0, Cp = 0, Cm = 0;
  dC.assign((size_t)nr * std::max(m, 1), T(0));
  dCs.assign((size_t)nr * std::max(m, 1), T(0));
  for (int c = 0; c < m; ++c)
    for (int r = 0; r < nr; ++r) {
      T a0 = a(A, r, c), a1 = a(A, r, c + 1), b0 = a(B, r, c), b1 = a(B, r, c + 1);
      C0 += (double)(a0 * b0);
      Cp += (double)(a0 * b1);
      Cm += (double)(a1 * b0);
      dC[r + (i64)c * nr] = a0 * b1 - a1 * b0;
    }
  s[0] += C0;
  s[1] += Cp;
  s[2] += Cm;
  const T quarter = T(1) / T(4);
  for (int c = 0; c < m; ++c)
    for (int r = 0; r < nr; ++r) {
      int cl = std::max(c - 1, 0), cr = std::min(c + 1, m - 1);
      dCs[r + (i64)c * nr] = quarter * (dC[r + (i64)cl * nr] + T(2) * dC[r + (i64)c * nr] + dC[r + (i64)cr * nr]);
    }
  double mu = 0;
  for (int c = 0; c < m; ++c)
    for (int r = 0; r < nr; ++r) mu += (double)dCs[r + (i64)c * nr];
  mu /= (double)(nr * m);
  double S00 = 0;
  for (int c = 0; c < m; ++c)
    for (int r = 0; r < nr; ++r) {
      double d = (double)dCs[r + (i64)c * nr] - mu;
      S00 += d * d;
    }
  s[3] += S00;
  for (int k = 0; k < 40; ++k) {
    int dr = UQ_OFF[k][0], dc = UQ_OFF[k][1];
    double Sk = 0;
    // 1-based ranges c in max(1,1-dc):min(m,m-dc), r in max(1,1-dr):min(nr,nr-dr)
    for (int c = std::max(1, 1 - dc); c <= std::min(m, m - dc); ++c)
      for (int r = std::max(1, 1 - dr); r <= std::min(nr, nr - dr); ++r)
        Sk += ((double)dCs[(r - 1) + (i64)(c - 1) * nr] - mu) *
              ((double)dCs[(r - 1 + dr) + (i64)(c - 1 + dc) * nr] - mu);
    s[4 + k] += Sk;
  }
}

// load_uncertainty_windows! :51-83 + accumulate_uncertainty! :87-96
template <class T>
static void uq_window_stats(double* stats /*2 x 44, row-major per component*/, const T* A, const T* B, i64 ld,
                            const uint8_t* m, i64 ldm, int wr, int wc, const T* apod) {
  uq_init();
  std::vector<T> wA((size_t)wr * wc), wB((size_t)wr * wc), dC, dCs;
  T meanA, meanB;
  if (!m) {
    T sA = A[0], sB = B[0];
    for (int k = 1; k < wr * wc; ++k) {
      sA += A[(k % wr) + (i64)(k / wr) * ld];
      sB += B[(k % wr) + (i64)(k / wr) * ld];
    }
    meanA = sA / (T)(wr * wc);
    meanB = sB / (T)(wr * wc);
  } else {
    T sA = 0, sB = 0;
    int n = 0;
    for (int j = 0; j < wc; ++j)
      for (int i = 0; i < wr; ++i) {
        if (m[i + j * ldm]) continue;
        sA += A[i + j * ld];
        sB += B[i + j * ld];
        ++n;
      }
    meanA = n > 0 ? sA / (T)n : T(0);
    meanB = n > 0 ? sB / (T)n : T(0);
  }
  for (int j = 0; j < wc; ++j)
    for (int i = 0; i < wr; ++i) {
      if (m && m[i + j * ldm]) {
        wA[i + j * wr] = 0;
        wB[i + j * wr] = 0;
      } else {
        wA[i + j * wr] = apod[i + j * wr] * (A[i + j * ld] - meanA);
        wB[i + j * wr] = apod[i + j * wr] * (B[i + j * ld] - meanB);
      }
    }
  uq_component(stats, wA.data(), wB.data(), wr, wc, 1, wr, dC, dCs);        // u: shift along columns
  uq_component(stats + 44, wA.data(), wB.data(), wc, wr, wr, 1, dC, dCs);   // v: transposed view
}

// finalize_uncertainty :162-179
template <class T> static T finalize_uq(const double* s) {
  uq_init();
  double C0 = s[0], Cp = s[1], Cm = s[2], S00 = s[3];
  double s2 = S00;
  for (int ring = 0; ring < 4; ++ring) {
    double mx = -INFINITY;
    for (int k = UQ_RING_START[ring]; k < UQ_RING_START[ring + 1]; ++k) mx = std::max(mx, s[4 + k]);
    if (mx < 0.05 * S00) break;
    for (int k = UQ_RING_START[ring]; k < UQ_RING_START[ring + 1]; ++k) s2 += 2 * s[4 + k];
  }
  double sdc = std::sqrt(std::max(s2, 0.0));
  double Cpm = (Cp + Cm) / 2, lo = Cpm - sdc / 2, hi = Cpm + sdc / 2;
  if (!(C0 > 0 && lo > 0)) return std::numeric_limits<T>::quiet_NaN();
  double denom = 2 * std::log(C0) - std::log(hi) - std::log(lo);
  if (!(denom > 0)) return std::numeric_limits<T>::quiet_NaN();
  return (T)((std::log(hi) - std::log(lo)) / (2 * denom));
}

// ---------------------------------------------------------------------------
// Vector-grid operations (src/quality.jl). Grids are column-major (ny, nx).

// universal_outlier_detection :244-293. Residuals in T; the normalisation
// widens to Float64 because epsilon is a Float64.
template <class T>
static void uod(const T* u, const T* v, int nr, int nc, double thr, int nb, double eps, const uint8_t* exclude,
                uint8_t* out) {
  std::vector<T> nu, nv, ru, rv;
  for (int c = 0; c < nc; ++c)
    for (int r = 0; r < nr; ++r) {
      out[r + (i64)c * nr] = 0;
      if (exclude && exclude[r + (i64)c * nr]) continue;
      nu.clear();
      nv.clear();
      for (int c2 = std::max(0, c - nb); c2 <= std::min(nc - 1, c + nb); ++c2)
        for (int r2 = std::max(0, r - nb); r2 <= std::min(nr - 1, r + nb); ++r2) {
          if (r2 == r && c2 == c) continue;
          if (exclude && exclude[r2 + (i64)c2 * nr]) continue;
          nu.push_back(u[r2 + (i64)c2 * nr]);
          nv.push_back(v[r2 + (i64)c2 * nr]);
        }
      int n = (int)nu.size();
      if (n == 0) continue;
      std::vector<T> su(nu), sv(nv);
      T um = median_inplace(su.data(), n), vm = median_inplace(sv.data(), n);
      ru.resize(n);
      rv.resize(n);
      for (int i = 0; i < n; ++i) {
        ru[i] = std::abs(nu[i] - um);
        rv[i] = std::abs(nv[i] - vm);
      }
      double un = (double)std::abs(u[r + (i64)c * nr] - um) / ((double)median_inplace(ru.data(), n) + eps);
      double vn = (double)std::abs(v[r + (i64)c * nr] - vm) / ((double)median_inplace(rv.data(), n) + eps);
      if (un > thr || vn > thr) out[r + (i64)c * nr] = 1;
    }
}

// replace_vectors! :85-114 (Float64 neighbour buffers, T store)
template <class T> static void replace_vectors(T* u, T* v, int nr, int nc, const uint8_t* invalid) {
  bool anyinv = false;
  for (i64 k = 0; k < (i64)nr * nc; ++k) anyinv |= invalid[k] != 0;
  if (!anyinv) return;
  std::vector<T> uref(u, u + (i64)nr * nc), vref(v, v + (i64)nr * nc);
  std::vector<double> bu, bv;
  int maxr = std::max(nr, nc) - 1;
  for (int c = 0; c < nc; ++c)
    for (int r = 0; r < nr; ++r) {
      if (!invalid[r + (i64)c * nr]) continue;
      for (int rad = 1; rad <= maxr; ++rad) {
        bu.clear();
        bv.clear();
        for (int c2 = std::max(0, c - rad); c2 <= std::min(nc - 1, c + rad); ++c2)
          for (int r2 = std::max(0, r - rad); r2 <= std::min(nr - 1, r + rad); ++r2) {
            if (invalid[r2 + (i64)c2 * nr]) continue;
            bu.push_back((double)uref[r2 + (i64)c2 * nr]);
            bv.push_back((double)vref[r2 + (i64)c2 * nr]);
          }
        if (bu.size() >= 3) {
          u[r + (i64)c * nr] = (T)median_inplace(bu.data(), (int)bu.size());
          v[r + (i64)c * nr] = (T)median_inplace(bv.data(), (int)bv.size());
          break;
        }
      }
    }
}

// smooth_field :123-136
template <class T> static void smooth_field(const T* f, int nr, int nc, T* out) {
  const T q = T(1) / T(4);
  std::vector<T> tmp((size_t)nr * nc);
  for (int c = 0; c < nc; ++c)
    for (int r = 0; r < nr; ++r)
      tmp[r + (i64)c * nr] =
          q * (f[r + (i64)std::max(c - 1, 0) * nr] + T(2) * f[r + (i64)c * nr] + f[r + (i64)std::min(c + 1, nc - 1) * nr]);
  for (int c = 0; c < nc; ++c)
    for (int r = 0; r < nr; ++r)
      out[r + (i64)c * nr] = q * (tmp[std::max(r - 1, 0) + (i64)c * nr] + T(2) * tmp[r + (i64)c * nr] +
                                  tmp[std::min(r + 1, nr - 1) + (i64)c * nr]);
}

// substitute_alternatives! :307-351. alt arrays are (nr, nc, nalt) column-major.
template <class T>
static int substitute(T* u, T* v, uint8_t* outl, const uint8_t* mask, const T* au_, const T* av_, int nalt, int nr,
                      int nc, int er, double thr) {
  bool any = false;
  for (i64 k = 0; k < (i64)nr * nc; ++k) any |= outl[k] != 0;
  if (!any) return 0;
  std::vector<T> uref(u, u + (i64)nr * nc), vref(v, v + (i64)nr * nc);
  std::vector<uint8_t> valid((size_t)nr * nc);
  for (i64 k = 0; k < (i64)nr * nc; ++k) valid[k] = !(outl[k] || (mask && mask[k]));
  std::vector<double> bu, bv;
  int nsub = 0;
  for (int c = 0; c < nc; ++c)
    for (int r = 0; r < nr; ++r) {
      i64 id = r + (i64)c * nr;
      if (!(outl[id] && !(mask && mask[id]))) continue;
      bu.clear();
      bv.clear();
      for (int c2 = std::max(0, c - er); c2 <= std::min(nc - 1, c + er); ++c2)
        for (int r2 = std::max(0, r - er); r2 <= std::min(nr - 1, r + er); ++r2) {
          if (r2 == r && c2 == c) continue;
          if (!valid[r2 + (i64)c2 * nr]) continue;
          bu.push_back((double)uref[r2 + (i64)c2 * nr]);
          bv.push_back((double)vref[r2 + (i64)c2 * nr]);
        }
      if (bu.size() < 3) continue;
      std::vector<double> tu(bu), tv(bv);
      double mu = median_inplace(tu.data(), (int)tu.size()), mv = median_inplace(tv.data(), (int)tv.size());
      for (auto& x : bu) x = std::abs(x - mu);
      for (auto& x : bv) x = std::abs(x - mv);
      double madu = median_inplace(bu.data(), (int)bu.size()), madv = median_inplace(bv.data(), (int)bv.size());
      for (int m = 0; m < nalt; ++m) {
        T au = au_[id + (i64)m * nr * nc], av = av_[id + (i64)m * nr * nc];
        if (!(std::isfinite(au) && std::isfinite(av))) break;
        if (std::abs((double)au - mu) / (madu + 0.1) <= thr && std::abs((double)av - mv) / (madv + 0.1) <= thr) {
          u[id] = au;
          v[id] = av;
          outl[id] = 0;
          ++nsub;
          break;
        }
      }
    }
  return nsub;
}

// validate_and_replace! src/pipeline.jl:617-645 (+ apply_validator!
// src/quality.jl:466-503)
template <class T>
static void validate_and_replace(T* u, T* v, const T* ratio, const T* moment, uint8_t* outl, const uint8_t* mask,
                                 int nr, int nc, const Pass& p, bool force_replace, const T* alt_u, const T* alt_v,
                                 int nalt) {
  const i64 P = (i64)nr * nc;
  bool anymask = false;
  if (mask)
    for (i64 k = 0; k < P; ++k) anymask |= mask[k] != 0;
  std::vector<uint8_t> tmp(P);
  if (p.uod_enable) {
    uod(u, v, nr, nc, p.uod_threshold, p.uod_neighborhood, 0.1, anymask ? mask : nullptr, tmp.data());
    for (i64 k = 0; k < P; ++k) outl[k] |= tmp[k];
  }
  if (p.min_peak_ratio > 1)
    for (i64 k = 0; k < P; ++k) outl[k] |= !((double)ratio[k] >= p.min_peak_ratio);
  for (int q = 0; q < p.n_validators; ++q) {
    const Validator& vd = p.validators[q];
    if (vd.kind == 0) {
      for (i64 k = 0; k < P; ++k) outl[k] |= !((double)ratio[k] >= vd.threshold);
    } else if (vd.kind == 1) {
      for (i64 k = 0; k < P; ++k) outl[k] |= !((double)moment[k] <= vd.threshold);
    } else if (vd.kind == 2) {
      for (i64 k = 0; k < P; ++k) {
        T mag = std::hypot(u[k], v[k]);
        if (!(vd.vmin <= (double)mag && (double)mag <= vd.vmax)) outl[k] = 1;
      }
    } else if (vd.kind == 3) {
      uod(u, v, nr, nc, vd.threshold, vd.neighborhood, vd.epsilon, anymask ? mask : nullptr, tmp.data());
      for (i64 k = 0; k < P; ++k) outl[k] |= tmp[k];
    }
  }
  if (mask)
    for (i64 k = 0; k < P; ++k) outl[k] &= !mask[k];
  if (alt_u) substitute(u, v, outl, mask, alt_u, alt_v, nalt, nr, nc, p.uod_neighborhood, p.uod_threshold);
  if (force_replace || p.replace_outliers) {
    std::vector<uint8_t> inv(P);
    bool any = false;
    for (i64 k = 0; k < P; ++k) {
      inv[k] = outl[k] || (mask && mask[k]);
      any |= inv[k] != 0;
    }
    if (any) {
      replace_vectors(u, v, nr, nc, inv.data());
      if (mask)
        for (i64 k = 0; k < P; ++k)
          if (mask[k]) u[k] = v[k] = std::numeric_limits<T>::quiet_NaN();
    }
  }
}

// field_change src/pipeline.jl:849-866 with quantile!(buf, 0.95) (type 7).
template <class T>
static T field_change(const T* u, const T* v, const T* pu, const T* pv, const uint8_t* mask, i64 P) {
  std::vector<T> buf;
  for (i64 i = 0; i < P; ++i) {
    if (mask && mask[i]) continue;
    T du = std::abs(u[i] - pu[i]), dv = std::abs(v[i] - pv[i]);
    if (std::isnan(du) || std::isnan(dv)) {
      if (std::isnan(u[i]) == std::isnan(pu[i]) && std::isnan(v[i]) == std::isnan(pv[i])) continue;
      buf.push_back(std::numeric_limits<T>::infinity());
      continue;
    }
    buf.push_back(std::max(du, dv));
  }
  if (buf.empty()) return T(0);
  const double p = 0.95;
  i64 n = (i64)buf.size();
  double aleph = std::fma((double)n, p, 1.0 - p);
  i64 j = std::min(std::max((i64)std::trunc(aleph), (i64)1), std::max(n - 1, (i64)1));
  double g = std::min(std::max(aleph - (double)j, 0.0), 1.0);
  std::sort(buf.begin(), buf.end());
  T a, b;
  if (n == 1) a = b = buf[0];
  else { a = buf[j - 1]; b = buf[j]; }
  double q;
  if (std::isfinite(a) && std::isfinite(b)) q = (double)a + g * (double)(b - a);
  else q = (1 - g) * (double)a + g * (double)b;
  return (T)q;
}

// ---------------------------------------------------------------------------
// Deformation: Interpolations.jl BSpline(Cubic(Line(OnGrid()))) restated.
// Padded (nr+2) x (nc+2) coefficient array; logical index k at parent k+1.
template <class T> static void bspline_line(T* x, i64 n, i64 stride) {
  // Solve, on the padded index set 1..n (n = m + 2):
  //   row 1: c1 - 2c2 + c3 = 0;   rows 2..n-1: (c_{i-1} + 4c_i + c_{i+1})/6 = b_i;
  //   row n: c_{n-2} - 2c_{n-1} + c_n = 0
  // with b_1 = b_n = 0 (zero padding). Eliminating the boundary rows gives
  // c2 = b2, c_{n-1} = b_{n-1}, a tridiagonal [1 4 1]/6 interior system, and
  // c1 = 2c2 - c3, cn = 2c_{n-1} - c_{n-2}. The interior system is solved in
  // T over the whole line by one forward and one backward Thomas sweep, with
  // elimination factors inv_k = 1/den_k and cp_k = inv_k/6.
  auto X = [&](i64 i) -> T& { return x[(i - 1) * stride]; };
  if (n < 4) return;
  const T sixth = T(1) / T(6), four6 = T(4) / T(6);
  i64 lo = 3, hi = n - 2;  // unknown interior rows
  T c2 = X(2), cn1 = X(n - 1);
  if (hi >= lo) {
    const i64 m = hi - lo + 1;
    std::vector<T> cp(m), inv(m), dp(m);
    for (i64 k = 0; k < m; ++k) {
      T den = k == 0 ? four6 : four6 - sixth * cp[k - 1];
      inv[k] = T(1) / den;
      cp[k] = sixth * inv[k];
    }
    auto rhs = [&](i64 k) {
      T r = X(lo + k);
      if (k == 0) r -= sixth * c2;
      if (k == m - 1) r -= sixth * cn1;
      return r;
    };
    T d = 0;
    for (i64 k = 0; k < m; ++k) {  // forward sweep
      d = k == 0 ? rhs(k) * inv[0] : (rhs(k) - sixth * d) * inv[k];
      dp[k] = d;
    }
    T xv = 0;
    for (i64 k = m - 1; k >= 0; --k) {  // backward sweep
      xv = k == m - 1 ? dp[k] : dp[k] - cp[k] * xv;
      X(lo + k) = xv;
    }
  }
  X(2) = c2;
  X(n - 1) = cn1;
  X(1) = T(2) * X(2) - X(3);
  X(n) = T(2) * X(n - 1) - X(n - 2);
}

template <class T> static void prefilter(const T* img, i64 nr, i64 nc, T* coef) {
  const i64 ld = nr + 2;
  std::fill(coef, coef + ld * (nc + 2), T(0));
  for (i64 j = 0; j < nc; ++j)
    for (i64 i = 0; i < nr; ++i) coef[(i + 1) + (j + 1) * ld] = img[i + j * nr];
  for (i64 j = 0; j < nc + 2; ++j) bspline_line(coef + j * ld, ld, 1);  // dim 1
  for (i64 i = 0; i < nr + 2; ++i) bspline_line(coef + i, nc + 2, ld);  // dim 2
}

// cubic B-spline weights (Interpolations value_weights for Cubic)
template <class T> static inline void cubw(T d, T* w) {
  T x3 = d * d * d, c = T(1) - d, c3 = c * c * c;
  w[0] = c3 / T(6);
  w[1] = T(2) / T(3) - d * d + x3 / T(2);
  w[2] = T(2) / T(3) - c * c + c3 / T(2);
  w[3] = x3 / T(6);
}

// zero-extrapolated cubic B-spline sample at 1-based (yy, xx)
template <class T> static T bspline_eval(const T* C, i64 nr, i64 nc, T yy, T xx) {
  if (yy < 1 || yy > (T)nr || xx < 1 || xx > (T)nc) return T(0);
  i64 iy = (i64)std::floor(yy);
  if (iy > nr - 1) iy = nr - 1;
  i64 ix = (i64)std::floor(xx);
  if (ix > nc - 1) ix = nc - 1;
  T wy[4], wx[4];
  cubw(yy - (T)iy, wy);
  cubw(xx - (T)ix, wx);
  const i64 ld = nr + 2;
  T s = 0;
  for (int a = 0; a < 4; ++a) {
    T t = 0;
    for (int b = 0; b < 4; ++b) t += wx[b] * C[(iy - 1 + a) + (ix - 1 + b) * ld];
    s += wy[a] * t;
  }
  return s;
}

// Gridded(Linear()) + Flat() along one axis of uniformly spaced knots
// q0 + k*step (k = 0..n-1): returns base index and fractional weight.
template <class T> static inline void lin_axis(T q, T q0, T step, int n, int& i, T& d) {
  if (n == 1) { i = 0; d = 0; return; }
  T last = q0 + (T)(n - 1) * step;
  if (q <= q0) { i = 0; d = 0; return; }
  if (q >= last) { i = n - 2; d = 1; return; }
  i = (int)std::floor((q - q0) / step);
  if (i > n - 2) i = n - 2;
  T k0 = q0 + (T)i * step, k1 = q0 + (T)(i + 1) * step;
  d = (q - k0) / (k1 - k0);
}

template <class T>
static T bilinear(const T* f, int gny, int gnx, T y0, T ysp, T x0, T xsp, T qy, T qx) {
  int iy, ix;
  T dy, dx;
  lin_axis(qy, y0, ysp, gny, iy, dy);
  lin_axis(qx, x0, xsp, gnx, ix, dx);
  int iy2 = gny == 1 ? iy : iy + 1, ix2 = gnx == 1 ? ix : ix + 1;
  T f00 = f[iy + (i64)ix * gny], f01 = f[iy + (i64)ix2 * gny], f10 = f[iy2 + (i64)ix * gny],
    f11 = f[iy2 + (i64)ix2 * gny];
  T a = (T(1) - dx) * f00 + dx * f01;
  T b = (T(1) - dx) * f10 + dx * f11;
  return (T(1) - dy) * a + dy * b;
}

struct Predictor {
  int gny = 0, gnx = 0;
  double y0 = 0, ysp = 1, x0 = 0, xsp = 1;
};

template <class T>
static void deform_columns(const T* CA, const T* CB, i64 nr, i64 nc, const T* pu, const T* pv, const Predictor& g,
                           T* wA, T* wB, i64 c0, i64 c1) {
  const T y0 = (T)g.y0, ysp = (T)g.ysp, x0 = (T)g.x0, xsp = (T)g.xsp;
  for (i64 c = c0; c < c1; ++c)
    for (i64 r = 0; r < nr; ++r) {
      T R = (T)(r + 1), Cc = (T)(c + 1);
      T du2 = bilinear(pu, g.gny, g.gnx, y0, ysp, x0, xsp, R, Cc) / T(2);
      T dv2 = bilinear(pv, g.gny, g.gnx, y0, ysp, x0, xsp, R, Cc) / T(2);
      wA[r + c * nr] = bspline_eval(CA, nr, nc, R - dv2, Cc - du2);
      wB[r + c * nr] = bspline_eval(CB, nr, nc, R + dv2, Cc + du2);
    }
}

// ---------------------------------------------------------------------------
// Differentiable correlation loss (no counterpart in the reference; the
// deformation it differentiates is deform_columns! above):
//   L(P) = - sum over windows j of NCC0_j,
//   NCC0_j = sum (a - abar)(b - bbar) / sqrt(sum (a - abar)^2 sum (b - bbar)^2)
// over the W x W pixels of window j of the pair deformed by the predictor
// P = (u, v) on a uniform node grid (bilinear, flat outside). Its gradient
// follows the chain: dL/da_i, dL/db_i of the normalised correlation; the
// sampling derivatives of the cubic B-spline at -+ (u, v)/2; the transpose of
// the bilinear predictor interpolation.

// derivative of the cubic B-spline weights with respect to the offset d
template <class T> static inline void cubw_d(T d, T* w) {
  T c = T(1) - d;
  w[0] = -c * c / T(2);
  w[1] = -T(2) * d + T(3) * d * d / T(2);
  w[2] = T(2) * c - T(3) * c * c / T(2);
  w[3] = d * d / T(2);
}

// value and gradient (d/dy, d/dx) of the zero-extrapolated B-spline sample
template <class T> static T bspline_eval_grad(const T* C, i64 nr, i64 nc, T yy, T xx, T& gy, T& gx) {
  gy = gx = T(0);
  if (yy < 1 || yy > (T)nr || xx < 1 || xx > (T)nc) return T(0);
  i64 iy = (i64)std::floor(yy);
  if (iy > nr - 1) iy = nr - 1;
  i64 ix = (i64)std::floor(xx);
  if (ix > nc - 1) ix = nc - 1;
  T wy[4], wx[4], dy[4], dx[4];
  cubw(yy - (T)iy, wy);
  cubw(xx - (T)ix, wx);
  cubw_d(yy - (T)iy, dy);
  cubw_d(xx - (T)ix, dx);
  const i64 ld = nr + 2;
  T s = 0, sy = 0, sx = 0;
  for (int a = 0; a < 4; ++a) {
    T t = 0, tx = 0;
    for (int b = 0; b < 4; ++b) {
      const T c = C[(iy - 1 + a) + (ix - 1 + b) * ld];
      t += wx[b] * c;
      tx += dx[b] * c;
    }
    s += wy[a] * t;
    sy += dy[a] * t;
    sx += wy[a] * tx;
  }
  gy = sy;
  gx = sx;
  return s;
}

// bilinear weights of the four nodes a query touches (flat outside)
template <class T> struct BilinW {
  int iy, ix, iy2, ix2;
  T w00, w01, w10, w11;
};
template <class T>
static BilinW<T> bilinear_w(int gny, int gnx, T y0, T ysp, T x0, T xsp, T qy, T qx) {
  BilinW<T> b;
  T dy, dx;
  lin_axis(qy, y0, ysp, gny, b.iy, dy);
  lin_axis(qx, x0, xsp, gnx, b.ix, dx);
  b.iy2 = gny == 1 ? b.iy : b.iy + 1;
  b.ix2 = gnx == 1 ? b.ix : b.ix + 1;
  b.w00 = (T(1) - dy) * (T(1) - dx);
  b.w01 = (T(1) - dy) * dx;
  b.w10 = dy * (T(1) - dx);
  b.w11 = dy * dx;
  return b;
}

// Loss over the windows with 0-based origins wins[2j], wins[2j+1]; the
// gradient (2 planes of gny x gnx: u then v) is accumulated when grad != 0.
template <class T>
static double ncc_loss_grad(const T* CA, const T* CB, i64 nr, i64 nc, const T* P, int gny, int gnx, T y0, T ysp, T x0,
                            T xsp, int W, const int32_t* wins, i64 nwin, T* grad) {
  const i64 G = (i64)gny * gnx;
  const T* pu = P;
  const T* pv = P + G;
  const int n = W * W;
  std::vector<T> a(n), b(n), ay(n), ax(n), by(n), bx(n);
  std::vector<BilinW<T>> bw(n);
  double L = 0;
  for (i64 j = 0; j < nwin; ++j) {
    const i64 rs = wins[2 * j], cs = wins[2 * j + 1];
    for (int q = 0; q < W; ++q)
      for (int p = 0; p < W; ++p) {
        const int k = p + q * W;
        const T R = (T)(rs + p + 1), Cc = (T)(cs + q + 1);
        const T u2 = bilinear(pu, gny, gnx, y0, ysp, x0, xsp, R, Cc) / T(2);
        const T v2 = bilinear(pv, gny, gnx, y0, ysp, x0, xsp, R, Cc) / T(2);
        a[k] = bspline_eval_grad(CA, nr, nc, R - v2, Cc - u2, ay[k], ax[k]);
        b[k] = bspline_eval_grad(CB, nr, nc, R + v2, Cc + u2, by[k], bx[k]);
        bw[k] = bilinear_w(gny, gnx, y0, ysp, x0, xsp, R, Cc);
      }
    T ma = 0, mb = 0;
    for (int k = 0; k < n; ++k) {
      ma += a[k];
      mb += b[k];
    }
    ma /= (T)n;
    mb /= (T)n;
    T saa = 0, sbb = 0, sab = 0;
    for (int k = 0; k < n; ++k) {
      const T da = a[k] - ma, db = b[k] - mb;
      saa += da * da;
      sbb += db * db;
      sab += da * db;
    }
    if (!(saa > 0 && sbb > 0)) continue;  // a flat window contributes nothing
    const T inv = T(1) / std::sqrt(saa * sbb), ncc = sab * inv;
    L -= (double)ncc;
    if (!grad) continue;
    const T ca = ncc / saa, cb = ncc / sbb;
    for (int k = 0; k < n; ++k) {
      const T da = a[k] - ma, db = b[k] - mb;
      const T ga = -db * inv + ca * da;  // dL/da_k
      const T gb = -da * inv + cb * db;  // dL/db_k
      const T gu = ga * (-ax[k] / T(2)) + gb * (bx[k] / T(2));
      const T gv = ga * (-ay[k] / T(2)) + gb * (by[k] / T(2));
      const BilinW<T>& w = bw[k];
      T* gu_ = grad;
      T* gv_ = grad + G;
      gu_[w.iy + (i64)w.ix * gny] += w.w00 * gu;
      gu_[w.iy + (i64)w.ix2 * gny] += w.w01 * gu;
      gu_[w.iy2 + (i64)w.ix * gny] += w.w10 * gu;
      gu_[w.iy2 + (i64)w.ix2 * gny] += w.w11 * gu;
      gv_[w.iy + (i64)w.ix * gny] += w.w00 * gv;
      gv_[w.iy + (i64)w.ix2 * gny] += w.w01 * gv;
      gv_[w.iy2 + (i64)w.ix * gny] += w.w10 * gv;
      gv_[w.iy2 + (i64)w.ix2 * gny] += w.w11 * gv;
    }
  }
  return L;
}

template <class F> static void parallel_for(int nthreads, i64 n, F f) {
  nthreads = (int)std::max<i64>(1, std::min<i64>(nthreads, n));
  if (nthreads == 1) { f(0, (i64)0, n); return; }
  i64 chunk = (n + nthreads - 1) / nthreads;
  std::vector<std::thread> th;
  for (int t = 0; t < nthreads; ++t) {
    i64 a = t * chunk, b = std::min(n, a + chunk);
    if (a >= b) break;
    th.emplace_back([=]() { f(t, a, b); });
  }
  for (auto& x : th) x.join();
}

// ---------------------------------------------------------------------------
// Pass grid: src/pipeline.jl:529-555
struct Grid {
  std::vector<int> rows, cols;  // 1-based window starts
  int ny = 0, nx = 0;
  std::vector<uint8_t> gmask;
  std::vector<int> jobs;  // 4 per job: gi, gj (0-based), rs, cs (1-based)
};

static int make_grid(i64 nr, i64 nc, const Pass& p, const uint8_t* mask, double thr, Grid& g) {
  int wr = p.window[0], wc = p.window[1], sr = p.search[0], sc = p.search[1];
  int mr = (sr - wr) / 2, mc = (sc - wc) / 2;
  if (sr > nr || sc > nc) return -1;
  g.rows.clear();
  g.cols.clear();
  for (i64 s = 1 + mr; s <= nr - wr - mr + 1; s += wr - p.overlap[0]) g.rows.push_back((int)s);
  for (i64 s = 1 + mc; s <= nc - wc - mc + 1; s += wc - p.overlap[1]) g.cols.push_back((int)s);
  g.ny = (int)g.rows.size();
  g.nx = (int)g.cols.size();
  g.gmask.assign((size_t)g.ny * g.nx, 0);
  if (mask) {
    for (int gj = 0; gj < g.nx; ++gj)
      for (int gi = 0; gi < g.ny; ++gi) {
        int rs = g.rows[gi], cs = g.cols[gj];
        i64 cw = 0, csr = 0;
        for (int j = 0; j < wc; ++j)
          for (int i = 0; i < wr; ++i) cw += mask[(rs - 1 + i) + (i64)(cs - 1 + j) * nr] != 0;
        int srs = rs - mr, scs = cs - mc;
        for (int j = 0; j < sc; ++j)
          for (int i = 0; i < sr; ++i) csr += mask[(srs - 1 + i) + (i64)(scs - 1 + j) * nr] != 0;
        double fw = (double)cw / (double)(wr * wc), fs = (double)csr / (double)(sr * sc);
        g.gmask[gi + (i64)gj * g.ny] = fw >= thr || fs >= thr;
      }
  }
  g.jobs.clear();
  for (int gj = 0; gj < g.nx; ++gj)
    for (int gi = 0; gi < g.ny; ++gi)
      if (!g.gmask[gi + (i64)gj * g.ny]) {
        g.jobs.push_back(gi);
        g.jobs.push_back(gj);
        g.jobs.push_back(g.rows[gi]);
        g.jobs.push_back(g.cols[gj]);
      }
  return 0;
}

template <class T> struct Field {
  int ny = 0, nx = 0;
  std::vector<T> x, y, u, v;
  std::vector<uint8_t> mask;
};

struct Timing {
  double deform = 0, correlate = 0, validate = 0, uq = 0, total = 0, final_pass = 0;
  int sweeps[64] = {0};
};

static double now_s() {
  return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

template <class T> struct Result {
  Grid grid;
  std::vector<T> x, y, u, v, ratio, moment, unc_u, unc_v;
  std::vector<uint8_t> outliers;
};

// process_windows! src/pipeline.jl:972-1027 over a chunk of jobs
template <class T>
static void process_chunk(const int* jobs, i64 njobs, const T* A, const T* B, i64 nr, const uint8_t* mask,
                          const Pass& p, Correlator<T>& c, T* ru, T* rv, T* ratio, T* moment, T* alt_u, T* alt_v,
                          T* unc_u, T* unc_v, int ny, int nx) {
  const int wr = p.window[0], wc = p.window[1];
  const int mr = (p.search[0] - wr) / 2, mc = (p.search[1] - wc) / 2;
  const int K = std::max(p.n_peaks, 2);
  std::vector<T> out(5 + 2 * (K - 1));
  const i64 G = (i64)ny * nx;
  for (i64 q = 0; q < njobs; ++q) {
    int gi = jobs[4 * q], gj = jobs[4 * q + 1], rs = jobs[4 * q + 2] - 1, cs = jobs[4 * q + 3] - 1;
    const T* subA = A + rs + (i64)cs * nr;
    const T* subB = B + (rs - mr) + (i64)(cs - mc) * nr;
    const uint8_t* mA = nullptr;
    const uint8_t* mB = nullptr;
    if (mask) {
      mA = mask + rs + (i64)cs * nr;
      bool any = false;
      for (int j = 0; j < wc && !any; ++j)
        for (int i = 0; i < wr; ++i)
          if (mA[i + (i64)j * nr]) { any = true; break; }
      if (!any) mA = nullptr;
      if (p.search[0] == wr && p.search[1] == wc) mB = mA;
      else {
        mB = mask + (rs - mr) + (i64)(cs - mc) * nr;
        bool anyb = false;
        for (int j = 0; j < p.search[1] && !anyb; ++j)
          for (int i = 0; i < p.search[0]; ++i)
            if (mB[i + (i64)j * nr]) { anyb = true; break; }
        if (!anyb) mB = nullptr;
      }
    }
    const T* R = correlation_plane(c, subA, subB, nr, mA, mB, nr);
    analyze_plane(R, c.nr, c.nc, p.n_peaks, p.finder, p.subpixel, out.data(), (int*)nullptr);
    i64 id = gi + (i64)gj * ny;
    ru[id] = out[0];
    rv[id] = out[1];
    ratio[id] = out[2];
    moment[id] = out[3];
    int found = (int)out[4];
    if (alt_u)
      for (int m = 2; m <= std::min(found, p.n_peaks); ++m) {
        alt_u[id + (i64)(m - 2) * G] = out[5 + (m - 2)];
        alt_v[id + (i64)(m - 2) * G] = out[5 + (K - 1) + (m - 2)];
      }
    if (unc_u) {
      double st[88] = {0};
      uq_window_stats(st, subA, B + rs + (i64)cs * nr, nr, mA, nr, wr, wc, c.apod.data());
      unc_u[id] = finalize_uq<T>(st);
      unc_v[id] = finalize_uq<T>(st + 44);
    }
  }
}

template <class T>
static void uq_chunk(const int* jobs, i64 njobs, const T* A, const T* B, i64 nr, const uint8_t* mask, const Pass& p,
                     const T* apod, T* unc_u, T* unc_v, int ny) {
  const int wr = p.window[0], wc = p.window[1];
  for (i64 q = 0; q < njobs; ++q) {
    int gi = jobs[4 * q], gj = jobs[4 * q + 1], rs = jobs[4 * q + 2] - 1, cs = jobs[4 * q + 3] - 1;
    const uint8_t* m = nullptr;
    if (mask) {
      m = mask + rs + (i64)cs * nr;
      bool any = false;
      for (int j = 0; j < wc && !any; ++j)
        for (int i = 0; i < wr; ++i)
          if (m[i + (i64)j * nr]) { any = true; break; }
      if (!any) m = nullptr;
    }
    double st[88] = {0};
    uq_window_stats(st, A + rs + (i64)cs * nr, B + rs + (i64)cs * nr, nr, m, nr, wr, wc, apod);
    i64 id = gi + (i64)gj * ny;
    unc_u[id] = finalize_uq<T>(st);
    unc_v[id] = finalize_uq<T>(st + 44);
  }
}

// run_piv src/pipeline.jl:361-449 with piv_pass :655-832 and
// build_predictor :454-464. Threads split the job list into contiguous
// chunks exactly like :711-754; results do not depend on the split.
template <class T>
static int run_piv(const T* A, const T* B, i64 nr, i64 nc, const Pass* passes, int npasses, const uint8_t* mask,
                   double mask_thr, bool smoothing, int nthreads, Result<T>& res, Timing* tm) {
  double t_start = now_s();
  const bool deforms = npasses > 1 || std::any_of(passes, passes + npasses, [](const Pass& p) { return p.max_iterations > 1; });
  std::vector<T> CA, CB, wA, wB;
  if (deforms) {
    CA.resize((size_t)(nr + 2) * (nc + 2));
    CB.resize((size_t)(nr + 2) * (nc + 2));
    double t0 = now_s();
    std::thread ta([&]() { prefilter(A, nr, nc, CA.data()); });
    prefilter(B, nr, nc, CB.data());
    ta.join();
    if (tm) tm->deform += now_s() - t0;
    wA.resize((size_t)nr * nc);
    wB.resize((size_t)nr * nc);
  }
  bool have_pred = false;
  std::vector<T> pred_u, pred_v;
  Predictor pg;
  Result<T> cur;
  for (int k = 0; k < npasses; ++k) {
    const Pass& p = passes[k];
    double t_pass = now_s();
    bool force_replace = k < npasses - 1;
    if (k > 0) {
      // build_predictor(prev result)
      std::vector<T> pu = cur.u, pv = cur.v;
      bool anym = false;
      for (auto m : cur.grid.gmask) anym |= m != 0;
      if (anym) replace_vectors(pu.data(), pv.data(), cur.grid.ny, cur.grid.nx, cur.grid.gmask.data());
      if (smoothing) {
        pred_u.resize(pu.size());
        pred_v.resize(pv.size());
        smooth_field(pu.data(), cur.grid.ny, cur.grid.nx, pred_u.data());
        smooth_field(pv.data(), cur.grid.ny, cur.grid.nx, pred_v.data());
      } else {
        pred_u = pu;
        pred_v = pv;
      }
      pg.gny = cur.grid.ny;
      pg.gnx = cur.grid.nx;
      pg.y0 = cur.y[0];
      pg.x0 = cur.x[0];
      pg.ysp = cur.grid.ny > 1 ? (double)(cur.y[1] - cur.y[0]) : 1.0;
      pg.xsp = cur.grid.nx > 1 ? (double)(cur.x[1] - cur.x[0]) : 1.0;
      have_pred = true;
    }
    Result<T> r;
    if (make_grid(nr, nc, p, mask, mask_thr, r.grid) != 0) return -1;
    const int ny = r.grid.ny, nx = r.grid.nx;
    const i64 G = (i64)ny * nx;
    r.x.resize(nx);
    r.y.resize(ny);
    for (int j = 0; j < nx; ++j) r.x[j] = (T)(r.grid.cols[j] + (p.window[1] - 1) / 2.0);
    for (int i = 0; i < ny; ++i) r.y[i] = (T)(r.grid.rows[i] + (p.window[0] - 1) / 2.0);
    const T NaN = std::numeric_limits<T>::quiet_NaN();
    std::vector<T> resu(G, 0), resv(G, 0), ratio(G, 0), moment(G, 0);
    int nalt = p.n_peaks - 1;
    std::vector<T> altu, altv;
    if (nalt > 0) {
      altu.assign(G * nalt, NaN);
      altv.assign(G * nalt, NaN);
    }
    bool unc = p.uncertainty && !force_replace;
    r.unc_u.assign(G, NaN);
    r.unc_v.assign(G, NaN);
    bool fused_unc = unc && p.max_iterations == 1;
    const i64 njobs = (i64)r.grid.jobs.size() / 4;
    int nch = (int)std::max<i64>(1, std::min<i64>(nthreads, njobs));
    std::vector<Correlator<T>*> cors;
    for (int t = 0; t < nch; ++t) cors.push_back(new Correlator<T>(p));
    bool keep_measured = p.max_iterations > 1 && !(force_replace || p.replace_outliers);
    std::vector<T> meas_u, meas_v, prev_u, prev_v;
    bool have_prev = false;
    const T* srcA = A;
    const T* srcB = B;
    std::vector<T> u, v;
    std::vector<uint8_t> outl;
    int sweeps = 0;
    for (int it = 1; it <= p.max_iterations; ++it) {
      ++sweeps;
      double t0 = now_s();
      u.assign(G, T(0));
      v.assign(G, T(0));
      if (have_pred) {
        for (int gj = 0; gj < nx; ++gj)
          for (int gi = 0; gi < ny; ++gi) {
            u[gi + (i64)gj * ny] = bilinear(pred_u.data(), pg.gny, pg.gnx, (T)pg.y0, (T)pg.ysp, (T)pg.x0, (T)pg.xsp,
                                            r.y[gi], r.x[gj]);
            v[gi + (i64)gj * ny] = bilinear(pred_v.data(), pg.gny, pg.gnx, (T)pg.y0, (T)pg.ysp, (T)pg.x0, (T)pg.xsp,
                                            r.y[gi], r.x[gj]);
          }
        parallel_for(nthreads, nc, [&](int, i64 a, i64 b) {
          deform_columns(CA.data(), CB.data(), nr, nc, pred_u.data(), pred_v.data(), pg, wA.data(), wB.data(), a, b);
        });
        srcA = wA.data();
        srcB = wB.data();
      } else {
        srcA = A;
        srcB = B;
      }
      double t1 = now_s();
      if (tm) tm->deform += t1 - t0;
      if (it > 1) {
        std::fill(resu.begin(), resu.end(), T(0));
        std::fill(resv.begin(), resv.end(), T(0));
        std::fill(altu.begin(), altu.end(), NaN);
        std::fill(altv.begin(), altv.end(), NaN);
      }
      i64 chunk = (njobs + nch - 1) / std::max(nch, 1);
      parallel_for(nch, nch, [&](int, i64 a, i64 b) {
        for (i64 t = a; t < b; ++t) {
          i64 j0 = t * chunk, j1 = std::min(njobs, j0 + chunk);
          if (j0 >= j1) continue;
          process_chunk(r.grid.jobs.data() + 4 * j0, j1 - j0, srcA, srcB, nr, mask, p, *cors[t], resu.data(),
                        resv.data(), ratio.data(), moment.data(), nalt > 0 ? altu.data() : nullptr,
                        nalt > 0 ? altv.data() : nullptr, fused_unc ? r.unc_u.data() : nullptr,
                        fused_unc ? r.unc_v.data() : nullptr, ny, nx);
        }
      });
      double t2 = now_s();
      if (tm) tm->correlate += t2 - t1;
      if (nalt > 0)
        for (int m = 0; m < nalt; ++m)
          for (i64 q = 0; q < G; ++q) {
            altu[q + m * G] += u[q];
            altv[q + m * G] += v[q];
          }
      for (i64 q = 0; q < G; ++q) {
        u[q] += resu[q];
        v[q] += resv[q];
      }
      for (i64 q = 0; q < G; ++q)
        if (r.grid.gmask[q]) u[q] = v[q] = ratio[q] = moment[q] = NaN;
      if (keep_measured) {
        meas_u = u;
        meas_v = v;
      }
      outl.assign(G, 0);
      validate_and_replace(u.data(), v.data(), ratio.data(), moment.data(), outl.data(), r.grid.gmask.data(), ny, nx,
                           p, force_replace || p.max_iterations > 1, nalt > 0 ? altu.data() : nullptr,
                           nalt > 0 ? altv.data() : nullptr, nalt);
      if (tm) tm->validate += now_s() - t2;
      if (it == p.max_iterations) break;
      if (p.convergence_tol > 0) {
        if (!have_prev) {
          prev_u = u;
          prev_v = v;
          have_prev = true;
        } else {
          T ch = field_change(u.data(), v.data(), prev_u.data(), prev_v.data(), r.grid.gmask.data(), G);
          if ((double)ch < p.convergence_tol) break;
          prev_u = u;
          prev_v = v;
        }
      }
      // build_predictor from this sweep's validated field
      std::vector<T> pu = u, pv = v;
      bool anym = false;
      for (auto m : r.grid.gmask) anym |= m != 0;
      if (anym) replace_vectors(pu.data(), pv.data(), ny, nx, r.grid.gmask.data());
      if (smoothing) {
        pred_u.resize(G);
        pred_v.resize(G);
        smooth_field(pu.data(), ny, nx, pred_u.data());
        smooth_field(pv.data(), ny, nx, pred_v.data());
      } else {
        pred_u = pu;
        pred_v = pv;
      }
      pg.gny = ny;
      pg.gnx = nx;
      pg.y0 = r.y[0];
      pg.x0 = r.x[0];
      pg.ysp = ny > 1 ? (double)(r.y[1] - r.y[0]) : 1.0;
      pg.xsp = nx > 1 ? (double)(r.x[1] - r.x[0]) : 1.0;
      have_pred = true;
    }
    if (unc && !fused_unc) {
      double t0 = now_s();
      std::vector<T> apod((size_t)p.window[0] * p.window[1]);
      apodization_window(p.window[0], p.window[1], p.apod, apod.data());
      i64 chunk = (njobs + nch - 1) / std::max(nch, 1);
      parallel_for(nch, nch, [&](int, i64 a, i64 b) {
        for (i64 t = a; t < b; ++t) {
          i64 j0 = t * chunk, j1 = std::min(njobs, j0 + chunk);
          if (j0 >= j1) continue;
          uq_chunk(r.grid.jobs.data() + 4 * j0, j1 - j0, srcA, srcB, nr, mask, p, apod.data(), r.unc_u.data(),
                   r.unc_v.data(), ny);
        }
      });
      if (tm) tm->uq += now_s() - t0;
    }
    if (keep_measured)
      for (i64 q = 0; q < G; ++q)
        if (outl[q]) {
          u[q] = meas_u[q];
          v[q] = meas_v[q];
        }
    for (auto* c : cors) delete c;
    r.u = u;
    r.v = v;
    r.ratio = ratio;
    r.moment = moment;
    r.outliers = outl;
    if (tm && k < 64) tm->sweeps[k] = sweeps;
    if (tm && k == npasses - 1) tm->final_pass = now_s() - t_pass;
    cur = std::move(r);
  }
  res = std::move(cur);
  if (tm) tm->total = now_s() - t_start;
  return 0;
}

// run_piv_ensemble (src/ensemble.jl:51-205): per pass, every pair is
// deformed by the shared predictor, each window's correlation planes are
// summed over the pairs in pair order (accumulate_planes!, :310-343) and
// analysed once (ensemble_analyze!, :273-305); the Wieneke statistics pool
// by summation; then validate_and_replace! with replacement forced on
// intermediate passes. One sweep per pass (max_iterations is not used).
template <class T>
static int run_ensemble(const T* const* As, const T* const* Bs, int npairs, i64 nr, i64 nc, const Pass* passes,
                        int npasses, const uint8_t* mask, double mask_thr, bool smoothing, int nthreads,
                        Result<T>& res) {
  std::vector<T> CA, CB, wA, wB;
  bool have_pred = false;
  std::vector<T> pred_u, pred_v;
  Predictor pg;
  Result<T> cur;
  const T NaN = std::numeric_limits<T>::quiet_NaN();
  for (int k = 0; k < npasses; ++k) {
    const Pass& p = passes[k];
    const bool force_replace = k < npasses - 1;
    if (k > 0) {
      std::vector<T> pu = cur.u, pv = cur.v;
      bool anym = false;
      for (auto m : cur.grid.gmask) anym |= m != 0;
      if (anym) replace_vectors(pu.data(), pv.data(), cur.grid.ny, cur.grid.nx, cur.grid.gmask.data());
      if (smoothing) {
        pred_u.resize(pu.size());
        pred_v.resize(pv.size());
        smooth_field(pu.data(), cur.grid.ny, cur.grid.nx, pred_u.data());
        smooth_field(pv.data(), cur.grid.ny, cur.grid.nx, pred_v.data());
      } else {
        pred_u = pu;
        pred_v = pv;
      }
      pg.gny = cur.grid.ny;
      pg.gnx = cur.grid.nx;
      pg.y0 = cur.y[0];
      pg.x0 = cur.x[0];
      pg.ysp = cur.grid.ny > 1 ? (double)(cur.y[1] - cur.y[0]) : 1.0;
      pg.xsp = cur.grid.nx > 1 ? (double)(cur.x[1] - cur.x[0]) : 1.0;
      have_pred = true;
    }
    Result<T> r;
    if (make_grid(nr, nc, p, mask, mask_thr, r.grid) != 0) return -1;
    const int ny = r.grid.ny, nx = r.grid.nx;
    const i64 G = (i64)ny * nx;
    r.x.resize(nx);
    r.y.resize(ny);
    for (int j = 0; j < nx; ++j) r.x[j] = (T)(r.grid.cols[j] + (p.window[1] - 1) / 2.0);
    for (int i = 0; i < ny; ++i) r.y[i] = (T)(r.grid.rows[i] + (p.window[0] - 1) / 2.0);
    const i64 njobs = (i64)r.grid.jobs.size() / 4;
    const int nalt = p.n_peaks - 1, K = std::max(p.n_peaks, 2);
    const bool unc = p.uncertainty && !force_replace;
    // node values of the shared predictor (zero without one)
    std::vector<T> u(G, T(0)), v(G, T(0));
    if (have_pred)
      for (int gj = 0; gj < nx; ++gj)
        for (int gi = 0; gi < ny; ++gi) {
          u[gi + (i64)gj * ny] =
              bilinear(pred_u.data(), pg.gny, pg.gnx, (T)pg.y0, (T)pg.ysp, (T)pg.x0, (T)pg.xsp, r.y[gi], r.x[gj]);
          v[gi + (i64)gj * ny] =
              bilinear(pred_v.data(), pg.gny, pg.gnx, (T)pg.y0, (T)pg.ysp, (T)pg.x0, (T)pg.xsp, r.y[gi], r.x[gj]);
        }
    int nch = (int)std::max<i64>(1, std::min<i64>(nthreads, njobs));
    std::vector<Correlator<T>*> cors;
    for (int t = 0; t < nch; ++t) cors.push_back(new Correlator<T>(p));
    const i64 PN = (i64)cors[0]->nr * cors[0]->nc;
    std::vector<T> acc((size_t)std::max<i64>(njobs, 1) * PN, T(0));
    std::vector<double> uacc(unc ? (size_t)njobs * 88 : 0, 0.0);
    std::vector<T> apod((size_t)p.window[0] * p.window[1]);
    apodization_window(p.window[0], p.window[1], p.apod, apod.data());
    const int wr = p.window[0], wc = p.window[1];
    const int mr = (p.search[0] - wr) / 2, mc = (p.search[1] - wc) / 2;
    for (int q = 0; q < npairs; ++q) {
      const T* srcA = As[q];
      const T* srcB = Bs[q];
      if (have_pred) {
        CA.resize((size_t)(nr + 2) * (nc + 2));
        CB.resize((size_t)(nr + 2) * (nc + 2));
        wA.resize((size_t)nr * nc);
        wB.resize((size_t)nr * nc);
        std::thread ta([&]() { prefilter(As[q], nr, nc, CA.data()); });
        prefilter(Bs[q], nr, nc, CB.data());
        ta.join();
        parallel_for(nthreads, nc, [&](int, i64 a, i64 b) {
          deform_columns(CA.data(), CB.data(), nr, nc, pred_u.data(), pred_v.data(), pg, wA.data(), wB.data(), a, b);
        });
        srcA = wA.data();
        srcB = wB.data();
      }
      const i64 chunk = (njobs + nch - 1) / std::max(nch, 1);
      parallel_for(nch, nch, [&](int, i64 a, i64 b) {
        for (i64 t = a; t < b; ++t) {
          const i64 j0 = t * chunk, j1 = std::min(njobs, j0 + chunk);
          for (i64 j = j0; j < j1; ++j) {
            const int* jb = r.grid.jobs.data() + 4 * j;
            const int rs = jb[2] - 1, cs = jb[3] - 1;
            const T* subA = srcA + rs + (i64)cs * nr;
            const T* subB = srcB + (rs - mr) + (i64)(cs - mc) * nr;
            const uint8_t* mA = nullptr;
            const uint8_t* mB = nullptr;
            if (mask) {
              mA = mask + rs + (i64)cs * nr;
              bool any = false;
              for (int jj = 0; jj < wc && !any; ++jj)
                for (int ii = 0; ii < wr; ++ii)
                  if (mA[ii + (i64)jj * nr]) { any = true; break; }
              if (!any) mA = nullptr;
              mB = mA;
            }
            const T* R = correlation_plane(*cors[t], subA, subB, nr, mA, mB, nr);
            T* dst = acc.data() + j * PN;
            for (i64 e = 0; e < PN; ++e) dst[e] += R[e];
            if (unc) {
              double st[88] = {0};
              uq_window_stats(st, subA, srcB + rs + (i64)cs * nr, nr, mA, nr, wr, wc, apod.data());
              for (int e = 0; e < 88; ++e) uacc[j * 88 + e] += st[e];
            }
          }
        }
      });
    }
    std::vector<T> ratio(G, T(0)), moment(G, T(0));
    std::vector<T> altu(nalt > 0 ? G * nalt : 0, NaN), altv(nalt > 0 ? G * nalt : 0, NaN);
    r.unc_u.assign(G, NaN);
    r.unc_v.assign(G, NaN);
    std::vector<T> out(5 + 2 * (K - 1));
    for (i64 j = 0; j < njobs; ++j) {
      const int gi = r.grid.jobs[4 * j], gj = r.grid.jobs[4 * j + 1];
      const i64 id = gi + (i64)gj * ny;
      analyze_plane(acc.data() + j * PN, cors[0]->nr, cors[0]->nc, p.n_peaks, p.finder, p.subpixel, out.data(),
                    (int*)nullptr);
      const int found = (int)out[4];
      for (int m = 2; m <= std::min(found, p.n_peaks); ++m) {
        altu[id + (i64)(m - 2) * G] = u[id] + out[5 + (m - 2)];
        altv[id + (i64)(m - 2) * G] = v[id] + out[5 + (K - 1) + (m - 2)];
      }
      u[id] += out[0];
      v[id] += out[1];
      ratio[id] = out[2];
      moment[id] = out[3];
      if (unc) {
        r.unc_u[id] = finalize_uq<T>(uacc.data() + j * 88);
        r.unc_v[id] = finalize_uq<T>(uacc.data() + j * 88 + 44);
      }
    }
    for (i64 q = 0; q < G; ++q)
      if (r.grid.gmask[q]) u[q] = v[q] = ratio[q] = moment[q] = NaN;
    std::vector<uint8_t> outl(G, 0);
    validate_and_replace(u.data(), v.data(), ratio.data(), moment.data(), outl.data(), r.grid.gmask.data(), ny, nx, p,
                         force_replace, nalt > 0 ? altu.data() : nullptr, nalt > 0 ? altv.data() : nullptr, nalt);
    for (auto* c : cors) delete c;
    r.u = u;
    r.v = v;
    r.ratio = ratio;
    r.moment = moment;
    r.outliers = outl;
    cur = std::move(r);
  }
  res = std::move(cur);
  return 0;
}

}  // namespace orc

// ===========================================================================
// C entry points (ctypes). Suffix _f32 = float instantiation, _f64 = double.
extern "C" {

struct orc_result_f32 {
  int32_t ny, nx;
  float *x, *y, *u, *v, *peak_ratio, *moment, *unc_u, *unc_v;
  uint8_t *outliers, *mask;
};
struct orc_result_f64 {
  int32_t ny, nx;
  double *x, *y, *u, *v, *peak_ratio, *moment, *unc_u, *unc_v;
  uint8_t *outliers, *mask;
};

int orc_sizeof_pass() { return (int)sizeof(orc::Pass); }

int orc_pass_grid(int64_t nr, int64_t nc, const orc::Pass* p, const uint8_t* mask, double thr, int32_t* ny,
                  int32_t* nx, uint8_t* gmask_out, int32_t* jobs_out) {
  orc::Grid g;
  if (orc::make_grid(nr, nc, *p, mask, thr, g) != 0) return -1;
  *ny = g.ny;
  *nx = g.nx;
  if (gmask_out) std::copy(g.gmask.begin(), g.gmask.end(), gmask_out);
  if (jobs_out) std::copy(g.jobs.begin(), g.jobs.end(), jobs_out);
  return (int)(g.jobs.size() / 4);
}

#define ORC_DEFINE(T, SUF)                                                                                          \
  int orc_run_piv_##SUF(const T* A, const T* B, int64_t nr, int64_t nc, const orc::Pass* passes, int npasses,      \
                        const uint8_t* mask, double thr, int smoothing, int nthreads, orc_result_##SUF* out,      \
                        double* timing /*6*/, int32_t* sweeps /*npasses*/) {                                      \
    orc::Result<T> r;                                                                                                \
    orc::Timing tm;                                                                                                  \
    if (orc::run_piv<T>(A, B, nr, nc, passes, npasses, mask, thr, smoothing != 0, nthreads, r, &tm) != 0)           \
      return -1;                                                                                                     \
    out->ny = r.grid.ny;                                                                                             \
    out->nx = r.grid.nx;                                                                                             \
    const size_t G = (size_t)r.grid.ny * r.grid.nx;                                                                  \
    if (out->x) std::copy(r.x.begin(), r.x.end(), out->x);                                                           \
    if (out->y) std::copy(r.y.begin(), r.y.end(), out->y);                                                           \
    if (out->u) std::copy(r.u.begin(), r.u.begin() + G, out->u);                                                     \
    if (out->v) std::copy(r.v.begin(), r.v.begin() + G, out->v);                                                     \
    if (out->peak_ratio) std::copy(r.ratio.begin(), r.ratio.end(), out->peak_ratio);                                 \
    if (out->moment) std::copy(r.moment.begin(), r.moment.end(), out->moment);                                       \
    if (out->unc_u) std::copy(r.unc_u.begin(), r.unc_u.end(), out->unc_u);                                           \
    if (out->unc_v) std::copy(r.unc_v.begin(), r.unc_v.end(), out->unc_v);                                           \
    if (out->outliers) std::copy(r.outliers.begin(), r.outliers.end(), out->outliers);                               \
    if (out->mask) std::copy(r.grid.gmask.begin(), r.grid.gmask.end(), out->mask);                                   \
    if (timing) {                                                                                                    \
      timing[0] = tm.deform;                                                                                         \
      timing[1] = tm.correlate;                                                                                      \
      timing[2] = tm.validate;                                                                                       \
      timing[3] = tm.uq;                                                                                             \
      timing[4] = tm.total;                                                                                          \
      timing[5] = tm.final_pass;                                                                                     \
    }                                                                                                                \
    if (sweeps)                                                                                                      \
      for (int k = 0; k < npasses && k < 64; ++k) sweeps[k] = tm.sweeps[k];                                          \
    return 0;                                                                                                        \
  }                                                                                                                  \
  int orc_find_peaks_##SUF(const T* R, int nr, int nc, int k, int finder, int excl, T* vals, int32_t* locs) {        \
    std::vector<int> l(2 * k);                                                                                       \
    int f = orc::find_peaks(vals, l.data(), R, nr, nc, k, finder, excl);                                             \
    for (int m = 0; m < 2 * f; ++m) locs[m] = l[m];                                                                  \
    return f;                                                                                                        \
  }                                                                                                                  \
  void orc_gauss3_##SUF(const T* R, int nr, int nc, int pr, int pc, T* out) { orc::gauss3(R, nr, nc, pr, pc, out); } \
  void orc_gauss9_##SUF(const T* R, int nr, int nc, int pr, int pc, T* out) { orc::gauss9(R, nr, nc, pr, pc, out); } \
  double orc_moment_##SUF(const T* R, int nr, int nc, T pr, T pc) {                                                  \
    return orc::correlation_moment(R, nr, nc, pr, pc);                                                               \
  }                                                                                                                  \
  T orc_peak_ratio_##SUF(const T* R, int nr, int nc, int pr, int pc, int excl, int finder) {                         \
    return orc::peak_ratio(R, nr, nc, pr, pc, excl, finder);                                                         \
  }                                                                                                                  \
  void orc_analyze_plane_##SUF(const T* R, int nr, int nc, int npeaks, int finder, int subpixel, T* out,             \
                               int32_t* locs) {                                                                      \
    std::vector<int> l(2 * std::max(npeaks, 2));                                                                     \
    orc::analyze_plane(R, nr, nc, npeaks, finder, subpixel, out, l.data());                                          \
    if (locs) std::copy(l.begin(), l.end(), locs);                                                                   \
  }                                                                                                                  \
  void orc_uod_##SUF(const T* u, const T* v, int nr, int nc, double thr, int nb, double eps,                         \
                     const uint8_t* exclude, uint8_t* out) {                                                         \
    orc::uod(u, v, nr, nc, thr, nb, eps, exclude, out);                                                              \
  }                                                                                                                  \
  void orc_replace_vectors_##SUF(T* u, T* v, int nr, int nc, const uint8_t* invalid) {                               \
    orc::replace_vectors(u, v, nr, nc, invalid);                                                                     \
  }                                                                                                                  \
  void orc_smooth_field_##SUF(const T* f, int nr, int nc, T* out) { orc::smooth_field(f, nr, nc, out); }             \
  int orc_substitute_##SUF(T* u, T* v, uint8_t* outl, const uint8_t* mask, const T* au, const T* av, int nalt,       \
                           int nr, int nc, int er, double thr) {                                                     \
    return orc::substitute(u, v, outl, mask, au, av, nalt, nr, nc, er, thr);                                         \
  }                                                                                                                  \
  void orc_validate_##SUF(T* u, T* v, const T* ratio, const T* moment, uint8_t* outl, const uint8_t* mask, int nr,   \
                          int nc, const orc::Pass* p, int force_replace, const T* au, const T* av, int nalt) {       \
    orc::validate_and_replace(u, v, ratio, moment, outl, mask, nr, nc, *p, force_replace != 0, au, av, nalt);        \
  }                                                                                                                  \
  void orc_fft2_##SUF(T* z /*interleaved re,im*/, int n1, int n2, int inverse) {                                     \
    orc::FFT2<T> f(n1, n2);                                                                                          \
    if (inverse) f.inverse((orc::cx<T>*)z);                                                                          \
    else f.forward((orc::cx<T>*)z);                                                                                  \
  }                                                                                                                  \
  int orc_correlation_plane_##SUF(const T* A, const T* B, int64_t ld, const orc::Pass* p, T* R_out) {               \
    orc::Correlator<T> c(*p);                                                                                        \
    const T* R = orc::correlation_plane(c, A, B, ld, (const uint8_t*)nullptr, (const uint8_t*)nullptr, 0);           \
    std::copy(R, R + (size_t)c.nr * c.nc, R_out);                                                                    \
    return c.nr;                                                                                                     \
  }                                                                                                                  \
  void orc_apodization_##SUF(int wr, int wc, int apod, T* out) { orc::apodization_window(wr, wc, apod, out); }       \
  void orc_overlap_gain_##SUF(int wr, int wc, int apod, T* out) {                                                   \
    std::vector<T> a((size_t)wr * wc);                                                                               \
    orc::apodization_window(wr, wc, apod, a.data());                                                                 \
    orc::overlap_gain(wr, wc, a.data(), 2 * wr, 2 * wc, out);                                                        \
  }                                                                                                                  \
  void orc_prefilter_##SUF(const T* img, int64_t nr, int64_t nc, T* coef) { orc::prefilter(img, nr, nc, coef); }     \
  T orc_bspline_eval_##SUF(const T* C, int64_t nr, int64_t nc, T yy, T xx) {                                         \
    return orc::bspline_eval(C, nr, nc, yy, xx);                                                                     \
  }                                                                                                                  \
  void orc_deform_##SUF(const T* CA, const T* CB, int64_t nr, int64_t nc, const T* pu, const T* pv, int gny,         \
                        int gnx, double y0, double ysp, double x0, double xsp, T* wA, T* wB, int nthreads) {         \
    orc::Predictor g;                                                                                                \
    g.gny = gny;                                                                                                     \
    g.gnx = gnx;                                                                                                     \
    g.y0 = y0;                                                                                                       \
    g.ysp = ysp;                                                                                                     \
    g.x0 = x0;                                                                                                       \
    g.xsp = xsp;                                                                                                     \
    orc::parallel_for(nthreads, nc, [&](int, int64_t a, int64_t b) {                                                 \
      orc::deform_columns(CA, CB, nr, nc, pu, pv, g, wA, wB, a, b);                                                  \
    });                                                                                                              \
  }                                                                                                                  \
  T orc_bilinear_##SUF(const T* f, int gny, int gnx, double y0, double ysp, double x0, double xsp, T qy, T qx) {     \
    return orc::bilinear(f, gny, gnx, (T)y0, (T)ysp, (T)x0, (T)xsp, qy, qx);                                         \
  }                                                                                                                  \
  void orc_uq_stats_##SUF(const T* A, const T* B, int64_t ld, int wr, int wc, int apod, const uint8_t* m,            \
                          double* stats) {                                                                           \
    std::vector<T> a((size_t)wr * wc);                                                                               \
    orc::apodization_window(wr, wc, apod, a.data());                                                                 \
    for (int k = 0; k < 88; ++k) stats[k] = 0;                                                                       \
    orc::uq_window_stats(stats, A, B, ld, m, ld, wr, wc, a.data());                                                  \
  }                                                                                                                  \
  T orc_finalize_uq_##SUF(const double* s) { return orc::finalize_uq<T>(s); }                                        \
  T orc_field_change_##SUF(const T* u, const T* v, const T* pu, const T* pv, const uint8_t* mask, int64_t n) {       \
    return orc::field_change(u, v, pu, pv, mask, n);                                                                 \
  }

ORC_DEFINE(float, f32)
ORC_DEFINE(double, f64)

// NCC loss (and gradient when grad != NULL, zeroed here) over the given
// windows of a prefiltered pair; threads split the windows, each thread
// accumulating its own gradient, summed in thread order.
#define ORC_NCC(T, SUF)                                                                                              \
  double orc_ncc_loss_grad_##SUF(const T* CA, const T* CB, int64_t nr, int64_t nc, const T* P, int gny, int gnx,    \
                                 double y0, double ysp, double x0, double xsp, int W, const int32_t* wins,          \
                                 int64_t nwin, T* grad, int nthreads) {                                              \
    const int64_t G2 = 2 * (int64_t)gny * gnx;                                                                       \
    nthreads = (int)std::max<int64_t>(1, std::min<int64_t>(nthreads, nwin));                                        \
    std::vector<double> Ls(nthreads, 0.0);                                                                           \
    std::vector<std::vector<T>> gs(grad ? nthreads : 0, std::vector<T>(grad ? G2 : 0, T(0)));                        \
    std::vector<std::thread> th;                                                                                     \
    for (int t = 0; t < nthreads; ++t)                                                                               \
      th.emplace_back([&, t]() {                                                                                     \
        const int64_t j0 = nwin * t / nthreads, j1 = nwin * (t + 1) / nthreads;                                      \
        Ls[t] = orc::ncc_loss_grad<T>(CA, CB, nr, nc, P, gny, gnx, (T)y0, (T)ysp, (T)x0, (T)xsp, W, wins + 2 * j0,  \
                                      j1 - j0, grad ? gs[t].data() : nullptr);                                       \
      });                                                                                                            \
    for (auto& x : th) x.join();                                                                                     \
    double L = 0;                                                                                                    \
    for (int t = 0; t < nthreads; ++t) L += Ls[t];                                                                   \
    if (grad) {                                                                                                      \
      std::fill(grad, grad + G2, T(0));                                                                              \
      for (int t = 0; t < nthreads; ++t)                                                                             \
        for (int64_t k = 0; k < G2; ++k) grad[k] += gs[t][k];                                                        \
    }                                                                                                                \
    return L;                                                                                                        \
  }
ORC_NCC(float, f32)
ORC_NCC(double, f64)

#define ORC_ENS(T, SUF)                                                                                              \
  int orc_run_ensemble_##SUF(const T* const* As, const T* const* Bs, int npairs, int64_t nr, int64_t nc,            \
                             const orc::Pass* passes, int npasses, const uint8_t* mask, double thr, int smoothing,  \
                             int nthreads, orc_result_##SUF* out) {                                                  \
    orc::Result<T> r;                                                                                                \
    if (orc::run_ensemble<T>(As, Bs, npairs, nr, nc, passes, npasses, mask, thr, smoothing != 0, nthreads, r) != 0) \
      return -1;                                                                                                     \
    out->ny = r.grid.ny;                                                                                             \
    out->nx = r.grid.nx;                                                                                             \
    if (out->x) std::copy(r.x.begin(), r.x.end(), out->x);                                                           \
    if (out->y) std::copy(r.y.begin(), r.y.end(), out->y);                                                           \
    if (out->u) std::copy(r.u.begin(), r.u.end(), out->u);                                                           \
    if (out->v) std::copy(r.v.begin(), r.v.end(), out->v);                                                           \
    if (out->peak_ratio) std::copy(r.ratio.begin(), r.ratio.end(), out->peak_ratio);                                 \
    if (out->moment) std::copy(r.moment.begin(), r.moment.end(), out->moment);                                       \
    if (out->unc_u) std::copy(r.unc_u.begin(), r.unc_u.end(), out->unc_u);                                           \
    if (out->unc_v) std::copy(r.unc_v.begin(), r.unc_v.end(), out->unc_v);                                           \
    if (out->outliers) std::copy(r.outliers.begin(), r.outliers.end(), out->outliers);                               \
    if (out->mask) std::copy(r.grid.gmask.begin(), r.grid.gmask.end(), out->mask);                                   \
    return 0;                                                                                                        \
  }
ORC_ENS(float, f32)
ORC_ENS(double, f64)

void orc_uq_offsets(int32_t* out /*40x2*/, int32_t* ring_start /*5*/) {
  orc::uq_init();
  for (int k = 0; k < 40; ++k) {
    out[2 * k] = orc::UQ_OFF[k][0];
    out[2 * k + 1] = orc::UQ_OFF[k][1];
  }
  for (int k = 0; k < 5; ++k) ring_start[k] = orc::UQ_RING_START[k];
}

}  // extern "C"
