// Fused window correlation for the planar WIDIM pass (sm_100a).
//
// One CTA holds WPC interrogation windows in shared memory and runs, per
// window, the whole of the reference's per-window chain
//   load_windows!  (src/correlators.jl:188-263: column-major mean, apodize)
//   FFT A, FFT B   (packed as one complex transform of A + iB)
//   spectrum!      (src/correlators.jl:266-279: conj(FA) FB, or filtered phase)
//   inverse FFT    (normalised by 1/N^2 like FFTW's inv(plan))
//   fftshift_abs!, overlap gain (src/correlators.jl:282-289, 338-339)
//   analyze_plane! (src/correlators.jl:459-468: regional-max or exclusion
//                   peaks with the tie rules of src/localmax.jl:3-19,
//                   gauss3/gauss9 in FP64, peak ratio, FP64 moment,
//                   gauss3-refined alternatives)
// writing the packed scalars of src/ka_backend.jl:497-506 straight into the
// vector grid. Nothing but images in and scalars out touches HBM.
//
// Shared-memory plane layout: element (p, q) (row p, column q) of window w
// lives at planes[w*N*LD + q*LD + p] with LD = N + 1, so a warp walking
// either axis with one line per lane is bank-conflict free.
//
// The 2-D transform runs each axis as an in-register radix-N1 pass and, for
// N > 32, a second radix-N2 pass (N = N1*N2). The forward transform leaves
// frequency k at position N2*(k % N1) + k / N1 along each axis; the spectrum
// step reads pairs (k, -k) from there and the inverse takes that order back
// to natural order, so no bit-reversal pass exists anywhere.
#include <math.h>
#include <stdint.h>

#include "hh_batch.h"
#include "hh_fft.cuh"
#include "hh_internal.h"

namespace hh {

// ---------------------------------------------------------------------------
// Global loads with L1 eviction hints. The shared-memory carveout leaves a
// small L1, and the window pixels, read once per window, would otherwise
// push out the small per-class tables (apodization, overlap gain, phase
// filter) that every window reads: the pixels stream past L1, the tables
// are kept. Inputs are read-only for the kernel's lifetime (.nc).
__device__ __forceinline__ float ld_stream(const float* p) {
  float v;
  asm("ld.global.nc.L1::no_allocate.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}
__device__ __forceinline__ uint8_t ld_stream(const uint8_t* p) {
  unsigned short v;
  asm("ld.global.nc.L1::no_allocate.u8 %0, [%1];" : "=h"(v) : "l"(p));
  return (uint8_t)v;
}
__device__ __forceinline__ float ld_keep(const float* p) {
  float v;
  asm("ld.global.nc.L1::evict_last.f32 %0, [%1];" : "=f"(v) : "l"(p));
  return v;
}

// Peak keys: larger key = larger value, ties broken by smaller column-major
// index (the reference's first-in-scan-order rule).
__device__ __forceinline__ uint32_t fkey(float v) {
  v = v + 0.0f;  // -0 -> +0 (they compare equal in the reference)
  uint32_t b = __float_as_uint(v);
  return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// Per-thread list of the best keys seen, descending, in KC register slots
// (KC >= K: 4 when the pass keeps at most 4 peaks, else KMAX).
template <int KC> struct TopK {
  uint32_t hi[KC];
  uint32_t lo[KC];
  int cnt;
  uint32_t thr;  // key of the K-th entry once the list is full, else 0
  __device__ __forceinline__ void init() {
    cnt = 0;
    thr = 0u;
#pragma unroll
    for (int m = 0; m < KC; ++m) hi[m] = lo[m] = 0u;
  }
  // the K-th (last retained) key, read with unrolled selects so the arrays
  // stay in registers for a run-time K
  __device__ __forceinline__ uint32_t last_hi(int K) const {
    uint32_t v = 0u;
#pragma unroll
    for (int m = 0; m < KC; ++m) v = (m == K - 1) ? hi[m] : v;
    return v;
  }
  __device__ __forceinline__ uint32_t last_lo(int K) const {
    uint32_t v = 0u;
#pragma unroll
    for (int m = 0; m < KC; ++m) v = (m == K - 1) ? lo[m] : v;
    return v;
  }
  // insert keeping (hi, lo) descending; K <= KC entries retained. Valid keys
  // are nonzero and empty slots hold 0, so the slots the new key beats are a
  // suffix of the first K: the first of them takes the new key, the others
  // their predecessor, and a key that beats none changes nothing. The
  // comparisons are independent of one another (no data-dependent indexing:
  // the list stays in registers).
  __device__ __forceinline__ void insert(uint32_t h, uint32_t l, int K) {
    bool b[KC];
#pragma unroll
    for (int m = 0; m < KC; ++m) b[m] = m < K && (h > hi[m] || (h == hi[m] && l > lo[m]));
#pragma unroll
    for (int m = KC - 1; m >= 0; --m) {
      const int q = m > 0 ? m - 1 : 0;
      const bool prev = m > 0 && b[q];
      const uint32_t ph = prev ? hi[q] : h, pl = prev ? lo[q] : l;
      hi[m] = b[m] ? ph : hi[m];
      lo[m] = b[m] ? pl : lo[m];
    }
    if (cnt < K) ++cnt;
    if (cnt == K) thr = last_hi(K);
  }
  __device__ __forceinline__ void pop() {
#pragma unroll
    for (int m = 0; m + 1 < KC; ++m) {
      hi[m] = hi[m + 1];
      lo[m] = lo[m + 1];
    }
    hi[KC - 1] = lo[KC - 1] = 0u;
    if (cnt > 0) --cnt;
    thr = 0u;
  }
};

// is_local_maximum (src/localmax.jl:3-19) on a column-major plane with
// leading dimension ldr: earlier neighbours (column-major) must be <=,
// later ones must be <; NaN is never a maximum.
__device__ __forceinline__ bool is_local_max(const float* R, int nr, int nc, int ldr, int r, int c, float I0) {
  if (isnan(I0)) return false;
  const int r0 = r > 0 ? r - 1 : 0, r1 = r < nr - 1 ? r + 1 : nr - 1;
  const int c0 = c > 0 ? c - 1 : 0, c1 = c < nc - 1 ? c + 1 : nc - 1;
  for (int jj = c0; jj <= c1; ++jj)
    for (int ii = r0; ii <= r1; ++ii) {
      if (ii == r && jj == c) continue;
      float In = R[jj * ldr + ii];
      bool earlier = (jj < c) || (jj == c && ii < r);
      if (earlier ? (In > I0) : (In >= I0)) return false;
    }
  return true;
}

// Lanes of the calling thread's group within its warp: the whole warp for
// groups of 32 threads or more, else the aligned block of `count` lanes
// (count a power of two below 32: two or more groups share a warp).
__device__ __forceinline__ unsigned grp_mask(int count) {
  return count >= 32 ? 0xffffffffu : (((1u << count) - 1u) << ((threadIdx.x & 31) & ~(count - 1)));
}

// Barrier of one thread group: lanes of a warp (count <= 32), the whole CTA
// (bar 0), or the named barrier `bar` shared by `count` threads (whole warps).
__device__ __forceinline__ void grp_sync(int bar, int count) {
  if (count <= 32) __syncwarp(grp_mask(count));
  else if (bar == 0) __syncthreads();
  else asm volatile("bar.sync %0, %1;" ::"r"(bar), "r"(count) : "memory");
}

// Group-wide argmax of (hi, lo) keys. Every thread of the group calls it (it
// synchronises the group); each group has its own reduction slots.
__device__ __forceinline__ void group_argmax(uint32_t hi, uint32_t lo, uint32_t* red, int gwarp, int gsize,
                                             uint32_t& whi, uint32_t& wlo, int bar) {
  const int lane = threadIdx.x & 31, nwarps = gsize >> 5;
  const unsigned m = grp_mask(gsize);
  uint32_t mhi = __reduce_max_sync(m, hi);
  uint32_t mlo = __reduce_max_sync(m, hi == mhi ? lo : 0u);
  if (nwarps <= 1) {  // one warp or part of one: the shuffle reduction is the answer
    whi = mhi;
    wlo = mlo;
    return;
  }
  if (lane == 0) {
    red[2 * gwarp] = mhi;
    red[2 * gwarp + 1] = mlo;
  }
  grp_sync(bar, nwarps * 32);
  whi = 0u;
  wlo = 0u;
  for (int w = 0; w < nwarps; ++w) {
    uint32_t h = red[2 * w], l = red[2 * w + 1];
    if (h > whi || (h == whi && l > wlo)) {
      whi = h;
      wlo = l;
    }
  }
  grp_sync(bar, nwarps * 32);
}

// The K best keys over the lists of the lanes in `mask` (a warp or the
// group's part of one), by K shuffle rounds (keys are unique, so exactly one
// lane pops each winner): lane m receives the m-th best in (mh, ml);
// returns how many exist (the same in every lane).
template <class TK>
__device__ __forceinline__ int warp_topk(TK& tk, int K, int lane, uint32_t& mh, uint32_t& ml, unsigned mask) {
  int n = 0;
  mh = ml = 0u;
  for (int round = 0; round < K; ++round) {
    const uint32_t h = tk.hi[0], l = tk.lo[0];  // empty slots hold 0
    const uint32_t wh = __reduce_max_sync(mask, h);
    if (wh == 0u) break;
    const uint32_t wl = __reduce_max_sync(mask, h == wh ? l : 0u);
    if (h == wh && l == wl) tk.pop();
    if (lane == round) {
      mh = wh;
      ml = wl;
    }
    n = round + 1;
  }
  return n;
}

// Plane access for the subpixel and moment arithmetic: value at (row i,
// column j), 0-based. PlaneAcc reads a column-major plane with leading
// dimension ld; RecAcc reads a w x w patch around a peak kept in a peak
// record (column-major, `stride` words between consecutive cells).
struct PlaneAcc {
  const float* p;
  int ld;
  __device__ __forceinline__ float operator()(int i, int j) const { return p[j * ld + i]; }
};
struct RecAcc {
  const float* p;
  int64_t stride;
  int i0, j0, w;  // patch origin and size
  __device__ __forceinline__ float operator()(int i, int j) const {
    // cells the arithmetic reads lie inside the patch; the clamp only keeps
    // every read inside the record
    const int di = min(max(i - i0, 0), w - 1), dj = min(max(j - j0, 0), w - 1);
    return __ldg(p + (int64_t)(dj * w + di) * stride);
  }
};

// subpixel_gauss3 (src/correlators.jl:499-520) with FP64 logarithms.
// (i, j) 0-based; returns 1-based refined (row, col).
// One axis: (ln Im - ln Ip) / (2 (ln Im - 2 ln I0 + ln Ip)), formed as
// ln(Im/Ip) / (2 ln(Im Ip / I0^2)) with the ratios in FP64 (exact products
// of floats, one rounding each): two logarithms instead of three.
__device__ __forceinline__ double gauss3_axis(float Im, float I0, float Ip) {
  if (!(Im > 0.f && I0 > 0.f && Ip > 0.f)) return 0.0;
  const double m = (double)Im, z = (double)I0, p = (double)Ip;
  const double den = log((m * p) / (z * z));
  return den != 0.0 ? log(m / p) / (2.0 * den) : 0.0;
}

template <class Acc> __device__ __forceinline__ void gauss3_fp64(const Acc& R, int nr, int nc, int i, int j, float* out) {
  double di = 0.0, dj = 0.0;
  const float I0 = R(i, j);
  if (i > 0 && i < nr - 1) di = gauss3_axis(R(i - 1, j), I0, R(i + 1, j));
  if (j > 0 && j < nc - 1) dj = gauss3_axis(R(i, j - 1), I0, R(i, j + 1));
  out[0] = (float)((double)(i + 1) + di);
  out[1] = (float)((double)(j + 1) + dj);
}

// subpixel_gauss9 (src/correlators.jl:534-564) with FP64 logarithms.
template <class Acc> __device__ __forceinline__ void gauss9_fp64(const Acc& R, int nr, int nc, int pr, int pc, float* out) {
  if (!(pr > 0 && pr < nr - 1 && pc > 0 && pc < nc - 1)) return gauss3_fp64(R, nr, nc, pr, pc, out);
  double sL = 0, sxL = 0, syL = 0, sxxL = 0, syyL = 0, sxyL = 0;
  for (int dj = -1; dj <= 1; ++dj)
    for (int di = -1; di <= 1; ++di) {
      float val = R(pr + di, pc + dj);
      if (!(val > 0.f)) return gauss3_fp64(R, nr, nc, pr, pc, out);
      double L = log((double)val);
      sL += L;
      sxL += dj * L;
      syL += di * L;
      sxxL += (dj * dj) * L;
      syyL += (di * di) * L;
      sxyL += (di * dj) * L;
    }
  double a1 = sxL / 6, a2 = syL / 6, a3 = sxxL / 2 - sL / 3, a4 = sxyL / 4, a5 = syyL / 2 - sL / 3;
  double D = 4 * a3 * a5 - a4 * a4;
  if (!(a3 < 0 && D > 0)) return gauss3_fp64(R, nr, nc, pr, pc, out);
  double dx = (a4 * a2 - 2 * a5 * a1) / D;
  double dy = (a4 * a1 - 2 * a3 * a2) / D;
  if (!(fabs(dx) <= 1 && fabs(dy) <= 1)) return gauss3_fp64(R, nr, nc, pr, pc, out);
  out[0] = (float)((double)(pr + 1) + dy);
  out[1] = (float)((double)(pc + 1) + dx);
}

// calculate_correlation_moment (src/quality.jl:49-74, neighbourhood 3):
// (c - pc)^2 in float like the Float32 reference, sums in FP64.
template <class Acc> __device__ __forceinline__ float moment_fp64(const Acc& R, int nr, int nc, float pr, float pc) {
  if (!(isfinite(pr) && isfinite(pc))) return __int_as_float(0x7fc00000);
  int r0 = (int)rintf(pr), c0 = (int)rintf(pc);  // 1-based, ties to even
  int rlo = max(1, r0 - 1), rhi = min(nr, r0 + 1), clo = max(1, c0 - 1), chi = min(nc, c0 + 1);
  if (rlo > rhi || clo > chi) return __int_as_float(0x7fc00000);
  // the 3 x 3 neighbourhood unrolled, clipped cells skipped: the loads issue
  // together and the sums keep the column-major order
  double sumC = 0, sdx = 0, sdy = 0;
#pragma unroll
  for (int dc = -1; dc <= 1; ++dc)
#pragma unroll
    for (int dr = -1; dr <= 1; ++dr) {
      const int c = c0 + dc, r = r0 + dr;
      if (c < clo || c > chi || r < rlo || r > rhi) continue;
      double w = fmax((double)R(r - 1, c - 1), 0.0);
      float dx = __fsub_rn((float)c, pc), dy = __fsub_rn((float)r, pr);
      sumC += w;
      sdx += (double)__fmul_rn(dx, dx) * w;
      sdy += (double)__fmul_rn(dy, dy) * w;
    }
  if (sumC < 1e-9) return __int_as_float(0x7fc00000);
  return (float)sqrt((sdx + sdy) / sumC);
}

struct PeakOut {
  float* du;
  float* dv;
  float* ratio;
  float* moment;
  float* alt_u;
  float* alt_v;
  int32_t nalt;
  int64_t G;
  float* packed;
  int32_t* locs;
};

// Peak record of one window (regional maxima), written by the correlation
// kernel in place of its epilogue and read by peak_epilogue_kernel: word w
// of job j at rec[w * njobs + j]. Words: 0 the number of peaks found (-1:
// window skipped), 1..K their values, then (row, col) per peak, then the
// 5 x 5 plane patch around the primary and a 3 x 3 patch around each
// alternative (column-major, cells outside the plane 0). A regional maximum
// is >= its neighbours, so its gauss3 offsets stay within 1/2 px and its
// gauss9 offsets within 1 px; the fits and the 3 x 3 moment around the
// refined primary therefore read only cells inside these patches.
__host__ __device__ constexpr int rec_words(int K) { return 17 + 12 * K; }
__device__ __forceinline__ int rec_patch(int K, int m) { return m == 0 ? 1 + 3 * K : 1 + 3 * K + 25 + 9 * (m - 1); }

// where the epilogue reads peak m's neighbourhood: the plane itself ...
struct PlaneSrc {
  const float* R;
  int ld;
  __device__ __forceinline__ PlaneAcc at(int, int, int) const { return PlaneAcc{R, ld}; }
};
// ... or the patches of a peak record
struct RecSrc {
  const float* rec;  // rec + job
  int64_t stride;
  int K;
  __device__ __forceinline__ RecAcc at(int m, int pr, int pc) const {
    const int h = m == 0 ? 2 : 1;
    return RecAcc{rec + (int64_t)rec_patch(K, m) * stride, stride, pr - h, pc - h, 2 * h + 1};
  }
};

// The per-window outputs from the peaks found (analyze_plane!'s tail,
// src/correlators.jl:459-468): the primary refined by the chosen subpixel
// method, displacement from the plane centre, peak ratio and moment; the
// alternatives 1..npeaks-1 refined by gauss3; 1-based peak locations.
template <class Src>
__device__ void peak_outputs(const Src& src, int nr, int nc, int K, int npeaks, int subpixel, int nfound,
                             const float* vals, const int* locs, int64_t grid_id, int64_t job, const PeakOut& o) {
  int found = 0;
  if (nfound > 0) {
    found = 1;
    while (found < nfound && vals[found] > 0.f) ++found;
  }
  const float NaN = __int_as_float(0x7fc00000);
  const int cr = nr / 2 + 1, cc = nc / 2 + 1;
  const int mmax = found < npeaks ? found : npeaks;  // peaks 1..mmax carry results
  float* pk = o.packed ? o.packed + job * (int64_t)(5 + 2 * (K - 1)) : nullptr;
  for (int m = 0; m < K; ++m) {
    float ref[2] = {NaN, NaN};
    if (m < found && (m == 0 || m < mmax)) {
      const int pr = locs[2 * m], pc = locs[2 * m + 1];
      const auto R = src.at(m, pr, pc);
      if (m == 0 && subpixel == 1) gauss9_fp64(R, nr, nc, pr, pc, ref);
      else if (m == 0 && subpixel == 3) {
        ref[0] = (float)(pr + 1);
        ref[1] = (float)(pc + 1);
      } else gauss3_fp64(R, nr, nc, pr, pc, ref);
    }
    const float d_col = ref[1] - (float)cc, d_row = ref[0] - (float)cr;
    if (m == 0) {
      float ratio = NaN, mom = NaN;
      if (found > 0) {
        const float v1 = vals[0];
        ratio = found >= 2 ? v1 / vals[1] : (v1 > 0.f ? INFINITY : NaN);
        mom = moment_fp64(src.at(0, locs[0], locs[1]), nr, nc, ref[0], ref[1]);
      }
      if (grid_id >= 0 && o.du) {
        o.du[grid_id] = d_col;
        o.dv[grid_id] = d_row;
        o.ratio[grid_id] = ratio;
        o.moment[grid_id] = mom;
      }
      if (pk) {
        pk[0] = d_col;
        pk[1] = d_row;
        pk[2] = ratio;
        pk[3] = mom;
        pk[4] = (float)found;
      }
    } else {
      // alternative peak m (0-based): result only while m < min(found, npeaks)
      const bool has = m < mmax;
      const float au = has ? d_col : NaN, av = has ? d_row : NaN;
      if (grid_id >= 0 && o.alt_u && m - 1 < o.nalt) {
        o.alt_u[grid_id + (int64_t)(m - 1) * o.G] = au;
        o.alt_v[grid_id + (int64_t)(m - 1) * o.G] = av;
      }
      if (pk) {
        pk[5 + (m - 1)] = au;
        pk[5 + (K - 1) + (m - 1)] = av;
      }
    }
    if (o.locs) {
      int32_t* lc = o.locs + job * (int64_t)(2 * K);
      lc[2 * m] = m < found ? locs[2 * m] + 1 : 0;
      lc[2 * m + 1] = m < found ? locs[2 * m + 1] + 1 : 0;
    }
  }
}

// Peak analysis of one plane by a group of threads (tid in [0, gsize)).
// Every thread of the group must call this (uniform K and finder), because
// the merge synchronises the group.
// Only the box rows [rlo, rhi] x columns [clo, chi] can hold positive
// values (outside it the overlap gain is zero, so R is exactly 0 there); the
// scans cover it, plus the last pixel, the only place outside where a zero
// can be a regional maximum (every other pixel has a later neighbour >= 0).
// A thread's share of the box scan, fixed for a launch (the box and the
// group size do not change), so the integer divisions are done once:
// column strips of rps rows, S strips per column; this thread's first
// strip is column c, rows [r0, r1).
struct ScanPlan {
  int rlo, rhi, clo, chi;
  int bw, S, rps;
  int c, r0, r1;
};
__device__ __forceinline__ ScanPlan scan_plan(int gtid, int gsize, int rlo, int rhi, int clo, int chi) {
  ScanPlan sp;
  sp.rlo = rlo;
  sp.rhi = rhi;
  sp.clo = clo;
  sp.chi = chi;
  sp.bw = chi - clo + 1;
  sp.S = gsize / sp.bw > 0 ? gsize / sp.bw : 1;  // row segments per column
  sp.rps = (rhi - rlo + 1 + sp.S - 1) / sp.S;
  sp.c = clo + gtid % sp.bw;
  sp.r0 = rlo + (gtid / sp.bw) * sp.rps;
  sp.r1 = min(rhi + 1, sp.r0 + sp.rps);
  return sp;
}

// One column strip of the regional-maximum scan (src/localmax.jl:3-19): the
// 3x3 neighbourhood rolls down the strip in registers, rows r - 1 (t) and r
// (m) of the left, centre and right columns (3 loads per pixel). Earlier
// neighbours in column-major order (the left column and the pixel above)
// must not exceed the value, later ones (the right column and the pixel
// below) must stay below it; fmaxf drops NaN neighbours, which never block
// in the reference either.
struct StripScan {
  const float* Cl;
  const float* Cc;
  const float* Cr;
  bool hl, hr;
  int c, r1;
  float lt, ct, rt, lm, cm, rm;
  __device__ __forceinline__ void init(const float* R, int ldr, int nc, int c_, int r0, int r1_) {
    const float NaNf = __int_as_float(0x7fc00000);
    c = c_;
    r1 = r1_;
    hl = c > 0;
    hr = c < nc - 1;
    Cc = R + c * ldr;
    Cl = hl ? Cc - ldr : Cc;
    Cr = hr ? Cc + ldr : Cc;
    lt = ct = rt = NaNf;
    if (r0 > 0) {
      lt = hl ? Cl[r0 - 1] : NaNf;
      ct = Cc[r0 - 1];
      rt = hr ? Cr[r0 - 1] : NaNf;
    }
    lm = hl ? Cl[r0] : NaNf;
    cm = Cc[r0];
    rm = hr ? Cr[r0] : NaNf;
  }
  // rows rb0 + 1 .. rb0 + SU of the three columns (NaN past the plane)
  template <int SU> __device__ __forceinline__ void load(int rb0, int nr, float* l, float* m, float* r) const {
    const float NaNf = __int_as_float(0x7fc00000);
#pragma unroll
    for (int u = 0; u < SU; ++u) {
      const int rr = rb0 + 1 + u;
      const bool ok = rr < nr;
      l[u] = ok && hl ? Cl[rr] : NaNf;
      m[u] = ok ? Cc[rr] : NaNf;
      r[u] = ok && hr ? Cr[rr] : NaNf;
    }
  }
  // tests row r (the centre value cm) and rolls down one row. Without TIES a
  // full list rejects a key equal to its K-th: the strips of a thread reach
  // the list in index order, so a later index cannot win the tie.
  template <bool TIES, class TK>
  __device__ __forceinline__ void step(int r, float lb, float cb, float rbv, int nr, TK& tk, int K) {
    const float v = cm;
    if (r < r1 && !isnan(v)) {
      const uint32_t h = fkey(v);
      if (TIES ? h >= tk.thr : h > tk.thr) {
        const float e = fmaxf(fmaxf(lt, lm), fmaxf(lb, ct));
        const float l = fmaxf(fmaxf(rt, rm), fmaxf(rbv, cb));
        if (!(e > v) && !(l >= v)) tk.insert(h, ~(uint32_t)(r + c * nr), K);
      }
    }
    lt = lm;
    ct = cm;
    rt = rm;
    lm = lb;
    cm = cb;
    rm = rbv;
  }
};

template <int KC, bool PAIRS>
__device__ __forceinline__ void analyze_body(const float* R, int nr, int nc, int ldr, int K, int npeaks, int finder,
                                             int subpixel, int gtid, int gsize, uint32_t* red, bool active,
                                             float* s_vals, int* s_locs, int64_t grid_id, int64_t job,
                                             const PeakOut* o, bool poison, int bar, const ScanPlan sp,
                                             float* rec, int64_t rec_stride) {
  const int rlo = sp.rlo, rhi = sp.rhi, clo = sp.clo, chi = sp.chi;
  // a poisoned plane (non-finite window data: the reference's plane is all
  // NaN there) yields no peak, so every output is NaN
  const bool scan = active && !poison;
  const int gwarp = gtid >> 5, nwarps = gsize >> 5;
  const int P = nr * nc;
  int nfound = 0;
  if (finder == 0) {
    // regional maxima (src/localmax.jl:3-19): each thread walks column strips
    // of the box top to bottom (StripScan), keeping its K best in registers
    TopK<KC> tk;
    tk.init();
    if (scan) {
      const int bw = sp.bw, S = sp.S, rps = sp.rps, ns = bw * S;
      // blocks of SU rows: the next SU rows of the three columns are loaded
      // together, so the loads of a block overlap instead of each row
      // waiting on its own
      constexpr int SU = 2;
      // strip `strip` of the box; an empty strip inside the box when it has
      // no rows (its addresses stay valid)
      auto strip_at = [&](int strip, int& c, int& r0, int& r1) {
        c = sp.c;
        r0 = sp.r0;
        r1 = sp.r1;
        if (strip != gtid) {  // a further strip: only when the box is wider than the group
          c = clo + strip % bw;
          r0 = rlo + (strip / bw) * rps;
          r1 = min(rhi + 1, r0 + rps);
        }
        if (strip >= ns || r0 >= r1) {
          c = clo;
          r0 = r1 = rlo;
        }
      };
      if (PAIRS && ns > gsize) {
        // Two strips per thread at a time, their rows interleaved, so the
        // two strips' loads and tests are independent chains. Their pixels
        // then reach the list out of index order, so a key equal to the
        // list's K-th goes to the insert's full (key, index) comparison.
        for (int sa = gtid; sa < ns; sa += 2 * gsize) {
          int ca, ra0, ra1, cb0, rb0, rb1;
          strip_at(sa, ca, ra0, ra1);
          strip_at(sa + gsize, cb0, rb0, rb1);
          StripScan A, B;
          A.init(R, ldr, nc, ca, ra0, ra1);
          B.init(R, ldr, nc, cb0, rb0, rb1);
          const int nrow = max(ra1 - ra0, rb1 - rb0);
          for (int rb = 0; rb < nrow; rb += SU) {
            float al[SU], ac[SU], ar[SU], bl[SU], bc[SU], br[SU];  // rows + 1 .. + SU
            A.load<SU>(ra0 + rb, nr, al, ac, ar);
            B.load<SU>(rb0 + rb, nr, bl, bc, br);
#pragma unroll
            for (int u = 0; u < SU; ++u) {
              A.template step<true>(ra0 + rb + u, al[u], ac[u], ar[u], nr, tk, K);
              B.template step<true>(rb0 + rb + u, bl[u], bc[u], br[u], nr, tk, K);
            }
          }
        }
      } else {
        for (int strip = gtid; strip < ns; strip += gsize) {
          int c, r0, r1;
          strip_at(strip, c, r0, r1);
          if (r0 >= r1) continue;
          StripScan A;
          A.init(R, ldr, nc, c, r0, r1);
          for (int rb0 = r0; rb0 < r1; rb0 += SU) {
            float lb[SU], cb[SU], rbv[SU];  // rows rb0 + 1 .. rb0 + SU
            A.load<SU>(rb0, nr, lb, cb, rbv);
#pragma unroll
            for (int u = 0; u < SU; ++u) A.template step<false>(rb0 + u, lb[u], cb[u], rbv[u], nr, tk, K);
          }
        }
      }
      if (gtid == 0 && (rhi < nr - 1 || chi < nc - 1)) {  // the last pixel, outside the box
        const int r = nr - 1, c = nc - 1;
        if (is_local_max(R, nr, nc, ldr, r, c, R[c * ldr + r])) tk.insert(fkey(R[c * ldr + r]), ~(uint32_t)(r + c * nr), K);
      }
    }
    // Merge: each warp takes its K best from its threads' lists by shuffle
    // rounds (lane m keeps the m-th); with several warps the warps' lists
    // meet in `red` behind one barrier and the first warp takes the group's
    // K best from them the same way.
    const int lane = gtid & 31;
    uint32_t mh = 0u, ml = 0u;
    int nw = warp_topk(tk, K, lane, mh, ml, grp_mask(gsize));
    if (nwarps > 1) {
      if (lane < K) {
        red[2 * (gwarp * K + lane)] = mh;
        red[2 * (gwarp * K + lane) + 1] = ml;
      }
      grp_sync(bar, gsize);
      if (gwarp == 0) {
        TopK<KC> tg;
        tg.init();
        for (int e = lane; e < nwarps * K; e += 32) {
          const uint32_t h = red[2 * e], l = red[2 * e + 1];
          if (h != 0u) tg.insert(h, l, K);
        }
        nw = warp_topk(tg, K, lane, mh, ml, 0xffffffffu);
      }
    }
    if (gwarp == 0) {
      nfound = nw;
      if (lane < nw) {
        const int lin = (int)(~ml);
        s_vals[lane] = R[(lin / nr) * ldr + (lin % nr)];
        s_locs[2 * lane] = lin % nr;
        s_locs[2 * lane + 1] = lin / nr;
      }
    }
  } else {
    // exclusion finder (src/correlators.jl:390-421): K scans, box +-2
    bool done = false;
    for (int round = 0; round < K; ++round) {  // every round runs: group_argmax synchronises the group
      // the box first; when its best is not positive the maximum can lie
      // outside it (a zero earlier in column-major order), so rescan all
      uint32_t whi = 0u, wlo = 0u;
      for (int pass = 0; pass < 2; ++pass) {
        const int bw = chi - clo + 1, bht = rhi - rlo + 1;
        const int n = pass == 0 ? bw * bht : P;
        uint32_t bh = 0u, bl = 0u;
        if (scan && !done) {
          for (int t = gtid; t < n; t += gsize) {
            const int r = pass == 0 ? rlo + t % bht : t % nr, c = pass == 0 ? clo + t / bht : t / nr;
            bool ex = false;
            for (int q = 0; q < nfound; ++q)
              if (abs(r - s_locs[2 * q]) <= 2 && abs(c - s_locs[2 * q + 1]) <= 2) { ex = true; break; }
            if (ex) continue;
            const float v = R[c * ldr + r];
            if (!(v > -INFINITY)) continue;  // NaN and -Inf never beat the initial -Inf
            const uint32_t h = fkey(v), l = ~(uint32_t)(r + c * nr);
            if (h > bh || (h == bh && l > bl)) { bh = h; bl = l; }
          }
        }
        group_argmax(bh, bl, red, gwarp, gsize, whi, wlo, bar);
        if (whi > fkey(0.f) || (rlo == 0 && clo == 0 && rhi == nr - 1 && chi == nc - 1)) break;  // positive, or the box is the plane
      }
      if (!done && whi != 0u) {
        const int lin = (int)(~wlo);
        const float best = R[(lin / nr) * ldr + (lin % nr)];
        if (nfound > 0 && !(best > 0.f)) {
          done = true;  // secondary peaks must be positive
        } else {
          if (gtid == 0) {
            s_vals[nfound] = best;
            s_locs[2 * nfound] = lin % nr;
            s_locs[2 * nfound + 1] = lin / nr;
          }
          ++nfound;
        }
      } else {
        done = true;
      }
      grp_sync(bar, gsize);  // s_locs visible to the next round's exclusion test
    }
  }
  // Epilogue on the group's first warp, after the last merge step wrote
  // s_vals / s_locs: with a record buffer (regional maxima) the lanes of the
  // peaks store the peak record and peak_epilogue_kernel forms the outputs;
  // otherwise lane 0 forms them here.
  if (gtid >= 32 || !active) return;
  __syncwarp(grp_mask(gsize));
  if (rec && finder == 0) {
    // the record's words spread over the lanes (a few each), so its shared
    // loads and global stores overlap instead of one lane walking the patches
    const int lanes = gsize < 32 ? gsize : 32, base0 = 1 + 3 * K, nw = rec_words(K);
    for (int wd = gtid; wd < nw; wd += lanes) {
      float val = 0.f;
      if (wd == 0) {
        val = __int_as_float(nfound);
      } else if (wd <= K) {
        val = wd - 1 < nfound ? s_vals[wd - 1] : 0.f;
      } else if (wd < base0) {
        const int m = (wd - 1 - K) >> 1;
        val = m < nfound ? __int_as_float(s_locs[wd - 1 - K]) : 0.f;
      } else {
        const int e = wd - base0;  // primary: 25 cells; alternative m: 9 cells
        const int m = e < 25 ? 0 : 1 + (e - 25) / 9, cell = e < 25 ? e : (e - 25) % 9;
        const int h = m == 0 ? 2 : 1, w = 2 * h + 1;
        if (m < nfound) {
          const int i = s_locs[2 * m] + cell % w - h, j = s_locs[2 * m + 1] + cell / w - h;
          val = (i >= 0 && i < nr && j >= 0 && j < nc) ? R[j * ldr + i] : 0.f;
        }
      }
      rec[(int64_t)wd * rec_stride + job] = val;
    }
    return;
  }
  if (gtid == 0) peak_outputs(PlaneSrc{R, ldr}, nr, nc, K, npeaks, subpixel, nfound, s_vals, s_locs, grid_id, job, *o);
}

// The analysis as a call: small planes keep it out of line (the kernel's
// transform stages then keep their registers); large planes inline it.
// PAIRS: walk two column strips per thread at a time, for groups with more
// strips than threads (half-warp groups of 32-point planes); elsewhere the
// second strip's registers would only add spills.
template <bool PAIRS = false>
__device__ __noinline__ void analyze_group(const float* R, int nr, int nc, int ldr, int K, int npeaks, int finder,
                                           int subpixel, int gtid, int gsize, uint32_t* red, bool active,
                                           float* s_vals, int* s_locs, int64_t grid_id, int64_t job,
                                           const PeakOut* o, bool poison, int bar, const ScanPlan sp,
                                           float* rec, int64_t rec_stride) {
  if (K <= 4)
    analyze_body<4, PAIRS>(R, nr, nc, ldr, K, npeaks, finder, subpixel, gtid, gsize, red, active, s_vals, s_locs, grid_id, job,
                    o, poison, bar, sp, rec, rec_stride);
  else
    analyze_body<KMAX, PAIRS>(R, nr, nc, ldr, K, npeaks, finder, subpixel, gtid, gsize, red, active, s_vals, s_locs, grid_id,
                       job, o, poison, bar, sp, rec, rec_stride);
}

// S(k) = conj(FA(k)) FB(k) of the packed transform Z = F(a + i b), from
// X = Z(k) and Zm = Z(-k): FA = (X + conj(Zm))/2, FB = (X - conj(Zm))/(2i)
// (spectrum!, src/correlators.jl:266-279); the phase method divides by
// |S| + eps(Float32) and applies the spectral filter weight wk.
__device__ __forceinline__ float2 cross_spectrum(float2 X, float2 Zm, int method, float wk) {
  const float2 Y = make_float2(Zm.x, -Zm.y);
  const float Ar = 0.5f * (X.x + Y.x), Ai = 0.5f * (X.y + Y.y);
  const float Br = 0.5f * (X.y - Y.y), Bi = -0.5f * (X.x - Y.x);
  float2 S = cmul(make_float2(Ar, -Ai), make_float2(Br, Bi));
  if (method == 1) {
    const float den = hypotf(S.x, S.y) + 1.1920929e-7f;
    S = make_float2((wk * S.x) / den, (wk * S.y) / den);
  }
  return S;
}

// the general-shape kernel (any FFT lengths, rectangular windows, planes
// larger than a CTA's shared memory)
#include "hh_corr_general.cuh"

// ---------------------------------------------------------------------------
// W is the extent of the data: the window, or with SRCH the frame-B search
// area that holds the (runtime) frame-A window at its centre. VAR selects the
// CTA shape (windows per CTA, threads per window) and register budget (CTAs
// per SM the registers are sized for) and FFT split among the five the
// autotuner times: 0 the default shape and budget, 1 the alternative shape,
// 2 the default shape with one CTA per SM more in the budget (fewer
// registers, more warps), 3 the default shape with one CTA less (more
// registers, no spills) -- or, where the default budget is one CTA, the
// alternative shape with one CTA more. Variants 0-3 compute the same
// arithmetic on another thread mapping or register allocation, so their
// results are identical. Variant 4 splits each axis's DFT differently
// (AxisSplitAlt), so its planes differ from variant 0's by rounding.
template <int N, int W, bool SRCH = false, int VAR = 0> struct CorrCfg {
  // variant 4: the alternative FFT split (AxisSplitAlt) in the default shape and budget
  static constexpr bool ALT = VAR == 4;
  static constexpr int N1 = ALT ? AxisSplitAlt<N>::N1 : AxisSplit<N>::N1;
  static constexpr int N2 = ALT ? AxisSplitAlt<N>::N2 : AxisSplit<N>::N2;
  // budget of the default shape; shape of this variant (0 default, 1 alternative)
  static constexpr int MINB0 = (N == 32 && W == 16) ? 3 : (N <= 48 ? 4 : (N <= 64 ? 3 : (N <= 96 ? 2 : 1)));
  static constexpr int SH = (VAR == 1 || (VAR == 3 && MINB0 == 1)) ? 1 : 0;
  // 16 x 16 windows padded to 32: every stage of the plane has at most 16
  // lines (16 data columns, 16 canonical column items, 16 row pairs), so
  // half a warp serves a window and each warp carries two
  static constexpr bool HALF = SH == 0 && N == 32 && W == 16;
  // alternatives: N <= 32 one window per warp in CTAs of 4 (half-warp
  // windows) or 8 warps; N = 48 a 3-CTA register budget; N = 64 one window
  // per 256-thread CTA; N = 96 512 threads and N = 128 256 threads per window
  static constexpr int WPC = SH == 0 ? (HALF ? 8 : (N <= 32 ? 4 : (N <= 64 ? 2 : 1)))  // windows per CTA
                                     : (N <= 32 ? (N == 32 && W == 16 ? 4 : 8) : (N <= 48 ? 2 : 1));
  static constexpr int NT = SH == 0 ? (N <= 48 ? 128 : (N <= 96 ? 256 : 512))
                                    : (N <= 32 ? (N == 32 && W == 16 ? 128 : 256)
                                               : (N <= 48 ? 128 : (N <= 64 ? 256 : (N <= 96 ? 512 : 256))));
  static constexpr int G = NT / WPC;  // threads per window
  // CTAs per SM the register budget is sized for
  static constexpr int MINB_SH = SH == 0 ? MINB0
                                         : (N <= 32 ? (N == 32 && W == 16 ? 4 : 2) : (N <= 48 ? 3 : (N <= 64 ? 3 : 1)));
  static constexpr int MINB = VAR == 2 ? MINB0 + 1
                                       : (VAR == 3 ? (MINB0 > 1 ? MINB0 - 1 : MINB_SH + 1) : MINB_SH);
  // the peak analysis inline (one window per CTA: its latency is the CTA's)
  static constexpr bool INLINE_ANALYSIS = N >= 96;
  // Canonical column c sits at storage column N2 (c % N1) + c / N1, and with
  // LD = N + 1 a 64-bit element's bank pair is (column + row) mod 16, so with
  // N2 = 8 consecutive canonical columns (8 storage columns apart) share two
  // bank pairs. The first inverse pass then walks c = N1 u + v with u
  // fastest (a model of the pass's addresses: 1088 wavefronts instead of
  // 2112 for 520 ideal at N = 128, 624 instead of 912 for 296 at N = 96).
  static constexpr bool SPREAD7 = N2 == 8;
  // The spectrum is Hermitian, so the inverse transforms only the N/2 + 1
  // canonical columns along p and then rows p and p + N/2 together along q
  // (their outputs are real: one lands in the real part, one in the
  // imaginary part). Every window is transformed on its own.
  static constexpr int NC = N / 2 + 1;
  static constexpr int IPT = ((N / 2) * N2 + G - 1) / G;  // final inverse items per thread
  static constexpr int LD = N + 1;    // complex plane leading dimension (float2)
  static constexpr int LDR = N + 1;   // real plane leading dimension (float), overlays the complex plane
  static constexpr bool PADDED = (W * 2 == N);
  static constexpr int NZ1 = PADDED ? (W / N2) : N1;  // nonzero inputs of a forward pass-A line

  static constexpr int EPT = (W * W + G - 1) / G;             // window pixels per thread
  static constexpr int NPART = SRCH ? 4 : 3;  // FP64 partial sums per warp: A, B, count (and count of B)
  // plane stride in float2; the two windows of a half-warp pair start 16
  // banks apart, so their 32-bit plane accesses (peak scan, real-plane
  // writes) do not meet in one bank
  static constexpr int PS = N * LD + (HALF ? 8 : 0);
  static constexpr size_t PLANE_B = (size_t)PS * sizeof(float2);
  static constexpr size_t BASE_B = WPC * PLANE_B + WPC * (G / 32) * NPART * sizeof(double) + N * sizeof(float2) +
                                   WPC * (G / 32) * 2 * KMAX * sizeof(uint32_t) +
                                   WPC * (KMAX * sizeof(float) + 2 * KMAX * sizeof(int)) + 3 * N * sizeof(int) + 64;
  // CTAs per SM that shared memory allows (228 KB per SM, 1 KB of it
  // reserved per CTA), capped by the register budget
  static constexpr int occ(size_t b) {
    return (int)((228 * 1024) / (b + 1024)) < MINB ? (int)((228 * 1024) / (b + 1024)) : MINB;
  }
  // The overlap gain table (N x N) is read by every window; from global
  // memory its L1 lines are flushed by the window pixels (it took a third of
  // the last inverse pass at 32 points, half of it at 128). It goes to shared
  // memory where that costs no CTA per SM: every size but 64 points. (The
  // apodization window in shared memory as well was no faster.)
  // Where the full table would cost a CTA (64 points), its quarter does not:
  // the gain of a symmetric apodization depends only on |lag| along each
  // axis, and the table builder appends the quarter when that holds exactly.
  static constexpr size_t GAIN_B = (size_t)N * N * sizeof(float);
  static constexpr size_t GQ_B = (size_t)(N / 2 + 1) * (N / 2 + 1) * sizeof(float);
  static constexpr bool GSM = occ(BASE_B + GAIN_B) >= occ(BASE_B);
  static constexpr bool QSM = !GSM && occ(BASE_B + GQ_B) >= occ(BASE_B);
  static constexpr size_t smem() { return BASE_B + (GSM ? GAIN_B : (QSM ? GQ_B : 0)); }
  static_assert(W == N || 2 * W == N, "window must equal the FFT size or half of it");
  static_assert((G >= 32 && G % 32 == 0) || G == 16, "a window group is whole warps or half a warp");
  static_assert(N * LDR <= 2 * N * LD, "real plane must fit in the complex plane");
};

template <int N, int W, bool SRCH, int VAR>
__global__ void __launch_bounds__(CorrCfg<N, W, SRCH, VAR>::NT, CorrCfg<N, W, SRCH, VAR>::MINB)
    correlate_kernel(const CorrArgs a) {
  using C = CorrCfg<N, W, SRCH, VAR>;
  constexpr int WPC = C::WPC, NT = C::NT, LD = C::LD, LDR = C::LDR, N1 = C::N1, N2 = C::N2, IPT = C::IPT;
  constexpr int G = C::G, EPT = C::EPT, NC = C::NC, H = N / 2;
  constexpr int PS = C::PS;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* planes = reinterpret_cast<float2*>(smem_raw);
  double* s_part = reinterpret_cast<double*>(smem_raw + WPC * C::PLANE_B);  // NPART per warp
  float2* tw = reinterpret_cast<float2*>(s_part + WPC * (G / 32) * C::NPART);
  uint32_t* red = reinterpret_cast<uint32_t*>(tw + N);
  float* s_vals = reinterpret_cast<float*>(red + WPC * (G / 32) * 2 * KMAX);
  int* s_locs = reinterpret_cast<int*>(s_vals + WPC * KMAX);
  // per-axis storage tables (N2 > 1): frequency of storage slot a, storage
  // slot of the negated frequency, canonical storage columns kq = 0..N/2
  int* s_freq = reinterpret_cast<int*>(s_locs + WPC * 2 * KMAX);
  int* s_neg = s_freq + N;
  int* s_canon = s_neg + N;
  float* s_gain = reinterpret_cast<float*>(s_canon + N);  // N x N when C::GSM

  const int tid = threadIdx.x;
  const int K = a.npeaks > 2 ? a.npeaks : 2;
  if (C::GSM && a.gain)
    for (int m = tid; m < N * N; m += NT) s_gain[m] = a.gain[m];
  // the quarter table (word N^2 of the gain buffer says whether it follows)
  const bool gq = C::QSM && a.gain && a.gain[N * N] != 0.f;
  if (gq)
    for (int m = tid; m < (N / 2 + 1) * (N / 2 + 1); m += NT) s_gain[m] = a.gain[N * N + 1 + m];

  if (N2 > 1) {
    for (int m = tid; m < N; m += NT) {
      double sn, cs;
      sincospi(-2.0 * (double)m / (double)N, &sn, &cs);
      tw[m] = make_float2((float)cs, (float)sn);  // W_N^m = exp(-2 pi i m / N)
    }
    for (int q = tid; q < N; q += NT) {
      const int k = q / N2 + N1 * (q % N2);  // storage slot q holds frequency k
      const int m = (N - k) % N;
      s_freq[q] = k;
      s_neg[q] = N2 * (m % N1) + m / N1;
      if (q <= N / 2) s_canon[q] = N2 * (q % N1) + q / N1;
    }
  }
  __syncthreads();  // the only CTA-wide barrier: from here on the window groups run independently

  // Thread group w (G threads, named barrier w + 1) owns plane w and walks
  // its own sequence of jobs; a group waits only for itself.
  const int w = tid / G, gt = tid % G, lane = tid & 31, gw = gt >> 5;
  const int bar = WPC == 1 ? 0 : w + 1;
  float2* P = planes + w * PS;
  float* Rw = reinterpret_cast<float*>(P);  // real plane, overlays the complex one after stage 8
  double* part = s_part + w * (G / 32) * C::NPART;
  const float scale = 1.0f / (float)(N * N);
  // fftshifted rows / columns that can hold a nonzero correlation value (the
  // support of the overlap gain; the whole plane without padding)
  const int blo = a.box_hi > 0 ? a.box_lo : 0, bhi = a.box_hi > 0 ? a.box_hi : N - 1;
  const ScanPlan sp = scan_plan(tid % G, G, blo, bhi, blo, bhi);
  PeakOut po{a.du, a.dv, a.ratio, a.moment, a.alt_u, a.alt_v, a.nalt, a.G, a.packed, a.locs};

  for (int64_t job = (int64_t)blockIdx.x * WPC + w; job < a.njobs; job += (int64_t)gridDim.x * WPC) {
    // ---- the window's source (every thread of the group reads the same
    //      descriptor words; they are broadcast from L1)
    int rs, cs;
    const float* A = a.A;
    const float* B = a.B;
    const uint8_t* M = a.mask;
    int64_t ld = a.ld, gid;
    PeakOut pw = po;
    if (a.bp) {
      const int p = a.jobs[4 * job];
      const BPair& b = a.bp[p];
      const int gij = a.jobs[4 * job + 1];
      const int64_t cell = (int64_t)(gij & 0xFFFF) + (int64_t)(gij >> 16) * b.ny;
      // pairs that converged or have no further sweep, and masked cells, are skipped
      if (!bp_live(b, a.it, a.done, p) || (b.gmask && b.gmask[cell])) {
        if (a.rec && a.finder == 0 && gt == 0) a.rec[job] = __int_as_float(-1);  // no record for the epilogue
        continue;
      }
      rs = a.jobs[4 * job + 2];
      cs = a.jobs[4 * job + 3];
      const bool warped = a.it > 1 || b.has_pred0;
      A = warped ? b.warpA : b.A;
      B = warped ? b.warpB : b.B;
      M = b.mask;
      ld = b.nr;
      gid = b.goff + cell;
      pw.G = (int64_t)b.ny * b.nx;
      pw.nalt = b.nalt;
      pw.alt_u = a.alt_u ? a.alt_u + b.aoff - b.goff : nullptr;  // indexed by gid + m*G
      pw.alt_v = a.alt_v ? a.alt_v + b.aoff - b.goff : nullptr;
    } else {
      rs = a.jobs[4 * job + 2];
      cs = a.jobs[4 * job + 3];
      gid = (int64_t)a.jobs[4 * job] + (int64_t)a.jobs[4 * job + 1] * a.ny;
    }
    // ---- stages 1-3: the group loads the window's pixels (coalesced down
    //      the columns), reduces the window means in FP64, and stores
    //      apod * (x - mean) into the plane; masked pixels enter as zero and
    //      leave the mean (load_windows!, src/correlators.jl:188-263). The
    //      mean is the exact sum over n rounded once, where the reference
    //      folds in Float32 left to right; the two differ by a few ulp.
    bool bad;
    if constexpr (SRCH) {
      // enlarged search area (load_windows!, src/correlators.jl:229-262):
      // the W x W frame-B area starts (W - win) / 2 before the window on
      // both axes; frame A enters only inside the centred window, apodized
      // and less its own mean, frame B everywhere, less its mean, without
      // apodization; a masked pixel is zero in both and leaves both means
      const int wa = a.win, oa = (W - wa) / 2;
      const int64_t r0 = rs - oa, c0 = cs - oa;
      float2 z[EPT];
      bool mk[EPT];
      double sa = 0.0, sb = 0.0, na = 0.0, nb = 0.0;
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int e = gt + i * G;
        z[i] = make_float2(0.f, 0.f);
        mk[i] = true;
        if (e < W * W) {
          const int p = e % W, q = e / W;
          const bool ina = (unsigned)(p - oa) < (unsigned)wa && (unsigned)(q - oa) < (unsigned)wa;
          const int64_t off = (r0 + p) + (c0 + q) * ld;
          z[i] = make_float2(ina ? ld_stream(A + off) : 0.f, ld_stream(B + off));
          mk[i] = M ? ld_stream(M + off) != 0 : false;
          if (!mk[i]) {
            sb += (double)z[i].y;
            nb += 1.0;
            if (ina) {
              sa += (double)z[i].x;
              na += 1.0;
            }
          }
        }
      }
      const unsigned gm = grp_mask(G);
#pragma unroll
      for (int o = (G < 32 ? G : 32) / 2; o > 0; o >>= 1) {
        sa += __shfl_xor_sync(gm, sa, o);
        sb += __shfl_xor_sync(gm, sb, o);
        na += __shfl_xor_sync(gm, na, o);
        nb += __shfl_xor_sync(gm, nb, o);
      }
      double ta = sa, tb = sb, tna = na, tnb = nb;
      if (G > 32) {
        if (lane == 0) {
          part[4 * gw] = sa;
          part[4 * gw + 1] = sb;
          part[4 * gw + 2] = na;
          part[4 * gw + 3] = nb;
        }
        grp_sync(bar, G);
        ta = tb = tna = tnb = 0.0;
        for (int k = 0; k < G / 32; ++k) {
          ta += part[4 * k];
          tb += part[4 * k + 1];
          tna += part[4 * k + 2];
          tnb += part[4 * k + 3];
        }
      }
      const float ma = tna > 0 ? (float)(ta / tna) : 0.f, mb = tnb > 0 ? (float)(tb / tnb) : 0.f;
      bad = !(isfinite(ta) && isfinite(tb));
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int e = gt + i * G;
        if (e < W * W) {
          const int p = e % W, q = e / W;
          const bool ina = (unsigned)(p - oa) < (unsigned)wa && (unsigned)(q - oa) < (unsigned)wa;
          float2 v = make_float2(0.f, 0.f);
          if (!(mk[i] || bad)) {
            v.y = z[i].y - mb;
            if (ina) v.x = ld_keep(a.apod + (p - oa) + (q - oa) * wa) * (z[i].x - ma);
          }
          P[q * LD + p] = v;
        }
      }
    } else {
      float2 z[EPT];
      bool mk[EPT];
      double sa = 0.0, sb = 0.0, cnt = 0.0;
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int e = gt + i * G;
        z[i] = make_float2(0.f, 0.f);
        mk[i] = true;
        if (e < W * W) {
          const int p = e % W, q = e / W;
          const int64_t off = (int64_t)(rs + p) + (int64_t)(cs + q) * ld;
          z[i] = make_float2(ld_stream(A + off), ld_stream(B + off));
          mk[i] = M ? ld_stream(M + off) != 0 : false;
          if (!mk[i]) {
            sa += (double)z[i].x;
            sb += (double)z[i].y;
            cnt += 1.0;
          }
        }
      }
      const unsigned gm = grp_mask(G);
#pragma unroll
      for (int o = (G < 32 ? G : 32) / 2; o > 0; o >>= 1) {
        sa += __shfl_xor_sync(gm, sa, o);
        sb += __shfl_xor_sync(gm, sb, o);
        cnt += __shfl_xor_sync(gm, cnt, o);
      }
      double ta = sa, tb = sb, tn = cnt;
      if (G > 32) {
        if (lane == 0) {
          part[3 * gw] = sa;
          part[3 * gw + 1] = sb;
          part[3 * gw + 2] = cnt;
        }
        grp_sync(bar, G);
        ta = tb = tn = 0.0;
        for (int k = 0; k < G / 32; ++k) {
          ta += part[3 * k];
          tb += part[3 * k + 1];
          tn += part[3 * k + 2];
        }
      }
      const float ma = tn > 0 ? (float)(ta / tn) : 0.f, mb = tn > 0 ? (float)(tb / tn) : 0.f;
      bad = !(isfinite(ta) && isfinite(tb));  // the window holds NaN or Inf
#pragma unroll
      for (int i = 0; i < EPT; ++i) {
        const int e = gt + i * G;
        if (e < W * W) {
          const int p = e % W, q = e / W;
          const float ap = ld_keep(a.apod + e);
          P[q * LD + p] = (mk[i] || bad) ? make_float2(0.f, 0.f) : make_float2(ap * (z[i].x - ma), ap * (z[i].y - mb));
        }
      }
    }
    grp_sync(bar, G);

    // ---- stage 4: forward transform along p (only the W data columns)
    for (int it = gt; it < W * N2; it += G) {
      const int q = it % W, n2 = it / W;
      float2* L = P + q * LD;
      float2 x[N1];
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) x[n1] = n1 < C::NZ1 ? L[N2 * n1 + n2] : make_float2(0.f, 0.f);
      RDFT<N1, false>::run(x, C::NZ1);
      if (N2 > 1) {
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) x[k1] = cmul(x[k1], tw[(n2 * k1) % N]);
      }
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) L[N2 * k1 + n2] = x[k1];
    }
    if (N2 > 1) {
      grp_sync(bar, G);
      for (int it = gt; it < W * N1; it += G) {
        const int q = it % W, k1 = it / W;
        float2* L = P + q * LD + N2 * k1;
        float2 x[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) x[n2] = L[n2];
        RDFT<N2, false>::run(x, N2);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) L[k2] = x[k2];
      }
    }
    grp_sync(bar, G);
    // ---- stage 5: forward transform along q for every row p
    for (int it = gt; it < N * N2; it += G) {
      const int p = it % N, n2 = it / N;
      float2* L = P + p;
      float2 x[N1];
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) x[n1] = n1 < C::NZ1 ? L[(N2 * n1 + n2) * LD] : make_float2(0.f, 0.f);
      RDFT<N1, false>::run(x, C::NZ1);
      if (N2 > 1) {
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) x[k1] = cmul(x[k1], tw[(n2 * k1) % N]);
      }
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) L[(N2 * k1 + n2) * LD] = x[k1];
    }
    if (N2 > 1) {
      grp_sync(bar, G);
      for (int it = gt; it < N * N1; it += G) {
        const int p = it % N, k1 = it / N;
        float2* L = P + p + (N2 * k1) * LD;
        float2 x[N2];
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) x[n2] = L[n2 * LD];
        RDFT<N2, false>::run(x, N2);
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) L[k2 * LD] = x[k2];
      }
    }
    grp_sync(bar, G);
    // ---- stages 6-7: cross-power (or filtered phase) spectrum over Hermitian
    //      pairs (k, -k) and the inverse along p, on the canonical columns
    //      kq = 0..N/2 only (frequencies in storage order for N2 > 1, natural
    //      order otherwise); the conjugate column -kq is then filled in as
    //      conj of column kq. (i) The two self-paired columns (kq = 0, N/2)
    //      pair rows within the column: their spectrum is formed first, in
    //      place (for N <= 32 every canonical column is done here: folding
    //      the spectrum into the single-pass inverse costs more registers
    //      than the separate pass costs time).
    if constexpr (N2 == 1 && G <= N && N % G == 0) {
      // each thread owns rows ap = gt + j G (j < N / G) of every canonical
      // column; the columns are unrolled, so every address is the row's base
      // plus a constant, and CB columns' operands are loaded before any of
      // their results is stored (no item reads a cell another item writes:
      // column -c is read only, and a self-paired column's rows ap and -ap
      // belong to one item)
      constexpr int RPT = G <= N ? N / G : 1, CB = RPT >= 2 ? 2 : 4;
      int ra[RPT], rb[RPT];
#pragma unroll
      for (int j = 0; j < RPT; ++j) {
        ra[j] = gt + j * G;
        rb[j] = (N - ra[j]) % N;
      }
#pragma unroll
      for (int c0 = 0; c0 < NC; c0 += CB) {
        float2 xa[CB][RPT], xb[CB][RPT];
        float wk[CB][RPT];
#pragma unroll
        for (int u = 0; u < CB; ++u) {
          const int c = c0 + u, cb = (N - c) % N;
          if (c < NC) {
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
              if (c == cb && ra[j] > rb[j]) continue;  // a self pair is done by its upper row
              xa[u][j] = P[c * LD + ra[j]];
              xb[u][j] = P[cb * LD + rb[j]];
              wk[u][j] = a.method == 1 ? ld_keep(a.phasew + c * N + ra[j]) : 1.f;
            }
          }
        }
#pragma unroll
        for (int u = 0; u < CB; ++u) {
          const int c = c0 + u, cb = (N - c) % N;
          if (c < NC) {
#pragma unroll
            for (int j = 0; j < RPT; ++j) {
              if (c == cb && ra[j] > rb[j]) continue;
              const float2 S = cross_spectrum(xa[u][j], xb[u][j], a.method, wk[u][j]);
              P[c * LD + ra[j]] = S;
              if (c == cb) P[c * LD + rb[j]] = make_float2(S.x, -S.y);
            }
          }
        }
      }
    } else if constexpr (N2 == 1) {
      // items (row ap, canonical column c) in batches of SB per thread: the
      // batch's operands are loaded before any of its results is stored (no
      // item reads a cell another item writes: column -c is read only, and a
      // self-paired column's rows ap and -ap belong to one item)
      constexpr int SB = 4, NIT = NC * N;  // (batches of 8 were slower: registers)
#pragma unroll 1
      for (int it0 = gt; it0 < NIT; it0 += SB * G) {
        float2 xa[SB], xb[SB];
        int ia[SB], ib[SB];
        bool on[SB], self[SB];
        float wk[SB];
#pragma unroll
        for (int u = 0; u < SB; ++u) {
          const int it = it0 + u * G;
          const int ap = it % N, c = it / N, bq = (N - c) % N, bp = (N - ap) % N;
          self[u] = c == bq;
          on[u] = it < NIT && !(self[u] && ap > bp);  // a self pair is done by its upper row
          ia[u] = c * LD + ap;
          ib[u] = bq * LD + bp;
          wk[u] = on[u] && a.method == 1 ? ld_keep(a.phasew + c * N + ap) : 1.f;
          if (on[u]) {
            xa[u] = P[ia[u]];
            xb[u] = P[ib[u]];
          }
        }
#pragma unroll
        for (int u = 0; u < SB; ++u)
          if (on[u]) {
            const float2 S = cross_spectrum(xa[u], xb[u], a.method, wk[u]);
            P[ia[u]] = S;
            if (self[u]) P[ib[u]] = make_float2(S.x, -S.y);
          }
      }
    } else {
      // the two self-paired columns kq = 0 and N/2 (storage order)
#pragma unroll 1
      for (int it = gt; it < 2 * N; it += G) {
        const int ap = it % N, c = (it / N) * H;
        const int aq = s_canon[c], bp = s_neg[ap], kp = s_freq[ap];
        if (ap > bp) continue;  // its partner row does this pair
        const float wk = a.method == 1 ? ld_keep(a.phasew + c * N + kp) : 1.f;
        const float2 S = cross_spectrum(P[aq * LD + ap], P[aq * LD + bp], a.method, wk);
        P[aq * LD + ap] = S;
        P[aq * LD + bp] = make_float2(S.x, -S.y);
      }
    }
    grp_sync(bar, G);
    //      (ii) for N > 32 every other canonical column forms its spectrum
    //      while it is read for its first inverse pass; its partner column
    //      -kq is read only by it, and written only after the pass.
    if (N2 > 1) {
#pragma unroll 1
      for (int it = gt; it < NC * N1; it += G) {
        int c, k1;
        if (C::SPREAD7) {  // c = N1 u + v with u fastest, then v, then k1; c = N/2 last
          if (it < H * N1) {
            constexpr int U = N2 / 2 > 0 ? N2 / 2 : 1;
            const int u = it % U, w = it / U;
            c = N1 * u + w % N1;
            k1 = w / N1;
          } else {
            c = H;
            k1 = it - H * N1;
          }
        } else {
          c = it % NC;
          k1 = it / NC;
        }
        const int aq = s_canon[c], bq = s_neg[aq];
        float2* L = P + aq * LD + N2 * k1;
        const float2* Lb = P + bq * LD;
        // slot N2 k1 + k2 holds frequency k1 + N1 k2; its negation sits at
        // slot N2 (N1 - k1) + N2 - 1 - k2 (k1 > 0), or N2 - k2 (k1 = 0, k2 > 0),
        // or 0: the row base is per item, the offsets constants
        const int nb0 = k1 == 0 ? N2 : N2 * (N1 - k1) + N2 - 1;
        float2 x[N2];
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
          x[k2] = L[k2];
          if (aq != bq) {
            const int neg = (k1 == 0 && k2 == 0) ? 0 : nb0 - k2;
            const float wk = a.method == 1 ? ld_keep(a.phasew + c * N + k1 + N1 * k2) : 1.f;
            x[k2] = cross_spectrum(x[k2], Lb[neg], a.method, wk);
          }
        }
        RDFT<N2, true>::run(x, N2);
#pragma unroll
        for (int n2 = 1; n2 < N2; ++n2) {
          const float2 t = tw[(n2 * k1) % N];
          x[n2] = cmul(x[n2], make_float2(t.x, -t.y));
        }
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) L[n2] = x[n2];
      }
      grp_sync(bar, G);
    }
#pragma unroll 1
    //      With N2 = 1 the two self-paired columns kq = 0 and N/2, whose
    //      results are real, share one transform as col0 + i col(N/2) (real
    //      part: column 0, imaginary part: column N/2): H items in all.
    //      With N2 > 1 consecutive threads take consecutive n2 of one column
    //      (the canonical columns sit N2 storage columns apart, which alias
    //      to two banks; rows n2 of one column do not).
    for (int it = gt; it < (N2 == 1 ? H : NC * N2); it += G) {
      const bool pk = N2 == 1 && it == 0;
      const int c = N2 == 1 ? it : it / N2, n2 = N2 == 1 ? 0 : it % N2;
      const int aq = N2 == 1 ? c : s_canon[c];
      const int bq = pk ? H : (N2 == 1 ? N - c : s_neg[aq]);
      float2* L = P + aq * LD;
      float2* Lb = P + bq * LD;
      float2 x[N1];
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) {
        const float2 u = L[N2 * k1 + n2];
        if (pk) {
          const float2 v = Lb[k1];
          x[k1] = make_float2(u.x - v.y, u.y + v.x);
        } else {
          x[k1] = u;
        }
      }
      RDFT<N1, true>::run(x, N1);
#pragma unroll
      for (int n1 = 0; n1 < N1; ++n1) {
        if (pk) {
          L[n1] = make_float2(x[n1].x, 0.f);
          Lb[n1] = make_float2(x[n1].y, 0.f);
        } else {
          L[N2 * n1 + n2] = x[n1];
          if (bq != aq) Lb[N2 * n1 + n2] = make_float2(x[n1].x, -x[n1].y);
        }
      }
    }
    grp_sync(bar, G);
    // ---- stage 8: inverse along q for the rows R needs: fftshifted rows
    //      blo..bhi (the overlap gain is zero on every other row, so R is
    //      exactly 0 there), taken in pairs (blo + t, blo + t + nh) packed as
    //      T(p) + i T(p'). The normalised, gain-weighted magnitudes are held
    //      in registers across a barrier, then written as the real plane R
    //      over the complex one; the other rows are written as zeros.
    const int nb = bhi - blo + 1, nh = (nb + 1) / 2;
    if (N2 > 1) {
#pragma unroll 1
      for (int it = gt; it < H * N1; it += G) {  // items (t, k1) at it = t + H k1, t < nh used
        const int t = it % H, k1 = it / H;
        if (t >= nh) continue;
        const bool hasb = t + nh < nb;
        const int pa = (blo + t + H) % N, pb = hasb ? (blo + t + nh + H) % N : pa;
        float2* La = P + pa + (N2 * k1) * LD;
        const float2* Lb = P + pb + (N2 * k1) * LD;
        float2 x[N2];
#pragma unroll
        for (int k2 = 0; k2 < N2; ++k2) {
          const float2 u = La[k2 * LD];
          const float2 v = hasb ? Lb[k2 * LD] : make_float2(0.f, 0.f);
          x[k2] = make_float2(u.x - v.y, u.y + v.x);
        }
        RDFT<N2, true>::run(x, N2);
#pragma unroll
        for (int n2 = 1; n2 < N2; ++n2) {
          const float2 tt = tw[(n2 * k1) % N];
          x[n2] = cmul(x[n2], make_float2(tt.x, -tt.y));
        }
#pragma unroll
        for (int n2 = 0; n2 < N2; ++n2) La[n2 * LD] = x[n2];
      }
      grp_sync(bar, G);
    }
    {
      float rv[IPT][2][N1];
#pragma unroll
      for (int i = 0; i < IPT; ++i) {
        const int it = gt + i * G;  // items (t, n2) at it = t + H n2, t < nh used
        if (it < H * N2 && it % H < nh) {
          const int t = it % H, n2 = it / H;
          const bool hasb = t + nh < nb;
          const int pa = (blo + t + H) % N, pb = hasb ? (blo + t + nh + H) % N : pa;
          const float2* La = P + pa;
          const float2* Lb = P + pb;
          float2 x[N1];
#pragma unroll
          for (int k1 = 0; k1 < N1; ++k1) {
            if (N2 == 1) {
              const float2 u = La[k1 * LD];
              const float2 v = hasb ? Lb[k1 * LD] : make_float2(0.f, 0.f);
              x[k1] = make_float2(u.x - v.y, u.y + v.x);
            } else {
              x[k1] = La[(N2 * k1 + n2) * LD];
            }
          }
          RDFT<N1, true>::run(x, N1);
          const int ps0 = blo + t, ps1 = blo + t + nh;  // fftshifted rows of pa and pb
#pragma unroll
          for (int n1 = 0; n1 < N1; ++n1) {
            const int qs = (N2 * n1 + n2 + H) % N;
            float r0 = fabsf(x[n1].x) * scale, r1 = fabsf(x[n1].y) * scale;
            if (a.gain) {
              if (C::GSM) {
                r0 *= s_gain[qs * N + ps0];
                r1 *= hasb ? s_gain[qs * N + ps1] : 0.f;
              } else if (gq) {
                const int bq = abs(qs - H) * (H + 1);
                r0 *= s_gain[abs(ps0 - H) + bq];
                r1 *= hasb ? s_gain[abs(ps1 - H) + bq] : 0.f;
              } else {
                r0 *= ld_keep(a.gain + qs * N + ps0);
                r1 *= hasb ? ld_keep(a.gain + qs * N + ps1) : 0.f;
              }
            }
            if (SRCH && (qs < blo || qs > bhi)) r0 = r1 = 0.f;  // lags outside the search range
            rv[i][0][n1] = r0;
            rv[i][1][n1] = r1;
          }
        }
      }
      grp_sync(bar, G);
#pragma unroll
      for (int i = 0; i < IPT; ++i) {
        const int it = gt + i * G;
        if (it < H * N2 && it % H < nh) {
          const int t = it % H, n2 = it / H;
          const bool hasb = t + nh < nb;
          const int ps0 = blo + t, ps1 = blo + t + nh;
#pragma unroll
          for (int n1 = 0; n1 < N1; ++n1) {
            const int qs = (N2 * n1 + n2 + H) % N;
            Rw[qs * LDR + ps0] = rv[i][0][n1];
            if (hasb) Rw[qs * LDR + ps1] = rv[i][1][n1];
          }
        }
      }
      const int nz = N - nb;  // rows outside [blo, bhi]
      for (int j = gt; j < nz; j += G) {
        const int ps = j < blo ? j : j + nb;
#pragma unroll 4
        for (int qs = 0; qs < N; ++qs) Rw[qs * LDR + ps] = 0.f;
      }
    }
    grp_sync(bar, G);
    if (a.planes) {
      float* dst = a.planes + job * (int64_t)(N * N);
      for (int it = gt; it < N * N; it += G) {
        const int p = it % N, q = it / N;
        const float r = Rw[q * LDR + p];
        // ensemble: per-pair planes summed in pair order; a window with
        // non-finite data poisons its sum as the reference's NaN plane does
        const float rr = bad ? __int_as_float(0x7fc00000) : r;
        dst[q * N + p] = a.accumulate ? dst[q * N + p] + rr : rr;
      }
      if (a.accumulate) {  // ensemble planes are analysed once, after the last pair
        grp_sync(bar, G);
        continue;
      }
    }
    // ---- stage 9: peak analysis by the group (the output pointers are
    //      needed only when the outputs are formed here, not from a record)
    const bool defer = a.rec && a.finder == 0;
    uint32_t* gred = red + w * (G / 32) * 2 * KMAX;
    if (C::INLINE_ANALYSIS && K <= 4)
      analyze_body<4, false>(Rw, N, N, LDR, K, a.npeaks, a.finder, a.subpixel, gt, G, gred, true, s_vals + w * KMAX,
                      s_locs + w * 2 * KMAX, gid, job, defer ? nullptr : &pw, bad, bar, sp, a.rec, a.njobs);
    else if (C::INLINE_ANALYSIS)
      analyze_body<KMAX, false>(Rw, N, N, LDR, K, a.npeaks, a.finder, a.subpixel, gt, G, gred, true, s_vals + w * KMAX,
                         s_locs + w * 2 * KMAX, gid, job, defer ? nullptr : &pw, bad, bar, sp, a.rec, a.njobs);
    else
      analyze_group<C::HALF>(Rw, N, N, LDR, K, a.npeaks, a.finder, a.subpixel, gt, G, gred, true, s_vals + w * KMAX,
                    s_locs + w * 2 * KMAX, gid, job, defer ? nullptr : &pw, bad, bar, sp, a.rec, a.njobs);
    grp_sync(bar, G);  // the plane is reused by the group's next window
  }
}

// Device analysis of caller-supplied planes (one CTA of 128 threads each).
// The plane is staged in shared memory when it fits (in_smem), else read in
// place from global memory (planes above 200 KB: 256 x 256 and larger).
__global__ void __launch_bounds__(128) analyze_planes_kernel(const AnalyzeArgs a, bool in_smem) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int P = a.nr * a.nc;
  float* R = reinterpret_cast<float*>(smem_raw);
  uint32_t* red = reinterpret_cast<uint32_t*>(smem_raw + (in_smem ? (size_t)P * sizeof(float) : 0));
  float* s_vals = reinterpret_cast<float*>(red + 8 * KMAX);
  int* s_locs = reinterpret_cast<int*>(s_vals + KMAX);
  const int K = a.npeaks > 2 ? a.npeaks : 2;
  PeakOut po{a.du, a.dv, a.ratio, a.moment, a.alt_u, a.alt_v, a.nalt, a.G, a.packed, a.locs};
  const ScanPlan sp = scan_plan(threadIdx.x, 128, 0, a.nr - 1, 0, a.nc - 1);
  for (int64_t pl = blockIdx.x; pl < a.nplanes; pl += gridDim.x) {
    const float* Rp = a.planes + pl * (int64_t)P;
    if (in_smem) {
      for (int k = threadIdx.x; k < P; k += blockDim.x) R[k] = Rp[k];
      Rp = R;
    }
    __syncthreads();
    const int64_t gid = a.jobs ? (int64_t)a.jobs[4 * pl] + (int64_t)a.jobs[4 * pl + 1] * a.ny : -1;
    analyze_group(Rp, a.nr, a.nc, a.nr, K, a.npeaks, a.finder, a.subpixel, threadIdx.x, 128, red, true, s_vals,
                  s_locs, gid, pl, &po, false, 0, sp, nullptr, 0);
    __syncthreads();
  }
}

// The per-window outputs from the peak records (one thread per window):
// the same arithmetic as the in-kernel epilogue, with every lane on its own
// window instead of one lane per window holding up the window's warp.
__global__ void __launch_bounds__(128) peak_epilogue_kernel(const CorrArgs a, int N) {
  const int K = a.npeaks > 2 ? a.npeaks : 2;
  const int64_t S = a.njobs;
  const PeakOut po{a.du, a.dv, a.ratio, a.moment, a.alt_u, a.alt_v, a.nalt, a.G, a.packed, a.locs};
  for (int64_t job = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; job < a.njobs;
       job += (int64_t)gridDim.x * blockDim.x) {
    const int nf = __float_as_int(__ldg(a.rec + job));
    if (nf < 0) continue;  // skipped by the correlation kernel
    int64_t gid;
    PeakOut pw = po;
    if (a.bp) {  // the correlation kernel's addressing of the window's grid cell
      const int p = a.jobs[4 * job];
      const BPair& b = a.bp[p];
      const int gij = a.jobs[4 * job + 1];
      gid = b.goff + (int64_t)(gij & 0xFFFF) + (int64_t)(gij >> 16) * b.ny;
      pw.G = (int64_t)b.ny * b.nx;
      pw.nalt = b.nalt;
      pw.alt_u = a.alt_u ? a.alt_u + b.aoff - b.goff : nullptr;
      pw.alt_v = a.alt_v ? a.alt_v + b.aoff - b.goff : nullptr;
    } else {
      gid = (int64_t)a.jobs[4 * job] + (int64_t)a.jobs[4 * job + 1] * a.ny;
    }
    float vals[KMAX];
    int locs[2 * KMAX];
    for (int m = 0; m < nf; ++m) {
      vals[m] = __ldg(a.rec + (int64_t)(1 + m) * S + job);
      locs[2 * m] = __float_as_int(__ldg(a.rec + (int64_t)(1 + K + 2 * m) * S + job));
      locs[2 * m + 1] = __float_as_int(__ldg(a.rec + (int64_t)(2 + K + 2 * m) * S + job));
    }
    peak_outputs(RecSrc{a.rec + job, S, K}, N, N, K, a.npeaks, a.subpixel, nf, vals, locs, gid, job, pw);
  }
}

size_t correlate_record_words(int npeaks) { return (size_t)rec_words(npeaks > 2 ? npeaks : 2); }

// ---------------------------------------------------------------------------
template <int N, int W, bool SRCH, int VAR>
static cudaError_t launch_nw(const CorrArgs& a, cudaStream_t s, int num_sms) {
  using C = CorrCfg<N, W, SRCH, VAR>;
  const size_t sm = C::smem();
  static bool attr_set = false;
  if (!attr_set) {
    cudaError_t e = cudaFuncSetAttribute(correlate_kernel<N, W, SRCH, VAR>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    // the planes live in shared memory: ask for the largest carveout so the
    // register budget, not the L1 split, sets the CTAs per SM
    e = cudaFuncSetAttribute(correlate_kernel<N, W, SRCH, VAR>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             (int)cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    attr_set = true;
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, correlate_kernel<N, W, SRCH, VAR>, C::NT, sm);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  const int64_t units = (a.njobs + C::WPC - 1) / C::WPC;
  int64_t grid = (int64_t)per_sm * num_sms;
  if (grid > units) grid = units;
  if (grid < 1) grid = 1;
  correlate_kernel<N, W, SRCH, VAR><<<(unsigned)grid, C::NT, sm, s>>>(a);
  if (a.rec && a.finder == 0 && !a.accumulate) {
    int64_t eb = (a.njobs + 127) / 128;
    if (eb > (int64_t)num_sms * 16) eb = (int64_t)num_sms * 16;
    peak_epilogue_kernel<<<(unsigned)eb, 128, 0, s>>>(a, N);
  }
  return cudaGetLastError();
}

#define HH_CORR_CASES(X) \
  X(16, 8) X(16, 16) X(24, 12) X(24, 24) X(32, 16) X(32, 32) X(48, 24) X(48, 48) X(64, 32) X(64, 64) X(96, 48) \
  X(96, 96) X(128, 64) X(128, 128)

bool correlate_supported(int N, int W) {
#define X(n, w) if (N == n && W == w) return true;
  HH_CORR_CASES(X)
#undef X
  return false;
}

size_t correlate_smem_bytes(int N, int W) {
#define X(n, w) if (N == n && W == w) return CorrCfg<n, w>::smem();
  HH_CORR_CASES(X)
#undef X
  return 0;
}

cudaError_t launch_correlate(const CorrArgs& a, int N, int W, cudaStream_t s, int num_sms) {
  if (a.njobs <= 0) return cudaSuccess;
#define X(n, w)                                                                         \
  if (N == n && W == w) {                                                              \
    if (a.win > 0 && a.win < w) return launch_nw<n, w, true, 0>(a, s, num_sms);       \
    switch (a.variant) {                                                               \
      case 1: return launch_nw<n, w, false, 1>(a, s, num_sms);                         \
      case 2: return launch_nw<n, w, false, 2>(a, s, num_sms);                         \
      case 3: return launch_nw<n, w, false, 3>(a, s, num_sms);                         \
      case 4: return launch_nw<n, w, false, 4>(a, s, num_sms);                         \
      default: return launch_nw<n, w, false, 0>(a, s, num_sms);                        \
    }                                                                                  \
  }
  HH_CORR_CASES(X)
#undef X
  return cudaErrorInvalidValue;
}

int gcorr_radix_plan(int n, int8_t* radix) {
  if (n < 1) return -1;
  int ns = 0;
  auto push = [&](int r) {
    if (ns >= 24) return false;
    radix[ns++] = (int8_t)r;
    return true;
  };
  while (n % 4 == 0) {
    if (!push(4)) return -1;
    n /= 4;
  }
  while (n % 2 == 0) {
    if (!push(2)) return -1;
    n /= 2;
  }
  for (int f = 3; f <= 61 && n > 1; f += 2)
    while (n % f == 0) {
      if (!push(f)) return -1;
      n /= f;
    }
  return n == 1 ? ns : -1;
}

size_t gcorr_smem_extra() {
  return 4 * GC_WARPS * sizeof(double) + GC_WARPS * 2 * KMAX * sizeof(uint32_t) + KMAX * sizeof(float) +
         2 * KMAX * sizeof(int) + 64;
}

cudaError_t launch_correlate_general(const CorrArgs& a, cudaStream_t s) {
  if (a.njobs <= 0) return cudaSuccess;
  if (!a.gscr || !a.twr || !a.twc || a.gscr_slices < 1 || a.gc_col_warps < 1 || a.gc_col_warps > GC_WARPS ||
      a.gc_chunk_c < 2)
    return cudaErrorInvalidValue;
  const size_t sm = (size_t)a.gc_smem_lines + gcorr_smem_extra();
  static size_t attr = 0;
  if (sm > attr) {
    cudaError_t e = cudaFuncSetAttribute(correlate_general_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    attr = sm;
  }
  const int64_t grid = a.njobs < a.gscr_slices ? a.njobs : a.gscr_slices;
  correlate_general_kernel<<<(unsigned)grid, GC_THREADS, sm, s>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_analyze_planes(const AnalyzeArgs& a, cudaStream_t s) {
  if (a.nplanes <= 0) return cudaSuccess;
  const size_t extra = 8 * KMAX * sizeof(uint32_t) + KMAX * sizeof(float) + 2 * KMAX * sizeof(int) + 16;
  size_t sm = (size_t)a.nr * a.nc * sizeof(float) + extra;
  const bool in_smem = sm <= 200 * 1024;
  if (!in_smem) sm = extra;
  cudaError_t e = cudaFuncSetAttribute(analyze_planes_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024);
  if (e != cudaSuccess) return e;
  int64_t grid = a.nplanes < 4096 ? a.nplanes : 4096;
  analyze_planes_kernel<<<(unsigned)grid, 128, sm, s>>>(a, in_smem);
  return cudaGetLastError();
}

}  // namespace hh
