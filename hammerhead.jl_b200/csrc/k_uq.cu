// Wieneke (2015) correlation-statistics uncertainty (sm_100a).
//
// One CTA per interrogation window (grid-stride over jobs). It restates
// src/uncertainty.jl:51-179: the windows are mean-subtracted and apodized
// like load_windows!, the per-pixel correlation
// difference dC = a0*b1 - a1*b0 and its (1,2,1)/4 smoothing are formed in
// FP32, and the 2 x 44 statistics (C0, C+, C-, S00 and the 40 half-plane
// covariance sums of rings 1..4) are reduced in FP64 across the CTA;
// finalize_uncertainty (:162-179) then runs on one thread per component.
#include <math.h>
#include <stdint.h>

#include <type_traits>

#include "hh_batch.h"
#include "hh_internal.h"

namespace hh {

// covariance offsets (dr, dc) of one half-plane, ring 1..4 (UQ_OFFSETS,
// src/uncertainty.jl:16-35): dc in 0:4, dr in (dc == 0 ? 1:4 : -4:4), stably
// ordered by ring max(|dr|, |dc|).
struct UQOffsets {
  int8_t dr[40], dc[40];
  int8_t ring_start[5];
  // ring position of the offset with natural index n: n = dr - 1 for dc = 0
  // (dr = 1..4), else 4 + 9 (dc - 1) + (dr + 4)
  int8_t nat2ring[40];
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
  for (int k2 = 0; k2 < 40; ++k2) {
    const int dr = o.dr[k2], dc = o.dc[k2];
    const int n = dc == 0 ? dr - 1 : 4 + 9 * (dc - 1) + (dr + 4);
    o.nat2ring[n] = (int8_t)k2;
  }
  return o;
}

// finalize_uncertainty (src/uncertainty.jl:162-179). The doubled covariance
// sums enter S00 one ring at a time (each ring summed in its own order, then
// added), the arithmetic of the lane-parallel form uq_finalize_seg, so every
// kernel gives a window the same sigma from the same statistics.
__device__ __forceinline__ float uq_finalize(const double* s, const UQOffsets& o) {
  const double C0 = s[0], Cp = s[1], Cm = s[2], S00 = s[3];
  double s2 = S00;
  for (int ring = 0; ring < 4; ++ring) {
    double mx = -INFINITY, rsum = 0.0;
    for (int k = o.ring_start[ring]; k < o.ring_start[ring + 1]; ++k) {
      mx = fmax(mx, s[4 + k]);
      rsum = fma(2.0, s[4 + k], rsum);
    }
    if (mx < __dmul_rn(0.05, S00)) break;
    s2 = __dadd_rn(s2, rsum);
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

// One CTA (4 warps) per window. Every reduction runs across lanes: the
// window means and the mean of the smoothed field are block-wide FP64 sums,
// and each of the 88 statistics is summed by one warp (lanes stride over the
// pixel pairs, then a shuffle reduction). The FP32 parts -- the apodized
// windows, dC and its smoothing -- use the reference's operation order.
constexpr int UQ_THREADS = 128;

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__global__ void __launch_bounds__(UQ_THREADS) uq_kernel(const UQArgs a, const UQOffsets o) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int W = a.W, m = W - 1, WM = W * m;
  double* dd = reinterpret_cast<double*>(smem_raw);       // 2*WM: smoothed dC minus its mean (u, v)
  double* stats = dd + 2 * WM;                             // 88
  double* part = stats + 88;                               // 4 warps x 3
  float* wa = reinterpret_cast<float*>(part + 12);         // W*W
  float* wb = wa + W * W;                                  // W*W
  float* dC = wb + W * W;                                  // 2*WM
  float* dCs = dC + 2 * WM;                                // 2*WM
  uint8_t* mf = reinterpret_cast<uint8_t*>(dCs + 2 * WM);  // W*W
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int64_t job = blockIdx.x; job < a.njobs; job += gridDim.x) {
    const int rs = a.jobs[4 * job + 2], cs = a.jobs[4 * job + 3];
    const float* A = a.A;
    const float* B = a.B;
    const uint8_t* M = a.mask;
    int64_t ld = a.ld, gid;
    if (a.bp) {  // batched: the pair's images and grid region; skip windows it does not need
      const int p = a.jobs[4 * job];
      const BPair& b = a.bp[p];
      const int gij = a.jobs[4 * job + 1];
      const int64_t cell = (int64_t)(gij & 0xFFFF) + (int64_t)(gij >> 16) * b.ny;
      const bool on = a.mode == 0 ? (b.unc_fused && bp_live(b, 1, a.done, p)) : (b.unc_post && b.live);
      if (!on || (b.gmask && b.gmask[cell])) continue;  // uniform across the CTA
      const bool warped = a.mode == 1 || b.has_pred0;
      A = warped ? b.warpA : b.A;
      B = warped ? b.warpB : b.B;
      M = b.mask;
      ld = b.nr;
      gid = b.goff + cell;
    } else {
      gid = (int64_t)a.jobs[4 * job] + (int64_t)a.jobs[4 * job + 1] * a.ny;
    }
    // windows and their means (load_uncertainty_windows!, :51-83)
    double sa = 0.0, sb = 0.0, cnt = 0.0;
    for (int k = tid; k < W * W; k += UQ_THREADS) {
      const int p = k % W, q = k / W;
      const int64_t off = (int64_t)(rs + p) + (int64_t)(cs + q) * ld;
      const float va = A[off], vb = B[off];
      const uint8_t mk = M ? M[off] : 0;
      wa[k] = va;
      wb[k] = vb;
      mf[k] = mk;
      if (!mk) {
        sa += (double)va;
        sb += (double)vb;
        cnt += 1.0;
      }
    }
    sa = warp_sum(sa);
    sb = warp_sum(sb);
    cnt = warp_sum(cnt);
    if (lane == 0) {
      part[3 * warp] = sa;
      part[3 * warp + 1] = sb;
      part[3 * warp + 2] = cnt;
    }
    __syncthreads();
    double ta = 0, tb = 0, tn = 0;
    for (int w = 0; w < UQ_THREADS / 32; ++w) {
      ta += part[3 * w];
      tb += part[3 * w + 1];
      tn += part[3 * w + 2];
    }
    const float ma = tn > 0 ? (float)(ta / tn) : 0.f, mb = tn > 0 ? (float)(tb / tn) : 0.f;
    for (int k = tid; k < W * W; k += UQ_THREADS) {
      const float ap = a.apod[k];
      wa[k] = mf[k] ? 0.f : __fmul_rn(ap, __fsub_rn(wa[k], ma));
      wb[k] = mf[k] ? 0.f : __fmul_rn(ap, __fsub_rn(wb[k], mb));
    }
    __syncthreads();
    // dC = a0 b1 - a1 b0 for both components: u views (r, c) = (p, q), v = (q, p)
    for (int k = tid; k < 2 * WM; k += UQ_THREADS) {
      const int comp = k / WM, e = k % WM, r = e % W, c = e / W;
      const int str = comp == 0 ? 1 : W, stc = comp == 0 ? W : 1;
      const float a0 = wa[r * str + c * stc], a1 = wa[r * str + (c + 1) * stc];
      const float b0 = wb[r * str + c * stc], b1 = wb[r * str + (c + 1) * stc];
      dC[k] = __fsub_rn(__fmul_rn(a0, b1), __fmul_rn(a1, b0));
    }
    __syncthreads();
    double s0 = 0.0, s1 = 0.0;
    for (int k = tid; k < 2 * WM; k += UQ_THREADS) {
      const int comp = k / WM, e = k % WM, r = e % W, c = e / W;
      const float* d = dC + comp * WM;
      const int cl = c > 0 ? c - 1 : 0, cr = c < m - 1 ? c + 1 : m - 1;
      const float v = __fmul_rn(0.25f, __fadd_rn(__fadd_rn(d[r + cl * W], __fmul_rn(2.0f, d[r + c * W])), d[r + cr * W]));
      dCs[k] = v;
      if (comp == 0) s0 += (double)v;
      else s1 += (double)v;
    }
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    __syncthreads();  // part reused
    if (lane == 0) {
      part[3 * warp] = s0;
      part[3 * warp + 1] = s1;
    }
    __syncthreads();
    double mu0 = 0, mu1 = 0;
    for (int w = 0; w < UQ_THREADS / 32; ++w) {
      mu0 += part[3 * w];
      mu1 += part[3 * w + 1];
    }
    mu0 /= (double)WM;
    mu1 /= (double)WM;
    for (int k = tid; k < 2 * WM; k += UQ_THREADS) dd[k] = (double)dCs[k] - (k < WM ? mu0 : mu1);
    __syncthreads();
    // the 2 x 44 statistics, one warp per statistic (uq_component!, :104-151)
    for (int st = warp; st < 88; st += UQ_THREADS / 32) {
      const int comp = st / 44, si = st % 44;
      const int str = comp == 0 ? 1 : W, stc = comp == 0 ? W : 1;
      const double* d = dd + comp * WM;
      double acc = 0.0;
      if (si < 3) {
        for (int t = lane; t < WM; t += 32) {
          const int r = t % W, c = t / W;
          const float a0 = wa[r * str + c * stc], a1 = wa[r * str + (c + 1) * stc];
          const float b0 = wb[r * str + c * stc], b1 = wb[r * str + (c + 1) * stc];
          const float pr = si == 0 ? __fmul_rn(a0, b0) : (si == 1 ? __fmul_rn(a0, b1) : __fmul_rn(a1, b0));
          acc += (double)pr;
        }
      } else if (si == 3) {
        for (int t = lane; t < WM; t += 32) acc = fma(d[t], d[t], acc);
      } else {
        const int k = si - 4, dr = o.dr[k], dc = o.dc[k];
        const int c0 = dc < 0 ? -dc : 0, c1 = dc > 0 ? m - dc : m;  // c in [c0, c1)
        const int r0 = dr < 0 ? -dr : 0, r1 = dr > 0 ? W - dr : W;  // r in [r0, r1)
        const int nrr = r1 - r0, ncc = c1 - c0;
        for (int t = lane; t < nrr * ncc; t += 32) {
          const int r = r0 + t % nrr, c = c0 + t / nrr;
          acc = fma(d[r + c * W], d[(r + dr) + (c + dc) * W], acc);
        }
      }
      acc = warp_sum(acc);
      if (lane == 0) stats[st] = acc;
    }
    __syncthreads();
    if (a.stats)
      for (int it = tid; it < 88; it += UQ_THREADS) {
        if (a.accumulate) a.stats[job * 88 + it] += stats[it];
        else a.stats[job * 88 + it] = stats[it];
      }
    if (a.unc_u && tid < 2) {
      const float sg = uq_finalize(stats + 44 * tid, o);
      if (tid == 0) a.unc_u[gid] = sg;
      else a.unc_v[gid] = sg;
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Register form for windows up to 32 px: two warps per window, one per
// component (u: the window as stored, v: its transpose). Lane c owns column c
// of the component's W x (W-1) difference field dC for every row in
// registers, so the smoothing along the columns is register arithmetic plus
// one shuffle per row. The mean-free smoothed field then goes to shared
// memory (one column per lane, zero columns past the last), and each lane
// reads its neighbour columns there in 16-byte row pairs for the 40
// half-plane covariance sums, which are register FMAs. The per-lane partial
// sums are combined across the window's lanes by transposed shuffle sums
// (each exchange halves the values a lane holds), so no shared memory holds
// per-lane partials. Same FP32 operations as uq_kernel, FP64 sums.
// When dC has at most 16 columns (W <= 17) a warp serves two windows, one
// per 16-lane segment (shuffles of width 16), so no lane idles for want of
// a column. Window means are one warp's job per window (all 32 lanes), and
// finalize_uncertainty is spread over the first lanes of each window (ring
// maxima and sums on lanes 0-3, one logarithm each on lanes 0-2).
constexpr int UQW_THREADS = 128;  // two warp pairs (u, v)

template <int W> struct UQWCfg {
  static constexpr int LD = W + 1;  // odd column stride: conflict-free column and row walks
  static constexpr int M = W - 1;   // columns of dC
  static constexpr int WPW = M <= 16 ? 2 : 1;  // windows per warp
  static constexpr int SEG = 32 / WPW;         // lanes per window
  static constexpr int NWIN = 2 * WPW;         // windows per CTA
  // the smoothed field of one window component: column c at c * DLD doubles.
  // DLD = W + 2 is 2 mod 4 (W is a multiple of 4), so the 16-byte row pairs
  // that 8 consecutive lanes read from 8 consecutive columns fall in distinct
  // bank groups. Columns SEG .. SEG+3 stay zero: the lag partners of the last
  // lanes.
  static constexpr int DLD = W + 2;
  static constexpr int DCOLS = SEG + 4;
  static constexpr size_t dd_bytes = (size_t)DCOLS * DLD * sizeof(double);
  // window buffers of consecutive slots start 16 banks apart (64 bytes mod
  // 128), so the two windows of a warp do not meet in one bank
  static constexpr size_t win_raw = 2 * (size_t)LD * W * sizeof(float) + (size_t)W * W;
  static constexpr size_t win_bytes = (win_raw + 127) / 128 * 128 + 64;
  // the next windows are copied in (cp.async) while the current ones are
  // reduced, into a second set of buffers (at 32 px the second set would
  // cost a CTA per SM)
  static constexpr bool PREFETCH = W <= 24;
  static constexpr int NBUF = PREFETCH ? 2 : 1;
  static constexpr size_t up128(size_t x) { return (x + 127) / 128 * 128; }
  // shared memory: smoothed fields (4 warps x WPW), totals (4 x WPW x 44),
  // window buffers, per-warp sums for the window means, apodization, offset
  // tables
  static constexpr size_t off_tot = up128(4 * WPW * dd_bytes);
  static constexpr size_t off_win = up128(off_tot + 4 * WPW * 44 * sizeof(double));
  static constexpr size_t off_mean = up128(off_win + NBUF * NWIN * win_bytes);
  static constexpr size_t off_apod = up128(off_mean + 4 * 3 * sizeof(double));
  static constexpr size_t off_offs = up128(off_apod + (size_t)W * W * sizeof(float));
  static constexpr size_t smem() { return off_offs + sizeof(UQOffsets) + 16; }
  static constexpr int MINB = W <= 24 ? 4 : 3;  // CTAs per SM the register budget is sized for
};

// sum over the lanes of one SEG-lane segment
template <int SEG> __device__ __forceinline__ double seg_sum(double v) {
#pragma unroll
  for (int o = SEG / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Transposed segment sum: N values per lane, summed over the lanes of a
// segment in log2(SEG) exchanges. At the exchange with the lane at xor O,
// the lower lane keeps the first half of its values and sends the second,
// the upper lane the reverse, and each adds what it receives; so the values
// a lane holds halve at every step. On return the lane holds the totals of
// values base + i in v[i] for i < n (n <= tsum_slots(N, SEG)).
constexpr int tsum_slots(int n, int seg) { return seg <= 1 ? n : tsum_slots((n + 1) / 2, seg / 2); }
template <int N, int O> __device__ __forceinline__ void seg_tsum(double* v, int c, int& base, int& n) {
  if constexpr (O > 0) {
    constexpr int H = (N + 1) / 2;
    const bool up = (c & O) != 0;
#pragma unroll
    for (int i = 0; i < H; ++i) {
      const double lo = v[i];
      const double hi = i + H < N ? v[i + H] : 0.0;
      const double send = up ? lo : hi;
      const double keep = up ? hi : lo;
      v[i] = keep + __shfl_xor_sync(0xffffffffu, send, O);
    }
    if (up) {
      base += H;
      n = n > H ? n - H : 0;
    } else {
      n = n < H ? n : H;
    }
    seg_tsum<H, O / 2>(v, c, base, n);
  }
}

// finalize_uncertainty (src/uncertainty.jl:162-179) of one window component
// from its 44 statistics in ring order (shared memory, visible to the
// segment), spread over the segment's first lanes: lane j < 4 forms ring
// j+1's maximum and doubled sum, lanes 0, 1, 2 one logarithm each. The
// result is valid on every lane of the segment.
template <int SEG> __device__ __forceinline__ float uq_finalize_seg(const double* s, const UQOffsets& o, int c) {
  constexpr unsigned FULL = 0xffffffffu;
  const int lb = (int)(threadIdx.x & 31) & ~(SEG - 1);  // the segment's first lane
  double mx = -INFINITY, rsum = 0.0;
  if (c < 4)
    for (int k = o.ring_start[c]; k < o.ring_start[c + 1]; ++k) {
      const double x = s[4 + k];
      mx = fmax(mx, x);
      rsum = fma(2.0, x, rsum);
    }
  const double C0 = s[0], Cp = s[1], Cm = s[2], S00 = s[3];
  const double thr = __dmul_rn(0.05, S00);
  double s2 = S00;
  bool go = true;
#pragma unroll
  for (int j = 0; j < 4; ++j) {
    const double m = __shfl_sync(FULL, mx, lb + j);
    const double t = __shfl_sync(FULL, rsum, lb + j);
    go = go && !(m < thr);  // a ring below 5 % of S00 ends the sum (NaN does not)
    if (go) s2 = __dadd_rn(s2, t);
  }
  const double sdc = sqrt(fmax(s2, 0.0));
  const double Cpm = __dmul_rn(__dadd_rn(Cp, Cm), 0.5);
  const double lo = __dsub_rn(Cpm, __dmul_rn(sdc, 0.5)), hi = __dadd_rn(Cpm, __dmul_rn(sdc, 0.5));
  const double lg = log(c == 0 ? C0 : (c == 1 ? hi : lo));
  const double lC0 = __shfl_sync(FULL, lg, lb), lhi = __shfl_sync(FULL, lg, lb + 1), llo = __shfl_sync(FULL, lg, lb + 2);
  if (!(C0 > 0 && lo > 0)) return __int_as_float(0x7fc00000);
  const double denom = __dsub_rn(__dsub_rn(__dmul_rn(2.0, lC0), lhi), llo);
  if (!(denom > 0)) return __int_as_float(0x7fc00000);
  return (float)(__dsub_rn(lhi, llo) / __dmul_rn(2.0, denom));
}

// Where window `job` comes from: on = the window is estimated in this launch.
struct UQSrc {
  bool on;
  const float* A;
  const float* B;
  const uint8_t* M;
  int64_t ld, gid;
  int rs, cs;
};
__device__ __forceinline__ UQSrc uq_src(const UQArgs& a, int64_t job) {
  UQSrc r{job < a.njobs, a.A, a.B, a.mask, a.ld, -1, 0, 0};
  if (r.on) {
    r.rs = a.jobs[4 * job + 2];
    r.cs = a.jobs[4 * job + 3];
    if (a.bp) {
      const int p = a.jobs[4 * job];
      const BPair& b = a.bp[p];
      const int gij = a.jobs[4 * job + 1];
      const int64_t cell = (int64_t)(gij & 0xFFFF) + (int64_t)(gij >> 16) * b.ny;
      r.on = a.mode == 0 ? (b.unc_fused && bp_live(b, 1, a.done, p)) : (b.unc_post && b.live);
      r.on = r.on && !(b.gmask && b.gmask[cell]);
      const bool warped = a.mode == 1 || b.has_pred0;
      r.A = warped ? b.warpA : b.A;
      r.B = warped ? b.warpB : b.B;
      r.M = b.mask;
      r.ld = b.nr;
      r.gid = b.goff + cell;
    } else {
      r.gid = (int64_t)a.jobs[4 * job] + (int64_t)a.jobs[4 * job + 1] * a.ny;
    }
  }
  return r;
}

// 4-byte asynchronous global -> shared copy and its group operations
__device__ __forceinline__ void cp_async4(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_prev() { asm volatile("cp.async.wait_group 1;\n" ::: "memory"); }

template <int W>
__global__ void __launch_bounds__(UQW_THREADS, UQWCfg<W>::MINB) uq_warp_kernel(const UQArgs a, const UQOffsets o) {
  using C = UQWCfg<W>;
  constexpr int LD = C::LD, M = C::M, WPW = C::WPW, SEG = C::SEG, NWIN = C::NWIN, DLD = C::DLD;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  unsigned char* wbase = smem_raw + C::off_win;
  double* msum = reinterpret_cast<double*>(smem_raw + C::off_mean);  // per warp: its share of (sum A, sum B, count)
  float* sap = reinterpret_cast<float*>(smem_raw + C::off_apod);    // the apodization window
  // the offset tables in shared memory (indexed at run time; a parameter
  // struct indexed that way would be copied to local memory)
  UQOffsets& so = *reinterpret_cast<UQOffsets*>(smem_raw + C::off_offs);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int comp = warp & 1, seg = lane / SEG, c = lane % SEG;
  const int slot = (warp >> 1) * WPW + seg;  // window of this lane
  const int ts = comp * SEG + c;             // this lane among the 2*SEG threads of its window
  double* dsm = reinterpret_cast<double*>(smem_raw + (size_t)(warp * WPW + seg) * C::dd_bytes);  // this segment's field
  double* tot = reinterpret_cast<double*>(smem_raw + C::off_tot) + (warp * WPW + seg) * 44;      // its 44 totals
  if (tid == 0) so = o;
  for (int k = tid; k < W * W; k += UQW_THREADS) sap[k] = __ldg(a.apod + k);
  {  // the zero columns past each segment's lanes (never written again)
    double* d0 = reinterpret_cast<double*>(smem_raw + (size_t)(warp * WPW) * C::dd_bytes);
    for (int k = lane; k < WPW * 4 * DLD; k += 32) {
      const int g = k / (4 * DLD), e = k % (4 * DLD);
      d0[(size_t)g * (C::dd_bytes / sizeof(double)) + SEG * DLD + e] = 0.0;
    }
  }
  __syncthreads();
  const int64_t stride = (int64_t)gridDim.x * NWIN;
  // copies the window's pixels into buffer set `ph` asynchronously
  auto prefetch = [&](const UQSrc& q0, int ph) {
    float* pa = reinterpret_cast<float*>(wbase + (ph * NWIN + slot) * C::win_bytes);
    float* pb = pa + LD * W;
    if (q0.on)
      for (int k = ts; k < W * W; k += 2 * SEG) {
        const int p = k % W, q = k / W;
        const int64_t off = (int64_t)(q0.rs + p) + (int64_t)(q0.cs + q) * q0.ld;
        cp_async4(pa + p + q * LD, q0.A + off);
        cp_async4(pb + p + q * LD, q0.B + off);
      }
  };
  int iter = 0;
  int64_t base = (int64_t)blockIdx.x * NWIN;
  // the source of this lane's window in the current iteration; the next
  // iteration's is looked up once, for its prefetch, and carried over
  UQSrc src = uq_src(a, base + slot);
  if (C::PREFETCH) {
    prefetch(src, 0);
    cp_async_commit();
  }
  for (; base < a.njobs; base += stride, ++iter) {
    const int64_t job = base + slot;
    const int ph = C::PREFETCH ? (iter & 1) : 0;
    float* wa = reinterpret_cast<float*>(wbase + (ph * NWIN + slot) * C::win_bytes);  // W x W, column stride LD
    float* wb = wa + LD * W;
    uint8_t* mf = reinterpret_cast<uint8_t*>(wb + LD * W);
    // ---- the window's source (uniform within the window's lanes)
    const UQSrc nxt = uq_src(a, base + stride + slot);
    const bool on = src.on;
    const float* A = src.A;
    const float* B = src.B;
    const uint8_t* Mk = src.M;
    const int64_t ld = src.ld, gid = src.gid;
    const int rs = src.rs, cs = src.cs;
    // with two windows per warp every lane runs the arithmetic below (the
    // shuffles span the warp, whose windows may differ in `on`); a window
    // that is off computes on zeros and writes nothing. With one window per
    // warp `on` is uniform and an idle warp pair skips the work.
    const bool run = WPW == 1 ? on : true;
    if (C::PREFETCH) {
      // the next windows go to the other buffer set while these are reduced
      // (that set was last read in the previous iteration, before its final
      // barrier); then wait for this set's copies, issued one group earlier
      prefetch(nxt, ph ^ 1);  // nothing for a window past the last job (nxt.on is false)
      cp_async_commit();
      cp_async_wait_prev();
      if (run)
        for (int k = ts; k < W * W; k += 2 * SEG) {
          const int p = k % W, q = k / W;
          uint8_t mk = 1;
          if (on) {
            mk = Mk ? __ldg(Mk + (int64_t)(rs + p) + (int64_t)(cs + q) * ld) : 0;
          } else {
            wa[p + q * LD] = 0.f;
            wb[p + q * LD] = 0.f;
          }
          mf[k] = mk;
        }
    } else if (run) {
      for (int k = ts; k < W * W; k += 2 * SEG) {
        const int p = k % W, q = k / W;
        float va = 0.f, vb = 0.f;
        uint8_t mk = 1;
        if (on) {
          const int64_t off = (int64_t)(rs + p) + (int64_t)(cs + q) * ld;
          va = __ldg(A + off);
          vb = __ldg(B + off);
          mk = Mk ? __ldg(Mk + off) : 0;
        }
        wa[p + q * LD] = va;
        wb[p + q * LD] = vb;
        mf[k] = mk;
      }
    }
    __syncthreads();
    // ---- window means (load_uncertainty_windows!), FP64: MW = 4 / NWIN warps
    //      per window slot, each summing its share of the pixels over all its
    //      lanes (a slot whose window is off and was not loaded yields values
    //      nobody reads)
    {
      constexpr int MW = 4 / NWIN;
      const int s = warp / MW, h = warp % MW;
      const float* pa = reinterpret_cast<const float*>(wbase + (ph * NWIN + s) * C::win_bytes);
      const float* pb = pa + LD * W;
      const uint8_t* pm = reinterpret_cast<const uint8_t*>(pb + LD * W);
      double sa = 0.0, sb = 0.0, cnt = 0.0;
#pragma unroll 4
      for (int k = h * 32 + lane; k < W * W; k += 32 * MW)
        if (!pm[k]) {
          const int p = k % W, q = k / W;
          sa += (double)pa[p + q * LD];
          sb += (double)pb[p + q * LD];
          cnt += 1.0;
        }
      sa = seg_sum<32>(sa);
      sb = seg_sum<32>(sb);
      cnt = seg_sum<32>(cnt);
      if (lane == 0) {
        msum[3 * warp] = sa;
        msum[3 * warp + 1] = sb;
        msum[3 * warp + 2] = cnt;
      }
    }
    __syncthreads();  // the sums are visible, and every read of the raw values precedes the apodized writes
    if (run) {
      constexpr int MW = 4 / NWIN;
      double sa = 0.0, sb = 0.0, cnt = 0.0;
#pragma unroll
      for (int h = 0; h < MW; ++h) {
        sa += msum[3 * (slot * MW + h)];
        sb += msum[3 * (slot * MW + h) + 1];
        cnt += msum[3 * (slot * MW + h) + 2];
      }
      const float ma = cnt > 0 ? (float)(sa / cnt) : 0.f, mb = cnt > 0 ? (float)(sb / cnt) : 0.f;
      for (int k = ts; k < W * W; k += 2 * SEG) {
        const int p = k % W, q = k / W;
        const float ap = sap[k];
        const float va = wa[p + q * LD], vb = wb[p + q * LD];
        wa[p + q * LD] = mf[k] ? 0.f : __fmul_rn(ap, __fsub_rn(va, ma));
        wb[p + q * LD] = mf[k] ? 0.f : __fmul_rn(ap, __fsub_rn(vb, mb));
      }
    }
    __syncthreads();
    if (run) {
      // ---- this component's dC column (lane c < M), and the C0 / C+ / C- sums
      const bool col = c < M;
      const int cc = col ? c : 0;
      float dcol[W];
      double s0 = 0.0, s1 = 0.0, s2 = 0.0;
#pragma unroll
      for (int r = 0; r < W; ++r) {
        // u: element (p, q) = (r, c); v: (p, q) = (c, r)
        const int i0 = comp == 0 ? r + cc * LD : cc + r * LD;
        const int i1 = comp == 0 ? r + (cc + 1) * LD : (cc + 1) + r * LD;
        const float a0 = wa[i0], a1 = wa[i1], b0 = wb[i0], b1 = wb[i1];
        dcol[r] = __fsub_rn(__fmul_rn(a0, b1), __fmul_rn(a1, b0));
        if (col) {
          s0 += (double)__fmul_rn(a0, b0);
          s1 += (double)__fmul_rn(a0, b1);
          s2 += (double)__fmul_rn(a1, b0);
        }
      }
      // ---- (1,2,1)/4 smoothing along the columns, and its mean
      double dd[W];
      double fs[2] = {0.0, 0.0};  // two interleaved partial sums (shorter dependency chains)
#pragma unroll
      for (int r = 0; r < W; ++r) {
        const float left = __shfl_up_sync(FULL, dcol[r], 1, SEG);
        const float right = __shfl_down_sync(FULL, dcol[r], 1, SEG);
        const float l = c > 0 ? left : dcol[r];
        const float rr = c < M - 1 ? right : dcol[r];
        const float v = __fmul_rn(0.25f, __fadd_rn(__fadd_rn(l, __fmul_rn(2.0f, dcol[r])), rr));
        dd[r] = (double)v;
        if (col) fs[r & 1] += dd[r];
      }
      constexpr double inv_n = 1.0 / (double)(W * M);  // the mean as a product (a division costs a long chain)
      const double mu = seg_sum<SEG>(fs[0] + fs[1]) * inv_n;
#pragma unroll
      for (int r = 0; r < W; ++r) dd[r] = col ? dd[r] - mu : 0.0;
      // this lane's column of the field into shared memory (lanes past M
      // store zeros), for the neighbour-column reads of the covariance sums
#pragma unroll
      for (int r = 0; r < W; r += 2) *reinterpret_cast<double2*>(dsm + c * DLD + r) = make_double2(dd[r], dd[r + 1]);
      // sums the per-lane partials v[0..N) of statistics first .. first+N-1
      // (natural order) over the window's lanes; the lanes holding totals
      // store them in ring order
      auto reduce_store = [&](double* v, auto n_tag, int first) {
        constexpr int N = decltype(n_tag)::value;
        int b = 0, n = N;
        seg_tsum<N, SEG / 2>(v, c, b, n);
#pragma unroll
        for (int i = 0; i < tsum_slots(N, SEG); ++i)
          if (i < n) {
            const int st = first + b + i;
            const int ri = st < 4 ? st : 4 + so.nat2ring[st - 4];
            tot[ri] = v[i];
            if (on && a.stats) {
              if (a.accumulate) a.stats[job * 88 + comp * 44 + ri] += v[i];
              else a.stats[job * 88 + comp * 44 + ri] = v[i];
            }
          }
      };
      // ---- C0, C+, C-, S00 and the lag-(dr, 0) sums (registers only)
      {
        double g1[8] = {s0, s1, s2, 0.0, 0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int r = 0; r < W; ++r) {
          g1[3] = fma(dd[r], dd[r], g1[3]);
#pragma unroll
          for (int dr = 1; dr <= 4; ++dr)
            if (r + dr < W) g1[3 + dr] = fma(dd[r], dd[r + dr], g1[3 + dr]);
        }
        reduce_store(g1, std::integral_constant<int, 8>{}, 0);
      }
      __syncwarp();  // the segment's columns are in shared memory
      // ---- the covariance sums of columns dc = 1..4: acc[9 i + dr + 4]
      //      pairs (r, c) with (r + dr, c + dc), dc = dg + i. Two neighbour
      //      columns at a time, so only 18 accumulators are live; a neighbour
      //      column past the window is one of the zero columns.
#pragma unroll
      for (int dg = 1; dg <= 3; dg += 2) {
        double acc[18];
#pragma unroll
        for (int jj = 0; jj < 18; ++jj) acc[jj] = 0.0;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const double* xc = dsm + (c + dg + i) * DLD;
#pragma unroll
          for (int r2 = 0; r2 < W; r2 += 2) {
            const double2 x2 = *reinterpret_cast<const double2*>(xc + r2);
#pragma unroll
            for (int h = 0; h < 2; ++h) {
              const double x = h ? x2.y : x2.x;
#pragma unroll
              for (int dr = -4; dr <= 4; ++dr) {
                const int r0 = r2 + h - dr;
                if (r0 >= 0 && r0 < W) acc[9 * i + dr + 4] = fma(dd[r0], x, acc[9 * i + dr + 4]);
              }
            }
          }
        }
        reduce_store(acc, std::integral_constant<int, 18>{}, 8 + 9 * (dg - 1));
      }
      __syncwarp();  // the totals are visible to the segment
      const float sg = uq_finalize_seg<SEG>(tot, so, c);
      if (c == 0 && on && a.unc_u) (comp == 0 ? a.unc_u : a.unc_v)[gid] = sg;
    }
    src = nxt;
    __syncthreads();  // the window buffers and fields are reused by the next iteration
  }
}

__global__ void uq_finalize_kernel(const double* __restrict__ stats, const int32_t* __restrict__ jobs, int64_t njobs,
                                   int32_t ny, float* unc_u, float* unc_v, const UQOffsets o) {
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < 2 * njobs; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t job = k >> 1;
    const int comp = (int)(k & 1);
    const int64_t gid = (int64_t)jobs[4 * job] + (int64_t)jobs[4 * job + 1] * ny;
    (comp == 0 ? unc_u : unc_v)[gid] = uq_finalize(stats + job * 88 + comp * 44, o);
  }
}

// ---------------------------------------------------------------------------
// General form: rectangular windows (wr x wc) and windows above 64 px. The
// same operations as uq_kernel, per component in its own frame (u: the
// window as stored, wr rows x wc columns, shifts along the columns; v: its
// transpose, wc rows x wr columns), with the windows, dC, its smoothing and
// the FP64 field in a global scratch slice per CTA instead of shared memory.
struct UQGeom {
  int R, C, m;          // rows, columns of the component's frame; m = C - 1 columns of dC
  int sr_, sc_;         // strides of (r, c) into the stored window
};
__device__ __forceinline__ UQGeom uq_geom(int comp, int wr, int wc) {
  return comp == 0 ? UQGeom{wr, wc, wc - 1, 1, wr} : UQGeom{wc, wr, wr - 1, wr, 1};
}

bool uq_general(int wr, int wc) { return wr != wc || wr > 64; }
int64_t uq_general_stride(int wr, int wc) {
  const int64_t n = (int64_t)wr * wc, mu = (int64_t)wr * (wc - 1), mv = (int64_t)wc * (wr - 1);
  // doubles: dd (mu + mv); floats: wa, wb (n each), dC and dCs (mu + mv each)
  const int64_t fl = 2 * n + 2 * (mu + mv);
  return ((mu + mv) + (fl + 1) / 2 + 31) & ~(int64_t)31;
}

__global__ void __launch_bounds__(UQ_THREADS) uq_general_kernel(const UQArgs a, const UQOffsets o) {
  __shared__ double stats[88];
  __shared__ double part[4 * (UQ_THREADS / 32)];
  const int wr = a.W, wc = a.Wc > 0 ? a.Wc : a.W, n = wr * wc;
  const int mu = wr * (wc - 1), mv = wc * (wr - 1);
  double* dd = a.gscr + (int64_t)blockIdx.x * a.gscr_stride;  // mu + mv
  float* wa = reinterpret_cast<float*>(dd + mu + mv);          // n
  float* wb = wa + n;                                          // n
  float* dC = wb + n;                                          // mu + mv
  float* dCs = dC + mu + mv;                                   // mu + mv
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int64_t job = blockIdx.x; job < a.njobs; job += gridDim.x) {
    const UQSrc src = uq_src(a, job);
    if (!src.on) continue;  // uniform across the CTA
    double sa = 0.0, sb = 0.0, cnt = 0.0;
    for (int k = tid; k < n; k += UQ_THREADS) {
      const int p = k % wr, q = k / wr;
      const int64_t off = (int64_t)(src.rs + p) + (int64_t)(src.cs + q) * src.ld;
      const float va = src.A[off], vb = src.B[off];
      const bool mk = src.M ? src.M[off] != 0 : false;
      wa[k] = mk ? __int_as_float(0x7fc00000) : va;  // NaN marks a masked pixel until the means are known
      wb[k] = vb;
      if (!mk) {
        sa += (double)va;
        sb += (double)vb;
        cnt += 1.0;
      }
    }
    sa = warp_sum(sa);
    sb = warp_sum(sb);
    cnt = warp_sum(cnt);
    if (lane == 0) {
      part[3 * warp] = sa;
      part[3 * warp + 1] = sb;
      part[3 * warp + 2] = cnt;
    }
    __syncthreads();
    double ta = 0, tb = 0, tn = 0;
    for (int w = 0; w < UQ_THREADS / 32; ++w) {
      ta += part[3 * w];
      tb += part[3 * w + 1];
      tn += part[3 * w + 2];
    }
    const float ma = tn > 0 ? (float)(ta / tn) : 0.f, mb = tn > 0 ? (float)(tb / tn) : 0.f;
    for (int k = tid; k < n; k += UQ_THREADS) {
      const int p = k % wr, q = k / wr;
      const int64_t off = (int64_t)(src.rs + p) + (int64_t)(src.cs + q) * src.ld;
      const bool mk = src.M ? src.M[off] != 0 : false;
      const float ap = a.apod[k];
      const float va = src.A[off];
      wa[k] = mk ? 0.f : __fmul_rn(ap, __fsub_rn(va, ma));
      wb[k] = mk ? 0.f : __fmul_rn(ap, __fsub_rn(wb[k], mb));
    }
    __syncthreads();
    // dC = a0 b1 - a1 b0 per component
    for (int k = tid; k < mu + mv; k += UQ_THREADS) {
      const int comp = k >= mu, e = comp ? k - mu : k;
      const UQGeom g = uq_geom(comp, wr, wc);
      const int r = e % g.R, c = e / g.R;
      const float a0 = wa[r * g.sr_ + c * g.sc_], a1 = wa[r * g.sr_ + (c + 1) * g.sc_];
      const float b0 = wb[r * g.sr_ + c * g.sc_], b1 = wb[r * g.sr_ + (c + 1) * g.sc_];
      dC[k] = __fsub_rn(__fmul_rn(a0, b1), __fmul_rn(a1, b0));
    }
    __syncthreads();
    double s0 = 0.0, s1 = 0.0;
    for (int k = tid; k < mu + mv; k += UQ_THREADS) {
      const int comp = k >= mu, e = comp ? k - mu : k;
      const UQGeom g = uq_geom(comp, wr, wc);
      const float* d = dC + (comp ? mu : 0);
      const int r = e % g.R, c = e / g.R;
      const int cl = c > 0 ? c - 1 : 0, cr = c < g.m - 1 ? c + 1 : g.m - 1;
      const float v = __fmul_rn(0.25f, __fadd_rn(__fadd_rn(d[r + cl * g.R], __fmul_rn(2.0f, d[r + c * g.R])), d[r + cr * g.R]));
      dCs[k] = v;
      if (comp == 0) s0 += (double)v;
      else s1 += (double)v;
    }
    s0 = warp_sum(s0);
    s1 = warp_sum(s1);
    __syncthreads();  // part reused
    if (lane == 0) {
      part[3 * warp] = s0;
      part[3 * warp + 1] = s1;
    }
    __syncthreads();
    double mu0 = 0, mu1 = 0;
    for (int w = 0; w < UQ_THREADS / 32; ++w) {
      mu0 += part[3 * w];
      mu1 += part[3 * w + 1];
    }
    mu0 /= (double)mu;
    mu1 /= (double)mv;
    for (int k = tid; k < mu + mv; k += UQ_THREADS) dd[k] = (double)dCs[k] - (k < mu ? mu0 : mu1);
    __syncthreads();
    // the 2 x 44 statistics, one warp per statistic (uq_component!, :104-151)
    for (int st = warp; st < 88; st += UQ_THREADS / 32) {
      const int comp = st / 44, si = st % 44;
      const UQGeom g = uq_geom(comp, wr, wc);
      const double* d = dd + (comp ? mu : 0);
      const int WM = g.R * g.m;
      double acc = 0.0;
      if (si < 3) {
        for (int t = lane; t < WM; t += 32) {
          const int r = t % g.R, c = t / g.R;
          const float a0 = wa[r * g.sr_ + c * g.sc_], a1 = wa[r * g.sr_ + (c + 1) * g.sc_];
          const float b0 = wb[r * g.sr_ + c * g.sc_], b1 = wb[r * g.sr_ + (c + 1) * g.sc_];
          const float pr = si == 0 ? __fmul_rn(a0, b0) : (si == 1 ? __fmul_rn(a0, b1) : __fmul_rn(a1, b0));
          acc += (double)pr;
        }
      } else if (si == 3) {
        for (int t = lane; t < WM; t += 32) acc = fma(d[t], d[t], acc);
      } else {
        const int k = si - 4, dr = o.dr[k], dc = o.dc[k];
        const int c0 = dc < 0 ? -dc : 0, c1 = dc > 0 ? g.m - dc : g.m;  // c in [c0, c1)
        const int r0 = dr < 0 ? -dr : 0, r1 = dr > 0 ? g.R - dr : g.R;  // r in [r0, r1)
        const int nrr = r1 - r0, ncc = c1 - c0;
        for (int t = lane; t < nrr * ncc; t += 32) {
          const int r = r0 + t % nrr, c = c0 + t / nrr;
          acc = fma(d[r + c * g.R], d[(r + dr) + (c + dc) * g.R], acc);
        }
      }
      acc = warp_sum(acc);
      if (lane == 0) stats[st] = acc;
    }
    __syncthreads();
    if (a.stats)
      for (int it = tid; it < 88; it += UQ_THREADS) {
        if (a.accumulate) a.stats[job * 88 + it] += stats[it];
        else a.stats[job * 88 + it] = stats[it];
      }
    if (a.unc_u && tid < 2) {
      const float sg = uq_finalize(stats + 44 * tid, o);
      if (tid == 0) a.unc_u[src.gid] = sg;
      else a.unc_v[src.gid] = sg;
    }
    __syncthreads();
  }
}

template <int W> static cudaError_t launch_uq_warp(const UQArgs& a, cudaStream_t s, int num_sms, const UQOffsets& offs) {
  using C = UQWCfg<W>;
  const size_t sm = C::smem();
  cudaError_t e = cudaFuncSetAttribute(uq_warp_kernel<W>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, uq_warp_kernel<W>, UQW_THREADS, sm);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * num_sms;
  const int64_t units = (a.njobs + C::NWIN - 1) / C::NWIN;
  if (grid > units) grid = units;
  uq_warp_kernel<W><<<(unsigned)grid, UQW_THREADS, sm, s>>>(a, offs);
  return cudaGetLastError();
}

cudaError_t launch_uq(const UQArgs& a, cudaStream_t s, int num_sms) {
  if (a.njobs <= 0) return cudaSuccess;
  static const UQOffsets offs = make_offsets();
  const int wc = a.Wc > 0 ? a.Wc : a.W;
  if (uq_general(a.W, wc)) {
    if (!a.gscr || a.gscr_slices < 1 || a.gscr_stride < uq_general_stride(a.W, wc) || a.W < 2 || wc < 2)
      return cudaErrorInvalidValue;
    const int64_t grid = a.njobs < a.gscr_slices ? a.njobs : a.gscr_slices;
    uq_general_kernel<<<(unsigned)grid, UQ_THREADS, 0, s>>>(a, offs);
    return cudaGetLastError();
  }
  switch (a.W) {
    case 8: return launch_uq_warp<8>(a, s, num_sms, offs);
    case 12: return launch_uq_warp<12>(a, s, num_sms, offs);
    case 16: return launch_uq_warp<16>(a, s, num_sms, offs);
    case 24: return launch_uq_warp<24>(a, s, num_sms, offs);
    case 32: return launch_uq_warp<32>(a, s, num_sms, offs);
    default: break;
  }
  auto smem_of = [](int W) {
    const int WM = W * (W - 1);
    return (size_t)(2 * WM + 88 + 12) * sizeof(double) + (size_t)(2 * W * W + 4 * WM) * sizeof(float) +
           (size_t)W * W + 16;
  };
  const size_t sm = smem_of(a.W);
  if (a.W > 64 || sm > 220 * 1024) return cudaErrorInvalidValue;
  // one attribute for every window size this kernel serves: the limit is a
  // property of the function, and launches of different sizes may share a graph
  cudaError_t e = cudaFuncSetAttribute(uq_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_of(64));
  if (e != cudaSuccess) return e;
  int per_sm = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, uq_kernel, UQ_THREADS, sm);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) per_sm = 1;
  int64_t grid = (int64_t)per_sm * num_sms;
  if (grid > a.njobs) grid = a.njobs;
  uq_kernel<<<(unsigned)grid, UQ_THREADS, sm, s>>>(a, offs);
  return cudaGetLastError();
}

cudaError_t launch_uq_finalize(const double* stats, const int32_t* jobs, int64_t njobs, int32_t ny, float* unc_u,
                               float* unc_v, cudaStream_t s) {
  if (njobs <= 0) return cudaSuccess;
  static const UQOffsets offs = make_offsets();
  int64_t blocks = (2 * njobs + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  uq_finalize_kernel<<<(unsigned)blocks, 256, 0, s>>>(stats, jobs, njobs, ny, unc_u, unc_v, offs);
  return cudaGetLastError();
}

}  // namespace hh
