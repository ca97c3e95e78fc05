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
// registers, so the smoothing along the columns and the 40 half-plane
// covariance sums are register FMAs plus one shuffle per neighbour column
// and row; the per-lane partial sums are combined through shared memory in
// a fixed order. Same FP32 operations as uq_kernel, FP64 sums.
// When dC has at most 16 columns (W <= 17) a warp serves two windows, one
// per 16-lane segment (shuffles of width 16), so no lane idles for want of
// a column.
constexpr int UQW_THREADS = 128;  // two warp pairs (u, v)

template <int W> struct UQWCfg {
  static constexpr int LD = W + 1;  // odd column stride: conflict-free column and row walks
  static constexpr int M = W - 1;   // columns of dC
  static constexpr int WPW = M <= 16 ? 2 : 1;  // windows per warp
  static constexpr int SEG = 32 / WPW;         // lanes per window
  static constexpr int NWIN = 2 * WPW;         // windows per CTA
  // window buffers of consecutive slots start 16 banks apart (64 bytes mod
  // 128), so the two windows of a warp do not meet in one bank
  static constexpr size_t win_raw = 2 * (size_t)LD * W * sizeof(float) + (size_t)W * W;
  static constexpr size_t win_bytes = (win_raw + 127) / 128 * 128 + 64;
  static constexpr size_t part_bytes = (44 * 33 + 44 * WPW) * sizeof(double);  // per warp: partials + totals
  // the next windows are copied in (cp.async) while the current ones are
  // reduced, into a second set of buffers (timed: faster up to 16 px, no
  // gain at 24 px, and at 32 px the buffers would cost a CTA per SM)
  static constexpr bool PREFETCH = W <= 16;
  static constexpr int NBUF = PREFETCH ? 2 : 1;
  static constexpr size_t smem() { return NBUF * NWIN * win_bytes + 4 * part_bytes + sizeof(UQOffsets) + 16; }
  static constexpr int MINB = 3;  // CTAs per SM the register budget is sized for
};

// sum over the lanes of one SEG-lane segment
template <int SEG> __device__ __forceinline__ double seg_sum(double v) {
#pragma unroll
  for (int o = SEG / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
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
  constexpr int LD = C::LD, M = C::M, WPW = C::WPW, SEG = C::SEG, NWIN = C::NWIN;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* part_all = reinterpret_cast<double*>(smem_raw);  // [warp][44][33] + totals
  unsigned char* wbase = smem_raw + 4 * C::part_bytes;
  // the offset tables in shared memory (indexed at run time; a parameter
  // struct indexed that way would be copied to local memory)
  UQOffsets& so = *reinterpret_cast<UQOffsets*>(wbase + C::NBUF * NWIN * C::win_bytes);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (tid == 0) so = o;
  __syncthreads();
  const int comp = warp & 1, seg = lane / SEG, c = lane % SEG;
  const int slot = (warp >> 1) * WPW + seg;  // window of this lane
  const int ts = comp * SEG + c;             // this lane among the 2*SEG threads of its window
  double* part = part_all + warp * (C::part_bytes / sizeof(double));
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
  if (C::PREFETCH) {
    const int64_t base0 = (int64_t)blockIdx.x * NWIN;
    if (base0 < a.njobs) prefetch(uq_src(a, base0 + slot), 0);
    cp_async_commit();
  }
  for (int64_t base = (int64_t)blockIdx.x * NWIN; base < a.njobs; base += stride, ++iter) {
    const int64_t job = base + slot;
    const int ph = C::PREFETCH ? (iter & 1) : 0;
    float* wa = reinterpret_cast<float*>(wbase + (ph * NWIN + slot) * C::win_bytes);  // W x W, column stride LD
    float* wb = wa + LD * W;
    uint8_t* mf = reinterpret_cast<uint8_t*>(wb + LD * W);
    // ---- the window's source (uniform within the window's lanes)
    const UQSrc src = uq_src(a, job);
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
      if (base + stride < a.njobs) prefetch(uq_src(a, base + stride + slot), ph ^ 1);
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
    // ---- window means (load_uncertainty_windows!), FP64, computed by each warp
    float ma = 0.f, mb = 0.f;
    if (run) {
      double sa = 0.0, sb = 0.0, cnt = 0.0;
      for (int k = c; k < W * W; k += SEG)
        if (!mf[k]) {
          const int p = k % W, q = k / W;
          sa += (double)wa[p + q * LD];
          sb += (double)wb[p + q * LD];
          cnt += 1.0;
        }
      sa = seg_sum<SEG>(sa);
      sb = seg_sum<SEG>(sb);
      cnt = seg_sum<SEG>(cnt);
      ma = cnt > 0 ? (float)(sa / cnt) : 0.f;
      mb = cnt > 0 ? (float)(sb / cnt) : 0.f;
    }
    __syncthreads();  // every read of the raw values precedes the apodized writes
    if (run)
      for (int k = ts; k < W * W; k += 2 * SEG) {
        const int p = k % W, q = k / W;
        const float ap = __ldg(a.apod + k);
        const float va = wa[p + q * LD], vb = wb[p + q * LD];
        wa[p + q * LD] = mf[k] ? 0.f : __fmul_rn(ap, __fsub_rn(va, ma));
        wb[p + q * LD] = mf[k] ? 0.f : __fmul_rn(ap, __fsub_rn(vb, mb));
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
      double msum = 0.0;
#pragma unroll
      for (int r = 0; r < W; ++r) {
        const float left = __shfl_up_sync(FULL, dcol[r], 1, SEG);
        const float right = __shfl_down_sync(FULL, dcol[r], 1, SEG);
        const float l = c > 0 ? left : dcol[r];
        const float rr = c < M - 1 ? right : dcol[r];
        const float v = __fmul_rn(0.25f, __fadd_rn(__fadd_rn(l, __fmul_rn(2.0f, dcol[r])), rr));
        dd[r] = (double)v;
        if (col) msum += dd[r];
      }
      const double mu = seg_sum<SEG>(msum) / (double)(W * M);
#pragma unroll
      for (int r = 0; r < W; ++r) dd[r] = col ? dd[r] - mu : 0.0;
      // ---- S00 and the covariance sums: acc[dc][dr + 4] pairs (r, c) with
      //      (r + dr, c + dc). Two neighbour columns at a time, so only 18
      //      accumulators are live; each group's per-lane partials go to
      //      shared [stat][lane] in natural order.
      part[0 * 33 + lane] = s0;
      part[1 * 33 + lane] = s1;
      part[2 * 33 + lane] = s2;
      {
        double sq = 0.0, acc0[4] = {0.0, 0.0, 0.0, 0.0};
#pragma unroll
        for (int r = 0; r < W; ++r) {
          sq = fma(dd[r], dd[r], sq);
#pragma unroll
          for (int dr = 1; dr <= 4; ++dr)
            if (r + dr < W) acc0[dr - 1] = fma(dd[r], dd[r + dr], acc0[dr - 1]);
        }
        part[3 * 33 + lane] = sq;
#pragma unroll
        for (int i = 0; i < 4; ++i) part[(4 + i) * 33 + lane] = acc0[i];
      }
#pragma unroll
      for (int dg = 1; dg <= 3; dg += 2) {
        double acc[2][9];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int jj = 0; jj < 9; ++jj) acc[i][jj] = 0.0;
#pragma unroll
        for (int i = 0; i < 2; ++i) {
          const int dc = dg + i;
          const bool ok = c + dc < M;
#pragma unroll
          for (int r2 = 0; r2 < W; ++r2) {
            double x = __shfl_down_sync(FULL, dd[r2], dc, SEG);
            x = ok ? x : 0.0;
#pragma unroll
            for (int dr = -4; dr <= 4; ++dr) {
              const int r0 = r2 - dr;
              if (r0 >= 0 && r0 < W) acc[i][dr + 4] = fma(dd[r0], x, acc[i][dr + 4]);
            }
          }
        }
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
          for (int jj = 0; jj < 9; ++jj) part[(8 + 9 * (dg - 1 + i) + jj) * 33 + lane] = acc[i][jj];
      }
      __syncwarp();
      // ---- per window and statistic, the sum of the M column lanes' partials
      //      in lane order (the other lanes hold zeros)
      double* tot = part + 44 * 33;
      bool on_s[WPW];
      int64_t job_s[WPW];
#pragma unroll
      for (int g = 0; g < WPW; ++g) {
        on_s[g] = __shfl_sync(FULL, on, g * SEG);
        job_s[g] = base + (warp >> 1) * WPW + g;
      }
      for (int j = lane; j < 44 * WPW; j += 32) {
        const int g = j / 44, st = j % 44;
        double t = 0.0;
        for (int l = 0; l < (WPW == 1 ? 32 : M); ++l) t += part[st * 33 + g * SEG + l];
        const int ri = st < 4 ? st : 4 + so.nat2ring[st - 4];
        tot[g * 44 + ri] = t;
        bool og = on_s[0];
        int64_t jg = job_s[0];
#pragma unroll
        for (int h = 1; h < WPW; ++h)
          if (g == h) {
            og = on_s[h];
            jg = job_s[h];
          }
        if (og && a.stats) {
          if (a.accumulate) a.stats[jg * 88 + comp * 44 + ri] += t;
          else a.stats[jg * 88 + comp * 44 + ri] = t;
        }
      }
      __syncwarp();
      if (c == 0 && on && a.unc_u) (comp == 0 ? a.unc_u : a.unc_v)[gid] = uq_finalize(tot + seg * 44, so);
    }
    __syncthreads();  // the window buffers are reused by the next iteration
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
