// General-shape window correlation (sm_100a), included by k_correlate.cu.
//
// The fused kernels of k_correlate.cu hold a whole plane in shared memory and
// are specialised per (FFT size, window). This kernel takes every other case
// the reference's correlators accept (src/correlators.jl:42-129, 188-355):
//   - FFT planes that do not fit a CTA: padded 128-px windows (256 x 256), or
//     larger;
//   - any window size, not only the specialised ones: FFT lengths with prime
//     factors up to 61 (FFTW plans any size; 2, 3 and 5 cover the usual ones);
//   - rectangular windows and search areas (window_size / search_area_size
//     tuples, src/types.jl:254-257), padded or not.
// One CTA per window (grid-stride over jobs) works on its own slice of a
// global scratch buffer -- the complex plane and the real correlation plane,
// about 0.8 MB for a 256 x 256 plane, so 148 slices stay resident in L2:
//   1. window means in FP64 (masked pixels excluded), then the data columns
//      of the packed plane Z = A + iB (mean-subtracted, apodized, zero-padded,
//      load_windows!) transformed along the rows axis, built directly from the
//      images (only the search-area columns are nonzero);
//   2. for each row pair (r, -r): both rows transformed along the columns
//      axis, the cross-power (or filtered phase) spectrum of each row formed
//      from Z(k) and Z(-k) (spectrum!), and both rows transformed back;
//   3. the columns transformed back, scaled by 1/(nr nc) like FFTW's inverse
//      plan, |.|, fftshifted, multiplied by the overlap gain, search lags
//      restricted (fftshift_abs!, restrict_search_lags!) into the real plane;
//   4. the plane analysed by the whole CTA (analyze_group: the same peak
//      search, subpixel fit, ratio, moment and alternatives as the fused
//      kernels).
// Lines are transformed in shared memory, one warp per line, by a Stockham
// (self-sorting) mixed-radix FFT with twiddles from a per-length table
// exp(-2 pi i t / n) computed in double and rounded once.
// (Included inside namespace hh, after analyze_group and cross_spectrum.)
#pragma once

constexpr int GC_THREADS = 512;
constexpr int GC_WARPS = GC_THREADS / 32;

// exp(-+2 pi i t / n) from the length-n table (inverse: the conjugate)
__device__ __forceinline__ float2 gc_tw(const float2* tw, int t, bool inv) {
  const float2 w = __ldg(tw + t);
  return inv ? make_float2(w.x, -w.y) : w;
}

// One radix-r Stockham stage of a length-n line: in -> out, p = product of
// the radices before this one (pm = p - 1 when p is a power of two, else
// -1), nr = n / r, tstep = n / (p r). Butterfly i (k = i mod p) reads
// in[i + m nr], applies the twiddles exp(-+2 pi i m k / (p r)), takes the
// r-point DFT and writes out[(i - k) r + k + q p].
__device__ __forceinline__ void gc_stage(const float2* __restrict__ in, float2* __restrict__ out, int r, int p, int pm,
                                         int nr, int tstep, const float2* tw, bool inv, int lane) {
  for (int i = lane; i < nr; i += 32) {
    const int k = pm >= 0 ? (i & pm) : i % p, j0 = (i - k) * r + k;
    if (r == 2) {
      float2 x0 = in[i], x1 = in[i + nr];
      if (k) x1 = cmul(x1, gc_tw(tw, k * tstep, inv));
      out[j0] = make_float2(x0.x + x1.x, x0.y + x1.y);
      out[j0 + p] = make_float2(x0.x - x1.x, x0.y - x1.y);
    } else if (r == 4) {
      float2 x0 = in[i], x1 = in[i + nr], x2 = in[i + 2 * nr], x3 = in[i + 3 * nr];
      if (k) {
        x1 = cmul(x1, gc_tw(tw, k * tstep, inv));
        x2 = cmul(x2, gc_tw(tw, 2 * k * tstep, inv));
        x3 = cmul(x3, gc_tw(tw, 3 * k * tstep, inv));
      }
      const float2 a = make_float2(x0.x + x2.x, x0.y + x2.y), b = make_float2(x0.x - x2.x, x0.y - x2.y);
      const float2 c = make_float2(x1.x + x3.x, x1.y + x3.y), d = make_float2(x1.x - x3.x, x1.y - x3.y);
      // forward: y1 = b - i d, y3 = b + i d; inverse swaps the signs of i
      const float2 md = inv ? make_float2(-d.y, d.x) : make_float2(d.y, -d.x);  // -+ i d
      out[j0] = make_float2(a.x + c.x, a.y + c.y);
      out[j0 + p] = make_float2(b.x + md.x, b.y + md.y);
      out[j0 + 2 * p] = make_float2(a.x - c.x, a.y - c.y);
      out[j0 + 3 * p] = make_float2(b.x - md.x, b.y - md.y);
    } else {
      // any other radix (3, 5, 7, ...): the r outputs summed directly, the
      // twiddled inputs read from shared memory (no register array); the
      // exponent e = m q mod r is stepped, not divided
      const int rstep = nr;  // n / r
      for (int q = 0; q < r; ++q) {
        float2 acc = make_float2(0.f, 0.f);
        int e = 0;
        for (int m = 0; m < r; ++m) {
          float2 x = in[i + m * nr];
          if (k && m) x = cmul(x, gc_tw(tw, m * k * tstep, inv));
          if (e) x = cmul(x, gc_tw(tw, e * rstep, inv));
          acc.x += x.x;
          acc.y += x.y;
          e += q;
          if (e >= r) e -= r;
        }
        out[j0 + q * p] = acc;
      }
    }
  }
}

// Length-n transform of one line held by a warp in buf0 (buf1 is the
// ping-pong partner); returns the buffer that holds the result.
__device__ __forceinline__ float2* gc_line(float2* buf0, float2* buf1, int n, const int8_t* radix, int nst,
                                           const float2* tw, bool inv, int lane) {
  float2* in = buf0;
  float2* out = buf1;
  int p = 1;
  for (int s = 0; s < nst; ++s) {
    const int r = radix[s];
    const int nr = n / r;  // once per stage, not per butterfly
    gc_stage(in, out, r, p, (p & (p - 1)) == 0 ? p - 1 : -1, nr, nr / p, tw, inv, lane);
    __syncwarp();
    p *= r;
    float2* t = in;
    in = out;
    out = t;
  }
  return in;
}

// Lengths n = 16 B (B = 2, 4, 8, 16: n = 32 .. 256) are transformed in
// registers by half a warp (hl = lane within the half): the four-step split
// n = 16 B with input index B n1 + n2 and output index k1 + 16 k2 -- a
// 16-point DFT over n1 per n2 (lanes n2 < B), the twiddle W_n^(n2 k1), a
// B-point DFT over n2 per k1 (lanes k1 < 16) -- with one exchange through
// `tmp` (row k1 padded to B + 1, so both access patterns are conflict-free).
// The result overwrites `line`. Two lines per warp, one per half.
template <int B, bool INV>
__device__ __forceinline__ void gc_fft16(float2* line, float2* tmp, const float2* tw, int hl, bool act) {
  if (act && hl < B) {
    float2 x[16];
#pragma unroll
    for (int n1 = 0; n1 < 16; ++n1) x[n1] = line[B * n1 + hl];
    RDFT<16, INV>::run(x, 16);
#pragma unroll
    for (int k1 = 0; k1 < 16; ++k1) {
      float2 v = x[k1];
      if (k1 && hl) v = cmul(v, gc_tw(tw, hl * k1, INV));
      tmp[k1 * (B + 1) + hl] = v;
    }
  }
  __syncwarp();
  if (act) {
    float2 t[B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) t[n2] = tmp[hl * (B + 1) + n2];
    RDFT<B, INV>::run(t, B);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) line[hl + 16 * k2] = t[k2];
  }
  __syncwarp();
}

// n = 32, 64, 128 or 256: the register form applies
__host__ __device__ __forceinline__ bool gc_reg_len(int n) { return n == 32 || n == 64 || n == 128 || n == 256; }

template <bool INV>
__device__ __forceinline__ void gc_fft16_n(float2* line, float2* tmp, int n, const float2* tw, int hl, bool act) {
  switch (n) {
    case 32: gc_fft16<2, INV>(line, tmp, tw, hl, act); break;
    case 64: gc_fft16<4, INV>(line, tmp, tw, hl, act); break;
    case 128: gc_fft16<8, INV>(line, tmp, tw, hl, act); break;
    default: gc_fft16<16, INV>(line, tmp, tw, hl, act); break;
  }
}

__global__ void __launch_bounds__(GC_THREADS, 1) correlate_general_kernel(const CorrArgs a) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int NR = a.nfr, NC = a.nfc, wr = a.wr, wc = a.wc, sr = a.sr, sc = a.sc;
  // staged line strides (float2): room for the register form's padded exchange
  const int LDR = NR + 16, LDC = NC + 16;
  const bool regR = gc_reg_len(NR), regC = gc_reg_len(NC);  // register-form lengths
  const int hw = (threadIdx.x & 31) >> 4, hl = threadIdx.x & 15;  // half-warp, lane within it
  const int CC = a.gc_chunk_c;  // rows-pass lines per chunk (length NC); the columns passes use a.gc_col_warps warps
  const size_t lines_b = a.gc_smem_lines;
  float2* buf0 = reinterpret_cast<float2*>(smem_raw);
  float2* buf1 = reinterpret_cast<float2*>(smem_raw + lines_b / 2);
  double* part = reinterpret_cast<double*>(smem_raw + lines_b);  // GC_WARPS x 4
  uint32_t* red = reinterpret_cast<uint32_t*>(part + 4 * GC_WARPS);
  float* s_vals = reinterpret_cast<float*>(red + GC_WARPS * 2 * KMAX);
  int* s_locs = reinterpret_cast<int*>(s_vals + KMAX);

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int K = a.npeaks > 2 ? a.npeaks : 2;
  const int64_t P = (int64_t)NR * NC;
  float2* Z = a.gscr + (int64_t)blockIdx.x * a.gscr_stride;  // complex plane, column-major, ld NR
  float* R = reinterpret_cast<float*>(Z + P);                 // real plane, column-major, ld NR
  const int oar = (sr - wr) / 2, oac = (sc - wc) / 2;  // frame-A window inside the search area
  const bool search = sr != wr || sc != wc;
  const float scale = 1.0f / (float)P;
  // rows / columns of the fftshifted plane that can be nonzero; outside this
  // box the gain (or the kept-lag restriction) makes the plane exactly zero,
  // so its columns skip the last inverse transform and the peak scan covers
  // the box (plus the last pixel, the one place outside where a zero can be
  // a regional maximum), as in the fused kernels
  const int rlo = a.gc_box[0], rhi = a.gc_box[1], clo = a.gc_box[2], chi = a.gc_box[3];
  const ScanPlan sp = scan_plan(tid, GC_THREADS, rlo, rhi, clo, chi);
  PeakOut po{a.du, a.dv, a.ratio, a.moment, a.alt_u, a.alt_v, a.nalt, a.G, a.packed, a.locs};

  // the real plane outside the box's columns is zero for every window of
  // this launch (the box is the launch's): cleared once here, never rewritten
  for (int c = warp; c < NC; c += GC_WARPS) {
    const int js = c;
    if (js >= clo && js <= chi) continue;
    float* rc = R + (int64_t)js * NR;
    for (int i = lane; i < NR; i += 32) rc[i] = 0.f;
  }
  __syncthreads();

  for (int64_t job = blockIdx.x; job < a.njobs; job += gridDim.x) {
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
      if (!bp_live(b, a.it, a.done, p) || (b.gmask && b.gmask[cell])) continue;  // uniform across the CTA
      const bool warped = a.it > 1 || b.has_pred0;
      A = warped ? b.warpA : b.A;
      B = warped ? b.warpB : b.B;
      M = b.mask;
      ld = b.nr;
      gid = b.goff + cell;
      pw.G = (int64_t)b.ny * b.nx;
      pw.nalt = b.nalt;
      pw.alt_u = a.alt_u ? a.alt_u + b.aoff - b.goff : nullptr;
      pw.alt_v = a.alt_v ? a.alt_v + b.aoff - b.goff : nullptr;
    } else {
      gid = (int64_t)a.jobs[4 * job] + (int64_t)a.jobs[4 * job + 1] * a.ny;
    }
    rs = a.jobs[4 * job + 2];
    cs = a.jobs[4 * job + 3];
    // search-area origin: the window's origin less the centring offset
    const int64_t r0 = (int64_t)rs - oar, c0 = (int64_t)cs - oac;

    // ---- 1a. means over the unmasked pixels (FP64, one rounding)
    double sa = 0.0, sb = 0.0, na = 0.0, nb = 0.0;
    for (int j = warp; j < sc; j += GC_WARPS)  // warps on columns, lanes down the rows
      for (int i = lane; i < sr; i += 32) {
        const int64_t off = (r0 + i) + (c0 + j) * ld;
        if (M && __ldg(M + off)) continue;
        sb += (double)__ldg(B + off);
        nb += 1.0;
        if ((unsigned)(i - oar) < (unsigned)wr && (unsigned)(j - oac) < (unsigned)wc) {
          sa += (double)__ldg(A + off);
          na += 1.0;
        }
      }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      sa += __shfl_xor_sync(0xffffffffu, sa, o);
      sb += __shfl_xor_sync(0xffffffffu, sb, o);
      na += __shfl_xor_sync(0xffffffffu, na, o);
      nb += __shfl_xor_sync(0xffffffffu, nb, o);
    }
    if (lane == 0) {
      part[4 * warp] = sa;
      part[4 * warp + 1] = sb;
      part[4 * warp + 2] = na;
      part[4 * warp + 3] = nb;
    }
    __syncthreads();
    double ta = 0.0, tb = 0.0, tna = 0.0, tnb = 0.0;
    for (int w = 0; w < GC_WARPS; ++w) {
      ta += part[4 * w];
      tb += part[4 * w + 1];
      tna += part[4 * w + 2];
      tnb += part[4 * w + 3];
    }
    const float ma = tna > 0 ? (float)(ta / tna) : 0.f, mb = tnb > 0 ? (float)(tb / tnb) : 0.f;
    const bool bad = !(isfinite(ta) && isfinite(tb));  // the window holds NaN or Inf: the reference's plane is NaN

    // ---- 1b. data columns j < sc of Z, transformed along the rows axis;
    //      each warp builds, transforms and stores its own columns (two at a
    //      time, one per half-warp, in the register form), so no CTA barrier
    //      is needed
    if (warp < a.gc_col_warps) {
      const int lpw = regR ? 2 : 1;  // lines per warp at a time
      float2* wbuf = buf0 + (size_t)warp * 2 * lpw * LDR;
      for (int jb = warp * lpw; jb < sc; jb += a.gc_col_warps * lpw) {
        const int j = jb + (regR ? hw : 0);
        const bool act = j < sc;
        const int i0 = regR ? hl : lane, st = regR ? 16 : 32;
        float2* l0 = wbuf + (regR ? hw * 2 * LDR : 0);
        float2* l1 = l0 + LDR;
        if (act) {
#pragma unroll 4
          for (int i = i0; i < NR; i += st) {
            float2 z = make_float2(0.f, 0.f);
            if (i < sr && !bad) {
              const int64_t off = (r0 + i) + (c0 + j) * ld;
              if (!(M && __ldg(M + off))) {
                const int ia = i - oar, ja = j - oac;
                const bool ina = (unsigned)ia < (unsigned)wr && (unsigned)ja < (unsigned)wc;
                if (search) {
                  z.y = __ldg(B + off) - mb;
                  if (ina) z.x = __ldg(a.apod + ia + ja * wr) * (__ldg(A + off) - ma);
                } else {
                  const float ap = __ldg(a.apod + i + j * wr);
                  z = make_float2(ap * (__ldg(A + off) - ma), ap * (__ldg(B + off) - mb));
                }
              }
            }
            l0[i] = z;
          }
        }
        __syncwarp();
        const float2* res = l0;
        if (regR) gc_fft16_n<false>(l0, l1, NR, a.twr, hl, act);
        else res = gc_line(l0, l1, NR, a.gc_radix_r, a.gc_nst_r, a.twr, false, lane);
        if (act) {
          float2* zc = Z + (int64_t)j * NR;
          for (int i = i0; i < NR; i += st) zc[i] = res[i];
        }
        __syncwarp();
      }
    }
    __syncthreads();

    // ---- 2. row pairs (r, -r): forward along columns, spectrum, inverse
    const int half = NR / 2;  // rows 0..half, each with its partner (NR - r) % NR
    const int CH = CC / 2;
    for (int h0 = 0; h0 <= half; h0 += CH) {
      const int nh = min(CH, half + 1 - h0);
      // lanes on the chunk's rows (consecutive rows and their partners), warps
      // on the columns: the reads of a column are two contiguous runs
      for (int l0 = lane; l0 < 2 * nh; l0 += 32) {
        const int ra = h0 + (l0 >> 1), row = (l0 & 1) ? (NR - ra) % NR : ra;
#pragma unroll 8
        for (int j = warp; j < NC; j += GC_WARPS)
          buf0[l0 * LDC + j] = j < sc ? Z[(int64_t)j * NR + row] : make_float2(0.f, 0.f);
      }
      __syncthreads();
      if (regC) {  // two lines per warp (its row pair), one per half-warp
        const int l = 2 * warp + hw;
        gc_fft16_n<false>(buf0 + l * LDC, buf1 + l * LDC, NC, a.twc, hl, l < 2 * nh);
      } else {
        for (int l = warp; l < 2 * nh; l += GC_WARPS)
          gc_line(buf0 + l * LDC, buf1 + l * LDC, NC, a.gc_radix_c, a.gc_nst_c, a.twc, false, lane);
      }
      __syncthreads();
      // the register form leaves its result in place
      float2* fz = (!regC && (a.gc_nst_c & 1)) ? buf1 : buf0;  // forward rows
      float2* sz = (!regC && (a.gc_nst_c & 1)) ? buf0 : buf1;  // spectrum rows
      for (int l = warp; l < 2 * nh; l += GC_WARPS) {
        const int ra = h0 + (l >> 1), row = (l & 1) ? (NR - ra) % NR : ra;
        const float2* Za = fz + l * LDC;          // this row
        const float2* Zb = fz + (l ^ 1) * LDC;    // its partner row (-r)
        for (int k2 = lane; k2 < NC; k2 += 32) {
          const float wk = a.phasew ? __ldg(a.phasew + row + (int64_t)k2 * NR) : 1.f;
          sz[l * LDC + k2] = cross_spectrum(Za[k2], Zb[k2 == 0 ? 0 : NC - k2], a.method, wk);
        }
      }
      __syncthreads();
      if (regC) {
        const int l = 2 * warp + hw;
        gc_fft16_n<true>(sz + l * LDC, fz + l * LDC, NC, a.twc, hl, l < 2 * nh);
      } else {
        for (int l = warp; l < 2 * nh; l += GC_WARPS)
          gc_line(sz + l * LDC, fz + l * LDC, NC, a.gc_radix_c, a.gc_nst_c, a.twc, true, lane);
      }
      __syncthreads();
      float2* iz = (!regC && (a.gc_nst_c & 1)) ? fz : sz;
      for (int l0 = lane; l0 < 2 * nh; l0 += 32) {
        const int ra = h0 + (l0 >> 1), row = (l0 & 1) ? (NR - ra) % NR : ra;
        if ((l0 & 1) && row == ra) continue;  // a self-paired row (0, NR/2) is written once
#pragma unroll 4
        for (int j = warp; j < NC; j += GC_WARPS) {
          const int js = j + NC / 2 < NC ? j + NC / 2 : j + NC / 2 - NC;
          if (js < clo || js > chi) continue;  // a column that step 3 writes as zeros
          Z[(int64_t)j * NR + row] = iz[l0 * LDC + j];
        }
      }
      __syncthreads();
    }

    // ---- 3. columns back, then |.| / (nr nc), fftshift, gain, kept lags;
    //      columns whose shifted position lies outside the box are zero
    //      (those columns were cleared at the start of the launch)
    const int nbox = chi - clo + 1;
    //      the box's columns, one warp each: unshifted column j = (js - NC/2) mod NC
    if (warp < a.gc_col_warps) {
      const int lpw = regR ? 2 : 1;
      float2* wbuf = buf0 + (size_t)warp * 2 * lpw * LDR;
      for (int bb = warp * lpw; bb < nbox; bb += a.gc_col_warps * lpw) {
        const int b = bb + (regR ? hw : 0);
        const bool act = b < nbox;
        const int i0 = regR ? hl : lane, st = regR ? 16 : 32;
        float2* l0 = wbuf + (regR ? hw * 2 * LDR : 0);
        float2* l1 = l0 + LDR;
        const int js = clo + (act ? b : 0), j = (js + NC - NC / 2) % NC;
        if (act) {
          const float2* zc = Z + (int64_t)j * NR;
#pragma unroll 8
          for (int i = i0; i < NR; i += st) l0[i] = zc[i];
        }
        __syncwarp();
        const float2* res = l0;
        if (regR) gc_fft16_n<true>(l0, l1, NR, a.twr, hl, act);
        else res = gc_line(l0, l1, NR, a.gc_radix_r, a.gc_nst_r, a.twr, true, lane);
        float* rc = R + (int64_t)js * NR;
        const bool colkept = !search || abs(js - NC / 2) <= oac;
        if (act)
        for (int i = i0; i < NR; i += st) {
          const float2 c = res[i];
          const int is = i + NR / 2 < NR ? i + NR / 2 : i + NR / 2 - NR;  // fftshifted row
          float v = hypotf(c.x * scale, c.y * scale);
          if (a.gain) v *= __ldg(a.gain + is + (int64_t)js * NR);
          if (!colkept || (search && abs(is - NR / 2) > oar)) v = 0.f;
          if (bad) v = __int_as_float(0x7fc00000);
          rc[is] = v;
        }
        __syncwarp();
      }
    }
    __syncthreads();

    // ---- 4. plane out (correlation_planes / ensemble sums) and analysis
    if (a.planes) {  // a window holding NaN or Inf has a NaN plane, as in the reference
      float* dst = a.planes + job * P;
      for (int64_t e = tid; e < P; e += GC_THREADS) {
        const float v = bad ? __int_as_float(0x7fc00000) : R[e];
        dst[e] = a.accumulate ? dst[e] + v : v;
      }
    }
    if (!a.accumulate) {
      analyze_group(R, NR, NC, NR, K, a.npeaks, a.finder, a.subpixel, tid, GC_THREADS, red, true, s_vals, s_locs,
                    gid, job, &pw, bad, 0, sp, nullptr, 0);
    }
    __syncthreads();  // the scratch plane and shared buffers are reused by the CTA's next window
  }
}
