// Library context and host-side helpers shared by the C-ABI translation units
// (hh_api.cu: single-pair schedule and hooks; hh_batch.cu: batched schedule).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <map>
#include <sstream>
#include <string>
#include <tuple>
#include <vector>

#include "hammerhead_b200.h"
#include "hh_internal.h"

using hh::CorrArgs;

namespace hhd {

inline thread_local std::string g_err;  // context-free failures

struct DevBuf {
  void* p = nullptr;
  size_t bytes = 0;
};

struct TableKey {
  int wr, wc, sr, sc, apod, method, padded;
  bool operator<(const TableKey& o) const {
    return std::tie(wr, wc, sr, sc, apod, method, padded) < std::tie(o.wr, o.wc, o.sr, o.sc, o.apod, o.method, o.padded);
  }
};
struct Tables {
  float* apod = nullptr;
  float* gain = nullptr;
  float* phasew = nullptr;
  // support of the gain, or the kept search lags, in fftshifted rows/columns (0, 0: whole plane)
  int box_lo = 0, box_hi = 0;
  // the same per axis for any plane shape (fftshifted rows rlo..rhi,
  // columns clo..chi; the whole plane when there is no gain or lag limit)
  int rlo = 0, rhi = -1, clo = 0, chi = -1;
};

}  // namespace hhd

struct hh_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  int num_sms = 148;
  std::string err;
  std::map<std::string, hhd::DevBuf> bufs;
  std::map<hhd::TableKey, hhd::Tables> tables;
  std::map<int64_t, std::pair<float*, float*>> bs_factors;  // line length -> (cp, inv)
  float* pinned = nullptr;  // small pinned scratch for scalar reads
  // staged pair for the hook-level entry points
  int64_t nr = 0, nc = 0;
  const float* curA = nullptr;
  const float* curB = nullptr;
  bool staged = false;
  const uint8_t* hook_mask = nullptr;  // image mask of the hook calls (hh_stage_mask), device
  // host-side allocation-failure injection (hh_debug_fail_alloc): the
  // allocation attempt that brings the count to zero fails with HH_ERR_OOM
  // as a failing cudaMalloc would; negative = off
  int64_t fail_alloc_after = -1;
  // timing of the last schedule
  std::vector<float> pass_ms;
  std::vector<int32_t> pass_sweeps;
  std::vector<cudaEvent_t> events;
  // kernel accounting (hh_set_profiling / hh_profile_read / hh_launch_count)
  bool prof = false;
  struct Pending {
    int cls;
    cudaEvent_t a, b;
    double flops, bytes;
    int64_t units, nk;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> evpool;
  hh_kernel_profile acc[HH_K_CLASSES] = {};
  int64_t launches = 0;
  // batched-schedule plans by batch shape (hh_batch.cu), most recent last
  std::vector<std::pair<std::string, void*>> bplans;
  void (*bplan_free)(void*) = nullptr;
  // cross-process reduction of the ensemble sums (hh_set_ensemble_reducer)
  hh_ensemble_reducer ens_reduce = nullptr;
  void* ens_reduce_user = nullptr;
  // correlation kernel CTA shape per (FFT size, data extent), from
  // hh_set_corr_variant / hh_autotune_correlation (absent: 0, the default)
  std::map<std::pair<int, int>, int> corr_var;
  // general-shape correlation: twiddle tables exp(-2 pi i t / n) by length
  std::map<int, float2*> gc_twiddles;
};

namespace hhd {

inline hh_status fail(hh_ctx* ctx, hh_status code, const std::string& msg) {
  if (ctx) ctx->err = msg;
  else g_err = msg;
  return code;
}

#define HH_CK(call)                                                                                  \
  do {                                                                                               \
    cudaError_t e_ = (call);                                                                         \
    if (e_ != cudaSuccess)                                                                           \
      return fail(ctx, e_ == cudaErrorMemoryAllocation ? HH_ERR_OOM : HH_ERR_CUDA,                   \
                  std::string(#call) + ": " + cudaGetErrorString(e_));                               \
  } while (0)

#define HH_TRY(expr)                  \
  do {                                \
    hh_status s_ = (expr);            \
    if (s_ != HH_OK) return s_;       \
  } while (0)

inline std::string tup(const int32_t* t) {
  std::ostringstream o;
  o << "(" << t[0] << ", " << t[1] << ")";
  return o.str();
}
inline std::string num(double x) {
  std::ostringstream o;
  o << x;
  return o.str();
}

// cudaMalloc through the context, with the injected failure of
// hh_debug_fail_alloc (no device call is made for an injected failure).
inline cudaError_t ctx_malloc(hh_ctx* ctx, void** p, size_t bytes) {
  if (ctx && ctx->fail_alloc_after >= 0 && ctx->fail_alloc_after-- == 0) {
    *p = nullptr;
    return cudaErrorMemoryAllocation;
  }
  return cudaMalloc(p, bytes);
}

// Device buffer by name, grown on demand (never shrunk): a steady state of
// equally sized calls allocates nothing.
template <class T> hh_status buf(hh_ctx* ctx, const char* name, size_t count, T** out) {
  DevBuf& b = ctx->bufs[name];
  const size_t need = std::max<size_t>(count, 1) * sizeof(T);
  if (b.bytes < need) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    cudaError_t e = ctx_malloc(ctx, &b.p, need);
    if (e != cudaSuccess)
      return fail(ctx, HH_ERR_OOM, std::string("device allocation of ") + std::to_string(need) + " bytes for " + name +
                                       " failed: " + cudaGetErrorString(e));
    b.bytes = need;
  }
  *out = static_cast<T*>(b.p);
  return HH_OK;
}

// ---------------------------------------------------------------------------
// Host grid: pass_grid (src/pipeline.jl:529-555)
struct Grid {
  int ny = 0, nx = 0;
  std::vector<float> x, y;
  std::vector<uint8_t> gmask;
  std::vector<int32_t> jobs;  // 0-based gi, gj, rs, cs
  bool any_mask = false;
};

inline hh_status make_grid(hh_ctx* ctx, int64_t nr, int64_t nc, const hh_pass_desc& p, const uint8_t* mask, double thr,
                    Grid& g) {
  const int wr = p.window[0], wc = p.window[1], sr = p.search[0], sc = p.search[1];
  const int mr = (sr - wr) / 2, mc = (sc - wc) / 2;
  if (sr > nr || sc > nc)
    return fail(ctx, HH_ERR_ARG, "search area " + tup(p.search) + " exceeds image size (" + std::to_string(nr) + ", " +
                                     std::to_string(nc) + ")");
  std::vector<int64_t> rows, cols;
  for (int64_t s = 1 + mr; s <= nr - wr - mr + 1; s += wr - p.overlap[0]) rows.push_back(s);
  for (int64_t s = 1 + mc; s <= nc - wc - mc + 1; s += wc - p.overlap[1]) cols.push_back(s);
  g.ny = (int)rows.size();
  g.nx = (int)cols.size();
  g.x.resize(g.nx);
  g.y.resize(g.ny);
  for (int j = 0; j < g.nx; ++j) g.x[j] = (float)((double)cols[j] + (wc - 1) / 2.0);
  for (int i = 0; i < g.ny; ++i) g.y[i] = (float)((double)rows[i] + (wr - 1) / 2.0);
  g.gmask.assign((size_t)g.ny * g.nx, 0);
  g.any_mask = false;
  if (mask) {
    for (int gj = 0; gj < g.nx; ++gj)
      for (int gi = 0; gi < g.ny; ++gi) {
        const int64_t rs = rows[gi], cs = cols[gj];
        int64_t cw = 0, csr = 0;
        for (int j = 0; j < wc; ++j)
          for (int i = 0; i < wr; ++i) cw += mask[(rs - 1 + i) + (cs - 1 + j) * nr] != 0;
        const int64_t srs = rs - mr, scs = cs - mc;
        for (int j = 0; j < sc; ++j)
          for (int i = 0; i < sr; ++i) csr += mask[(srs - 1 + i) + (scs - 1 + j) * nr] != 0;
        const double fw = (double)cw / (double)(wr * wc), fs = (double)csr / (double)(sr * sc);
        const uint8_t m = fw >= thr || fs >= thr;
        g.gmask[gi + (size_t)gj * g.ny] = m;
        g.any_mask |= m != 0;
      }
  }
  g.jobs.clear();
  for (int gj = 0; gj < g.nx; ++gj)
    for (int gi = 0; gi < g.ny; ++gi)
      if (!g.gmask[gi + (size_t)gj * g.ny]) {
        g.jobs.push_back(gi);
        g.jobs.push_back(gj);
        g.jobs.push_back((int32_t)(rows[gi] - 1));
        g.jobs.push_back((int32_t)(cols[gj] - 1));
      }
  return HH_OK;
}

inline int fft_size(const hh_pass_desc& p) { return p.padding ? 2 * p.search[0] : p.search[0]; }
inline int fft_rows(const hh_pass_desc& p) { return p.padding ? 2 * p.search[0] : p.search[0]; }
inline int fft_cols(const hh_pass_desc& p) { return p.padding ? 2 * p.search[1] : p.search[1]; }

// A fused shared-memory kernel exists for this pass (square window and
// search area of a specialised size); otherwise the general-shape kernel runs.
inline bool corr_special(const hh_pass_desc& p) {
  return p.window[0] == p.window[1] && p.search[0] == p.search[1] && hh::correlate_supported(fft_size(p), p.search[0]);
}

// The CTA shape chosen for a pass's correlation launches.
inline int32_t corr_variant(const hh_ctx* ctx, const hh_pass_desc& p) {
  auto it = ctx->corr_var.find({fft_size(p), (int)p.search[0]});
  return it == ctx->corr_var.end() ? 0 : it->second;
}

// apodization_window (src/correlators.jl:18-25), computed in double like
// Julia: centre (w + 1)/2 and sigma w/4 per axis, wr x wc column-major
inline void apod_table(int wr, int wc, int apod, std::vector<float>& out) {
  out.assign((size_t)wr * wc, 1.0f);
  if (apod == HH_APOD_NONE) return;
  const double cr = (wr + 1) / 2.0, cc = (wc + 1) / 2.0, sr = wr / 4.0, sc = wc / 4.0;
  for (int j = 1; j <= wc; ++j)
    for (int i = 1; i <= wr; ++i)
      out[(i - 1) + (size_t)(j - 1) * wr] =
          (float)std::exp(-((i - cr) * (i - cr) / (2 * sr * sr) + (j - cc) * (j - cc) / (2 * sc * sc)));
}

// overlap gain (src/correlators.jl:170-181): the weight of each lag is the
// autocorrelation of the apodization window (the reference forms it with an
// FFT in T); gain = wmax / w where w >= wmax / 2, else 0, in the fftshifted
// layout of the 2wr x 2wc plane. Square windows up to 64 px sum the float
// window's products directly in double; larger or rectangular windows use
// the separable form of the same window (the product of the row and column
// autocorrelations of the double-precision factors), the same quantity to
// within the float rounding of the window values.
inline void gain_table(int wr, int wc, int apod, const std::vector<float>& ap, std::vector<float>& out) {
  const int NR = 2 * wr, NC = 2 * wc;
  std::vector<float> wt((size_t)NR * NC, 0.f);
  if (wr == wc && wr <= 64) {
    const int W = wr, N = NR;
    for (int qs = 0; qs < N; ++qs)
      for (int ps = 0; ps < N; ++ps) {
        const int dp = ps - N / 2, dq = qs - N / 2;
        if (std::abs(dp) >= W || std::abs(dq) >= W) continue;
        double acc = 0;
        for (int q = std::max(0, -dq); q < std::min(W, W - dq); ++q)
          for (int p = std::max(0, -dp); p < std::min(W, W - dp); ++p)
            acc += (double)ap[p + (size_t)q * W] * (double)ap[(p + dp) + (size_t)(q + dq) * W];
        wt[ps + (size_t)qs * N] = (float)std::fabs(acc);
      }
  } else {
    auto axis = [apod](int w, std::vector<double>& ac) {
      std::vector<double> g(w, 1.0);
      if (apod == HH_APOD_GAUSS) {
        const double c = (w + 1) / 2.0, s = w / 4.0;
        for (int i = 1; i <= w; ++i) g[i - 1] = std::exp(-(i - c) * (i - c) / (2 * s * s));
      }
      ac.assign(2 * w, 0.0);  // lag d at index d + w
      for (int d = -(w - 1); d <= w - 1; ++d) {
        double a = 0;
        for (int i = std::max(0, -d); i < std::min(w, w - d); ++i) a += g[i] * g[i + d];
        ac[d + w] = a;
      }
    };
    std::vector<double> ar, acol;
    axis(wr, ar);
    axis(wc, acol);
    for (int qs = 0; qs < NC; ++qs)
      for (int ps = 0; ps < NR; ++ps) {
        const int dp = ps - NR / 2, dq = qs - NC / 2;
        if (std::abs(dp) >= wr || std::abs(dq) >= wc) continue;
        wt[ps + (size_t)qs * NR] = (float)std::fabs(ar[dp + wr] * acol[dq + wc]);
      }
  }
  float wmax = 0.f;
  for (float w : wt) wmax = std::max(wmax, w);
  out.resize(wt.size());
  for (size_t k = 0; k < wt.size(); ++k) out[k] = wt[k] >= wmax / 2 ? wmax / wt[k] : 0.f;
}

// PhaseCorrelator Gaussian spectral filter (src/correlators.jl:96-129):
// fftfreq bins of each axis, sigma = min(nr, nc) / 8, natural FFT order
inline void phase_table(int NR, int NC, std::vector<float>& out) {
  out.resize((size_t)NR * NC);
  const double fs = std::min(NR, NC) / 8.0;
  for (int j = 0; j < NC; ++j)
    for (int i = 0; i < NR; ++i) {
      const double fi = i < (NR + 1) / 2 ? i : i - NR, fj = j < (NC + 1) / 2 ? j : j - NC;
      out[i + (size_t)j * NR] = (float)std::exp(-(fi * fi + fj * fj) / (2 * fs * fs));
    }
}

inline hh_status get_tables(hh_ctx* ctx, const hh_pass_desc& p, Tables& t) {
  const int wr = p.window[0], wc = p.window[1], sr = p.search[0], sc = p.search[1];
  const int NR = fft_rows(p), NC = fft_cols(p);
  TableKey key{wr, wc, sr, sc, p.apodization, p.method, p.padding};
  auto it = ctx->tables.find(key);
  if (it != ctx->tables.end()) {
    t = it->second;
    return HH_OK;
  }
  std::vector<float> ap, gn, ph;
  apod_table(wr, wc, p.apodization, ap);
  Tables nt;
  nt.rhi = NR - 1;
  nt.chi = NC - 1;
  HH_CK(cudaMalloc(&nt.apod, ap.size() * sizeof(float)));
  HH_CK(cudaMemcpy(nt.apod, ap.data(), ap.size() * sizeof(float), cudaMemcpyHostToDevice));
  if (sr != wr || sc != wc) {
    // enlarged search area: no overlap gain (CrossCorrelator, src/correlators.jl:73);
    // only lags with |lag| <= (S - W) / 2 are kept (restrict_search_lags!, :347-355)
    nt.rlo = NR / 2 - (sr - wr) / 2;
    nt.rhi = NR / 2 + (sr - wr) / 2;
    nt.clo = NC / 2 - (sc - wc) / 2;
    nt.chi = NC / 2 + (sc - wc) / 2;
    if (NR == NC && sr == sc && wr == wc) {
      const int m = (sr - wr) / 2;
      nt.box_lo = NR / 2 - m;
      nt.box_hi = NR / 2 + m;
    }
  } else if (p.padding) {
    gain_table(wr, wc, p.apodization, ap, gn);
    {  // bounding rows and columns of the nonzero gain
      int rl = NR, rh = -1, cl = NC, ch = -1;
      for (int q = 0; q < NC; ++q)
        for (int r = 0; r < NR; ++r)
          if (gn[r + (size_t)q * NR] != 0.f) {
            rl = std::min(rl, r);
            rh = std::max(rh, r);
            cl = std::min(cl, q);
            ch = std::max(ch, q);
          }
      if (rh >= 0) {
        nt.rlo = rl;
        nt.rhi = rh;
        nt.clo = cl;
        nt.chi = ch;
      }
    }
    if (NR == NC) {
      // bounding box of the nonzero gain (square and centred, by symmetry)
      int lo = NR, hi = -1;
      for (int q = 0; q < NC; ++q)
        for (int r = 0; r < NR; ++r)
          if (gn[r + (size_t)q * NR] != 0.f) {
            lo = std::min(lo, std::min(r, q));
            hi = std::max(hi, std::max(r, q));
          }
      if (hi > 0) {
        nt.box_lo = lo;
        nt.box_hi = hi;
      }
    }
    // after the table: a flag word and, for a square table whose values
    // depend only on |lag| along each axis (a symmetric apodization window),
    // its quarter q[a + b (N/2 + 1)] = gain at lags (-a, -b) for kernels that
    // keep the quarter in shared memory; the flag is 1 when the quarter is exact
    std::vector<float> gq;
    if (NR == NC) {
      const int H = NR / 2, HQ = H + 1;
      gq.assign((size_t)HQ * HQ, 0.f);
      for (int b = 0; b <= H; ++b)
        for (int a = 0; a <= H; ++a) gq[a + (size_t)b * HQ] = gn[(H - a) + (size_t)(H - b) * NR];
      bool sym = true;
      for (int c = 0; c < NC && sym; ++c)
        for (int r = 0; r < NR && sym; ++r)
          sym = gn[r + (size_t)c * NR] == gq[std::abs(r - H) + (size_t)std::abs(c - H) * HQ];
      if (!sym) gq.clear();
    }
    gn.push_back(gq.empty() ? 0.f : 1.f);
    gn.insert(gn.end(), gq.begin(), gq.end());
    HH_CK(cudaMalloc(&nt.gain, gn.size() * sizeof(float)));
    HH_CK(cudaMemcpy(nt.gain, gn.data(), gn.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  if (p.method == HH_PHASE) {
    phase_table(NR, NC, ph);
    HH_CK(cudaMalloc(&nt.phasew, ph.size() * sizeof(float)));
    HH_CK(cudaMemcpy(nt.phasew, ph.data(), ph.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  ctx->tables[key] = nt;
  t = nt;
  return HH_OK;
}

// Twiddle table exp(-2 pi i t / n), t = 0 .. n-1, of one FFT length, built
// once per context (double-precision angles, each entry rounded once).
inline hh_status gc_twiddles(hh_ctx* ctx, int n, const float2** out) {
  auto it = ctx->gc_twiddles.find(n);
  if (it == ctx->gc_twiddles.end()) {
    std::vector<float2> h(n);
    for (int t = 0; t < n; ++t) {
      // the angle in double (relative error ~1e-16, far below float rounding)
      const double a = -2.0 * M_PI * (double)t / (double)n;
      h[t] = make_float2((float)std::cos(a), (float)std::sin(a));
    }
    float2* d = nullptr;
    HH_CK(cudaMalloc(&d, (size_t)n * sizeof(float2)));
    HH_CK(cudaMemcpy(d, h.data(), (size_t)n * sizeof(float2), cudaMemcpyHostToDevice));
    it = ctx->gc_twiddles.emplace(n, d).first;
  }
  *out = it->second;
  return HH_OK;
}

// Shared memory of the general kernel's two line buffers (at most this much)
constexpr size_t GC_SMEM_LINES = 192 * 1024;
// planes the general kernel accepts (complex + real plane per CTA slice)
constexpr int64_t GC_MAX_POINTS = (int64_t)1 << 22;

// FFT lengths the general kernel transforms in registers (16 x B, two lines per warp)
inline bool gc_reg_length(int n) { return n == 32 || n == 64 || n == 128 || n == 256; }

// Is the pass's FFT shape one the general kernel can run?
inline bool gcorr_shape_ok(const hh_pass_desc& p) {
  int8_t rr[24];
  const int NR = fft_rows(p), NC = fft_cols(p);
  return NR >= 2 && NC >= 2 && (int64_t)NR * NC <= GC_MAX_POINTS && hh::gcorr_radix_plan(NR, rr) > 0 &&
         hh::gcorr_radix_plan(NC, rr) > 0 && 2 * (size_t)(NC + 16) * 2 * sizeof(float2) <= GC_SMEM_LINES &&
         2 * 2 * (size_t)(NR + 16) * sizeof(float2) <= GC_SMEM_LINES;
}

// Fill the general-shape fields of a correlation launch: shapes, radix
// plans, twiddles, chunking and the scratch slice geometry (one slice per
// CTA, as many as SMs); gcorr_prepare also points it at the context's
// scratch buffer (grown on demand), a batched plan at its own.
inline hh_status gcorr_setup(hh_ctx* ctx, const hh_pass_desc& p, CorrArgs& ca) {
  ca.wr = p.window[0];
  ca.wc = p.window[1];
  ca.sr = p.search[0];
  ca.sc = p.search[1];
  ca.nfr = fft_rows(p);
  ca.nfc = fft_cols(p);
  ca.gc_nst_r = hh::gcorr_radix_plan(ca.nfr, ca.gc_radix_r);
  ca.gc_nst_c = hh::gcorr_radix_plan(ca.nfc, ca.gc_radix_c);
  if (ca.gc_nst_r < 0 || ca.gc_nst_c < 0 || !gcorr_shape_ok(p))
    return fail(ctx, HH_ERR_UNSUPPORTED,
                "backend :b200 has no correlation kernel for an FFT plane of " + std::to_string(ca.nfr) + " x " +
                    std::to_string(ca.nfc));
  HH_TRY(gc_twiddles(ctx, ca.nfr, &ca.twr));
  HH_TRY(gc_twiddles(ctx, ca.nfc, &ca.twc));
  // columns passes: per warp one line (two, one per half-warp, for the
  // register-form lengths 32..256), two buffers per line, as many warps (of
  // 16) as fit; rows pass: chunks of row pairs, two buffers each. Lines are
  // staged with 16 elements of padding (the register form's exchange).
  const size_t ldr = (size_t)ca.nfr + 16, ldc = (size_t)ca.nfc + 16;
  const int lpw = gc_reg_length(ca.nfr) ? 2 : 1;
  ca.gc_col_warps = std::max(1, std::min(16, (int)(GC_SMEM_LINES / (2 * lpw * ldr * sizeof(float2)))));
  ca.gc_chunk_c = std::max(2, std::min(32, (int)(GC_SMEM_LINES / (2 * ldc * sizeof(float2)))) & ~1);
  const size_t lines = std::max((size_t)ca.gc_col_warps * lpw * ldr, (size_t)ca.gc_chunk_c * ldc);
  ca.gc_smem_lines = (int64_t)(2 * lines * sizeof(float2));
  const int64_t P = (int64_t)ca.nfr * ca.nfc;
  ca.gscr_stride = (P + (P + 1) / 2 + 31) & ~(int64_t)31;  // complex plane + real plane, 256-byte aligned slices
  ca.gscr_slices = ctx->num_sms;
  Tables tb;
  HH_TRY(get_tables(ctx, p, tb));
  ca.gc_box[0] = tb.rlo;
  ca.gc_box[1] = tb.rhi;
  ca.gc_box[2] = tb.clo;
  ca.gc_box[3] = tb.chi;
  return HH_OK;
}
inline hh_status gcorr_prepare(hh_ctx* ctx, const hh_pass_desc& p, CorrArgs& ca) {
  HH_TRY(gcorr_setup(ctx, p, ca));
  return buf(ctx, "gcorr_scratch", (size_t)ca.gscr_slices * ca.gscr_stride, &ca.gscr);
}

// The window shape of an uncertainty launch (rows W, columns Wc), and for
// rectangular or large windows the general form's scratch slices (one per
// CTA; the buffer is the context's and grows on demand).
inline void uq_setup(hh_ctx* ctx, int wr, int wc, hh::UQArgs& ua) {
  ua.W = wr;
  ua.Wc = wc;
  if (!hh::uq_general(wr, wc)) return;
  ua.gscr_stride = hh::uq_general_stride(wr, wc);
  ua.gscr_slices = 4 * ctx->num_sms;
}
inline hh_status uq_prepare(hh_ctx* ctx, int wr, int wc, hh::UQArgs& ua) {
  uq_setup(ctx, wr, wc, ua);
  if (!hh::uq_general(wr, wc)) return HH_OK;
  return buf(ctx, "uq_scratch", (size_t)ua.gscr_slices * ua.gscr_stride, &ua.gscr);
}

// Launch the correlation of one pass: the fused kernel where one exists,
// else the general-shape kernel (gcorr_prepare must have filled ca).
inline cudaError_t corr_launch(hh_ctx* ctx, const hh_pass_desc& p, const CorrArgs& ca, cudaStream_t s) {
  if (corr_special(p)) return hh::launch_correlate(ca, fft_size(p), p.search[0], s, ctx->num_sms);
  return hh::launch_correlate_general(ca, s);
}

inline hh_status set_device(hh_ctx* ctx) {
  HH_CK(cudaSetDevice(ctx->device));
  return HH_OK;
}

// B-spline elimination factors of one line length, built once per context.
inline hh_status bs_factors(hh_ctx* ctx, int64_t n, float** cp, float** inv) {
  auto it = ctx->bs_factors.find(n);
  if (it == ctx->bs_factors.end()) {
    float *a = nullptr, *b = nullptr;
    HH_CK(cudaMalloc(&a, std::max<int64_t>(n, 1) * sizeof(float)));
    HH_CK(cudaMalloc(&b, std::max<int64_t>(n, 1) * sizeof(float)));
    HH_CK(hh::launch_bspline_factors(n, a, b, ctx->stream));
    ctx->launches += 1;
    it = ctx->bs_factors.emplace(n, std::make_pair(a, b)).first;
  }
  *cp = it->second.first;
  *inv = it->second.second;
  return HH_OK;
}

inline cudaEvent_t pool_event(hh_ctx* ctx) {
  if (!ctx->evpool.empty()) {
    cudaEvent_t e = ctx->evpool.back();
    ctx->evpool.pop_back();
    return e;
  }
  cudaEvent_t e = nullptr;
  cudaEventCreate(&e);
  return e;
}

// Launch one or more kernels of class cls; count them, and when profiling
// bracket them with events on the context stream.
template <class F>
inline hh_status run_k(hh_ctx* ctx, int cls, int nk, double flops, double bytes, int64_t units, F&& f) {
  cudaEvent_t a = nullptr;
  if (ctx->prof) {
    a = pool_event(ctx);
    cudaEventRecord(a, ctx->stream);
  }
  cudaError_t e = f();
  if (e != cudaSuccess)
    return fail(ctx, e == cudaErrorMemoryAllocation ? HH_ERR_OOM : HH_ERR_CUDA,
                std::string("kernel launch failed: ") + cudaGetErrorString(e));
  ctx->launches += nk;
  if (ctx->prof) {
    cudaEvent_t b = pool_event(ctx);
    cudaEventRecord(b, ctx->stream);
    ctx->pending.push_back({cls, a, b, flops, bytes, units, nk});
  }
  return HH_OK;
}
#define HH_K(cls, nk, fl, by, un, call) HH_TRY(run_k(ctx, cls, nk, (double)(fl), (double)(by), (int64_t)(un), [&]() { return (call); }))

// Fold completed event pairs into the per-class totals (stream synchronised).
inline hh_status flush_profile(hh_ctx* ctx) {
  for (auto& q : ctx->pending) {
    float ms = 0.f;
    HH_CK(cudaEventElapsedTime(&ms, q.a, q.b));
    hh_kernel_profile& t = ctx->acc[q.cls];
    t.launches += q.nk;
    t.ms += ms;
    t.flops += q.flops;
    t.bytes += q.bytes;
    t.units += q.units;
    ctx->evpool.push_back(q.a);
    ctx->evpool.push_back(q.b);
  }
  ctx->pending.clear();
  return HH_OK;
}

// algorithmic work of one correlation launch: 2 forward + 1 inverse real
// 2-D FFT (2.5 M log2 M each, M = N^2) + 8 M for spectrum and gain per
// window; bytes: both windows read once, packed scalars written.
inline double corr_flops(int N, int64_t njobs) {
  const double M = (double)N * N;
  return (double)njobs * (3.0 * 2.5 * M * std::log2(M) + 8.0 * M);
}
inline double corr_bytes(int W, int nalt, int64_t njobs) { return (double)njobs * (2.0 * W * W * 4 + 4.0 * (4 + 2 * nalt)); }
// the same for a pass of any shape: FFT plane NR x NC, frame-A window and
// frame-B search area read once
inline double corr_flops(const hh_pass_desc& p, int64_t njobs) {
  const double M = (double)fft_rows(p) * fft_cols(p);
  return (double)njobs * (3.0 * 2.5 * M * std::log2(M) + 8.0 * M);
}
inline double corr_bytes(const hh_pass_desc& p, int nalt, int64_t njobs) {
  return (double)njobs * (4.0 * ((double)p.window[0] * p.window[1] + (double)p.search[0] * p.search[1]) +
                          4.0 * (4 + 2 * nalt));
}
inline double uq_flops(int W, int64_t njobs) { return (double)njobs * 2.0 * 2.0 * (3 + 41) * W * (W - 1); }
inline double uq_flops(const hh_pass_desc& p, int64_t njobs) {
  const double wr = p.window[0], wc = p.window[1];
  return (double)njobs * 2.0 * (3 + 41) * (wr * (wc - 1) + wc * (wr - 1));
}

// Cubic B-spline coefficients of both images of a pair.
inline hh_status prefilter_pair(hh_ctx* ctx, const float* dA, const float* dB, int64_t nr, int64_t nc, float* cA, float* cB) {
  float *cpc, *ivc, *cpr, *ivr, *bsd;
  HH_TRY(bs_factors(ctx, nr + 2, &cpc, &ivc));
  HH_TRY(bs_factors(ctx, nc + 2, &cpr, &ivr));
  HH_TRY(buf(ctx, "bs_dbuf", (size_t)2 * (nr + 2) * (nc + 2), &bsd));
  const double P = (double)nr * nc;
  HH_K(HH_K_PREFILTER, 4, 24 * P, 16 * P, (int64_t)(2 * P),
       hh::launch_prefilter_pair(dA, dB, nr, nc, cA, cB, bsd, cpc, ivc, cpr, ivr, ctx->stream));
  return HH_OK;
}


// validate_and_replace! (src/pipeline.jl:617-645) on device buffers.
inline hh_status validate_device(hh_ctx* ctx, const hh_pass_desc& p, int ny, int nx, float* u, float* v, const float* ratio,
                          const float* moment, uint8_t* outl, uint8_t* outl2, const uint8_t* gmask, bool any_mask,
                          const float* alt_u, const float* alt_v, int nalt, bool force_replace) {
  cudaStream_t s = ctx->stream;
  const int64_t G = (int64_t)ny * nx;
  HH_CK(cudaMemsetAsync(outl, 0, G, s));
  const uint8_t* excl = any_mask ? gmask : nullptr;
  if (p.uod_enable) HH_K(HH_K_VECTOR, 1, 0, 48 * G, G, hh::launch_uod(u, v, ny, nx, p.uod_threshold, p.uod_neighborhood, 0.1, excl, outl, 1, s));
  if (p.min_peak_ratio > 1) HH_K(HH_K_VECTOR, 1, 0, 5 * G, G, hh::launch_flag_ratio(ratio, G, p.min_peak_ratio, outl, s));
  for (int q = 0; q < p.n_validators; ++q) {
    const hh_validator& vd = p.validators[q];
    if (vd.kind == HH_VAL_PEAK_RATIO) HH_K(HH_K_VECTOR, 1, 0, 5 * G, G, hh::launch_flag_ratio(ratio, G, vd.threshold, outl, s));
    else if (vd.kind == HH_VAL_MOMENT) HH_K(HH_K_VECTOR, 1, 0, 5 * G, G, hh::launch_flag_moment(moment, G, vd.threshold, outl, s));
    else if (vd.kind == HH_VAL_VELOCITY) HH_K(HH_K_VECTOR, 1, 0, 9 * G, G, hh::launch_flag_velocity(u, v, G, vd.vmin, vd.vmax, outl, s));
    else if (vd.kind == HH_VAL_UOD)
      HH_K(HH_K_VECTOR, 1, 0, 48 * G, G, hh::launch_uod(u, v, ny, nx, vd.threshold, vd.neighborhood, vd.epsilon, excl, outl, 1, s));
  }
  if (any_mask) HH_K(HH_K_VECTOR, 1, 0, 2 * G, G, hh::launch_mask_flags(outl, gmask, G, s));
  if (alt_u && nalt > 0) {
    HH_K(HH_K_VECTOR, 1, 0, (10 + 8 * nalt) * G, G, hh::launch_substitute(u, v, outl, outl2, gmask, alt_u, alt_v, nalt, ny, nx, p.uod_neighborhood,
                                p.uod_threshold, s));
    HH_CK(cudaMemcpyAsync(outl, outl2, G, cudaMemcpyDeviceToDevice, s));
  }
  if (force_replace || p.replace_outliers) HH_K(HH_K_VECTOR, 1, 0, 10 * G, G, hh::launch_replace(u, v, outl, gmask, ny, nx, 1, s));
  return HH_OK;
}

inline hh_status read_scalar(hh_ctx* ctx, const float* dptr, float* out) {
  HH_CK(cudaMemcpyAsync(ctx->pinned, dptr, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream));
  HH_CK(cudaStreamSynchronize(ctx->stream));
  *out = ctx->pinned[0];
  return HH_OK;
}

inline hh_status check_passes(hh_ctx* ctx, const hh_pass_desc* passes, int np) {
  if (!passes || np < 1) return fail(ctx, HH_ERR_ARG, "at least one pass is required");
  for (int k = 0; k < np; ++k) {
    hh_status s = hh_pass_validate(&passes[k]);
    if (s != HH_OK) return fail(ctx, s, hh_last_error(nullptr));
  }
  hh_status s = hh_check_backend_params(passes, np);
  if (s != HH_OK) return fail(ctx, s, hh_last_error(nullptr));
  return HH_OK;
}


}  // namespace hhd
