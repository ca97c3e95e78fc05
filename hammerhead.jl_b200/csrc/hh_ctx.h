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
  int W, S, N, apod, method, padded;
  bool operator<(const TableKey& o) const {
    return std::tie(W, S, N, apod, method, padded) < std::tie(o.W, o.S, o.N, o.apod, o.method, o.padded);
  }
};
struct Tables {
  float* apod = nullptr;
  float* gain = nullptr;
  float* phasew = nullptr;
  // support of the gain, or the kept search lags, in fftshifted rows/columns (0, 0: whole plane)
  int box_lo = 0, box_hi = 0;
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

// Device buffer by name, grown on demand (never shrunk): a steady state of
// equally sized calls allocates nothing.
template <class T> hh_status buf(hh_ctx* ctx, const char* name, size_t count, T** out) {
  DevBuf& b = ctx->bufs[name];
  const size_t need = std::max<size_t>(count, 1) * sizeof(T);
  if (b.bytes < need) {
    if (b.p) cudaFree(b.p);
    b.p = nullptr;
    b.bytes = 0;
    cudaError_t e = cudaMalloc(&b.p, need);
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

// The CTA shape chosen for a pass's correlation launches.
inline int32_t corr_variant(const hh_ctx* ctx, const hh_pass_desc& p) {
  auto it = ctx->corr_var.find({fft_size(p), (int)p.search[0]});
  return it == ctx->corr_var.end() ? 0 : it->second;
}

// apodization_window (src/correlators.jl:18-25), computed in double like Julia
inline void apod_table(int W, int apod, std::vector<float>& out) {
  out.assign((size_t)W * W, 1.0f);
  if (apod == HH_APOD_NONE) return;
  const double c = (W + 1) / 2.0, s = W / 4.0;
  for (int j = 1; j <= W; ++j)
    for (int i = 1; i <= W; ++i)
      out[(i - 1) + (size_t)(j - 1) * W] =
          (float)std::exp(-((i - c) * (i - c) / (2 * s * s) + (j - c) * (j - c) / (2 * s * s)));
}

// overlap gain (src/correlators.jl:170-181): the reference forms the
// autocorrelation of the apodization window with an FFT; here it is summed
// directly in double (the same quantity without transform round-off), then
// thresholded at half the zero-lag weight in float.
inline void gain_table(int W, const std::vector<float>& apod, std::vector<float>& out) {
  const int N = 2 * W;
  std::vector<float> wt((size_t)N * N, 0.f);
  for (int qs = 0; qs < N; ++qs)
    for (int ps = 0; ps < N; ++ps) {
      const int dp = ps - N / 2, dq = qs - N / 2;
      if (std::abs(dp) >= W || std::abs(dq) >= W) continue;
      double acc = 0;
      for (int q = std::max(0, -dq); q < std::min(W, W - dq); ++q)
        for (int p = std::max(0, -dp); p < std::min(W, W - dp); ++p)
          acc += (double)apod[p + (size_t)q * W] * (double)apod[(p + dp) + (size_t)(q + dq) * W];
      wt[ps + (size_t)qs * N] = (float)std::fabs(acc);
    }
  float wmax = 0.f;
  for (float w : wt) wmax = std::max(wmax, w);
  out.resize(wt.size());
  for (size_t k = 0; k < wt.size(); ++k) out[k] = wt[k] >= wmax / 2 ? wmax / wt[k] : 0.f;
}

// PhaseCorrelator Gaussian spectral filter (src/correlators.jl:96-129)
inline void phase_table(int N, std::vector<float>& out) {
  out.resize((size_t)N * N);
  const double fs = N / 8.0;
  for (int j = 0; j < N; ++j)
    for (int i = 0; i < N; ++i) {
      const double fi = i < (N + 1) / 2 ? i : i - N, fj = j < (N + 1) / 2 ? j : j - N;
      out[i + (size_t)j * N] = (float)std::exp(-(fi * fi + fj * fj) / (2 * fs * fs));
    }
}

inline hh_status get_tables(hh_ctx* ctx, const hh_pass_desc& p, Tables& t) {
  const int W = p.window[0], S = p.search[0], N = fft_size(p);
  TableKey key{W, S, N, p.apodization, p.method, p.padding};
  auto it = ctx->tables.find(key);
  if (it != ctx->tables.end()) {
    t = it->second;
    return HH_OK;
  }
  std::vector<float> ap, gn, ph;
  apod_table(W, p.apodization, ap);
  Tables nt;
  HH_CK(cudaMalloc(&nt.apod, ap.size() * sizeof(float)));
  HH_CK(cudaMemcpy(nt.apod, ap.data(), ap.size() * sizeof(float), cudaMemcpyHostToDevice));
  if (S != W) {
    // enlarged search area: no overlap gain (CrossCorrelator, src/correlators.jl:73);
    // only lags with |lag| <= (S - W) / 2 are kept (restrict_search_lags!, :347-355)
    const int m = (S - W) / 2;
    nt.box_lo = N / 2 - m;
    nt.box_hi = N / 2 + m;
  } else if (p.padding) {
    gain_table(W, ap, gn);
    // bounding box of the nonzero gain (square and centred, by symmetry)
    int lo = N, hi = -1;
    for (int q = 0; q < N; ++q)
      for (int r = 0; r < N; ++r)
        if (gn[r + (size_t)q * N] != 0.f) {
          lo = std::min(lo, std::min(r, q));
          hi = std::max(hi, std::max(r, q));
        }
    if (hi > 0) {
      nt.box_lo = lo;
      nt.box_hi = hi;
    }
    HH_CK(cudaMalloc(&nt.gain, gn.size() * sizeof(float)));
    HH_CK(cudaMemcpy(nt.gain, gn.data(), gn.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  if (p.method == HH_PHASE) {
    phase_table(N, ph);
    HH_CK(cudaMalloc(&nt.phasew, ph.size() * sizeof(float)));
    HH_CK(cudaMemcpy(nt.phasew, ph.data(), ph.size() * sizeof(float), cudaMemcpyHostToDevice));
  }
  ctx->tables[key] = nt;
  t = nt;
  return HH_OK;
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
inline double uq_flops(int W, int64_t njobs) { return (double)njobs * 2.0 * 2.0 * (3 + 41) * W * (W - 1); }

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
