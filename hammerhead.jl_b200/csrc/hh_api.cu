// C ABI of the B200 planar-WIDIM library: parameter validation, grids,
// contexts, and the device-resident pass schedule (run_piv / piv_pass of
// src/pipeline.jl:361-832). Kernels live in k_*.cu.
#include "hh_ctx.h"

using namespace hhd;
using hh::CorrArgs;

namespace hhd {

// The device-resident schedule: run_piv + piv_pass with every sweep, the
// deformation, validation and uncertainty on the context stream.
hh_status run_schedule(hh_ctx* ctx, const float* dA, const float* dB, int64_t nr, int64_t nc,
                       const hh_pass_desc* passes, int np, const uint8_t* hmask, const uint8_t* dmask, double thr,
                       bool smoothing, hh_result* out) {
  cudaStream_t s = ctx->stream;
  HH_TRY(check_passes(ctx, passes, np));
  if (nr < 1 || nc < 1) return fail(ctx, HH_ERR_ARG, "images must be non-empty");
  if (!(thr > 0 && thr <= 1)) return fail(ctx, HH_ERR_ARG, "mask_threshold must be in (0, 1], got " + num(thr));
  const bool deforms = np > 1 || std::any_of(passes, passes + np, [](const hh_pass_desc& p) { return p.max_iterations > 1; });
  const int64_t P = nr * nc;
  float *coefA = nullptr, *coefB = nullptr, *warpA = nullptr, *warpB = nullptr;
  if (deforms) {
    HH_TRY(buf(ctx, "coefA", (size_t)(nr + 2) * (nc + 2), &coefA));
    HH_TRY(buf(ctx, "coefB", (size_t)(nr + 2) * (nc + 2), &coefB));
    HH_TRY(buf(ctx, "warpA", (size_t)P, &warpA));
    HH_TRY(buf(ctx, "warpB", (size_t)P, &warpB));
  }
  // grids of every pass (host) and the largest grid
  std::vector<Grid> grids(np);
  int64_t Gmax = 1, Jmax = 1;
  int nalt_max = 0;
  for (int k = 0; k < np; ++k) {
    HH_TRY(make_grid(ctx, nr, nc, passes[k], hmask, thr, grids[k]));
    Gmax = std::max<int64_t>(Gmax, (int64_t)grids[k].ny * grids[k].nx);
    Jmax = std::max<int64_t>(Jmax, (int64_t)grids[k].jobs.size() / 4);
    nalt_max = std::max(nalt_max, passes[k].n_peaks - 1);
  }
  float *u, *v, *resu, *resv, *ratio, *moment, *uncu, *uncv, *altu = nullptr, *altv = nullptr;
  float *predu, *predv, *predw_u, *predw_v, *prevu, *prevv, *measu, *measv, *dx, *dy, *fc, *fcout;
  uint8_t *outl, *outl2, *gm;
  int32_t* djobs;
  HH_TRY(buf(ctx, "u", Gmax, &u));
  HH_TRY(buf(ctx, "v", Gmax, &v));
  HH_TRY(buf(ctx, "resu", Gmax, &resu));
  HH_TRY(buf(ctx, "resv", Gmax, &resv));
  HH_TRY(buf(ctx, "ratio", Gmax, &ratio));
  HH_TRY(buf(ctx, "moment", Gmax, &moment));
  HH_TRY(buf(ctx, "uncu", Gmax, &uncu));
  HH_TRY(buf(ctx, "uncv", Gmax, &uncv));
  if (nalt_max > 0) {
    HH_TRY(buf(ctx, "altu", Gmax * nalt_max, &altu));
    HH_TRY(buf(ctx, "altv", Gmax * nalt_max, &altv));
  }
  HH_TRY(buf(ctx, "predu", Gmax, &predu));
  HH_TRY(buf(ctx, "predv", Gmax, &predv));
  HH_TRY(buf(ctx, "predwu", Gmax, &predw_u));
  HH_TRY(buf(ctx, "predwv", Gmax, &predw_v));
  HH_TRY(buf(ctx, "prevu", Gmax, &prevu));
  HH_TRY(buf(ctx, "prevv", Gmax, &prevv));
  HH_TRY(buf(ctx, "measu", Gmax, &measu));
  HH_TRY(buf(ctx, "measv", Gmax, &measv));
  HH_TRY(buf(ctx, "gx", Gmax, &dx));
  HH_TRY(buf(ctx, "gy", Gmax, &dy));
  HH_TRY(buf(ctx, "fc", Gmax + 64, &fc));
  HH_TRY(buf(ctx, "fcout", 4, &fcout));
  HH_TRY(buf(ctx, "outl", Gmax, &outl));
  HH_TRY(buf(ctx, "outl2", Gmax, &outl2));
  HH_TRY(buf(ctx, "gmask", Gmax, &gm));
  HH_TRY(buf(ctx, "jobs", 4 * Jmax, &djobs));
  size_t recw = 0;
  for (int k = 0; k < np; ++k) recw = std::max(recw, hh::correlate_record_words(passes[k].n_peaks));
  float* prec;
  HH_TRY(buf(ctx, "peakrec", (size_t)Jmax * recw, &prec));

  // events for per-pass device time
  while ((int)ctx->events.size() < np + 1) {
    cudaEvent_t e;
    HH_CK(cudaEventCreate(&e));
    ctx->events.push_back(e);
  }
  ctx->pass_ms.assign(np, 0.f);
  ctx->pass_sweeps.assign(np, 0);

  HH_CK(cudaEventRecord(ctx->events[0], s));
  if (deforms) {
    HH_TRY(prefilter_pair(ctx, dA, dB, nr, nc, coefA, coefB));
  }
  bool have_pred = false;
  hh::PredGrid pg{};
  const float* pred_src_u = nullptr;
  const float* pred_src_v = nullptr;
  for (int k = 0; k < np; ++k) {
    const hh_pass_desc& p = passes[k];
    const Grid& g = grids[k];
    const bool force_replace = k < np - 1;
    const int ny = g.ny, nx = g.nx;
    const int64_t G = (int64_t)ny * nx;
    const int64_t njobs = (int64_t)g.jobs.size() / 4;
    const int W = p.window[0], N = fft_size(p);
    const int nalt = p.n_peaks - 1;
    Tables tb;
    HH_TRY(get_tables(ctx, p, tb));
    if (k > 0) {
      // build_predictor (src/pipeline.jl:454-464) from the previous pass
      const Grid& pgd = grids[k - 1];
      const int64_t Gp = (int64_t)pgd.ny * pgd.nx;
      HH_CK(cudaMemcpyAsync(predw_u, u, Gp * sizeof(float), cudaMemcpyDeviceToDevice, s));
      HH_CK(cudaMemcpyAsync(predw_v, v, Gp * sizeof(float), cudaMemcpyDeviceToDevice, s));
      if (pgd.any_mask) HH_K(HH_K_VECTOR, 1, 0, 10 * Gp, Gp, hh::launch_replace(predw_u, predw_v, nullptr, gm, pgd.ny, pgd.nx, 0, s));
      if (smoothing) {
        HH_K(HH_K_VECTOR, 1, 0, 8 * Gp, Gp, hh::launch_smooth(predw_u, pgd.ny, pgd.nx, predu, s));
        HH_K(HH_K_VECTOR, 1, 0, 8 * Gp, Gp, hh::launch_smooth(predw_v, pgd.ny, pgd.nx, predv, s));
        pred_src_u = predu;
        pred_src_v = predv;
      } else {
        pred_src_u = predw_u;
        pred_src_v = predw_v;
      }
      pg.gny = pgd.ny;
      pg.gnx = pgd.nx;
      pg.y0 = pgd.y[0];
      pg.x0 = pgd.x[0];
      pg.ysp = pgd.ny > 1 ? pgd.y[1] - pgd.y[0] : 1.f;
      pg.xsp = pgd.nx > 1 ? pgd.x[1] - pgd.x[0] : 1.f;
      have_pred = true;
    }
    // this pass's grid
    HH_CK(cudaMemcpyAsync(djobs, g.jobs.data(), g.jobs.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    HH_CK(cudaMemcpyAsync(gm, g.gmask.data(), G, cudaMemcpyHostToDevice, s));
    HH_CK(cudaMemcpyAsync(dx, g.x.data(), nx * sizeof(float), cudaMemcpyHostToDevice, s));
    HH_CK(cudaMemcpyAsync(dy, g.y.data(), ny * sizeof(float), cudaMemcpyHostToDevice, s));
    HH_CK(cudaMemsetAsync(resu, 0, G * sizeof(float), s));
    HH_CK(cudaMemsetAsync(resv, 0, G * sizeof(float), s));
    HH_CK(cudaMemsetAsync(ratio, 0, G * sizeof(float), s));
    HH_CK(cudaMemsetAsync(moment, 0, G * sizeof(float), s));
    const float NaN = std::nanf("");
    HH_K(HH_K_VECTOR, 1, 0, 4 * G, G, hh::launch_fill(uncu, NaN, G, s));
    HH_K(HH_K_VECTOR, 1, 0, 4 * G, G, hh::launch_fill(uncv, NaN, G, s));
    if (nalt > 0) {
      HH_K(HH_K_VECTOR, 1, 0, 4 * G * nalt, G, hh::launch_fill(altu, NaN, G * nalt, s));
      HH_K(HH_K_VECTOR, 1, 0, 4 * G * nalt, G, hh::launch_fill(altv, NaN, G * nalt, s));
    }
    const bool unc = p.uncertainty && !force_replace;
    const bool fused_unc = unc && p.max_iterations == 1;
    const bool keep_measured = p.max_iterations > 1 && !(force_replace || p.replace_outliers);
    bool have_prev = false;
    const float* srcA = dA;
    const float* srcB = dB;
    int sweeps = 0;
    for (int it = 1; it <= p.max_iterations; ++it) {
      ++sweeps;
      if (have_pred) {
        HH_K(HH_K_VECTOR, 1, 0, 8 * G, G, hh::launch_node_values(pred_src_u, pred_src_v, pg, dy, ny, dx, nx, u, v, s));
        HH_K(HH_K_DEFORM, 1, 120 * P, 16 * P, P, hh::launch_deform(coefA, coefB, nr, nc, pred_src_u, pred_src_v, pg, warpA, warpB, s));
        srcA = warpA;
        srcB = warpB;
      } else {
        HH_CK(cudaMemsetAsync(u, 0, G * sizeof(float), s));
        HH_CK(cudaMemsetAsync(v, 0, G * sizeof(float), s));
        srcA = dA;
        srcB = dB;
      }
      CorrArgs ca{};
      ca.A = srcA;
      ca.B = srcB;
      ca.mask = dmask;
      ca.ld = nr;
      ca.jobs = djobs;
      ca.njobs = njobs;
      ca.ny = ny;
      ca.G = G;
      ca.apod = tb.apod;
      ca.gain = tb.gain;
      ca.phasew = tb.phasew;
      ca.box_lo = tb.box_lo;
      ca.box_hi = tb.box_hi;
      ca.method = p.method;
      ca.npeaks = p.n_peaks;
      ca.finder = p.peak_finder;
      ca.subpixel = p.subpixel;
      ca.du = resu;
      ca.dv = resv;
      ca.ratio = ratio;
      ca.moment = moment;
      ca.alt_u = nalt > 0 ? altu : nullptr;
      ca.alt_v = nalt > 0 ? altv : nullptr;
      ca.nalt = nalt;
      ca.rec = prec;
      ca.win = p.search[0] != W ? W : 0;
      ca.variant = corr_variant(ctx, p);
      if (!corr_special(p)) HH_TRY(gcorr_prepare(ctx, p, ca));
      HH_K(HH_K_CORRELATE, 1, corr_flops(p, njobs), corr_bytes(p, nalt, njobs), njobs, corr_launch(ctx, p, ca, s));
      if (fused_unc) {
        hh::UQArgs ua{srcA, srcB, dmask, nr, djobs, njobs, ny, W, tb.apod, nullptr, uncu, uncv};
        HH_TRY(uq_prepare(ctx, p.window[0], p.window[1], ua));
        HH_K(HH_K_UQ, 1, uq_flops(p, njobs), 8.0 * p.window[0] * p.window[1] * njobs, njobs,
             hh::launch_uq(ua, s, ctx->num_sms));
      }
      HH_K(HH_K_VECTOR, 1, 0, (28 + 8 * nalt) * G, G, hh::launch_combine(u, v, resu, resv, ratio, moment, nalt > 0 ? altu : nullptr, nalt > 0 ? altv : nullptr,
                               nalt, g.any_mask ? gm : nullptr, G, keep_measured ? measu : nullptr,
                               keep_measured ? measv : nullptr, s));
      HH_TRY(validate_device(ctx, p, ny, nx, u, v, ratio, moment, outl, outl2, gm, g.any_mask,
                             nalt > 0 ? altu : nullptr, nalt > 0 ? altv : nullptr, nalt,
                             force_replace || p.max_iterations > 1));
      if (it == p.max_iterations) break;
      if (p.convergence_tol > 0) {
        if (!have_prev) {
          have_prev = true;
        } else {
          HH_K(HH_K_VECTOR, 1, 0, 24 * G, G, hh::launch_field_change(u, v, prevu, prevv, g.any_mask ? gm : nullptr, G, fc, fcout, s));
          float change = 0.f;
          HH_TRY(read_scalar(ctx, fcout, &change));
          if ((double)change < p.convergence_tol) break;
        }
        HH_CK(cudaMemcpyAsync(prevu, u, G * sizeof(float), cudaMemcpyDeviceToDevice, s));
        HH_CK(cudaMemcpyAsync(prevv, v, G * sizeof(float), cudaMemcpyDeviceToDevice, s));
      }
      // predictor for the next sweep from this sweep's validated field
      HH_CK(cudaMemcpyAsync(predw_u, u, G * sizeof(float), cudaMemcpyDeviceToDevice, s));
      HH_CK(cudaMemcpyAsync(predw_v, v, G * sizeof(float), cudaMemcpyDeviceToDevice, s));
      if (g.any_mask) HH_K(HH_K_VECTOR, 1, 0, 10 * G, G, hh::launch_replace(predw_u, predw_v, nullptr, gm, ny, nx, 0, s));
      if (smoothing) {
        HH_K(HH_K_VECTOR, 1, 0, 8 * G, G, hh::launch_smooth(predw_u, ny, nx, predu, s));
        HH_K(HH_K_VECTOR, 1, 0, 8 * G, G, hh::launch_smooth(predw_v, ny, nx, predv, s));
        pred_src_u = predu;
        pred_src_v = predv;
      } else {
        pred_src_u = predw_u;
        pred_src_v = predw_v;
      }
      pg.gny = ny;
      pg.gnx = nx;
      pg.y0 = g.y[0];
      pg.x0 = g.x[0];
      pg.ysp = ny > 1 ? g.y[1] - g.y[0] : 1.f;
      pg.xsp = nx > 1 ? g.x[1] - g.x[0] : 1.f;
      have_pred = true;
    }
    if (unc && !fused_unc) {
      hh::UQArgs ua{srcA, srcB, dmask, nr, djobs, njobs, ny, W, tb.apod, nullptr, uncu, uncv};
      HH_TRY(uq_prepare(ctx, p.window[0], p.window[1], ua));
      HH_K(HH_K_UQ, 1, uq_flops(p, njobs), 8.0 * p.window[0] * p.window[1] * njobs, njobs,
           hh::launch_uq(ua, s, ctx->num_sms));
    }
    if (keep_measured) HH_K(HH_K_VECTOR, 1, 0, 20 * G, G, hh::launch_restore_measured(u, v, measu, measv, outl, G, s));
    ctx->pass_sweeps[k] = sweeps;
    HH_CK(cudaEventRecord(ctx->events[k + 1], s));
  }
  // final pass -> host
  const Grid& g = grids[np - 1];
  const int64_t G = (int64_t)g.ny * g.nx;
  if (out) {
    out->ny = g.ny;
    out->nx = g.nx;
    if (out->x) memcpy(out->x, g.x.data(), g.nx * sizeof(float));
    if (out->y) memcpy(out->y, g.y.data(), g.ny * sizeof(float));
    if (out->u) HH_CK(cudaMemcpyAsync(out->u, u, G * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out->v) HH_CK(cudaMemcpyAsync(out->v, v, G * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out->peak_ratio) HH_CK(cudaMemcpyAsync(out->peak_ratio, ratio, G * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out->correlation_moment)
      HH_CK(cudaMemcpyAsync(out->correlation_moment, moment, G * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out->uncertainty_u) HH_CK(cudaMemcpyAsync(out->uncertainty_u, uncu, G * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out->uncertainty_v) HH_CK(cudaMemcpyAsync(out->uncertainty_v, uncv, G * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out->outliers) HH_CK(cudaMemcpyAsync(out->outliers, outl, G, cudaMemcpyDeviceToHost, s));
    if (out->mask) memcpy(out->mask, g.gmask.data(), G);
  }
  HH_CK(cudaStreamSynchronize(s));
  for (int k = 0; k < np; ++k) HH_CK(cudaEventElapsedTime(&ctx->pass_ms[k], ctx->events[k], ctx->events[k + 1]));
  return flush_profile(ctx);
}

}  // namespace

// ===========================================================================
extern "C" {

const char* hh_version(void) { return "hammerhead_b200 0.1.0 (sm_100a)"; }

const char* hh_last_error(const hh_ctx* ctx) { return ctx ? ctx->err.c_str() : g_err.c_str(); }

hh_status hh_pass_validate(const hh_pass_desc* p) {
  hh_ctx* ctx = nullptr;
  if (!p) return fail(ctx, HH_ERR_ARG, "pass descriptor is NULL");
  const int32_t *ws = p->window, *ss = p->search, *ov = p->overlap;
  if (!(ws[0] >= 4 && ws[1] >= 4))
    return fail(ctx, HH_ERR_ARG, "window_size must be at least 4 in each dimension, got " + tup(ws));
  if (!(ss[0] >= ws[0] && ss[1] >= ws[1]))
    return fail(ctx, HH_ERR_ARG, "search_area_size must be at least window_size in each dimension, got search_area_size=" +
                                     tup(ss) + " for window_size=" + tup(ws));
  if ((ss[0] - ws[0]) % 2 != 0 || (ss[1] - ws[1]) % 2 != 0)
    return fail(ctx, HH_ERR_ARG,
                "search_area_size - window_size must be even in each dimension so the areas share a center, got "
                "search_area_size=" + tup(ss) + " for window_size=" + tup(ws));
  if (!(ov[0] >= 0 && ov[1] >= 0 && ov[0] < ws[0] && ov[1] < ws[1]))
    return fail(ctx, HH_ERR_ARG, "overlap must satisfy 0 \xe2\x89\xa4 overlap < window_size, got overlap=" + tup(ov) +
                                     " for window_size=" + tup(ws));
  if (p->method != HH_CROSS && p->method != HH_PHASE)
    return fail(ctx, HH_ERR_ARG, "correlation_method must be :cross or :phase, got code " + std::to_string(p->method));
  if (p->apodization != HH_APOD_NONE && p->apodization != HH_APOD_GAUSS)
    return fail(ctx, HH_ERR_ARG, "apodization must be :none or :gauss, got code " + std::to_string(p->apodization));
  if (p->subpixel < HH_GAUSS3 || p->subpixel > HH_SUBPIXEL_NONE)
    return fail(ctx, HH_ERR_ARG, "subpixel_method must be :gauss3, :gauss9, :gauss2d, or :none, got code " +
                                     std::to_string(p->subpixel));
  if (p->n_peaks < 1) return fail(ctx, HH_ERR_ARG, "n_peaks must be at least 1, got " + std::to_string(p->n_peaks));
  if (p->peak_finder != HH_REGIONALMAX && p->peak_finder != HH_EXCLUSION)
    return fail(ctx, HH_ERR_ARG, "peak_finder must be :exclusion or :regionalmax, got code " + std::to_string(p->peak_finder));
  if (!(p->uod_threshold > 0)) return fail(ctx, HH_ERR_ARG, "uod_threshold must be positive, got " + num(p->uod_threshold));
  if (p->uod_neighborhood < 1)
    return fail(ctx, HH_ERR_ARG, "uod_neighborhood must be at least 1, got " + std::to_string(p->uod_neighborhood));
  if (!(p->min_peak_ratio >= 0))
    return fail(ctx, HH_ERR_ARG, "min_peak_ratio must be non-negative, got " + num(p->min_peak_ratio));
  if (p->max_iterations < 1)
    return fail(ctx, HH_ERR_ARG, "max_iterations must be at least 1, got " + std::to_string(p->max_iterations));
  if (!(p->convergence_tol >= 0))
    return fail(ctx, HH_ERR_ARG, "convergence_tol must be non-negative, got " + num(p->convergence_tol));
  if (p->n_validators < 0 || p->n_validators > HH_MAX_VALIDATORS)
    return fail(ctx, HH_ERR_ARG, "at most " + std::to_string(HH_MAX_VALIDATORS) + " extra validators are supported");
  for (int q = 0; q < p->n_validators; ++q) {
    const hh_validator& v = p->validators[q];
    if (v.kind < HH_VAL_PEAK_RATIO || v.kind > HH_VAL_UOD)
      return fail(ctx, HH_ERR_ARG, "unknown validator code " + std::to_string(v.kind));
    if (v.kind == HH_VAL_UOD && v.neighborhood < 1)
      return fail(ctx, HH_ERR_ARG, "neighborhood_size must be at least 1, got " + std::to_string(v.neighborhood));
    if (v.kind == HH_VAL_UOD && !(v.epsilon > 0))
      return fail(ctx, HH_ERR_ARG, "epsilon must be positive, got " + num(v.epsilon));
  }
  return HH_OK;
}

hh_status hh_check_backend_params(const hh_pass_desc* passes, int32_t npasses) {
  hh_ctx* ctx = nullptr;
  for (int k = 0; k < npasses; ++k) {
    const hh_pass_desc& p = passes[k];
    if (!(p.subpixel == HH_GAUSS3 || p.subpixel == HH_GAUSS9 || p.subpixel == HH_SUBPIXEL_NONE))
      return fail(ctx, HH_ERR_UNSUPPORTED,
                  "backend :b200 supports subpixel_method :gauss3, :gauss9 or :none only (got :gauss2d); use backend = :cpu");
    if (p.keep_correlation_planes)
      return fail(ctx, HH_ERR_UNSUPPORTED,
                  "backend :b200 does not support keep_correlation_planes yet; use backend = :cpu");
    // every window and search-area shape runs: the fused kernels where one
    // exists, the general-shape kernel otherwise (FFT lengths whose prime
    // factors are at most 61, planes up to 4 M points)
    if (!corr_special(p) && !gcorr_shape_ok(p))
      return fail(ctx, HH_ERR_UNSUPPORTED,
                  "backend :b200 has no correlation kernel for an FFT plane of " + std::to_string(fft_rows(p)) + " x " +
                      std::to_string(fft_cols(p)) + " (window_size=" + tup(p.window) + ", search_area_size=" +
                      tup(p.search) + (p.padding ? ", padded" : "") +
                      "): FFT lengths need prime factors of at most 61 and planes at most 4194304 points");
    if (p.n_peaks > hh::KMAX)
      return fail(ctx, HH_ERR_UNSUPPORTED,
                  "backend :b200 locates at most " + std::to_string(hh::KMAX) + " peaks, got n_peaks=" + std::to_string(p.n_peaks));
    if (p.uod_neighborhood > 4)
      return fail(ctx, HH_ERR_UNSUPPORTED, "backend :b200 supports uod_neighborhood <= 4, got " + std::to_string(p.uod_neighborhood));
    for (int q = 0; q < p.n_validators; ++q)
      if (p.validators[q].kind == HH_VAL_UOD && p.validators[q].neighborhood > 4)
        return fail(ctx, HH_ERR_UNSUPPORTED, "backend :b200 supports UOD neighborhood_size <= 4");
  }
  return HH_OK;
}

hh_status hh_pass_grid(int64_t nr, int64_t nc, const hh_pass_desc* p, const uint8_t* mask, double thr, int32_t* ny,
                       int32_t* nx, float* x, float* y, uint8_t* grid_mask, int32_t* jobs, int64_t* njobs) {
  hh_ctx* ctx = nullptr;
  HH_TRY(hh_pass_validate(p));
  Grid g;
  HH_TRY(make_grid(ctx, nr, nc, *p, mask, thr, g));
  if (ny) *ny = g.ny;
  if (nx) *nx = g.nx;
  if (x) memcpy(x, g.x.data(), g.nx * sizeof(float));
  if (y) memcpy(y, g.y.data(), g.ny * sizeof(float));
  if (grid_mask) memcpy(grid_mask, g.gmask.data(), g.gmask.size());
  if (jobs)
    for (size_t k = 0; k < g.jobs.size(); ++k) jobs[k] = g.jobs[k] + 1;
  if (njobs) *njobs = (int64_t)g.jobs.size() / 4;
  return HH_OK;
}

hh_status hh_ctx_create(int32_t device, hh_ctx** out) {
  hh_ctx* ctx = nullptr;
  if (!out) return fail(ctx, HH_ERR_ARG, "output pointer is NULL");
  int n = 0;
  cudaError_t e = cudaGetDeviceCount(&n);
  if (e != cudaSuccess || n == 0)
    return fail(ctx, HH_ERR_CUDA, std::string("no CUDA device available: ") + cudaGetErrorString(e));
  if (device < 0 || device >= n) return fail(ctx, HH_ERR_ARG, "device index out of range");
  ctx = new hh_ctx();
  ctx->device = device;
  hh_status s = set_device(ctx);
  if (s != HH_OK) {
    g_err = ctx->err;
    delete ctx;
    return s;
  }
  cudaDeviceProp prop;
  if (cudaGetDeviceProperties(&prop, device) == cudaSuccess) {
    ctx->num_sms = prop.multiProcessorCount;
    if (prop.major != 10) {
      g_err = "hammerhead_b200 is built for sm_100a (B200); device " + std::to_string(device) + " is sm_" +
              std::to_string(prop.major) + std::to_string(prop.minor);
      delete ctx;
      return HH_ERR_UNSUPPORTED;
    }
  }
  if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMallocHost(&ctx->pinned, 64) != cudaSuccess) {
    g_err = "stream or pinned buffer creation failed";
    delete ctx;
    return HH_ERR_CUDA;
  }
  *out = ctx;
  return HH_OK;
}

void hh_ctx_destroy(hh_ctx* ctx) {
  if (!ctx) return;
  cudaSetDevice(ctx->device);
  if (ctx->stream) cudaStreamSynchronize(ctx->stream);
  if (ctx->bplan_free)
    for (auto& kv : ctx->bplans) ctx->bplan_free(kv.second);
  for (auto& kv : ctx->bufs)
    if (kv.second.p) cudaFree(kv.second.p);
  for (auto& kv : ctx->tables) {
    cudaFree(kv.second.apod);
    if (kv.second.gain) cudaFree(kv.second.gain);
    if (kv.second.phasew) cudaFree(kv.second.phasew);
  }
  for (auto& kv : ctx->bs_factors) {
    cudaFree(kv.second.first);
    cudaFree(kv.second.second);
  }
  for (auto e : ctx->events) cudaEventDestroy(e);
  for (auto e : ctx->evpool) cudaEventDestroy(e);
  for (auto& q : ctx->pending) {
    cudaEventDestroy(q.a);
    cudaEventDestroy(q.b);
  }
  if (ctx->pinned) cudaFreeHost(ctx->pinned);
  if (ctx->stream) cudaStreamDestroy(ctx->stream);
  delete ctx;
}

void* hh_ctx_stream(hh_ctx* ctx) { return ctx ? (void*)ctx->stream : nullptr; }

hh_status hh_run_piv(hh_ctx* ctx, const float* A, const float* B, int64_t nr, int64_t nc, const hh_pass_desc* passes,
                     int32_t npasses, const uint8_t* mask, double thr, int32_t smoothing, hh_result* out) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  if (!A || !B) return fail(ctx, HH_ERR_ARG, "image pointers must not be NULL");
  if (nr < 1 || nc < 1) return fail(ctx, HH_ERR_ARG, "images must be non-empty");
  const int64_t P = nr * nc;
  float *dA, *dB;
  uint8_t* dm = nullptr;
  HH_TRY(buf(ctx, "imgA", (size_t)P, &dA));
  HH_TRY(buf(ctx, "imgB", (size_t)P, &dB));
  HH_CK(cudaMemcpyAsync(dA, A, P * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  HH_CK(cudaMemcpyAsync(dB, B, P * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  if (mask) {
    HH_TRY(buf(ctx, "imgmask", (size_t)P, &dm));
    HH_CK(cudaMemcpyAsync(dm, mask, P, cudaMemcpyHostToDevice, ctx->stream));
  }
  return run_schedule(ctx, dA, dB, nr, nc, passes, npasses, mask, dm, thr, smoothing != 0, out);
}

hh_status hh_run_piv_device(hh_ctx* ctx, const float* dA, const float* dB, int64_t nr, int64_t nc,
                            const hh_pass_desc* passes, int32_t npasses, const uint8_t* dmask, double thr,
                            int32_t smoothing, hh_result* out) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  if (!dA || !dB) return fail(ctx, HH_ERR_ARG, "image pointers must not be NULL");
  std::vector<uint8_t> hmask;
  if (dmask) {
    hmask.resize((size_t)(nr * nc));
    HH_CK(cudaMemcpyAsync(hmask.data(), dmask, hmask.size(), cudaMemcpyDeviceToHost, ctx->stream));
    HH_CK(cudaStreamSynchronize(ctx->stream));
  }
  return run_schedule(ctx, dA, dB, nr, nc, passes, npasses, dmask ? hmask.data() : nullptr, dmask, thr, smoothing != 0,
                      out);
}

hh_status hh_last_pass_times(const hh_ctx* ctx, int32_t npasses, float* ms, int32_t* sweeps) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  for (int k = 0; k < npasses; ++k) {
    if (k >= (int)ctx->pass_ms.size()) return fail(const_cast<hh_ctx*>(ctx), HH_ERR_STATE, "no such pass in the last run");
    if (ms) ms[k] = ctx->pass_ms[k];
    if (sweeps) sweeps[k] = ctx->pass_sweeps[k];
  }
  return HH_OK;
}

// ---- hook-level entry points ---------------------------------------------

hh_status hh_stage_pair(hh_ctx* ctx, const float* A, const float* B, int64_t nr, int64_t nc) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  if (!A || !B || nr < 1 || nc < 1) return fail(ctx, HH_ERR_ARG, "invalid image arguments");
  const int64_t P = nr * nc;
  float *dA, *dB, *cA, *cB;
  HH_TRY(buf(ctx, "imgA", (size_t)P, &dA));
  HH_TRY(buf(ctx, "imgB", (size_t)P, &dB));
  HH_TRY(buf(ctx, "coefA", (size_t)(nr + 2) * (nc + 2), &cA));
  HH_TRY(buf(ctx, "coefB", (size_t)(nr + 2) * (nc + 2), &cB));
  HH_CK(cudaMemcpyAsync(dA, A, P * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  HH_CK(cudaMemcpyAsync(dB, B, P * sizeof(float), cudaMemcpyHostToDevice, ctx->stream));
  HH_TRY(prefilter_pair(ctx, dA, dB, nr, nc, cA, cB));
  HH_CK(cudaStreamSynchronize(ctx->stream));
  ctx->nr = nr;
  ctx->nc = nc;
  ctx->curA = dA;
  ctx->curB = dB;
  ctx->staged = true;
  ctx->hook_mask = nullptr;  // a new pair starts unmasked (hh_stage_mask)
  return HH_OK;
}

hh_status hh_ncc_loss_grad(hh_ctx* ctx, const float* P, int32_t gny, int32_t gnx, float y0, float ysp, float x0,
                           float xsp, int32_t window, int32_t overlap, int32_t device_ptrs, double* loss,
                           float* dLdP) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  if (!ctx->staged) return fail(ctx, HH_ERR_STATE, "no staged pair: call hh_stage_pair first");
  if (!P || !loss) return fail(ctx, HH_ERR_ARG, "predictor and loss pointers must not be NULL");
  if (gny < 1 || gnx < 1) return fail(ctx, HH_ERR_ARG, "predictor grid must be non-empty");
  if (!(ysp > 0) || !(xsp > 0)) return fail(ctx, HH_ERR_ARG, "predictor node spacing must be positive");
  if (window < 2 || window > 64) return fail(ctx, HH_ERR_UNSUPPORTED, "loss windows must be 2..64 px");
  if (overlap < 0 || overlap >= window)
    return fail(ctx, HH_ERR_ARG, "overlap must satisfy 0 \xe2\x89\xa4 overlap < window_size");
  if (window > ctx->nr || window > ctx->nc) return fail(ctx, HH_ERR_ARG, "window exceeds the image size");
  cudaStream_t s = ctx->stream;
  const int64_t G2 = 2 * (int64_t)gny * gnx, Px = ctx->nr * ctx->nc;
  hh::NccArgs a{};
  a.CA = (const float*)ctx->bufs["coefA"].p;
  a.CB = (const float*)ctx->bufs["coefB"].p;
  a.nr = ctx->nr;
  a.nc = ctx->nc;
  a.gny = gny;
  a.gnx = gnx;
  a.y0 = y0;
  a.ysp = ysp;
  a.x0 = x0;
  a.xsp = xsp;
  a.W = window;
  a.step = window - overlap;
  a.wy = (int32_t)((ctx->nr - window) / a.step + 1);
  a.wx = (int32_t)((ctx->nc - window) / a.step + 1);
  float* dP = nullptr;
  if (device_ptrs) {
    a.P = P;
  } else {
    HH_TRY(buf(ctx, "ncc_P", (size_t)G2, &dP));
    HH_CK(cudaMemcpyAsync(dP, P, G2 * sizeof(float), cudaMemcpyHostToDevice, s));
    a.P = dP;
  }
  HH_TRY(buf(ctx, "ncc_wstat", (size_t)6 * a.wy * a.wx, &a.wstat));
  HH_TRY(buf(ctx, "ncc_loss", 1, &a.loss));
  float* dG = nullptr;
  if (dLdP) {
    HH_TRY(buf(ctx, "ncc_gpix", (size_t)2 * Px, &a.gpix));
    if (device_ptrs) {
      a.grad = dLdP;
    } else {
      HH_TRY(buf(ctx, "ncc_grad", (size_t)G2, &dG));
      a.grad = dG;
    }
  }
  const double nwin = (double)a.wy * a.wx;
  HH_K(HH_K_DEFORM, dLdP ? 4 : 2, nwin * window * window * 80.0 + (dLdP ? Px * 240.0 : 0.0), 16.0 * Px,
       (int64_t)nwin, hh::launch_ncc_loss_grad(a, s));
  if (dLdP && !device_ptrs) HH_CK(cudaMemcpyAsync(dLdP, dG, G2 * sizeof(float), cudaMemcpyDeviceToHost, s));
  double* hl = reinterpret_cast<double*>(ctx->pinned);
  HH_CK(cudaMemcpyAsync(hl, a.loss, sizeof(double), cudaMemcpyDeviceToHost, s));
  HH_CK(cudaStreamSynchronize(s));
  *loss = *hl;
  return flush_profile(ctx);
}

hh_status hh_apply_predictor(hh_ctx* ctx, const float* pu, const float* pv, int32_t gny, int32_t gnx, float y0,
                             float ysp, float x0, float xsp, const float* y, int32_t ny, const float* x, int32_t nx,
                             float* node_u, float* node_v, float* warpA_out, float* warpB_out) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  if (!ctx->staged) return fail(ctx, HH_ERR_STATE, "no staged pair: call hh_stage_pair first");
  cudaStream_t s = ctx->stream;
  const int64_t P = ctx->nr * ctx->nc;
  float *dA = (float*)ctx->bufs["imgA"].p, *dB = (float*)ctx->bufs["imgB"].p;
  if (!pu) {
    ctx->curA = dA;
    ctx->curB = dB;
    if (node_u) memset(node_u, 0, (size_t)ny * nx * sizeof(float));
    if (node_v) memset(node_v, 0, (size_t)ny * nx * sizeof(float));
    if (warpA_out) HH_CK(cudaMemcpy(warpA_out, dA, P * sizeof(float), cudaMemcpyDeviceToHost));
    if (warpB_out) HH_CK(cudaMemcpy(warpB_out, dB, P * sizeof(float), cudaMemcpyDeviceToHost));
    return HH_OK;
  }
  if (gny < 1 || gnx < 1) return fail(ctx, HH_ERR_ARG, "predictor grid must be non-empty");
  float *dpu, *dpv, *wA, *wB, *cA = (float*)ctx->bufs["coefA"].p, *cB = (float*)ctx->bufs["coefB"].p;
  HH_TRY(buf(ctx, "hook_pu", (size_t)gny * gnx, &dpu));
  HH_TRY(buf(ctx, "hook_pv", (size_t)gny * gnx, &dpv));
  HH_TRY(buf(ctx, "warpA", (size_t)P, &wA));
  HH_TRY(buf(ctx, "warpB", (size_t)P, &wB));
  HH_CK(cudaMemcpyAsync(dpu, pu, (size_t)gny * gnx * sizeof(float), cudaMemcpyHostToDevice, s));
  HH_CK(cudaMemcpyAsync(dpv, pv, (size_t)gny * gnx * sizeof(float), cudaMemcpyHostToDevice, s));
  hh::PredGrid g{gny, gnx, y0, ysp, x0, xsp};
  HH_K(HH_K_DEFORM, 1, 0, 0, 0, hh::launch_deform(cA, cB, ctx->nr, ctx->nc, dpu, dpv, g, wA, wB, s));
  if (node_u && node_v && ny > 0 && nx > 0) {
    float *dy, *dx, *nu, *nv;
    HH_TRY(buf(ctx, "hook_y", ny, &dy));
    HH_TRY(buf(ctx, "hook_x", nx, &dx));
    HH_TRY(buf(ctx, "hook_nu", (size_t)ny * nx, &nu));
    HH_TRY(buf(ctx, "hook_nv", (size_t)ny * nx, &nv));
    HH_CK(cudaMemcpyAsync(dy, y, ny * sizeof(float), cudaMemcpyHostToDevice, s));
    HH_CK(cudaMemcpyAsync(dx, x, nx * sizeof(float), cudaMemcpyHostToDevice, s));
    HH_K(HH_K_VECTOR, 1, 0, 0, 0, hh::launch_node_values(dpu, dpv, g, dy, ny, dx, nx, nu, nv, s));
    HH_CK(cudaMemcpyAsync(node_u, nu, (size_t)ny * nx * sizeof(float), cudaMemcpyDeviceToHost, s));
    HH_CK(cudaMemcpyAsync(node_v, nv, (size_t)ny * nx * sizeof(float), cudaMemcpyDeviceToHost, s));
  }
  if (warpA_out) HH_CK(cudaMemcpyAsync(warpA_out, wA, P * sizeof(float), cudaMemcpyDeviceToHost, s));
  if (warpB_out) HH_CK(cudaMemcpyAsync(warpB_out, wB, P * sizeof(float), cudaMemcpyDeviceToHost, s));
  HH_CK(cudaStreamSynchronize(s));
  ctx->curA = wA;
  ctx->curB = wB;
  return HH_OK;
}

// Jobs of a hook call (1-based, from the caller) checked and copied to the
// device 0-based; the window is wr x wc and (mr, mc) the margins of an
// enlarged search area around it.
static hh_status hook_jobs(hh_ctx* ctx, const int32_t* jobs, int64_t njobs, int64_t nr, int64_t nc, int wr, int wc,
                           int32_t** djobs_out, int32_t* ny_out, int mr = 0, int mc = 0) {
  std::vector<int32_t> hj((size_t)4 * njobs);
  int32_t ny = 1;
  for (int64_t k = 0; k < njobs; ++k) {
    const int32_t gi = jobs[4 * k] - 1, gj = jobs[4 * k + 1] - 1, rs = jobs[4 * k + 2] - 1, cs = jobs[4 * k + 3] - 1;
    if (rs - mr < 0 || cs - mc < 0 || rs + wr + mr > nr || cs + wc + mc > nc || gi < 0 || gj < 0)
      return fail(ctx, HH_ERR_ARG, "job " + std::to_string(k + 1) + " lies outside the image");
    hj[4 * k] = gi;
    hj[4 * k + 1] = gj;
    hj[4 * k + 2] = rs;
    hj[4 * k + 3] = cs;
    ny = std::max(ny, gi + 1);
  }
  int32_t* dj;
  HH_TRY(buf(ctx, "hook_jobs", (size_t)4 * std::max<int64_t>(njobs, 1), &dj));
  HH_CK(cudaMemcpyAsync(dj, hj.data(), hj.size() * sizeof(int32_t), cudaMemcpyHostToDevice, ctx->stream));
  *djobs_out = dj;
  *ny_out = ny;
  return HH_OK;
}

static hh_status hook_correlate(hh_ctx* ctx, const hh_pass_desc* p, const int32_t* jobs, int64_t njobs, float* out,
                                int32_t* locs, double* uq, float* planes) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  if (!ctx->staged) return fail(ctx, HH_ERR_STATE, "no staged pair: call hh_stage_pair first");
  HH_TRY(check_passes(ctx, p, 1));
  if (njobs <= 0) return HH_OK;
  cudaStream_t s = ctx->stream;
  const int W = p->window[0], K = std::max(p->n_peaks, 2);
  const int64_t PL = (int64_t)fft_rows(*p) * fft_cols(*p);  // plane size
  int32_t* dj;
  int32_t ny;
  HH_TRY(hook_jobs(ctx, jobs, njobs, ctx->nr, ctx->nc, p->window[0], p->window[1], &dj, &ny,
                   (p->search[0] - p->window[0]) / 2, (p->search[1] - p->window[1]) / 2));
  Tables tb;
  HH_TRY(get_tables(ctx, *p, tb));
  float *dpk = nullptr, *dpl = nullptr;
  int32_t* dlc = nullptr;
  double* duq = nullptr;
  if (out) HH_TRY(buf(ctx, "hook_packed", (size_t)(5 + 2 * (K - 1)) * njobs, &dpk));
  if (locs) HH_TRY(buf(ctx, "hook_locs", (size_t)2 * K * njobs, &dlc));
  if (planes) HH_TRY(buf(ctx, "hook_planes", (size_t)PL * njobs, &dpl));
  float* drec;
  HH_TRY(buf(ctx, "hook_rec", hh::correlate_record_words(p->n_peaks) * njobs, &drec));
  CorrArgs ca{};
  ca.A = ctx->curA;
  ca.B = ctx->curB;
  ca.ld = ctx->nr;
  ca.jobs = dj;
  ca.njobs = njobs;
  ca.ny = ny;
  ca.G = 0;
  ca.apod = tb.apod;
  ca.gain = tb.gain;
  ca.phasew = tb.phasew;
  ca.box_lo = tb.box_lo;
  ca.box_hi = tb.box_hi;
  ca.method = p->method;
  ca.npeaks = p->n_peaks;
  ca.finder = p->peak_finder;
  ca.subpixel = p->subpixel;
  ca.mask = ctx->hook_mask;
  ca.packed = dpk;
  ca.locs = dlc;
  ca.planes = dpl;
  ca.rec = drec;
  ca.win = p->search[0] != W ? W : 0;
  ca.variant = corr_variant(ctx, *p);
  if (!corr_special(*p)) HH_TRY(gcorr_prepare(ctx, *p, ca));
  HH_K(HH_K_CORRELATE, 1, 0, 0, 0, corr_launch(ctx, *p, ca, s));
  if (uq) {
    HH_TRY(buf(ctx, "hook_uq", (size_t)88 * njobs, &duq));
    hh::UQArgs ua{ctx->curA, ctx->curB, ctx->hook_mask, ctx->nr, dj, njobs, ny, W, tb.apod, duq, nullptr, nullptr};
    HH_TRY(uq_prepare(ctx, p->window[0], p->window[1], ua));
    HH_K(HH_K_UQ, 1, 0, 0, 0, hh::launch_uq(ua, s, ctx->num_sms));
    HH_CK(cudaMemcpyAsync(uq, duq, (size_t)88 * njobs * sizeof(double), cudaMemcpyDeviceToHost, s));
  }
  if (out) HH_CK(cudaMemcpyAsync(out, dpk, (size_t)(5 + 2 * (K - 1)) * njobs * sizeof(float), cudaMemcpyDeviceToHost, s));
  if (locs) HH_CK(cudaMemcpyAsync(locs, dlc, (size_t)2 * K * njobs * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  if (planes) HH_CK(cudaMemcpyAsync(planes, dpl, (size_t)PL * njobs * sizeof(float), cudaMemcpyDeviceToHost, s));
  HH_CK(cudaStreamSynchronize(s));
  return HH_OK;
}

hh_status hh_stage_mask(hh_ctx* ctx, const uint8_t* mask) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  if (!ctx->staged) return fail(ctx, HH_ERR_STATE, "no staged pair: call hh_stage_pair first");
  if (!mask) {
    ctx->hook_mask = nullptr;
    return HH_OK;
  }
  uint8_t* dm;
  HH_TRY(buf(ctx, "hook_mask", (size_t)(ctx->nr * ctx->nc), &dm));
  HH_CK(cudaMemcpyAsync(dm, mask, (size_t)(ctx->nr * ctx->nc), cudaMemcpyHostToDevice, ctx->stream));
  HH_CK(cudaStreamSynchronize(ctx->stream));
  ctx->hook_mask = dm;
  return HH_OK;
}

hh_status hh_process_windows(hh_ctx* ctx, const hh_pass_desc* p, const int32_t* jobs, int64_t njobs, float* out,
                             int32_t* locs, double* uq) {
  return hook_correlate(ctx, p, jobs, njobs, out, locs, uq, nullptr);
}

hh_status hh_correlation_planes(hh_ctx* ctx, const hh_pass_desc* p, const int32_t* jobs, int64_t njobs, float* planes) {
  if (!planes) return fail(ctx, HH_ERR_ARG, "planes pointer is NULL");
  return hook_correlate(ctx, p, jobs, njobs, nullptr, nullptr, nullptr, planes);
}

hh_status hh_analyze_planes(hh_ctx* ctx, const float* planes, int64_t nplanes, int32_t nr, int32_t nc, int32_t n_peaks,
                            int32_t peak_finder, int32_t subpixel, float* out, int32_t* locs) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  if (nr < 1 || nc < 1 || nplanes < 0 || !planes) return fail(ctx, HH_ERR_ARG, "invalid plane arguments");
  if (n_peaks < 1) return fail(ctx, HH_ERR_ARG, "n_peaks must be at least 1, got " + std::to_string(n_peaks));
  if (n_peaks > hh::KMAX) return fail(ctx, HH_ERR_UNSUPPORTED, "at most 8 peaks per plane on the device");
  if ((int64_t)nr * nc * 4 > 180 * 1024) return fail(ctx, HH_ERR_UNSUPPORTED, "plane too large for the analysis kernel");
  if (subpixel == HH_GAUSS2D) return fail(ctx, HH_ERR_UNSUPPORTED, "subpixel_method :gauss2d is not on the device path");
  const int K = std::max(n_peaks, 2);
  cudaStream_t s = ctx->stream;
  float *dp, *dout;
  int32_t* dl;
  HH_TRY(buf(ctx, "ana_planes", (size_t)nr * nc * std::max<int64_t>(nplanes, 1), &dp));
  HH_TRY(buf(ctx, "ana_out", (size_t)(5 + 2 * (K - 1)) * std::max<int64_t>(nplanes, 1), &dout));
  HH_TRY(buf(ctx, "ana_locs", (size_t)2 * K * std::max<int64_t>(nplanes, 1), &dl));
  HH_CK(cudaMemcpyAsync(dp, planes, (size_t)nr * nc * nplanes * sizeof(float), cudaMemcpyHostToDevice, s));
  hh::AnalyzeArgs aa{dp, nplanes, nr, nc, n_peaks, peak_finder, subpixel, dout, dl};
  HH_K(HH_K_CORRELATE, 1, 0, 0, 0, hh::launch_analyze_planes(aa, s));
  if (out) HH_CK(cudaMemcpyAsync(out, dout, (size_t)(5 + 2 * (K - 1)) * nplanes * sizeof(float), cudaMemcpyDeviceToHost, s));
  if (locs) HH_CK(cudaMemcpyAsync(locs, dl, (size_t)2 * K * nplanes * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
  HH_CK(cudaStreamSynchronize(s));
  return HH_OK;
}

hh_status hh_validate(hh_ctx* ctx, const hh_pass_desc* p, int32_t ny, int32_t nx, float* u, float* v,
                      const float* peak_ratio, const float* moment, uint8_t* outliers, const uint8_t* mask,
                      const float* alt_u, const float* alt_v, int32_t nalt, int32_t force_replace) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  HH_TRY(check_passes(ctx, p, 1));
  const int64_t G = (int64_t)ny * nx;
  if (G <= 0) return HH_OK;
  cudaStream_t s = ctx->stream;
  float *du, *dv, *dr, *dm, *au = nullptr, *av = nullptr;
  uint8_t *o1, *o2, *gm;
  HH_TRY(buf(ctx, "val_u", G, &du));
  HH_TRY(buf(ctx, "val_v", G, &dv));
  HH_TRY(buf(ctx, "val_r", G, &dr));
  HH_TRY(buf(ctx, "val_m", G, &dm));
  HH_TRY(buf(ctx, "val_o1", G, &o1));
  HH_TRY(buf(ctx, "val_o2", G, &o2));
  HH_TRY(buf(ctx, "val_gm", G, &gm));
  HH_CK(cudaMemcpyAsync(du, u, G * 4, cudaMemcpyHostToDevice, s));
  HH_CK(cudaMemcpyAsync(dv, v, G * 4, cudaMemcpyHostToDevice, s));
  if (peak_ratio) HH_CK(cudaMemcpyAsync(dr, peak_ratio, G * 4, cudaMemcpyHostToDevice, s));
  else HH_K(HH_K_VECTOR, 1, 0, 0, 0, hh::launch_fill(dr, 2.0f, G, s));
  if (moment) HH_CK(cudaMemcpyAsync(dm, moment, G * 4, cudaMemcpyHostToDevice, s));
  else HH_K(HH_K_VECTOR, 1, 0, 0, 0, hh::launch_fill(dm, 0.0f, G, s));
  bool any_mask = false;
  if (mask) {
    for (int64_t k = 0; k < G; ++k) any_mask |= mask[k] != 0;
    HH_CK(cudaMemcpyAsync(gm, mask, G, cudaMemcpyHostToDevice, s));
  } else {
    HH_CK(cudaMemsetAsync(gm, 0, G, s));
  }
  if (alt_u && nalt > 0) {
    HH_TRY(buf(ctx, "val_au", G * nalt, &au));
    HH_TRY(buf(ctx, "val_av", G * nalt, &av));
    HH_CK(cudaMemcpyAsync(au, alt_u, G * nalt * 4, cudaMemcpyHostToDevice, s));
    HH_CK(cudaMemcpyAsync(av, alt_v, G * nalt * 4, cudaMemcpyHostToDevice, s));
  }
  // outliers start from all-false, as in piv_pass; the array is output only
  HH_TRY(validate_device(ctx, *p, ny, nx, du, dv, dr, dm, o1, o2, gm, any_mask, au, av, au ? nalt : 0,
                         force_replace != 0));
  std::vector<uint8_t> o(G);
  HH_CK(cudaMemcpyAsync(o.data(), o1, G, cudaMemcpyDeviceToHost, s));
  HH_CK(cudaMemcpyAsync(u, du, G * 4, cudaMemcpyDeviceToHost, s));
  HH_CK(cudaMemcpyAsync(v, dv, G * 4, cudaMemcpyDeviceToHost, s));
  HH_CK(cudaStreamSynchronize(s));
  for (int64_t k = 0; k < G; ++k) outliers[k] = o[k];
  return HH_OK;
}

hh_status hh_uod(hh_ctx* ctx, const float* u, const float* v, int32_t ny, int32_t nx, double thr, int32_t nb,
                 double eps, const uint8_t* exclude, uint8_t* flags) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  if (nb < 1) return fail(ctx, HH_ERR_ARG, "neighborhood_size must be at least 1, got " + std::to_string(nb));
  if (!(eps > 0)) return fail(ctx, HH_ERR_ARG, "epsilon must be positive, got " + num(eps));
  if (nb > 4) return fail(ctx, HH_ERR_UNSUPPORTED, "neighborhood_size <= 4 on the device");
  const int64_t G = (int64_t)ny * nx;
  if (G <= 0) return HH_OK;
  cudaStream_t s = ctx->stream;
  float *du, *dv;
  uint8_t *dx = nullptr, *df;
  HH_TRY(buf(ctx, "uod_u", G, &du));
  HH_TRY(buf(ctx, "uod_v", G, &dv));
  HH_TRY(buf(ctx, "uod_f", G, &df));
  HH_CK(cudaMemcpyAsync(du, u, G * 4, cudaMemcpyHostToDevice, s));
  HH_CK(cudaMemcpyAsync(dv, v, G * 4, cudaMemcpyHostToDevice, s));
  if (exclude) {
    HH_TRY(buf(ctx, "uod_x", G, &dx));
    HH_CK(cudaMemcpyAsync(dx, exclude, G, cudaMemcpyHostToDevice, s));
  }
  HH_K(HH_K_VECTOR, 1, 0, 0, 0, hh::launch_uod(du, dv, ny, nx, thr, nb, eps, dx, df, 0, s));
  HH_CK(cudaMemcpyAsync(flags, df, G, cudaMemcpyDeviceToHost, s));
  HH_CK(cudaStreamSynchronize(s));
  return HH_OK;
}

hh_status hh_replace_vectors(hh_ctx* ctx, float* u, float* v, int32_t ny, int32_t nx, const uint8_t* invalid) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  const int64_t G = (int64_t)ny * nx;
  if (G <= 0) return HH_OK;
  cudaStream_t s = ctx->stream;
  float *du, *dv;
  uint8_t* di;
  HH_TRY(buf(ctx, "rep_u", G, &du));
  HH_TRY(buf(ctx, "rep_v", G, &dv));
  HH_TRY(buf(ctx, "rep_i", G, &di));
  HH_CK(cudaMemcpyAsync(du, u, G * 4, cudaMemcpyHostToDevice, s));
  HH_CK(cudaMemcpyAsync(dv, v, G * 4, cudaMemcpyHostToDevice, s));
  HH_CK(cudaMemcpyAsync(di, invalid, G, cudaMemcpyHostToDevice, s));
  HH_K(HH_K_VECTOR, 1, 0, 0, 0, hh::launch_replace(du, dv, di, nullptr, ny, nx, 0, s));
  HH_CK(cudaMemcpyAsync(u, du, G * 4, cudaMemcpyDeviceToHost, s));
  HH_CK(cudaMemcpyAsync(v, dv, G * 4, cudaMemcpyDeviceToHost, s));
  HH_CK(cudaStreamSynchronize(s));
  return HH_OK;
}

hh_status hh_smooth_field(hh_ctx* ctx, const float* f, int32_t ny, int32_t nx, float* out) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  const int64_t G = (int64_t)ny * nx;
  if (G <= 0) return HH_OK;
  cudaStream_t s = ctx->stream;
  float *df, *dout;
  HH_TRY(buf(ctx, "sm_in", G, &df));
  HH_TRY(buf(ctx, "sm_out", G, &dout));
  HH_CK(cudaMemcpyAsync(df, f, G * 4, cudaMemcpyHostToDevice, s));
  HH_K(HH_K_VECTOR, 1, 0, 0, 0, hh::launch_smooth(df, ny, nx, dout, s));
  HH_CK(cudaMemcpyAsync(out, dout, G * 4, cudaMemcpyDeviceToHost, s));
  HH_CK(cudaStreamSynchronize(s));
  return HH_OK;
}

hh_status hh_field_change(hh_ctx* ctx, const float* u, const float* v, const float* pu, const float* pv,
                          const uint8_t* mask, int64_t n, float* change) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  if (n <= 0) {
    *change = 0.f;
    return HH_OK;
  }
  cudaStream_t s = ctx->stream;
  float *d[4], *sc, *o;
  uint8_t* dm = nullptr;
  const char* names[4] = {"fc_u", "fc_v", "fc_pu", "fc_pv"};
  const float* src[4] = {u, v, pu, pv};
  for (int q = 0; q < 4; ++q) {
    HH_TRY(buf(ctx, names[q], n, &d[q]));
    HH_CK(cudaMemcpyAsync(d[q], src[q], n * 4, cudaMemcpyHostToDevice, s));
  }
  if (mask) {
    HH_TRY(buf(ctx, "fc_m", n, &dm));
    HH_CK(cudaMemcpyAsync(dm, mask, n, cudaMemcpyHostToDevice, s));
  }
  HH_TRY(buf(ctx, "fc_s", n + 64, &sc));
  HH_TRY(buf(ctx, "fc_o", 4, &o));
  HH_K(HH_K_VECTOR, 1, 0, 0, 0, hh::launch_field_change(d[0], d[1], d[2], d[3], dm, n, sc, o, s));
  return read_scalar(ctx, o, change);
}

hh_status hh_finalize_uncertainty(const double* stats, int64_t n, float* su, float* sv) {
  // host restatement of finalize_uncertainty for callers holding raw stats
  static int dr[40], dc[40], rs[5];
  static bool init = false;
  if (!init) {
    int tmp[40][2], q = 0;
    for (int c = 0; c <= 4; ++c)
      for (int r = (c == 0 ? 1 : -4); r <= 4; ++r) {
        tmp[q][0] = r;
        tmp[q][1] = c;
        ++q;
      }
    int k = 0;
    for (int ring = 1; ring <= 4; ++ring) {
      rs[ring - 1] = k;
      for (int t = 0; t < 40; ++t)
        if (std::max(std::abs(tmp[t][0]), tmp[t][1]) == ring) {
          dr[k] = tmp[t][0];
          dc[k] = tmp[t][1];
          ++k;
        }
    }
    rs[4] = 40;
    init = true;
  }
  auto fin = [&](const double* s) -> float {
    const double C0 = s[0], Cp = s[1], Cm = s[2], S00 = s[3];
    double s2 = S00;
    for (int ring = 0; ring < 4; ++ring) {
      double mx = -INFINITY;
      for (int k = rs[ring]; k < rs[ring + 1]; ++k) mx = std::max(mx, s[4 + k]);
      if (mx < 0.05 * S00) break;
      for (int k = rs[ring]; k < rs[ring + 1]; ++k) s2 += 2 * s[4 + k];
    }
    const double sdc = std::sqrt(std::max(s2, 0.0)), Cpm = (Cp + Cm) / 2, lo = Cpm - sdc / 2, hi = Cpm + sdc / 2;
    if (!(C0 > 0 && lo > 0)) return std::nanf("");
    const double den = 2 * std::log(C0) - std::log(hi) - std::log(lo);
    if (!(den > 0)) return std::nanf("");
    return (float)((std::log(hi) - std::log(lo)) / (2 * den));
  };
  for (int64_t j = 0; j < n; ++j) {
    if (su) su[j] = fin(stats + 88 * j);
    if (sv) sv[j] = fin(stats + 88 * j + 44);
  }
  (void)dr;
  (void)dc;
  return HH_OK;
}

hh_status hh_set_profiling(hh_ctx* ctx, int32_t enable) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  ctx->prof = enable != 0;
  return HH_OK;
}

hh_status hh_profile_read(hh_ctx* ctx, hh_kernel_profile* out, int32_t reset) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  HH_CK(cudaStreamSynchronize(ctx->stream));
  HH_TRY(flush_profile(ctx));
  if (out)
    for (int k = 0; k < HH_K_CLASSES; ++k) out[k] = ctx->acc[k];
  if (reset)
    for (int k = 0; k < HH_K_CLASSES; ++k) ctx->acc[k] = hh_kernel_profile{};
  return HH_OK;
}

int64_t hh_launch_count(const hh_ctx* ctx) { return ctx ? ctx->launches : 0; }

}  // extern "C"

// ---------------------------------------------------------------------------
// Autotuning of the correlation kernel's CTA shape.
static void drop_plans(hh_ctx* ctx) {  // batched graphs captured with an older choice
  if (ctx->bplan_free)
    for (auto& kv : ctx->bplans) ctx->bplan_free(kv.second);
  ctx->bplans.clear();
}

extern "C" hh_status hh_debug_fail_alloc(hh_ctx* ctx, int64_t after) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  ctx->fail_alloc_after = after < 0 ? -1 : after;
  return HH_OK;
}

extern "C" int32_t hh_corr_fused(const hh_pass_desc* p) { return p && corr_special(*p) ? 1 : 0; }

extern "C" hh_status hh_set_corr_variant(hh_ctx* ctx, int32_t fft_size_, int32_t window, int32_t variant) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  if (variant < 0 || variant >= HH_CORR_VARIANTS)
    return fail(ctx, HH_ERR_ARG, "variant must be in [0, " + std::to_string(HH_CORR_VARIANTS) + "), got " +
                                     std::to_string(variant));
  if (!hh::correlate_supported(fft_size_, window))
    return fail(ctx, HH_ERR_ARG, "no correlation kernel for FFT size " + std::to_string(fft_size_) + " and window " +
                                     std::to_string(window));
  HH_TRY(set_device(ctx));
  HH_CK(cudaStreamSynchronize(ctx->stream));
  ctx->corr_var[{fft_size_, window}] = variant;
  drop_plans(ctx);
  return HH_OK;
}

extern "C" hh_status hh_autotune_correlation(hh_ctx* ctx, const hh_pass_desc* p, int32_t reps, float* variant_ms,
                                             int32_t* best) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  if (!ctx->staged) return fail(ctx, HH_ERR_STATE, "no staged pair: call hh_stage_pair first");
  HH_TRY(check_passes(ctx, p, 1));
  const hh_status cs = hh_check_backend_params(p, 1);
  if (cs != HH_OK) return fail(ctx, cs, hh_last_error(nullptr));
  if (p->search[0] != p->window[0])
    return fail(ctx, HH_ERR_ARG, "autotuning covers passes with equal window and search area");
  if (!corr_special(*p))
    return fail(ctx, HH_ERR_ARG, "autotuning covers the fused correlation kernels (square windows of the specialised "
                                 "sizes); the general-shape kernel has one shape");
  if (reps < 1) return fail(ctx, HH_ERR_ARG, "reps must be at least 1, got " + std::to_string(reps));
  Grid g;
  HH_TRY(make_grid(ctx, ctx->nr, ctx->nc, *p, nullptr, 0.5, g));
  const int64_t njobs = (int64_t)g.jobs.size() / 4;
  if (njobs < 1) return fail(ctx, HH_ERR_ARG, "the staged pair holds no window of this pass");
  cudaStream_t s = ctx->stream;
  const int N = fft_size(*p);
  const int64_t G = (int64_t)g.ny * g.nx;
  Tables tb;
  HH_TRY(get_tables(ctx, *p, tb));
  int32_t* dj;
  float *du, *dv, *ratio, *moment, *alt = nullptr, *rec;
  const int nalt = p->n_peaks - 1;
  HH_TRY(buf(ctx, "tune_jobs", (size_t)g.jobs.size(), &dj));
  HH_TRY(buf(ctx, "tune_out", (size_t)4 * G, &du));
  dv = du + G;
  ratio = dv + G;
  moment = ratio + G;
  if (nalt > 0) HH_TRY(buf(ctx, "tune_alt", (size_t)2 * nalt * G, &alt));
  HH_TRY(buf(ctx, "tune_rec", hh::correlate_record_words(p->n_peaks) * njobs, &rec));
  HH_CK(cudaMemcpyAsync(dj, g.jobs.data(), g.jobs.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
  CorrArgs ca{};
  ca.A = ctx->curA;
  ca.B = ctx->curB;
  ca.ld = ctx->nr;
  ca.jobs = dj;
  ca.njobs = njobs;
  ca.ny = g.ny;
  ca.G = G;
  ca.apod = tb.apod;
  ca.gain = tb.gain;
  ca.phasew = tb.phasew;
  ca.box_lo = tb.box_lo;
  ca.box_hi = tb.box_hi;
  ca.method = p->method;
  ca.npeaks = p->n_peaks;
  ca.finder = p->peak_finder;
  ca.subpixel = p->subpixel;
  ca.du = du;
  ca.dv = dv;
  ca.ratio = ratio;
  ca.moment = moment;
  ca.alt_u = alt;
  ca.alt_v = nalt > 0 ? alt + (int64_t)nalt * G : nullptr;
  ca.nalt = nalt;
  ca.rec = rec;
  cudaEvent_t e0, e1;
  HH_CK(cudaEventCreate(&e0));
  HH_CK(cudaEventCreate(&e1));
  double tot[HH_CORR_VARIANTS] = {};
  cudaError_t err = cudaSuccess;
  for (int r = -1; r < reps && err == cudaSuccess; ++r)  // round -1 warms every shape up
    for (int v = 0; v < HH_CORR_VARIANTS && err == cudaSuccess; ++v) {
      ca.variant = v;
      err = cudaEventRecord(e0, s);
      if (err == cudaSuccess) err = hh::launch_correlate(ca, N, p->search[0], s, ctx->num_sms);
      if (err == cudaSuccess) err = cudaEventRecord(e1, s);
      if (err == cudaSuccess) err = cudaEventSynchronize(e1);
      float ms = 0.f;
      if (err == cudaSuccess) err = cudaEventElapsedTime(&ms, e0, e1);
      if (r >= 0) tot[v] += ms;
    }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  HH_CK(err);
  int b = 0;
  for (int v = 0; v < HH_CORR_VARIANTS; ++v) {
    if (variant_ms) variant_ms[v] = (float)(tot[v] / reps);
    if (tot[v] < tot[b]) b = v;
  }
  if (best) *best = b;
  ctx->corr_var[{N, (int)p->search[0]}] = b;
  drop_plans(ctx);
  return HH_OK;
}
