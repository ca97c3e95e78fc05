// Ensemble (sum-of-correlation) PIV on the device: run_piv_ensemble
// (src/ensemble.jl:51-205). Per pass, every pair is staged and deformed by
// the shared predictor, the correlation kernel adds each window's plane to a
// device-resident accumulator (and the Wieneke statistics to FP64 sums), and
// after the last pair the summed planes are analysed once, combined with the
// predictor and validated exactly like a WIDIM sweep. Only the final vector
// grid returns to the host. With the pairs split over processes, the context
// reducer (hh_set_ensemble_reducer) turns each pass's partial sums into the
// sums over all processes before the analysis.
#include "hh_ctx.h"

using namespace hhd;

extern "C" hh_status hh_run_ensemble(hh_ctx* ctx, const hh_batch_pair* pairs, int32_t npairs,
                                     const hh_pass_desc* passes, int32_t np, const uint8_t* hmask, double thr,
                                     int32_t smoothing, int32_t flags, hh_result* out) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  if (!pairs || npairs < 1) return fail(ctx, HH_ERR_ARG, "pairs must not be empty");
  HH_TRY(check_passes(ctx, passes, np));
  if (!(thr > 0 && thr <= 1)) return fail(ctx, HH_ERR_ARG, "mask_threshold must be in (0, 1], got " + num(thr));
  const int64_t nr = pairs[0].nr, nc = pairs[0].nc, P = nr * nc;
  if (nr < 1 || nc < 1) return fail(ctx, HH_ERR_ARG, "images must be non-empty");
  for (int q = 0; q < npairs; ++q) {
    if (pairs[q].nr != nr || pairs[q].nc != nc)
      return fail(ctx, HH_ERR_ARG, "all pairs must share the image size (" + std::to_string(nr) + ", " +
                                       std::to_string(nc) + "), got (" + std::to_string(pairs[q].nr) + ", " +
                                       std::to_string(pairs[q].nc) + ")");
    if (!pairs[q].A || !pairs[q].B) return fail(ctx, HH_ERR_ARG, "image pointer is NULL");
    if (pairs[q].format < HH_PIX_F32 || pairs[q].format > HH_PIX_U16_RAW)
      return fail(ctx, HH_ERR_ARG, "unknown pixel format " + std::to_string(pairs[q].format));
  }
  const bool device_inputs = (flags & HH_BATCH_DEVICE_INPUTS) != 0;
  cudaStream_t s = ctx->stream;
  std::vector<Grid> grids(np);
  int64_t Gmax = 1, Jmax = 1, accmax = 1;
  int nalt_max = 0;
  for (int k = 0; k < np; ++k) {
    HH_TRY(make_grid(ctx, nr, nc, passes[k], hmask, thr, grids[k]));
    const int64_t nj = (int64_t)grids[k].jobs.size() / 4;
    const int64_t PL = (int64_t)fft_rows(passes[k]) * fft_cols(passes[k]);
    Gmax = std::max<int64_t>(Gmax, (int64_t)grids[k].ny * grids[k].nx);
    Jmax = std::max<int64_t>(Jmax, nj);
    accmax = std::max<int64_t>(accmax, nj * PL);
    nalt_max = std::max(nalt_max, passes[k].n_peaks - 1);
  }
  float *dA = nullptr, *dB = nullptr, *coefA, *coefB, *warpA, *warpB, *acc;
  uint8_t* dmask = nullptr;
  double* stats;
  bool any_u16 = false;
  for (int q = 0; q < npairs; ++q) any_u16 |= pairs[q].format != HH_PIX_F32;
  uint16_t *d16A = nullptr, *d16B = nullptr;
  if (!device_inputs || any_u16) {
    HH_TRY(buf(ctx, "ens_A", (size_t)P, &dA));
    HH_TRY(buf(ctx, "ens_B", (size_t)P, &dB));
  }
  if (!device_inputs && any_u16) {
    HH_TRY(buf(ctx, "ens_A16", (size_t)P, &d16A));
    HH_TRY(buf(ctx, "ens_B16", (size_t)P, &d16B));
  }
  if (hmask) {
    HH_TRY(buf(ctx, "ens_mask", (size_t)P, &dmask));
    HH_CK(cudaMemcpyAsync(dmask, hmask, (size_t)P, cudaMemcpyHostToDevice, s));
  }
  HH_TRY(buf(ctx, "coefA", (size_t)(nr + 2) * (nc + 2), &coefA));
  HH_TRY(buf(ctx, "coefB", (size_t)(nr + 2) * (nc + 2), &coefB));
  HH_TRY(buf(ctx, "warpA", (size_t)P, &warpA));
  HH_TRY(buf(ctx, "warpB", (size_t)P, &warpB));
  HH_TRY(buf(ctx, "ens_acc", (size_t)accmax, &acc));
  HH_TRY(buf(ctx, "ens_stats", (size_t)Jmax * 88, &stats));
  float *u, *v, *resu, *resv, *ratio, *moment, *uncu, *uncv, *altu = nullptr, *altv = nullptr, *predu, *predv, *predw_u,
        *predw_v, *dx, *dy;
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
  HH_TRY(buf(ctx, "gx", Gmax, &dx));
  HH_TRY(buf(ctx, "gy", Gmax, &dy));
  HH_TRY(buf(ctx, "outl", Gmax, &outl));
  HH_TRY(buf(ctx, "outl2", Gmax, &outl2));
  HH_TRY(buf(ctx, "gmask", Gmax, &gm));
  HH_TRY(buf(ctx, "jobs", 4 * Jmax, &djobs));
  while ((int)ctx->events.size() < np + 1) {
    cudaEvent_t e;
    HH_CK(cudaEventCreate(&e));
    ctx->events.push_back(e);
  }
  ctx->pass_ms.assign(np, 0.f);
  ctx->pass_sweeps.assign(np, 1);
  HH_CK(cudaEventRecord(ctx->events[0], s));

  const float NaN = std::nanf("");
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
    const int W = p.window[0], NR = fft_rows(p), NC = fft_cols(p);
    const int64_t PL = (int64_t)NR * NC;
    const int nalt = p.n_peaks - 1;
    const bool unc = p.uncertainty && !force_replace;
    Tables tb;
    HH_TRY(get_tables(ctx, p, tb));
    if (k > 0) {  // build_predictor from the previous pass's result (src/pipeline.jl:454-464)
      const Grid& pgd = grids[k - 1];
      const int64_t Gp = (int64_t)pgd.ny * pgd.nx;
      HH_CK(cudaMemcpyAsync(predw_u, u, Gp * sizeof(float), cudaMemcpyDeviceToDevice, s));
      HH_CK(cudaMemcpyAsync(predw_v, v, Gp * sizeof(float), cudaMemcpyDeviceToDevice, s));
      if (pgd.any_mask) {
        HH_CK(cudaMemcpyAsync(gm, pgd.gmask.data(), Gp, cudaMemcpyHostToDevice, s));
        HH_K(HH_K_VECTOR, 1, 0, 10 * Gp, Gp, hh::launch_replace(predw_u, predw_v, nullptr, gm, pgd.ny, pgd.nx, 0, s));
      }
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
    }
    HH_CK(cudaMemcpyAsync(djobs, g.jobs.data(), g.jobs.size() * sizeof(int32_t), cudaMemcpyHostToDevice, s));
    HH_CK(cudaMemcpyAsync(gm, g.gmask.data(), G, cudaMemcpyHostToDevice, s));
    HH_CK(cudaMemcpyAsync(dx, g.x.data(), nx * sizeof(float), cudaMemcpyHostToDevice, s));
    HH_CK(cudaMemcpyAsync(dy, g.y.data(), ny * sizeof(float), cudaMemcpyHostToDevice, s));
    // the shared predictor's node values (zero without one)
    if (k > 0) {
      HH_K(HH_K_VECTOR, 1, 0, 8 * G, G, hh::launch_node_values(pred_src_u, pred_src_v, pg, dy, ny, dx, nx, u, v, s));
    } else {
      HH_CK(cudaMemsetAsync(u, 0, G * sizeof(float), s));
      HH_CK(cudaMemsetAsync(v, 0, G * sizeof(float), s));
    }
    HH_CK(cudaMemsetAsync(acc, 0, (size_t)njobs * PL * sizeof(float), s));
    if (unc) HH_CK(cudaMemsetAsync(stats, 0, (size_t)njobs * 88 * sizeof(double), s));
    for (int q = 0; q < npairs; ++q) {
      const float* A = pairs[q].A;
      const float* B = pairs[q].B;
      if (pairs[q].format != HH_PIX_F32) {  // UInt16 frames: (copy and) convert on the device
        const uint16_t* a16 = reinterpret_cast<const uint16_t*>(A);
        const uint16_t* b16 = reinterpret_cast<const uint16_t*>(B);
        if (!device_inputs) {
          HH_CK(cudaMemcpyAsync(d16A, a16, P * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
          HH_CK(cudaMemcpyAsync(d16B, b16, P * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
          a16 = d16A;
          b16 = d16B;
        }
        const int norm = pairs[q].format == HH_PIX_U16;
        HH_K(HH_K_PREFILTER, 2, 0, 12.0 * P, P, hh::launch_u16_to_f32(a16, P, norm, dA, s));
        HH_K(HH_K_PREFILTER, 0, 0, 0, 0, hh::launch_u16_to_f32(b16, P, norm, dB, s));
        A = dA;
        B = dB;
      } else if (!device_inputs) {
        HH_CK(cudaMemcpyAsync(dA, A, P * sizeof(float), cudaMemcpyHostToDevice, s));
        HH_CK(cudaMemcpyAsync(dB, B, P * sizeof(float), cudaMemcpyHostToDevice, s));
        A = dA;
        B = dB;
      }
      if (k > 0) {
        HH_TRY(prefilter_pair(ctx, A, B, nr, nc, coefA, coefB));
        HH_K(HH_K_DEFORM, 1, 120.0 * P, 16.0 * P, P,
             hh::launch_deform(coefA, coefB, nr, nc, pred_src_u, pred_src_v, pg, warpA, warpB, s));
        A = warpA;
        B = warpB;
      }
      if (njobs > 0) {
        CorrArgs ca{};
        ca.A = A;
        ca.B = B;
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
        ca.planes = acc;
        ca.accumulate = 1;
        ca.win = p.search[0] != W ? W : 0;
        ca.variant = corr_variant(ctx, p);
        if (!corr_special(p)) HH_TRY(gcorr_prepare(ctx, p, ca));
        HH_K(HH_K_CORRELATE, 1, corr_flops(p, njobs), corr_bytes(p, 0, njobs) + 8.0 * PL * njobs, njobs,
             corr_launch(ctx, p, ca, s));
        if (unc) {
          hh::UQArgs ua{};
          ua.A = A;
          ua.B = B;
          ua.mask = dmask;
          ua.ld = nr;
          ua.jobs = djobs;
          ua.njobs = njobs;
          ua.ny = ny;
          ua.W = W;
          ua.apod = tb.apod;
          ua.stats = stats;
          ua.accumulate = 1;
          HH_TRY(uq_prepare(ctx, p.window[0], p.window[1], ua));
          HH_K(HH_K_UQ, 1, uq_flops(p, njobs), 8.0 * p.window[0] * p.window[1] * njobs, njobs,
               hh::launch_uq(ua, s, ctx->num_sms));
        }
      }
    }
    // partial sums of this process's pairs -> sums over all processes
    if (ctx->ens_reduce && njobs > 0) {
      const int64_t nst = unc ? njobs * 88 : 0;
      if (ctx->ens_reduce(ctx->ens_reduce_user, k, acc, njobs * PL, unc ? stats : nullptr, nst, (void*)s) != 0)
        return fail(ctx, HH_ERR_STATE, "ensemble reducer failed in pass " + std::to_string(k + 1));
    }
    // ensemble_analyze! (src/ensemble.jl:273-305): one analysis of every summed plane
    HH_K(HH_K_VECTOR, 1, 0, 4 * G, G, hh::launch_fill(uncu, NaN, G, s));
    HH_K(HH_K_VECTOR, 1, 0, 4 * G, G, hh::launch_fill(uncv, NaN, G, s));
    if (nalt > 0) {
      HH_K(HH_K_VECTOR, 1, 0, 4 * G * nalt, G, hh::launch_fill(altu, NaN, G * nalt, s));
      HH_K(HH_K_VECTOR, 1, 0, 4 * G * nalt, G, hh::launch_fill(altv, NaN, G * nalt, s));
    }
    if (njobs > 0) {
      hh::AnalyzeArgs aa{};
      aa.planes = acc;
      aa.nplanes = njobs;
      aa.nr = NR;
      aa.nc = NC;
      aa.npeaks = p.n_peaks;
      aa.finder = p.peak_finder;
      aa.subpixel = p.subpixel;
      aa.jobs = djobs;
      aa.ny = ny;
      aa.G = G;
      aa.du = resu;
      aa.dv = resv;
      aa.ratio = ratio;
      aa.moment = moment;
      aa.alt_u = nalt > 0 ? altu : nullptr;
      aa.alt_v = nalt > 0 ? altv : nullptr;
      aa.nalt = nalt;
      HH_K(HH_K_CORRELATE, 1, 0, 4.0 * PL * njobs, njobs, hh::launch_analyze_planes(aa, s));
      if (unc) HH_K(HH_K_UQ, 1, 0, 88.0 * 8 * njobs, njobs, hh::launch_uq_finalize(stats, djobs, njobs, ny, uncu, uncv, s));
    }
    HH_K(HH_K_VECTOR, 1, 0, (28 + 8 * nalt) * G, G,
         hh::launch_combine(u, v, resu, resv, ratio, moment, nalt > 0 ? altu : nullptr, nalt > 0 ? altv : nullptr, nalt,
                            g.any_mask ? gm : nullptr, G, nullptr, nullptr, s));
    HH_TRY(validate_device(ctx, p, ny, nx, u, v, ratio, moment, outl, outl2, gm, g.any_mask,
                           nalt > 0 ? altu : nullptr, nalt > 0 ? altv : nullptr, nalt, force_replace));
    HH_CK(cudaEventRecord(ctx->events[k + 1], s));
  }
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

extern "C" hh_status hh_set_ensemble_reducer(hh_ctx* ctx, hh_ensemble_reducer fn, void* user) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  ctx->ens_reduce = fn;
  ctx->ens_reduce_user = fn ? user : nullptr;
  return HH_OK;
}
