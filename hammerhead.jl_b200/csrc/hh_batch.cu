// Batched planar-WIDIM schedule (hh_batch_grid, hh_run_batched).
//
// A plan is built once per batch shape (pair sizes, schedules, mask
// presence): the grids of every pass slot, the descriptor tables
// (hh_batch.h), the per-(FFT size, window, options) job lists, and all
// device storage. The launch sequence of a run -- prefilter, then per slot
// and sweep: node values, deformation, one correlation launch per job class,
// uncertainty, the vector-grid stage with the device-side convergence test,
// the predictor -- depends only on the plan, so it is captured once in a CUDA
// graph and replayed; a call uploads the descriptor tables (image pointers,
// grid masks), replays, and reads back the compact results.
#include "hh_batch.h"
#include "hh_ctx.h"

using namespace hhd;
using hh::BPair;

namespace hhd {

struct BClass {
  int N = 0, W = 0, S = 0, method = 0, npeaks = 1, finder = 0, subpixel = 0, apod = 0, padding = 0;  // S: search area
  hh_pass_desc pd{};  // a pass of this class (its shape and options)
  bool special = true;  // a fused kernel exists; else the general-shape kernel (fields in gen)
  CorrArgs gen{};
  Tables tb;
  std::vector<int32_t> hjobs;
  int32_t* jobs = nullptr;
  int64_t njobs = 0;
  std::vector<int64_t> pair_jobs;  // jobs of each pair in this class
  bool unc_fused = false, unc_post = false;
};

struct BSlot {
  int64_t gtot = 0, ptot = 0;
  int max_maxit = 0;
  bool any_nalt = false, any_replace = false, any_tol = false, any_keep = false, any_next = false;
  bool any_deform = false, any_pred0 = false;
  std::vector<BClass> classes;
};

struct BPlan {
  int npairs = 0, nslots = 0;
  std::vector<int> sched, npass;
  std::vector<std::vector<Grid>> grids;  // [pair][slot], without masks
  std::vector<BPair> tables;             // [slot * npairs + pair], pointers of the last call
  std::vector<BSlot> slots;
  std::vector<int64_t> ioff;             // input staging offsets (host inputs)
  std::vector<uint8_t> has_mask;
  int64_t gcap = 0, atot = 0, wtot = 0, qtot = 0, wcol = 0, wrow = 0, rtot = 0, itot = 0;
  // device storage
  std::vector<void*> allocs;
  BPair* d_tables = nullptr;
  // Pinned upload staging of the descriptor tables and grid masks, two sets
  // used in turn. A kernel reads a set from host memory when the stream
  // reaches the call's upload, so with asynchronous calls (HH_BATCH_ASYNC)
  // the next call fills the other set, and a set is refilled only after the
  // event recorded behind its last upload has completed.
  BPair* h_tables_set[2] = {nullptr, nullptr};
  uint8_t* h_gmask_set[2] = {nullptr, nullptr};  // nslots * gcap each, when masks
  cudaEvent_t upload_ev[2] = {nullptr, nullptr};
  int upload_set = 0;
  // recorded behind the last asynchronous call's read-back; the plan's
  // storage is released only after it completes
  cudaEvent_t done_ev = nullptr;
  bool async_pending = false;
  int32_t* d_done = nullptr;
  int32_t* d_sweeps = nullptr;
  int32_t* d_slot_sweeps = nullptr;  // nslots x npairs: sweeps run by each pair in each slot
  uint8_t* d_gmask = nullptr;
  float *warpA = nullptr, *warpB = nullptr, *coefA = nullptr, *coefB = nullptr, *dbuf = nullptr;
  float* rec = nullptr;  // peak records of a correlation launch
  float2* gscr = nullptr;  // general-shape correlation scratch (plan-owned: captured graphs keep the pointer)
  double* uqscr = nullptr; // general-form uncertainty scratch
  float *stageA = nullptr, *stageB = nullptr;
  uint16_t *stage16A = nullptr, *stage16B = nullptr;  // host UInt16 frames before conversion
  uint8_t* stageM = nullptr;
  hh::BGrid g{};
  hh::BResult r{};
  std::vector<uint8_t> final_gmask;  // rtot, host
  bool smoothing = true;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  int64_t graph_launches = 0;
  // profiled runs: the launches whose algorithmic work depends on which
  // pairs are live (converged pairs and pairs without the slot are skipped
  // by the kernels); their charge is recomputed from the sweeps each pair
  // ran once the run has finished
  struct Charge {
    size_t pending;  // index into ctx->pending
    int cls, slot, it, jclass, mode;
  };
  std::vector<Charge> charges;
};

static void free_plan(void* vp) {
  BPlan* P = static_cast<BPlan*>(vp);
  if (!P) return;
  // work of an asynchronous call may still read the plan's storage
  if (P->async_pending && P->done_ev) cudaEventSynchronize(P->done_ev);
  for (cudaEvent_t e : P->upload_ev)
    if (e) cudaEventSynchronize(e);
  if (P->exec) cudaGraphExecDestroy(P->exec);
  if (P->graph) cudaGraphDestroy(P->graph);
  for (void* a : P->allocs) cudaFree(a);
  for (auto& S : P->slots)
    for (auto& c : S.classes)
      if (c.jobs) cudaFree(c.jobs);
  for (int i = 0; i < 2; ++i) {
    if (P->h_tables_set[i]) cudaFreeHost(P->h_tables_set[i]);
    if (P->h_gmask_set[i]) cudaFreeHost(P->h_gmask_set[i]);
    if (P->upload_ev[i]) cudaEventDestroy(P->upload_ev[i]);
  }
  if (P->done_ev) cudaEventDestroy(P->done_ev);
  delete P;
}

template <class T> static hh_status plan_alloc(hh_ctx* ctx, BPlan& P, size_t count, T** out) {
  void* p = nullptr;
  cudaError_t e = ctx_malloc(ctx, &p, std::max<size_t>(count, 1) * sizeof(T));
  if (e != cudaSuccess)
    return fail(ctx, HH_ERR_OOM, std::string("device allocation of ") + std::to_string(count * sizeof(T)) +
                                     " bytes for the batched plan failed: " + cudaGetErrorString(e));
  P.allocs.push_back(p);
  *out = static_cast<T*>(p);
  return HH_OK;
}

// Host-side argument checks and the passes of each pair.
static hh_status check_batch(hh_ctx* ctx, const hh_batch_pair* pairs, int npairs, const hh_pass_desc* passes,
                             const int32_t* so, int nsched) {
  if (!pairs || npairs < 1) return fail(ctx, HH_ERR_ARG, "pairs must not be empty");
  if (!passes || !so || nsched < 1) return fail(ctx, HH_ERR_ARG, "at least one pass schedule is required");
  if (so[0] != 0) return fail(ctx, HH_ERR_ARG, "schedule_offsets[0] must be 0");
  for (int s = 0; s < nsched; ++s) {
    if (so[s + 1] <= so[s]) return fail(ctx, HH_ERR_ARG, "at least one pass is required");
    HH_TRY(check_passes(ctx, passes + so[s], so[s + 1] - so[s]));
  }
  for (int p = 0; p < npairs; ++p) {
    const hh_batch_pair& q = pairs[p];
    if (q.schedule < 0 || q.schedule >= nsched)
      return fail(ctx, HH_ERR_ARG, "pair " + std::to_string(p + 1) + ": schedule index out of range");
    if (q.nr < 1 || q.nc < 1) return fail(ctx, HH_ERR_ARG, "images must be non-empty");
    if (!q.A || !q.B) return fail(ctx, HH_ERR_ARG, "pair " + std::to_string(p + 1) + ": image pointer is NULL");
    if (q.format < HH_PIX_F32 || q.format > HH_PIX_U16_RAW)
      return fail(ctx, HH_ERR_ARG, "pair " + std::to_string(p + 1) + ": unknown pixel format " + std::to_string(q.format));
  }
  return HH_OK;
}

// Plan key: everything the launch sequence depends on.
static std::string plan_key(const hh_batch_pair* pairs, int npairs, const hh_pass_desc* passes, const int32_t* so,
                            int nsched, bool smoothing) {
  std::string k;
  auto put = [&k](const void* d, size_t n) { k.append(static_cast<const char*>(d), n); };
  put(&npairs, sizeof npairs);
  put(&nsched, sizeof nsched);
  const int sm = smoothing;
  put(&sm, sizeof sm);
  for (int p = 0; p < npairs; ++p) {
    put(&pairs[p].nr, 8);
    put(&pairs[p].nc, 8);
    put(&pairs[p].schedule, 4);
    const int hm = pairs[p].mask != nullptr;
    put(&hm, 4);
    put(&pairs[p].format, 4);
  }
  for (int i = 0; i < so[nsched]; ++i) {
    hh_pass_desc d = passes[i];
    d.reserved0 = 0;
    for (int q = d.n_validators; q < HH_MAX_VALIDATORS; ++q) memset(&d.validators[q], 0, sizeof(hh_validator));
    put(&d, sizeof d);
  }
  for (int s = 0; s <= nsched; ++s) put(&so[s], 4);
  return k;
}


static hh_status build_plan(hh_ctx* ctx, BPlan& P, const hh_batch_pair* pairs, int npairs, const hh_pass_desc* passes,
                            const int32_t* so, double thr, bool smoothing) {
  P.npairs = npairs;
  P.smoothing = smoothing;
  P.sched.resize(npairs);
  P.npass.resize(npairs);
  P.grids.resize(npairs);
  P.has_mask.resize(npairs);
  P.ioff.resize(npairs + 1);
  std::vector<int64_t> gcap(npairs), acap(npairs);
  std::vector<int> deforms(npairs);
  int nslots = 0;
  bool any_mask = false;
  for (int p = 0; p < npairs; ++p) {
    const hh_batch_pair& q = pairs[p];
    const int s = q.schedule, n = so[s + 1] - so[s];
    const hh_pass_desc* ps = passes + so[s];
    P.sched[p] = s;
    P.npass[p] = n;
    P.has_mask[p] = q.mask != nullptr;
    any_mask |= q.mask != nullptr;
    nslots = std::max(nslots, n);
    P.grids[p].resize(n);
    int64_t gc = 1;
    int nalt = 0;
    bool iter = false;
    for (int k = 0; k < n; ++k) {
      HH_TRY(make_grid(ctx, q.nr, q.nc, ps[k], nullptr, thr, P.grids[p][k]));
      const Grid& g = P.grids[p][k];
      if (g.ny > 65535 || g.nx > 65535) return fail(ctx, HH_ERR_UNSUPPORTED, "batched grids are limited to 65535 x 65535 cells");
      gc = std::max<int64_t>(gc, (int64_t)g.ny * g.nx);
      nalt = std::max(nalt, ps[k].n_peaks - 1);
      iter |= ps[k].max_iterations > 1;
    }
    gcap[p] = gc;
    acap[p] = (int64_t)nalt * gc;
    deforms[p] = n > 1 || iter;
  }
  P.nslots = nslots;
  // storage offsets
  std::vector<int64_t> goff(npairs), aoff(npairs), poff(npairs), qoff(npairs), wcol(npairs), wrow(npairs), roff(npairs);
  int64_t G = 0, A = 0, Wt = 0, Q = 0, WC = 0, WR = 0, R = 0, I = 0;
  for (int p = 0; p < npairs; ++p) {
    const int64_t nr = pairs[p].nr, nc = pairs[p].nc;
    goff[p] = G;
    G += gcap[p];
    aoff[p] = A;
    A += acap[p];
    poff[p] = Wt;
    qoff[p] = Q;
    wcol[p] = WC;
    wrow[p] = WR;
    if (deforms[p]) {
      Wt += (nr * nc + 3) / 4 * 4;  // 16-byte aligned per pair: the deformation stores pixel quads
      Q += (nr + 2) * (nc + 2);
      WC += (nc + 31) / 32 * hh::b_nseg(nr + 2);  // column tiles x segments
      WR += (nr + 2 + 31) / 32 * hh::b_nseg(nc + 2);  // 32-row groups x segments
    }
    roff[p] = R;
    const Grid& gf = P.grids[p].back();
    R += (int64_t)gf.ny * gf.nx;
    P.ioff[p] = I;
    I += nr * nc;
  }
  P.ioff[npairs] = I;
  P.gcap = G;
  P.atot = A;
  P.wtot = Wt;
  P.qtot = Q;
  P.wcol = WC;
  P.wrow = WR;
  P.rtot = R;
  P.itot = I;
  // device storage
  hh::BGrid& g = P.g;
  float** fl[] = {&g.u, &g.v, &g.resu, &g.resv, &g.ratio, &g.moment, &g.meas_u, &g.meas_v, &g.prev_u,
                  &g.prev_v, &g.predw_u, &g.predw_v, &g.pred_u, &g.pred_v, &g.unc_u, &g.unc_v};
  for (float** f : fl) HH_TRY(plan_alloc(ctx, P, G, f));
  HH_TRY(plan_alloc(ctx, P, A, &g.alt_u));
  HH_TRY(plan_alloc(ctx, P, A, &g.alt_v));
  HH_TRY(plan_alloc(ctx, P, G, &g.outl));
  HH_TRY(plan_alloc(ctx, P, G, &g.outl2));
  HH_TRY(plan_alloc(ctx, P, G, &g.keys));
  HH_CK(cudaMemsetAsync(g.pred_u, 0, G * sizeof(float), ctx->stream));
  HH_CK(cudaMemsetAsync(g.pred_v, 0, G * sizeof(float), ctx->stream));
  HH_CK(cudaMemsetAsync(g.predw_u, 0, G * sizeof(float), ctx->stream));
  HH_CK(cudaMemsetAsync(g.predw_v, 0, G * sizeof(float), ctx->stream));
  HH_TRY(plan_alloc(ctx, P, Wt, &P.warpA));
  HH_TRY(plan_alloc(ctx, P, Wt, &P.warpB));
  HH_TRY(plan_alloc(ctx, P, Q, &P.coefA));
  HH_TRY(plan_alloc(ctx, P, Q, &P.coefB));
  HH_TRY(plan_alloc(ctx, P, 2 * Q, &P.dbuf));
  HH_TRY(plan_alloc(ctx, P, (size_t)npairs, &P.d_done));
  HH_TRY(plan_alloc(ctx, P, (size_t)npairs, &P.d_sweeps));
  HH_TRY(plan_alloc(ctx, P, (size_t)npairs * std::max(P.nslots, 1), &P.d_slot_sweeps));
  HH_TRY(plan_alloc(ctx, P, (size_t)nslots * npairs, &P.d_tables));
  hh::BResult& r = P.r;
  float** rf[] = {&r.u, &r.v, &r.ratio, &r.moment, &r.unc_u, &r.unc_v};
  for (float** f : rf) HH_TRY(plan_alloc(ctx, P, R, f));
  HH_TRY(plan_alloc(ctx, P, R, &r.outl));
  for (int i = 0; i < 2; ++i) {
    if (any_mask) HH_CK(cudaMallocHost(&P.h_gmask_set[i], std::max<size_t>((size_t)nslots * G, 1)));
    HH_CK(cudaMallocHost(&P.h_tables_set[i], sizeof(BPair) * std::max<size_t>((size_t)nslots * npairs, 1)));
    HH_CK(cudaEventCreateWithFlags(&P.upload_ev[i], cudaEventDisableTiming));
  }
  HH_CK(cudaEventCreateWithFlags(&P.done_ev, cudaEventDisableTiming));
  if (any_mask) HH_TRY(plan_alloc(ctx, P, (size_t)nslots * G, &P.d_gmask));
  P.final_gmask.assign(R, 0);
  // descriptor tables and job classes, slot by slot
  P.tables.assign((size_t)nslots * npairs, BPair{});
  P.slots.resize(nslots);
  for (int k = 0; k < nslots; ++k) {
    BSlot& S = P.slots[k];
    std::map<std::tuple<int, int, int, int, int, int, int, int, int, int, int, int>, int> cls;
    int64_t coff = 0, pcoff = 0;
    for (int p = 0; p < npairs; ++p) {
      const hh_batch_pair& q = pairs[p];
      const hh_pass_desc* ps = passes + so[P.sched[p]];
      const int n = P.npass[p];
      BPair& b = P.tables[(size_t)k * npairs + p];
      b.nr = q.nr;
      b.nc = q.nc;
      b.poff = poff[p];
      b.qoff = qoff[p];
      b.wcol = wcol[p];
      b.wrow = wrow[p];
      b.goff = goff[p];
      b.aoff = aoff[p];
      b.roff = roff[p];
      b.coff = coff;
      b.pcoff = pcoff;
      b.deforms = deforms[p];
      b.coefA = P.coefA + qoff[p];
      b.coefB = P.coefB + qoff[p];
      b.warpA = P.warpA + poff[p];
      b.warpB = P.warpB + poff[p];
      const Grid& gf = P.grids[p].back();
      b.fgny = gf.ny;
      b.fgnx = gf.nx;
      if (deforms[p]) {
        float *cp, *iv;
        HH_TRY(bs_factors(ctx, q.nr + 2, &cp, &iv));
        b.cpc = cp;
        b.ivc = iv;
        HH_TRY(bs_factors(ctx, q.nc + 2, &cp, &iv));
        b.cpr = cp;
        b.ivr = iv;
      }
      if (k >= n) continue;  // the pair has no pass in this slot
      const hh_pass_desc& pd = ps[k];
      const Grid& gr = P.grids[p][k];
      b.live = 1;
      b.ny = gr.ny;
      b.nx = gr.nx;
      b.gy0 = gr.y[0];
      b.gysp = gr.ny > 1 ? gr.y[1] - gr.y[0] : 1.f;
      b.gx0 = gr.x[0];
      b.gxsp = gr.nx > 1 ? gr.x[1] - gr.x[0] : 1.f;
      if (k > 0) {
        const Grid& pg = P.grids[p][k - 1];
        b.has_pred0 = 1;
        b.pgny = pg.ny;
        b.pgnx = pg.nx;
        b.py0 = pg.y[0];
        b.pysp = pg.ny > 1 ? pg.y[1] - pg.y[0] : 1.f;
        b.px0 = pg.x[0];
        b.pxsp = pg.nx > 1 ? pg.x[1] - pg.x[0] : 1.f;
      }
      b.has_next = k < n - 1;
      b.is_final = k == n - 1;
      b.maxit = pd.max_iterations;
      b.nalt = pd.n_peaks - 1;
      b.W = pd.window[0];
      b.uod_enable = pd.uod_enable;
      b.uod_nb = pd.uod_neighborhood;
      b.uod_thr = pd.uod_threshold;
      b.min_peak_ratio = pd.min_peak_ratio;
      b.nval = pd.n_validators;
      for (int v = 0; v < pd.n_validators; ++v) b.val[v] = pd.validators[v];
      const bool force = k < n - 1;
      b.replace = force || pd.max_iterations > 1 || pd.replace_outliers;
      b.keep_measured = pd.max_iterations > 1 && !(force || pd.replace_outliers);
      const bool unc = pd.uncertainty && !force;
      b.unc_fused = unc && pd.max_iterations == 1;
      b.unc_post = unc && pd.max_iterations > 1;
      b.tol = pd.convergence_tol;
      const int64_t Gk = (int64_t)gr.ny * gr.nx;
      coff += Gk;
      if (deforms[p]) pcoff += (q.nr * q.nc + 3) / 4 * 4;  // quads of pixels never straddle two pairs
      S.max_maxit = std::max(S.max_maxit, (int)pd.max_iterations);
      S.any_nalt |= b.nalt > 0;
      S.any_replace |= b.replace != 0;
      S.any_tol |= pd.convergence_tol > 0 && pd.max_iterations > 2;
      S.any_keep |= b.keep_measured != 0;
      S.any_next |= b.has_next != 0;
      S.any_deform |= deforms[p] != 0;
      S.any_pred0 |= k > 0;
      // job class of this pass
      const auto key = std::make_tuple(fft_rows(pd), fft_cols(pd), (int)pd.window[0], (int)pd.window[1],
                                       (int)pd.search[0], (int)pd.search[1], (int)pd.method, (int)pd.n_peaks,
                                       (int)pd.peak_finder, (int)pd.subpixel, (int)pd.apodization, (int)pd.padding);
      auto it = cls.find(key);
      if (it == cls.end()) {
        it = cls.emplace(key, (int)S.classes.size()).first;
        BClass c;
        c.N = fft_size(pd);
        c.W = pd.window[0];
        c.S = pd.search[0];
        c.method = pd.method;
        c.npeaks = pd.n_peaks;
        c.finder = pd.peak_finder;
        c.subpixel = pd.subpixel;
        c.apod = pd.apodization;
        c.padding = pd.padding;
        c.pd = pd;
        c.special = corr_special(pd);
        if (!c.special) HH_TRY(gcorr_setup(ctx, pd, c.gen));
        HH_TRY(get_tables(ctx, pd, c.tb));
        S.classes.push_back(std::move(c));
      }
      BClass& c = S.classes[it->second];
      c.unc_fused |= b.unc_fused != 0;
      c.unc_post |= b.unc_post != 0;
      c.pair_jobs.resize(npairs, 0);
      c.pair_jobs[p] += (int64_t)gr.jobs.size() / 4;
      for (size_t j = 0; j + 3 < gr.jobs.size(); j += 4) {
        c.hjobs.push_back(p);
        c.hjobs.push_back(gr.jobs[j] | (gr.jobs[j + 1] << 16));
        c.hjobs.push_back(gr.jobs[j + 2]);
        c.hjobs.push_back(gr.jobs[j + 3]);
      }
    }
    S.gtot = coff;
    S.ptot = pcoff;
    for (auto& c : S.classes) {
      c.njobs = (int64_t)c.hjobs.size() / 4;
      void* d = nullptr;
      HH_CK(ctx_malloc(ctx, &d, std::max<size_t>(c.hjobs.size(), 1) * sizeof(int32_t)));
      c.jobs = static_cast<int32_t*>(d);
      HH_CK(cudaMemcpy(c.jobs, c.hjobs.data(), c.hjobs.size() * sizeof(int32_t), cudaMemcpyHostToDevice));
      c.hjobs.clear();
      c.hjobs.shrink_to_fit();
    }
  }
  // peak records of the largest correlation launch (launches of a sweep run
  // one after another on the stream, so they share it)
  size_t recw = 0, gw = 0, uw = 0;
  for (const auto& S : P.slots)
    for (const auto& c : S.classes) {
      recw = std::max(recw, (size_t)c.njobs * hh::correlate_record_words(c.npeaks));
      if (!c.special) gw = std::max(gw, (size_t)(c.gen.gscr_slices * c.gen.gscr_stride));
      if ((c.unc_fused || c.unc_post) && hh::uq_general(c.pd.window[0], c.pd.window[1])) {
        hh::UQArgs ua{};  // the launch's slices, as uq_setup sizes them
        uq_setup(ctx, c.pd.window[0], c.pd.window[1], ua);
        uw = std::max(uw, (size_t)ua.gscr_slices * (size_t)ua.gscr_stride);
      }
    }
  HH_TRY(plan_alloc(ctx, P, recw, &P.rec));
  if (gw) HH_TRY(plan_alloc(ctx, P, gw, &P.gscr));
  if (uw) HH_TRY(plan_alloc(ctx, P, uw, &P.uqscr));
  return HH_OK;
}

// The launch sequence of one batched run on the context stream.
static hh_status issue(hh_ctx* ctx, BPlan& P) {
  cudaStream_t s = ctx->stream;
  const int np = P.npairs;
  const hh::BGrid& g = P.g;
  HH_CK(cudaMemsetAsync(P.d_sweeps, 0, np * sizeof(int32_t), s));
  HH_CK(cudaMemsetAsync(P.d_slot_sweeps, 0, (size_t)np * P.nslots * sizeof(int32_t), s));
  P.charges.clear();
  // remember the profiled launch just issued for the live-work charge
  auto charge = [&](int cls, int slot, int it, int jclass, int mode) {
    if (ctx->prof && !ctx->pending.empty()) P.charges.push_back({ctx->pending.size() - 1, cls, slot, it, jclass, mode});
  };
  if (P.qtot > 0) {
    const double px = (double)P.wtot;
    HH_K(HH_K_PREFILTER, 10, 24 * px, 16 * px, (int64_t)px,
         hh::launch_b_prefilter(P.d_tables, np, P.qtot, P.wcol, P.wrow, P.dbuf, s));
  }
  const float* pu = P.smoothing ? g.pred_u : g.predw_u;
  const float* pv = P.smoothing ? g.pred_v : g.predw_v;
  for (int k = 0; k < P.nslots; ++k) {
    const BSlot& S = P.slots[k];
    const BPair* T = P.d_tables + (size_t)k * np;
    const double Gs = (double)S.gtot, Ps = (double)S.ptot;
    HH_CK(cudaMemsetAsync(P.d_done, 0, np * sizeof(int32_t), s));
    for (int it = 1; it <= S.max_maxit; ++it) {
      HH_K(HH_K_VECTOR, 1, 0, 8 * Gs, S.gtot,
           hh::launch_b_sweep_begin(T, np, P.d_done, it, S.gtot, pu, pv, g.u, g.v, g.unc_u, g.unc_v, P.d_sweeps,
                                    P.d_slot_sweeps + (size_t)k * np, s));
      charge(HH_K_VECTOR, k, it, -1, 0);
      if (S.any_deform && (it > 1 || S.any_pred0)) {
        HH_K(HH_K_DEFORM, 1, 120 * Ps, 16 * Ps, S.ptot, hh::launch_b_deform(T, np, P.d_done, it, S.ptot, pu, pv, s));
        charge(HH_K_DEFORM, k, it, -1, 0);
      }
      for (size_t ci = 0; ci < S.classes.size(); ++ci) {
        const BClass& c = S.classes[ci];
        CorrArgs ca = c.gen;  // general-shape fields (zero for the fused kernels)
        ca.gscr = P.gscr;
        ca.jobs = c.jobs;
        ca.njobs = c.njobs;
        ca.apod = c.tb.apod;
        ca.gain = c.tb.gain;
        ca.phasew = c.tb.phasew;
        ca.box_lo = c.tb.box_lo;
        ca.box_hi = c.tb.box_hi;
        ca.method = c.method;
        ca.npeaks = c.npeaks;
        ca.finder = c.finder;
        ca.subpixel = c.subpixel;
        ca.du = g.resu;
        ca.dv = g.resv;
        ca.ratio = g.ratio;
        ca.moment = g.moment;
        ca.nalt = c.npeaks - 1;
        ca.alt_u = c.npeaks > 1 ? g.alt_u : nullptr;
        ca.alt_v = c.npeaks > 1 ? g.alt_v : nullptr;
        ca.bp = T;
        ca.done = P.d_done;
        ca.it = it;
        ca.rec = P.rec;
        ca.win = c.S != c.W ? c.W : 0;
        {
          auto cv = ctx->corr_var.find({c.N, c.S});
          ca.variant = cv == ctx->corr_var.end() ? 0 : cv->second;
        }
        HH_K(HH_K_CORRELATE, 1, corr_flops(c.pd, c.njobs), corr_bytes(c.pd, c.npeaks - 1, c.njobs), c.njobs,
             corr_launch(ctx, c.pd, ca, s));
        charge(HH_K_CORRELATE, k, it, (int)ci, 0);
      }
      if (it == 1)
        for (size_t ci = 0; ci < S.classes.size(); ++ci) {
          const BClass& c = S.classes[ci];
          if (c.unc_fused) {
            hh::UQArgs ua{};
            ua.jobs = c.jobs;
            ua.njobs = c.njobs;
            ua.W = c.W;
            ua.apod = c.tb.apod;
            ua.unc_u = g.unc_u;
            ua.unc_v = g.unc_v;
            ua.bp = T;
            ua.done = P.d_done;
            ua.mode = 0;
            uq_setup(ctx, c.pd.window[0], c.pd.window[1], ua);
            ua.gscr = P.uqscr;
            HH_K(HH_K_UQ, 1, uq_flops(c.pd, c.njobs), 8.0 * c.pd.window[0] * c.pd.window[1] * c.njobs, c.njobs,
                 hh::launch_uq(ua, s, ctx->num_sms));
            charge(HH_K_UQ, k, 1, (int)ci, 0);
          }
        }
      const bool fc = S.any_tol && it >= 2 && it < S.max_maxit;
      const int nv = 2 + S.any_nalt + S.any_replace + fc;
      HH_K(HH_K_VECTOR, nv, 0, 120 * Gs, S.gtot,
           hh::launch_b_vector(T, np, P.d_done, it, S.gtot, g, S.any_nalt, S.any_replace, S.any_tol, S.max_maxit, s,
                               nullptr));
      charge(HH_K_VECTOR, k, it, -1, 1);
      if (it < S.max_maxit) {
        HH_K(HH_K_VECTOR, P.smoothing ? 2 : 1, 0, 24 * Gs, S.gtot,
             hh::launch_b_predictor(T, np, P.d_done, it, 0, S.gtot, g, P.smoothing, s, nullptr));
        charge(HH_K_VECTOR, k, it, -1, 2);
      }
    }
    for (size_t ci = 0; ci < S.classes.size(); ++ci) {
      const BClass& c = S.classes[ci];
      if (c.unc_post) {
        hh::UQArgs ua{};
        ua.jobs = c.jobs;
        ua.njobs = c.njobs;
        ua.W = c.W;
        ua.apod = c.tb.apod;
        ua.unc_u = g.unc_u;
        ua.unc_v = g.unc_v;
        ua.bp = T;
        ua.done = P.d_done;
        ua.mode = 1;
        uq_setup(ctx, c.pd.window[0], c.pd.window[1], ua);
        ua.gscr = P.uqscr;
        HH_K(HH_K_UQ, 1, uq_flops(c.pd, c.njobs), 8.0 * c.pd.window[0] * c.pd.window[1] * c.njobs, c.njobs,
             hh::launch_uq(ua, s, ctx->num_sms));
        charge(HH_K_UQ, k, 0, (int)ci, 1);
      }
    }
    if (S.any_keep) HH_K(HH_K_VECTOR, 1, 0, 20 * Gs, S.gtot, hh::launch_b_restore(T, np, S.gtot, g, s));
    if (S.any_next)
      HH_K(HH_K_VECTOR, P.smoothing ? 2 : 1, 0, 24 * Gs, S.gtot,
           hh::launch_b_predictor(T, np, P.d_done, S.max_maxit, 1, S.gtot, g, P.smoothing, s, nullptr));
  }
  HH_K(HH_K_VECTOR, 1, 0, 50.0 * P.rtot, P.rtot, hh::launch_b_gather(P.d_tables, np, P.rtot, g, P.r, s));
  return HH_OK;
}

// Algorithmic work of the profiled launches of the last run, counted over
// the pairs each launch actually served: a pair takes part in sweep `it` of
// slot k when it has the slot and ran at least `it` sweeps there (converged
// pairs are skipped by the kernels). Replaces the launch-time charge, which
// counted every pair of the slot.
static hh_status recharge_live(hh_ctx* ctx, BPlan& P) {
  if (P.charges.empty()) return HH_OK;
  const int np = P.npairs;
  std::vector<int32_t> sw((size_t)np * P.nslots);
  HH_CK(cudaMemcpy(sw.data(), P.d_slot_sweeps, sw.size() * sizeof(int32_t), cudaMemcpyDeviceToHost));
  for (const auto& ch : P.charges) {
    if (ch.pending >= ctx->pending.size()) continue;
    auto& q = ctx->pending[ch.pending];
    const BSlot& S = P.slots[ch.slot];
    const int32_t* ran = sw.data() + (size_t)ch.slot * np;
    const BPair* tb = P.tables.data() + (size_t)ch.slot * np;
    auto live = [&](int p, int it) { return tb[p].live && ran[p] >= it; };
    double units = 0;
    if (ch.cls == HH_K_CORRELATE) {
      const BClass& c = S.classes[ch.jclass];
      for (int p = 0; p < np && p < (int)c.pair_jobs.size(); ++p)
        if (live(p, ch.it)) units += (double)c.pair_jobs[p];
      q.flops = corr_flops(c.pd, (int64_t)units);
      q.bytes = corr_bytes(c.pd, c.npeaks - 1, (int64_t)units);
    } else if (ch.cls == HH_K_UQ) {
      const BClass& c = S.classes[ch.jclass];
      for (int p = 0; p < np && p < (int)c.pair_jobs.size(); ++p) {
        const bool on = ch.mode == 0 ? (tb[p].unc_fused && live(p, 1)) : (tb[p].unc_post && tb[p].live);
        if (on) units += (double)c.pair_jobs[p];
      }
      q.flops = uq_flops(c.pd, (int64_t)units);
      q.bytes = 8.0 * c.pd.window[0] * c.pd.window[1] * units;
    } else if (ch.cls == HH_K_DEFORM) {
      for (int p = 0; p < np; ++p)
        if (live(p, ch.it) && tb[p].deforms && (ch.it > 1 || tb[p].has_pred0)) units += (double)(tb[p].nr * tb[p].nc);
      q.flops = 120 * units;
      q.bytes = 16 * units;
    } else {  // vector-grid stages: cells of the live pairs
      for (int p = 0; p < np; ++p)
        if (live(p, ch.it)) units += (double)tb[p].ny * tb[p].nx;
      q.bytes = (ch.mode == 0 ? 8.0 : ch.mode == 1 ? 120.0 : 24.0) * units;
    }
    q.units = (int64_t)units;
  }
  P.charges.clear();
  return HH_OK;
}

static hh_status find_plan(hh_ctx* ctx, const hh_batch_pair* pairs, int npairs, const hh_pass_desc* passes,
                           const int32_t* so, int nsched, double thr, bool smoothing, BPlan** out) {
  const std::string key = plan_key(pairs, npairs, passes, so, nsched, smoothing);
  for (size_t i = 0; i < ctx->bplans.size(); ++i)
    if (ctx->bplans[i].first == key) {
      auto e = ctx->bplans[i];
      ctx->bplans.erase(ctx->bplans.begin() + i);
      ctx->bplans.push_back(e);
      *out = static_cast<BPlan*>(e.second);
      return HH_OK;
    }
  constexpr size_t kMaxPlans = 4;
  ctx->bplan_free = free_plan;
  if (ctx->bplans.size() >= kMaxPlans) {
    HH_CK(cudaStreamSynchronize(ctx->stream));
    free_plan(ctx->bplans.front().second);
    ctx->bplans.erase(ctx->bplans.begin());
  }
  BPlan* P = new BPlan();
  hh_status st = build_plan(ctx, *P, pairs, npairs, passes, so, thr, smoothing);
  if (st != HH_OK) {
    cudaStreamSynchronize(ctx->stream);
    free_plan(P);
    return st;
  }
  ctx->bplans.emplace_back(key, P);
  *out = P;
  return HH_OK;
}

// Per-call inputs: image pointers (or staged host images) and grid masks.
static hh_status stage_inputs(hh_ctx* ctx, BPlan& P, const hh_batch_pair* pairs, const hh_pass_desc* passes,
                              const int32_t* so, double thr, bool device_inputs) {
  cudaStream_t s = ctx->stream;
  const int np = P.npairs;
  const bool any_mask = P.d_gmask != nullptr;
  // this call's staging set: the upload that last read it must have run
  const int set = P.upload_set;
  HH_CK(cudaEventSynchronize(P.upload_ev[set]));
  BPair* h_tables = P.h_tables_set[set];
  uint8_t* h_gmask = P.h_gmask_set[set];
  bool any_u16 = false;
  for (int p = 0; p < np; ++p) any_u16 |= pairs[p].format != HH_PIX_F32;
  if ((!device_inputs || any_u16) && !P.stageA) {
    HH_TRY(plan_alloc(ctx, P, P.itot, &P.stageA));
    HH_TRY(plan_alloc(ctx, P, P.itot, &P.stageB));
  }
  if (!device_inputs && any_mask && !P.stageM) HH_TRY(plan_alloc(ctx, P, P.itot, &P.stageM));
  if (!device_inputs && any_u16 && !P.stage16A) {
    HH_TRY(plan_alloc(ctx, P, P.itot, &P.stage16A));
    HH_TRY(plan_alloc(ctx, P, P.itot, &P.stage16B));
  }
  for (int p = 0; p < np; ++p) {
    const size_t n = (size_t)(pairs[p].nr * pairs[p].nc);
    const int fmt = pairs[p].format;
    if (fmt == HH_PIX_F32) {
      if (!device_inputs) {
        HH_CK(cudaMemcpyAsync(P.stageA + P.ioff[p], pairs[p].A, n * sizeof(float), cudaMemcpyHostToDevice, s));
        HH_CK(cudaMemcpyAsync(P.stageB + P.ioff[p], pairs[p].B, n * sizeof(float), cudaMemcpyHostToDevice, s));
      }
    } else {  // UInt16 frames: (copy and) convert into the float staging
      const uint16_t* a16 = reinterpret_cast<const uint16_t*>(pairs[p].A);
      const uint16_t* b16 = reinterpret_cast<const uint16_t*>(pairs[p].B);
      if (!device_inputs) {
        HH_CK(cudaMemcpyAsync(P.stage16A + P.ioff[p], a16, n * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
        HH_CK(cudaMemcpyAsync(P.stage16B + P.ioff[p], b16, n * sizeof(uint16_t), cudaMemcpyHostToDevice, s));
        a16 = P.stage16A + P.ioff[p];
        b16 = P.stage16B + P.ioff[p];
      }
      const int norm = fmt == HH_PIX_U16;
      HH_K(HH_K_PREFILTER, 2, 0, 12.0 * n, (int64_t)n, hh::launch_u16_to_f32(a16, (int64_t)n, norm, P.stageA + P.ioff[p], s));
      HH_K(HH_K_PREFILTER, 0, 0, 0, 0, hh::launch_u16_to_f32(b16, (int64_t)n, norm, P.stageB + P.ioff[p], s));
    }
    if (!device_inputs && pairs[p].mask)
      HH_CK(cudaMemcpyAsync(P.stageM + P.ioff[p], pairs[p].mask, n, cudaMemcpyHostToDevice, s));
  }
  std::vector<uint8_t> hmask;
  for (int p = 0; p < np; ++p) {
    const hh_batch_pair& q = pairs[p];
    const bool staged = !device_inputs || q.format != HH_PIX_F32;
    const float* A = staged ? P.stageA + P.ioff[p] : q.A;
    const float* B = staged ? P.stageB + P.ioff[p] : q.B;
    const uint8_t* M = q.mask ? (device_inputs ? q.mask : P.stageM + P.ioff[p]) : nullptr;
    const uint8_t* hm = nullptr;
    if (q.mask) {
      if (device_inputs) {
        hmask.resize((size_t)(q.nr * q.nc));
        HH_CK(cudaMemcpyAsync(hmask.data(), q.mask, hmask.size(), cudaMemcpyDeviceToHost, s));
        HH_CK(cudaStreamSynchronize(s));
        hm = hmask.data();
      } else {
        hm = q.mask;
      }
    }
    const hh_pass_desc* ps = passes + so[P.sched[p]];
    for (int k = 0; k < P.nslots; ++k) {
      BPair& b = P.tables[(size_t)k * np + p];
      b.A = A;
      b.B = B;
      b.mask = M;
      b.gmask = nullptr;
      if (k < P.npass[p] && hm) {
        Grid gm;
        HH_TRY(make_grid(ctx, q.nr, q.nc, ps[k], hm, thr, gm));
        if (gm.any_mask) {
          memcpy(h_gmask + (size_t)k * P.gcap + b.goff, gm.gmask.data(), gm.gmask.size());
          b.gmask = P.d_gmask + (size_t)k * P.gcap + b.goff;
        }
        if (k == P.npass[p] - 1) memcpy(P.final_gmask.data() + b.roff, gm.gmask.data(), gm.gmask.size());
      } else if (k == P.npass[p] - 1) {
        const Grid& gf = P.grids[p][k];
        memset(P.final_gmask.data() + b.roff, 0, (size_t)gf.ny * gf.nx);
      }
    }
  }
  // the tables and grid masks are read from their page-locked staging by a
  // kernel: an upload through the copy engine would queue behind frame
  // copies that a caller streams in on another stream meanwhile
  memcpy(h_tables, P.tables.data(), sizeof(BPair) * P.tables.size());
  HH_CK(hh::launch_host_read_copy(P.d_tables, h_tables, sizeof(BPair) * P.tables.size(), s));
  if (any_mask) HH_CK(hh::launch_host_read_copy(P.d_gmask, h_gmask, (size_t)P.nslots * P.gcap, s));
  HH_CK(cudaEventRecord(P.upload_ev[set], s));
  P.upload_set = set ^ 1;
  return HH_OK;
}

}  // namespace hhd

extern "C" {

hh_status hh_batch_grid(const hh_batch_pair* pairs, int32_t npairs, const hh_pass_desc* passes,
                        const int32_t* schedule_offsets, int32_t nschedules, int32_t* ny, int32_t* nx,
                        int64_t* offsets) {
  hh_ctx* ctx = nullptr;
  HH_TRY(check_batch(ctx, pairs, npairs, passes, schedule_offsets, nschedules));
  int64_t off = 0;
  for (int p = 0; p < npairs; ++p) {
    const hh_batch_pair& q = pairs[p];
    Grid g;
    for (int k = schedule_offsets[q.schedule]; k < schedule_offsets[q.schedule + 1]; ++k)
      HH_TRY(make_grid(ctx, q.nr, q.nc, passes[k], nullptr, 0.5, g));
    if (ny) ny[p] = g.ny;
    if (nx) nx[p] = g.nx;
    if (offsets) offsets[p] = off;
    off += (int64_t)g.ny * g.nx;
  }
  if (offsets) offsets[npairs] = off;
  return HH_OK;
}

hh_status hh_run_batched(hh_ctx* ctx, const hh_batch_pair* pairs, int32_t npairs, const hh_pass_desc* passes,
                         const int32_t* schedule_offsets, int32_t nschedules, double thr, int32_t smoothing,
                         int32_t flags, hh_batch_result* out) {
  if (!ctx) return fail(nullptr, HH_ERR_ARG, "context is NULL");
  HH_TRY(set_device(ctx));
  HH_TRY(check_batch(ctx, pairs, npairs, passes, schedule_offsets, nschedules));
  if (!(thr > 0 && thr <= 1)) return fail(ctx, HH_ERR_ARG, "mask_threshold must be in (0, 1], got " + num(thr));
  BPlan* P = nullptr;
  HH_TRY(find_plan(ctx, pairs, npairs, passes, schedule_offsets, nschedules, thr, smoothing != 0, &P));
  HH_TRY(stage_inputs(ctx, *P, pairs, passes, schedule_offsets, thr, (flags & HH_BATCH_DEVICE_INPUTS) != 0));
  cudaStream_t s = ctx->stream;
  const bool use_graph = !(flags & HH_BATCH_NO_GRAPH) && !ctx->prof;
  if (use_graph) {
    if (!P->exec) {
      const int64_t before = ctx->launches;
      HH_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
      const hh_status st = issue(ctx, *P);
      cudaGraph_t graph = nullptr;
      const cudaError_t ec = cudaStreamEndCapture(s, &graph);
      if (st != HH_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
      }
      HH_CK(ec);
      P->graph = graph;
      HH_CK(cudaGraphInstantiate(&P->exec, graph, 0));
      P->graph_launches = ctx->launches - before;
      ctx->launches = before;
    }
    HH_CK(cudaGraphLaunch(P->exec, s));
    ctx->launches += P->graph_launches;
  } else {
    HH_TRY(issue(ctx, *P));
  }
  if (out) {
    const int64_t R = P->rtot;
    const hh::BResult& r = P->r;
    if (out->u) HH_CK(cudaMemcpyAsync(out->u, r.u, R * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out->v) HH_CK(cudaMemcpyAsync(out->v, r.v, R * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out->peak_ratio) HH_CK(cudaMemcpyAsync(out->peak_ratio, r.ratio, R * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out->correlation_moment)
      HH_CK(cudaMemcpyAsync(out->correlation_moment, r.moment, R * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out->uncertainty_u)
      HH_CK(cudaMemcpyAsync(out->uncertainty_u, r.unc_u, R * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out->uncertainty_v)
      HH_CK(cudaMemcpyAsync(out->uncertainty_v, r.unc_v, R * sizeof(float), cudaMemcpyDeviceToHost, s));
    if (out->outliers) HH_CK(cudaMemcpyAsync(out->outliers, r.outl, R, cudaMemcpyDeviceToHost, s));
    if (out->sweeps)
      HH_CK(cudaMemcpyAsync(out->sweeps, P->d_sweeps, npairs * sizeof(int32_t), cudaMemcpyDeviceToHost, s));
    if (out->mask) memcpy(out->mask, P->final_gmask.data(), R);
    for (int p = 0; p < npairs; ++p) {
      const BPair& b = P->tables[p];
      if (out->ny) out->ny[p] = b.fgny;
      if (out->nx) out->nx[p] = b.fgnx;
      if (out->offsets) out->offsets[p] = b.roff;
    }
    if (out->offsets) out->offsets[npairs] = R;
  }
  if ((flags & HH_BATCH_ASYNC) && !ctx->prof) {
    // the caller waits on the context stream before it reads the results
    HH_CK(cudaEventRecord(P->done_ev, s));
    P->async_pending = true;
    return HH_OK;
  }
  HH_CK(cudaStreamSynchronize(s));
  P->async_pending = false;
  if (ctx->prof) HH_TRY(recharge_live(ctx, *P));
  return flush_profile(ctx);
}

}  // extern "C"
