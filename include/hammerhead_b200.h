/*
 * hammerhead_b200.h — C ABI of the B200 (sm_100a) planar-WIDIM library.
 *
 * The library is the device half of a Hammerhead.jl backend: every entry
 * point takes plain pointers and sizes (no Julia, Python or torch types), so
 * the Julia package extension binds it with `ccall` and the Python host layer
 * with ctypes. Images are Julia column-major matrices: element (i, j), 1-based,
 * of an nr x nc image lives at offset (i-1) + (j-1)*nr. Vector grids are
 * column-major (ny, nx) like `PIVResult{Float32}` fields.
 *
 * Each entry point names the reference interface it replaces
 * (stillyslalom/Hammerhead.jl, path:line).
 *
 * Conventions
 *   - Return value: hh_status (HH_OK == 0). On failure, hh_last_error(ctx)
 *     (or hh_last_error(NULL) for context-free calls) gives the message.
 *     Argument errors carry the same text as the reference's ArgumentError.
 *   - Host pointers are borrowed for the duration of the call. Calls are
 *     synchronous unless their name ends in _async (stream-ordered on the
 *     context's stream).
 *   - One context per PIVWorkspace; a context is not thread-safe
 *     (src/pipeline.jl:16-19).
 */
#ifndef HAMMERHEAD_B200_H
#define HAMMERHEAD_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int32_t hh_status;
enum {
  HH_OK = 0,
  HH_ERR_ARG = 1,          /* invalid argument (ArgumentError / DimensionMismatch) */
  HH_ERR_OOM = 2,          /* device allocation failed */
  HH_ERR_CUDA = 3,         /* CUDA runtime error */
  HH_ERR_TIMEOUT = 4,      /* a bounded device wait gave up */
  HH_ERR_UNSUPPORTED = 5,  /* option outside the device scope (_ka_scope_check) */
  HH_ERR_STATE = 6         /* call out of order (e.g. no staged pair) */
};

/* Correlation method, apodization, subpixel, peak finder: the Symbol
 * arguments of PIVParameters (src/types.jl:212-291). */
enum { HH_CROSS = 0, HH_PHASE = 1 };
enum { HH_APOD_NONE = 0, HH_APOD_GAUSS = 1 };
enum { HH_GAUSS3 = 0, HH_GAUSS9 = 1, HH_GAUSS2D = 2, HH_SUBPIXEL_NONE = 3 };
enum { HH_REGIONALMAX = 0, HH_EXCLUSION = 1 };
/* Extra validators (src/quality.jl:360-503, parse_validator). */
enum { HH_VAL_PEAK_RATIO = 0, HH_VAL_MOMENT = 1, HH_VAL_VELOCITY = 2, HH_VAL_UOD = 3 };

#define HH_MAX_VALIDATORS 8

typedef struct hh_validator {
  int32_t kind;          /* HH_VAL_* */
  int32_t neighborhood;  /* UOD neighbourhood layers */
  double threshold;      /* peak-ratio / moment / UOD threshold */
  double vmin, vmax;     /* velocity magnitude bounds */
  double epsilon;        /* UOD epsilon */
} hh_validator;

/* Mirror of PIVParameters (src/types.jl:212-291), one per pass. */
typedef struct hh_pass_desc {
  int32_t window[2];     /* (rows, cols) */
  int32_t search[2];     /* search_area_size (rows, cols) */
  int32_t overlap[2];
  int32_t method;        /* HH_CROSS / HH_PHASE */
  int32_t padding;       /* bool */
  int32_t apodization;   /* HH_APOD_* */
  int32_t subpixel;      /* HH_GAUSS3 / ... */
  int32_t n_peaks;
  int32_t peak_finder;   /* HH_REGIONALMAX / HH_EXCLUSION */
  int32_t uncertainty;   /* bool */
  int32_t uod_enable;    /* bool */
  double uod_threshold;
  int32_t uod_neighborhood;
  int32_t replace_outliers; /* bool */
  double min_peak_ratio;
  int32_t max_iterations;
  int32_t keep_correlation_planes; /* bool (rejected by the device scope check) */
  double convergence_tol;
  int32_t n_validators;
  int32_t reserved0;
  hh_validator validators[HH_MAX_VALIDATORS];
} hh_pass_desc;

/* Caller-owned host buffers for the final pass of run_piv: the fields of
 * PIVResult{Float32} (src/types.jl:359-373). Grid dims come from
 * hh_pass_grid on the final pass. Any pointer may be NULL (not returned). */
typedef struct hh_result {
  int32_t ny, nx;        /* filled by the library */
  float *x, *y;          /* nx, ny */
  float *u, *v, *peak_ratio, *correlation_moment, *uncertainty_u, *uncertainty_v; /* ny*nx */
  uint8_t *outliers, *mask;                                                        /* ny*nx */
} hh_result;

typedef struct hh_ctx hh_ctx;

/* Library identification. */
const char* hh_version(void);
/* Message of the last failure on ctx (ctx == NULL: last context-free failure). */
const char* hh_last_error(const hh_ctx* ctx);

/* Validate one pass descriptor with the checks and messages of the
 * PIVParameters constructor (src/types.jl:254-285). Host-only. */
hh_status hh_pass_validate(const hh_pass_desc* p);

/* Reject options the device path does not implement, before any work:
 * replaces _check_backend_params / _ka_scope_check (src/ka_backend.jl:13-29).
 * Wider than the reference's device backends: enlarged search areas,
 * rectangular windows and search areas, and every FFT plane whose lengths
 * factor into primes up to 61 (at most 4194304 points) are accepted;
 * rejected are subpixel_method :gauss2d, keep_correlation_planes,
 * n_peaks > 8 and UOD neighbourhoods above 4. */
hh_status hh_check_backend_params(const hh_pass_desc* passes, int32_t npasses);

/* Interrogation grid of one pass: replaces pass_grid (src/pipeline.jl:529-555).
 * x (nx), y (ny): window centres; grid_mask (ny*nx) and jobs (4*njobs int32:
 * gi, gj 1-based grid index, rs, cs 1-based window origin) may be NULL.
 * Returns the number of jobs in *njobs. Host-only. */
hh_status hh_pass_grid(int64_t nr, int64_t nc, const hh_pass_desc* p, const uint8_t* mask,
                       double mask_threshold, int32_t* ny, int32_t* nx, float* x, float* y,
                       uint8_t* grid_mask, int32_t* jobs, int64_t* njobs);

/* Context: one device, one stream, a growable device arena.
 * Replaces piv_workspace(; backend = :b200) (src/pipeline.jl:33-44). */
hh_status hh_ctx_create(int32_t device, hh_ctx** out);
void hh_ctx_destroy(hh_ctx* ctx);
/* The context's cudaStream_t (as void*), for callers that time or order work. */
void* hh_ctx_stream(hh_ctx* ctx);

/* Whole planar-WIDIM schedule for one pair, all passes and sweeps on the
 * device: replaces run_piv(imgA, imgB, passes; backend) with its pass loop
 * piv_pass (src/pipeline.jl:361-449, 655-832). A, B host images (nr x nc,
 * column-major float32), mask optional (uint8, nonzero = excluded). */
hh_status hh_run_piv(hh_ctx* ctx, const float* A, const float* B, int64_t nr, int64_t nc,
                     const hh_pass_desc* passes, int32_t npasses, const uint8_t* mask,
                     double mask_threshold, int32_t predictor_smoothing, hh_result* out);

/* Same, with A, B (and mask) already in device memory of the context's
 * device; the result is still returned into the host buffers of *out. */
hh_status hh_run_piv_device(hh_ctx* ctx, const float* dA, const float* dB, int64_t nr, int64_t nc,
                            const hh_pass_desc* passes, int32_t npasses, const uint8_t* dmask,
                            double mask_threshold, int32_t predictor_smoothing, hh_result* out);

/* ---- Batched schedule: many pairs of uneven size and schedule at once ------
 *
 * The reference analyses a stream of pairs with run_piv_sequence
 * (src/io.jl:229-247, _run_sequence :307-361): one run_piv per pair, in
 * order, with results identical to separate calls. hh_run_batched runs every pair's whole
 * schedule together: pass slot k (the k-th pass of every pair that has one)
 * is one launch per kernel for all pairs, each sweep's convergence test is
 * decided on the device (no host round trip), and the launch sequence of a
 * given batch shape is captured once in a CUDA graph and replayed. Results
 * equal hh_run_piv on each pair.
 *
 * Pair p uses passes[schedule_offsets[s] .. schedule_offsets[s+1]) with
 * s = pairs[p].schedule. Images are column-major float32 (host memory, or
 * device memory of the context's device with HH_BATCH_DEVICE_INPUTS; then
 * they must stay valid until the call returns). */
typedef struct hh_batch_pair {
  const float* A;       /* frame data; with format != HH_PIX_F32 a const uint16_t* cast to float* */
  const float* B;
  const uint8_t* mask;  /* nonzero = excluded, or NULL */
  int64_t nr, nc;
  int32_t schedule;
  int32_t format;       /* HH_PIX_*: pixel type of A and B */
} hh_batch_pair;

/* Pixel formats of a batch pair. Camera frames (12- or 16-bit counts stored
 * as UInt16) cross PCIe at half the bytes and are converted on the device:
 * HH_PIX_U16 gives value / 65535 (the Float32 of a Gray{N0f16} pixel, as
 * load_image returns it, src/io.jl:20-25), HH_PIX_U16_RAW the count itself
 * (value * 1). Both are correctly rounded IEEE operations. */
#define HH_PIX_F32 0
#define HH_PIX_U16 1
#define HH_PIX_U16_RAW 2

/* Final-pass results in compact host arrays: pair p's ny[p] x nx[p] grid
 * (column-major) occupies [offsets[p], offsets[p+1]). Any pointer may be
 * NULL. Page-locked buffers make the read-back one asynchronous copy each. */
typedef struct hh_batch_result {
  int32_t *ny, *nx;       /* npairs */
  int64_t* offsets;       /* npairs + 1 */
  float *u, *v, *peak_ratio, *correlation_moment, *uncertainty_u, *uncertainty_v;
  uint8_t *outliers, *mask;
  int32_t* sweeps;        /* npairs: sweeps run in each pair's final pass */
} hh_batch_result;

#define HH_BATCH_DEVICE_INPUTS 1 /* A, B, mask are device pointers */
#define HH_BATCH_NO_GRAPH 2      /* launch directly instead of replaying a captured graph */
/* Return once the run and its read-back are queued on the context stream
 * (hh_ctx_stream) instead of after they finish: the result arrays in *out
 * (page-locked host memory, or the copies are not asynchronous) and device
 * inputs must stay untouched until the caller has waited on that stream, for
 * example through an event recorded on it after the call. Calls on one
 * context run in call order; a call may fill its host staging while an
 * earlier call is still queued. Ignored while profiling. */
#define HH_BATCH_ASYNC 4

/* Final grid sizes and result offsets of a batch (host-only). */
hh_status hh_batch_grid(const hh_batch_pair* pairs, int32_t npairs, const hh_pass_desc* passes,
                        const int32_t* schedule_offsets, int32_t nschedules, int32_t* ny, int32_t* nx,
                        int64_t* offsets);
hh_status hh_run_batched(hh_ctx* ctx, const hh_batch_pair* pairs, int32_t npairs, const hh_pass_desc* passes,
                         const int32_t* schedule_offsets, int32_t nschedules, double mask_threshold,
                         int32_t predictor_smoothing, int32_t flags, hh_batch_result* out);

/* ---- Ensemble (sum-of-correlation) PIV -----------------------------------
 * Replaces run_piv_ensemble (src/ensemble.jl:51-205): per pass, every pair
 * is deformed by the shared predictor, each window's correlation planes are
 * summed over the pairs on the device (in pair order) and analysed once; the
 * uncertainty statistics pool by summation; one sweep per pass. Pairs share
 * one image size; pairs[q].schedule is ignored. mask is a HOST image mask
 * (or NULL) shared by every pair. Images are host pointers, or device
 * pointers with HH_BATCH_DEVICE_INPUTS. The final pass is returned in *out
 * (grid dims from hh_pass_grid of the final pass). */
hh_status hh_run_ensemble(hh_ctx* ctx, const hh_batch_pair* pairs, int32_t npairs, const hh_pass_desc* passes,
                          int32_t npasses, const uint8_t* mask, double mask_threshold,
                          int32_t predictor_smoothing, int32_t flags, hh_result* out);

/* ---- Autotuning of the correlation kernel --------------------------------
 * The correlation kernel of each (FFT size, window) comes in
 * HH_CORR_VARIANTS variants: two CTA shapes (windows per CTA, threads per
 * window) and, for the default shape, register budgets of one CTA per SM
 * more and one less (variants 0-3, identical results), and the default
 * shape with another split of each axis's DFT into an in-register radix and
 * a second pass (variant 4, results differ by rounding). hh_autotune_correlation
 * times every shape on the windows of `pass` over the staged pair
 * (hh_stage_pair first), `reps` launches each, interleaved, writes the mean
 * ms per launch of each shape into variant_ms (HH_CORR_VARIANTS entries)
 * and makes the fastest the context's choice for that (FFT size, window),
 * returned in *best. hh_set_corr_variant sets a choice directly (for
 * example from a cache of earlier tuning). Both drop the context's batched
 * plans, whose graphs hold the old choice. Enlarged search areas have one
 * shape. No counterpart in the reference. */
#define HH_CORR_VARIANTS 5
hh_status hh_autotune_correlation(hh_ctx* ctx, const hh_pass_desc* pass, int32_t reps, float* variant_ms,
                                  int32_t* best);
hh_status hh_set_corr_variant(hh_ctx* ctx, int32_t fft_size, int32_t window, int32_t variant);
/* 1 when a fused shared-memory correlation kernel (the shapes the
 * autotuner chooses between) serves the pass: square windows and search
 * areas of FFT size 16, 24, 32, 48, 64, 96 or 128; 0 when the general-shape
 * kernel does (any other window or search-area shape, rectangular ones and
 * planes that exceed a CTA's shared memory, such as the 256 x 256 planes of
 * padded 128-px windows). Host-only; no counterpart in the reference. */
int32_t hh_corr_fused(const hh_pass_desc* p);

/* Cross-process reduction of the ensemble sums (multi-GPU ensemble: each
 * process holds a share of the pairs). The reference sums every plane on one
 * host (accum[j] .+= plane, src/ensemble.jl:170-171; the uncertainty sums,
 * :182-183); with the pairs split over processes each hh_run_ensemble call
 * sums its own pairs and the reducer turns the partial sums into the sums
 * over all processes before the planes are analysed. It is called once per
 * pass that has windows, after the last local pair, with
 *   planes : nplanes device floats (njobs x N x N, window-major),
 *   stats  : nstats device doubles (njobs x 88), or NULL / 0 when the pass
 *            carries no uncertainty,
 *   stream : the context stream (cudaStream_t) the sums were produced on,
 * and must leave in both arrays their element-wise sum over the processes,
 * ordered on that stream (an in-place all-reduce, e.g. NCCL). Every process
 * makes the same calls in the same order: the grids depend only on the image
 * size, mask and passes, which must agree. A nonzero return fails the call
 * with HH_ERR_STATE. fn == NULL removes the reducer. No counterpart in the
 * reference (single-process only). */
typedef int32_t (*hh_ensemble_reducer)(void* user, int32_t pass, float* planes, int64_t nplanes, double* stats,
                                       int64_t nstats, void* stream);
hh_status hh_set_ensemble_reducer(hh_ctx* ctx, hh_ensemble_reducer fn, void* user);

/* ---- Differentiation: adjoint of deformation + correlation -------------
 *
 * No counterpart in the reference: a correlation loss of the predictor
 * field, for gradient-based refinement of the field, built on the same
 * symmetric deformation as a WIDIM sweep (deform_columns!,
 * src/pipeline.jl:957-965; bilinear predictor with flat extrapolation,
 * src/pipeline.jl:561-569):
 *   L(P) = - sum over windows j of NCC0_j,
 *   NCC0_j = sum (a - abar)(b - bbar) / sqrt(sum (a - abar)^2 sum (b - bbar)^2)
 * over W x W windows at origins (jr*(W - overlap), jc*(W - overlap)) (the
 * pass_grid rows and columns of a pass with that window and overlap) of the
 * staged pair (hh_stage_pair) deformed by P. P holds u (gny x gnx,
 * column-major) followed by v on nodes y0 + i*ysp, x0 + j*xsp. Returns L in
 * *loss and, when dLdP != NULL, dL/dP in the layout of P. The deformed
 * windows are recomputed, not stored. With device_ptrs, P and dLdP are
 * device pointers and the call is stream-ordered on the context stream up
 * to the final loss read. */
hh_status hh_ncc_loss_grad(hh_ctx* ctx, const float* P, int32_t gny, int32_t gnx, float y0, float ysp, float x0,
                           float xsp, int32_t window, int32_t overlap, int32_t device_ptrs, double* loss,
                           float* dLdP);

/* Per-pass timing of the last hh_run_piv* call on ctx, measured with CUDA
 * events on the context stream: ms[k] = device time of pass k (all sweeps,
 * deformation, validation, uncertainty); sweeps[k] = sweeps run. */
hh_status hh_last_pass_times(const hh_ctx* ctx, int32_t npasses, float* ms, int32_t* sweeps);

/* ---- Backend-hook level entry points (the plugin seam of
 *      docs/src/reference/backends.md:40-71) ---------------------------- */

/* _deform_context: stage a pair (host, column-major) and build its cubic
 * B-spline coefficients on the device (src/ka_backend.jl:335-351 +
 * Interpolations prefilter, src/pipeline.jl:75-85). */
hh_status hh_stage_pair(hh_ctx* ctx, const float* A, const float* B, int64_t nr, int64_t nc);

/* apply_predictor: deform the staged pair by a coarse predictor field
 * (gny x gnx, column-major, uniform knots y0 + k*ysp, x0 + k*xsp) on the
 * device; optionally return the warped images (host, nr x nc) and the
 * predictor at the nodes (ny x nx) of a target grid (y: ny, x: nx).
 * Replaces apply_predictor / _ka_apply_predictor_ctx (src/pipeline.jl:575-600,
 * src/ka_backend.jl:357-378). pu == NULL means no predictor (pass-through). */
hh_status hh_apply_predictor(hh_ctx* ctx, const float* pu, const float* pv, int32_t gny, int32_t gnx,
                             float y0, float ysp, float x0, float xsp, const float* y, int32_t ny,
                             const float* x, int32_t nx, float* node_u, float* node_v, float* warpA,
                             float* warpB);

/* The image mask (nr x nc of the staged pair, column-major uint8, nonzero =
 * excluded) of the next hh_process_windows / hh_correlation_planes calls:
 * masked pixels leave the window means and enter as zero (load_windows!,
 * src/correlators.jl:188-263; the mask argument of process_windows!,
 * ext/HammerheadCUDAExt.jl:303-308). NULL clears it; hh_stage_pair clears
 * it too. */
hh_status hh_stage_mask(hh_ctx* ctx, const uint8_t* mask);

/* process_windows!: correlate the jobs of one pass on the current (warped
 * or raw) staged pair and return the packed per-window scalars, layout of
 * src/ka_backend.jl:497-506: out[(5 + 2*(K-1)) * njobs], K = max(n_peaks, 2),
 * column j = [du, dv, peak_ratio, moment, found, alt du (K-1), alt dv (K-1)].
 * jobs: 4*njobs int32 (gi, gj, rs, cs; 1-based). locs (2*K*njobs int32,
 * 1-based (row, col) plane peaks) and uq (2*44*njobs float64 Wieneke
 * statistics, src/uncertainty.jl:40-151) may be NULL. Replaces
 * process_windows! (ext/HammerheadCUDAExt.jl:303-398). */
hh_status hh_process_windows(hh_ctx* ctx, const hh_pass_desc* p, const int32_t* jobs, int64_t njobs,
                             float* out, int32_t* locs, double* uq);

/* Device plane analysis on caller-supplied correlation planes (nplanes
 * column-major nr x nc float32 planes): peak search, subpixel fit, ratio,
 * moment and alternatives, the same device code process_windows runs.
 * Output layout as hh_process_windows. Replaces _ka_analyze!
 * (src/ka_backend.jl:521-687); used for the crafted-plane golden vectors
 * of test/test_ka.jl:28-71. */
hh_status hh_analyze_planes(hh_ctx* ctx, const float* planes, int64_t nplanes, int32_t nr, int32_t nc,
                            int32_t n_peaks, int32_t peak_finder, int32_t subpixel, float* out,
                            int32_t* locs);

/* Correlation planes (fftshifted, gain-normalised, the plane
 * correlation_plane! returns, src/correlators.jl:326-341) of the jobs on the
 * staged pair: planes[fft_rows * fft_cols * njobs]. */
hh_status hh_correlation_planes(hh_ctx* ctx, const hh_pass_desc* p, const int32_t* jobs, int64_t njobs,
                                float* planes);

/* validate_and_replace! on a host vector grid, run on the device
 * (src/pipeline.jl:617-645): UOD, peak ratio, extra validators, mask,
 * peak substitution (alt_u/alt_v: (ny, nx, nalt) or NULL), replacement.
 * u, v, outliers are updated in place. */
hh_status hh_validate(hh_ctx* ctx, const hh_pass_desc* p, int32_t ny, int32_t nx, float* u, float* v,
                      const float* peak_ratio, const float* moment, uint8_t* outliers, const uint8_t* mask,
                      const float* alt_u, const float* alt_v, int32_t nalt, int32_t force_replace);

/* universal_outlier_detection (src/quality.jl:244-293) on the device. */
hh_status hh_uod(hh_ctx* ctx, const float* u, const float* v, int32_t ny, int32_t nx, double threshold,
                 int32_t neighborhood, double epsilon, const uint8_t* exclude, uint8_t* flags);

/* replace_vectors! (src/quality.jl:85-114) and smooth_field (:123-136). */
hh_status hh_replace_vectors(hh_ctx* ctx, float* u, float* v, int32_t ny, int32_t nx, const uint8_t* invalid);
hh_status hh_smooth_field(hh_ctx* ctx, const float* f, int32_t ny, int32_t nx, float* out);

/* field_change (src/pipeline.jl:849-866): 95th-percentile change. */
hh_status hh_field_change(hh_ctx* ctx, const float* u, const float* v, const float* pu, const float* pv,
                          const uint8_t* mask, int64_t n, float* change);

/* finalize_uncertainty (src/uncertainty.jl:162-179) of n windows' Wieneke
 * statistics (2*44 float64 each) into sigma_u, sigma_v. Host-only. */
hh_status hh_finalize_uncertainty(const double* stats, int64_t n, float* sigma_u, float* sigma_v);

/* ---- Measurement (no counterpart in the reference) --------------------- */

/* Per-kernel-class device time. When profiling is on, every launch of the
 * correlation, deformation, prefilter, uncertainty and vector-grid kernels
 * on ctx is bracketed by CUDA events on the context stream, and the
 * algorithmic work of the launch (FLOPs, bytes) is accumulated with it. */
enum { HH_K_CORRELATE = 0, HH_K_DEFORM = 1, HH_K_PREFILTER = 2, HH_K_UQ = 3, HH_K_VECTOR = 4, HH_K_CLASSES = 5 };
typedef struct hh_kernel_profile {
  int64_t launches;
  double ms;       /* summed device time */
  double flops;    /* algorithmic floating-point operations */
  double bytes;    /* algorithmic DRAM bytes */
  int64_t units;   /* windows (correlate, uq), pixels (deform, prefilter), vectors */
} hh_kernel_profile;
hh_status hh_set_profiling(hh_ctx* ctx, int32_t enable);
hh_status hh_profile_read(hh_ctx* ctx, hh_kernel_profile* out /* HH_K_CLASSES entries */, int32_t reset);
/* Kernels launched on ctx since creation (all classes, profiling or not). */
int64_t hh_launch_count(const hh_ctx* ctx);

/* Failure injection for tests of the out-of-memory path (no counterpart in
 * the reference; host side only, no device fault): the device allocation
 * attempt `after` calls from now (0 = the next one) through the context's
 * arena or a batched plan fails with HH_ERR_OOM exactly as a failing
 * cudaMalloc would, without calling it; later allocations proceed. A
 * negative value switches the injection off. The failing call leaves the
 * context usable: its partly built plan or buffer is released and the next
 * call allocates again. */
hh_status hh_debug_fail_alloc(hh_ctx* ctx, int64_t after);

/* ---- Allocation-free convergence norm (no counterpart in the reference) --
 *
 * For callers that must not have the library allocate device memory: a host
 * runtime whose GPU memory belongs to its own pool allocator, a loop that
 * cannot absorb an allocation stall, or a process held to a fixed memory
 * budget. Computes what hh_field_change computes (the 95th-percentile
 * vector change of src/pipeline.jl:849-866) on caller-owned device buffers
 * d_u, d_v, d_pu, d_pv (n float32 each) and optional d_mask (n uint8,
 * nonzero = masked), writing the result to the device float *d_change,
 * asynchronously on `stream` (a cudaStream_t; NULL = the legacy default
 * stream). It allocates nothing: its scratch is a fixed array of
 * HH_NOALLOC_MAX_VECTORS 32-bit keys compiled into the library, which every
 * GPU that loads the library holds until the process exits (4 MiB).
 *   - n > HH_NOALLOC_MAX_VECTORS is rejected with HH_ERR_ARG.
 *   - The first call on a device looks up the scratch address for that
 *     device (the device current at the call) and keeps it for the life of
 *     the process; make that first call before any stream capture. Calls
 *     after cudaDeviceReset (or any other teardown of the device's primary
 *     context) are not supported: the kept address belongs to the old
 *     context.
 *   - All calls on a device share the scratch; each call rewrites the
 *     entries it reads, so nothing carries over, but calls whose kernels
 *     overlap on the GPU (different streams, no ordering) race on it.
 * Errors are reported through hh_noalloc_last_error(), which is empty after
 * a call that succeeded. */
#define HH_NOALLOC_MAX_VECTORS (1 << 20)
hh_status hh_field_change_noalloc(const float* d_u, const float* d_v, const float* d_pu, const float* d_pv,
                                  const uint8_t* d_mask, int64_t n, float* d_change, void* stream);
const char* hh_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif
#endif /* HAMMERHEAD_B200_H */
