// Internal declarations shared by the C-ABI layer and the kernel files.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace hh {

struct BPair;

constexpr int KMAX = 8;  // peaks tracked per window on the device (n_peaks <= 8)

// B-spline prefilter: each line's two Thomas sweeps are cut into independent
// segments of BS_SEG unknowns whose sweeps start BS_WARM unknowns early from a
// zero state (k_deform.cu). Segments of a padded line of n elements (n - 4
// unknowns); the batched plan counts its work items with it.
constexpr int BS_SEG = 64, BS_WARM = 32;
__host__ __device__ __forceinline__ int64_t b_nseg(int64_t n) { return n >= 5 ? (n - 4 + BS_SEG - 1) / BS_SEG : 1; }

// Arguments of the fused correlation kernel (one pass, one image pair).
struct CorrArgs {
  const float* A;            // deformed (or raw) frame A, column-major nr x nc
  const float* B;            // frame B
  const uint8_t* mask;       // image mask (nonzero = excluded) or nullptr
  int64_t ld;                // leading dimension (= nr)
  const int32_t* jobs;       // 4 int32 per job: gi, gj, rs, cs (0-based)
  int64_t njobs;
  int32_t ny;                // grid rows; grid index id = gi + gj * ny
  int64_t G;                 // grid size ny * nx
  const float* apod;         // W x W apodization window (column-major)
  const float* gain;         // N x N overlap gain (fftshifted layout) or nullptr
  const float* phasew;       // N x N phase filter (natural FFT order) or nullptr
  int32_t method, npeaks, finder, subpixel;
  // grid-indexed outputs (residual displacement of this sweep)
  float* du;
  float* dv;
  float* ratio;
  float* moment;
  float* alt_u;              // G x nalt or nullptr
  float* alt_v;
  int32_t nalt;
  // optional per-job outputs
  float* packed;             // (5 + 2(K-1)) x njobs
  int32_t* locs;             // 2K x njobs (1-based row, col)
  float* planes;             // N*N x njobs correlation planes
  // batched mode (bp != nullptr): jobs are (pair, gi | gj << 16, rs, cs);
  // images, grid offsets and sizes come from bp[pair]; windows of pairs not
  // live in sweep `it` are skipped
  const BPair* bp;
  const int32_t* done;
  int32_t it;
  // ensemble mode: planes += R (planes != nullptr) and no peak analysis
  int32_t accumulate;
  // fftshifted rows/columns [box_lo, box_hi] outside which the overlap gain
  // is zero (box_hi == 0: the whole plane); with an enlarged search area the
  // lags kept by restrict_search_lags! (src/correlators.jl:347-355)
  int32_t box_lo, box_hi;
  // enlarged search area: the launch's W is the frame-B search area and win
  // the frame-A window centred in it (jobs give the window's origin); 0 when
  // the two are equal
  int32_t win;
  // CTA shape of the launch (0: default, 1: the alternative; equal areas only)
  int32_t variant;
  // peak records (correlate_record_words(npeaks) x njobs floats) or nullptr:
  // with regional maxima the per-window outputs are then formed by a
  // one-thread-per-window epilogue kernel after the correlation kernel
  float* rec;
  // general-shape path (correlate_general_kernel): window wr x wc, search
  // area sr x sc, FFT plane nfr x nfc; gscr holds one scratch slice of
  // gscr_stride float2 per CTA (complex plane + real plane); twr / twc the
  // twiddle tables exp(-2 pi i t / n) of the two lengths and their radix
  // plans; the line buffers' layout and shared bytes
  int32_t wr, wc, sr, sc, nfr, nfc;
  float2* gscr;
  int64_t gscr_stride;
  int32_t gscr_slices;
  const float2* twr;
  const float2* twc;
  int8_t gc_radix_r[24], gc_radix_c[24];
  int32_t gc_nst_r, gc_nst_c;
  int32_t gc_col_warps, gc_chunk_c;  // warps of the columns passes (one line each); rows-pass lines per chunk
  int64_t gc_smem_lines;
  // fftshifted rows [0], [1] and columns [2], [3] outside which the plane is
  // zero (overlap-gain support or kept search lags; the whole plane otherwise)
  int32_t gc_box[4];
};

// Launch the correlation kernel for FFT size N (square) and window W (the
// search area when a.win is set).
cudaError_t launch_correlate(const CorrArgs& a, int N, int W, cudaStream_t s, int num_sms);
bool correlate_supported(int N, int W);
// The general-shape correlation (any FFT lengths, rectangular windows and
// search areas): a.wr .. a.gc_smem_lines set by the host (gcorr_prepare).
cudaError_t launch_correlate_general(const CorrArgs& a, cudaStream_t s);
// Radix plan of an FFT length (factors 4, 2, then odd primes <= 61);
// returns the stage count, or -1 when a factor exceeds 61 or there are more
// than 24 stages.
int gcorr_radix_plan(int n, int8_t* radix);
// Shared bytes the general kernel needs beyond its line buffers.
size_t gcorr_smem_extra();
size_t correlate_record_words(int npeaks);  // per job
size_t correlate_smem_bytes(int N, int W);

// Device peak analysis of caller-supplied planes.
struct AnalyzeArgs {
  const float* planes;
  int64_t nplanes;
  int32_t nr, nc;
  int32_t npeaks, finder, subpixel;
  float* packed;
  int32_t* locs;
  // optional grid outputs (as CorrArgs): plane j is job j of `jobs`
  const int32_t* jobs;
  int32_t ny;
  int64_t G;
  float *du, *dv, *ratio, *moment, *alt_u, *alt_v;
  int32_t nalt;
};
cudaError_t launch_analyze_planes(const AnalyzeArgs& a, cudaStream_t s);

// --- deformation -----------------------------------------------------------
cudaError_t launch_bspline_factors(int64_t n, float* cp, float* inv, cudaStream_t s);
// Cubic B-spline coefficients ((nr + 2) x (nc + 2), padded) of both frames of
// a pair; dbuf: 2 (nr + 2) (nc + 2) floats for the forward sweeps.
cudaError_t launch_prefilter_pair(const float* imgA, const float* imgB, int64_t nr, int64_t nc, float* coefA,
                                  float* coefB, float* dbuf, const float* cpc, const float* ivc, const float* cpr,
                                  const float* ivr, cudaStream_t s);
struct PredGrid {
  int32_t gny, gnx;
  float y0, ysp, x0, xsp;
};
cudaError_t launch_deform(const float* CA, const float* CB, int64_t nr, int64_t nc, const float* pu,
                          const float* pv, PredGrid g, float* wA, float* wB, cudaStream_t s);
cudaError_t launch_node_values(const float* pu, const float* pv, PredGrid g, const float* y, int32_t ny,
                               const float* x, int32_t nx, float* u, float* v, cudaStream_t s);

// --- vector-grid kernels -----------------------------------------------------
cudaError_t launch_combine(float* u, float* v, const float* resu, const float* resv, float* ratio, float* moment,
                           float* alt_u, float* alt_v, int32_t nalt, const uint8_t* gmask, int64_t G,
                           float* meas_u, float* meas_v, cudaStream_t s);
cudaError_t launch_uod(const float* u, const float* v, int32_t ny, int32_t nx, double thr, int32_t nb, double eps,
                       const uint8_t* exclude, uint8_t* flags, int32_t or_into, cudaStream_t s);
cudaError_t launch_flag_ratio(const float* ratio, int64_t G, double thr, uint8_t* flags, cudaStream_t s);
cudaError_t launch_flag_moment(const float* moment, int64_t G, double thr, uint8_t* flags, cudaStream_t s);
cudaError_t launch_flag_velocity(const float* u, const float* v, int64_t G, double vmin, double vmax,
                                 uint8_t* flags, cudaStream_t s);
cudaError_t launch_mask_flags(uint8_t* flags, const uint8_t* gmask, int64_t G, cudaStream_t s);
cudaError_t launch_substitute(float* u, float* v, const uint8_t* outl_in, uint8_t* outl_out, const uint8_t* gmask,
                              const float* alt_u, const float* alt_v, int32_t nalt, int32_t ny, int32_t nx,
                              int32_t er, double thr, cudaStream_t s);
// replace_vectors!: invalid = flags | gmask (either may be nullptr); masked
// cells are set to NaN afterwards when nan_mask is nonzero.
cudaError_t launch_replace(float* u, float* v, const uint8_t* flags, const uint8_t* gmask, int32_t ny, int32_t nx,
                           int32_t nan_mask, cudaStream_t s);
cudaError_t launch_smooth(const float* f, int32_t ny, int32_t nx, float* out, cudaStream_t s);
// field_change -> *out (device float); scratch: G floats + 2 KB
cudaError_t launch_field_change(const float* u, const float* v, const float* pu, const float* pv,
                                const uint8_t* gmask, int64_t G, float* scratch, float* out, cudaStream_t s);
cudaError_t launch_restore_measured(float* u, float* v, const float* meas_u, const float* meas_v,
                                    const uint8_t* outl, int64_t G, cudaStream_t s);
cudaError_t launch_fill(float* p, float value, int64_t n, cudaStream_t s);

// --- ingestion -------------------------------------------------------------------
// UInt16 frame -> float32: value / 65535 (normalise) or value * 1
cudaError_t launch_u16_to_f32(const uint16_t* src, int64_t n, int32_t normalise, float* dst, cudaStream_t s);

// --- uncertainty -------------------------------------------------------------
struct UQArgs {
  const float* A;
  const float* B;
  const uint8_t* mask;
  int64_t ld;
  const int32_t* jobs;
  int64_t njobs;
  int32_t ny;
  int32_t W;
  const float* apod;
  double* stats;     // 88 per job, or nullptr
  float* unc_u;      // grid-indexed outputs, or nullptr
  float* unc_v;
  // batched mode (bp != nullptr): jobs as in CorrArgs; mode 0 = the fused
  // estimate of a single-sweep pass (sweep 1), 1 = the post-loop estimate
  const BPair* bp;
  const int32_t* done;
  int32_t mode;
  // ensemble mode: stats += this pair's statistics
  int32_t accumulate;
  // rectangular windows (W rows x Wc columns; Wc == 0: square) and windows
  // above 64 px run the general form, whose per-window buffers live in a
  // global scratch slice per CTA (gscr_slices slices of gscr_stride doubles)
  int32_t Wc;
  double* gscr;
  int64_t gscr_stride;
  int32_t gscr_slices;
};
cudaError_t launch_uq(const UQArgs& a, cudaStream_t s, int num_sms);
// Does this window shape run the general (global-scratch) form, and how many
// doubles does one window's scratch slice take?
bool uq_general(int wr, int wc);
int64_t uq_general_stride(int wr, int wc);
// finalize_uncertainty of pooled statistics (88 per job) into grid cells
cudaError_t launch_uq_finalize(const double* stats, const int32_t* jobs, int64_t njobs, int32_t ny, float* unc_u,
                               float* unc_v, cudaStream_t s);

// --- adjoint of deformation + zero-lag correlation --------------------------
struct NccArgs {
  const float* CA;  // B-spline coefficients of both frames, (nr + 2) x (nc + 2)
  const float* CB;
  int64_t nr, nc;
  const float* P;   // predictor: u plane then v plane, gny x gnx each
  int32_t gny, gnx;
  float y0, ysp, x0, xsp;
  int32_t W, step;  // windows: W x W at origins (jr * step, jc * step)
  int32_t wy, wx;   // window grid
  double* wstat;    // 6 per window (scratch)
  float* gpix;      // 2 x nr x nc pixel gradient (scratch), when grad
  float* grad;      // 2 x gny x gnx dL/dP, or nullptr (loss only)
  double* loss;     // device scalar
};
cudaError_t launch_ncc_loss_grad(const NccArgs& a, cudaStream_t s);

}  // namespace hh
