// Batched schedule: one descriptor per (image pair, pass slot), shared by the
// host orchestrator (hh_batch.cu) and the batched kernels (k_batch.cu,
// k_deform.cu, and the batched modes of k_correlate.cu / k_uq.cu).
//
// Every pair owns fixed storage regions of the concatenated arrays for the
// whole run: grid cells [goff, goff + gcap) (gcap = its largest grid over the
// schedule), alternatives [aoff, aoff + nalt*gcap), pixels [poff, poff +
// nr*nc) of the warped pair, padded pixels [qoff, ...) of the B-spline
// coefficients. A pass slot k is the k-th pass of every pair whose schedule
// has one; a pair is live in sweep `it` of slot k when the slot exists for
// it, it <= max_iterations, and it has not converged (done[p]).
//
// Kernels of a slot iterate over slot-compact index spaces (coff: cells of
// the pairs that have the slot; pcoff: their pixels) and find the owning
// pair by binary search, so one launch covers every pair and pairs of
// uneven size cost nothing extra. Everything a kernel needs about a pair is
// read from this table at run time, so a captured graph stays valid when
// only the image pointers or masks of a call change.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "hammerhead_b200.h"

namespace hh {

struct BPair {
  // inputs, valid for the call
  const float* A;
  const float* B;
  const uint8_t* mask;   // image mask or nullptr
  const uint8_t* gmask;  // this slot's grid mask (ny*nx) or nullptr when no cell is masked
  // per-pair library storage
  float* coefA;
  float* coefB;
  float* warpA;
  float* warpB;
  const float* cpc;  // B-spline elimination factors of the column length nr + 2
  const float* ivc;
  const float* cpr;  // ... and of the row length nc + 2
  const float* ivr;
  int64_t nr, nc;
  int64_t poff;   // warped-pixel storage offset (a multiple of 4)
  int64_t qoff;   // padded-pixel (coefficient) storage offset, compact over deforming pairs
  int64_t wcol;   // prefilter work offsets (32-column tiles x segments, 32-row groups x segments)
  int64_t wrow;
  int64_t goff;   // cell storage offset
  int64_t aoff;   // alternatives storage offset (nalt planes of ny*nx cells)
  int64_t coff;   // slot-compact cell offset
  int64_t pcoff;  // slot-compact pixel offset (a multiple of 4)
  int64_t roff;   // offset of the pair's final-pass result
  int32_t ny, nx;      // this slot's grid (0 when the slot does not exist)
  int32_t pgny, pgnx;  // previous slot's grid (predictor of sweep 1)
  float gy0, gysp, gx0, gxsp;  // this slot's node coordinates y0 + i*ysp, x0 + j*xsp
  float py0, pysp, px0, pxsp;  // previous slot's
  int32_t live;       // the pair has this pass slot
  int32_t deforms;    // the pair's schedule deforms (several passes or sweeps)
  int32_t has_pred0;  // a predictor from the previous slot exists (sweep 1)
  int32_t has_next;   // the pair has a later slot
  int32_t is_final;   // this slot is the pair's final pass
  int32_t maxit;      // max_iterations
  int32_t nalt;       // n_peaks - 1
  int32_t W;
  int32_t uod_enable, uod_nb;
  double uod_thr;
  double min_peak_ratio;
  int32_t nval;
  int32_t replace;        // replace_vectors! after validation
  int32_t keep_measured;  // restore measured vectors at flagged cells after the sweeps
  int32_t unc_fused;      // uncertainty estimated in sweep 1 (single-sweep final pass)
  int32_t unc_post;       // uncertainty estimated after the sweeps
  int32_t fgny, fgnx;     // final-pass grid (result region size)
  double tol;             // convergence_tol
  hh_validator val[HH_MAX_VALIDATORS];
};

// live in sweep `it` (1-based)?
__host__ __device__ __forceinline__ bool bp_live(const BPair& b, int it, const int32_t* done, int p) {
  return b.live && it <= b.maxit && !done[p];
}

// The pair whose region [off_p, off_{p+1}) holds index k: the last pair with
// off <= k (offsets ascending; empty regions are skipped).
template <int64_t BPair::*OFF>
__device__ __forceinline__ int bp_find(const BPair* bp, int npairs, int64_t k) {
  int lo = 0, hi = npairs - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (bp[mid].*OFF <= k) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// --- batched launches (k_batch.cu, k_deform.cu) --------------------------------
// Totals of the index spaces a launch covers are passed by the host; the
// kernels stop at them and skip pairs that are not live.
// Copy `bytes` from page-locked host memory (addressable from the device
// under unified addressing) to device memory with a kernel, not a copy-engine
// transfer: the small per-call uploads then never wait behind large frame
// copies that other streams have queued on the host-to-device copy engine.
cudaError_t launch_host_read_copy(void* dst, const void* host_src, size_t bytes, cudaStream_t s);
cudaError_t launch_b_prefilter(const BPair* bp, int npairs, int64_t qtot, int64_t wcol_tot, int64_t wrow_tot,
                               float* dbuf, cudaStream_t s);
cudaError_t launch_b_sweep_begin(const BPair* bp, int npairs, const int32_t* done, int it, int64_t gtot,
                                 const float* pu, const float* pv, float* u, float* v, float* uncu, float* uncv,
                                 int32_t* sweeps, int32_t* slot_sweeps, cudaStream_t s);
cudaError_t launch_b_deform(const BPair* bp, int npairs, const int32_t* done, int it, int64_t ptot, const float* pu,
                            const float* pv, cudaStream_t s);
struct BGrid {  // concatenated grid arrays, indexed by goff + cell
  float *u, *v, *resu, *resv, *ratio, *moment, *alt_u, *alt_v, *meas_u, *meas_v;
  float *prev_u, *prev_v, *predw_u, *predw_v, *pred_u, *pred_v, *unc_u, *unc_v;
  uint8_t *outl, *outl2;
  uint32_t* keys;
};
cudaError_t launch_b_vector(const BPair* bp, int npairs, int32_t* done, int it, int64_t gtot, const BGrid& g,
                            bool any_nalt, bool any_replace, bool any_tol, int max_maxit, cudaStream_t s, int* nlaunch);
cudaError_t launch_b_predictor(const BPair* bp, int npairs, const int32_t* done, int it, int mode, int64_t gtot,
                               const BGrid& g, bool smoothing, cudaStream_t s, int* nlaunch);
cudaError_t launch_b_restore(const BPair* bp, int npairs, int64_t gtot, const BGrid& g, cudaStream_t s);
struct BResult {  // compact final-pass results, indexed by roff + cell
  float *u, *v, *ratio, *moment, *unc_u, *unc_v;
  uint8_t* outl;
};
cudaError_t launch_b_gather(const BPair* bp, int npairs, int64_t rtot, const BGrid& g, const BResult& r,
                            cudaStream_t s);

}  // namespace hh
