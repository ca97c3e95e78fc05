// Batched vector-grid kernels of a WIDIM sweep (sm_100a): one launch covers
// the grids of every image pair of a pass slot. Each thread owns one cell of
// the slot-compact cell space, finds its pair in the descriptor table, and
// applies the same per-cell operations as the single-pair kernels
// (hh_grid.cuh) to that pair's grid region, so results are bit-identical to
// the single-pair schedule. Convergence is decided on the device: the
// field-change kernel marks a pair done and later launches skip it.
#include <math.h>
#include <stdint.h>

#include "hh_batch.h"
#include "hh_grid.cuh"
#include "hh_internal.h"

namespace hh {

#define B_STRIDE(k, n) for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (n); k += (int64_t)gridDim.x * blockDim.x)

static unsigned bb_blocks(int64_t n, int threads) {
  int64_t b = (n + threads - 1) / threads;
  if (b > 148 * 16) b = 148 * 16;
  return (unsigned)(b < 1 ? 1 : b);
}

// Resolve cell k of the slot-compact space: the pair, its local cell index,
// and whether the pair takes part (cond evaluated by the caller's predicate).
#define B_CELL(k, p, b, l)                                   \
  const int p = bp_find<&BPair::coff>(bp, npairs, k);        \
  const BPair& b = bp[p];                                    \
  const int64_t l = k - b.coff;                              \
  if (l >= (int64_t)b.ny * b.nx) continue;

// combine (src/pipeline.jl:755-770)
__global__ void b_combine_kernel(const BPair* __restrict__ bp, int npairs, const int32_t* __restrict__ done, int it,
                                 int64_t gtot, BGrid g) {
  B_STRIDE(k, gtot) {
    B_CELL(k, p, b, l)
    if (!bp_live(b, it, done, p)) continue;
    const int64_t G = (int64_t)b.ny * b.nx, o = b.goff;
    float* au = b.nalt > 0 ? g.alt_u + b.aoff : nullptr;
    float* av = b.nalt > 0 ? g.alt_v + b.aoff : nullptr;
    const bool km = b.keep_measured;
    float* base_u = g.u + o;
    float* base_v = g.v + o;
    const float pu = base_u[l], pv = base_v[l];
    for (int m = 0; m < b.nalt; ++m) {
      au[l + m * G] = FADD(au[l + m * G], pu);
      av[l + m * G] = FADD(av[l + m * G], pv);
    }
    float uu = FADD(pu, g.resu[o + l]), vv = FADD(pv, g.resv[o + l]);
    if (b.gmask && b.gmask[l]) {
      uu = vv = f_nan();
      g.ratio[o + l] = f_nan();
      g.moment[o + l] = f_nan();
    }
    base_u[l] = uu;
    base_v[l] = vv;
    if (km) {
      g.meas_u[o + l] = uu;
      g.meas_v[o + l] = vv;
    }
  }
}

// validate_and_replace! flags (src/pipeline.jl:617-645): UOD, peak ratio,
// the extra validators, masked cells cleared; written to outl and outl2.
__global__ void b_flags_kernel(const BPair* __restrict__ bp, int npairs, const int32_t* __restrict__ done, int it,
                               int64_t gtot, BGrid g) {
  B_STRIDE(k, gtot) {
    B_CELL(k, p, b, l)
    if (!bp_live(b, it, done, p)) continue;
    const int64_t o = b.goff;
    const uint8_t* gm = b.gmask;
    uint8_t f = 0;
    if (!(gm && gm[l])) {
      const int r = (int)(l % b.ny), c = (int)(l / b.ny);
      const float* u = g.u + o;
      const float* v = g.v + o;
      if (b.uod_enable) f |= uod_cell(u, v, b.ny, b.nx, r, c, b.uod_thr, b.uod_nb, 0.1, gm);
      if (b.min_peak_ratio > 1 && !((double)g.ratio[o + l] >= b.min_peak_ratio)) f = 1;
      for (int q = 0; q < b.nval; ++q) {
        const hh_validator& vd = b.val[q];
        if (vd.kind == HH_VAL_PEAK_RATIO) {
          if (!((double)g.ratio[o + l] >= vd.threshold)) f = 1;
        } else if (vd.kind == HH_VAL_MOMENT) {
          if (!((double)g.moment[o + l] <= vd.threshold)) f = 1;
        } else if (vd.kind == HH_VAL_VELOCITY) {
          const double mag = (double)hypotf(u[l], v[l]);
          if (!(vd.vmin <= mag && mag <= vd.vmax)) f = 1;
        } else if (vd.kind == HH_VAL_UOD) {
          f |= uod_cell(u, v, b.ny, b.nx, r, c, vd.threshold, vd.neighborhood, vd.epsilon, gm);
        }
      }
    }
    g.outl[o + l] = f;
    g.outl2[o + l] = f;
  }
}

// secondary-peak substitution (src/quality.jl:307-351): outl -> outl2
__global__ void b_substitute_kernel(const BPair* __restrict__ bp, int npairs, const int32_t* __restrict__ done, int it,
                                    int64_t gtot, BGrid g) {
  B_STRIDE(k, gtot) {
    B_CELL(k, p, b, l)
    if (!bp_live(b, it, done, p) || b.nalt < 1) continue;
    const int64_t o = b.goff;
    const int r = (int)(l % b.ny), c = (int)(l / b.ny);
    g.outl2[o + l] = substitute_cell(g.u + o, g.v + o, g.outl + o, b.gmask, g.alt_u + b.aoff, g.alt_v + b.aoff,
                                     b.nalt, b.ny, b.nx, r, c, b.uod_nb, b.uod_thr);
  }
}

// replace_vectors! at outl2 | gmask, masked cells -> NaN
__global__ void b_replace_kernel(const BPair* __restrict__ bp, int npairs, const int32_t* __restrict__ done, int it,
                                 int64_t gtot, BGrid g) {
  B_STRIDE(k, gtot) {
    B_CELL(k, p, b, l)
    if (!bp_live(b, it, done, p) || !b.replace) continue;
    const int64_t o = b.goff;
    const uint8_t* fl = g.outl2 + o;
    if (!repl_invalid(fl, b.gmask, l)) continue;
    float nu = g.u[o + l], nv = g.v[o + l];
    replace_cell(g.u + o, g.v + o, fl, b.gmask, b.ny, b.nx, (int)(l % b.ny), (int)(l / b.ny), nu, nv);
    if (b.gmask && b.gmask[l]) nu = nv = f_nan();
    g.u[o + l] = nu;
    g.v[o + l] = nv;
  }
}

// field_change (src/pipeline.jl:849-866), one CTA per pair; a pair whose
// change falls below convergence_tol is marked done.
constexpr int BFC_THREADS = 1024;

__global__ void __launch_bounds__(BFC_THREADS) b_field_change_kernel(const BPair* __restrict__ bp, int32_t* done, int it,
                                                                     BGrid g) {
  __shared__ uint32_t hist[256];
  __shared__ uint32_t s_bucket;
  __shared__ int64_t s_k;
  __shared__ unsigned long long s_n;
  const int p = blockIdx.x;
  const BPair& b = bp[p];
  if (!bp_live(b, it, done, p) || !(it < b.maxit) || !(b.tol > 0)) return;  // uniform across the CTA
  const int64_t G = (int64_t)b.ny * b.nx, o = b.goff;
  uint32_t* keys = g.keys + o;
  if (threadIdx.x == 0) s_n = 0;
  __syncthreads();
  unsigned long long n_local = 0;
  for (int64_t i = threadIdx.x; i < G; i += blockDim.x) {
    bool counts;
    keys[i] = change_key(g.u[o + i], g.v[o + i], g.prev_u[o + i], g.prev_v[o + i], b.gmask && b.gmask[i], counts);
    n_local += counts;
  }
  atomicAdd(&s_n, n_local);
  __syncthreads();
  const int64_t n = (int64_t)s_n;
  float change = 0.f;
  if (n > 0) {
    int64_t ka, kb;
    double gq;
    quantile95_index(n, ka, kb, gq);
    const uint32_t a = cta_radix_select(keys, G, ka, hist, &s_bucket, &s_k);
    const uint32_t c = kb == ka ? a : cta_radix_select(keys, G, kb, hist, &s_bucket, &s_k);
    change = quantile95_value(a, c, gq);
  }
  if (threadIdx.x == 0 && (double)change < b.tol) done[p] = 1;
}

cudaError_t launch_b_vector(const BPair* bp, int npairs, int32_t* done, int it, int64_t gtot, const BGrid& g,
                            bool any_nalt, bool any_replace, bool any_tol, int max_maxit, cudaStream_t s, int* nlaunch) {
  if (gtot <= 0) return cudaSuccess;
  int n = 0;
  b_combine_kernel<<<bb_blocks(gtot, 256), 256, 0, s>>>(bp, npairs, done, it, gtot, g);
  b_flags_kernel<<<bb_blocks(gtot, 128), 128, 0, s>>>(bp, npairs, done, it, gtot, g);
  n += 2;
  if (any_nalt) {
    b_substitute_kernel<<<bb_blocks(gtot, 128), 128, 0, s>>>(bp, npairs, done, it, gtot, g);
    ++n;
  }
  if (any_replace) {
    b_replace_kernel<<<bb_blocks(gtot, 128), 128, 0, s>>>(bp, npairs, done, it, gtot, g);
    ++n;
  }
  if (any_tol && it >= 2 && it < max_maxit) {
    b_field_change_kernel<<<npairs, BFC_THREADS, 0, s>>>(bp, done, it, g);
    ++n;
  }
  if (nlaunch) *nlaunch = n;
  return cudaGetLastError();
}

// Predictor for the next sweep (mode 0: pairs live in sweep `it` that sweep
// again) or for the next pass slot (mode 1: pairs with a later slot):
// build_predictor (src/pipeline.jl:454-464) -- masked cells replaced from
// their valid neighbours, then [1 2 1] smoothing. Mode 0 also keeps the
// field for the convergence test of the next sweep.
__device__ __forceinline__ bool b_pred_on(const BPair& b, int mode, int it, const int32_t* done, int p) {
  return mode == 0 ? (bp_live(b, it, done, p) && it < b.maxit) : (b.live && b.has_next);
}

__global__ void b_pred_build_kernel(const BPair* __restrict__ bp, int npairs, const int32_t* __restrict__ done, int it,
                                    int mode, int64_t gtot, BGrid g) {
  B_STRIDE(k, gtot) {
    B_CELL(k, p, b, l)
    if (!b_pred_on(b, mode, it, done, p)) continue;
    const int64_t o = b.goff;
    float nu = g.u[o + l], nv = g.v[o + l];
    if (mode == 0 && b.tol > 0) {
      g.prev_u[o + l] = nu;
      g.prev_v[o + l] = nv;
    }
    if (b.gmask && b.gmask[l])
      replace_cell(g.u + o, g.v + o, nullptr, b.gmask, b.ny, b.nx, (int)(l % b.ny), (int)(l / b.ny), nu, nv);
    g.predw_u[o + l] = nu;
    g.predw_v[o + l] = nv;
  }
}

__global__ void b_smooth_kernel(const BPair* __restrict__ bp, int npairs, const int32_t* __restrict__ done, int it,
                                int mode, int64_t gtot, BGrid g) {
  B_STRIDE(k, gtot) {
    B_CELL(k, p, b, l)
    if (!b_pred_on(b, mode, it, done, p)) continue;
    const int64_t o = b.goff;
    const int r = (int)(l % b.ny), c = (int)(l / b.ny);
    g.pred_u[o + l] = smooth_cell(g.predw_u + o, b.ny, b.nx, r, c);
    g.pred_v[o + l] = smooth_cell(g.predw_v + o, b.ny, b.nx, r, c);
  }
}

cudaError_t launch_b_predictor(const BPair* bp, int npairs, const int32_t* done, int it, int mode, int64_t gtot,
                               const BGrid& g, bool smoothing, cudaStream_t s, int* nlaunch) {
  if (gtot <= 0) return cudaSuccess;
  b_pred_build_kernel<<<bb_blocks(gtot, 128), 128, 0, s>>>(bp, npairs, done, it, mode, gtot, g);
  int n = 1;
  if (smoothing) {
    b_smooth_kernel<<<bb_blocks(gtot, 256), 256, 0, s>>>(bp, npairs, done, it, mode, gtot, g);
    ++n;
  }
  if (nlaunch) *nlaunch = n;
  return cudaGetLastError();
}

// measured vectors back at flagged cells (src/pipeline.jl:800-806)
__global__ void b_restore_kernel(const BPair* __restrict__ bp, int npairs, int64_t gtot, BGrid g) {
  B_STRIDE(k, gtot) {
    B_CELL(k, p, b, l)
    if (!b.live || !b.keep_measured) continue;
    const int64_t o = b.goff;
    if (g.outl2[o + l]) {
      g.u[o + l] = g.meas_u[o + l];
      g.v[o + l] = g.meas_v[o + l];
    }
  }
}

cudaError_t launch_b_restore(const BPair* bp, int npairs, int64_t gtot, const BGrid& g, cudaStream_t s) {
  if (gtot <= 0) return cudaSuccess;
  b_restore_kernel<<<bb_blocks(gtot, 256), 256, 0, s>>>(bp, npairs, gtot, g);
  return cudaGetLastError();
}

// final-pass fields of every pair into the compact result arrays
__global__ void b_gather_kernel(const BPair* __restrict__ bp, int npairs, int64_t rtot, BGrid g, BResult r) {
  B_STRIDE(k, rtot) {
    const int p = bp_find<&BPair::roff>(bp, npairs, k);
    const BPair& b = bp[p];
    const int64_t l = k - b.roff;
    if (l >= (int64_t)b.fgny * b.fgnx) continue;
    const int64_t o = b.goff + l;
    r.u[k] = g.u[o];
    r.v[k] = g.v[o];
    r.ratio[k] = g.ratio[o];
    r.moment[k] = g.moment[o];
    r.unc_u[k] = g.unc_u[o];
    r.unc_v[k] = g.unc_v[o];
    r.outl[k] = g.outl2[o];
  }
}

cudaError_t launch_b_gather(const BPair* bp, int npairs, int64_t rtot, const BGrid& g, const BResult& r,
                            cudaStream_t s) {
  if (rtot <= 0) return cudaSuccess;
  b_gather_kernel<<<bb_blocks(rtot, 256), 256, 0, s>>>(bp, npairs, rtot, g, r);
  return cudaGetLastError();
}

// 16-byte words while both addresses and the length allow, then the tail by
// bytes; the source is page-locked host memory read over the bus
__global__ void host_read_copy_kernel(uint8_t* __restrict__ dst, const uint8_t* __restrict__ src, size_t bytes) {
  const size_t n16 = ((reinterpret_cast<uintptr_t>(dst) | reinterpret_cast<uintptr_t>(src)) & 15) ? 0 : bytes / 16;
  const size_t t = blockIdx.x * (size_t)blockDim.x + threadIdx.x, nt = (size_t)gridDim.x * blockDim.x;
  for (size_t k = t; k < n16; k += nt) reinterpret_cast<uint4*>(dst)[k] = reinterpret_cast<const uint4*>(src)[k];
  for (size_t k = n16 * 16 + t; k < bytes; k += nt) dst[k] = src[k];
}

cudaError_t launch_host_read_copy(void* dst, const void* host_src, size_t bytes, cudaStream_t s) {
  if (bytes == 0) return cudaSuccess;
  size_t blocks = (bytes / 16 + 255) / 256;
  if (blocks < 1) blocks = 1;
  if (blocks > 148 * 4) blocks = 148 * 4;
  host_read_copy_kernel<<<(unsigned)blocks, 256, 0, s>>>(static_cast<uint8_t*>(dst), static_cast<const uint8_t*>(host_src),
                                                         bytes);
  return cudaGetLastError();
}

}  // namespace hh
