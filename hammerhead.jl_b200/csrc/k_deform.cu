// Symmetric image deformation for WIDIM sweeps (sm_100a).
//
// prefilter: cubic B-spline coefficients of Interpolations.jl's
//   BSpline(Cubic(Line(OnGrid()))) on the (nr+2) x (nc+2) padded index set
//   (the coefficient array image_interpolant builds, src/pipeline.jl:75-85,
//   909-915): per line, rows [1 4 1]/6 inside and the "Line" boundary rows
//   c0 - 2c1 + c2 = 0. Eliminating the boundary rows leaves c1 = b1,
//   c_{n-2} = b_{n-2} and a constant-coefficient tridiagonal system, solved
//   by the Thomas algorithm with the line-independent elimination factors
//   precomputed once. Separable: every column, then every row.
// deform: one thread per output pixel evaluates the predictor by bilinear
//   interpolation with flat extrapolation (Gridded(Linear()) + Flat(),
//   src/pipeline.jl:561-600) and samples both coefficient arrays with the
//   4x4 cubic B-spline at -+ half the displacement, zero outside the image
//   (deform_columns!, src/pipeline.jl:957-965; _ka_deform!,
//   src/ka_backend.jl:266-312).
// All floating-point operations use explicit round-to-nearest intrinsics so
// no multiply-add is fused: results equal the CPU restatement bit for bit.
#include <math.h>
#include <stdint.h>

#include "hh_batch.h"
#include "hh_internal.h"

namespace hh {

#define FM(a, b) __fmul_rn((a), (b))
#define FA(a, b) __fadd_rn((a), (b))
#define FS(a, b) __fsub_rn((a), (b))
#define FD(a, b) __fdiv_rn((a), (b))

// Correctly rounded float constants of 1/6 and 2/3 (what 1f0/6 and 2f0/3
// evaluate to), and x/2 taken as x*0.5: halving by a power of two is the
// same correctly rounded value either way, so the results are unchanged.
static __device__ __forceinline__ float k_sixth() { return __int_as_float(0x3E2AAAAB); }
static __device__ __forceinline__ float k_two_thirds() { return __int_as_float(0x3F2AAAAB); }
#define kSixth k_sixth()
#define kTwoThirds k_two_thirds()

// x / 6 correctly rounded for every x whose quotient is a normal float (and
// x = 0), without a division: q0 = x * RN(1/6), then one residual correction
// by fused multiply-add (Markstein's correction for a divisor known in
// advance; Brisebarre, Muller and Raina, IEEE Trans. Computers 53(8), 2004).
// A comparison with IEEE division over every positive float with a normal
// quotient finds no difference. The B-spline weights (1-d)^3 and d^3 it
// divides are 0 or at least 2^-72 (d is 0 or a multiple of 2^-23 in [0, 1]),
// so their quotients are normal.
static __device__ __forceinline__ float div6(float x) {
  const float r = k_sixth();
  const float q0 = __fmul_rn(x, r);
  const float e = __fmaf_rn(-q0, 6.0f, x);
  return __fmaf_rn(e, r, q0);
}

// Elimination factors for a line of padded length n: unknown rows
// i = 3..n-2 (1-based). inv[k] = 1/den_k, cp[k] = (1/6)*inv[k], k = i - 3.
__global__ void bspline_factors_kernel(int64_t n, float* cp, float* inv) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const float sixth = FD(1.0f, 6.0f), b = FD(4.0f, 6.0f);
  const int64_t m = n - 4;  // number of unknowns
  float cprev = 0.f;
  for (int64_t k = 0; k < m; ++k) {
    float den = k == 0 ? b : FS(b, FM(sixth, cprev));
    float iv = FD(1.0f, den);
    inv[k] = iv;
    cprev = FM(sixth, iv);
    cp[k] = cprev;
  }
}

// Both Thomas sweeps are contractions (|cp_k| -> 0.268), so each line is cut
// into independent segments of BS_SEG unknowns whose sweeps start BS_WARM
// unknowns early from a zero state; the neglected term is below
// 0.268^32 ~ 5e-19 of the value, far under float rounding. The CPU
// restatement solves each line in one sweep; the deformed images are held to
// 4 ulp of the image scale against it. The forward sweep is
// d_k = (rhs_k - d_{k-1}/6) inv_k (unknown k at line element k + 2; rhs_0 and
// rhs_{m-1} carry the known c1 and c_{n-2}), the backward sweep
// x_k = d_k - cp_k x_{k+1}, followed by the "Line" boundary coefficients
// c0 = 2c1 - c2 and c_{n-1} = 2c_{n-2} - c_{n-3}. BS_SEG, BS_WARM and the
// segment count b_nseg are in hh_internal.h (the batched plan counts work
// items with them).

cudaError_t launch_bspline_factors(int64_t n, float* cp, float* inv, cudaStream_t s) {
  bspline_factors_kernel<<<1, 1, 0, s>>>(n, cp, inv);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Gridded(Linear()) + Flat() along one axis of uniform knots q0 + k*step.
__device__ __forceinline__ void lin_axis(float q, float q0, float step, int n, int& i, float& d) {
  if (n == 1) { i = 0; d = 0.f; return; }
  const float last = FA(q0, FM((float)(n - 1), step));
  if (q <= q0) { i = 0; d = 0.f; return; }
  if (q >= last) { i = n - 2; d = 1.f; return; }
  i = (int)floorf(FD(FS(q, q0), step));
  if (i > n - 2) i = n - 2;
  const float k0 = FA(q0, FM((float)i, step)), k1 = FA(q0, FM((float)(i + 1), step));
  d = FD(FS(q, k0), FS(k1, k0));
}

// the bilinear combination at cell (iy, ix) with fractions (dy, dx)
__device__ __forceinline__ float bilinear_at(const float* f, const PredGrid& g, int iy, float dy, int ix, float dx) {
  const int iy2 = g.gny == 1 ? iy : iy + 1, ix2 = g.gnx == 1 ? ix : ix + 1;
  const float f00 = f[iy + ix * g.gny], f01 = f[iy + ix2 * g.gny], f10 = f[iy2 + ix * g.gny],
              f11 = f[iy2 + ix2 * g.gny];
  const float a = FA(FM(FS(1.f, dx), f00), FM(dx, f01));
  const float b = FA(FM(FS(1.f, dx), f10), FM(dx, f11));
  return FA(FM(FS(1.f, dy), a), FM(dy, b));
}

__device__ __forceinline__ float bilinear(const float* f, const PredGrid& g, float qy, float qx) {
  int iy, ix;
  float dy, dx;
  lin_axis(qy, g.y0, g.ysp, g.gny, iy, dy);
  lin_axis(qx, g.x0, g.xsp, g.gnx, ix, dx);
  const int iy2 = g.gny == 1 ? iy : iy + 1, ix2 = g.gnx == 1 ? ix : ix + 1;
  const float f00 = f[iy + ix * g.gny], f01 = f[iy + ix2 * g.gny], f10 = f[iy2 + ix * g.gny],
              f11 = f[iy2 + ix2 * g.gny];
  const float a = FA(FM(FS(1.f, dx), f00), FM(dx, f01));
  const float b = FA(FM(FS(1.f, dx), f10), FM(dx, f11));
  return FA(FM(FS(1.f, dy), a), FM(dy, b));
}

// Interpolations' cubic B-spline weights at fractional offset d.
__device__ __forceinline__ void cubw(float d, float* w) {
  const float x3 = FM(FM(d, d), d), c = FS(1.f, d), c3 = FM(FM(c, c), c);
  const float two3 = kTwoThirds;
  w[0] = div6(c3);
  w[1] = FA(FS(two3, FM(d, d)), FM(x3, 0.5f));
  w[2] = FA(FS(two3, FM(c, c)), FM(c3, 0.5f));
  w[3] = div6(x3);
}

__device__ __forceinline__ float bspline_eval(const float* C, int64_t nr, int64_t nc, float yy, float xx) {
  if (yy < 1.f || yy > (float)nr || xx < 1.f || xx > (float)nc) return 0.f;
  int64_t iy = (int64_t)floorf(yy);
  if (iy > nr - 1) iy = nr - 1;
  int64_t ix = (int64_t)floorf(xx);
  if (ix > nc - 1) ix = nc - 1;
  float wy[4], wx[4];
  cubw(FS(yy, (float)iy), wy);
  cubw(FS(xx, (float)ix), wx);
  const int64_t ld = nr + 2;
  const float* base = C + (iy - 1) + (ix - 1) * ld;
  float s = 0.f;
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    float t = 0.f;
#pragma unroll
    for (int b = 0; b < 4; ++b) t = FA(t, FM(wx[b], __ldg(base + a + b * ld)));
    s = FA(s, FM(wy[a], t));
  }
  return s;
}

__global__ void __launch_bounds__(256) deform_kernel(const float* __restrict__ CA, const float* __restrict__ CB,
                                                     int64_t nr, int64_t nc, const float* __restrict__ pu,
                                                     const float* __restrict__ pv, PredGrid g, float* wA, float* wB) {
  const int64_t total = nr * nc;
  const bool small = total <= 0x7fffffff;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    const int64_t r = small ? (int64_t)((uint32_t)k % (uint32_t)nr) : k % nr;
    const int64_t c = small ? (int64_t)((uint32_t)k / (uint32_t)nr) : k / nr;
    const float R = (float)(r + 1), Cc = (float)(c + 1);
    const float du2 = FM(bilinear(pu, g, R, Cc), 0.5f);
    const float dv2 = FM(bilinear(pv, g, R, Cc), 0.5f);
    wA[k] = bspline_eval(CA, nr, nc, FS(R, dv2), FS(Cc, du2));
    wB[k] = bspline_eval(CB, nr, nc, FA(R, dv2), FA(Cc, du2));
  }
}

cudaError_t launch_deform(const float* CA, const float* CB, int64_t nr, int64_t nc, const float* pu,
                          const float* pv, PredGrid g, float* wA, float* wB, cudaStream_t s) {
  const int64_t total = nr * nc;
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 32) blocks = 148 * 32;
  deform_kernel<<<(unsigned)blocks, 256, 0, s>>>(CA, CB, nr, nc, pu, pv, g, wA, wB);
  return cudaGetLastError();
}

__global__ void node_values_kernel(const float* pu, const float* pv, PredGrid g, const float* y, int32_t ny,
                                   const float* x, int32_t nx, float* u, float* v) {
  const int64_t total = (int64_t)ny * nx;
  for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < total; k += (int64_t)gridDim.x * blockDim.x) {
    const int gi = (int)(k % ny), gj = (int)(k / ny);
    u[k] = bilinear(pu, g, y[gi], x[gj]);
    v[k] = bilinear(pv, g, y[gi], x[gj]);
  }
}

cudaError_t launch_node_values(const float* pu, const float* pv, PredGrid g, const float* y, int32_t ny,
                               const float* x, int32_t nx, float* u, float* v, cudaStream_t s) {
  const int64_t total = (int64_t)ny * nx;
  int64_t blocks = (total + 255) / 256;
  if (blocks > 148 * 8) blocks = 148 * 8;
  if (blocks < 1) blocks = 1;
  node_values_kernel<<<(unsigned)blocks, 256, 0, s>>>(pu, pv, g, y, ny, x, nx, u, v);
  return cudaGetLastError();
}

// ===========================================================================
// Batched forms: every pair of a pass slot in one launch (see hh_batch.h).

#define B_STRIDE(k, n) for (int64_t k = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; k < (n); k += (int64_t)gridDim.x * blockDim.x)

static unsigned b_blocks(int64_t n, int cap_per_sm = 16) {
  int64_t b = (n + 255) / 256;
  if (b > 148 * (int64_t)cap_per_sm) b = 148 * (int64_t)cap_per_sm;
  return (unsigned)(b < 1 ? 1 : b);
}

// prefilter of both frames (blockIdx.y: 0 = A, 1 = B) of every deforming pair.
//
// dim 1 (down the image columns, contiguous in memory) runs on 32-column
// tiles: a warp takes 32 neighbouring columns and one segment, the lanes
// load and store down each column together (coalesced) through a staged
// tile in shared memory, and each lane then runs its own column's sweep
// from the tile with the arithmetic of bs_fwd_item / bs_bwd_item. The
// forward pass reads the image itself (padded element e of column j + 1 is
// image row e - 1), and the backward pass writes every element of the
// padded column, the copied rows 1 and n - 2 included, so no padded copy of
// the image is made first. Work items: (column tile, segment) per pair,
// counted from BPair::wcol.

constexpr int BS_TILE = BS_WARM + BS_SEG;  // rows staged per column
constexpr int BS_TLD = BS_TILE + 1;        // odd stride: conflict-free by lane and by row
constexpr int BSC_WARPS = 4;
constexpr int BS_RPL = (BS_TILE + 31) / 32;  // staged rows per lane and column
// per warp: a tile (32 columns x BS_TILE rows at stride BS_TLD, or BS_TILE
// columns x 32 rows at stride 33) and the elimination factors of its
// BS_TILE unknowns
constexpr int BS_WTILE = BS_TILE * 33 > 32 * BS_TLD ? BS_TILE * 33 : 32 * BS_TLD;
constexpr int BS_WSTRIDE = BS_WTILE + BS_TILE;
constexpr size_t BSC_SMEM = (size_t)BSC_WARPS * BS_WSTRIDE * sizeof(float);

// The factors f[0 .. cnt) into F: every lane of a sweep uses the same factor
// at each step, and staging them keeps an L2 round trip out of the sweep's
// dependent chain. The copies join the tile's asynchronous copies, and
// stage_factors waits for all of them.
__device__ __forceinline__ void bs_cp_async4(float* dst, const float* src);
__device__ __forceinline__ void bs_cp_async_wait_all();
__device__ __forceinline__ void stage_factors(float* F, const float* f, int cnt, int lane) {
  for (int j = lane; j < cnt; j += 32) bs_cp_async4(F + j, f + j);
  bs_cp_async_wait_all();
}

// Rows [0, cnt) (cnt <= BS_TILE) of `ncol` columns between global memory (column
// c at g + c * gld) and a staged tile (column c at T + c * BS_TLD). The
// lanes walk down the columns. Loads are asynchronous copies straight into
// shared memory, all of the tile's issued before the first is waited for (in
// stage_factors): one memory round trip per item instead of one per batch of
// registers.
__device__ __forceinline__ void bs_cp_async4(float* dst, const float* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void bs_cp_async_wait_all() {
  asm volatile("cp.async.commit_group;\n" ::: "memory");
  asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}
__device__ __forceinline__ void tile_load(float* T, const float* g, int64_t gld, int ncol, int cnt, int lane) {
  for (int c = 0; c < ncol; ++c)
#pragma unroll
    for (int j = 0; j < BS_RPL; ++j) {
      const int r = lane + 32 * j;
      if (r < cnt) bs_cp_async4(T + c * BS_TLD + r, g + c * gld + r);
    }
}
__device__ __forceinline__ void tile_store(const float* T, float* g, int64_t gld, int ncol, int cnt, int lane) {
  for (int c0 = 0; c0 < ncol; c0 += 8) {
    float v[8][BS_RPL];
#pragma unroll
    for (int u = 0; u < 8; ++u)
#pragma unroll
      for (int j = 0; j < BS_RPL; ++j) {
        const int c = c0 + u, r = lane + 32 * j;
        v[u][j] = (c < ncol && r < cnt) ? T[c * BS_TLD + r] : 0.f;
      }
#pragma unroll
    for (int u = 0; u < 8; ++u)
#pragma unroll
      for (int j = 0; j < BS_RPL; ++j) {
        const int c = c0 + u, r = lane + 32 * j;
        if (c < ncol && r < cnt) g[c * gld + r] = v[u][j];
      }
  }
}

// Work item l of the column pass of one image (nr x nc, column-major): a
// tile of 32 columns and one segment of their unknowns. coef0 / d0: the
// padded coefficients and the forward-sweep buffer ((nr + 2) x (nc + 2)).
template <int PASS>
__device__ __forceinline__ void bs_col_item(const float* __restrict__ img0, float* coef0, float* d0, int64_t nr,
                                            int64_t nc, const float* __restrict__ cpc, const float* __restrict__ ivc,
                                            int64_t l, float* T, float* F, int lane) {
  {
    const int64_t n = nr + 2, m = n - 4;
    const int64_t ncg = (nc + 31) / 32;
    const int64_t cg = l % ncg, seg = l / ncg;
    const int ncol = (int)min((int64_t)32, nc - cg * 32);  // columns of this tile
    const float* im = img0 + cg * 32 * nr;                     // image column cg*32
    float* coef = coef0 + (cg * 32 + 1) * n;                   // padded column cg*32 + 1
    float* d = d0 + (cg * 32 + 1) * n;
    const bool mine = lane < ncol;
    if (m < 1) {  // n <= 4: nothing to solve; the backward pass writes the column
      if (PASS == 1 && mine) {
        const float* ic = im + lane * nr;
        float* x = coef + lane * n;
        if (n == 4) {
          const float c1 = ic[0], c2 = ic[1];
          x[0] = FS(FM(2.0f, c1), c2);
          x[1] = c1;
          x[2] = c2;
          x[3] = FS(FM(2.0f, c2), c1);
        } else {  // n == 3: the padded copy as it stands
          x[0] = 0.f;
          x[1] = ic[0];
          x[2] = 0.f;
        }
      }
      return;
    }
    const int64_t k0 = seg * BS_SEG, k1 = min(m, k0 + BS_SEG);
    if (PASS == 0) {
      const int64_t ks = max((int64_t)0, k0 - BS_WARM);
      const int cnt = (int)(k1 - ks);
      // stage the right-hand sides: unknown k is padded element k + 2 = image row k + 1
      tile_load(T, im + ks + 1, nr, ncol, cnt, lane);
      stage_factors(F, ivc + ks, cnt, lane);
      __syncwarp();
      if (mine) {
        const float* ic = im + lane * nr;
        const float sixth = kSixth;
        const float c2 = __ldg(ic), cn1 = __ldg(ic + nr - 1);  // padded elements 1 and n - 2
        float* x = T + lane * BS_TLD;
        float dv = 0.f;
#pragma unroll 4
        for (int64_t k = ks; k < k1; ++k) {
          float rhs = x[k - ks];
          if (k == 0) rhs = FS(rhs, FM(sixth, c2));
          if (k == m - 1) rhs = FS(rhs, FM(sixth, cn1));
          dv = k == 0 ? FM(rhs, F[0]) : FM(FS(rhs, FM(sixth, dv)), F[k - ks]);
          x[k - ks] = dv;
        }
      }
      __syncwarp();
      const int nout = (int)(k1 - k0), o = (int)(k0 - ks);
      tile_store(T + o, d + k0 + 2, n, ncol, nout, lane);
      __syncwarp();  // the tile is restaged by the next item
    } else {
      const int64_t ke = min(m - 1, k1 - 1 + BS_WARM);
      const int cnt = (int)(ke - k0 + 1);
      tile_load(T, d + k0 + 2, n, ncol, cnt, lane);
      stage_factors(F, cpc + k0, cnt, lane);
      __syncwarp();
      if (mine) {
        float* x = T + lane * BS_TLD;
        float xv = 0.f, xlast = 0.f;
#pragma unroll 4
        for (int64_t k = ke; k >= k0; --k) {
          const float dk = x[k - k0];
          xv = k == ke ? dk : FS(dk, FM(F[k - k0], xv));
          x[k - k0] = xv;
          if (k == m - 1) xlast = xv;
        }
        const float* ic = im + lane * nr;
        float* xc = coef + lane * n;
        if (k0 == 0) {  // padded element 1 is image row 0; element 0 the "Line" boundary
          const float c1 = __ldg(ic);
          xc[1] = c1;
          xc[0] = FS(FM(2.0f, c1), xv);  // xv == x_0 here
        }
        if (k1 == m) {
          const float cn = __ldg(ic + nr - 1);
          xc[n - 2] = cn;
          xc[n - 1] = FS(FM(2.0f, cn), xlast);
        }
      }
      __syncwarp();
      const int nout = (int)(k1 - k0);
      tile_store(T, coef + k0 + 2, n, ncol, nout, lane);
      __syncwarp();
    }
  }
}

template <int PASS>
__global__ void __launch_bounds__(32 * BSC_WARPS) b_bspline_col_kernel(const BPair* __restrict__ bp, int npairs,
                                                                      int64_t witems, float* dbuf, int64_t qtot) {
  extern __shared__ float bsc_tile[];
  const int img = blockIdx.y, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* T = bsc_tile + warp * BS_WSTRIDE;
  float* F = T + BS_WTILE;
  for (int64_t t = (int64_t)blockIdx.x * BSC_WARPS + warp; t < witems; t += (int64_t)gridDim.x * BSC_WARPS) {
    const BPair& b = bp[bp_find<&BPair::wcol>(bp, npairs, t)];
    if (!b.deforms) continue;  // uniform across the warp
    const int64_t l = t - b.wcol;
    if (l >= (b.nc + 31) / 32 * b_nseg(b.nr + 2)) continue;
    bs_col_item<PASS>(img ? b.B : b.A, img ? b.coefB : b.coefA, dbuf + (int64_t)img * qtot + b.qoff, b.nr, b.nc,
                      b.cpc, b.ivc, l, T, F, lane);
  }
}

// Padding columns 0 and nc + 1 are written by the row pass's "Line"
// boundary; only rows too short to solve (nc + 2 < 4) keep them zero.
__global__ void b_pad_cols_kernel(const BPair* __restrict__ bp, int npairs) {
  const int img = blockIdx.y;
  for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
    const BPair& b = bp[p];
    if (!b.deforms || b.nc + 2 >= 4) continue;
    const int64_t n = b.nr + 2;
    float* coef = img ? b.coefB : b.coefA;
    for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
      coef[i] = 0.f;
      coef[(b.nc + 1) * n + i] = 0.f;
    }
  }
}

// dim 2: a warp takes 32 consecutive padded rows and one segment of their
// unknowns. The segment's columns are staged in shared memory (each column's
// 32 rows are one coalesced 128-byte copy, every column in flight at once),
// the lanes sweep their rows there (row r of staged column j at
// T[33 j + r]: conflict-free), and the results leave the same way. The
// arithmetic is bs_fwd_item / bs_bwd_item's, step for step.
__device__ __forceinline__ void row_tile_load(float* T, const float* g, int64_t gld, int nrow, int cnt, int lane) {
  if (lane < nrow)
    for (int j = 0; j < cnt; ++j) bs_cp_async4(T + j * 33 + lane, g + j * gld + lane);
}
__device__ __forceinline__ void row_tile_store(const float* T, float* g, int64_t gld, int nrow, int cnt, int lane) {
  if (lane >= nrow) return;
  for (int j = 0; j < cnt; ++j) g[j * gld + lane] = T[j * 33 + lane];
}

// Work item l of the row pass of one image's padded coefficients coef0
// ((nr + 2) x (nc + 2)), with the forward-sweep buffer d0 of the same shape.
template <int PASS>
__device__ __forceinline__ void bs_row_item(float* coef0, float* d0, int64_t nr, int64_t nc,
                                            const float* __restrict__ cpr, const float* __restrict__ ivr, int64_t l,
                                            float* T, float* F, int lane) {
  {
    const int64_t ld = nr + 2, n = nc + 2, m = n - 4;
    const int64_t nrg = (ld + 31) / 32;
    const int64_t rg = l % nrg, seg = l / nrg, r0 = rg * 32;
    const int nrow = (int)min((int64_t)32, ld - r0);
    const bool mine = lane < nrow;
    float* coef = coef0 + r0;  // row r0 of the padded coefficients
    float* d = d0 + r0;
    if (PASS == 0) {
      if (m < 1) return;
      const int64_t k0 = seg * BS_SEG, k1 = min(m, k0 + BS_SEG), ks = max((int64_t)0, k0 - BS_WARM);
      const int cnt = (int)(k1 - ks);
      row_tile_load(T, coef + (ks + 2) * ld, ld, nrow, cnt, lane);  // unknown k is padded column k + 2
      stage_factors(F, ivr + ks, cnt, lane);
      __syncwarp();
      if (mine) {
        const float sixth = kSixth;
        const float c2 = coef[ld + lane], cn1 = coef[(n - 2) * ld + lane];
        float dv = 0.f;
#pragma unroll 4
        for (int64_t k = ks; k < k1; ++k) {
          float* x = T + (k - ks) * 33 + lane;
          float rhs = *x;
          if (k == 0) rhs = FS(rhs, FM(sixth, c2));
          if (k == m - 1) rhs = FS(rhs, FM(sixth, cn1));
          dv = k == 0 ? FM(rhs, F[0]) : FM(FS(rhs, FM(sixth, dv)), F[k - ks]);
          *x = dv;
        }
      }
      __syncwarp();
      row_tile_store(T + (k0 - ks) * 33, d + (k0 + 2) * ld, ld, nrow, (int)(k1 - k0), lane);
      __syncwarp();  // the tile is restaged by the next item
    } else {
      if (n < 4) return;
      if (m < 1) {  // n == 4: c1 = b1, c2 = b2 only
        if (mine) {
          const float c1 = coef[ld + lane], c2 = coef[2 * ld + lane];
          coef[lane] = FS(FM(2.0f, c1), c2);
          coef[3 * ld + lane] = FS(FM(2.0f, c2), c1);
        }
        return;
      }
      const int64_t k0 = seg * BS_SEG, k1 = min(m, k0 + BS_SEG), ke = min(m - 1, k1 - 1 + BS_WARM);
      const int cnt = (int)(ke - k0 + 1);
      row_tile_load(T, d + (k0 + 2) * ld, ld, nrow, cnt, lane);
      stage_factors(F, cpr + k0, cnt, lane);
      __syncwarp();
      if (mine) {
        float xv = 0.f, xlast = 0.f;
#pragma unroll 4
        for (int64_t k = ke; k >= k0; --k) {
          float* x = T + (k - k0) * 33 + lane;
          const float dk = *x;
          xv = k == ke ? dk : FS(dk, FM(F[k - k0], xv));
          *x = xv;
          if (k == m - 1) xlast = xv;
        }
        // "Line" boundary columns from the copied columns 1 and n - 2
        if (k0 == 0) coef[lane] = FS(FM(2.0f, coef[ld + lane]), xv);  // xv == x_0 here
        if (k1 == m) coef[(n - 1) * ld + lane] = FS(FM(2.0f, coef[(n - 2) * ld + lane]), xlast);
      }
      __syncwarp();
      row_tile_store(T, coef + (k0 + 2) * ld, ld, nrow, (int)(k1 - k0), lane);
      __syncwarp();
    }
  }
}

template <int PASS>
__global__ void __launch_bounds__(32 * BSC_WARPS) b_bspline_row_kernel(const BPair* __restrict__ bp, int npairs,
                                                                      int64_t witems, float* dbuf, int64_t qtot) {
  extern __shared__ float bsc_tile[];
  const int img = blockIdx.y, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* T = bsc_tile + warp * BS_WSTRIDE;
  float* F = T + BS_WTILE;
  for (int64_t t = (int64_t)blockIdx.x * BSC_WARPS + warp; t < witems; t += (int64_t)gridDim.x * BSC_WARPS) {
    const BPair& b = bp[bp_find<&BPair::wrow>(bp, npairs, t)];
    if (!b.deforms) continue;  // uniform across the warp
    const int64_t l = t - b.wrow;
    if (l >= (b.nr + 2 + 31) / 32 * b_nseg(b.nc + 2)) continue;
    bs_row_item<PASS>(img ? b.coefB : b.coefA, dbuf + (int64_t)img * qtot + b.qoff, b.nr, b.nc, b.cpr, b.ivr, l, T, F,
                      lane);
  }
}

// The same passes over the two frames of one pair (blockIdx.y: frame), for
// the single-pair schedule and the hooks.
struct PrefFrames {
  const float* img[2];
  float* coef[2];
  float* d[2];
};

template <int PASS>
__global__ void __launch_bounds__(32 * BSC_WARPS) bspline_col_tiles_kernel(PrefFrames P, int64_t nr, int64_t nc,
                                                                          const float* cpc, const float* ivc,
                                                                          int64_t witems) {
  extern __shared__ float bsc_tile[];
  const int img = blockIdx.y, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* T = bsc_tile + warp * BS_WSTRIDE;
  float* F = T + BS_WTILE;
  for (int64_t t = (int64_t)blockIdx.x * BSC_WARPS + warp; t < witems; t += (int64_t)gridDim.x * BSC_WARPS)
    bs_col_item<PASS>(P.img[img], P.coef[img], P.d[img], nr, nc, cpc, ivc, t, T, F, lane);
}

template <int PASS>
__global__ void __launch_bounds__(32 * BSC_WARPS) bspline_row_tiles_kernel(PrefFrames P, int64_t nr, int64_t nc,
                                                                          const float* cpr, const float* ivr,
                                                                          int64_t witems) {
  extern __shared__ float bsc_tile[];
  const int img = blockIdx.y, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  float* T = bsc_tile + warp * BS_WSTRIDE;
  float* F = T + BS_WTILE;
  for (int64_t t = (int64_t)blockIdx.x * BSC_WARPS + warp; t < witems; t += (int64_t)gridDim.x * BSC_WARPS)
    bs_row_item<PASS>(P.coef[img], P.d[img], nr, nc, cpr, ivr, t, T, F, lane);
}

static cudaError_t set_tile_smem() {
  static bool done = false;
  if (done) return cudaSuccess;
  for (cudaError_t e : {cudaFuncSetAttribute(b_bspline_col_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)BSC_SMEM),
                        cudaFuncSetAttribute(b_bspline_col_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)BSC_SMEM),
                        cudaFuncSetAttribute(b_bspline_row_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)BSC_SMEM),
                        cudaFuncSetAttribute(b_bspline_row_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)BSC_SMEM),
                        cudaFuncSetAttribute(bspline_col_tiles_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)BSC_SMEM),
                        cudaFuncSetAttribute(bspline_col_tiles_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)BSC_SMEM),
                        cudaFuncSetAttribute(bspline_row_tiles_kernel<0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)BSC_SMEM),
                        cudaFuncSetAttribute(bspline_row_tiles_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)BSC_SMEM)})
    if (e != cudaSuccess) return e;
  done = true;
  return cudaSuccess;
}

static unsigned tile_blocks(int64_t witems) {
  int64_t blocks = (witems + BSC_WARPS - 1) / BSC_WARPS;
  if (blocks > 148 * 8) blocks = 148 * 8;
  return (unsigned)(blocks < 1 ? 1 : blocks);
}

cudaError_t launch_prefilter_pair(const float* imgA, const float* imgB, int64_t nr, int64_t nc, float* coefA,
                                  float* coefB, float* dbuf, const float* cpc, const float* ivc, const float* cpr,
                                  const float* ivr, cudaStream_t s) {
  cudaError_t e = set_tile_smem();
  if (e != cudaSuccess) return e;
  const int64_t ld = nr + 2, q = ld * (nc + 2);
  const PrefFrames P{{imgA, imgB}, {coefA, coefB}, {dbuf, dbuf + q}};
  const int64_t wc = (nc + 31) / 32 * b_nseg(ld), wr = (ld + 31) / 32 * b_nseg(nc + 2);
  bspline_col_tiles_kernel<0><<<dim3(tile_blocks(wc), 2), 32 * BSC_WARPS, BSC_SMEM, s>>>(P, nr, nc, cpc, ivc, wc);
  bspline_col_tiles_kernel<1><<<dim3(tile_blocks(wc), 2), 32 * BSC_WARPS, BSC_SMEM, s>>>(P, nr, nc, cpc, ivc, wc);
  if (nc + 2 < 4)  // padding columns 0 and nc + 1 stay zero: no row to solve writes them
    for (float* c : {coefA, coefB}) {
      e = cudaMemsetAsync(c, 0, ld * sizeof(float), s);
      if (e == cudaSuccess) e = cudaMemsetAsync(c + (nc + 1) * ld, 0, ld * sizeof(float), s);
      if (e != cudaSuccess) return e;
    }
  bspline_row_tiles_kernel<0><<<dim3(tile_blocks(wr), 2), 32 * BSC_WARPS, BSC_SMEM, s>>>(P, nr, nc, cpr, ivr, wr);
  bspline_row_tiles_kernel<1><<<dim3(tile_blocks(wr), 2), 32 * BSC_WARPS, BSC_SMEM, s>>>(P, nr, nc, cpr, ivr, wr);
  return cudaGetLastError();
}

cudaError_t launch_b_prefilter(const BPair* bp, int npairs, int64_t qtot, int64_t wcol_tot, int64_t wrow_tot,
                               float* dbuf, cudaStream_t s) {
  if (qtot <= 0) return cudaSuccess;
  cudaError_t e = set_tile_smem();
  if (e != cudaSuccess) return e;
  if (wcol_tot > 0) {
    int64_t blocks = (wcol_tot + BSC_WARPS - 1) / BSC_WARPS;
    if (blocks > 148 * 8) blocks = 148 * 8;
    b_bspline_col_kernel<0><<<dim3((unsigned)blocks, 2), 32 * BSC_WARPS, BSC_SMEM, s>>>(bp, npairs, wcol_tot, dbuf, qtot);
    b_bspline_col_kernel<1><<<dim3((unsigned)blocks, 2), 32 * BSC_WARPS, BSC_SMEM, s>>>(bp, npairs, wcol_tot, dbuf, qtot);
  }
  b_pad_cols_kernel<<<dim3(npairs < 148 ? npairs : 148, 2), 128, 0, s>>>(bp, npairs);
  if (wrow_tot > 0) {
    int64_t blocks = (wrow_tot + BSC_WARPS - 1) / BSC_WARPS;
    if (blocks > 148 * 8) blocks = 148 * 8;
    b_bspline_row_kernel<0><<<dim3((unsigned)blocks, 2), 32 * BSC_WARPS, BSC_SMEM, s>>>(bp, npairs, wrow_tot, dbuf, qtot);
    b_bspline_row_kernel<1><<<dim3((unsigned)blocks, 2), 32 * BSC_WARPS, BSC_SMEM, s>>>(bp, npairs, wrow_tot, dbuf, qtot);
  }
  return cudaGetLastError();
}

// the predictor grid of sweep `it`: the previous slot's grid in sweep 1,
// this slot's grid afterwards
__device__ __forceinline__ PredGrid b_pred_grid(const BPair& b, int it) {
  PredGrid g;
  if (it == 1) {
    g.gny = b.pgny; g.gnx = b.pgnx; g.y0 = b.py0; g.ysp = b.pysp; g.x0 = b.px0; g.xsp = b.pxsp;
  } else {
    g.gny = b.ny; g.gnx = b.nx; g.y0 = b.gy0; g.ysp = b.gysp; g.x0 = b.gx0; g.xsp = b.gxsp;
  }
  return g;
}

// Start of sweep `it`: the node values of the predictor (zero without one),
// NaN uncertainties at the start of the slot, and the sweep count of pairs
// in their final pass.
__global__ void b_sweep_begin_kernel(const BPair* __restrict__ bp, int npairs, const int32_t* __restrict__ done, int it,
                                     int64_t gtot, const float* __restrict__ pu, const float* __restrict__ pv, float* u,
                                     float* v, float* uncu, float* uncv, int32_t* sweeps, int32_t* slot_sweeps) {
  B_STRIDE(k, gtot) {
    const int p = bp_find<&BPair::coff>(bp, npairs, k);
    const BPair& b = bp[p];
    const int64_t l = k - b.coff;
    if (!bp_live(b, it, done, p) || l >= (int64_t)b.ny * b.nx) continue;
    const int64_t id = b.goff + l;
    if (l == 0) {
      slot_sweeps[p] = it;
      if (b.is_final) sweeps[p] = it;
    }
    if (it == 1) {
      uncu[id] = __int_as_float(0x7fc00000);
      uncv[id] = __int_as_float(0x7fc00000);
    }
    if (it > 1 || b.has_pred0) {
      const PredGrid g = b_pred_grid(b, it);
      const int gi = (int)(l % b.ny), gj = (int)(l / b.ny);
      const float y = FA(b.gy0, FM((float)gi, b.gysp)), x = FA(b.gx0, FM((float)gj, b.gxsp));
      u[id] = bilinear(pu + b.goff, g, y, x);
      v[id] = bilinear(pv + b.goff, g, y, x);
    } else {
      u[id] = 0.f;
      v[id] = 0.f;
    }
  }
}

cudaError_t launch_b_sweep_begin(const BPair* bp, int npairs, const int32_t* done, int it, int64_t gtot,
                                 const float* pu, const float* pv, float* u, float* v, float* uncu, float* uncv,
                                 int32_t* sweeps, int32_t* slot_sweeps, cudaStream_t s) {
  if (gtot <= 0) return cudaSuccess;
  b_sweep_begin_kernel<<<b_blocks(gtot), 256, 0, s>>>(bp, npairs, done, it, gtot, pu, pv, u, v, uncu, uncv, sweeps,
                                                      slot_sweeps);
  return cudaGetLastError();
}

// Four consecutive pixels (a quad; pairs start on multiples of 4 in the
// slot-compact index and in the warped arrays) per thread: the pair lookup,
// the pair's fields, the pixel index division and the predictor's column
// interpolation are done once per quad (again only where the quad wraps to
// the next column), and a full quad is stored as one 16-byte vector.
__global__ void __launch_bounds__(256) b_deform_kernel(const BPair* __restrict__ bp, int npairs,
                                                       const int32_t* __restrict__ done, int it, int64_t ptot,
                                                       const float* __restrict__ pu, const float* __restrict__ pv) {
  B_STRIDE(t, (ptot + 3) / 4) {
    const int64_t k = 4 * t;
    const int p = bp_find<&BPair::pcoff>(bp, npairs, k);
    const BPair& b = bp[p];
    const int64_t l0 = k - b.pcoff, npx = b.nr * b.nc;
    if (!bp_live(b, it, done, p) || !(it > 1 || b.has_pred0) || !b.deforms || l0 >= npx) continue;
    const PredGrid g = b_pred_grid(b, it);
    const float* fu = pu + b.goff;
    const float* fv = pv + b.goff;
    const int64_t nr = b.nr, nc = b.nc;
    int64_t r, c;
    if (npx <= 0x7fffffff) {  // 32-bit division when the pair's pixel index fits
      r = (uint32_t)l0 % (uint32_t)nr;
      c = (uint32_t)l0 / (uint32_t)nr;
    } else {
      r = l0 % nr;
      c = l0 / nr;
    }
    float wa[4], wb[4];
    int ix = 0;
    float dx = 0.f;
    int64_t cx = -1;  // column whose x interpolation (ix, dx) is held
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      wa[j] = wb[j] = 0.f;
      if (l0 + j < npx) {
        int64_t rj = r + j, cj = c;
        while (rj >= nr) {  // the quad wraps to the next column
          rj -= nr;
          ++cj;
        }
        const float R = (float)(rj + 1), Cc = (float)(cj + 1);
        if (cj != cx) {
          lin_axis(Cc, g.x0, g.xsp, g.gnx, ix, dx);
          cx = cj;
        }
        int iy;
        float dy;
        lin_axis(R, g.y0, g.ysp, g.gny, iy, dy);
        const float du2 = FM(bilinear_at(fu, g, iy, dy, ix, dx), 0.5f);
        const float dv2 = FM(bilinear_at(fv, g, iy, dy, ix, dx), 0.5f);
        wa[j] = bspline_eval(b.coefA, nr, nc, FS(R, dv2), FS(Cc, du2));
        wb[j] = bspline_eval(b.coefB, nr, nc, FA(R, dv2), FA(Cc, du2));
      }
    }
    if (l0 + 3 < npx) {
      *reinterpret_cast<float4*>(b.warpA + l0) = make_float4(wa[0], wa[1], wa[2], wa[3]);
      *reinterpret_cast<float4*>(b.warpB + l0) = make_float4(wb[0], wb[1], wb[2], wb[3]);
    } else {
#pragma unroll
      for (int j = 0; j < 4; ++j)
        if (l0 + j < npx) {
          b.warpA[l0 + j] = wa[j];
          b.warpB[l0 + j] = wb[j];
        }
    }
  }
}

cudaError_t launch_b_deform(const BPair* bp, int npairs, const int32_t* done, int it, int64_t ptot, const float* pu,
                            const float* pv, cudaStream_t s) {
  if (ptot <= 0) return cudaSuccess;
  b_deform_kernel<<<b_blocks((ptot + 3) / 4, 32), 256, 0, s>>>(bp, npairs, done, it, ptot, pu, pv);
  return cudaGetLastError();
}

}  // namespace hh
