// Batched dense equilibrated LU with FP64 residual refinement.
//
// Replaces the reference's cuBLAS dgetrfBatched/dgetrsBatched path
// (PyMHM 1.3.2 src/pymhm/execution/cuda.py:114-288, BatchedFactorization):
//   * row then column max-equilibration, zero row/column rejection (:201-211)
//   * partial-pivoting LU, exact-zero pivot -> "singular pivot" (:127-131)
//   * rank test min |u_ii| <= eps * n * max |LU| -> "rank deficient" (:132-135)
//   * solve with the equilibrated factors, FP64 residual on the original matrix,
//     at most two corrections, columnwise acceptance (:230-255)
// One CTA owns one matrix.  The working matrix lives in shared memory when it fits
// (n <= 160, unblocked right-looking LU).  Up to n = 640 it lives in the caller's
// `factors` array (L2-resident) and is factored in blocks of 32 columns: the panel
// in shared memory with partial pivoting, the trailing matrix updated in 64 x 64
// tiles.  Larger n use the unblocked algorithm on `factors`.  Solves keep the
// right-hand sides in shared memory and read the factors in 32-row chunks (one
// batch of loads per chunk) when they fit, else one warp per column.
#include <cmath>

#include "mhm_common.cuh"

namespace mhm {
namespace {

constexpr int kLuThreads = 256;

__global__ void __launch_bounds__(kLuThreads) batched_factor_kernel(
    int n, const double* __restrict__ mats, double* __restrict__ factors, int32_t* __restrict__ piv,
    double* __restrict__ rs, double* __restrict__ cs, int32_t* __restrict__ status, int in_smem) {
  extern __shared__ __align__(16) double sm[];
  __shared__ double red[32];
  __shared__ int sp;
  const int m = blockIdx.x, tid = threadIdx.x;
  const size_t nn = (size_t)n * n;
  const double* A = mats + nn * m;
  double* F = factors + nn * m;
  double* L = in_smem ? sm : F;
  double* rsc = rs + (size_t)n * m;
  double* csc = cs + (size_t)n * m;
  int st = MHM_CELL_OK;
  // row scaling
  int zero_row = 0, nonfinite = 0;
  for (int i = tid; i < n; i += blockDim.x) {
    double mx = 0.0;
    for (int j = 0; j < n; ++j) {
      const double v = A[(size_t)i * n + j];
      if (!isfinite(v)) nonfinite = 1;
      mx = fmax(mx, fabs(v));
    }
    if (mx == 0.0) zero_row = 1;
    rsc[i] = (mx > 0.0) ? 1.0 / mx : 0.0;
  }
  nonfinite = __syncthreads_or(nonfinite);
  zero_row = __syncthreads_or(zero_row);
  if (nonfinite) st = MHM_CELL_NONFINITE;
  else if (zero_row) st = MHM_CELL_ZERO_ROW;
  // column scaling of the row-scaled matrix
  int zero_col = 0;
  for (int j = tid; j < n; j += blockDim.x) {
    double mx = 0.0;
    for (int i = 0; i < n; ++i) mx = fmax(mx, fabs(A[(size_t)i * n + j] * rsc[i]));
    if (mx == 0.0) zero_col = 1;
    csc[j] = (mx > 0.0) ? 1.0 / mx : 0.0;
  }
  zero_col = __syncthreads_or(zero_col);
  if (st == MHM_CELL_OK && zero_col) st = MHM_CELL_ZERO_COLUMN;
  for (size_t idx = tid; idx < nn; idx += blockDim.x) {
    const int i = (int)(idx / n), j = (int)(idx % n);
    L[idx] = A[idx] * rsc[i] * csc[j];
  }
  __syncthreads();
  // right-looking LU with partial pivoting
  if (st == MHM_CELL_OK) {
    for (int k = 0; k < n; ++k) {
      // pivot search: warp 0
      if (tid < 32) {
        double best = -1.0;
        int bi = k;
        for (int i = k + tid; i < n; i += 32) {
          const double v = fabs(L[(size_t)i * n + k]);
          if (v > best) { best = v; bi = i; }
        }
        for (int o = 16; o > 0; o >>= 1) {
          const double ob = __shfl_xor_sync(0xffffffffu, best, o);
          const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
          if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        if (tid == 0) sp = bi;
      }
      __syncthreads();
      const int p = sp;
      if (tid == 0) piv[(size_t)m * n + k] = p;
      if (p != k)
        for (int j = tid; j < n; j += blockDim.x) {
          const double tmp = L[(size_t)k * n + j];
          L[(size_t)k * n + j] = L[(size_t)p * n + j];
          L[(size_t)p * n + j] = tmp;
        }
      __syncthreads();
      const double d = L[(size_t)k * n + k];
      if (d == 0.0) { st = MHM_CELL_SINGULAR_PIVOT; break; }
      const double inv = 1.0 / d;
      for (int i = k + 1 + tid; i < n; i += blockDim.x) L[(size_t)i * n + k] *= inv;
      __syncthreads();
      const int rem = n - k - 1;
      for (int idx = tid; idx < rem * rem; idx += blockDim.x) {
        const int i = k + 1 + idx / rem, j = k + 1 + idx % rem;
        L[(size_t)i * n + j] = fma(-L[(size_t)i * n + k], L[(size_t)k * n + j], L[(size_t)i * n + j]);
      }
      __syncthreads();
    }
  }
  if (st == MHM_CELL_OK) {
    double dmin = 1e300, amax = 0.0;
    for (int i = tid; i < n; i += blockDim.x) dmin = fmin(dmin, fabs(L[(size_t)i * n + i]));
    for (size_t idx = tid; idx < nn; idx += blockDim.x) amax = fmax(amax, fabs(L[idx]));
    dmin = block_min(dmin, red);
    amax = block_max(amax, red);
    if (dmin <= 2.220446049250313e-16 * n * amax) st = MHM_CELL_RANK_DEFICIENT;
  }
  __syncthreads();
  if (in_smem)
    for (size_t idx = tid; idx < nn; idx += blockDim.x) F[idx] = L[idx];
  if (tid == 0) status[m] = st;
}

// y = col_scale .* U^-1 L^-1 P (row_scale .* r) for one column, one warp.
__device__ void lu_apply_col(int n, int nrhs, const double* LU, const int32_t* piv, const double* rsc,
                             const double* csc, double* v /* column, stride nrhs */, int lane) {
  if (lane == 0) {
    for (int i = 0; i < n; ++i) v[(size_t)i * nrhs] *= rsc[i];
    for (int k = 0; k < n; ++k) {
      const int p = piv[k];
      if (p != k) {
        const double tmp = v[(size_t)k * nrhs];
        v[(size_t)k * nrhs] = v[(size_t)p * nrhs];
        v[(size_t)p * nrhs] = tmp;
      }
    }
  }
  __syncwarp();
  for (int i = 0; i < n; ++i) {  // unit lower
    double acc = 0.0;
    for (int j = lane; j < i; j += 32) acc = fma(LU[(size_t)i * n + j], v[(size_t)j * nrhs], acc);
    acc = warp_sum(acc);
    if (lane == 0) v[(size_t)i * nrhs] -= acc;
    __syncwarp();
  }
  for (int i = n - 1; i >= 0; --i) {  // upper
    double acc = 0.0;
    for (int j = i + 1 + lane; j < n; j += 32) acc = fma(LU[(size_t)i * n + j], v[(size_t)j * nrhs], acc);
    acc = warp_sum(acc);
    if (lane == 0) v[(size_t)i * nrhs] = (v[(size_t)i * nrhs] - acc) / LU[(size_t)i * n + i];
    __syncwarp();
  }
  for (int i = lane; i < n; i += 32) v[(size_t)i * nrhs] *= csc[i];
  __syncwarp();
}

__global__ void __launch_bounds__(kLuThreads) batched_solve_kernel(
    int n, int nrhs, const double* __restrict__ mats, const double* __restrict__ factors,
    const int32_t* __restrict__ piv, const double* __restrict__ rs, const double* __restrict__ cs,
    const double* __restrict__ rhs, double* __restrict__ x, double* __restrict__ work, double rtol,
    double atol, int max_refine, int32_t* __restrict__ status) {
  __shared__ int ok_all;
  const int m = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
  const int nw = blockDim.x >> 5;
  const size_t nn = (size_t)n * n, nb = (size_t)n * nrhs;
  const double* A = mats + nn * m;
  const double* LU = factors + nn * m;
  const int32_t* pv = piv + (size_t)n * m;
  const double* rsc = rs + (size_t)n * m;
  const double* csc = cs + (size_t)n * m;
  const double* B = rhs + nb * m;
  double* X = x + nb * m;
  double* R = work + nb * m;
  if (status[m] != MHM_CELL_OK) return;
  int nonfinite = 0;
  for (size_t idx = tid; idx < nb; idx += blockDim.x) {
    if (!isfinite(B[idx])) nonfinite = 1;
    X[idx] = B[idx];
  }
  if (__syncthreads_or(nonfinite)) {
    if (tid == 0) status[m] = MHM_CELL_NONFINITE;
    return;
  }
  for (int c = wid; c < nrhs; c += nw) lu_apply_col(n, nrhs, LU, pv, rsc, csc, X + c, lane);
  __syncthreads();
  for (int pass = 0; pass <= max_refine; ++pass) {
    // residual R = B - A X and columnwise acceptance with max-scaling
    if (tid == 0) ok_all = 1;
    __syncthreads();
    int bad = 0;
    for (size_t idx = tid; idx < nb; idx += blockDim.x) {
      const int i = (int)(idx / nrhs), c = (int)(idx % nrhs);
      double hi = B[idx], lo = 0.0;
      for (int j = 0; j < n; ++j) dd_fma(hi, lo, -A[(size_t)i * n + j], X[(size_t)j * nrhs + c]);
      R[idx] = hi + lo;
      if (!isfinite(X[idx])) bad = 1;
    }
    if (__syncthreads_or(bad)) {
      if (tid == 0) status[m] = MHM_CELL_NONFINITE;
      return;
    }
    for (int c = wid; c < nrhs; c += nw) {
      double bmax = 0.0;
      for (int i = lane; i < n; i += 32) bmax = fmax(bmax, fabs(B[(size_t)i * nrhs + c]));
      bmax = warp_max(bmax);
      double scale = fmax(atol, bmax);
      if (!(scale > 0.0)) scale = 1.0;
      double r2 = 0.0, b2 = 0.0;
      for (int i = lane; i < n; i += 32) {
        const double rv = R[(size_t)i * nrhs + c] / scale, bv = B[(size_t)i * nrhs + c] / scale;
        r2 += rv * rv;
        b2 += bv * bv;
      }
      r2 = warp_sum(r2);
      b2 = warp_sum(b2);
      const double limit = fmax(atol / scale, rtol * sqrt(b2));
      if (lane == 0 && !(sqrt(r2) <= limit)) ok_all = 0;
    }
    __syncthreads();
    if (ok_all) return;
    if (pass == max_refine) break;
    for (int c = wid; c < nrhs; c += nw) lu_apply_col(n, nrhs, LU, pv, rsc, csc, R + c, lane);
    __syncthreads();
    for (size_t idx = tid; idx < nb; idx += blockDim.x) X[idx] += R[idx];
    __syncthreads();
  }
  if (tid == 0) status[m] = MHM_CELL_RESIDUAL;
}


constexpr int kPanel = 32;
constexpr int kPanelStride = kPanel + 1;  // odd: a column of the panel spans all banks
constexpr int kBlockedMaxN = 640;
constexpr int kListed = 1 << 30;  // marks a listed position in the swap composition

// D = A B + D on one 8 x 8 x 4 FP64 tensor-core step (fragments as documented at the
// call site).
__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Row then column max-equilibration of A into F (cuda.py:201-211); the status of
// zero rows / columns and non-finite entries.
__device__ int equilibrate(int n, const double* A, double* F, double* rsc, double* csc) {
  int st = MHM_CELL_OK;
  const int tid = threadIdx.x;
  int zero_row = 0, nonfinite = 0;
  // row maxima: a warp per row, lanes over the columns (coalesced)
  const int lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  for (int i = wid; i < n; i += nw) {
    double mx = 0.0;
    for (int j = lane; j < n; j += 32) {
      const double v = A[(size_t)i * n + j];
      if (!isfinite(v)) nonfinite = 1;
      mx = fmax(mx, fabs(v));
    }
    mx = warp_max(mx);
    if (lane == 0) {
      if (mx == 0.0) zero_row = 1;
      rsc[i] = (mx > 0.0) ? 1.0 / mx : 0.0;
    }
  }
  nonfinite = __syncthreads_or(nonfinite);
  zero_row = __syncthreads_or(zero_row);
  if (nonfinite) st = MHM_CELL_NONFINITE;
  else if (zero_row) st = MHM_CELL_ZERO_ROW;
  int zero_col = 0;
  for (int j = tid; j < n; j += blockDim.x) {
    double mx = 0.0;
#pragma unroll 8
    for (int i = 0; i < n; ++i) mx = fmax(mx, fabs(A[(size_t)i * n + j] * rsc[i]));
    if (mx == 0.0) zero_col = 1;
    csc[j] = (mx > 0.0) ? 1.0 / mx : 0.0;
  }
  zero_col = __syncthreads_or(zero_col);
  if (st == MHM_CELL_OK && zero_col) st = MHM_CELL_ZERO_COLUMN;
  // a warp per row (no index division)
  for (int i = wid; i < n; i += nw) {
    const double ri = rsc[i];
    for (int j = lane; j < n; j += 32) F[(size_t)i * n + j] = A[(size_t)i * n + j] * ri * csc[j];
  }
  __syncthreads();
  return st;
}

// Blocked right-looking LU with partial pivoting of one matrix held in `factors`
// (32 < n <= 640).  Per panel of 32 columns: (a) the panel rows kb..n-1 are factored
// in shared memory, pivots by first maximum as the unblocked kernel; (b) the panel's
// row swaps are applied to the other columns, a thread per column, in order;
// (c) U12 = L11^-1 A12, a thread per column; (d) A22 -= L21 U12 on the FP64 tensor
// cores, a warp per 8-row block, without a CTA barrier inside.
// With desc (ragged batches), CTA m factors the matrix desc[m] describes (its order,
// offsets and status word); matrices larger than max_n get MHM_CELL_SIZE.
__global__ void __launch_bounds__(kLuThreads) batched_factor_blocked_kernel(
    int n_uniform, const double* __restrict__ mats, double* __restrict__ factors, int32_t* __restrict__ piv,
    double* __restrict__ rs, double* __restrict__ cs, int32_t* __restrict__ status,
    const mhm_ragged_matrix* __restrict__ desc, int max_n) {
  extern __shared__ __align__(16) double sm[];
  double* Pn = sm;                                   // (n, kPanelStride) panel
  __shared__ double red[32];
  __shared__ double wbest[32];
  __shared__ int wrow[32];
  __shared__ int sperm[kPanel];
  __shared__ int apos[2 * kPanel], asrc[2 * kPanel];  // rows the panel's swaps move: position <- source
  __shared__ int naff;
  __shared__ int srcrow[kBlockedMaxN];
  const int m = blockIdx.x, tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  int n = n_uniform, sidx = m;
  size_t moff = (size_t)n_uniform * n_uniform * m, voff = (size_t)n_uniform * m;
  if (desc) {
    const mhm_ragged_matrix d = desc[m];
    n = d.n;
    sidx = d.slot;
    moff = (size_t)d.mat_off;
    voff = (size_t)d.vec_off;
    if (n < 1 || n > max_n) {
      if (tid == 0) status[sidx] = MHM_CELL_SIZE;
      return;
    }
  }
  double* F = factors + moff;
  int st = equilibrate(n, mats + moff, F, rs + voff, cs + voff);
  for (int kb = 0; kb < n && st == MHM_CELL_OK; kb += kPanel) {
    const int w = min(kPanel, n - kb), rows = n - kb;
    for (int r = wid; r < rows; r += nw)
      if (lane < w) Pn[r * kPanelStride + lane] = F[(size_t)(kb + r) * n + kb + lane];
    __syncthreads();
    for (int c = 0; c < w; ++c) {
      // pivot search on column c; the previous column's multipliers are scaled in the
      // same phase (its elimination ended at the last barrier; columns differ)
      if (c > 0) {
        const double pinv = 1.0 / Pn[(c - 1) * kPanelStride + (c - 1)];
        for (int r = c + tid; r < rows; r += blockDim.x) Pn[r * kPanelStride + c - 1] *= pinv;
      }
      double best = -1.0;
      int bi = c;
      for (int r = c + tid; r < rows; r += blockDim.x) {
        const double v = fabs(Pn[r * kPanelStride + c]);
        if (v > best) { best = v; bi = r; }
      }
      for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_xor_sync(0xffffffffu, best, o);
        const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
        if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
      }
      if (lane == 0) { wbest[wid] = best; wrow[wid] = bi; }
      __syncthreads();
      // every thread reduces the warps' candidates (first maximum) itself
      int p = wrow[0];
      {
        double b = wbest[0];
        for (int q = 1; q < nw; ++q)
          if (wbest[q] > b || (wbest[q] == b && wrow[q] < p)) { b = wbest[q]; p = wrow[q]; }
      }
      if (tid == 0) sperm[c] = p;
      if (p != c)
        for (int j = tid; j < w; j += blockDim.x) {
          const double t = Pn[c * kPanelStride + j];
          Pn[c * kPanelStride + j] = Pn[p * kPanelStride + j];
          Pn[p * kPanelStride + j] = t;
        }
      __syncthreads();
      const double d = Pn[c * kPanelStride + c];
      if (d == 0.0) { st = MHM_CELL_SINGULAR_PIVOT; break; }
      const double inv = 1.0 / d;
      {
        // every (row below the pivot, panel column right of it) pair is independent (the
        // multiplier l = a_rc / d formed where used; column c is scaled in the next
        // column's first phase): a warp per row, a lane per panel column, four rows'
        // loads before their stores
        const int j = c + 1 + lane;
        const bool jv = j < w;
        const double u = jv ? Pn[c * kPanelStride + j] : 0.0;
        for (int r = c + 1 + wid; r < rows; r += 4 * nw) {
          double l[4], a[4];
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int rk = r + k * nw;
            const bool ok = rk < rows && jv;
            l[k] = ok ? Pn[rk * kPanelStride + c] * inv : 0.0;
            a[k] = ok ? Pn[rk * kPanelStride + j] : 0.0;
          }
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            const int rk = r + k * nw;
            if (rk < rows && jv) Pn[rk * kPanelStride + j] = fma(-l[k], u, a[k]);
          }
        }
      }
      __syncthreads();
    }
    if (st == MHM_CELL_OK) {  // the last column's multipliers
      const double pinv = 1.0 / Pn[(w - 1) * kPanelStride + (w - 1)];
      for (int r = w + tid; r < rows; r += blockDim.x) Pn[r * kPanelStride + w - 1] *= pinv;
      __syncthreads();
    }
    if (st != MHM_CELL_OK) break;
    for (int r = wid; r < rows; r += nw)
      if (lane < w) F[(size_t)(kb + r) * n + kb + lane] = Pn[r * kPanelStride + lane];
    for (int c = tid; c < w; c += blockDim.x) piv[voff + kb + c] = kb + sperm[c];
    // compose the panel's swaps: srcrow[r] = the panel row that ends at position r; the
    // moved positions (at most 2 w) are listed with their sources
    for (int r = tid; r < rows; r += blockDim.x) srcrow[r] = r;
    __syncthreads();
    if (tid == 0) {
      for (int c = 0; c < w; ++c) {
        const int p = sperm[c];
        if (p != c) {
          const int t = srcrow[c];
          srcrow[c] = srcrow[p];
          srcrow[p] = t;
        }
      }
      int cnt = 0;
      for (int c = 0; c < w; ++c)
        if (srcrow[c] != c) {
          apos[cnt] = c;
          asrc[cnt] = srcrow[c];
          ++cnt;
        }
      for (int c = 0; c < w; ++c) {
        const int p = sperm[c];
        if (p >= w && !(srcrow[p] & kListed) && srcrow[p] != p) {
          apos[cnt] = p;
          asrc[cnt] = srcrow[p];
          srcrow[p] |= kListed;
          ++cnt;
        }
      }
      naff = cnt;
    }
    __syncthreads();
    // the other columns: every moved entry of a column is loaded before any is stored
    for (int j = tid; j < n - w; j += blockDim.x) {
      const int col = j < kb ? j : j + w;
      double v[2 * kPanel];
#pragma unroll
      for (int k = 0; k < 2 * kPanel; ++k) v[k] = k < naff ? F[(size_t)(kb + asrc[k]) * n + col] : 0.0;
#pragma unroll
      for (int k = 0; k < 2 * kPanel; ++k)
        if (k < naff) F[(size_t)(kb + apos[k]) * n + col] = v[k];
    }
    __syncthreads();
    for (int j = kb + w + tid; j < n; j += blockDim.x) {
      double x[kPanel];
#pragma unroll
      for (int r = 0; r < kPanel; ++r) x[r] = r < w ? F[(size_t)(kb + r) * n + j] : 0.0;
#pragma unroll
      for (int r = 1; r < kPanel; ++r)
#pragma unroll
        for (int q = 0; q < r; ++q) x[r] = fma(-Pn[r * kPanelStride + q], x[q], x[r]);
#pragma unroll
      for (int r = 0; r < kPanel; ++r)
        if (r < w) F[(size_t)(kb + r) * n + j] = x[r];
    }
    __syncthreads();
    const int m2 = n - kb - w, base = kb + w;
    // A22 -= L21 U12 on the tensor cores with no CTA barrier inside: warp wid takes the
    // 8-row blocks wid, wid + nw, ... of the trailing matrix and walks its columns in
    // blocks of 64 (eight 8 x 8 outputs, FP64 mma.sync m8n8k4 over the panel's columns
    // in steps of 4).  A = -L21 comes from the panel in shared memory once per row
    // block; all B = U12 fragments of a column block are loaded from global memory (L2)
    // before its tensor-core steps, so their latency is paid once.  Fragments:
    // A[lane/4][lane%4], B[lane%4][lane/4], C[lane/4][2 (lane%4) + {0, 1}]; panel
    // columns past w are masked to 0.
    const int fr = lane >> 2, fc = lane & 3;
    const int ksteps = (w + 3) >> 2;
    for (int rb = 8 * wid; rb < m2; rb += 8 * nw) {
      const int i = rb + fr;  // this lane's A / C row in the trailing block
      const int prow = w + (i < m2 ? i : m2 - 1);  // panel row of L21 (clamped rows are not stored)
      double av[kPanel / 4];
#pragma unroll
      for (int s = 0; s < kPanel / 4; ++s) {
        const int q = 4 * s + fc;
        av[s] = q < w ? -Pn[prow * kPanelStride + q] : 0.0;
      }
      for (int tj = 0; tj < m2; tj += 64) {
        double bv[kPanel / 4][8];
#pragma unroll
        for (int s = 0; s < kPanel / 4; ++s) {
          const int q = 4 * s + fc;
#pragma unroll
          for (int b = 0; b < 8; ++b) {
            const int col = tj + 8 * b + fr;
            bv[s][b] = (q < w && col < m2) ? F[(size_t)(kb + q) * n + base + col] : 0.0;
          }
        }
        double acc[8][2];
#pragma unroll
        for (int b = 0; b < 8; ++b)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int j = tj + 8 * b + 2 * fc + e;
            acc[b][e] = (i < m2 && j < m2) ? F[(size_t)(base + i) * n + base + j] : 0.0;
          }
#pragma unroll
        for (int s = 0; s < kPanel / 4; ++s) {
          if (s >= ksteps) break;
#pragma unroll
          for (int b = 0; b < 8; ++b) dmma_8x8x4(acc[b][0], acc[b][1], av[s], bv[s][b]);
        }
        if (i < m2) {
#pragma unroll
          for (int b = 0; b < 8; ++b)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int j = tj + 8 * b + 2 * fc + e;
              if (j < m2) F[(size_t)(base + i) * n + base + j] = acc[b][e];
            }
        }
      }
    }
    __syncthreads();
  }
  if (st == MHM_CELL_OK) {
    double dmin = 1e300, amax = 0.0;
    for (int i = tid; i < n; i += blockDim.x) dmin = fmin(dmin, fabs(F[(size_t)i * n + i]));
    for (int i = wid; i < n; i += nw)
      for (int j = lane; j < n; j += 32) amax = fmax(amax, fabs(F[(size_t)i * n + j]));
    dmin = block_min(dmin, red);
    amax = block_max(amax, red);
    if (dmin <= 2.220446049250313e-16 * n * amax) st = MHM_CELL_RANK_DEFICIENT;
  }
  if (tid == 0) status[sidx] = st;
}

// ---------------------------------------------------------------------------------
// Large orders (640 < n <= kLargeMaxN): blocked right-looking LU of one matrix per CTA
// held in `factors` (HBM), with the row search of each column restricted to the
// panel's diagonal window: rows kb .. kb + w of the panel kb .. kb + w - 1 (w <= 32
// columns, one row past the block).  The local systems this serves are bordered
// positive semi-definite matrices [[A, c], [c^T, 0]] (A with the constants as its
// kernel, c^T 1 != 0) padded with identity rows.  For such a matrix every leading
// block of node rows is positive definite, and the Schur complement left after any
// panel does not depend on the row order inside the panel's window, so the trailing
// matrix stays positive definite up to the last node row; the one pivot that needs a
// row exchange is the last node's (zero in exact arithmetic), which the window's extra
// row (the bordering row, directly below it) supplies.  Rows below the window are
// never searched: their multipliers are the independent substitutions
// L21 = A21 U11^-1, and no column has to be read whole before its pivot is known.
// Per panel:
//   (a) the window ((w + 1) x w) is factored in shared memory with partial pivoting
//       over its rows (first maximum, as the other kernels);
//   (b) the window's row exchanges are applied to the other columns of its rows;
//   (c) U12 = L11^-1 A12, a thread per column;
//   (d) L21 = A21 U11^-1 for the rows below the window, a thread per row;
//   (e) A22 -= L21 U12 on the FP64 tensor cores: U12 is staged in shared memory 64
//       columns at a time and each warp walks its 8-row blocks of the trailing matrix
//       against that tile (A = -L21 and C from global memory, B from shared memory).
// The pivot sequence is LAPACK's (piv[k] = row exchanged with k at step k), so the
// solves of the blocked kernel apply unchanged.  The rank test is the same.
// ---------------------------------------------------------------------------------
constexpr int kLargeMaxN = 4096;
constexpr int kUTile = 64;
constexpr int kUStride = kUTile + 4;  // row stride of the staged U12 tile
// The factorization runs kLargeThreads threads a CTA; in the trailing update each warp
// takes blocks of kBlockRows rows (kHalves 8-row halves).  Per-warp stages: kBlockRows
// C rows of 64 columns, the row stride chosen so that the fragment loads (two doubles
// a lane) hit distinct banks.
constexpr int kLargeThreads = 512;
constexpr int kBlockRows = 8;
constexpr int kHalves = kBlockRows / 8;
constexpr int kCStride = kUTile + 8;
constexpr int kStageDoubles = kBlockRows * kCStride;
constexpr size_t kLargeStageBytes = (size_t)(kLargeThreads / 32) * 2 * kStageDoubles * sizeof(double);
constexpr long long kSpinLimit = 1ll << 24;  // polls of an mbarrier before a copy is given up

__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
               : "memory");
}
// Polls the barrier's phase with a limit; false when the limit ran out.
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  for (long long k = 0; k < kSpinLimit; ++k) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_addr(bar)), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}
// Bulk copy (TMA engine, no multicast) of `bytes` (a multiple of 16; both addresses
// 16-byte aligned) from global to this CTA's shared memory, completing on `bar`.
__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_addr(dst)),
               "l"(src), "r"(bytes), "r"(smem_addr(bar))
               : "memory");
}
// Orders this thread's earlier shared-memory accesses before later async-proxy writes.
__device__ __forceinline__ void fence_proxy_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// (c) U12 = L11^-1 A12, a thread per column, and (d) L21 = A21 U11^-1 for the rows
// below the window, a thread per row (kept out of line: their 32-entry rows need
// registers that the trailing update uses for its accumulators).
__device__ __noinline__ void panel_solves(double* F, int n, int kb, int w, int h, const double* Pn) {
  const int tid = threadIdx.x;
    // (c) U12 = L11^-1 A12
    for (int j = kb + w + tid; j < n; j += blockDim.x) {
      double x[kPanel];
#pragma unroll
      for (int r = 0; r < kPanel; ++r) x[r] = r < w ? F[(size_t)(kb + r) * n + j] : 0.0;
#pragma unroll
      for (int r = 1; r < kPanel; ++r)
#pragma unroll
        for (int q = 0; q < r; ++q) x[r] = fma(-Pn[r * kPanelStride + q], x[q], x[r]);
#pragma unroll
      for (int r = 0; r < kPanel; ++r)
        if (r < w) F[(size_t)(kb + r) * n + j] = x[r];
    }
    // (d) L21 = A21 U11^-1 for the rows below the window
    for (int r = kb + h + tid; r < n; r += blockDim.x) {
      double x[kPanel];
#pragma unroll
      for (int j = 0; j < kPanel; ++j) x[j] = j < w ? F[(size_t)r * n + kb + j] : 0.0;
#pragma unroll
      for (int j = 0; j < kPanel; ++j) {
        double v = x[j];
#pragma unroll
        for (int q = 0; q < j; ++q) v = fma(-x[q], Pn[q * kPanelStride + j], v);
        x[j] = j < w ? v * (1.0 / Pn[j * kPanelStride + j]) : 0.0;
      }
#pragma unroll
      for (int j = 0; j < kPanel; ++j)
        if (j < w) F[(size_t)r * n + kb + j] = x[j];
    }
}

__global__ void __launch_bounds__(kLargeThreads, 1) large_factor_kernel(
    const mhm_ragged_matrix* __restrict__ desc, int max_n, const double* __restrict__ mats,
    double* __restrict__ factors, int32_t* __restrict__ piv, double* __restrict__ rs, double* __restrict__ cs,
    int32_t* __restrict__ status) {
  extern __shared__ __align__(16) double stages[];    // per warp: two trailing-update stages
  __shared__ double Pn[(kPanel + 1) * kPanelStride];  // the window: (w + 1) x w
  __shared__ __align__(16) double Us[kPanel * kUStride];  // U12 tile: 32 x 64
  __shared__ double red[32];
  __shared__ __align__(8) uint64_t bars[2 * (kLargeThreads / 32)];
  __shared__ int sperm[kPanel];
  __shared__ int apos[2 * kPanel + 2], asrc[2 * kPanel + 2];
  __shared__ int srcrow[kPanel + 1];
  __shared__ int naff, abort_all;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  const mhm_ragged_matrix d = desc[blockIdx.x];
  const int n = d.n, sidx = d.slot;
  if (n < 1 || n > max_n) {
    if (tid == 0) status[sidx] = MHM_CELL_SIZE;
    return;
  }
  const size_t voff = (size_t)d.vec_off;
  double* F = factors + d.mat_off;
  // bulk copies need 16-byte aligned rows: an even order and an aligned matrix
  const bool bulk = (n % 2 == 0) && ((reinterpret_cast<uintptr_t>(F) & 15) == 0);
  uint32_t qcount = 0;     // this warp's bulk-copy stages used so far (stage q & 1, phase q >> 1)
  bool prefetched = false;  // the next tile's first block is already in flight
  if (lane == 0) {
    mbar_init(&bars[2 * wid], 1);
    mbar_init(&bars[2 * wid + 1], 1);
  }
  if (tid == 0) abort_all = 0;
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  __syncthreads();
  int st = equilibrate(n, mats + d.mat_off, F, rs + voff, cs + voff);
  for (int kb = 0; kb < n && st == MHM_CELL_OK; kb += kPanel) {
    const int w = min(kPanel, n - kb), h = min(w + 1, n - kb);
    for (int idx = tid; idx < h * kPanel; idx += blockDim.x) {
      const int r = idx >> 5, c = idx & 31;
      if (c < w) Pn[r * kPanelStride + c] = F[(size_t)(kb + r) * n + kb + c];
    }
    __syncthreads();
    for (int c = 0; c < w; ++c) {
      // the previous column's multipliers are scaled in the pivot-search phase (its
      // elimination ended at the last barrier; the columns differ)
      if (c > 0) {
        const double pinv = 1.0 / Pn[(c - 1) * kPanelStride + (c - 1)];
        for (int r = c + tid; r < h; r += blockDim.x) Pn[r * kPanelStride + c - 1] *= pinv;
      }
      if (wid == nw - 1) {
        double best = -1.0;
        int bi = c;
        for (int r = c + lane; r < h; r += 32) {
          const double v = fabs(Pn[r * kPanelStride + c]);
          if (v > best) { best = v; bi = r; }
        }
        for (int o = 16; o > 0; o >>= 1) {
          const double ob = __shfl_xor_sync(0xffffffffu, best, o);
          const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
          if (ob > best || (ob == best && oi < bi)) { best = ob; bi = oi; }
        }
        if (lane == 0) sperm[c] = bi;
      }
      __syncthreads();
      const int p = sperm[c];
      if (p != c && tid < w) {
        const double t = Pn[c * kPanelStride + tid];
        Pn[c * kPanelStride + tid] = Pn[p * kPanelStride + tid];
        Pn[p * kPanelStride + tid] = t;
      }
      __syncthreads();
      const double dg = Pn[c * kPanelStride + c];
      if (dg == 0.0) { st = MHM_CELL_SINGULAR_PIVOT; break; }
      const double inv = 1.0 / dg;
      // (row below the pivot, column right of it): at most 32 x 31 independent pairs
      const int cols = w - c - 1, rows = h - c - 1;
      for (int idx = tid; idx < rows * 32; idx += blockDim.x) {
        const int r = c + 1 + (idx >> 5), j = c + 1 + (idx & 31);
        if (j - c - 1 < cols)
          Pn[r * kPanelStride + j] = fma(-Pn[r * kPanelStride + c] * inv, Pn[c * kPanelStride + j],
                                         Pn[r * kPanelStride + j]);
      }
      __syncthreads();
    }
    if (st != MHM_CELL_OK) break;
    {
      const double pinv = 1.0 / Pn[(w - 1) * kPanelStride + (w - 1)];
      for (int r = w + tid; r < h; r += blockDim.x) Pn[r * kPanelStride + w - 1] *= pinv;
    }
    __syncthreads();
    for (int idx = tid; idx < h * kPanel; idx += blockDim.x) {
      const int r = idx >> 5, c = idx & 31;
      if (c < w) F[(size_t)(kb + r) * n + kb + c] = Pn[r * kPanelStride + c];
    }
    for (int c = tid; c < w; c += blockDim.x) piv[voff + kb + c] = kb + sperm[c];
    // (b) compose the window's exchanges: srcrow[r] = the window row that ends at r
    if (tid == 0) {
      for (int r = 0; r < h; ++r) srcrow[r] = r;
      for (int c = 0; c < w; ++c) {
        const int p = sperm[c];
        if (p != c) {
          const int t = srcrow[c];
          srcrow[c] = srcrow[p];
          srcrow[p] = t;
        }
      }
      int cnt = 0;
      for (int r = 0; r < h; ++r)
        if (srcrow[r] != r) {
          apos[cnt] = r;
          asrc[cnt] = srcrow[r];
          ++cnt;
        }
      naff = cnt;
    }
    __syncthreads();
    const int moved = naff;
    if (moved > 0)
      for (int j = tid; j < n - w; j += blockDim.x) {
        const int col = j < kb ? j : j + w;
        double v[kPanel + 1];
#pragma unroll
        for (int k = 0; k < kPanel + 1; ++k) v[k] = k < moved ? F[(size_t)(kb + asrc[k]) * n + col] : 0.0;
#pragma unroll
        for (int k = 0; k < kPanel + 1; ++k)
          if (k < moved) F[(size_t)(kb + apos[k]) * n + col] = v[k];
      }
    __syncthreads();
    panel_solves(F, n, kb, w, h, Pn);
    __syncthreads();
    // (e) A22 -= L21 U12.  Fragments: A[lane/4][lane%4], B[lane%4][lane/4],
    // C[lane/4][2 (lane%4) + {0, 1}]; panel columns past w are masked to 0.
    const int m2 = n - kb - w, base = kb + w;
    const int fr = lane >> 2, fc = lane & 3;
    const int ksteps = (w + 3) >> 2;
    for (int tj = 0; tj < m2 && !abort_all; tj += kUTile) {
      for (int idx = tid; idx < kPanel * kUTile; idx += blockDim.x) {
        const int r = idx >> 6, c = idx & (kUTile - 1);
        Us[r * kUStride + c] = (r < w && tj + c < m2) ? F[(size_t)(kb + r) * n + base + tj + c] : 0.0;
      }
      // this thread's earlier global writes (factors, swaps, trailing stores) before the
      // bulk copies that read them
      if (bulk) asm volatile("fence.proxy.async;" ::: "memory");
      __syncthreads();
      if (bulk) {
        // Each warp's 16-row blocks of C arrive by bulk copies (the TMA engine, one copy
        // per row) into the warp's two shared-memory stages: block t + 1 is in flight,
        // and its L21 rows are loaded into registers, while block t is on the tensor
        // cores (16 independent accumulator tiles per k-step).  Here w = 32 (a trailing
        // matrix exists only below a full panel).
        // The first block of the next tile is issued during this tile's last block, so
        // the pipeline does not drain at the tile boundary (C blocks do not depend on
        // the U12 tile).
        const int cols = min(kUTile, m2 - tj);
        const uint32_t cbytes = (uint32_t)cols * 8u;
        const int nblk = kBlockRows * wid < m2 ? (m2 - kBlockRows * wid + kBlockRows * nw - 1) / (kBlockRows * nw) : 0;
        double* stg = stages + (size_t)wid * 2 * kStageDoubles;
        auto issue_at = [&](int t, uint32_t q, int tjx) {
          const int rb = kBlockRows * wid + kBlockRows * nw * t;
          const int rows = min(kBlockRows, m2 - rb);
          const uint32_t cb = (uint32_t)min(kUTile, m2 - tjx) * 8u;
          uint64_t* bar = &bars[2 * wid + (q & 1u)];
          fence_proxy_async_smem();
          if (lane == 0) mbar_arrive_expect_tx(bar, (uint32_t)rows * cb);
          __syncwarp();
          if (lane < rows)
            bulk_copy_g2s(stg + (q & 1u) * kStageDoubles + lane * kCStride,
                          F + (size_t)(base + rb + lane) * n + base + tjx, cb, bar);
        };
        auto issue = [&](int t, uint32_t q) { issue_at(t, q, tj); };
        auto load_l21 = [&](int t, double (&a)[kHalves][kPanel / 4]) {
          const int rb = kBlockRows * wid + kBlockRows * nw * t;
#pragma unroll
          for (int h = 0; h < kHalves; ++h) {
            const int i = min(rb + 8 * h + fr, m2 - 1);
#pragma unroll
            for (int s = 0; s < kPanel / 4; ++s) a[h][s] = -F[(size_t)(base + i) * n + kb + 4 * s + fc];
          }
        };
        double av[kHalves][kPanel / 4];
        if (nblk > 0) {
          if (!prefetched) issue(0, qcount);
          load_l21(0, av);
        }
        prefetched = false;
        for (int t = 0; t < nblk; ++t) {
          const uint32_t q = qcount + (uint32_t)t;
          double an[kHalves][kPanel / 4];
          if (t + 1 < nblk) {
            issue(t + 1, q + 1);
            load_l21(t + 1, an);
          } else if (tj + kUTile < m2) {
            issue_at(0, q + 1, tj + kUTile);
            prefetched = true;
          }
          if (!mbar_wait_bounded(&bars[2 * wid + (q & 1u)], (q >> 1) & 1u)) {
            // a copy that never lands: wait once more (bounded) for it and the next one,
            // then give up on this matrix without issuing more copies
            mbar_wait_bounded(&bars[2 * wid + (q & 1u)], (q >> 1) & 1u);
            if (t + 1 < nblk || prefetched)
              mbar_wait_bounded(&bars[2 * wid + ((q + 1) & 1u)], ((q + 1) >> 1) & 1u);
            if (lane == 0) abort_all = 1;
            break;
          }
          const double* sC = stg + (q & 1u) * kStageDoubles;
          const int rb = kBlockRows * wid + kBlockRows * nw * t;
          double acc[kHalves][8][2];
#pragma unroll
          for (int h = 0; h < kHalves; ++h) {
            const int i = rb + 8 * h + fr;
#pragma unroll
            for (int b = 0; b < 8; ++b) {
              const int jj = 8 * b + 2 * fc;
              const bool ok = i < m2 && jj < cols;  // cols is even: a pair is in or out
              const double2 v =
                  ok ? *reinterpret_cast<const double2*>(sC + (8 * h + fr) * kCStride + jj) : make_double2(0.0, 0.0);
              acc[h][b][0] = v.x;
              acc[h][b][1] = v.y;
            }
          }
#pragma unroll
          for (int s = 0; s < kPanel / 4; ++s) {
            double bv[8];
#pragma unroll
            for (int b = 0; b < 8; ++b) bv[b] = Us[(4 * s + fc) * kUStride + 8 * b + fr];
#pragma unroll
            for (int b = 0; b < 8; ++b)
#pragma unroll
              for (int h = 0; h < kHalves; ++h) dmma_8x8x4(acc[h][b][0], acc[h][b][1], av[h][s], bv[b]);
          }
#pragma unroll
          for (int h = 0; h < kHalves; ++h) {
            const int i = rb + 8 * h + fr;
            if (i < m2) {
              double* crow = F + (size_t)(base + i) * n + base + tj;
#pragma unroll
              for (int b = 0; b < 8; ++b) {
                const int jj = 8 * b + 2 * fc;
                if (jj < cols) *reinterpret_cast<double2*>(crow + jj) = make_double2(acc[h][b][0], acc[h][b][1]);
              }
            }
          }
          __syncwarp();  // every lane has read the stage before block t + 2 is copied into it
          if (t + 1 < nblk) {
#pragma unroll
            for (int h = 0; h < kHalves; ++h)
#pragma unroll
              for (int s = 0; s < kPanel / 4; ++s) av[h][s] = an[h][s];
          }
          if (t + 1 == nblk) qcount += (uint32_t)nblk;
        }
      } else {
        for (int rb = 8 * wid; rb < m2; rb += 8 * nw) {
          const int i = rb + fr;
          const size_t row = (size_t)(base + (i < m2 ? i : m2 - 1)) * n;
          double av[kPanel / 4];
#pragma unroll
          for (int s = 0; s < kPanel / 4; ++s) {
            const int q = 4 * s + fc;
            av[s] = q < w ? -F[row + kb + q] : 0.0;
          }
          double acc[8][2];
#pragma unroll
          for (int b = 0; b < 8; ++b)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int j = tj + 8 * b + 2 * fc + e;
              acc[b][e] = (i < m2 && j < m2) ? F[row + base + j] : 0.0;
            }
#pragma unroll
          for (int s = 0; s < kPanel / 4; ++s) {
            if (s >= ksteps) break;
            double bv[8];
#pragma unroll
            for (int b = 0; b < 8; ++b) bv[b] = Us[(4 * s + fc) * kUStride + 8 * b + fr];
#pragma unroll
            for (int b = 0; b < 8; ++b) dmma_8x8x4(acc[b][0], acc[b][1], av[s], bv[b]);
          }
          if (i < m2) {
#pragma unroll
            for (int b = 0; b < 8; ++b)
#pragma unroll
              for (int e = 0; e < 2; ++e) {
                const int j = tj + 8 * b + 2 * fc + e;
                if (j < m2) F[row + base + j] = acc[b][e];
              }
          }
        }
      }
      __syncthreads();
    }
    if (abort_all) st = MHM_CELL_TIMEOUT;
  }
  if (st == MHM_CELL_OK) {
    double dmin = 1e300, amax = 0.0;
    for (int i = tid; i < n; i += blockDim.x) dmin = fmin(dmin, fabs(F[(size_t)i * n + i]));
    for (int i = wid; i < n; i += nw)
      for (int j = lane; j < n; j += 32) amax = fmax(amax, fabs(F[(size_t)i * n + j]));
    dmin = block_min(dmin, red);
    amax = block_max(amax, red);
    if (dmin <= 2.220446049250313e-16 * n * amax) st = MHM_CELL_RANK_DEFICIENT;
  }
  if (tid == 0) status[sidx] = st;
}

// W <- U^-1 L^-1 W for the shared-memory block W (n, nrhs), in place, by chunks of
// 32 rows (right-looking): the chunk's diagonal block (in Dg) is solved with one
// warp per column, a lane per row; then every row beyond the chunk subtracts its
// 32 factor entries times the chunk's solution, a thread per row with the 32
// loads issued together.  The threads whose rows form the next chunk also load
// that chunk's diagonal block (into the other half of Dg) in the same pass.
// W (n, nrhs) with row stride ws.
template <int NCB = 2>
__device__ void chunked_lu_solve(int n, int nrhs, int ws, const double* LU, double* W, double* Dg) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  const int nchunk = (n + 31) / 32;
  for (int dir = 0; dir < 2; ++dir) {
    const bool lower = dir == 0;
    int cur = 0;
    {  // the first diagonal block
      const int i0 = lower ? 0 : (nchunk - 1) * 32, h = min(32, n - i0);
      for (int idx = tid; idx < 32 * 32; idx += blockDim.x) {
        const int r = idx >> 5, c = idx & 31;
        Dg[r * 33 + c] = (r < h && c < h) ? LU[(size_t)(i0 + r) * n + i0 + c] : 0.0;
      }
      __syncthreads();
    }
    for (int q = 0; q < nchunk; ++q) {
      const int i0 = lower ? q * 32 : (nchunk - 1 - q) * 32;
      const int h = min(32, n - i0);
      const double* D = Dg + cur * 32 * 33;
      double* Dn = Dg + (1 - cur) * 32 * 33;
      for (int c = wid; c < nrhs; c += nw) {
        double v = lane < h ? W[(size_t)(i0 + lane) * ws + c] : 0.0;
        if (lower) {
          for (int sidx = 0; sidx < h; ++sidx) {
            const double xs = __shfl_sync(0xffffffffu, v, sidx);
            if (lane > sidx && lane < h) v = fma(-D[lane * 33 + sidx], xs, v);
          }
        } else {
          for (int sidx = h - 1; sidx >= 0; --sidx) {
            if (lane == sidx) v = v / D[sidx * 33 + sidx];
            const double xs = __shfl_sync(0xffffffffu, v, sidx);
            if (lane < sidx) v = fma(-D[lane * 33 + sidx], xs, v);
          }
        }
        if (lane < h) W[(size_t)(i0 + lane) * ws + c] = v;
      }
      __syncthreads();
      // rows beyond the chunk (below for L, above for U):
      //   W[i] -= LU[i][i0 .. i0 + h) W[i0 .. i0 + h)
      // on the tensor cores, a warp per block of 8 rows, the chunk's columns in steps of
      // 4 (past h masked to 0), the right-hand sides in blocks of 8 (FP64 mma.sync
      // m8n8k4; fragments A[lane/4][lane%4], B[lane%4][lane/4], C[lane/4][2 (lane%4) +
      // {0, 1}]).  The next chunk's diagonal block is staged beside it.
      const int r0 = lower ? i0 + h : 0, r1 = lower ? n : i0;
      const int n0 = lower ? i0 + h : i0 - 32;  // first row of the next chunk
      const int hn = lower ? min(32, n - n0) : 32;
      const int fr = lane >> 2, fc = lane & 3;
      const int ncb = (nrhs + 7) >> 3;
      for (int rb = r0 + 8 * wid; rb < r1; rb += 8 * nw) {
        const int i = rb + fr;
        const bool iv = i < r1;
        double acc[NCB][2];
#pragma unroll
        for (int cb = 0; cb < NCB; ++cb)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int col = 8 * cb + 2 * fc + e;
            acc[cb][e] = (cb < ncb && iv && col < nrhs) ? W[(size_t)i * ws + col] : 0.0;
          }
        const double* row = LU + (size_t)(iv ? i : rb) * n + i0;
#pragma unroll
        for (int k0 = 0; k0 < 32; k0 += 4) {
          const int k = k0 + fc;
          const double av = (iv && k < h) ? -row[k] : 0.0;
#pragma unroll
          for (int cb = 0; cb < NCB; ++cb) {
            if (cb >= ncb) break;
            const int col = 8 * cb + fr;
            const double bv = (k < h && col < nrhs) ? W[(size_t)(i0 + k) * ws + col] : 0.0;
            dmma_8x8x4(acc[cb][0], acc[cb][1], av, bv);
          }
        }
        if (iv) {
#pragma unroll
          for (int cb = 0; cb < NCB; ++cb)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int col = 8 * cb + 2 * fc + e;
              if (cb < ncb && col < nrhs) W[(size_t)i * ws + col] = acc[cb][e];
            }
        }
      }
      if (q + 1 < nchunk)
        for (int idx = tid; idx < 32 * 32; idx += blockDim.x) {
          const int r = idx >> 5, c = idx & 31;
          Dn[r * 33 + c] = (r < hn && c < hn) ? LU[(size_t)(n0 + r) * n + n0 + c] : 0.0;
        }
      __syncthreads();
      cur = 1 - cur;
    }
  }
}

// W <- U^-1 L^-1 W for a block W (n, nrhs <= 32, row stride ws) in global memory
// (large orders), left-looking by chunks of 32 rows: each chunk's rows first subtract
// the already solved rows' contributions, LU[chunk, solved] W[solved] (one GEMM on the
// FP64 tensor cores streaming the factor rows and the solved rows from global memory;
// the warps split the inner dimension, each forming all 16 output tiles of 8 x 8 over
// its share, and the 8 partials are summed in warp order through `part` (8 x 32 x 32)),
// then the chunk is solved against its diagonal block in shared memory (a warp per
// column, a lane per row).  Every factor entry is read once per direction.  Dg holds
// the diagonal block and Wc the chunk's right-hand sides (32 x 33 each).
__device__ void gw_lu_solve(int n, int nrhs, int ws, const double* LU, double* W, double* Dg, double* Wc,
                            double* part) {
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  const int fr = lane >> 2, fc = lane & 3;
  const int nchunk = (n + 31) / 32;
  const int ncb = (nrhs + 7) >> 3;
  for (int dir = 0; dir < 2; ++dir) {
    const bool lower = dir == 0;
    for (int q = 0; q < nchunk; ++q) {
      const int i0 = lower ? q * 32 : (nchunk - 1 - q) * 32;
      const int h = min(32, n - i0);
      const int k0 = lower ? 0 : i0 + h, k1 = lower ? i0 : n;
      for (int idx = tid; idx < 32 * 32; idx += blockDim.x) {
        const int r = idx >> 5, c = idx & 31;
        Dg[r * 33 + c] = (r < h && c < h) ? LU[(size_t)(i0 + r) * n + i0 + c] : 0.0;
        Wc[r * 33 + c] = (r < h && c < nrhs) ? W[(size_t)(i0 + r) * ws + c] : 0.0;
      }
      // warp wid takes the k-steps wid, wid + nw, ... of [k0, k1) and forms the whole
      // 32 x 32 partial product (16 tiles of 8 x 8) over them
      double acc[4][4][2] = {};
      const double* arow[4];
#pragma unroll
      for (int rb = 0; rb < 4; ++rb) {
        const int row = min(i0 + 8 * rb + fr, i0 + h - 1);
        arow[rb] = LU + (size_t)row * n;
      }
#pragma unroll 4
      for (int k = k0 + 4 * wid; k < k1; k += 4 * nw) {
        const int kk = k + fc;
        const bool kv = kk < k1;
        double a[4], b[4];
#pragma unroll
        for (int rb = 0; rb < 4; ++rb) a[rb] = kv ? arow[rb][kk] : 0.0;
#pragma unroll
        for (int cb = 0; cb < 4; ++cb) {
          const int col = 8 * cb + fr;
          b[cb] = (kv && cb < ncb && col < nrhs) ? W[(size_t)kk * ws + col] : 0.0;
        }
#pragma unroll
        for (int rb = 0; rb < 4; ++rb)
#pragma unroll
          for (int cb = 0; cb < 4; ++cb) dmma_8x8x4(acc[rb][cb][0], acc[rb][cb][1], a[rb], b[cb]);
      }
      // the warps' partials, summed in warp order (deterministic)
#pragma unroll
      for (int rb = 0; rb < 4; ++rb)
#pragma unroll
        for (int cb = 0; cb < 4; ++cb)
#pragma unroll
          for (int e = 0; e < 2; ++e) part[wid * 1024 + (8 * rb + fr) * 32 + 8 * cb + 2 * fc + e] = acc[rb][cb][e];
      __syncthreads();
      for (int idx = tid; idx < 32 * 32; idx += blockDim.x) {
        double t = 0.0;
        for (int w = 0; w < nw; ++w) t += part[w * 1024 + idx];
        const int r = idx >> 5, c = idx & 31;
        Wc[r * 33 + c] -= t;
      }
      __syncthreads();
      for (int c = wid; c < nrhs; c += nw) {
        double v = lane < h ? Wc[lane * 33 + c] : 0.0;
        if (lower) {
          for (int sidx = 0; sidx < h; ++sidx) {
            const double xs = __shfl_sync(0xffffffffu, v, sidx);
            if (lane > sidx && lane < h) v = fma(-Dg[lane * 33 + sidx], xs, v);
          }
        } else {
          for (int sidx = h - 1; sidx >= 0; --sidx) {
            if (lane == sidx) v = v / Dg[sidx * 33 + sidx];
            const double xs = __shfl_sync(0xffffffffu, v, sidx);
            if (lane < sidx) v = fma(-Dg[lane * 33 + sidx], xs, v);
          }
        }
        if (lane < h) W[(size_t)(i0 + lane) * ws + c] = v;
      }
      __syncthreads();
    }
  }
}

// Solve with the right-hand sides in shared memory (n nrhs small enough): the
// permutation is composed once, every application reads the factors in chunks, the
// residual B - A X is one warp per row in double-double arithmetic, then the
// reference's columnwise max-scaled acceptance (cuda.py:230-255).
// With desc (ragged batches), CTA m solves columns c0 .. c0 + NR - 1 of the system
// desc[m] describes (order n, nrhs columns, offsets, status word); a system with no
// column in that range is skipped.  With GW (large orders), the solution and the
// correction blocks X and W live in gwork (2 x (KC + 1) doubles per row of the
// system, at 2 (KC + 1) vec_off) instead of shared memory, and the accurate residual
// reads its rows without the register prefetch.
template <int NR, bool GW = false>
__global__ void __launch_bounds__(kLuThreads) batched_solve_chunked_kernel(
    int n_uniform, int nrhs_uniform, int ldr_uniform, int c0, const double* __restrict__ mats,
    const double* __restrict__ factors, const int32_t* __restrict__ piv, const double* __restrict__ rs,
    const double* __restrict__ cs, const double* __restrict__ rhs, double* __restrict__ x, double rtol, double atol,
    int max_refine, int32_t* __restrict__ status, const mhm_ragged_matrix* __restrict__ desc, int max_n,
    double* __restrict__ gwork) {
  constexpr int KC = NR > 16 ? NR : 16;  // column capacity of the partial sums
  constexpr int NCB = KC / 8;            // 8-column blocks of the tensor-core steps
  extern __shared__ __align__(16) double sm[];
  int n = n_uniform, nrhs = nrhs_uniform, ldr = ldr_uniform, sidx = blockIdx.x;
  size_t moff = (size_t)n_uniform * n_uniform * blockIdx.x, voff = (size_t)n_uniform * blockIdx.x,
         roff = (size_t)n_uniform * ldr_uniform * blockIdx.x;
  if (desc) {
    const mhm_ragged_matrix d = desc[blockIdx.x];
    n = d.n;
    ldr = d.nrhs;
    nrhs = min(NR, d.nrhs - c0);
    sidx = d.slot;
    moff = (size_t)d.mat_off;
    voff = (size_t)d.vec_off;
    roff = (size_t)d.rhs_off;
    if (n < 1 || n > max_n) {
      if (threadIdx.x == 0 && c0 == 0) status[sidx] = MHM_CELL_SIZE;
      return;
    }
    if (nrhs < 1) return;
  }
  // X and W are (n, nrhs) with an odd row stride ws = nrhs | 1, so that lanes reading
  // consecutive rows of one column hit distinct shared-memory banks
  const int ws = nrhs | 1;
  double* X = GW ? gwork + 2 * (KC + 1) * voff : sm;              // (n, ws)
  double* W = GW ? X + (size_t)n * (KC + 1) : X + (size_t)n * ws; // (n, ws)
  double* Dg = GW ? sm : W + (size_t)n * ws;                      // 2 x 32 x 33
  double* part = Dg + 2 * 32 * 33;         // 32 x KC
  double* colr = part + 32 * KC;           // (3, KC): bmax, b2, r2 per column
  // GW: the triangular solves' partial products (8 x 32 x 32) follow colr
  int* perm = reinterpret_cast<int*>(colr + 3 * KC + (GW ? 8 * 1024 : 0));
  int* iperm = perm + n;
  __shared__ int flag;
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  const double* A = mats + moff;
  const double* LU = factors + moff;
  const double* rsc = rs + voff;
  const double* csc = cs + voff;
  // columns c0 .. c0 + nrhs - 1 of (n, ldr) row-major right-hand sides and solutions
  const double* B = rhs + roff + c0;
  double* Xg = x + roff + c0;
  if (status[sidx] != MHM_CELL_OK) return;
  if (tid == 0) {
    for (int i = 0; i < n; ++i) perm[i] = i;
    const int32_t* pv = piv + voff;
    for (int k = 0; k < n; ++k) {
      const int p = pv[k];
      if (p != k) { const int t = perm[k]; perm[k] = perm[p]; perm[p] = t; }
    }
    for (int i = 0; i < n; ++i) iperm[perm[i]] = i;
    flag = 0;
  }
  if (tid < KC) colr[tid] = colr[KC + tid] = 0.0;
  __syncthreads();
  int nonfinite = 0;
  // (row, column) loops run over n x NR slots (NR a power of two: shift and mask, no
  // division), skipping the columns past nrhs
  for (int idx = tid; idx < n * NR; idx += blockDim.x)
    if (idx % NR < nrhs && !isfinite(B[(size_t)(idx / NR) * ldr + idx % NR])) nonfinite = 1;
  if (__syncthreads_or(nonfinite)) {
    for (int idx = tid; idx < n * NR; idx += blockDim.x) {
      if (idx % NR >= nrhs) continue;
      const size_t g = (size_t)(idx / NR) * ldr + idx % NR;
      Xg[g] = B[g];
    }
    if (tid == 0) status[sidx] = MHM_CELL_NONFINITE;
    return;
  }
  // per column: max |b| and ||b / scale||^2
  for (int c = wid; c < nrhs; c += nw) {
    double bmax = 0.0;
    for (int i = lane; i < n; i += 32) bmax = fmax(bmax, fabs(B[(size_t)i * ldr + c]));
    bmax = warp_max(bmax);
    double scale = fmax(atol, bmax);
    if (!(scale > 0.0)) scale = 1.0;
    double b2 = 0.0;
    for (int i = lane; i < n; i += 32) {
      const double bv = B[(size_t)i * ldr + c] / scale;
      b2 += bv * bv;
    }
    b2 = warp_sum(b2);
    if (lane == 0) { colr[c] = scale; colr[KC + c] = b2; }
  }
  // X = csc .* U^-1 L^-1 P (rsc .* B)
  for (int idx = tid; idx < n * NR; idx += blockDim.x) {
    const int i = idx / NR, c = idx % NR;
    if (c >= nrhs) continue;
    const int src = perm[i];
    W[i * ws + c] = B[(size_t)src * ldr + c] * rsc[src];
  }
  __syncthreads();
  if constexpr (GW)
    gw_lu_solve(n, nrhs, ws, LU, W, Dg, Dg + 32 * 33, colr + 3 * KC);
  else
    chunked_lu_solve<NCB>(n, nrhs, ws, LU, W, Dg);
  for (int idx = tid; idx < n * NR; idx += blockDim.x) {
    const int i = idx / NR, c = idx % NR;
    if (c < nrhs) X[i * ws + c] = W[i * ws + c] * csc[i];
  }
  __syncthreads();
  int result = MHM_CELL_RESIDUAL;
  for (int pass = 0; pass <= max_refine; ++pass) {
    int bad = 0;
    for (int idx = tid; idx < n * NR; idx += blockDim.x)
      if (idx % NR < nrhs && !isfinite(X[(idx / NR) * ws + idx % NR])) bad = 1;
    if (__syncthreads_or(bad)) { result = MHM_CELL_NONFINITE; break; }
    // As the reference's _checked (linalg/linear.py:132-152): first the plain binary64
    // residual, here on the FP64 tensor cores (a warp per 8-row block, A fragments from
    // global memory, X fragments from shared memory; fragments A[lane/4][lane%4],
    // B[lane%4][lane/4], C[lane/4][2 (lane%4) + {0, 1}]), with per lane the sums of
    // (r / scale)^2 of its columns; only when it fails the acceptance, the accurate
    // residual below, which also feeds the correction.
    if constexpr (GW) {
      // large orders: 32 rows at a time, the eight warps splitting the inner dimension
      // (each forms the 32-row block's partial product for all columns over its share
      // of k, the partials summed in warp order through the shared buffer after colr),
      // so X is read once per 32 rows and every warp streams a short k-range.  Thread
      // t keeps the sum of (r / scale)^2 of column t % 32 over its rows.
      const int fr = lane >> 2, fc = lane & 3;
      const int ncb = (nrhs + 7) >> 3;
      double* pp = colr + 3 * KC;  // (8, 32, 32) partials
      double s2c = 0.0;
      for (int i0 = 0; i0 < n; i0 += 32) {
        double acc[4][NCB][2] = {};
        const double* arow[4];
#pragma unroll
        for (int rb = 0; rb < 4; ++rb) arow[rb] = A + (size_t)min(i0 + 8 * rb + fr, n - 1) * n;
#pragma unroll 4
        for (int k = 4 * wid; k < n; k += 4 * nw) {
          const int kk = k + fc;
          const bool kv = kk < n;
          double a[4], b[NCB];
#pragma unroll
          for (int rb = 0; rb < 4; ++rb) a[rb] = kv ? arow[rb][kk] : 0.0;
#pragma unroll
          for (int cb = 0; cb < NCB; ++cb) {
            const int col = 8 * cb + fr;
            b[cb] = (kv && cb < ncb && col < nrhs) ? X[(size_t)kk * ws + col] : 0.0;
          }
#pragma unroll
          for (int rb = 0; rb < 4; ++rb)
#pragma unroll
            for (int cb = 0; cb < NCB; ++cb) dmma_8x8x4(acc[rb][cb][0], acc[rb][cb][1], a[rb], b[cb]);
        }
#pragma unroll
        for (int rb = 0; rb < 4; ++rb)
#pragma unroll
          for (int cb = 0; cb < NCB; ++cb)
#pragma unroll
            for (int e = 0; e < 2; ++e) pp[wid * 1024 + (8 * rb + fr) * 32 + 8 * cb + 2 * fc + e] = acc[rb][cb][e];
        __syncthreads();
        for (int idx = tid; idx < 32 * 32; idx += blockDim.x) {
          const int r = idx >> 5, c = idx & 31;
          if (i0 + r < n && c < nrhs) {
            double t = 0.0;
            for (int q = 0; q < nw; ++q) t += pp[q * 1024 + idx];
            const double rv = (B[(size_t)(i0 + r) * ldr + c] - t) / colr[c];
            s2c = fma(rv, rv, s2c);
          }
        }
        __syncthreads();
      }
      part[wid * KC + lane] = s2c;  // column lane of this warp's rows
      __syncthreads();
      if (tid == 0) {
        int ok = 1;
        for (int c = 0; c < nrhs; ++c) {
          double t = 0.0;
          for (int q = 0; q < nw; ++q) t += part[q * KC + c];
          const double limit = fmax(atol / colr[c], rtol * sqrt(colr[KC + c]));
          if (!(sqrt(t) <= limit)) ok = 0;
        }
        flag = ok;
      }
      __syncthreads();
      if (flag) { result = MHM_CELL_OK; break; }
    } else {
      const int fr = lane >> 2, fc = lane & 3;
      const int ncb = (nrhs + 7) >> 3;
      double s2[NCB][2] = {};
      for (int rb = 8 * wid; rb < n; rb += 8 * nw) {
        const int i = rb + fr;
        const bool iv = i < n;
        const double* arow = A + (size_t)(iv ? i : rb) * n;
        double acc[NCB][2] = {};
#pragma unroll 8
        for (int k0 = 0; k0 < n; k0 += 4) {
          const int kk = k0 + fc;
          const double a = (iv && kk < n) ? arow[kk] : 0.0;
#pragma unroll
          for (int cb = 0; cb < NCB; ++cb) {
            if (cb >= ncb) break;
            const int col = 8 * cb + fr;
            const double bx = (kk < n && col < nrhs) ? X[(size_t)kk * ws + col] : 0.0;
            dmma_8x8x4(acc[cb][0], acc[cb][1], a, bx);
          }
        }
        if (iv) {
#pragma unroll
          for (int cb = 0; cb < NCB; ++cb)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int col = 8 * cb + 2 * fc + e;
              if (cb < ncb && col < nrhs) {
                const double rv = (B[(size_t)i * ldr + col] - acc[cb][e]) / colr[col];
                s2[cb][e] = fma(rv, rv, s2[cb][e]);
              }
            }
        }
      }
#pragma unroll
      for (int cb = 0; cb < NCB; ++cb)
#pragma unroll
        for (int e = 0; e < 2; ++e) {
          double v = s2[cb][e];
          v += __shfl_xor_sync(0xffffffffu, v, 4);
          v += __shfl_xor_sync(0xffffffffu, v, 8);
          v += __shfl_xor_sync(0xffffffffu, v, 16);
          const int col = 8 * cb + 2 * fc + e;
          if (fr == 0 && cb < ncb && col < nrhs) part[wid * KC + col] = v;
        }
      __syncthreads();
      if (tid == 0) {
        int ok = 1;
        for (int c = 0; c < nrhs; ++c) {
          double t = 0.0;
          for (int q = 0; q < nw; ++q) t += part[q * KC + c];
          const double limit = fmax(atol / colr[c], rtol * sqrt(colr[KC + c]));
          if (!(sqrt(t) <= limit)) ok = 0;
        }
        flag = ok;
      }
      __syncthreads();
      if (flag) { result = MHM_CELL_OK; break; }
    }
    // R = B - A X, one warp per row; the scaled residual goes to W at the row's
    // permuted position (ready for the correction solve); per warp the sums of
    // (r / scale)^2 per column, added in warp order below
    double wr2[NR];
#pragma unroll
    for (int c = 0; c < NR; ++c) wr2[c] = 0.0;
    // each lane's (at most 20) entries of the warp's next row are loaded while the
    // current row is summed
    constexpr int kPer = GW ? 1 : kBlockedMaxN / 32;
    double av[kPer], an[kPer];
    if (!GW && wid < n) {
      const double* row = A + (size_t)wid * n;
#pragma unroll
      for (int u = 0; u < kPer; ++u) av[u] = lane + 32 * u < n ? row[lane + 32 * u] : 0.0;
    }
    for (int i = wid; i < n; i += nw) {
      if (!GW && i + nw < n) {
        const double* nrow = A + (size_t)(i + nw) * n;
#pragma unroll
        for (int u = 0; u < kPer; ++u) an[u] = lane + 32 * u < n ? nrow[lane + 32 * u] : 0.0;
      }
      double hi[NR], lo[NR];
#pragma unroll
      for (int c = 0; c < NR; ++c) hi[c] = lo[c] = 0.0;
      if constexpr (GW) {
        const double* row = A + (size_t)i * n;
        for (int j = lane; j < n; j += 32) {
          const double a = row[j];
#pragma unroll
          for (int c = 0; c < NR; ++c)
            if (c < nrhs) dd_fma(hi[c], lo[c], -a, X[(size_t)j * ws + c]);
        }
      } else {
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
          const int j = lane + 32 * u;
          if (j < n) {
#pragma unroll
            for (int c = 0; c < NR; ++c)
              if (c < nrhs) dd_fma(hi[c], lo[c], -av[u], X[(size_t)j * ws + c]);
          }
        }
      }
#pragma unroll
      for (int c = 0; c < NR; ++c) {
        if (c >= nrhs) continue;
        double h = hi[c], l = lo[c];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          const double oh = __shfl_xor_sync(0xffffffffu, h, o);
          const double ol = __shfl_xor_sync(0xffffffffu, l, o);
          double sres, e;
          two_sum(h, oh, sres, e);
          h = sres;
          l += ol + e;
        }
        if (lane == 0) {
          double sres, e;
          two_sum(B[(size_t)i * ldr + c], h, sres, e);
          const double r = sres + (e + l);
          W[(size_t)iperm[i] * ws + c] = r * rsc[i];
          const double rv = r / colr[c];
          wr2[c] = fma(rv, rv, wr2[c]);
        }
      }
      if constexpr (!GW) {
#pragma unroll
        for (int u = 0; u < kPer; ++u) av[u] = an[u];
      }
    }
    if (lane == 0)
#pragma unroll
      for (int c = 0; c < NR; ++c) part[wid * KC + c] = wr2[c];
    __syncthreads();
    if (tid == 0) {
      for (int c = 0; c < nrhs; ++c) {
        double t = 0.0;
        for (int q = 0; q < nw; ++q) t += part[q * KC + c];
        colr[2 * KC + c] = t;
      }
      int ok = 1;
      for (int c = 0; c < nrhs; ++c) {
        const double scale = colr[c];
        const double limit = fmax(atol / scale, rtol * sqrt(colr[KC + c]));
        if (!(sqrt(colr[2 * KC + c]) <= limit)) ok = 0;
      }
      flag = ok;
    }
    __syncthreads();
    if (flag) { result = MHM_CELL_OK; break; }
    if (pass == max_refine) break;
    if constexpr (GW)
    gw_lu_solve(n, nrhs, ws, LU, W, Dg, Dg + 32 * 33, colr + 3 * KC);
  else
    chunked_lu_solve<NCB>(n, nrhs, ws, LU, W, Dg);
    for (int idx = tid; idx < n * NR; idx += blockDim.x) {
      const int i = idx / NR, c = idx % NR;
      if (c < nrhs) X[i * ws + c] += W[i * ws + c] * csc[i];
    }
    __syncthreads();
  }
  for (int idx = tid; idx < n * NR; idx += blockDim.x) {
    const int i = idx / NR, c = idx % NR;
    if (c < nrhs) Xg[(size_t)i * ldr + c] = X[i * ws + c];
  }
  if (tid == 0 && result != MHM_CELL_OK) status[sidx] = result;
}

// Shared memory of the GW solve: the diagonal blocks, partial sums and the row
// permutation (X and W are in global memory).
size_t large_solve_smem(int n) { return ((size_t)2 * 32 * 33 + 32 * 32 + 3 * 32 + 8 * 1024) * 8 + (size_t)2 * n * 4; }

size_t chunked_solve_smem(int n, int nrhs) {
  return ((size_t)2 * n * (nrhs | 1) + 2 * 32 * 33 + 32 * 16 + 3 * 16) * 8 + (size_t)2 * n * 4;
}
}  // namespace
}  // namespace mhm

using namespace mhm;

extern "C" int mhm_batched_factor(int64_t count, int32_t n, const double* matrices, double* factors,
                                  int32_t* pivots, double* row_scale, double* col_scale,
                                  int32_t* status, void* stream) {
  if (count < 1 || n < 1 || !matrices || !factors || !pivots || !row_scale || !col_scale || !status)
    return MHM_ERR_ARGUMENT;
  if (count > 0x7fffffff) return MHM_ERR_UNSUPPORTED;
  const size_t bytes = (size_t)n * n * 8;
  const int in_smem = bytes <= 200 * 1024;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (!in_smem && n <= kBlockedMaxN) {
    const size_t smem = (size_t)n * kPanelStride * 8;
    if (cudaFuncSetAttribute(batched_factor_blocked_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
      return MHM_ERR_LAUNCH;
    batched_factor_blocked_kernel<<<(unsigned)count, kLuThreads, smem, st>>>(n, matrices, factors, pivots,
                                                                             row_scale, col_scale, status,
                                                                             nullptr, n);
    return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
  }
  const size_t smem = in_smem ? bytes : 0;
  if (in_smem && smem > 48 * 1024 &&
      cudaFuncSetAttribute(batched_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  batched_factor_kernel<<<(unsigned)count, kLuThreads, smem, st>>>(
      n, matrices, factors, pivots, row_scale, col_scale, status, in_smem);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_batched_solve(int64_t count, int32_t n, int32_t nrhs, const double* matrices,
                                 const double* factors, const int32_t* pivots,
                                 const double* row_scale, const double* col_scale, const double* rhs,
                                 double* x, double* work, double rtol, double atol,
                                 int32_t max_refine, int32_t* status, void* stream) {
  if (count < 1 || n < 1 || nrhs < 1 || !matrices || !factors || !pivots || !row_scale ||
      !col_scale || !rhs || !x || !work || !status || max_refine < 0 || !(rtol >= 0) || !(atol >= 0))
    return MHM_ERR_ARGUMENT;
  if (count > 0x7fffffff) return MHM_ERR_UNSUPPORTED;
  // the residual's row prefetch covers n <= kBlockedMaxN columns
  // more than 16 right-hand sides: column groups of 16 (each column's acceptance is
  // its own, and a matrix that failed in one group is skipped by the next)
  const int group = nrhs <= 16 ? nrhs : 16;
  if (n <= kBlockedMaxN && chunked_solve_smem(n, group) <= 200 * 1024) {
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    auto go = [&](auto kernel, int c0, int cols) {
      const size_t sm = chunked_solve_smem(n, cols);
      if (sm > 48 * 1024 &&
          cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) != cudaSuccess)
        return MHM_ERR_LAUNCH;
      kernel<<<(unsigned)count, kLuThreads, sm, st>>>(n, cols, nrhs, c0, matrices, factors, pivots, row_scale,
                                                      col_scale, rhs, x, rtol, atol, max_refine, status, nullptr,
                                                      n, nullptr);
      return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
    };
    for (int c0 = 0; c0 < nrhs; c0 += group) {
      const int cols = nrhs - c0 < group ? nrhs - c0 : group;
      const int rc = cols <= 4 ? go(batched_solve_chunked_kernel<4>, c0, cols)
                     : cols <= 8 ? go(batched_solve_chunked_kernel<8>, c0, cols)
                                 : go(batched_solve_chunked_kernel<16>, c0, cols);
      if (rc != MHM_OK) return rc;
    }
    return MHM_OK;
  }
  batched_solve_kernel<<<(unsigned)count, kLuThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      n, nrhs, matrices, factors, pivots, row_scale, col_scale, rhs, x, work, rtol, atol, max_refine,
      status);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_batched_factor_ragged(int64_t count, const mhm_ragged_matrix* desc, int32_t max_n,
                                         const double* matrices, double* factors, int32_t* pivots,
                                         double* row_scale, double* col_scale, int32_t* status, void* stream) {
  if (count < 1 || !desc || max_n < 1 || max_n > kBlockedMaxN || !matrices || !factors || !pivots || !row_scale ||
      !col_scale || !status)
    return MHM_ERR_ARGUMENT;
  if (count > 0x7fffffff) return MHM_ERR_UNSUPPORTED;
  const size_t smem = (size_t)max_n * kPanelStride * 8;
  if (cudaFuncSetAttribute(batched_factor_blocked_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return MHM_ERR_LAUNCH;
  batched_factor_blocked_kernel<<<(unsigned)count, kLuThreads, smem, static_cast<cudaStream_t>(stream)>>>(
      max_n, matrices, factors, pivots, row_scale, col_scale, status, desc, max_n);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_batched_solve_ragged(int64_t count, const mhm_ragged_matrix* desc, int32_t max_n,
                                        int32_t max_nrhs, const double* matrices, const double* factors,
                                        const int32_t* pivots, const double* row_scale, const double* col_scale,
                                        const double* rhs, double* x, double rtol, double atol, int32_t max_refine,
                                        int32_t* status, void* stream) {
  if (count < 1 || !desc || max_n < 1 || max_n > kBlockedMaxN || max_nrhs < 1 || !matrices || !factors ||
      !pivots || !row_scale || !col_scale || !rhs || !x || !status || max_refine < 0 || !(rtol >= 0) ||
      !(atol >= 0))
    return MHM_ERR_ARGUMENT;
  if (count > 0x7fffffff) return MHM_ERR_UNSUPPORTED;
  const int group = max_nrhs < 16 ? max_nrhs : 16;
  const size_t sm = chunked_solve_smem(max_n, group);
  if (sm > 200 * 1024) return MHM_ERR_UNSUPPORTED;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaFuncSetAttribute(batched_solve_chunked_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm) !=
      cudaSuccess)
    return MHM_ERR_LAUNCH;
  for (int c0 = 0; c0 < max_nrhs; c0 += 16) {
    batched_solve_chunked_kernel<16><<<(unsigned)count, kLuThreads, sm, st>>>(
        max_n, group, group, c0, matrices, factors, pivots, row_scale, col_scale, rhs, x, rtol, atol, max_refine,
        status, desc, max_n, nullptr);
    if (cudaGetLastError() != cudaSuccess) return MHM_ERR_LAUNCH;
  }
  return MHM_OK;
}

extern "C" int mhm_batched_factor_large(int64_t count, const mhm_ragged_matrix* desc, int32_t max_n,
                                        const double* matrices, double* factors, int32_t* pivots,
                                        double* row_scale, double* col_scale, int32_t* status, void* stream) {
  if (count < 1 || !desc || max_n < 1 || max_n > kLargeMaxN || !matrices || !factors || !pivots || !row_scale ||
      !col_scale || !status)
    return MHM_ERR_ARGUMENT;
  if (count > 0x7fffffff) return MHM_ERR_UNSUPPORTED;
  if (cudaFuncSetAttribute(large_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kLargeStageBytes) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  large_factor_kernel<<<(unsigned)count, kLargeThreads, kLargeStageBytes, static_cast<cudaStream_t>(stream)>>>(
      desc, max_n, matrices, factors, pivots, row_scale, col_scale, status);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_batched_solve_large(int64_t count, const mhm_ragged_matrix* desc, int32_t max_n,
                                       int32_t max_nrhs, const double* matrices, const double* factors,
                                       const int32_t* pivots, const double* row_scale, const double* col_scale,
                                       const double* rhs, double* x, double* work, double rtol, double atol,
                                       int32_t max_refine, int32_t* status, void* stream) {
  if (count < 1 || !desc || max_n < 1 || max_n > kLargeMaxN || max_nrhs < 1 || !matrices || !factors ||
      !pivots || !row_scale || !col_scale || !rhs || !x || !work || !status || max_refine < 0 || !(rtol >= 0) ||
      !(atol >= 0))
    return MHM_ERR_ARGUMENT;
  if (count > 0x7fffffff) return MHM_ERR_UNSUPPORTED;
  const int group = max_nrhs < 32 ? max_nrhs : 32;
  const size_t sm = large_solve_smem(max_n);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (cudaFuncSetAttribute(batched_solve_chunked_kernel<32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)sm) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  for (int c0 = 0; c0 < max_nrhs; c0 += 32) {
    batched_solve_chunked_kernel<32, true><<<(unsigned)count, kLuThreads, sm, st>>>(
        max_n, group, group, c0, matrices, factors, pivots, row_scale, col_scale, rhs, x, rtol, atol, max_refine,
        status, desc, max_n, work);
    if (cudaGetLastError() != cudaSuccess) return MHM_ERR_LAUNCH;
  }
  return MHM_OK;
}

extern "C" const char* mhm_version(void) { return "mhm_b200 0.1.0 (sm_100a)"; }
