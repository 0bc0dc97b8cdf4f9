// Batched dense equilibrated LU with FP64 residual refinement.
//
// Replaces the reference's cuBLAS dgetrfBatched/dgetrsBatched path
// (PyMHM 1.3.2 src/pymhm/execution/cuda.py:114-288, BatchedFactorization):
//   * row then column max-equilibration, zero row/column rejection (:201-211)
//   * partial-pivoting LU, exact-zero pivot -> "singular pivot" (:127-131)
//   * rank test min |u_ii| <= eps * n * max |LU| -> "rank deficient" (:132-135)
//   * solve with the equilibrated factors, FP64 residual on the original matrix,
//     at most two corrections, columnwise acceptance (:230-255)
// One CTA owns one matrix; the working matrix lives in shared memory when it
// fits and in the caller's `factors` array (L2-resident) otherwise.
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
  const size_t smem = in_smem ? bytes : 0;
  if (in_smem && smem > 48 * 1024 &&
      cudaFuncSetAttribute(batched_factor_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  batched_factor_kernel<<<(unsigned)count, kLuThreads, smem, static_cast<cudaStream_t>(stream)>>>(
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
  batched_solve_kernel<<<(unsigned)count, kLuThreads, 0, static_cast<cudaStream_t>(stream)>>>(
      n, nrhs, matrices, factors, pivots, row_scale, col_scale, rhs, x, work, rtol, atol, max_refine,
      status);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" const char* mhm_version(void) { return "mhm_b200 0.1.0 (sm_100a)"; }
