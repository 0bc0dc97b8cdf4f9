// Global skeleton solve for macro meshes of any shape (tetrahedra, polygons, ...).
//
// Reference: solve_hybrid_system's global solve (PyMHM 1.3.2, core/system.py:355-528,
// SuperLU at rtol 1e-10 through linalg/linear.py:798).  Here the assembled system
//
//   K = [[S, -G], [-G^T, -C]]   (trace unknowns lambda, one coarse unknown per cell)
//
// is solved by an outer FP64 defect correction x += K0^-1 (b - K x) on the assembled
// CSR matrix, with K0 = [[S, -G0], [-G0^T, 0]] and G0 = B^T 1 the exact geometric
// net-flux operator (K - K0 is at rounding level).  K0 is solved by projected CG
// (the FETI natural coarse space):
//
//   lambda0 = G0 Q (-r_c),  Q = (G0^T G0)^-1 (dense, built once per mesh);
//   P S P mu = P (r_lambda - S lambda0),  P = I - G0 Q G0^T,
//   preconditioner P M^-1 P, M^-1 either block Jacobi over the skeleton faces or,
//   when the caller passes the cells' condensed blocks, the cell-Dirichlet sum
//   sum_c R_c^T D_c S_c^-1 D_c R_c (S_c the cell's trace-trace block, D_c the
//   stiffness weights S_c,aa / S_aa), the FETI Dirichlet preconditioner with the
//   roles of the Neumann and Dirichlet operators exchanged (S_c maps fluxes to
//   traces here);
//   c = Q G0^T (S lambda - r_lambda),  lambda = lambda0 + mu.
//
// One persistent cooperative launch does everything.  Vectors live in the caller's
// workspace; the trace-trace block S is read from the CSR rows (columns < T).  Every
// sum runs in a fixed order (per-CTA partials summed identically in every CTA), so
// results are bitwise reproducible.  Seven grid barriers per CG iteration: the
// residual and the search direction are double-buffered so that values another CTA
// still reads are never overwritten in the same phase, and the updated residual that
// the cell sums need is recomputed where it is read, with the same arithmetic.  Every
// barrier is bounded: a CTA that waits too long sets the error flag, and all return.
#include <cmath>
#include <cstdint>

#include "mhm_common.cuh"

namespace mhm {
namespace {

constexpr int kGThreads = 512;
constexpr long long kGSpinLimit = 1ll << 26;
constexpr int kMaxFace = 8;  // DOFs per skeleton face
constexpr int kSlots = 4;    // reduction slots per CTA

struct GWork {
  double* mu;
  double* rt[2];
  double* p[2];
  double* q;
  double* r;
  double* z0;
  double* z;
  double* lam0;
  double* w;
  double* v;
  double* w2;
  double* v2;
  double* rfull;
  double* finv;
  double* dof_g;   // (T, 2): G0 entry of the DOF in its first and second cell
  double* ypart;   // (cell entries): a cell's preconditioned residual on its DOFs
  double* dsum;    // (T): sum of the DOF's diagonal entries over its cells' blocks
  double* cinv;    // (cell entries^2 ragged): D S_c^-1 D of every cell
  double* part;
  unsigned* bar;
  int* err;
};

struct GParams {
  mhm_general_system s;
  GWork w;
  const double* rhs;
  double* x;
  double rtol, inner_rtol;
  int max_inner, max_outer;
  int* info;
  double* stats;
};

__device__ __forceinline__ unsigned g_ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void g_red_release_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded grid barrier on a monotonic arrival counter zeroed by the host.
__device__ bool g_sync(const GWork& w, unsigned& epoch) {
  __shared__ int bad;
  __syncthreads();
  ++epoch;
  if (threadIdx.x == 0) {
    const unsigned target = epoch * gridDim.x;
    g_red_release_add(w.bar, 1u);
    long long spins = 0;
    while (g_ld_acquire(w.bar) < target) {
      if (++spins > kGSpinLimit) {
        atomicExch(w.err, 1);
        break;
      }
      if ((spins & 1023) == 0 && *reinterpret_cast<volatile int*>(w.err) != 0) break;
      if (spins > 64) __nanosleep(20);
    }
    bad = *reinterpret_cast<volatile int*>(w.err);
  }
  __syncthreads();
  return bad == 0;
}

__device__ void g_partial(const GWork& w, int slot, double v, double* red) {
  v = block_sum(v, red);
  if (threadIdx.x == 0) w.part[blockIdx.x * kSlots + slot] = v;
}

__device__ void g_partial_max(const GWork& w, int slot, double v, double* red) {
  v = block_max(v, red);
  if (threadIdx.x == 0) w.part[blockIdx.x * kSlots + slot] = v;
}

// Totals of slots [0, n) over all CTAs, in CTA order (the same bits in every CTA); the
// slots whose bit is set in max_mask are combined by maximum instead of sum.
__device__ void g_totals(const GWork& w, int n, double* out, double* sh, unsigned max_mask = 0u) {
  if (threadIdx.x < 32) {
    for (int k = 0; k < n; ++k) {
      const bool mx = (max_mask >> k) & 1u;
      double a = 0.0;
      for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) {
        const double v = __ldcg(w.part + i * kSlots + k);
        a = mx ? fmax(a, v) : a + v;
      }
      a = mx ? warp_max(a) : warp_sum(a);
      if (threadIdx.x == 0) sh[k] = a;
    }
  }
  __syncthreads();
  for (int k = 0; k < n; ++k) out[k] = sh[k];
  __syncthreads();
}

// (G0 v)_i: the DOF's entries in its (at most two) cells, first cell then second
// (dof_g holds the entries, 0 for a missing second cell).
__device__ __forceinline__ double g0_apply(const mhm_general_system& s, const double* dof_g, int64_t i,
                                           const double* v) {
  const int2 c = reinterpret_cast<const int2*>(s.dof_cells)[i];
  double acc = dof_g[2 * i] * __ldcg(v + c.x);
  if (c.y >= 0) acc = fma(dof_g[2 * i + 1], __ldcg(v + c.y), acc);
  return acc;
}

// y = Q x, one warp per row, lanes over the columns (fixed order).
__device__ void q_gemv(const mhm_general_system& s, const double* xin, double* yout) {
  const int M = s.cells;
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = wid; c < M; c += nw) {
    const double* row = s.coarse_inverse + c * (int64_t)M;
    double acc = 0.0;
    for (int d = lane; d < M; d += 32) acc = fma(__ldg(row + d), __ldcg(xin + d), acc);
    acc = warp_sum(acc);
    if (lane == 0) yout[c] = acc;
  }
}

// Face block-Jacobi: z0 on the DOFs of face f from the projected residual rt - G0 v.
__device__ __forceinline__ void face_apply(const GParams& P, int64_t f, const double* rt, const double* v,
                                           double* z0) {
  const mhm_general_system& s = P.s;
  const int64_t f0 = s.face_ptr[f];
  const int fs = (int)(s.face_ptr[f + 1] - f0);
  double rv[kMaxFace];
  for (int j = 0; j < fs; ++j) rv[j] = __ldcg(rt + f0 + j) - g0_apply(s, P.w.dof_g, f0 + j, v);
  const double* inv = P.w.finv + f * kMaxFace * kMaxFace;
  for (int i = 0; i < fs; ++i) {
    double acc = 0.0;
    for (int j = 0; j < fs; ++j) acc = fma(inv[i * kMaxFace + j], rv[j], acc);
    z0[f0 + i] = acc;
  }
}

// Cell-Dirichlet: y_c = D S_c^-1 D r_c on the cell's DOFs, r = rt - G0 v, one warp per
// cell (lane a computes row a; t <= 32).
__device__ __forceinline__ void cell_apply(const GParams& P, int64_t c, const double* rt, const double* v,
                                           int lane) {
  const mhm_general_system& s = P.s;
  const int64_t e0 = s.cell_ptr[c];
  const int t = (int)(s.cell_ptr[c + 1] - e0);
  double ra = 0.0;
  if (lane < t) {
    const int64_t i = s.cell_dofs[e0 + lane];
    ra = __ldcg(rt + i) - g0_apply(s, P.w.dof_g, i, v);
  }
  const double* W = P.w.cinv + s.block_off[c];
  double acc = 0.0;
  for (int b = 0; b < t; ++b) {
    const double rb = __shfl_sync(0xffffffffu, ra, b);
    if (lane < t) acc = fma(W[lane * t + b], rb, acc);
  }
  if (lane < t) P.w.ypart[e0 + lane] = acc;
}

// The DOF's preconditioned value: the sum of its cells' parts, first cell then second.
__device__ __forceinline__ double dof_gather(const GParams& P, int64_t i) {
  const mhm_general_system& s = P.s;
  const int2 c = reinterpret_cast<const int2*>(s.dof_cells)[i];
  double acc = __ldcg(P.w.ypart + s.dof_entry[2 * i]);
  if (c.y >= 0) acc += __ldcg(P.w.ypart + s.dof_entry[2 * i + 1]);
  return acc;
}

// Inverse of the face's diagonal block of S (SPD): Cholesky, then the inverse from
// the factor, by one thread.
__device__ void face_inverse(const mhm_general_system& s, int f, double* out) {
  const int64_t f0 = s.face_ptr[f];
  const int fs = (int)(s.face_ptr[f + 1] - f0);
  double a[kMaxFace][kMaxFace];
  for (int r = 0; r < fs; ++r) {
    for (int c = 0; c < fs; ++c) a[r][c] = 0.0;
    const int64_t row = f0 + r;
    for (int64_t k = s.indptr[row]; k < s.indptr[row + 1]; ++k) {
      const int64_t col = s.indices[k];
      if (col >= f0 && col < f0 + fs) a[r][col - f0] = s.values[k];
    }
  }
  // lower Cholesky in place
  for (int j = 0; j < fs; ++j) {
    double d = a[j][j];
    for (int k = 0; k < j; ++k) d -= a[j][k] * a[j][k];
    d = d > 0.0 ? sqrt(d) : 0.0;
    a[j][j] = d;
    for (int i = j + 1; i < fs; ++i) {
      double v = a[i][j];
      for (int k = 0; k < j; ++k) v -= a[i][k] * a[j][k];
      a[i][j] = d > 0.0 ? v / d : 0.0;
    }
  }
  // columns of the inverse: solve L L^T x = e_c
  for (int c = 0; c < fs; ++c) {
    double y[kMaxFace];
    for (int i = 0; i < fs; ++i) {
      double v = (i == c) ? 1.0 : 0.0;
      for (int k = 0; k < i; ++k) v -= a[i][k] * y[k];
      y[i] = a[i][i] > 0.0 ? v / a[i][i] : 0.0;
    }
    for (int i = fs - 1; i >= 0; --i) {
      double v = y[i];
      for (int k = i + 1; k < fs; ++k) v -= a[k][i] * y[k];
      y[i] = a[i][i] > 0.0 ? v / a[i][i] : 0.0;
    }
    for (int i = 0; i < fs; ++i) out[i * kMaxFace + c] = y[i];
  }
}

// D S_c^-1 D of one cell, by one warp: S_c is the top-left t x t of the cell's block
// (row length t + 1); Gauss-Jordan in place on W (lane j owns column j; SPD, no
// pivoting), then the stiffness weights D_a = S_aa / (sum over the DOF's cells).
__device__ void cell_inverse(const GParams& P, int64_t c, int lane) {
  const mhm_general_system& s = P.s;
  const int64_t e0 = s.cell_ptr[c];
  const int t = (int)(s.cell_ptr[c + 1] - e0);
  const double* S = s.cell_blocks + s.block_off[c];
  double* W = P.w.cinv + s.block_off[c];
  if (lane < t)
    for (int i = 0; i < t; ++i) W[i * t + lane] = S[i * (t + 1) + lane];
  __syncwarp();
  for (int k = 0; k < t; ++k) {
    const double a = 1.0 / W[k * t + k];
    __syncwarp();
    if (lane < t && lane != k) W[k * t + lane] *= a;
    __syncwarp();
    // column k is left untouched until its own update below
    if (lane < t && lane != k)
      for (int i = 0; i < t; ++i)
        if (i != k) W[i * t + lane] = fma(-W[i * t + k], W[k * t + lane], W[i * t + lane]);
    __syncwarp();
    if (lane == k) {
      for (int i = 0; i < t; ++i)
        if (i != k) W[i * t + k] = -W[i * t + k] * a;
      W[k * t + k] = a;
    }
    __syncwarp();
  }
  double d = 0.0;
  if (lane < t) d = S[lane * (t + 1) + lane] / __ldcg(P.w.dsum + s.cell_dofs[e0 + lane]);
  for (int i = 0; i < t; ++i) {
    const double di = __shfl_sync(0xffffffffu, d, i);
    if (lane < t) W[i * t + lane] *= di * d;
  }
  __syncwarp();
}

// r = rt - G0 v on every DOF; z0 = M^-1 r (face blocks, or the cells' D S^-1 D summed
// per DOF); w2 = G0^T z0 per cell.  Two grid barriers; false when one timed out.
__device__ __noinline__ bool precondition(const GParams& P, const double* rt, unsigned& epoch) {
  const mhm_general_system& s = P.s;
  const GWork& w = P.w;
  const int64_t T = s.trace_size;
  const int M = s.cells;
  const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
  const bool cellmode = s.cell_blocks != nullptr;
  for (int64_t i = gtid; i < T; i += gstride) w.r[i] = __ldcg(rt + i) - g0_apply(s, w.dof_g, i, w.v);
  if (cellmode) {
    const int lane = threadIdx.x & 31;
    for (int64_t c = gtid >> 5; c < M; c += gstride >> 5) cell_apply(P, c, rt, w.v, lane);
  } else {
    for (int64_t f = gtid; f < s.faces; f += gstride) face_apply(P, f, rt, w.v, w.z0);
  }
  if (!g_sync(w, epoch)) return false;
  if (cellmode)
    for (int64_t i = gtid; i < T; i += gstride) w.z0[i] = dof_gather(P, i);
  for (int64_t c = gtid; c < M; c += gstride) {
    double acc = 0.0;
    for (int64_t e = s.cell_ptr[c]; e < s.cell_ptr[c + 1]; ++e) {
      const int64_t i = s.cell_dofs[e];
      acc = fma(s.cell_g0[e], cellmode ? dof_gather(P, i) : __ldcg(w.z0 + i), acc);
    }
    w.w2[c] = acc;
  }
  return g_sync(w, epoch);
}

// Per-DOF setup: the DOF's G0 entries, and the sum of its diagonal entries over its
// cells' blocks (cell-Dirichlet) or, per face, the face block inverses.
__global__ void general_setup_kernel(const GParams P) {
  const mhm_general_system& s = P.s;
  const GWork& w = P.w;
  const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
  const bool cellmode = s.cell_blocks != nullptr;
  for (int64_t i = gtid; i < s.trace_size; i += gstride) {
    const int2 c = reinterpret_cast<const int2*>(s.dof_cells)[i];
    w.dof_g[2 * i] = s.cell_g0[s.dof_entry[2 * i]];
    w.dof_g[2 * i + 1] = c.y >= 0 ? s.cell_g0[s.dof_entry[2 * i + 1]] : 0.0;
    if (cellmode) {
      double d = 0.0;
      for (int k = 0; k < 2; ++k) {
        const int cc = k ? c.y : c.x;
        if (cc < 0) continue;
        const int64_t a = s.dof_entry[2 * i + k] - s.cell_ptr[cc];
        const int tc = (int)(s.cell_ptr[cc + 1] - s.cell_ptr[cc]);
        d += s.cell_blocks[s.block_off[cc] + a * (tc + 1) + a];
      }
      w.dsum[i] = d;
    }
  }
  if (!cellmode)
    for (int64_t f = gtid; f < s.faces; f += gstride) face_inverse(s, (int)f, w.finv + f * kMaxFace * kMaxFace);
}

// One warp per cell: D S_c^-1 D (after general_setup_kernel's DOF sums).
__global__ void general_cell_inverse_kernel(const GParams P) {
  const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t nwarps = ((int64_t)gridDim.x * blockDim.x) >> 5;
  for (int64_t c = gtid >> 5; c < P.s.cells; c += nwarps) cell_inverse(P, c, threadIdx.x & 31);
}

__global__ void __launch_bounds__(kGThreads, 1) general_pcg_kernel(const GParams P) {
  __shared__ double red[32];
  __shared__ double sh[kSlots];
  const mhm_general_system& s = P.s;
  const GWork& w = P.w;
  const int64_t T = s.trace_size, N = s.size;
  const int M = s.cells;
  const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
  unsigned epoch = 0;
  int status = MHM_SOLVE_OK;
  int total_inner = 0, outer = 0;
  double tot[kSlots];
  double bnorm = 0.0, res = 0.0, omega = INFINITY;
#define GSYNC()                                                              \
  do {                                                                       \
    if (!g_sync(w, epoch)) { status = MHM_SOLVE_BARRIER_TIMEOUT; goto done; } \
  } while (0)
#define PRECONDITION(RT)                                          \
  do {                                                            \
    if (!precondition(P, (RT), epoch)) {                          \
      status = MHM_SOLVE_BARRIER_TIMEOUT;                         \
      goto done;                                                  \
    }                                                             \
  } while (0)
  {
    double b2 = 0.0;
    for (int64_t i = gtid; i < N; i += gstride) {
      P.x[i] = 0.0;
      const double b = P.rhs[i];
      b2 = fma(b, b, b2);
    }
    g_partial(w, 0, b2, red);
  }
  GSYNC();
  g_totals(w, 1, tot, sh);
  bnorm = sqrt(tot[0]);
  if (!(bnorm > 0.0)) {
    if (!isfinite(bnorm)) status = MHM_SOLVE_NONFINITE;
    goto done;
  }
  for (;;) {
    // ---- outer residual rfull = b - K x over all rows, its norm and the componentwise
    //      backward error max_i |r_i| / (|b_i| + sum_j |K_ij| |x_j|) ----------------------
    {
      double r2 = 0.0, om = 0.0;
      for (int64_t i = gtid; i < N; i += gstride) {
        const double b = P.rhs[i];
        double acc = b, den = fabs(b);
        for (int64_t k = s.indptr[i]; k < s.indptr[i + 1]; ++k) {
          const double t = s.values[k] * __ldcg(P.x + s.indices[k]);
          acc = fma(-s.values[k], __ldcg(P.x + s.indices[k]), acc);
          den += fabs(t);
        }
        w.rfull[i] = acc;
        r2 = fma(acc, acc, r2);
        om = fmax(om, den > 0.0 ? fabs(acc) / den : (acc != 0.0 ? INFINITY : 0.0));
      }
      g_partial(w, 0, r2, red);
      g_partial_max(w, 1, om, red);
    }
    GSYNC();
    g_totals(w, 2, tot, sh, 2u);
    res = sqrt(tot[0]) / bnorm;
    if (!isfinite(res)) { status = MHM_SOLVE_NONFINITE; goto done; }
    // Converged when the normwise residual meets rtol and every row's residual is
    // within rtol of that row's scale (rows of short faces have tiny entries that a
    // normwise test alone leaves unresolved), or the latter stopped improving.
    if (res <= P.rtol && (tot[1] <= P.rtol || tot[1] > 0.5 * omega)) {
      omega = tot[1];
      break;
    }
    omega = tot[1];
    if (outer >= P.max_outer || total_inner >= P.max_inner) { status = MHM_SOLVE_NOT_CONVERGED; goto done; }
    ++outer;
    // ---- lambda0 = G0 Q (-r_c) ---------------------------------------------------
    for (int64_t c = gtid; c < M; c += gstride) w.w[c] = -w.rfull[T + c];
    GSYNC();
    q_gemv(s, w.w, w.v);
    GSYNC();
    for (int64_t i = gtid; i < T; i += gstride) {
      w.lam0[i] = g0_apply(s, w.dof_g, i, w.v);
      w.mu[i] = 0.0;
      w.p[0][i] = 0.0;
    }
    GSYNC();
    // ---- initial residual rt = r_lambda - S lambda0 (trace-trace block of K) ------
    for (int64_t i = gtid; i < T; i += gstride) {
      double acc = w.rfull[i];
      for (int64_t k = s.indptr[i]; k < s.indptr[i + 1]; ++k) {
        const int64_t j = s.indices[k];
        if (j < T) acc = fma(-s.values[k], __ldcg(w.lam0 + j), acc);
      }
      w.rt[0][i] = acc;
    }
    GSYNC();
    // ---- projection and preconditioning of the initial residual ------------------
    for (int64_t c = gtid; c < M; c += gstride) {
      double acc = 0.0;
      for (int64_t e = s.cell_ptr[c]; e < s.cell_ptr[c + 1]; ++e)
        acc = fma(s.cell_g0[e], __ldcg(w.rt[0] + s.cell_dofs[e]), acc);
      w.w[c] = acc;
    }
    GSYNC();
    q_gemv(s, w.w, w.v);
    GSYNC();
    PRECONDITION(w.rt[0]);
    q_gemv(s, w.w2, w.v2);
    GSYNC();
    double gamma, rr0;
    {
      double rz = 0.0, rr = 0.0;
      for (int64_t i = gtid; i < T; i += gstride) {
        const double zi = __ldcg(w.z0 + i) - g0_apply(s, w.dof_g, i, w.v2);
        w.z[i] = zi;
        const double ri = __ldcg(w.r + i);
        rz = fma(ri, zi, rz);
        rr = fma(ri, ri, rr);
      }
      g_partial(w, 0, rz, red);
      g_partial(w, 1, rr, red);
    }
    GSYNC();
    g_totals(w, 2, tot, sh);
    gamma = tot[0];
    rr0 = tot[1];
    {
      // stop once the preconditioned residual norm (r, z)^1/2 fell by inner_rtol
      const double target = P.inner_rtol * sqrt(fmax(gamma, 0.0));
      double beta = 0.0;
      int cur = 0;
      double rr = rr0;
      while (sqrt(fmax(gamma, 0.0)) > target && total_inner < P.max_inner) {
        if (!(gamma > 0.0)) { status = MHM_SOLVE_BREAKDOWN; goto done; }
        const int nxt = cur ^ 1;
        // P1: direction p = z + beta p_prev, q = S p
        {
          double pq = 0.0;
          for (int64_t i = gtid; i < T; i += gstride) {
            const double pi = fma(beta, __ldcg(w.p[cur] + i), __ldcg(w.z + i));
            double qi = 0.0;
            for (int64_t k = s.indptr[i]; k < s.indptr[i + 1]; ++k) {
              const int64_t j = s.indices[k];
              if (j < T) qi = fma(s.values[k], fma(beta, __ldcg(w.p[cur] + j), __ldcg(w.z + j)), qi);
            }
            w.p[nxt][i] = pi;
            w.q[i] = qi;
            pq = fma(pi, qi, pq);
          }
          g_partial(w, 0, pq, red);
        }
        GSYNC();
        g_totals(w, 1, tot, sh);
        if (!(tot[0] > 0.0)) { status = isfinite(tot[0]) ? MHM_SOLVE_BREAKDOWN : MHM_SOLVE_NONFINITE; goto done; }
        const double alpha = gamma / tot[0];
        // P2: mu += alpha p, rt_next = rt - alpha q; the cells' G0^T rt_next
        for (int64_t i = gtid; i < T; i += gstride) {
          w.mu[i] = fma(alpha, __ldcg(w.p[nxt] + i), w.mu[i]);
          w.rt[nxt][i] = fma(-alpha, __ldcg(w.q + i), __ldcg(w.rt[cur] + i));
        }
        for (int64_t c = gtid; c < M; c += gstride) {
          double acc = 0.0;
          for (int64_t e = s.cell_ptr[c]; e < s.cell_ptr[c + 1]; ++e) {
            const int64_t i = s.cell_dofs[e];
            acc = fma(s.cell_g0[e], fma(-alpha, __ldcg(w.q + i), __ldcg(w.rt[cur] + i)), acc);
          }
          w.w[c] = acc;
        }
        GSYNC();
        // P3: v = Q G0^T rt
        q_gemv(s, w.w, w.v);
        GSYNC();
        // P4: r = P rt, z0 = M^-1 r; the cells' G0^T z0 (two barriers)
        PRECONDITION(w.rt[nxt]);
        // P5: v2 = Q G0^T z0
        q_gemv(s, w.w2, w.v2);
        GSYNC();
        // P6: z = P z0; (r, z) and (r, r)
        {
          double rz = 0.0, r2 = 0.0;
          for (int64_t i = gtid; i < T; i += gstride) {
            const double zi = __ldcg(w.z0 + i) - g0_apply(s, w.dof_g, i, w.v2);
            w.z[i] = zi;
            const double ri = __ldcg(w.r + i);
            rz = fma(ri, zi, rz);
            r2 = fma(ri, ri, r2);
          }
          g_partial(w, 0, rz, red);
          g_partial(w, 1, r2, red);
        }
        GSYNC();
        g_totals(w, 2, tot, sh);
        beta = tot[0] / gamma;
        gamma = tot[0];
        rr = tot[1];
        if (!isfinite(rr) || !isfinite(gamma)) { status = MHM_SOLVE_NONFINITE; goto done; }
        cur = nxt;
        ++total_inner;
      }
    }
    // ---- coarse unknowns c = Q G0^T (S lambda - r_lambda), then the update -----------
    for (int64_t i = gtid; i < T; i += gstride) {
      double acc = -w.rfull[i];
      for (int64_t k = s.indptr[i]; k < s.indptr[i + 1]; ++k) {
        const int64_t j = s.indices[k];
        if (j < T) acc = fma(s.values[k], __ldcg(w.lam0 + j) + __ldcg(w.mu + j), acc);
      }
      w.q[i] = acc;
    }
    GSYNC();
    for (int64_t c = gtid; c < M; c += gstride) {
      double acc = 0.0;
      for (int64_t e = s.cell_ptr[c]; e < s.cell_ptr[c + 1]; ++e)
        acc = fma(s.cell_g0[e], __ldcg(w.q + s.cell_dofs[e]), acc);
      w.w[c] = acc;
    }
    GSYNC();
    q_gemv(s, w.w, w.v);
    GSYNC();
    for (int64_t i = gtid; i < T; i += gstride) P.x[i] += __ldcg(w.lam0 + i) + __ldcg(w.mu + i);
    for (int64_t c = gtid; c < M; c += gstride) P.x[T + c] += __ldcg(w.v + c);
    GSYNC();
  }
done:
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.info[0] = status;
    P.info[1] = total_inner;
    P.info[2] = outer;
    P.info[3] = *reinterpret_cast<volatile int*>(w.err);
    P.stats[0] = res;
    P.stats[1] = bnorm;
    P.stats[2] = omega;
  }
#undef GSYNC
#undef PRECONDITION
}

struct GLayout {
  size_t mu, rt0, rt1, p0, p1, q, r, z0, z, lam0, w, v, w2, v2, rfull, finv, dof_g, ypart, dsum, cinv, part,
      bar, err, total;
};

GLayout g_layout(const mhm_general_system* s, int grid) {
  GLayout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off = align16(off + bytes);
    return at;
  };
  const size_t T = (size_t)s->trace_size, N = (size_t)s->size, M = (size_t)s->cells;
  L.mu = take(T * 8);
  L.rt0 = take(T * 8);
  L.rt1 = take(T * 8);
  L.p0 = take(T * 8);
  L.p1 = take(T * 8);
  L.q = take(T * 8);
  L.r = take(T * 8);
  L.z0 = take(T * 8);
  L.z = take(T * 8);
  L.lam0 = take(T * 8);
  L.w = take(M * 8);
  L.v = take(M * 8);
  L.w2 = take(M * 8);
  L.v2 = take(M * 8);
  L.rfull = take(N * 8);
  L.finv = take((size_t)s->faces * kMaxFace * kMaxFace * 8);
  L.dof_g = take(T * 2 * 8);
  L.ypart = take((size_t)s->cell_entries * 8);
  L.dsum = take(T * 8);
  L.cinv = take((size_t)(s->block_off ? s->blocks_size : 1) * 8);
  L.part = take((size_t)grid * kSlots * 8);
  L.bar = take(2 * sizeof(unsigned));
  L.err = take(sizeof(int));
  L.total = off;
  return L;
}

// The layout (everything but the matrix values, which change from solve to solve).
bool g_valid_layout(const mhm_general_system* s) {
  return s && s->trace_size >= 1 && s->cells >= 1 && s->size == s->trace_size + s->cells && s->faces >= 1 &&
         s->indptr && s->indices && s->face_ptr && s->cell_ptr && s->cell_dofs && s->cell_g0 && s->dof_cells &&
         s->dof_entry && s->coarse_inverse && s->max_face_size >= 1 && s->max_face_size <= kMaxFace &&
         s->trace_size <= INT32_MAX && s->cell_entries >= 1 &&
         (!s->block_off || (s->blocks_size >= 1 && s->max_cell_dofs >= 1 && s->max_cell_dofs <= 32)) &&
         (!s->cell_blocks || s->block_off);
}

int g_grid() {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, general_pcg_kernel, kGThreads, 0) != cudaSuccess)
    return -1;
  if (per_sm < 1) return 0;
  return sms;  // one CTA per SM: all co-resident for the cooperative launch
}

}  // namespace
}  // namespace mhm

using namespace mhm;

extern "C" int64_t mhm_general_workspace_bytes(const mhm_general_system* s) {
  if (!g_valid_layout(s)) return -1;
  const int grid = g_grid();
  if (grid <= 0) return -1;
  return (int64_t)g_layout(s, grid).total;
}

extern "C" int mhm_general_solve(const mhm_general_system* s, const double* rhs, double* x, void* workspace,
                                 int64_t workspace_bytes, double rtol, double inner_rtol, int32_t max_inner,
                                 int32_t max_outer, int32_t* info, double* stats, void* stream) {
  if (!g_valid_layout(s) || !s->values || !rhs || !x || !workspace || !info || !stats || !(rtol > 0.0) || !(inner_rtol > 0.0) ||
      max_inner < 1 || max_outer < 1)
    return MHM_ERR_ARGUMENT;
  const int grid = g_grid();
  if (grid < 0) return MHM_ERR_LAUNCH;
  if (grid == 0) return MHM_ERR_UNSUPPORTED;
  const GLayout L = g_layout(s, grid);
  if (workspace_bytes < (int64_t)L.total) return MHM_ERR_ARGUMENT;
  unsigned char* base = static_cast<unsigned char*>(workspace);
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  GParams P{};
  P.s = *s;
  auto d = [&](size_t o) { return reinterpret_cast<double*>(base + o); };
  P.w.mu = d(L.mu);
  P.w.rt[0] = d(L.rt0);
  P.w.rt[1] = d(L.rt1);
  P.w.p[0] = d(L.p0);
  P.w.p[1] = d(L.p1);
  P.w.q = d(L.q);
  P.w.r = d(L.r);
  P.w.z0 = d(L.z0);
  P.w.z = d(L.z);
  P.w.lam0 = d(L.lam0);
  P.w.w = d(L.w);
  P.w.v = d(L.v);
  P.w.w2 = d(L.w2);
  P.w.v2 = d(L.v2);
  P.w.rfull = d(L.rfull);
  P.w.finv = d(L.finv);
  P.w.dof_g = d(L.dof_g);
  P.w.ypart = d(L.ypart);
  P.w.dsum = d(L.dsum);
  P.w.cinv = d(L.cinv);
  P.w.part = d(L.part);
  P.w.bar = reinterpret_cast<unsigned*>(base + L.bar);
  P.w.err = reinterpret_cast<int*>(base + L.err);
  P.rhs = rhs;
  P.x = x;
  P.rtol = rtol;
  P.inner_rtol = inner_rtol;
  P.max_inner = max_inner;
  P.max_outer = max_outer;
  P.info = info;
  P.stats = stats;
  if (cudaMemsetAsync(base + L.bar, 0, L.total - L.bar, st) != cudaSuccess) return MHM_ERR_LAUNCH;
  general_setup_kernel<<<grid * 2, 256, 0, st>>>(P);
  if (s->cell_blocks) general_cell_inverse_kernel<<<grid * 2, 256, 0, st>>>(P);
  void* args[] = {&P};
  if (cudaLaunchCooperativeKernel((const void*)general_pcg_kernel, grid, kGThreads, args, 0, st) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}
