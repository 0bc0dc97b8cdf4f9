// Global skeleton solve for macro meshes of any shape (tetrahedra, polygons, ...).
//
// Reference: solve_hybrid_system's global solve (PyMHM 1.3.2, core/system.py:355-528,
// SuperLU at rtol 1e-10 through linalg/linear.py:798).  Here the assembled system
//
//   K = [[S, -G], [-G^T, -C]]   (trace unknowns lambda, one coarse unknown per cell)
//
// is solved by flexible GMRES on the assembled CSR matrix in FP64, right-preconditioned
// by solves with K0 = [[S, -G0], [-G0^T, 0]], G0 = B^T 1 the exact geometric net-flux
// operator.  K - K0 is at rounding level for most cells, where GMRES takes the two
// steps of a plain defect correction; cells whose retained basis was corrected
// (A 1 != 0) carry G != G0 and a coarse term C, and K0^-1 K is then the identity plus
// a low-rank term, which GMRES resolves in a few more steps (a defect correction
// alone diverges once that term exceeds one).  K0 is solved by projected CG (the FETI
// natural coarse space):
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
// workspace.  Every sum runs in a fixed order (per-CTA partials summed identically in
// every CTA, the small least-squares problem solved the same way in every CTA), so
// results are bitwise reproducible.  The trace-trace block is re-laid as column-major
// ELL at setup, the coarse vector of each Q product is staged in shared memory, and
// per-cell sums run a warp per cell.  Seven grid barriers per CG iteration: the
// residual and the search direction are double-buffered so that values another CTA
// still reads are never overwritten in the same phase, and the updated residual that
// the cell sums need is recomputed where it is read, with the same arithmetic.  Every
// barrier is bounded: a CTA that waits too long sets the error flag, and all return.
#include <cmath>
#include <cstdint>

#include "mhm_common.cuh"

namespace mhm {
namespace {

constexpr int kGThreads = 256;
constexpr long long kGSpinLimit = 1ll << 26;
constexpr int kMaxFace = 8;  // DOFs per skeleton face
constexpr int kMaxKrylov = 8;  // flexible GMRES steps per cycle
constexpr int kSlots = 8;      // reduction slots per CTA (>= kMaxKrylov)

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
  double* kv;  // (kMaxKrylov, N): Krylov basis; v_0 holds the cycle's residual unscaled
  double* kz;  // (kMaxKrylov, N): the inner solves' results z_j = K0^-1 v_j
  double* ku;  // (N): K z_j during its orthogonalisation
  double* finv;
  double* dof_g;   // (T, 2): G0 entry of the DOF in its first and second cell
  double* ypart;   // (cell entries): a cell's preconditioned residual on its DOFs
  double* dsum;    // (T): sum of the DOF's diagonal entries over its cells' blocks
  double* cinv;    // (cell entries^2 ragged): D S_c^-1 D of every cell
  int32_t* ell_cols;  // (max_trace_row, T): trace-trace block of S, column-major ELL
  double* ell_vals;   //   (padding: the row's own column with value 0)
  int2* ent_cells;    // (cell entries): the entry's DOF's first and second cell
  double2* ent_g;     //   its G0 entries in those cells
  int2* ent_pair;     //   its flat entries in those cells (-1: none)
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
  int qvec;  // Q rows 16-byte aligned with an even length: double2 loads
  int qsmem; // the coarse vector of a Q product is staged in shared memory
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

// y = Q x, one warp per row, lanes over the columns (fixed order).  With qsmem the
// CTA first copies x into shared memory; with qvec each lane streams its columns
// as double2, four loads in flight.
__device__ void q_gemv(const GParams& P, const double* xin, double* yout) {
  extern __shared__ double2 xs2[];
  const mhm_general_system& s = P.s;
  const int M = s.cells;
  const int lane = threadIdx.x & 31;
  const int64_t wid = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int64_t nw = ((int64_t)gridDim.x * blockDim.x) >> 5;
  if (P.qsmem) {
    double* xs = reinterpret_cast<double*>(xs2);
    for (int d = threadIdx.x; d < M; d += blockDim.x) xs[d] = __ldcg(xin + d);
    __syncthreads();
  }
  if (P.qsmem && P.qvec) {
    const int H = M >> 1;
    for (int64_t c = wid; c < M; c += nw) {
      const double2* row = reinterpret_cast<const double2*>(s.coarse_inverse + c * (int64_t)M);
      double acc = 0.0;
      int d = lane;
      for (; d + 96 < H; d += 128) {
        const double2 q0 = __ldg(row + d), q1 = __ldg(row + d + 32), q2 = __ldg(row + d + 64),
                      q3 = __ldg(row + d + 96);
        const double2 x0 = xs2[d], x1 = xs2[d + 32], x2 = xs2[d + 64], x3 = xs2[d + 96];
        acc = fma(q0.x, x0.x, acc);
        acc = fma(q0.y, x0.y, acc);
        acc = fma(q1.x, x1.x, acc);
        acc = fma(q1.y, x1.y, acc);
        acc = fma(q2.x, x2.x, acc);
        acc = fma(q2.y, x2.y, acc);
        acc = fma(q3.x, x3.x, acc);
        acc = fma(q3.y, x3.y, acc);
      }
      for (; d < H; d += 32) {
        const double2 q0 = __ldg(row + d), x0 = xs2[d];
        acc = fma(q0.x, x0.x, acc);
        acc = fma(q0.y, x0.y, acc);
      }
      acc = warp_sum(acc);
      if (lane == 0) yout[c] = acc;
    }
    return;
  }
  const double* xs = reinterpret_cast<const double*>(xs2);
  for (int64_t c = wid; c < M; c += nw) {
    const double* row = s.coarse_inverse + c * (int64_t)M;
    double acc = 0.0;
    if (P.qsmem)
      for (int d = lane; d < M; d += 32) acc = fma(__ldg(row + d), xs[d], acc);
    else
      for (int d = lane; d < M; d += 32) acc = fma(__ldg(row + d), __ldcg(xin + d), acc);
    acc = warp_sum(acc);
    if (lane == 0) yout[c] = acc;
  }
}

// q_i = sum_k S_ik y_k over the trace-trace ELL row of DOF i, y = z + beta p, in
// the CSR column order (chunks of eight: the loads of a chunk are all in flight).
__device__ __forceinline__ double ell_row(const GParams& P, int64_t i, double beta, const double* pc,
                                          const double* z) {
  const int64_t T = P.s.trace_size;
  const int W = P.s.max_trace_row;
  double qi = 0.0;
  for (int k0 = 0; k0 < W; k0 += 8) {
    int col[8];
    double val[8], y[8];
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (k0 + u < W) {
        col[u] = P.w.ell_cols[(int64_t)(k0 + u) * T + i];
        val[u] = P.w.ell_vals[(int64_t)(k0 + u) * T + i];
      }
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (k0 + u < W) y[u] = fma(beta, __ldcg(pc + col[u]), __ldcg(z + col[u]));
#pragma unroll
    for (int u = 0; u < 8; ++u)
      if (k0 + u < W) qi = fma(val[u], y[u], qi);
  }
  return qi;
}

// sum over the cell's entries e of cell_g0[e] * value(e, DOF), one warp per cell
// (lanes over the entries, then a warp sum): the same bits in every call.
template <class F>
__device__ __forceinline__ double cell_reduce(const mhm_general_system& s, int64_t c, int lane, F value) {
  const int64_t e0 = s.cell_ptr[c], e1 = s.cell_ptr[c + 1];
  double acc = 0.0;
  for (int64_t e = e0 + lane; e < e1; e += 32) acc = fma(s.cell_g0[e], value(e, s.cell_dofs[e]), acc);
  return warp_sum(acc);
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
    // r_i = rt_i - (G0 v)_i with the DOF's cells and entries in g0_apply's order
    const int64_t e = e0 + lane;
    const int64_t i = s.cell_dofs[e];
    const int2 cc = P.w.ent_cells[e];
    const double2 g = P.w.ent_g[e];
    double gv = g.x * __ldcg(v + cc.x);
    if (cc.y >= 0) gv = fma(g.y, __ldcg(v + cc.y), gv);
    ra = __ldcg(rt + i) - gv;
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
  {
    const int lane = threadIdx.x & 31;
    for (int64_t c = gtid >> 5; c < M; c += gstride >> 5) {
      const double acc = cellmode ? cell_reduce(s, c, lane, [&](int64_t e, int64_t) {
        const int2 pr = w.ent_pair[e];
        double y = __ldcg(w.ypart + pr.x);
        if (pr.y >= 0) y += __ldcg(w.ypart + pr.y);
        return y;
      })
                                  : cell_reduce(s, c, lane, [&](int64_t, int64_t i) { return __ldcg(w.z0 + i); });
      if (lane == 0) w.w2[c] = acc;
    }
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
  // the trace-trace block as column-major ELL, in CSR column order
  const int64_t T = s.trace_size;
  const int W = s.max_trace_row;
  for (int64_t i = gtid; i < T; i += gstride) {
    int k = 0;
    for (int64_t q = s.indptr[i]; q < s.indptr[i + 1]; ++q) {
      const int32_t j = s.indices[q];
      if (j < T && k < W) {
        w.ell_cols[(int64_t)k * T + i] = j;
        w.ell_vals[(int64_t)k * T + i] = s.values[q];
        ++k;
      }
    }
    for (; k < W; ++k) {
      w.ell_cols[(int64_t)k * T + i] = (int32_t)i;
      w.ell_vals[(int64_t)k * T + i] = 0.0;
    }
  }
  // per cell entry: its DOF's cells, G0 entries and flat entries (g0_apply's order)
  for (int64_t e = gtid; e < s.cell_entries; e += gstride) {
    const int64_t i = s.cell_dofs[e];
    const int2 c = reinterpret_cast<const int2*>(s.dof_cells)[i];
    w.ent_cells[e] = c;
    w.ent_g[e] = make_double2(s.cell_g0[s.dof_entry[2 * i]], c.y >= 0 ? s.cell_g0[s.dof_entry[2 * i + 1]] : 0.0);
    w.ent_pair[e] = make_int2((int)s.dof_entry[2 * i], c.y >= 0 ? (int)s.dof_entry[2 * i + 1] : -1);
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

// z = K0^-1 v (v = ib * isc): lambda0 = G0 Q (-v_c), projected PCG on the trace part,
// c = Q G0^T (S lambda - v_lambda).  Returns the solve status (barrier timeouts and
// breakdowns end it early).
__device__ __forceinline__ int inner_solve(const GParams& P, const double* ib, double isc, double* zj, double need,
                                        unsigned& epoch, int& total_inner) {
  __shared__ double red[32];
  __shared__ double sh[kSlots];
  const mhm_general_system& s = P.s;
  const GWork& w = P.w;
  const int64_t T = s.trace_size;
  const int M = s.cells;
  const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
  const int lane = threadIdx.x & 31;
  const int64_t gwarp = gtid >> 5, nwarps = gstride >> 5;
  double tot[kSlots];
  int status = MHM_SOLVE_OK;
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
  // ---- inner solve z_j = K0^-1 v_j: lambda0 = G0 Q (-v_c) ------------------------
  for (int64_t c = gtid; c < M; c += gstride) w.w[c] = -__ldcg(ib + T + c) * isc;
  GSYNC();
  q_gemv(P, w.w, w.v);
  GSYNC();
  for (int64_t i = gtid; i < T; i += gstride) {
    w.lam0[i] = g0_apply(s, w.dof_g, i, w.v);
    w.mu[i] = 0.0;
    w.p[0][i] = 0.0;
  }
  GSYNC();
  // initial residual rt = v_lambda - S lambda0 (trace-trace block of K)
  for (int64_t i = gtid; i < T; i += gstride) w.rt[0][i] = __ldcg(ib + i) * isc - ell_row(P, i, 0.0, w.lam0, w.lam0);
  GSYNC();
  // projection and preconditioning of the initial residual
  for (int64_t c = gwarp; c < M; c += nwarps) {
    const double acc = cell_reduce(s, c, lane, [&](int64_t, int64_t i) { return __ldcg(w.rt[0] + i); });
    if (lane == 0) w.w[c] = acc;
  }
  GSYNC();
  q_gemv(P, w.w, w.v);
  GSYNC();
  PRECONDITION(w.rt[0]);
  q_gemv(P, w.w2, w.v2);
  GSYNC();
  double gamma;
  {
    double rz = 0.0;
    for (int64_t i = gtid; i < T; i += gstride) {
      const double zi = __ldcg(w.z0 + i) - g0_apply(s, w.dof_g, i, w.v2);
      w.z[i] = zi;
      rz = fma(__ldcg(w.r + i), zi, rz);
    }
    g_partial(w, 0, rz, red);
  }
  GSYNC();
  g_totals(w, 1, tot, sh);
  gamma = tot[0];
  {
    // stop once the preconditioned residual norm (r, z)^1/2 fell by inner_rtol, or
    // by `need` (inexact Krylov: later steps need less)
    const double target = fmax(P.inner_rtol, need) * sqrt(fmax(gamma, 0.0));
    double beta = 0.0;
    int cur = 0;
    while (sqrt(fmax(gamma, 0.0)) > target && total_inner < P.max_inner) {
      if (!(gamma > 0.0)) { status = MHM_SOLVE_BREAKDOWN; goto done; }
      const int nxt = cur ^ 1;
      // P1: direction p = z + beta p_prev, q = S p
      {
        double pq = 0.0;
        for (int64_t i = gtid; i < T; i += gstride) {
          const double pi = fma(beta, __ldcg(w.p[cur] + i), __ldcg(w.z + i));
          const double qi = ell_row(P, i, beta, w.p[cur], w.z);
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
      for (int64_t c = gwarp; c < M; c += nwarps) {
        const double acc = cell_reduce(s, c, lane, [&](int64_t, int64_t i) {
          return fma(-alpha, __ldcg(w.q + i), __ldcg(w.rt[cur] + i));
        });
        if (lane == 0) w.w[c] = acc;
      }
      GSYNC();
      // P3: v = Q G0^T rt
      q_gemv(P, w.w, w.v);
      GSYNC();
      // P4: r = P rt, z0 = M^-1 r; the cells' G0^T z0 (two barriers)
      PRECONDITION(w.rt[nxt]);
      // P5: v2 = Q G0^T z0
      q_gemv(P, w.w2, w.v2);
      GSYNC();
      // P6: z = P z0; (r, z)
      {
        double rz = 0.0;
        for (int64_t i = gtid; i < T; i += gstride) {
          const double zi = __ldcg(w.z0 + i) - g0_apply(s, w.dof_g, i, w.v2);
          w.z[i] = zi;
          rz = fma(__ldcg(w.r + i), zi, rz);
        }
        g_partial(w, 0, rz, red);
      }
      GSYNC();
      g_totals(w, 1, tot, sh);
      beta = tot[0] / gamma;
      gamma = tot[0];
      if (!isfinite(gamma)) { status = MHM_SOLVE_NONFINITE; goto done; }
      cur = nxt;
      ++total_inner;
    }
  }
  // coarse unknowns c = Q G0^T (S lambda - v_lambda); z_j = (lambda0 + mu, c)
  for (int64_t i = gtid; i < T; i += gstride) {
    const double li = __ldcg(w.lam0 + i) + __ldcg(w.mu + i);
    w.q[i] = ell_row(P, i, 1.0, w.mu, w.lam0) - __ldcg(ib + i) * isc;
    zj[i] = li;
  }
  GSYNC();
  for (int64_t c = gwarp; c < M; c += nwarps) {
    const double acc = cell_reduce(s, c, lane, [&](int64_t, int64_t i) { return __ldcg(w.q + i); });
    if (lane == 0) w.w[c] = acc;
  }
  GSYNC();
  q_gemv(P, w.w, w.v);
  GSYNC();
  for (int64_t c = gtid; c < M; c += gstride) zj[T + c] = __ldcg(w.v + c);
  GSYNC();
done:
  return status;
#undef GSYNC
#undef PRECONDITION
}

// u = K z_j over all rows, then classical Gram-Schmidt of u against v_0..v_j, twice
// (v_0 scaled by 1 / beta0 on read); h[0..j] the projections, h[j+1] = ||u||, u left
// in ku.  False when a grid barrier timed out.
__device__ __noinline__ bool orthogonalise(const GParams& P, const double* zj, int j, double beta0, double* h,
                                           unsigned& epoch) {
  __shared__ double red[32];
  __shared__ double sh[kSlots];
  const mhm_general_system& s = P.s;
  const GWork& w = P.w;
  const int64_t N = s.size;
  const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
  double tot[kSlots];
#define GSYNC()                          \
  do {                                   \
    if (!g_sync(w, epoch)) return false; \
  } while (0)
  // ---- u = K z_j (all rows), then classical Gram-Schmidt against v_0..v_j, twice --
  for (int64_t i = gtid; i < N; i += gstride) {
    double acc = 0.0;
    for (int64_t k = s.indptr[i]; k < s.indptr[i + 1]; ++k)
      acc = fma(s.values[k], __ldcg(zj + s.indices[k]), acc);
    w.ku[i] = acc;
  }
  GSYNC();
  for (int k = 0; k <= j + 1; ++k) h[k] = 0.0;
  for (int pass = 0; pass < 2; ++pass) {
    {
      double d[kMaxKrylov];
      for (int k = 0; k <= j; ++k) d[k] = 0.0;
      for (int64_t i = gtid; i < N; i += gstride) {
        const double u = __ldcg(w.ku + i);
        for (int k = 0; k <= j; ++k) d[k] = fma(__ldcg(w.kv + (int64_t)k * N + i) * (k == 0 ? 1.0 / beta0 : 1.0), u, d[k]);
      }
      for (int k = 0; k <= j; ++k) g_partial(w, k, d[k], red);
    }
    GSYNC();
    g_totals(w, j + 1, tot, sh);
    for (int k = 0; k <= j; ++k) h[k] += tot[k];
    {
      double n2 = 0.0;
      for (int64_t i = gtid; i < N; i += gstride) {
        double u = __ldcg(w.ku + i);
        for (int k = 0; k <= j; ++k)
          u = fma(-tot[k], __ldcg(w.kv + (int64_t)k * N + i) * (k == 0 ? 1.0 / beta0 : 1.0), u);
        w.ku[i] = u;
        n2 = fma(u, u, n2);
      }
      if (pass == 1) g_partial(w, 0, n2, red);
    }
    GSYNC();
  }
  g_totals(w, 1, tot, sh);
  h[j + 1] = sqrt(tot[0]);
  return true;
#undef GSYNC
}

__global__ void __launch_bounds__(kGThreads, 1) general_pcg_kernel(const GParams P) {
  __shared__ double red[32];
  __shared__ double sh[kSlots];
  const mhm_general_system& s = P.s;
  const GWork& w = P.w;
  const int64_t N = s.size;
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
  // ---- flexible GMRES on K, right-preconditioned by inner solves of K0 -----------
  // Each cycle starts from the true residual; step j solves K0 z_j = v_j by projected
  // PCG, orthogonalises K z_j against the basis (classical Gram-Schmidt, twice) and
  // updates the Givens-rotated least-squares problem.  Where K - K0 is at rounding
  // level this takes the two steps the plain defect correction took; where a few
  // cells' coupling or coarse terms differ from G0 and 0 (corrected cells), K0^-1 K
  // is the identity plus a low-rank term and the cycle still converges.
  __shared__ double kr[kMaxKrylov + 1][kMaxKrylov];  // R (upper triangle) of the cycle
  __shared__ double kcs[kMaxKrylov], ksn[kMaxKrylov], kg[kMaxKrylov + 1], ky[kMaxKrylov];
  for (;;) {
    // ---- true residual v0 = b - K x over all rows, its norm and the componentwise
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
        w.kv[i] = acc;
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
    const double beta0 = sqrt(tot[0]);
    if (threadIdx.x == 0) {
      kg[0] = beta0;
      for (int k = 1; k <= kMaxKrylov; ++k) kg[k] = 0.0;
    }
    __syncthreads();
    int steps = 0;
    for (int j = 0; j < kMaxKrylov; ++j) {
      const double* ib = w.kv + (int64_t)j * N;  // v_j (v_0 scaled by 1 / beta0 on read)
      const double isc = j == 0 ? 1.0 / beta0 : 1.0;
      double* zj = w.kz + (int64_t)j * N;
      const double est = fabs(kg[j]);
      ++outer;
      ++steps;
      {
        // the componentwise error is taken to shrink with the cycle's residual estimate
        // (omega was measured at the cycle's start, where the estimate is beta0)
        const double need = 0.1 * fmin(P.rtol * bnorm / est, P.rtol / (omega * (est / beta0)));
        status = inner_solve(P, ib, isc, zj, need, epoch, total_inner);
        if (status != MHM_SOLVE_OK) goto done;
      }
      double h[kMaxKrylov + 1];
      if (!orthogonalise(P, zj, j, beta0, h, epoch)) { status = MHM_SOLVE_BARRIER_TIMEOUT; goto done; }
      if (!isfinite(h[j + 1])) { status = MHM_SOLVE_NONFINITE; goto done; }
      // ---- Givens rotations of the new column (every CTA, the same bits) ---------------
      if (threadIdx.x == 0) {
        for (int k = 0; k < j; ++k) {
          const double a = kcs[k] * h[k] + ksn[k] * h[k + 1];
          h[k + 1] = -ksn[k] * h[k] + kcs[k] * h[k + 1];
          h[k] = a;
        }
        const double den = hypot(h[j], h[j + 1]);
        kcs[j] = den > 0.0 ? h[j] / den : 1.0;
        ksn[j] = den > 0.0 ? h[j + 1] / den : 0.0;
        for (int k = 0; k < j; ++k) kr[k][j] = h[k];
        kr[j][j] = den;
        kg[j + 1] = -ksn[j] * kg[j];
        kg[j] = kcs[j] * kg[j];
      }
      __syncthreads();
      const double next = fabs(kg[j + 1]);
      const bool last = next <= 0.1 * P.rtol * bnorm || !(h[j + 1] > 0.0) || j + 1 == kMaxKrylov ||
                        outer >= P.max_outer || total_inner >= P.max_inner;
      if (!last) {
        double* vn = w.kv + (int64_t)(j + 1) * N;
        const double inv = 1.0 / h[j + 1];
        for (int64_t i = gtid; i < N; i += gstride) vn[i] = __ldcg(w.ku + i) * inv;
        GSYNC();
        continue;
      }
      break;
    }
    // ---- x += Z y with R y = g (back substitution, every CTA) ------------------------
    if (threadIdx.x == 0) {
      for (int k = steps - 1; k >= 0; --k) {
        double a = kg[k];
        for (int l = k + 1; l < steps; ++l) a = fma(-kr[k][l], ky[l], a);
        ky[k] = kr[k][k] != 0.0 ? a / kr[k][k] : 0.0;
      }
    }
    __syncthreads();
    for (int64_t i = gtid; i < N; i += gstride) {
      double a = P.x[i];
      for (int k = 0; k < steps; ++k) a = fma(ky[k], __ldcg(w.kz + (int64_t)k * N + i), a);
      P.x[i] = a;
    }
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
}

struct GLayout {
  size_t mu, rt0, rt1, p0, p1, q, r, z0, z, lam0, w, v, w2, v2, kv, kz, ku, finv, dof_g, ypart, dsum, cinv, ell_cols,
      ell_vals, ent_cells, ent_g, ent_pair, part, bar, err, total;
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
  L.kv = take(N * 8 * kMaxKrylov);
  L.kz = take(N * 8 * kMaxKrylov);
  L.ku = take(N * 8);
  L.finv = take((size_t)s->faces * kMaxFace * kMaxFace * 8);
  L.dof_g = take(T * 2 * 8);
  L.ypart = take((size_t)s->cell_entries * 8);
  L.dsum = take(T * 8);
  L.cinv = take((size_t)(s->block_off ? s->blocks_size : 1) * 8);
  L.ell_cols = take((size_t)s->max_trace_row * T * 4);
  L.ell_vals = take((size_t)s->max_trace_row * T * 8);
  L.ent_cells = take((size_t)s->cell_entries * 8);
  L.ent_g = take((size_t)s->cell_entries * 16);
  L.ent_pair = take((size_t)s->cell_entries * 8);
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
         s->trace_size <= INT32_MAX && s->cell_entries >= 1 && s->cell_entries <= INT32_MAX &&
         s->max_trace_row >= 1 && s->max_trace_row <= 1024 &&
         (!s->block_off || (s->blocks_size >= 1 && s->max_cell_dofs >= 1 && s->max_cell_dofs <= 32)) &&
         (!s->cell_blocks || s->block_off);
}

// Dynamic shared memory of the solve: the coarse vector of a Q product, when it fits.
constexpr size_t kQSmemMax = 192 * 1024;
size_t g_smem(const mhm_general_system* s) {
  const size_t bytes = (size_t)s->cells * sizeof(double);
  return bytes <= kQSmemMax ? bytes : 0;
}

int g_grid(size_t smem) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  if (cudaFuncSetAttribute(general_pcg_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
      cudaSuccess)
    return -1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, general_pcg_kernel, kGThreads, smem) != cudaSuccess)
    return -1;
  if (per_sm < 1) return 0;
  return sms;  // one CTA per SM: all co-resident for the cooperative launch
}

}  // namespace
}  // namespace mhm

using namespace mhm;

extern "C" int64_t mhm_general_workspace_bytes(const mhm_general_system* s) {
  if (!g_valid_layout(s)) return -1;
  const int grid = g_grid(g_smem(s));
  if (grid <= 0) return -1;
  return (int64_t)g_layout(s, grid).total;
}

extern "C" int mhm_general_solve(const mhm_general_system* s, const double* rhs, double* x, void* workspace,
                                 int64_t workspace_bytes, double rtol, double inner_rtol, int32_t max_inner,
                                 int32_t max_outer, int32_t* info, double* stats, void* stream) {
  if (!g_valid_layout(s) || !s->values || !rhs || !x || !workspace || !info || !stats || !(rtol > 0.0) || !(inner_rtol > 0.0) ||
      max_inner < 1 || max_outer < 1)
    return MHM_ERR_ARGUMENT;
  const size_t smem = g_smem(s);
  const int grid = g_grid(smem);
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
  P.w.kv = d(L.kv);
  P.w.kz = d(L.kz);
  P.w.ku = d(L.ku);
  P.w.finv = d(L.finv);
  P.w.dof_g = d(L.dof_g);
  P.w.ypart = d(L.ypart);
  P.w.dsum = d(L.dsum);
  P.w.cinv = d(L.cinv);
  P.w.ell_cols = reinterpret_cast<int32_t*>(base + L.ell_cols);
  P.w.ell_vals = d(L.ell_vals);
  P.w.ent_cells = reinterpret_cast<int2*>(base + L.ent_cells);
  P.w.ent_g = reinterpret_cast<double2*>(base + L.ent_g);
  P.w.ent_pair = reinterpret_cast<int2*>(base + L.ent_pair);
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
  P.qsmem = smem > 0;
  P.qvec = (s->cells % 2 == 0) && (reinterpret_cast<uintptr_t>(s->coarse_inverse) % 16 == 0);
  if (cudaMemsetAsync(base + L.bar, 0, L.total - L.bar, st) != cudaSuccess) return MHM_ERR_LAUNCH;
  general_setup_kernel<<<grid * 2, 256, 0, st>>>(P);
  if (s->cell_blocks) general_cell_inverse_kernel<<<grid * 2, 256, 0, st>>>(P);
  void* args[] = {&P};
  if (cudaLaunchCooperativeKernel((const void*)general_pcg_kernel, grid, kGThreads, args, smem, st) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}
