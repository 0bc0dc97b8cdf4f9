// Global skeleton system: ordered reduction of the cell blocks and the projected
// preconditioned CG solve.
//
// Reference algorithm (PyMHM 1.3.2, src/pymhm/):
//   assemble_hybrid_contributions   core/contributions.py:77-195, core/_assembly.py:10-42
//   solve_hybrid_system             core/system.py:355-528 (SuperLU at rtol 1e-10 there)
//
// The global unknown is (lambda, c): skeleton traces and one retained constant per
// macrocell.  Its operator is the symmetric saddle K = [[S, -G], [-G^T, -C]] with
// C at rounding level.  The solver here is an outer FP64 defect correction on K
// (residuals from the assembled CSR matrix) whose inner solve is a FETI-style
// projected CG on
//     K0 = [[S, -G0], [-G0^T, 0]],
// G0 the exact geometric net-flux operator of the Cartesian macro grid.
// G0^T G0 = ay (T_y (x) I) + ax (I (x) T_x) is a scaled 2-D Dirichlet Laplacian
// on the macro cells; it is inverted exactly by an orthonormal sine transform
// along x (Q), the inverse of one tridiagonal Toeplitz matrix along y per sine
// mode (closed form through Chebyshev polynomials of the second kind), and the
// inverse transform.  K - K0 is at rounding level, so two or three outer
// corrections reach FP64 accuracy.
//
// Cell form.  S = sum_c R_c^T S_c R_c over macrocells c (S_c the t x t trace
// block each cell contributes), so S u is applied as per-cell products S_c u_c
// whose face partials are summed per DOF (first cell + second cell, a fixed
// order).  With the cells' own blocks available the preconditioner is the
// cell-Dirichlet one, M^-1 = sum_c R_c^T D_c S_c^-1 D_c R_c with stiffness
// weights D_c,a = S_c,aa / sum_{c' containing the DOF} S_c',a'a'.  From an
// assembled matrix alone, S is split exactly into cell parts (entries of a face
// shared by two cells halved) and the preconditioner is additive Schwarz over
// the cells' principal t x t submatrices.
//
// The inner CG uses the single-reduction recurrence of Chronopoulos and Gear
// (J. Comput. Appl. Math. 25 (1989) 153-168): with u = P M^-1 r and w = S u,
//   gamma = (r, u), delta = (u, w), beta = gamma / gamma_prev,
//   alpha = gamma / (delta - beta gamma / alpha_prev),
//   p = u + beta p, P S p = P w + beta P S p_prev, r -= alpha P S p,
// P = I - G0 (G0^T G0)^-1 G0^T.  Every kReproject iterations r and P S p are
// projected again, which removes the drift of the recurrences out of range(P).
//
// Everything runs in one persistent cooperative kernel with one CTA per macro
// row.  CTA r owns the DOFs first met by the cells of row r (a contiguous range
// in the reference's numbering) and keeps the iteration vectors on the DOFs of
// its own cells (owned DOFs plus the bottom faces).  A coarse solve takes two
// steps between grid barriers: row owners transform their rows along x (their
// cells' partials also reach the two neighbouring rows through the shared
// faces); then CTA k solves sine mode k along y for all rows; the row owners
// read back the three rows they need.  Every cross-CTA value a step reads
// arrives in one batch of loads after a barrier.  The barrier is a monotonic
// arrival counter with a bounded spin: on timeout every CTA sets the error flag
// and returns (MHM_SOLVE_BARRIER_TIMEOUT).
#include <cmath>

#include "mhm_common.cuh"

namespace mhm {
namespace {

constexpr int kSolveThreads = 512;
constexpr int kWarps = kSolveThreads / 32;
constexpr int kReproject = 16;
constexpr long long kSpinLimit = 1ll << 26;

struct Sys {
  int64_t N, T;
  const int64_t* indptr;
  const int32_t* indices;
  const double* values;
  const int64_t* trace_end;
  int F, fs, M, t;
  const int64_t* cell_dofs;
  const double* g0;
  const int32_t* dof_cells;
  const int32_t* dof_slot;
  int nx, ny;
  double ax, ay;
  const double* blocks;
  int ld;
  const uint8_t* fixed;  // T: 1 = fixed trace DOF (null: none)
  int yneu;              // coarse T_y ends: bit 0 bottom, bit 1 top Neumann
  const double* qx;      // nx x nx eigenvectors [k][i] of the coarse T_x (null: the sine basis)
  const double* lamx;    // nx eigenvalues of T_x (with qx)
  const double* pinv0;   // ny x ny pseudo-inverse of mode 0's T_y when every side is fixed (else null)
  // Neumann faces on part of a side: the coarse operator is the separable one less
  // E D E^T on wbm boundary cells; y = A_sep^-1 r is corrected by wbR (E^T y)
  int wbm;
  const int32_t* wbcell;  // wbm cells
  const double* wbR;      // cells x wbm, [cell][l]
};

// Row-transformed coarse data of one quantity, layout [mode][row]:
// U = self + below + above, `below` written by the CTA of row-1 and `above` by
// the CTA of row+1 (null: absent).
struct Coarse {
  double *self, *below, *above;
};

struct Work {
  double *Zf, *Zs, *Vf, *Vs;       // T each: per-DOF partials of the first / second cell
  Coarse Uz, Uw;                   // M each part
  double *Ux1, *Ux2;               // M each: coarse data of DOF vectors
  double *Wz, *Ww, *Wx1, *Wx2;     // M each, [row][mode]: solved coarse data
  double* rfull;                   // N: outer residual
  double* part;                    // grid * 4 partial sums
  unsigned* bar;                   // arrival counter
  int* err;
};

struct Params {
  Sys s;
  Work w;
  const double* rhs;
  const double* load_scale;
  double* x;
  double rtol, inner_rtol;
  int max_inner, max_outer;
  int32_t* info;
  double* stats;
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
  unsigned v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}

__device__ __forceinline__ void red_release_add(unsigned* p, unsigned v) {
  asm volatile("red.release.gpu.global.add.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Bounded grid barrier on a monotonic arrival counter (zeroed by the host before
// the launch): arrival k of every CTA completes when the counter reaches
// k * gridDim.x.  Returns false when the error flag is set.
__device__ bool grid_sync(const Work& w, unsigned& epoch) {
  __shared__ int bad;
  __syncthreads();
  ++epoch;
  if (threadIdx.x == 0) {
    const unsigned target = epoch * gridDim.x;
    // the release orders every write of the CTA before the bar.sync above
    red_release_add(w.bar, 1u);
    long long spins = 0;
    while (ld_acquire(w.bar) < target) {
      if (++spins > kSpinLimit) {
        atomicExch(w.err, 1);
        break;
      }
      // another CTA gave up: it will not arrive
      if ((spins & 1023) == 0 && *reinterpret_cast<volatile int*>(w.err) != 0) break;
      if (spins > 64) __nanosleep(20);
    }
    bad = *reinterpret_cast<volatile int*>(w.err);
  }
  __syncthreads();
  return bad == 0;
}

// Sums of the per-CTA partials in slots [slot, slot + NS) (fixed order, identical
// in every CTA); the loads of all slots are issued together.
template <int NS>
__device__ void grid_totals(const Work& w, int slot, double (&out)[NS], double* sh) {
  if (threadIdx.x < 32) {
    double v[NS][4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = threadIdx.x + 32 * q;
#pragma unroll
      for (int n = 0; n < NS; ++n) v[n][q] = i < (int)gridDim.x ? __ldcg(w.part + i * 4 + slot + n) : 0.0;
    }
    for (int i0 = threadIdx.x + 128; i0 < (int)gridDim.x; i0 += 32)
#pragma unroll
      for (int n = 0; n < NS; ++n) v[n][0] += __ldcg(w.part + i0 * 4 + slot + n);
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      const double a = warp_sum((v[n][0] + v[n][1]) + (v[n][2] + v[n][3]));
      if (threadIdx.x == 0) sh[n] = a;
    }
  }
  __syncthreads();
#pragma unroll
  for (int n = 0; n < NS; ++n) out[n] = sh[n];
  __syncthreads();
}

__device__ double grid_total(const Work& w, int slot, double* sh) {
  double o[1];
  grid_totals<1>(w, slot, o, sh);
  return o[0];
}

__device__ void put_partial(const Work& w, int slot, double v, double* red) {
  v = block_sum(v, red);
  if (threadIdx.x == 0) w.part[blockIdx.x * 4 + slot] = v;
}

// Two partials in one block reduction (red >= 64 doubles).
__device__ void put_partial2(const Work& w, int slot, double a, double b, double* red) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  __syncthreads();
  if (lane == 0) {
    red[wid] = a;
    red[32 + wid] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double sa = 0.0, sb = 0.0;
    for (int i = 0; i < nw; ++i) {
      sa += red[i];
      sb += red[32 + i];
    }
    w.part[blockIdx.x * 4 + slot] = sa;
    w.part[blockIdx.x * 4 + slot + 1] = sb;
  }
}

__device__ __forceinline__ double krow(const Sys& s, int64_t i, const double* v) {
  double acc = 0.0;
  for (int64_t e = s.indptr[i]; e < s.indptr[i + 1]; ++e) acc = fma(s.values[e], __ldcg(v + s.indices[e]), acc);
  return acc;
}

// S[i][j] of the assembled CSR (0 when the entry is not stored).
__device__ double csr_entry(const Sys& s, int64_t i, int64_t j) {
  int64_t lo = s.indptr[i], hi = s.indptr[i + 1];
  while (lo < hi) {
    const int64_t mid = (lo + hi) / 2;
    const int64_t c = s.indices[mid];
    if (c == j) return s.values[mid];
    if (c < j) lo = mid + 1; else hi = mid;
  }
  return 0.0;
}

// Row stride of the shared-memory sine transform: = 4 (mod 16) doubles, so the four
// rows that a half-warp reads in one transform step fall in disjoint banks.
__host__ __device__ inline int q_stride(int nx) { return nx + ((4 - nx % 16) + 16) % 16; }

// Per-CTA state.  CTA r owns macro row r and the DOFs [d0, d1) first met in it.
// Local DOFs ("G"): l < nown are the owned DOFs d0 + l; l >= nown (rows r > 0)
// are the bottom faces of the row's cells, nown + cx * fs + j.  These are all
// the DOFs of the row's cells; their cells lie in rows r-1 .. r+1, whose coarse
// values are kept in yrow slots 0..2 (slot = row - r + 1).  The CTA also solves
// sine modes blockIdx.x + j * gridDim.x (Chebyshev tables in mcheb).
struct Row {
  int r, c0, nown, ng, qs, nmode;
  int64_t d0, d1;
  double* Q;      // nx x qs: Q[k][i] = sqrt(2/(nx+1)) sin(pi (k+1)(i+1) / (nx+1))
  double* yrow;   // 3 nx
  double* col;    // 12 nx: faces' coarse sums across (1-4) and to the cell (8-11); combined (5)
  double* wrow;   // 3 nx
  double* mcheb;  // nmode 2 (ny + 1): U_m(theta_k); with Neumann ends u then v (see mode_solve)
  double* mcinv;  // nmode: 1 / (ay U_ny(theta_k)), or 1 / C
  double* ucol;   // ny
  double *vr, *vps, *vp, *vlam, *vu, *vt;  // G vectors: r, P S p, p, lambda, u, staging
  double* Sb;     // nx np: packed symmetric S_c
  double* Pb;     // nx np: packed symmetric preconditioner block
  double *ga, *gb;  // G: G0 coefficient of the first / second cell
  int16_t *ya, *yb; // G: yrow index of the first / second cell (second: -1 = none)
  int32_t* gdof;    // G: global DOF
  // per cell slot, stored [slot][cell] so that the lanes of a warp (one cell each)
  // read consecutive entries:
  int16_t* cl;      // t nx: local DOF
  double* gself;    // t nx: g0 of the cell on the slot
  double* gnb;      // t nx: g0 of the other cell on the same DOF (0: none)
  uint8_t* role;    // t nx: bit 0 = the cell is the DOF's second cell, bit 1 = the DOF has two cells
  double* wbe;      // fixed-DOF instantiation: y at the Woodbury cells (2 (nx + ny))
  double* scratch;  // kWarps t t (aliases the G vectors during setup)
};

__device__ __forceinline__ double g0y(const Row& R, int l) {
  double v = R.ga[l] * R.yrow[R.ya[l]];
  const int b = R.yb[l];
  if (b >= 0) v = fma(R.gb[l], R.yrow[b], v);
  return v;
}

// Packed index of (i, j) in a symmetric T x T block stored by upper rows.
template <int T>
__host__ __device__ __forceinline__ constexpr int packed(int a, int b) {
  return a < b ? a * T - (a * (a - 1)) / 2 + (b - a) : b * T - (b * (b - 1)) / 2 + (a - b);
}

// Distance between the packed blocks of consecutive cells: T (T + 1) / 2 rounded up
// to an odd count of doubles, so that the lanes of a warp (one cell each) read
// distinct shared-memory banks.
__host__ __device__ __forceinline__ constexpr int block_stride(int t) { return (t * (t + 1) / 2) | 1; }

// out(j, i, v): v = sum_k in[j][k] Q[k][i] (TR: Q[i][k]) for j < nin (in[j] in
// shared memory), i < nx.  Q[cell][mode] holds the coarse T_x eigenvectors, so the
// forward transform reads it as is and the inverse transposed (the sine basis is
// symmetric; a host table with Neumann x-ends is not).  Warp w takes columns
// 4w .. 4w+3 (repeating every 64); lane bits 2-4 split k eight ways, reduced by
// shuffles.
template <bool TR = false, typename F>
__device__ void sine_apply(const Row& R, int nx, int nin, const double* const* in, F out) {
  const int lane = threadIdx.x & 31, q = lane >> 2;
  for (int base = (threadIdx.x >> 5) * 4; base < nx; base += kWarps * 4) {
    const int i = base + (lane & 3);
    double acc[3] = {0.0, 0.0, 0.0};
    if (i < nx) {
      const double* qc = R.Q + i;
#pragma unroll 4
      for (int k = q; k < nx; k += 8) {
        const double qv = TR ? R.Q[i * R.qs + k] : qc[k * R.qs];
#pragma unroll
        for (int j = 0; j < 3; ++j)
          if (j < nin) acc[j] = fma(in[j][k], qv, acc[j]);
      }
    }
#pragma unroll
    for (int j = 0; j < 3; ++j) {
      acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], 4);
      acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], 8);
      acc[j] += __shfl_xor_sync(0xffffffffu, acc[j], 16);
    }
    if (i < nx && q == 0)
      for (int j = 0; j < nin; ++j) out(j, i, acc[j]);
  }
}

// Row transform of nin column vectors R.col + src[j] nx into dst[j] at row
// R.r + shift[j] (layout [mode][row]; null dst: skipped).
__device__ void coarse_rowfwd(const Sys& s, const Row& R, int nin, const int* src, double* const* dst,
                              const int* shift) {
  __syncthreads();
  const double* in[3] = {R.col + src[0] * s.nx, R.col + src[nin > 1 ? 1 : 0] * s.nx,
                         R.col + src[nin > 2 ? 2 : 0] * s.nx};
  sine_apply(R, s.nx, nin, in, [&](int j, int k, double v) {
    if (dst[j]) dst[j][(size_t)k * s.ny + R.r + shift[j]] = v;
  });
}

__device__ void coarse_rowfwd1(const Sys& s, const Row& R, double* dst) {
  const int src[1] = {0};
  double* const d[1] = {dst};
  const int sh[1] = {0};
  coarse_rowfwd(s, R, 1, src, d, sh);
}

// After every row's coarse data is written: for each sine mode k this CTA owns,
// W[ir][k] = sum_iy Tinv_k[ir][iy] U[k][iy] for every row ir, with
// Tinv_k[i][j] = U_i U_{ny-1-j} / (ay U_ny) for i <= j (U the mode's Chebyshev
// values; symmetric).  With Neumann ends (whole bottom / top sides fixed) the end
// rows of T_k lose one neighbour and Tinv_k[i][j] = u_i v_j / C for i <= j, u and v
// the solutions of the homogeneous recurrence from the bottom and the top end.
// NEU: the solve may have fixed DOFs (compile-time switch; the Dirichlet-only
// instantiation carries none of their code).
template <bool NEU>
__device__ void mode_solve(const Sys& s, const Row& R, const Coarse& U, double* W) {
  const int ny = s.ny, nx = s.nx;
  for (int j = 0; j < R.nmode; ++j) {
    const int k = blockIdx.x + j * gridDim.x;
    __syncthreads();
    for (int iy = threadIdx.x; iy < ny; iy += blockDim.x) {
      const size_t at = (size_t)k * ny + iy;
      const double v0 = __ldcg(U.self + at);
      const double v1 = (iy > 0 && U.below) ? __ldcg(U.below + at) : 0.0;
      const double v2 = (iy < ny - 1 && U.above) ? __ldcg(U.above + at) : 0.0;
      R.ucol[iy] = (v0 + v1) + v2;
    }
    __syncthreads();
    const double* u = R.mcheb + (size_t)j * (NEU ? 2 : 1) * (ny + 1);
    const double* v = u + (ny + 1);
    const double c = R.mcinv[j];
    const int lane8 = threadIdx.x & 7, grp = threadIdx.x >> 3, ngrp = blockDim.x >> 3;
    for (int base = 0; base < ny; base += ngrp) {
      const int ir = base + grp;
      double acc = 0.0;
      if (ir < ny) {
        if (NEU && s.pinv0 && k == 0) {
          const double* prow = s.pinv0 + (size_t)ir * ny;
          for (int iy = lane8; iy < ny; iy += 8) acc = fma(__ldg(prow + iy), R.ucol[iy], acc);
        } else if (!NEU || s.yneu == 0) {
          const double uir = u[ir], unir = u[ny - 1 - ir];
          for (int iy = lane8; iy < ny; iy += 8)
            acc = fma((ir < iy ? uir * u[ny - 1 - iy] : u[iy] * unir), R.ucol[iy], acc);
        } else {
          const double uir = u[ir], vir = v[ir];
          for (int iy = lane8; iy < ny; iy += 8)
            acc = fma((ir <= iy ? uir * v[iy] : u[iy] * vir), R.ucol[iy], acc);
        }
      }
      acc += __shfl_xor_sync(0xffffffffu, acc, 4);
      acc += __shfl_xor_sync(0xffffffffu, acc, 2);
      acc += __shfl_xor_sync(0xffffffffu, acc, 1);
      if (ir < ny && lane8 == 0) W[(size_t)ir * nx + k] = acc * c;
    }
  }
}

// Neumann faces on part of a side (fixed-DOF instantiation): the coarse operator is
// A = A_sep - E D E^T, A_sep the separable operator with those sides taken as
// Dirichlet and E the wbm boundary cells that lose a face.  By the Woodbury identity
// A^-1 r = y + wbR (E^T y), y = A_sep^-1 r, wbR = A_sep^-1 E (D^-1 - E^T A_sep^-1 E)^-1.
// Every CTA forms E^T y from the solved mode data W itself (y at a cell is its row of
// W through the inverse transform), so no grid barrier is added; it then corrects its
// coarse rows [lo, hi) in yrow.
template <bool NEU>
__device__ void woodbury_rows(const Sys& s, const Row& R, const double* W, int lo, int hi) {
  if (!NEU || s.wbm == 0) return;
  const int nx = s.nx, r0 = R.r - 1;
  for (int l = threadIdx.x; l < s.wbm; l += blockDim.x) {
    const int c = s.wbcell[l], ir = c / nx, ix = c - ir * nx;
    const double* wr = W + (size_t)ir * nx;
    double acc = 0.0;
    for (int k = 0; k < nx; ++k) acc = fma(__ldcg(wr + k), s.qx ? R.Q[ix * R.qs + k] : R.Q[k * R.qs + ix], acc);
    R.wbe[l] = acc;
  }
  __syncthreads();
  for (int idx = threadIdx.x; idx < 3 * nx; idx += blockDim.x) {
    const int ir = r0 + idx / nx;
    if (ir < lo || ir >= hi) continue;
    const double* rr = s.wbR + ((size_t)ir * nx + idx % nx) * s.wbm;
    double acc = 0.0;
    for (int l = 0; l < s.wbm; ++l) acc = fma(__ldg(rr + l), R.wbe[l], acc);
    R.yrow[idx] += acc;
  }
  __syncthreads();
}

// Coarse solution rows [lo, hi) (clipped to the grid, within r-1 .. r+1) from W
// into yrow; other slots zero.  Y row = W row Q.
template <bool NEU>
__device__ void coarse_rows(const Sys& s, const Row& R, const double* W, int lo, int hi) {
  const int ny = s.ny, nx = s.nx, r0 = R.r - 1;
  if (lo < 0) lo = 0;
  if (hi > ny) hi = ny;
  __syncthreads();
  for (int idx = threadIdx.x; idx < 3 * nx; idx += blockDim.x) {
    const int ir = r0 + idx / nx;
    R.wrow[idx] = (ir >= lo && ir < hi) ? __ldcg(W + (size_t)ir * nx + idx % nx) : 0.0;
  }
  __syncthreads();
  const double* in[3] = {R.wrow, R.wrow + nx, R.wrow + 2 * nx};
  auto put = [&](int j, int i, double v) { R.yrow[j * nx + i] = v; };
  if (NEU && s.qx)
    sine_apply<true>(R, nx, 3, in, put);  // inverse transform
  else
    sine_apply<false>(R, nx, 3, in, put);
  __syncthreads();
  woodbury_rows<NEU>(s, R, W, lo, hi);
}

// Start of an inner half-step after a grid barrier: the partial sums in slots
// [slot, slot + NS), the per-DOF exchange sums Xf + Xs on the G DOFs (into out) and
// the solved coarse rows r-1 .. r+1 of W (into wrow; rows outside [0, ny) zero)
// are all loaded in one batch before any of them is used; then the coarse rows Y
// are formed.  tot receives the partial sums (identical in every CTA).
template <int NS, bool NEU>
__device__ void phase_begin(const Sys& s, const Work& w, const Row& R, int slot, double (&tot)[NS], double* sh,
                            const double* Xf, const double* Xs, double* out, const double* W) {
  const int nx = s.nx, ny = s.ny, r0 = R.r - 1, tid = threadIdx.x, nth = blockDim.x;
  __syncthreads();
  double pv[NS][4];
  if (tid < 32) {
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int i = tid + 32 * q;
#pragma unroll
      for (int n = 0; n < NS; ++n) pv[n][q] = i < (int)gridDim.x ? __ldcg(w.part + i * 4 + slot + n) : 0.0;
    }
  }
  double xa[2], xb[2], wv;
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int l = tid + q * nth;
    const int64_t i = l < R.ng ? R.gdof[l] : 0;
    xa[q] = l < R.ng ? __ldcg(Xf + i) : 0.0;
    xb[q] = l < R.ng ? __ldcg(Xs + i) : 0.0;
  }
  {
    const int ir = r0 + tid / nx;
    wv = (tid < 3 * nx && ir >= 0 && ir < ny) ? __ldcg(W + (size_t)ir * nx + tid % nx) : 0.0;
  }
  // remainders (rows wider than the block; not reached for the supported sizes)
  for (int l = tid + 2 * nth; l < R.ng; l += nth) out[l] = __ldcg(Xf + R.gdof[l]) + __ldcg(Xs + R.gdof[l]);
  for (int idx = tid + nth; idx < 3 * nx; idx += nth) {
    const int ir = r0 + idx / nx;
    R.wrow[idx] = (ir >= 0 && ir < ny) ? __ldcg(W + (size_t)ir * nx + idx % nx) : 0.0;
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int l = tid + q * nth;
    if (l < R.ng) out[l] = xa[q] + xb[q];
  }
  if (tid < 3 * nx) R.wrow[tid] = wv;
  if (tid < 32) {
    for (int i0 = tid + 128; i0 < (int)gridDim.x; i0 += 32)
#pragma unroll
      for (int n = 0; n < NS; ++n) pv[n][0] += __ldcg(w.part + i0 * 4 + slot + n);
#pragma unroll
    for (int n = 0; n < NS; ++n) {
      const double a = warp_sum((pv[n][0] + pv[n][1]) + (pv[n][2] + pv[n][3]));
      if (tid == 0) sh[n] = a;
    }
  }
  __syncthreads();
#pragma unroll
  for (int n = 0; n < NS; ++n) tot[n] = sh[n];
  const double* in[3] = {R.wrow, R.wrow + nx, R.wrow + 2 * nx};
  auto put = [&](int j, int i, double v) { R.yrow[j * nx + i] = v; };
  if (NEU && s.qx)
    sine_apply<true>(R, nx, 3, in, put);  // inverse transform
  else
    sine_apply<false>(R, nx, 3, in, put);
  __syncthreads();
  woodbury_rows<NEU>(s, R, W, 0, ny);
}

// Rows Q FS .. Q FS + FS - 1 (face Q) of one cell's product B_c v_c, with B_c
// packed symmetric at blk and v_c in xv.  The face's rows go to the per-DOF
// exchange arrays (first / second cell; skipped for null Xf) and, with `coarse`,
// into the coarse sums of the face: col[(1 + Q) nx + cx] across the face to the
// neighbour, col[(8 + Q) nx + cx] to the cell itself.  Returns the face's share of
// v_c . B_c v_c.
template <int FS, int Q, bool NEU>
__device__ __forceinline__ double face_rows(const Row& R, const double* blk, int cx, int nx,
                                            const double (&xv)[4 * FS], double* Xf, double* Xs, bool coarse) {
  constexpr int T = 4 * FS;
  double acc[FS];
#pragma unroll
  for (int j = 0; j < FS; ++j) {
    double a = 0.0;
#pragma unroll
    for (int b = 0; b < T; ++b) a = fma(blk[packed<T>(Q * FS + j, b)], xv[b], a);
    acc[j] = a;
  }
  double dot = 0.0, self = 0.0, across = 0.0;
#pragma unroll
  for (int j = 0; j < FS; ++j) {
    const int idx = (Q * FS + j) * nx + cx;
    dot = fma(xv[Q * FS + j], acc[j], dot);
    if (Xf) ((R.role[idx] & 1) ? Xs : Xf)[R.gdof[R.cl[idx]]] = (NEU && (R.role[idx] & 4)) ? 0.0 : acc[j];
    if (coarse) {
      self = fma(R.gself[idx], acc[j], self);
      across = fma(R.gnb[idx], acc[j], across);
    }
  }
  if (coarse) {
    R.col[(1 + Q) * nx + cx] = across;
    R.col[(8 + Q) * nx + cx] = self;
  }
  return dot;
}

// B_c v_c for every cell of the row (B packed symmetric, block_stride apart),
// written to the exchange arrays and, with `coarse`, reduced to the faces' coarse
// sums (see face_rows).  Warp w computes face w % 4 of cells 32 (w / 4) + lane, so
// every block index is a compile-time constant within a warp.  Returns this
// thread's part of sum_c v_c . B_c v_c.
template <int FS, bool NEU>
__device__ double cell_apply(const Sys& s, const Row& R, const double* B, const double* v, double* Xf, double* Xs,
                             bool coarse) {
  constexpr int T = 4 * FS;
  __syncthreads();
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, face = wid & 3, nx = s.nx;
  const int step = 32 * ((int)(blockDim.x >> 5) >> 2);
  double dot = 0.0;
  for (int cx = lane + 32 * (wid >> 2); cx < nx; cx += step) {
    const double* blk = B + (size_t)cx * block_stride(T);
    double xv[T];
#pragma unroll
    for (int b = 0; b < T; ++b) xv[b] = v[R.cl[b * nx + cx]];
    switch (face) {
      case 0: dot += face_rows<FS, 0, NEU>(R, blk, cx, nx, xv, Xf, Xs, coarse); break;
      case 1: dot += face_rows<FS, 1, NEU>(R, blk, cx, nx, xv, Xf, Xs, coarse); break;
      case 2: dot += face_rows<FS, 2, NEU>(R, blk, cx, nx, xv, Xf, Xs, coarse); break;
      default: dot += face_rows<FS, 3, NEU>(R, blk, cx, nx, xv, Xf, Xs, coarse); break;
    }
  }
  return dot;
}

// out[l] = Xf + Xs over the G DOFs (four loads of each array in flight per thread).
__device__ void read_exchange(const Row& R, const double* Xf, const double* Xs, double* out) {
  for (int base = threadIdx.x; base < R.ng; base += 4 * blockDim.x) {
    double a[4], b[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int l = base + q * blockDim.x;
      const int64_t i = l < R.ng ? R.gdof[l] : 0;
      a[q] = l < R.ng ? __ldcg(Xf + i) : 0.0;
      b[q] = l < R.ng ? __ldcg(Xs + i) : 0.0;
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int l = base + q * blockDim.x;
      if (l < R.ng) out[l] = a[q] + b[q];
    }
  }
}

// Row-transformed coarse data of the cell products of the last cell_apply (with
// `coarse`), minus G0^T of the G vector `minus` if given, for this row and,
// through the shared faces, rows r+1 and r-1.
__device__ void coarse_combine(const Sys& s, const Row& R, const Coarse& U, const double* minus) {
  const int nx = s.nx, t = s.t;
  __syncthreads();
  const double* own = R.col + 8 * nx;
  for (int cx = threadIdx.x; cx < nx; cx += blockDim.x) {
    double self = (own[cx] + own[nx + cx]) + (own[2 * nx + cx] + own[3 * nx + cx]);
    if (minus) {
      double m = 0.0;
      for (int a = 0; a < t; ++a) m = fma(R.gself[a * nx + cx], minus[R.cl[a * nx + cx]], m);
      self -= m;
    }
    const double from_left = cx > 0 ? R.col[2 * nx + cx - 1] : 0.0;       // right face of cx-1
    const double from_right = cx + 1 < nx ? R.col[4 * nx + cx + 1] : 0.0;  // left face of cx+1
    R.col[5 * nx + cx] = (self + from_left) + from_right;
  }
  // to row r+1: the top faces' sums; to row r-1: the bottom faces'
  const int src[3] = {5, 3, 1};
  double* const dst[3] = {U.self, R.r + 1 < s.ny ? U.below : nullptr, R.r > 0 ? U.above : nullptr};
  const int shift[3] = {0, 1, -1};
  coarse_rowfwd(s, R, 3, src, dst, shift);
}

// col[j nx + cx] = sum_a g0[c][a] v_j[cl] over the row's cells, for up to two vectors.
__device__ void dof_coarse(const Sys& s, const Row& R, const double* v0, const double* v1) {
  __syncthreads();
  const int nx = s.nx, t = s.t, n = v1 ? 2 : 1;
  for (int idx = threadIdx.x; idx < n * nx; idx += blockDim.x) {
    const int j = idx / nx, cx = idx - j * nx;
    const double* v = j ? v1 : v0;
    double acc = 0.0;
    for (int a = 0; a < t; ++a) acc = fma(R.gself[a * nx + cx], v[R.cl[a * nx + cx]], acc);
    R.col[idx] = acc;
  }
}

// In-place Gauss-Jordan inverse of the t x t matrix a (symmetric positive definite,
// no pivoting) by one warp.
__device__ void warp_invert(double* a, int t) {
  const int lane = threadIdx.x & 31;
  for (int k = 0; k < t; ++k) {
    __syncwarp();
    const double d = 1.0 / a[k * t + k];
    __syncwarp();
    for (int j = lane; j < t; j += 32)
      if (j != k) a[k * t + j] *= d;
    __syncwarp();
    for (int e = lane; e < t * t; e += 32) {
      const int i = e / t, j = e - i * t;
      if (i != k && j != k) a[e] = fma(-a[i * t + k], a[k * t + j], a[e]);
    }
    __syncwarp();
    for (int i = lane; i < t; i += 32)
      if (i != k) a[i * t + k] = -a[i * t + k] * d;
    __syncwarp();
    if (lane == 0) a[k * t + k] = d;
  }
  __syncwarp();
}

constexpr int kSmemArrays = 23;

__host__ __device__ size_t smem_layout(int nx, int ny, int fs, int t, int grid, bool neu, size_t* off) {
  // a row owns at most 3 nx + 1 faces (row 0); later rows own 2 nx + 1 and add the
  // nx bottom faces of their cells
  const size_t g = (size_t)(3 * nx + 1) * fs;
  const size_t np = (size_t)block_stride(t);
  const size_t scratch = (size_t)kWarps * t * (t + 1);  // per warp: a t x t block and t weights
  const size_t vec = 6 * g > scratch ? 6 * g : scratch;
  const size_t nmode = grid > 0 ? (size_t)((nx + grid - 1) / grid) : 1;
  size_t o = 0;
  int k = 0;
  auto take = [&](size_t bytes) {
    off[k++] = o;
    o = align16(o + bytes);
  };
  take((size_t)nx * q_stride(nx) * 8);   // 0 Q
  take(3 * (size_t)nx * 8);              // 1 yrow
  take(12 * (size_t)nx * 8);             // 2 col
  take(3 * (size_t)nx * 8);              // 3 wrow
  take(nmode * (neu ? 2 : 1) * (ny + 1) * 8);  // 4 mcheb
  take(nmode * 8);                       // 5 mcinv
  take((size_t)ny * 8);                  // 6 ucol
  take(vec * 8);                         // 7 G vectors (6 g) / setup scratch
  take((size_t)nx * np * 8);             // 8 Sb
  take((size_t)nx * np * 8);             // 9 Pb
  take(g * 8);                           // 10 ga
  take(g * 8);                           // 11 gb
  take(g * 2);                           // 12 ya
  take(g * 2);                           // 13 yb
  take(g * 4);                           // 14 gdof
  take((size_t)nx * t * 2);              // 15 cl
  take((size_t)nx * t * 8);              // 16 gself
  take((size_t)nx * t * 8);              // 17 gnb
  take((size_t)nx * t);                  // 18 role
  if (neu) take(2 * (size_t)(nx + ny) * 8);  // 19 wbe
  off[k] = o;
  return o;
}

template <int FS, bool NEU>
__global__ void __launch_bounds__(kSolveThreads, 1) skeleton_pcg_kernel(const Params P) {
  constexpr int T = 4 * FS;
  constexpr int np = block_stride(T);
  const Sys& s = P.s;
  const Work& w = P.w;
  __shared__ double red[64];
  __shared__ double sh[4];
  __shared__ size_t off[kSmemArrays + 1];
  extern __shared__ __align__(16) unsigned char dyn[];
  const int tid = threadIdx.x, nth = blockDim.x;
  const int nx = s.nx, ny = s.ny;
  unsigned epoch = 0;
  int status = MHM_SOLVE_OK;
  int total_inner = 0, outer = 0;
  double bnorm = 0.0, res = 1.0;
  Row R;
#define SYNC_OR_EXIT() \
  do {                 \
    if (!grid_sync(w, epoch)) { status = MHM_SOLVE_BARRIER_TIMEOUT; goto done; } \
  } while (0)
  if (tid == 0) smem_layout(nx, ny, FS, T, gridDim.x, NEU, off);
  __syncthreads();
  R.r = blockIdx.x;
  R.c0 = R.r * nx;
  R.qs = q_stride(nx);
  R.nmode = (nx - (int)blockIdx.x + (int)gridDim.x - 1) / (int)gridDim.x;
  if (R.nmode < 0) R.nmode = 0;
  R.Q = reinterpret_cast<double*>(dyn + off[0]);
  R.yrow = reinterpret_cast<double*>(dyn + off[1]);
  R.col = reinterpret_cast<double*>(dyn + off[2]);
  R.wrow = reinterpret_cast<double*>(dyn + off[3]);
  R.mcheb = reinterpret_cast<double*>(dyn + off[4]);
  R.mcinv = reinterpret_cast<double*>(dyn + off[5]);
  R.ucol = reinterpret_cast<double*>(dyn + off[6]);
  {
    double* v = reinterpret_cast<double*>(dyn + off[7]);
    const int g = (3 * nx + 1) * FS;
    R.vr = v; R.vps = v + g; R.vp = v + 2 * g; R.vlam = v + 3 * g; R.vu = v + 4 * g; R.vt = v + 5 * g;
    R.scratch = v;
  }
  R.Sb = reinterpret_cast<double*>(dyn + off[8]);
  R.Pb = reinterpret_cast<double*>(dyn + off[9]);
  R.ga = reinterpret_cast<double*>(dyn + off[10]);
  R.gb = reinterpret_cast<double*>(dyn + off[11]);
  R.ya = reinterpret_cast<int16_t*>(dyn + off[12]);
  R.yb = reinterpret_cast<int16_t*>(dyn + off[13]);
  R.gdof = reinterpret_cast<int32_t*>(dyn + off[14]);
  R.cl = reinterpret_cast<int16_t*>(dyn + off[15]);
  R.gself = reinterpret_cast<double*>(dyn + off[16]);
  R.gnb = reinterpret_cast<double*>(dyn + off[17]);
  R.role = reinterpret_cast<uint8_t*>(dyn + off[18]);
  R.wbe = NEU ? reinterpret_cast<double*>(dyn + off[19]) : nullptr;
  {
    // DOFs are numbered by their first cell: binary search the row boundaries
    auto lower = [&](int cell) {
      int64_t lo = 0, hi = s.T;
      while (lo < hi) {
        const int64_t mid = (lo + hi) / 2;
        if (s.dof_cells[2 * mid] < cell) lo = mid + 1; else hi = mid;
      }
      return lo;
    };
    R.d0 = lower(R.c0);
    R.d1 = lower(R.c0 + nx);
    R.nown = (int)(R.d1 - R.d0);
    R.ng = R.nown + (R.r > 0 ? nx * FS : 0);
  }
  for (int e = tid; e < nx * nx; e += nth) {
    const int k = e / nx, i = e - k * nx;
    const int m = ((k + 1) * (i + 1)) % (2 * (nx + 1));
    R.Q[k * R.qs + i] = (NEU && s.qx) ? s.qx[e] : sqrt(2.0 / (nx + 1)) * sinpi((double)m / (double)(nx + 1));
  }
  // Chebyshev values of this CTA's sine modes: T_k = ay tridiag(-1, 2 theta_k, -1),
  // theta_k = 1 + ax lam_k / (2 ay); U_m(theta_k), m = 0..ny
  for (int j = tid; j < R.nmode; j += nth) {
    const int k = blockIdx.x + j * gridDim.x;
    double* u = R.mcheb + (size_t)j * (NEU ? 2 : 1) * (ny + 1);
    const double lam = (NEU && s.lamx) ? s.lamx[k] : 2.0 - 2.0 * cospi((double)(k + 1) / (double)(nx + 1));
    const double two_theta = 2.0 + s.ax * lam / s.ay;
    if (NEU && s.pinv0 && k == 0) {
      R.mcinv[j] = 1.0;  // the singular constant mode: mode_solve applies pinv0
    } else if (!NEU || s.yneu == 0) {
      double um1 = 0.0, u0 = 1.0;
      u[0] = 1.0;
      for (int m = 1; m <= ny; ++m) {
        const double un = two_theta * u0 - um1;
        u[m] = un;
        um1 = u0;
        u0 = un;
      }
      R.mcinv[j] = 1.0 / (s.ay * u[ny]);
    } else {
      // rows of T_k / ay: diagonal e_i = 2 theta_k, minus 1 on a Neumann end row
      double* v = u + (ny + 1);
      auto e = [&](int i) {
        double d = two_theta;
        if (i == 0 && (s.yneu & 1)) d -= 1.0;
        if (i == ny - 1 && (s.yneu & 2)) d -= 1.0;
        return d;
      };
      u[0] = 1.0;
      if (ny > 1) u[1] = e(0);
      for (int m = 1; m + 1 < ny; ++m) u[m + 1] = e(m) * u[m] - u[m - 1];
      v[ny - 1] = 1.0;
      if (ny > 1) v[ny - 2] = e(ny - 1);
      for (int m = ny - 2; m >= 1; --m) v[m - 1] = e(m) * v[m] - v[m + 1];
      R.mcinv[j] = 1.0 / (s.ay * (e(0) * v[0] - (ny > 1 ? v[1] : 0.0)));
    }
  }
  // G DOFs
  for (int l = tid; l < R.ng; l += nth) {
    int64_t i;
    if (l < R.nown) {
      i = R.d0 + l;
    } else {
      const int q = l - R.nown, cx = q / FS, j = q - cx * FS;
      i = s.cell_dofs[(size_t)(R.c0 + cx) * T + j];  // bottom side: slots 0 .. fs-1
    }
    R.gdof[l] = (int32_t)i;
    for (int k = 0; k < 2; ++k) {
      const int c = s.dof_cells[2 * i + k];
      double g = 0.0;
      int y = -1;
      if (c >= 0) {
        g = s.g0[(size_t)c * T + s.dof_slot[2 * i + k]];
        const int cy = c / nx;
        y = (cy - R.r + 1) * nx + (c - cy * nx);
      }
      if (NEU && s.fixed[i]) g = 0.0;  // fixed DOFs are outside the coarse space
      if (k == 0) { R.ga[l] = g; R.ya[l] = (int16_t)(y < 0 ? 0 : y); }
      else { R.gb[l] = g; R.yb[l] = (int16_t)y; }
    }
  }
  // the row's cells: local DOF, role and G0 coefficients of each slot
  for (int idx = tid; idx < nx * T; idx += nth) {
    const int cx = idx / T, a = idx - cx * T;
    const int c = R.c0 + cx;
    const int64_t i = s.cell_dofs[(size_t)c * T + a];
    const int sl = a * nx + cx;
    R.cl[sl] = (int16_t)(i >= R.d0 && i < R.d1 ? i - R.d0 : R.nown + cx * FS + a);
    const int first = s.dof_cells[2 * i];
    const bool second = first != c;
    const bool fix = NEU && s.fixed[i];
    R.role[sl] = (uint8_t)((second ? 1 : 0) | (s.dof_cells[2 * i + 1] >= 0 ? 2 : 0) | (fix ? 4 : 0));
    R.gself[sl] = fix ? 0.0 : s.g0[(size_t)c * T + a];
    const int other = second ? first : s.dof_cells[2 * i + 1];
    const int oslot = second ? s.dof_slot[2 * i] : s.dof_slot[2 * i + 1];
    R.gnb[sl] = (other >= 0 && !fix) ? s.g0[(size_t)other * T + oslot] : 0.0;
  }
  // DOFs met by one cell only: their second-cell partials stay zero
  for (int64_t i = R.d0 + tid; i < R.d1; i += nth)
    if (s.dof_cells[2 * i + 1] < 0) {
      w.Zs[i] = 0.0;
      w.Vs[i] = 0.0;
    }
  __syncthreads();
  // packed symmetric S_c (operator) of the row's cells
  for (int idx = tid; idx < nx * T * T; idx += nth) {
    const int cx = idx / (T * T), e = idx - cx * T * T, a = e / T, b = e - a * T;
    if (a > b) continue;
    const int c = R.c0 + cx;
    double v;
    if (s.blocks) {
      const double* B = s.blocks + (size_t)c * s.ld * s.ld;
      v = 0.5 * (B[a * s.ld + b] + B[b * s.ld + a]);
    } else {
      const int64_t ia = s.cell_dofs[(size_t)c * T + a], ib = s.cell_dofs[(size_t)c * T + b];
      v = 0.5 * (csr_entry(s, ia, ib) + csr_entry(s, ib, ia));
      // an entry between two DOFs of a face shared with another cell is split evenly
      if (a / FS == b / FS && (R.role[a * nx + cx] & 2)) v *= 0.5;
    }
    R.Sb[(size_t)cx * np + packed<T>(a, b)] = v;
  }
  __syncthreads();
  // preconditioner blocks: D B^-1 D, B = S_c (cell blocks) or the assembled principal
  // submatrix (D = 1); one warp inverts one cell's block in the setup scratch.  The
  // stiffness weights D of the cell's T slots (a dependent chain of global loads
  // each) are formed first, one lane per slot.
  {
    const int warp = tid >> 5, lane = tid & 31;
    double* a = R.scratch + (size_t)warp * T * (T + 1);
    double* wts = a + T * T;
    for (int cx = warp; cx < nx; cx += kWarps) {
      const int c = R.c0 + cx;
      if (s.blocks && lane < T) {
        const int64_t dof = s.cell_dofs[(size_t)c * T + lane];
        const int c1 = s.dof_cells[2 * dof], c2 = s.dof_cells[2 * dof + 1];
        const double d1 = s.blocks[(size_t)c1 * s.ld * s.ld + (size_t)s.dof_slot[2 * dof] * (s.ld + 1)];
        const double d2 =
            c2 >= 0 ? s.blocks[(size_t)c2 * s.ld * s.ld + (size_t)s.dof_slot[2 * dof + 1] * (s.ld + 1)] : 0.0;
        wts[lane] = s.blocks[(size_t)c * s.ld * s.ld + (size_t)lane * (s.ld + 1)] / (d1 + d2);
      }
      for (int e = lane; e < T * T; e += 32) {
        const int i = e / T, j = e - i * T;
        double v;
        if (s.blocks) {
          v = R.Sb[(size_t)cx * np + packed<T>(i, j)];
        } else {
          const int64_t ia = s.cell_dofs[(size_t)c * T + i], ib = s.cell_dofs[(size_t)c * T + j];
          v = 0.5 * (csr_entry(s, ia, ib) + csr_entry(s, ib, ia));
        }
        a[e] = v;
      }
      warp_invert(a, T);
      for (int e = lane; e < T * T; e += 32) {
        const int i = e / T, j = e - i * T;
        if (i > j) continue;
        const double di = s.blocks ? wts[i] : 1.0, dj = s.blocks ? wts[j] : 1.0;
        R.Pb[(size_t)cx * np + packed<T>(i, j)] = di * (0.5 * (a[i * T + j] + a[j * T + i])) * dj;
      }
      __syncwarp();
    }
  }
  // x = 0, r_full = rhs on owned rows; ||rhs||
  {
    double b2 = 0.0;
    for (int64_t i = R.d0 + tid; i < R.d1; i += nth) {
      P.x[i] = 0.0;
      const double v = P.rhs[i];
      w.rfull[i] = v;
      b2 += v * v;
    }
    for (int cx = tid; cx < nx; cx += nth) {
      const int64_t i = s.T + R.c0 + cx;
      P.x[i] = 0.0;
      const double v = P.rhs[i];
      w.rfull[i] = v;
      b2 += v * v;
    }
    put_partial(w, 0, b2, red);
  }
  SYNC_OR_EXIT();
  bnorm = sqrt(grid_total(w, 0, sh));
  if (bnorm == 0.0) goto finish;
  for (outer = 0; outer < P.max_outer; ++outer) {
    if (outer > 0) {
      double r2 = 0.0;
      for (int64_t i = R.d0 + tid; i < R.d1; i += nth) {
        const double v = (NEU && s.fixed[i]) ? 0.0 : P.rhs[i] - krow(s, i, P.x);
        w.rfull[i] = v;
        r2 += v * v;
      }
      for (int cx = tid; cx < nx; cx += nth) {
        const int64_t i = s.T + R.c0 + cx;
        const double v = P.rhs[i] - krow(s, i, P.x);
        w.rfull[i] = v;
        r2 += v * v;
      }
      put_partial(w, 0, r2, red);
      SYNC_OR_EXIT();
      res = sqrt(grid_total(w, 0, sh)) / bnorm;
      if (outer == 1 && blockIdx.x == 0 && tid == 0) P.stats[2] = res;
      if (!isfinite(res)) { status = MHM_SOLVE_NONFINITE; goto finish; }
      if (res <= P.rtol) break;
    }
    {
      // the first inner solve to inner_rtol; a later correction only has to win the
      // factor between the current outer residual and rtol.  Either one also stops
      // once its residual is below half of what rtol asks of the outer residual
      // (res bnorm): a right-hand side whose projected part is at rounding level, as
      // for a correction carried by the coarse unknowns alone, then needs no inner
      // iteration instead of chasing rounding noise into a breakdown
      const double itol = (outer == 0) ? P.inner_rtol : fmin(0.1, fmax(P.rtol / res, 1e-12));
      const double afloor = 0.5 * P.rtol * res * bnorm;
      const Coarse Cx1{w.Ux1, nullptr, nullptr}, Cx2{w.Ux2, nullptr, nullptr};
      // coarse data of r2
      for (int cx = tid; cx < nx; cx += nth) R.col[cx] = w.rfull[s.T + R.c0 + cx];
      coarse_rowfwd1(s, R, w.Ux1);
      SYNC_OR_EXIT();
      mode_solve<NEU>(s, R, Cx1, w.Wx1);
      SYNC_OR_EXIT();
      // lambda0 = -G0 (G0^T G0)^-1 r2 on G; cell partials of S lambda0; r1 on G
      coarse_rows<NEU>(s, R, w.Wx1, R.r - 1, R.r + 2);
      for (int l = tid; l < R.ng; l += nth) R.vlam[l] = -g0y(R, l);
      for (int l = tid; l < R.ng; l += nth) R.vt[l] = __ldcg(w.rfull + R.gdof[l]);
      cell_apply<FS, NEU>(s, R, R.Sb, R.vlam, w.Vf, w.Vs, false);
      SYNC_OR_EXIT();
      // rhoP = r1 - S lambda0 on G; its coarse data
      read_exchange(R, w.Vf, w.Vs, R.vu);
      __syncthreads();
      for (int l = tid; l < R.ng; l += nth) R.vr[l] = R.vt[l] - R.vu[l];
      dof_coarse(s, R, R.vr, nullptr);
      coarse_rowfwd1(s, R, w.Ux1);
      SYNC_OR_EXIT();
      mode_solve<NEU>(s, R, Cx1, w.Wx1);
      SYNC_OR_EXIT();
      // r0 = P rhoP; preconditioned partials and their coarse data; |r0|^2
      coarse_rows<NEU>(s, R, w.Wx1, R.r - 1, R.r + 2);
      for (int l = tid; l < R.ng; l += nth) R.vr[l] -= g0y(R, l);
      {
        double r2 = 0.0;
        for (int l = tid; l < R.nown; l += nth) r2 = fma(R.vr[l], R.vr[l], r2);
        cell_apply<FS, NEU>(s, R, R.Pb, R.vr, w.Zf, w.Zs, true);
        coarse_combine(s, R, w.Uz, nullptr);
        put_partial(w, 0, r2, red);
      }
      SYNC_OR_EXIT();
      mode_solve<NEU>(s, R, w.Uz, w.Wz);
      SYNC_OR_EXIT();
      double r0 = 0.0, gam_prev = 1.0, alpha_prev = 1.0;
      int k = 0;
      for (;; ++k) {
        // (1) u = P M^-1 r and w = S u (cell partials) on G; gamma, delta
        double rr[1];
        phase_begin<1, NEU>(s, w, R, 0, rr, sh, w.Zf, w.Zs, R.vt, w.Wz);
        const double rn = sqrt(rr[0]);
        if (!isfinite(rn)) { status = MHM_SOLVE_NONFINITE; break; }
        if (k == 0) {
          r0 = rn;
          if (r0 == 0.0 || r0 <= afloor) break;
        } else if (rn <= itol * r0 || rn <= afloor) {
          break;
        }
        if (k >= P.max_inner) { status = MHM_SOLVE_NOT_CONVERGED; break; }
#pragma unroll 2
        for (int l = tid; l < R.ng; l += nth) R.vu[l] = R.vt[l] - g0y(R, l);
        double gam = 0.0;
        for (int l = tid; l < R.nown; l += nth) gam = fma(R.vr[l], R.vu[l], gam);
        {
          const double del = cell_apply<FS, NEU>(s, R, R.Sb, R.vu, w.Vf, w.Vs, true);
          coarse_combine(s, R, w.Uw, nullptr);
          put_partial2(w, 1, gam, del, red);
        }
        SYNC_OR_EXIT();
        mode_solve<NEU>(s, R, w.Uw, w.Ww);
        SYNC_OR_EXIT();
        // (2) step: P S p by recurrence, r -= alpha P S p; preconditioned partials
        {
          double gd[2];
          phase_begin<2, NEU>(s, w, R, 1, gd, sh, w.Vf, w.Vs, R.vt, w.Ww);
          const double g = gd[0], d = gd[1];
          const double beta = k > 0 ? g / gam_prev : 0.0;
          const double pq = k > 0 ? d - beta * g / alpha_prev : d;
          if (!(pq > 0.0) || !isfinite(g)) { status = MHM_SOLVE_BREAKDOWN; break; }
          const double alpha = g / pq;
#pragma unroll 2
          for (int l = tid; l < R.ng; l += nth) {
            const double pw = R.vt[l] - g0y(R, l);
            const double ps = k > 0 ? fma(beta, R.vps[l], pw) : pw;
            R.vps[l] = ps;
            R.vr[l] = fma(-alpha, ps, R.vr[l]);
            const double p = k > 0 ? fma(beta, R.vp[l], R.vu[l]) : R.vu[l];
            R.vp[l] = p;
            R.vlam[l] = fma(alpha, p, R.vlam[l]);
          }
          gam_prev = g;
          alpha_prev = alpha;
        }
        if ((k + 1) % kReproject == 0) {
          // project r and P S p again
          dof_coarse(s, R, R.vr, R.vps);
          {
            const int src[2] = {0, 1};
            double* const dst[2] = {w.Ux1, w.Ux2};
            const int shift[2] = {0, 0};
            coarse_rowfwd(s, R, 2, src, dst, shift);
          }
          SYNC_OR_EXIT();
          mode_solve<NEU>(s, R, Cx1, w.Wx1);
          mode_solve<NEU>(s, R, Cx2, w.Wx2);
          SYNC_OR_EXIT();
          coarse_rows<NEU>(s, R, w.Wx1, R.r - 1, R.r + 2);
          for (int l = tid; l < R.ng; l += nth) R.vr[l] -= g0y(R, l);
          coarse_rows<NEU>(s, R, w.Wx2, R.r - 1, R.r + 2);
          for (int l = tid; l < R.ng; l += nth) R.vps[l] -= g0y(R, l);
        }
        {
          double r2 = 0.0;
          for (int l = tid; l < R.nown; l += nth) r2 = fma(R.vr[l], R.vr[l], r2);
          cell_apply<FS, NEU>(s, R, R.Pb, R.vr, w.Zf, w.Zs, true);
          coarse_combine(s, R, w.Uz, nullptr);
          put_partial(w, 0, r2, red);
        }
        SYNC_OR_EXIT();
        mode_solve<NEU>(s, R, w.Uz, w.Wz);
        SYNC_OR_EXIT();
      }
      total_inner += k;
      if (status != MHM_SOLVE_OK) goto finish;
      // c = (G0^T G0)^-1 G0^T (S lambda - r1): cell partials of S lambda, minus r1
      for (int l = tid; l < R.ng; l += nth) R.vt[l] = __ldcg(w.rfull + R.gdof[l]);
      cell_apply<FS, NEU>(s, R, R.Sb, R.vlam, nullptr, nullptr, true);
      coarse_combine(s, R, w.Uw, R.vt);
      SYNC_OR_EXIT();
      mode_solve<NEU>(s, R, w.Uw, w.Ww);
      SYNC_OR_EXIT();
      coarse_rows<NEU>(s, R, w.Ww, R.r, R.r + 1);
      for (int l = tid; l < R.nown; l += nth) P.x[R.d0 + l] += R.vlam[l];
      for (int cx = tid; cx < nx; cx += nth) P.x[s.T + R.c0 + cx] += R.yrow[nx + cx];
      SYNC_OR_EXIT();
    }
  }
  if (outer >= P.max_outer) {
    double r2 = 0.0;
    for (int64_t i = R.d0 + tid; i < R.d1; i += nth) {
      const double v = (NEU && s.fixed[i]) ? 0.0 : P.rhs[i] - krow(s, i, P.x);
      r2 += v * v;
    }
    for (int cx = tid; cx < nx; cx += nth) {
      const int64_t i = s.T + R.c0 + cx;
      const double v = P.rhs[i] - krow(s, i, P.x);
      r2 += v * v;
    }
    put_partial(w, 0, r2, red);
    SYNC_OR_EXIT();
    res = sqrt(grid_total(w, 0, sh)) / bnorm;
    if (!(res <= P.rtol) && status == MHM_SOLVE_OK) status = MHM_SOLVE_NOT_CONVERGED;
  }
finish:
  // every CTA has finished reading the partial sums before they are reused
  SYNC_OR_EXIT();
  // physical certificate (system.py:481-507): ||K x - b|| / max(||b||, ||load_scale||, || |K||x| ||)
  {
    double d2 = 0.0, a2 = 0.0, l2 = 0.0;
    auto row = [&](int64_t i) {
      double acc = 0.0, aacc = 0.0;
      for (int64_t e = s.indptr[i]; e < s.indptr[i + 1]; ++e) {
        const double xv = __ldcg(P.x + s.indices[e]);
        acc = fma(s.values[e], xv, acc);
        aacc = fma(fabs(s.values[e]), fabs(xv), aacc);
      }
      const double d = acc - P.rhs[i];
      d2 += d * d;
      a2 += aacc * aacc;
      const double ls = P.load_scale ? P.load_scale[i] : 0.0;
      l2 += ls * ls;
    };
    for (int64_t i = R.d0 + tid; i < R.d1; i += nth)
      if (!(NEU && s.fixed[i])) row(i);  // the reduced system's rows only
    for (int cx = tid; cx < nx; cx += nth) row(s.T + R.c0 + cx);
    put_partial(w, 0, d2, red);
    put_partial(w, 1, a2, red);
    put_partial(w, 2, l2, red);
    if (!grid_sync(w, epoch)) { status = MHM_SOLVE_BARRIER_TIMEOUT; goto done; }
    double tot[3];
    grid_totals<3>(w, 0, tot, sh);
    const double dn = sqrt(tot[0]), an = sqrt(tot[1]), ln = sqrt(tot[2]);
    const double scale = fmax(fmax(bnorm, ln), fmax(an, 2.2250738585072014e-308));
    if (blockIdx.x == 0 && tid == 0) {
      P.stats[0] = (bnorm > 0.0) ? dn / bnorm : 0.0;
      P.stats[1] = dn / scale;
    }
  }
done:
  if (blockIdx.x == 0 && tid == 0) {
    P.info[0] = status;
    P.info[1] = total_inner;
    P.info[2] = outer;
    P.info[3] = *reinterpret_cast<volatile int*>(w.err);
  }
#undef SYNC_OR_EXIT
}

// Ordered reduction: slot sums in ascending cell order.
__global__ void scatter_kernel(int64_t nnz, const int64_t* slot_ptr, const int64_t* contrib,
                               const double* blocks, double* vals, int64_t size, int64_t trace_size,
                               const int64_t* load_ptr, const int64_t* load_contrib,
                               const double* loads, const double* boundary, double* rhs,
                               double* load_scale) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t sidx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; sidx < nnz; sidx += stride) {
    double acc = 0.0;
    for (int64_t e = slot_ptr[sidx]; e < slot_ptr[sidx + 1]; ++e) acc += blocks[contrib[e]];
    vals[sidx] = acc;
  }
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < size; g += stride) {
    double acc = 0.0, sc = 0.0;
    for (int64_t e = load_ptr[g]; e < load_ptr[g + 1]; ++e) {
      const double v = loads[load_contrib[e]];
      acc += v;
      sc += fabs(v);
    }
    if (g < trace_size && boundary) {
      acc -= boundary[g];
      sc += fabs(boundary[g]);
    }
    rhs[g] = acc;
    if (load_scale) load_scale[g] = sc;
  }
}

// CSC export with exact zeros dropped.  The structural pattern is symmetric, so column
// j of the CSC matrix lists the same indices as CSR row j; its entry in row i is the
// CSR value of slot (i, j) = vals[transpose[k]] for the CSR slot k of (j, i).
__global__ void csc_count_kernel(int64_t size, const int64_t* indptr, const int64_t* transpose,
                                 const double* vals, int64_t* csc_indptr) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < size; j += stride) {
    int64_t c = 0;
    for (int64_t k = indptr[j]; k < indptr[j + 1]; ++k) c += vals[transpose[k]] != 0.0;
    csc_indptr[j + 1] = c;
    if (j == 0) csc_indptr[0] = 0;
  }
}

// In-place inclusive scan of ptr[1..size] in one block: each thread sums a contiguous
// chunk, the chunk totals are scanned in shared memory, and each thread rewrites its
// chunk from its prefix.  Sums of int64 counts: order-free and exact.
constexpr int kScanThreads = 1024;
__global__ void __launch_bounds__(kScanThreads) csc_scan_kernel(int64_t size, int64_t* ptr) {
  __shared__ int64_t part[kScanThreads];
  const int tid = threadIdx.x;
  const int64_t chunk = (size + kScanThreads - 1) / kScanThreads;
  const int64_t lo = 1 + tid * chunk;
  const int64_t hi = lo + chunk < size + 1 ? lo + chunk : size + 1;
  int64_t s = 0;
  for (int64_t i = lo; i < hi; ++i) s += ptr[i];
  part[tid] = s;
  __syncthreads();
  for (int off = 1; off < kScanThreads; off <<= 1) {
    const int64_t v = tid >= off ? part[tid - off] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  int64_t run = tid ? part[tid - 1] : 0;
  for (int64_t i = lo; i < hi; ++i) {
    run += ptr[i];
    ptr[i] = run;
  }
}

__global__ void csc_write_kernel(int64_t size, const int64_t* indptr, const int32_t* indices,
                                 const int64_t* transpose, const double* vals,
                                 const int64_t* csc_indptr, int32_t* csc_indices, double* csc_data) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t j = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; j < size; j += stride) {
    int64_t out = csc_indptr[j];
    for (int64_t k = indptr[j]; k < indptr[j + 1]; ++k) {
      const double v = vals[transpose[k]];
      if (v != 0.0) {
        csc_indices[out] = indices[k];
        csc_data[out] = v;
        ++out;
      }
    }
  }
}

struct Layout {
  size_t Zf, Zs, Vf, Vs, U[12], rfull, part, bar, err, total;
};

Layout layout(const mhm_skeleton_system* s, int grid) {
  Layout L{};
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t at = off;
    off = align16(off + bytes);
    return at;
  };
  const size_t T = (size_t)s->trace_size, N = (size_t)s->size, M = (size_t)s->cells;
  L.Zf = take(T * 8);
  L.Zs = take(T * 8);
  L.Vf = take(T * 8);
  L.Vs = take(T * 8);
  for (int k = 0; k < 12; ++k) L.U[k] = take(M * 8);
  L.rfull = take(N * 8);
  L.part = take((size_t)grid * 4 * 8);
  L.bar = take(2 * sizeof(unsigned));
  L.err = take(sizeof(int));
  L.total = off;
  return L;
}

size_t dyn_smem(const mhm_skeleton_system* s, int grid) {
  size_t off[kSmemArrays + 1];
  return smem_layout(s->nx, s->ny, s->face_size, s->cell_width, grid, s->fixed != nullptr, off);
}

const void* kernel_for(int fs, bool neu) {
  switch (fs * 2 + (neu ? 1 : 0)) {
    case 2: return (const void*)skeleton_pcg_kernel<1, false>;
    case 3: return (const void*)skeleton_pcg_kernel<1, true>;
    case 4: return (const void*)skeleton_pcg_kernel<2, false>;
    case 5: return (const void*)skeleton_pcg_kernel<2, true>;
    case 6: return (const void*)skeleton_pcg_kernel<3, false>;
    case 7: return (const void*)skeleton_pcg_kernel<3, true>;
    case 8: return (const void*)skeleton_pcg_kernel<4, false>;
    case 9: return (const void*)skeleton_pcg_kernel<4, true>;
    default: return nullptr;
  }
}

// One CTA per macro row; all rows must be co-resident for the cooperative launch.
// Local DOF indices are int16 and the DOF ids int32.
int resolve_grid(const mhm_skeleton_system* s) {
  int dev = 0, sms = 0, per_sm = 0;
  const void* kern = kernel_for(s->face_size, s->fixed != nullptr);
  if (!kern) return 0;
  if ((int64_t)(3 * (int64_t)s->nx + 1) * s->face_size > 32767 || s->trace_size > INT32_MAX) return 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  const size_t smem = dyn_smem(s, s->ny);
  if (smem > 227 * 1024) return 0;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return -1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kSolveThreads, smem) != cudaSuccess)
    return -1;
  const int cap = sms * per_sm;
  if (s->ny > cap) return 0;
  return s->ny;
}

bool valid(const mhm_skeleton_system* s) {
  return s && s->size == s->trace_size + s->cells && s->face_size >= 1 && s->face_size <= 4 &&
         (int64_t)s->faces * s->face_size == s->trace_size && s->cell_width == 4 * s->face_size &&
         s->nx >= 1 && s->ny >= 1 && (int64_t)s->nx * s->ny == s->cells && s->indptr &&
         s->indices && s->values && s->trace_end && s->cell_dofs && s->cell_g0 && s->dof_cells &&
         s->dof_slot && std::isfinite(s->coarse_ax) && std::isfinite(s->coarse_ay) &&
         s->coarse_ax > 0 && s->coarse_ay > 0 && (!s->cell_blocks || s->block_ld >= s->cell_width) &&
         s->coarse_neumann >= 0 && s->coarse_neumann <= 15 && (s->fixed || s->coarse_neumann == 0) &&
         (!(s->coarse_neumann & 12) || (s->coarse_qx && s->coarse_lamx)) &&
         (s->coarse_neumann != 15 || s->coarse_pinv0) &&
         (s->coarse_partial == 0 || (s->fixed && s->coarse_partial > 0 &&
                                     s->coarse_partial <= 2 * (s->nx + s->ny) && s->coarse_partial_cells &&
                                     s->coarse_partial_R));
}

// The Chebyshev values U_m(theta) grow like rho^m, rho = theta + sqrt(theta^2 - 1);
// the coarse inverse needs U_ny of the stiffest sine mode to stay far from overflow.
bool coarse_representable(const mhm_skeleton_system* s) {
  const double lam = 2.0 - 2.0 * std::cos(M_PI * s->nx / (s->nx + 1.0));
  const double theta = 1.0 + 0.5 * s->coarse_ax * lam / s->coarse_ay;
  const double rho = theta + std::sqrt(theta * theta - 1.0);
  return std::isfinite(rho) && s->ny * std::log(rho) < 600.0;
}

}  // namespace
}  // namespace mhm

using namespace mhm;

extern "C" int mhm_skeleton_scatter(int64_t nnz, const int64_t* slot_ptr, const int64_t* contrib,
                                    const double* blocks, double* vals, int64_t size,
                                    int64_t trace_size, const int64_t* load_ptr,
                                    const int64_t* load_contrib, const double* loads,
                                    const double* boundary, double* rhs, double* load_scale,
                                    void* stream) {
  if (nnz < 0 || size < 1 || trace_size < 0 || trace_size > size || !slot_ptr || !contrib ||
      !blocks || !vals || !load_ptr || !load_contrib || !loads || !rhs)
    return MHM_ERR_ARGUMENT;
  const int64_t work = nnz > size ? nnz : size;
  int blocks_n = (int)((work + 255) / 256);
  if (blocks_n > 4096) blocks_n = 4096;
  if (blocks_n < 1) blocks_n = 1;
  scatter_kernel<<<blocks_n, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      nnz, slot_ptr, contrib, blocks, vals, size, trace_size, load_ptr, load_contrib, loads,
      boundary, rhs, load_scale);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_skeleton_export_csc(int64_t size, const int64_t* indptr, const int32_t* indices,
                                       const int64_t* transpose, const double* vals,
                                       int64_t* csc_indptr, int32_t* csc_indices, double* csc_data,
                                       void* stream) {
  if (size < 1 || !indptr || !indices || !transpose || !vals || !csc_indptr || !csc_indices ||
      !csc_data)
    return MHM_ERR_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  int blocks_n = (int)((size + 255) / 256);
  if (blocks_n > 4096) blocks_n = 4096;
  csc_count_kernel<<<blocks_n, 256, 0, st>>>(size, indptr, transpose, vals, csc_indptr);
  csc_scan_kernel<<<1, kScanThreads, 0, st>>>(size, csc_indptr);
  csc_write_kernel<<<blocks_n, 256, 0, st>>>(size, indptr, indices, transpose, vals, csc_indptr,
                                              csc_indices, csc_data);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int64_t mhm_skeleton_workspace_bytes(const mhm_skeleton_system* s, int32_t grid) {
  (void)grid;
  if (!s || s->face_size < 1 || s->face_size > 4 || s->ny < 1 || s->nx < 1) return -1;
  return (int64_t)layout(s, s->ny).total;
}

namespace mhm {
namespace {
// reduced = rhs - K xfixed on the free rows (double-double row sums), 0 on the fixed
// rows (the elimination of prescribed DOFs, core/system.py:421-447).  One thread per
// row reads its row before writing it, so reduced may alias rhs.
__global__ void fixed_rhs_kernel(int64_t size, int64_t trace_size, const int64_t* indptr, const int32_t* indices,
                                 const double* values, const uint8_t* fixed, const double* xfixed,
                                 const double* rhs, double* reduced) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < size; i += stride) {
    if (i < trace_size && fixed[i]) {
      reduced[i] = 0.0;
      continue;
    }
    double hi = rhs[i], lo = 0.0;
    for (int64_t e = indptr[i]; e < indptr[i + 1]; ++e) {
      const double xv = xfixed[indices[e]];
      if (xv != 0.0) dd_add(hi, lo, -values[e] * xv);
    }
    reduced[i] = hi + lo;
  }
}
}  // namespace
}  // namespace mhm

extern "C" int mhm_skeleton_fixed_rhs(int64_t size, int64_t trace_size, const int64_t* indptr,
                                      const int32_t* indices, const double* values, const uint8_t* fixed,
                                      const double* xfixed, const double* rhs, double* reduced, void* stream) {
  if (size < 1 || trace_size < 0 || trace_size > size || !indptr || !indices || !values || !fixed || !xfixed ||
      !rhs || !reduced)
    return MHM_ERR_ARGUMENT;
  int64_t grid = (size + 255) / 256;
  if (grid > 148 * 8) grid = 148 * 8;
  fixed_rhs_kernel<<<(int)grid, 256, 0, static_cast<cudaStream_t>(stream)>>>(size, trace_size, indptr, indices,
                                                                           values, fixed, xfixed, rhs, reduced);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_skeleton_solve(const mhm_skeleton_system* s, const double* rhs,
                                  const double* load_scale, double* x, double rtol,
                                  double inner_rtol, int32_t max_inner, int32_t max_outer,
                                  int32_t grid, void* workspace, int64_t workspace_bytes,
                                  int32_t* info, double* stats, void* stream) {
  (void)grid;
  if (!valid(s) || !rhs || !x || !workspace || !info || !stats || max_inner < 1 || max_outer < 1 ||
      !(rtol > 0) || !(inner_rtol > 0))
    return MHM_ERR_ARGUMENT;
  if (!coarse_representable(s)) return MHM_ERR_UNSUPPORTED;
  const int g = resolve_grid(s);
  if (g < 0) return MHM_ERR_LAUNCH;
  if (g == 0) return MHM_ERR_UNSUPPORTED;
  const Layout L = layout(s, g);
  if ((int64_t)L.total > workspace_bytes) return MHM_ERR_ARGUMENT;
  char* base = static_cast<char*>(workspace);
  Params P{};
  P.s = Sys{s->size, s->trace_size, s->indptr, s->indices, s->values, s->trace_end, s->faces,
            s->face_size, s->cells, s->cell_width, s->cell_dofs, s->cell_g0, s->dof_cells,
            s->dof_slot, s->nx, s->ny, s->coarse_ax, s->coarse_ay, s->cell_blocks, s->block_ld,
            s->fixed, s->fixed ? (s->coarse_neumann & 3) : 0,
            (s->fixed && (s->coarse_neumann & 12)) ? s->coarse_qx : nullptr,
            (s->fixed && (s->coarse_neumann & 12)) ? s->coarse_lamx : nullptr,
            (s->fixed && s->coarse_neumann == 15) ? s->coarse_pinv0 : nullptr,
            s->fixed ? s->coarse_partial : 0, s->fixed ? s->coarse_partial_cells : nullptr,
            s->fixed ? s->coarse_partial_R : nullptr};
  auto at = [&](size_t o) { return reinterpret_cast<double*>(base + o); };
  P.w.Zf = at(L.Zf);
  P.w.Zs = at(L.Zs);
  P.w.Vf = at(L.Vf);
  P.w.Vs = at(L.Vs);
  P.w.Uz = Coarse{at(L.U[0]), at(L.U[1]), at(L.U[2])};
  P.w.Uw = Coarse{at(L.U[3]), at(L.U[4]), at(L.U[5])};
  P.w.Ux1 = at(L.U[6]);
  P.w.Ux2 = at(L.U[7]);
  P.w.Wz = at(L.U[8]);
  P.w.Ww = at(L.U[9]);
  P.w.Wx1 = at(L.U[10]);
  P.w.Wx2 = at(L.U[11]);
  P.w.rfull = at(L.rfull);
  P.w.part = at(L.part);
  P.w.bar = reinterpret_cast<unsigned*>(base + L.bar);
  P.w.err = reinterpret_cast<int*>(base + L.err);
  P.rhs = rhs; P.load_scale = load_scale; P.x = x; P.rtol = rtol; P.inner_rtol = inner_rtol;
  P.max_inner = max_inner; P.max_outer = max_outer; P.info = info; P.stats = stats;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // barrier counter and error flag start at zero on every call
  if (cudaMemsetAsync(base + L.bar, 0, L.total - L.bar, st) != cudaSuccess) return MHM_ERR_LAUNCH;
  if (cudaMemsetAsync(stats, 0, 4 * sizeof(double), st) != cudaSuccess) return MHM_ERR_LAUNCH;
  void* args[] = {&P};
  cudaError_t e = cudaLaunchCooperativeKernel(kernel_for(s->face_size, s->fixed != nullptr), dim3(g), dim3(kSolveThreads),
                                              args, dyn_smem(s, g), st);
  return e == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}
