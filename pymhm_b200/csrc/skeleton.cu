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
// whose inner solve is a FETI-style projected CG on
//     K0 = [[S, -G0], [-G0^T, 0]],
// G0 the exact geometric net-flux operator of the Cartesian macro grid.
// G0^T G0 = ay (T_y (x) I) + ax (I (x) T_x) is a scaled 2-D Dirichlet Laplacian
// on the macro cells; it is inverted exactly by an orthonormal sine transform
// along x, the inverse of one tridiagonal Toeplitz matrix along y per sine mode
// (closed form through Chebyshev polynomials of the second kind), and the
// inverse transform.  The preconditioner is block Jacobi over skeleton faces.
// K - K0 is at rounding level, so two or three outer corrections reach FP64
// accuracy.
//
// Everything runs in one persistent cooperative kernel with one CTA per macro
// row: CTA r owns the faces first met by the cells of row r (a contiguous DOF
// range in the reference's numbering), the row's coarse unknowns and the row's
// sine transform.  An inner iteration needs four grid barriers.  Each phase
// stages what it reads from other CTAs into shared memory with batched loads
// and computes from there.  The barrier is a monotonic arrival counter with a
// bounded spin: on timeout every CTA sets the error flag and returns
// (MHM_SOLVE_BARRIER_TIMEOUT).
#include <cmath>

#include "mhm_common.cuh"

namespace mhm {
namespace {

constexpr int kSolveThreads = 512;
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
  const double* qx;
  double ax, ay;
};

struct Work {
  double *lam, *rho, *rhoP, *z, *zt, *p, *q, *tmp;  // T each
  double* rfull;                                    // N
  double *U, *U2;                                   // M each ([iy][k]), two buffers
  double* cheb;                                     // nx * (ny + 1) Chebyshev tables
  double* part;                                     // grid * 4
  unsigned* bar;                                    // arrival counter
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
    __threadfence();
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

// Sum of the per-CTA partials `slot` (fixed order, identical in every CTA).
__device__ double grid_total(const Work& w, int slot, double* sh) {
  if (threadIdx.x < 32) {
    double v = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) v += __ldcg(w.part + i * 4 + slot);
    v = warp_sum(v);
    if (threadIdx.x == 0) sh[0] = v;
  }
  __syncthreads();
  const double r = sh[0];
  __syncthreads();
  return r;
}

__device__ void put_partial(const Work& w, int slot, double v, double* red) {
  v = block_sum(v, red);
  if (threadIdx.x == 0) w.part[blockIdx.x * 4 + slot] = v;
}

__device__ __forceinline__ double krow(const Sys& s, int64_t i, const double* v) {
  double acc = 0.0;
  for (int64_t e = s.indptr[i]; e < s.indptr[i + 1]; ++e) acc = fma(s.values[e], __ldcg(v + s.indices[e]), acc);
  return acc;
}

// Per-CTA state.  CTA r owns macro row r: DOFs [d0, d1) (the faces first met by
// the row's cells), the row's coarse unknowns and sine mode r.  The "G range"
// [gs, d1) covers row r-1's and row r's DOFs: every DOF whose G0 coefficients,
// face inverse or preconditioned residual the CTA needs; all of their cells lie
// in rows r-1..r+1.  The window [w0, w1) covers rows r-1..r+1 (SpMV columns).
struct Row {
  int r, c0;
  int64_t d0, d1, gs, w0, w1;
  double* qx;    // nx*nx
  double* yrow;  // 3*nx: Y of rows r-1, r, r+1
  double* col;   // max(nx, ny) scratch
  double* win;   // staged vector (window or G range)
  double* ga;    // G range: G0 coefficient of the first / second cell
  double* gb;
  int16_t* ya;   // yrow index of the first / second cell (second: -1 = none)
  int16_t* yb;
  double* minv;  // face inverses of the G range
  int16_t* cl;   // own cells: G-range index of each cell DOF (nx*t)
  double* cg;    // own cells: G0 coefficient of each cell DOF
  double* cheb;  // Chebyshev tables U_m(theta_k), m = 0..ny, of every sine mode
  double* wrow;  // W rows r-1..r+1 (sine space along x)
  double* cinv;  // 1 / (ay U_ny(theta_k)) per mode
  double* ust;   // staged U, transposed [k][iy] with row pitch ny+1
};

__device__ __forceinline__ double g0y(const Row& R, int64_t l) {
  double v = R.ga[l] * R.yrow[R.ya[l]];
  const int b = R.yb[l];
  if (b >= 0) v = fma(R.gb[l], R.yrow[b], v);
  return v;
}

// dst[k] = src[k] (k < n) through L2; each thread issues eight loads before it stores
// any of them, so a staging pass costs one round trip instead of one per element.
__device__ __forceinline__ void copy_l2(double* dst, const double* src, int64_t n) {
  for (int64_t base = threadIdx.x; base < n; base += 8 * (int64_t)blockDim.x) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int64_t k = base + (int64_t)u * blockDim.x;
      v[u] = k < n ? __ldcg(src + k) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int64_t k = base + (int64_t)u * blockDim.x;
      if (k < n) dst[k] = v[u];
    }
  }
}

// Stage v over the SpMV window [w0, w1) or over the G range [gs, d1) into R.win.
__device__ void stage(const Row& R, const double* v) {
  __syncthreads();
  copy_l2(R.win, v + R.w0, R.w1 - R.w0);
  __syncthreads();
}

__device__ void stage_g(const Row& R, const double* v) {
  __syncthreads();
  copy_l2(R.win, v + R.gs, R.d1 - R.gs);
  __syncthreads();
}

// (S v)_i with v staged in R.win over the window; matrix entries are fetched
// sixteen at a time, all loads of a chunk in flight together.
__device__ __forceinline__ double srow_win(const Sys& s, const Row& R, int64_t i) {
  const int64_t e1 = s.trace_end[i];
  double acc = 0.0;
  for (int64_t e = s.indptr[i]; e < e1; e += 16) {
    double v[16];
    int c[16];
#pragma unroll
    for (int u = 0; u < 16; ++u) {
      const bool ok = e + u < e1;
      v[u] = ok ? s.values[e + u] : 0.0;
      c[u] = ok ? s.indices[e + u] : (int)R.w0;
    }
#pragma unroll
    for (int u = 0; u < 16; ++u) acc = fma(v[u], R.win[c[u] - R.w0], acc);
  }
  return acc;
}

// Dot products by 8-lane groups: out o = sum over lanes of partial(o, lane).  Every
// lane of the block runs the same number of rounds, so the shuffles never diverge.
template <typename F, typename G>
__device__ __forceinline__ void group8(int nout, F partial, G store) {
  const int lane8 = threadIdx.x & 7, grp = threadIdx.x >> 3, ngrp = blockDim.x >> 3;
  for (int base = 0; base < nout; base += ngrp) {
    const int o = base + grp;
    double v = (o < nout) ? partial(o, lane8) : 0.0;
    v += __shfl_xor_sync(0xffffffffu, v, 4);
    v += __shfl_xor_sync(0xffffffffu, v, 2);
    v += __shfl_xor_sync(0xffffffffu, v, 1);
    if (o < nout && lane8 == 0) store(o, v);
  }
}

// U[r][:] = v_row Qx  (v_row in R.col, nx values; Qx symmetric).  U is one of two
// buffers: a phase that reads one may write the other before the next barrier.
__device__ void coarse_rowfwd(const Sys& s, double* U, const Row& R) {
  __syncthreads();
  group8(
      s.nx,
      [&](int k, int l) {
        double acc = 0.0;
#pragma unroll 8
        for (int ix = l; ix < s.nx; ix += 8) acc = fma(R.col[ix], R.qx[k * s.nx + ix], acc);
        return acc;
      },
      [&](int k, double v) { U[(size_t)R.r * s.nx + k] = v; });
}

// After every row's U is written: W rows r-1+j (j in [j0, j1)) = T_k^-1 U[:, k]
// restricted to those rows, then Y rows = W rows Qx.  Inverse entry (i, j) of mode k
// (i <= j): U_i U_{ny-1-j} / (ay U_ny), U the Chebyshev table of the mode.
__device__ void coarse_rows(const Sys& s, const double* U, const Row& R, int j0, int j1) {
  __syncthreads();
  const int ny = s.ny, nx = s.nx;
  for (int base = threadIdx.x; base < nx * ny; base += 8 * blockDim.x) {
    double v[8];
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int idx = base + u * blockDim.x;
      v[u] = idx < nx * ny ? __ldcg(U + idx) : 0.0;
    }
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int idx = base + u * blockDim.x;
      if (idx < nx * ny) {
        const int iy = idx / nx, k = idx - iy * nx;
        R.ust[k * (ny + 1) + iy] = v[u];
      }
    }
  }
  __syncthreads();
  {
    const int lane8 = threadIdx.x & 7, grp = threadIdx.x >> 3, ngrp = blockDim.x >> 3;
    for (int base = 0; base < nx; base += ngrp) {
      const int k = base + grp;
      double a0 = 0.0, a1 = 0.0, a2 = 0.0;
      if (k < nx) {
        const double* u = R.cheb + (size_t)k * (ny + 1);
        const double* uc = R.ust + (size_t)k * (ny + 1);
        const int r0 = R.r - 1;
#pragma unroll 4
        for (int iy = lane8; iy < ny; iy += 8) {
          const double v = uc[iy];
          const double ulo = u[iy], uhi = u[ny - 1 - iy];
          // row ir = r0 + j, column iy: U_min U_{ny-1-max}
          if (r0 >= 0) a0 = fma((r0 < iy ? u[r0] * uhi : ulo * u[ny - 1 - r0]), v, a0);
          if (r0 + 1 < ny) a1 = fma((r0 + 1 < iy ? u[r0 + 1] * uhi : ulo * u[ny - 2 - r0]), v, a1);
          if (r0 + 2 < ny) a2 = fma((r0 + 2 < iy ? u[r0 + 2] * uhi : ulo * u[ny - 3 - r0]), v, a2);
        }
      }
      for (int o = 4; o > 0; o >>= 1) {
        a0 += __shfl_xor_sync(0xffffffffu, a0, o);
        a1 += __shfl_xor_sync(0xffffffffu, a1, o);
        a2 += __shfl_xor_sync(0xffffffffu, a2, o);
      }
      if (k < nx && lane8 == 0) {
        const double c = R.cinv[k];
        R.wrow[k] = (j0 <= 0 && j1 > 0) ? a0 * c : 0.0;
        R.wrow[nx + k] = (j0 <= 1 && j1 > 1) ? a1 * c : 0.0;
        R.wrow[2 * nx + k] = (j0 <= 2 && j1 > 2) ? a2 * c : 0.0;
      }
    }
  }
  __syncthreads();
  group8(
      3 * nx,
      [&](int o, int l) {
        const int j = o / nx, ix = o - j * nx;
        double acc = 0.0;
#pragma unroll 8
        for (int k = l; k < nx; k += 8) acc = fma(R.wrow[j * nx + k], R.qx[ix * nx + k], acc);
        return acc;
      },
      [&](int o, double v) { R.yrow[o] = v; });
  __syncthreads();
}

// R.col[cx] = sum_a g0[c,a] v[cl] over the row's cells (v over the G range, shared memory).
__device__ void row_g0t(const Sys& s, const Row& R, const double* v) {
  __syncthreads();
  group8(
      s.nx,
      [&](int cx, int l) {
        double acc = 0.0;
        for (int a = l; a < s.t; a += 8) acc = fma(R.cg[cx * s.t + a], v[R.cl[cx * s.t + a]], acc);
        return acc;
      },
      [&](int cx, double v2) { R.col[cx] = v2; });
}

// Projected residual rho = rhoP - G0 Y and zt = Minv rho on the face whose first DOF is
// at G-range position l0; rhoP is staged over the G range in shared memory.
template <int FS>
__device__ __forceinline__ void face_precondition(const Row& R, int l0, const double* rhoP_win,
                                                  double (&rho_out)[FS], double (&z_out)[FS]) {
#pragma unroll
  for (int r = 0; r < FS; ++r) rho_out[r] = rhoP_win[l0 + r] - g0y(R, l0 + r);
  const double* m = R.minv + (l0 / FS) * FS * FS;
#pragma unroll
  for (int r = 0; r < FS; ++r) {
    double acc = 0.0;
#pragma unroll
    for (int c = 0; c < FS; ++c) acc = fma(m[r * FS + c], rho_out[c], acc);
    z_out[r] = acc;
  }
}

__host__ __device__ size_t smem_layout(const mhm_skeleton_system* s, size_t* off) {
  // bounds: a row owns at most (3 nx + 1) faces (row 0), later rows 2 nx + 1
  const int fs = s->face_size;
  const size_t own0 = (size_t)(3 * s->nx + 1) * fs, own = (size_t)(2 * s->nx + 1) * fs;
  const size_t own_max = own0 > own ? own0 : own;
  const size_t g = own_max + own;              // rows r-1 and r
  const size_t wmax = own_max + 2 * own_max;   // rows r-1..r+1
  const size_t m = s->nx > s->ny ? s->nx : s->ny;
  const size_t win = wmax > 3 * (size_t)s->nx ? wmax : 3 * (size_t)s->nx;
  size_t o = 0;
  auto take = [&](int k, size_t bytes) {
    off[k] = o;
    o = align16(o + bytes);
  };
  take(0, (size_t)s->nx * s->nx * 8);           // qx
  take(1, 3 * (size_t)s->nx * 8);               // yrow
  take(2, m * 8);                               // col
  take(3, win * 8);                             // win
  take(4, g * 8);                               // ga
  take(5, g * 8);                               // gb
  take(6, g * 2);                               // ya
  take(7, g * 2);                               // yb
  take(8, (g / fs + 1) * fs * fs * 8);          // minv
  take(9, (size_t)s->nx * s->cell_width * 2);   // cl
  take(10, (size_t)s->nx * s->cell_width * 8);  // cg
  take(11, (size_t)s->nx * (s->ny + 1) * 8);    // cheb
  take(12, 3 * (size_t)s->nx * 8);              // wrow
  take(13, (size_t)s->nx * 8);                  // cinv
  take(14, (size_t)s->nx * (s->ny + 1) * 8);    // ust (transposed, padded)
  off[15] = o;
  return o;
}

template <int FS>
__global__ void __launch_bounds__(kSolveThreads, 1) skeleton_pcg_kernel(const Params P) {
  const Sys& s = P.s;
  const Work& w = P.w;
  __shared__ double red[32];
  __shared__ double sh[2];
  __shared__ size_t off[16];
  extern __shared__ __align__(16) unsigned char dyn[];
  constexpr int fs = FS;
  const int tid = threadIdx.x, nth = blockDim.x;
  unsigned epoch = 0;
  int status = MHM_SOLVE_OK;
  int total_inner = 0, outer = 0;
  double bnorm = 0.0, res = 1.0;
  Row R;
#define SYNC_OR_EXIT() \
  do {                 \
    if (!grid_sync(w, epoch)) { status = MHM_SOLVE_BARRIER_TIMEOUT; goto done; } \
  } while (0)
  if (tid == 0) {
    mhm_skeleton_system tmp{};
    tmp.nx = s.nx; tmp.ny = s.ny; tmp.face_size = s.fs; tmp.cell_width = s.t;
    smem_layout(&tmp, off);
  }
  __syncthreads();
  R.r = blockIdx.x;
  R.c0 = R.r * s.nx;
  R.qx = reinterpret_cast<double*>(dyn + off[0]);
  R.yrow = reinterpret_cast<double*>(dyn + off[1]);
  R.col = reinterpret_cast<double*>(dyn + off[2]);
  R.win = reinterpret_cast<double*>(dyn + off[3]);
  R.ga = reinterpret_cast<double*>(dyn + off[4]);
  R.gb = reinterpret_cast<double*>(dyn + off[5]);
  R.ya = reinterpret_cast<int16_t*>(dyn + off[6]);
  R.yb = reinterpret_cast<int16_t*>(dyn + off[7]);
  R.minv = reinterpret_cast<double*>(dyn + off[8]);
  R.cl = reinterpret_cast<int16_t*>(dyn + off[9]);
  R.cg = reinterpret_cast<double*>(dyn + off[10]);
  R.cheb = reinterpret_cast<double*>(dyn + off[11]);
  R.wrow = reinterpret_cast<double*>(dyn + off[12]);
  R.cinv = reinterpret_cast<double*>(dyn + off[13]);
  R.ust = reinterpret_cast<double*>(dyn + off[14]);
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
    R.d1 = lower(R.c0 + s.nx);
    R.gs = R.r > 0 ? lower(R.c0 - s.nx) : R.d0;
    R.w0 = R.gs;
    R.w1 = R.r + 1 < s.ny ? lower(R.c0 + 2 * s.nx) : R.d1;
  }
  for (int idx = tid; idx < s.nx * s.nx; idx += nth) R.qx[idx] = s.qx[idx];
  // G-range coefficients: (G0 Y)_i = ga Y(first cell) + gb Y(second cell)
  for (int64_t l = tid; l < R.d1 - R.gs; l += nth) {
    const int64_t i = R.gs + l;
    for (int k = 0; k < 2; ++k) {
      const int c = s.dof_cells[2 * i + k];
      double g = 0.0;
      int y = -1;
      if (c >= 0) {
        g = s.g0[(size_t)c * s.t + s.dof_slot[2 * i + k]];
        const int cy = c / s.nx;
        y = (cy - R.r + 1) * s.nx + (c - cy * s.nx);
      }
      if (k == 0) { R.ga[l] = g; R.ya[l] = (int16_t)(y < 0 ? 0 : y); }
      else { R.gb[l] = g; R.yb[l] = (int16_t)y; }
    }
  }
  // own cells: G-range position and G0 coefficient of each cell DOF
  for (int idx = tid; idx < s.nx * s.t; idx += nth) {
    const int cx = idx / s.t, a = idx - cx * s.t;
    const int c = R.c0 + cx;
    R.cl[idx] = (int16_t)(s.cell_dofs[(size_t)c * s.t + a] - R.gs);
    R.cg[idx] = s.g0[(size_t)c * s.t + a];
  }
  // Chebyshev table of mode k: T_k = ay tridiag(-1, 2 theta_k, -1), theta_k =
  // 1 + ax lam_k / (2 ay); U_m(theta_k), m = 0..ny.  Row CTA k owns mode k.
  if (tid == 0) {
    for (int k = blockIdx.x; k < s.nx; k += gridDim.x) {
      double* u = w.cheb + (size_t)k * (s.ny + 1);
      const double lam = 2.0 - 2.0 * cos(M_PI * (k + 1) / (s.nx + 1));
      const double two_theta = 2.0 + s.ax * lam / s.ay;
      double um1 = 0.0, u0 = 1.0;
      u[0] = 1.0;
      for (int m = 1; m <= s.ny; ++m) {
        const double un = two_theta * u0 - um1;
        u[m] = un;
        um1 = u0;
        u0 = un;
      }
    }
  }
  // face-block Jacobi inverses of the G range (Gauss-Jordan, partial pivoting)
  for (int64_t fl = tid; fl < (R.d1 - R.gs) / fs; fl += nth) {
    const int64_t f = R.gs / fs + fl;
    double a[FS][2 * FS];
    for (int r = 0; r < fs; ++r) {
      const int64_t row = f * fs + r;
      for (int c = 0; c < 2 * fs; ++c) a[r][c] = (c - fs == r) ? 1.0 : 0.0;
      for (int64_t e = s.indptr[row]; e < s.trace_end[row]; ++e) {
        const int64_t cidx = s.indices[e];
        if (cidx >= f * fs && cidx < (f + 1) * fs) a[r][cidx - f * fs] = s.values[e];
      }
    }
    for (int k = 0; k < fs; ++k) {
      int piv = k;
      for (int r = k + 1; r < fs; ++r)
        if (fabs(a[r][k]) > fabs(a[piv][k])) piv = r;
      if (piv != k)
        for (int c = 0; c < 2 * fs; ++c) { const double tmp = a[k][c]; a[k][c] = a[piv][c]; a[piv][c] = tmp; }
      const double d = a[k][k];
      const double inv = (d != 0.0) ? 1.0 / d : 0.0;
      for (int c = 0; c < 2 * fs; ++c) a[k][c] *= inv;
      for (int r = 0; r < fs; ++r) {
        if (r == k) continue;
        const double m = a[r][k];
        for (int c = 0; c < 2 * fs; ++c) a[r][c] = fma(-m, a[k][c], a[r][c]);
      }
    }
    for (int r = 0; r < fs; ++r)
      for (int c = 0; c < fs; ++c) R.minv[fl * fs * fs + r * fs + c] = a[r][fs + c];
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
    for (int cx = tid; cx < s.nx; cx += nth) {
      const int64_t i = s.T + R.c0 + cx;
      P.x[i] = 0.0;
      const double v = P.rhs[i];
      w.rfull[i] = v;
      b2 += v * v;
    }
    put_partial(w, 0, b2, red);
  }
  SYNC_OR_EXIT();
  // every mode's Chebyshev table (complete now) into shared memory
  copy_l2(R.cheb, w.cheb, (int64_t)s.nx * (s.ny + 1));
  __syncthreads();
  for (int k = tid; k < s.nx; k += nth) R.cinv[k] = 1.0 / (s.ay * R.cheb[(size_t)k * (s.ny + 1) + s.ny]);
  __syncthreads();
  bnorm = sqrt(grid_total(w, 0, sh));
  if (bnorm == 0.0) goto finish;
  for (outer = 0; outer < P.max_outer; ++outer) {
    if (outer > 0) {
      double r2 = 0.0;
      for (int64_t i = R.d0 + tid; i < R.d1; i += nth) {
        const double v = P.rhs[i] - krow(s, i, P.x);
        w.rfull[i] = v;
        r2 += v * v;
      }
      for (int cx = tid; cx < s.nx; cx += nth) {
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
      const double itol = (outer == 0) ? P.inner_rtol : fmax(P.inner_rtol, 1e-4);
      // lambda0 = -G0 C^-1 r2
      for (int cx = tid; cx < s.nx; cx += nth) R.col[cx] = w.rfull[s.T + R.c0 + cx];
      coarse_rowfwd(s, w.U, R);
      SYNC_OR_EXIT();
      coarse_rows(s, w.U, R, 1, 3);
      for (int64_t i = R.d0 + tid; i < R.d1; i += nth) w.lam[i] = -g0y(R, i - R.gs);
      SYNC_OR_EXIT();
      // rhoP = r1 - S lam
      stage(R, w.lam);
      for (int64_t i = R.d0 + tid; i < R.d1; i += nth) w.rhoP[i] = w.rfull[i] - srow_win(s, R, i);
      SYNC_OR_EXIT();
      stage_g(R, w.rhoP);
      row_g0t(s, R, R.win);
      coarse_rowfwd(s, w.U, R);
      SYNC_OR_EXIT();
      coarse_rows(s, w.U, R, 0, 3);
      stage_g(R, w.rhoP);
      double r2 = 0.0;
      for (int64_t f = R.d0 / fs + tid; f < R.d1 / fs; f += nth) {
        double rl[FS], zl[FS];
        face_precondition<FS>(R, (int)(f * fs - R.gs), R.win, rl, zl);
        for (int r = 0; r < fs; ++r) {
          w.rho[f * fs + r] = rl[r];
          w.zt[f * fs + r] = zl[r];
          r2 += rl[r] * rl[r];
        }
      }
      put_partial(w, 1, r2, red);
      SYNC_OR_EXIT();  // zt of neighbouring rows is needed below
      const double r0 = sqrt(grid_total(w, 1, sh));
      stage_g(R, w.zt);
      row_g0t(s, R, R.win);
      coarse_rowfwd(s, w.U, R);
      SYNC_OR_EXIT();
      coarse_rows(s, w.U, R, 1, 3);
      {
        double rz = 0.0;
        for (int64_t i = R.d0 + tid; i < R.d1; i += nth) {
          const double zi = w.zt[i] - g0y(R, i - R.gs);
          w.z[i] = zi;
          w.p[i] = zi;
          rz += w.rho[i] * zi;
        }
        put_partial(w, 2, rz, red);
      }
      SYNC_OR_EXIT();
      double rz = grid_total(w, 2, sh);
      {
        stage(R, w.p);
        double pq = 0.0;
        for (int64_t i = R.d0 + tid; i < R.d1; i += nth) {
          const double qi = srow_win(s, R, i);
          w.q[i] = qi;
          pq += R.win[i - R.w0] * qi;
        }
        put_partial(w, 3, pq, red);
      }
      SYNC_OR_EXIT();
      int k = 0;
      if (r0 > 0.0) {
        for (k = 0; k < P.max_inner; ++k) {
          // A: step along p; coarse data of the updated residual
          const double pq = grid_total(w, 3, sh);
          if (!(pq > 0.0)) { status = MHM_SOLVE_BREAKDOWN; break; }
          const double alpha = rz / pq;
          for (int64_t i = R.d0 + tid; i < R.d1; i += nth) {
            w.lam[i] = fma(alpha, w.p[i], w.lam[i]);
            w.rhoP[i] = fma(-alpha, w.q[i], w.rho[i]);
          }
          __syncthreads();
          {
            const int64_t ng = R.d1 - R.gs;
            for (int64_t base = tid; base < ng; base += 4 * (int64_t)nth) {
              double qv[4], rv[4];
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const int64_t k2 = base + (int64_t)u * nth;
                qv[u] = k2 < ng ? __ldcg(w.q + R.gs + k2) : 0.0;
                rv[u] = k2 < ng ? __ldcg(w.rho + R.gs + k2) : 0.0;
              }
#pragma unroll
              for (int u = 0; u < 4; ++u) {
                const int64_t k2 = base + (int64_t)u * nth;
                if (k2 < ng) R.win[k2] = fma(-alpha, qv[u], rv[u]);
              }
            }
          }
          row_g0t(s, R, R.win);
          coarse_rowfwd(s, w.U, R);
          SYNC_OR_EXIT();
          // B: W and Y rows of the projection; project and precondition the owned faces;
          //    coarse data of G0^T Minv rho
          coarse_rows(s, w.U, R, 0, 3);
          stage_g(R, w.rhoP);
          double r2b = 0.0;
          for (int64_t f = R.d0 / fs + tid; f < R.d1 / fs; f += nth) {
            double rl[FS], zl[FS];
            face_precondition<FS>(R, (int)(f * fs - R.gs), R.win, rl, zl);
            for (int r = 0; r < fs; ++r) {
              w.rho[f * fs + r] = rl[r];
              w.zt[f * fs + r] = zl[r];
              r2b += rl[r] * rl[r];
            }
          }
          // four threads per cell, one per side, reduced over 4-lane groups
          for (int base = 0; base < 4 * s.nx; base += nth) {
            const int idx = base + tid;
            const int cx = idx >> 2, side = idx & 3;
            double acc = 0.0;
            if (cx < s.nx) {
              const int a = side * fs;
              double rl[FS], zl[FS];
              face_precondition<FS>(R, R.cl[cx * s.t + a], R.win, rl, zl);
#pragma unroll
              for (int r = 0; r < FS; ++r) acc = fma(R.cg[cx * s.t + a + r], zl[r], acc);
            }
            acc += __shfl_xor_sync(0xffffffffu, acc, 2);
            acc += __shfl_xor_sync(0xffffffffu, acc, 1);
            if (cx < s.nx && side == 0) R.col[cx] = acc;
          }
          coarse_rowfwd(s, w.U2, R);
          put_partial(w, 1, r2b, red);
          SYNC_OR_EXIT();
          // C: convergence test; projected preconditioned residual
          {
            const double rn = sqrt(grid_total(w, 1, sh));
            if (!isfinite(rn)) { status = MHM_SOLVE_NONFINITE; break; }
            if (rn <= itol * r0) { ++k; break; }
          }
          coarse_rows(s, w.U2, R, 1, 3);
          {
            double rzn = 0.0;
            for (int64_t i = R.d0 + tid; i < R.d1; i += nth) {
              const double zi = w.zt[i] - g0y(R, i - R.gs);
              w.z[i] = zi;
              rzn += w.rho[i] * zi;
            }
            put_partial(w, 2, rzn, red);
          }
          SYNC_OR_EXIT();
          // D: new direction, q = S p by recurrence
          {
            const double rzn = grid_total(w, 2, sh);
            const double beta = rzn / rz;
            rz = rzn;
            stage(R, w.z);
            double pq2 = 0.0;
            for (int64_t i = R.d0 + tid; i < R.d1; i += nth) {
              const double pi = fma(beta, w.p[i], R.win[i - R.w0]);
              const double qi = fma(beta, w.q[i], srow_win(s, R, i));
              w.p[i] = pi;
              w.q[i] = qi;
              pq2 += pi * qi;
            }
            put_partial(w, 3, pq2, red);
          }
          SYNC_OR_EXIT();
        }
        if (k >= P.max_inner && status == MHM_SOLVE_OK) status = MHM_SOLVE_NOT_CONVERGED;
      }
      total_inner += k;
      if (status != MHM_SOLVE_OK) goto finish;
      // c = C^-1 G0^T (S lam - r1)
      stage(R, w.lam);
      for (int64_t i = R.d0 + tid; i < R.d1; i += nth) w.tmp[i] = srow_win(s, R, i) - w.rfull[i];
      SYNC_OR_EXIT();
      stage_g(R, w.tmp);
      row_g0t(s, R, R.win);
      coarse_rowfwd(s, w.U, R);
      SYNC_OR_EXIT();
      coarse_rows(s, w.U, R, 1, 2);
      for (int64_t i = R.d0 + tid; i < R.d1; i += nth) P.x[i] += w.lam[i];
      for (int cx = tid; cx < s.nx; cx += nth) P.x[s.T + R.c0 + cx] += R.yrow[s.nx + cx];
      SYNC_OR_EXIT();
    }
  }
  if (outer >= P.max_outer) {
    double r2 = 0.0;
    for (int64_t i = R.d0 + tid; i < R.d1; i += nth) {
      const double v = P.rhs[i] - krow(s, i, P.x);
      r2 += v * v;
    }
    for (int cx = tid; cx < s.nx; cx += nth) {
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
    for (int64_t i = R.d0 + tid; i < R.d1; i += nth) row(i);
    for (int cx = tid; cx < s.nx; cx += nth) row(s.T + R.c0 + cx);
    put_partial(w, 0, d2, red);
    put_partial(w, 1, a2, red);
    put_partial(w, 2, l2, red);
    if (!grid_sync(w, epoch)) { status = MHM_SOLVE_BARRIER_TIMEOUT; goto done; }
    const double dn = sqrt(grid_total(w, 0, sh));
    const double an = sqrt(grid_total(w, 1, sh));
    const double ln = sqrt(grid_total(w, 2, sh));
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

struct Layout {
  size_t lam, rho, rhoP, z, zt, p, q, tmp, rfull, U, U2, cheb, part, bar, err, total;
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
  L.lam = take(T * 8); L.rho = take(T * 8); L.rhoP = take(T * 8); L.z = take(T * 8);
  L.zt = take(T * 8); L.p = take(T * 8); L.q = take(T * 8); L.tmp = take(T * 8);
  L.rfull = take(N * 8);
  L.U = take(M * 8); L.U2 = take(M * 8);
  L.cheb = take((size_t)s->nx * (s->ny + 1) * 8);
  L.part = take((size_t)grid * 4 * 8);
  L.bar = take(2 * sizeof(unsigned));
  L.err = take(sizeof(int));
  L.total = off;
  return L;
}

size_t dyn_smem(const mhm_skeleton_system* s) {
  size_t off[16];
  return smem_layout(s, off);
}

const void* kernel_for(int fs) {
  switch (fs) {
    case 1: return (const void*)skeleton_pcg_kernel<1>;
    case 2: return (const void*)skeleton_pcg_kernel<2>;
    case 3: return (const void*)skeleton_pcg_kernel<3>;
    case 4: return (const void*)skeleton_pcg_kernel<4>;
    default: return nullptr;
  }
}

// One CTA per macro row; all rows must be co-resident for the cooperative launch.
int resolve_grid(const mhm_skeleton_system* s) {
  int dev = 0, sms = 0, per_sm = 0;
  const void* kern = kernel_for(s->face_size);
  if (!kern) return 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  const size_t smem = dyn_smem(s);
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
         s->nx >= 1 && s->ny >= 1 && (int64_t)s->nx * s->ny == s->cells && s->qx && s->indptr &&
         s->indices && s->values && s->trace_end && s->cell_dofs && s->cell_g0 && s->dof_cells &&
         s->dof_slot && std::isfinite(s->coarse_ax) && std::isfinite(s->coarse_ay) &&
         s->coarse_ax > 0 && s->coarse_ay > 0;
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

extern "C" int64_t mhm_skeleton_workspace_bytes(const mhm_skeleton_system* s, int32_t grid) {
  (void)grid;
  if (!s || s->face_size < 1 || s->face_size > 4 || s->ny < 1 || s->nx < 1) return -1;
  return (int64_t)layout(s, s->ny).total;
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
            s->dof_slot, s->nx, s->ny, s->qx, s->coarse_ax, s->coarse_ay};
  P.w.lam = (double*)(base + L.lam); P.w.rho = (double*)(base + L.rho);
  P.w.rhoP = (double*)(base + L.rhoP); P.w.z = (double*)(base + L.z);
  P.w.zt = (double*)(base + L.zt); P.w.p = (double*)(base + L.p); P.w.q = (double*)(base + L.q);
  P.w.tmp = (double*)(base + L.tmp); P.w.rfull = (double*)(base + L.rfull);
  P.w.U = (double*)(base + L.U); P.w.U2 = (double*)(base + L.U2);
  P.w.cheb = (double*)(base + L.cheb); P.w.part = (double*)(base + L.part);
  P.w.bar = (unsigned*)(base + L.bar); P.w.err = (int*)(base + L.err);
  P.rhs = rhs; P.load_scale = load_scale; P.x = x; P.rtol = rtol; P.inner_rtol = inner_rtol;
  P.max_inner = max_inner; P.max_outer = max_outer; P.info = info; P.stats = stats;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // barrier counter and error flag start at zero on every call
  if (cudaMemsetAsync(base + L.bar, 0, L.total - L.bar, st) != cudaSuccess) return MHM_ERR_LAUNCH;
  if (cudaMemsetAsync(stats, 0, 4 * sizeof(double), st) != cudaSuccess) return MHM_ERR_LAUNCH;
  void* args[] = {&P};
  cudaError_t e = cudaLaunchCooperativeKernel(kernel_for(s->face_size), dim3(g), dim3(kSolveThreads),
                                              args, dyn_smem(s), st);
  return e == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}
