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
// G0 the exact geometric net-flux operator of the Cartesian macro grid.  G0^T G0
// is a scaled 2-D Dirichlet Laplacian on the macro cells, applied exactly by two
// orthonormal sine transforms (dense 64x64-class products).  The preconditioner
// is block Jacobi over skeleton faces.  K - K0 is at rounding level, so two or
// three outer corrections reach FP64 accuracy.
//
// Everything runs in one persistent cooperative kernel.  Its grid barrier is a
// counter/generation pair with a bounded spin: on timeout every CTA sets the
// error flag and returns, and the host reports MHM_SOLVE_BARRIER_TIMEOUT.
#include <cmath>

#include "mhm_common.cuh"

namespace mhm {
namespace {

constexpr int kSolveThreads = 256;
constexpr long long kSpinLimit = 1ll << 25;

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
  const double* qy;
  const double* eig;
};

struct Work {
  double *lam, *rho, *rhoP, *z, *zt, *p, *q, *tmp;  // T each
  double *rfull;                                    // N
  double *V, *W, *Y;                                // M each
  double *minv;                                     // F * fs * fs
  double *part;                                     // grid * 4
  unsigned* bar;                                    // [count, gen]
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

// Bounded grid barrier.  Returns false when the error flag is set.
__device__ bool grid_sync(const Work& w) {
  __shared__ int bad;
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned* count = w.bar;
    unsigned* gen = w.bar + 1;
    const unsigned my = atomicOr(gen, 0u);
    __threadfence();
    if (atomicAdd(count, 1u) == gridDim.x - 1) {
      atomicExch(count, 0u);
      __threadfence();
      atomicAdd(gen, 1u);
    } else {
      long long spins = 0;
      while (atomicOr(gen, 0u) == my) {
        if (++spins > kSpinLimit) {
          atomicExch(w.err, 1);
          break;
        }
        __nanosleep(64);
      }
    }
    __threadfence();
    bad = atomicOr(w.err, 0);
  }
  __syncthreads();
  return bad == 0;
}

// Sum of the per-CTA partials `slot` (fixed order, identical in every CTA).
__device__ double grid_total(const Work& w, int slot, double* sh) {
  if (threadIdx.x < 32) {
    double v = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) v += w.part[i * 4 + slot];
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

// out[i] = (S v)_i over trace rows (columns < T); scale/shift variants.
__device__ __forceinline__ double srow(const Sys& s, int64_t i, const double* v) {
  double acc = 0.0;
  for (int64_t e = s.indptr[i]; e < s.trace_end[i]; ++e) acc = fma(s.values[e], v[s.indices[e]], acc);
  return acc;
}

__device__ __forceinline__ double krow(const Sys& s, int64_t i, const double* v) {
  double acc = 0.0;
  for (int64_t e = s.indptr[i]; e < s.indptr[i + 1]; ++e) acc = fma(s.values[e], v[s.indices[e]], acc);
  return acc;
}

// (G0 y)_i for trace DOF i.
__device__ __forceinline__ double g0_apply(const Sys& s, int64_t i, const double* y) {
  double acc = 0.0;
  for (int k = 0; k < 2; ++k) {
    const int c = s.dof_cells[2 * i + k];
    if (c >= 0) acc = fma(s.g0[(size_t)c * s.t + s.dof_slot[2 * i + k]], y[c], acc);
  }
  return acc;
}

// Coarse solve stage 1: W[:, kx] = Qy (V Qx)[:, kx] / eig[:, kx].
__device__ void coarse_stage1(const Sys& s, const Work& w, const double* V, double* col) {
  for (int kx = blockIdx.x; kx < s.nx; kx += gridDim.x) {
    for (int iy = threadIdx.x; iy < s.ny; iy += blockDim.x) {
      double acc = 0.0;
      for (int ix = 0; ix < s.nx; ++ix) acc = fma(V[(size_t)iy * s.nx + ix], s.qx[(size_t)ix * s.nx + kx], acc);
      col[iy] = acc;
    }
    __syncthreads();
    for (int ky = threadIdx.x; ky < s.ny; ky += blockDim.x) {
      double acc = 0.0;
      for (int iy = 0; iy < s.ny; ++iy) acc = fma(s.qy[(size_t)ky * s.ny + iy], col[iy], acc);
      w.W[(size_t)ky * s.nx + kx] = acc / s.eig[(size_t)ky * s.nx + kx];
    }
    __syncthreads();
  }
}

// Coarse solve stage 2: Y[:, ix] = Qy (W Qx)[:, ix].
__device__ void coarse_stage2(const Sys& s, const Work& w, double* Y, double* col) {
  for (int ix = blockIdx.x; ix < s.nx; ix += gridDim.x) {
    for (int ky = threadIdx.x; ky < s.ny; ky += blockDim.x) {
      double acc = 0.0;
      for (int kx = 0; kx < s.nx; ++kx) acc = fma(w.W[(size_t)ky * s.nx + kx], s.qx[(size_t)kx * s.nx + ix], acc);
      col[ky] = acc;
    }
    __syncthreads();
    for (int iy = threadIdx.x; iy < s.ny; iy += blockDim.x) {
      double acc = 0.0;
      for (int ky = 0; ky < s.ny; ++ky) acc = fma(s.qy[(size_t)iy * s.ny + ky], col[ky], acc);
      Y[(size_t)iy * s.nx + ix] = acc;
    }
    __syncthreads();
  }
}

// V_K = sum_a g0[K,a] * v[dof(K,a)]
__device__ void g0t(const Sys& s, const double* v, double* V, int64_t gtid, int64_t gstride) {
  for (int64_t c = gtid; c < s.M; c += gstride) {
    double acc = 0.0;
    for (int a = 0; a < s.t; ++a) acc = fma(s.g0[(size_t)c * s.t + a], v[s.cell_dofs[(size_t)c * s.t + a]], acc);
    V[c] = acc;
  }
}

__global__ void __launch_bounds__(kSolveThreads) skeleton_pcg_kernel(const Params P) {
  const Sys& s = P.s;
  const Work& w = P.w;
  __shared__ double red[32];
  __shared__ double sh[2];
  extern __shared__ double col[];
  const int64_t gtid = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t gstride = (int64_t)gridDim.x * blockDim.x;
  const int fs = s.fs;
  int status = MHM_SOLVE_OK;
  int total_inner = 0, outer = 0;
#define SYNC_OR_EXIT() \
  do {                 \
    if (!grid_sync(w)) { status = MHM_SOLVE_BARRIER_TIMEOUT; goto done; } \
  } while (0)

  // ---- face-block Jacobi inverses (Gauss-Jordan with partial pivoting) -------
  for (int64_t f = gtid; f < s.F; f += gstride) {
    double a[8][16];
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
      for (int c = 0; c < fs; ++c) w.minv[(size_t)f * fs * fs + r * fs + c] = a[r][fs + c];
  }
  // x = 0, r_full = rhs, ||rhs||
  {
    double b2 = 0.0;
    for (int64_t i = gtid; i < s.N; i += gstride) {
      P.x[i] = 0.0;
      const double v = P.rhs[i];
      w.rfull[i] = v;
      b2 += v * v;
    }
    put_partial(w, 0, b2, red);
  }
  SYNC_OR_EXIT();
  {
    const double bnorm = sqrt(grid_total(w, 0, sh));
    double res = 1.0;
    if (bnorm == 0.0) goto finish;
    for (outer = 0; outer < P.max_outer; ++outer) {
      if (outer > 0) {
        // r_full = rhs - K x
        double r2 = 0.0;
        for (int64_t i = gtid; i < s.N; i += gstride) {
          const double v = P.rhs[i] - krow(s, i, P.x);
          w.rfull[i] = v;
          r2 += v * v;
        }
        put_partial(w, 0, r2, red);
        SYNC_OR_EXIT();
        res = sqrt(grid_total(w, 0, sh)) / bnorm;
        if (outer == 1 && blockIdx.x == 0 && threadIdx.x == 0) P.stats[2] = res;
        if (!isfinite(res)) { status = MHM_SOLVE_NONFINITE; goto finish; }
        if (res <= P.rtol) break;
      }
      const double itol = (outer == 0) ? P.inner_rtol : fmax(P.inner_rtol, 1e-4);
      // lambda0 = -G0 C^-1 r2
      for (int64_t c = gtid; c < s.M; c += gstride) w.V[c] = w.rfull[s.T + c];
      SYNC_OR_EXIT();
      coarse_stage1(s, w, w.V, col);
      SYNC_OR_EXIT();
      coarse_stage2(s, w, w.Y, col);
      SYNC_OR_EXIT();
      for (int64_t i = gtid; i < s.T; i += gstride) w.lam[i] = -g0_apply(s, i, w.Y);
      SYNC_OR_EXIT();
      // rhoP = r1 - S lam ; V = G0^T rhoP
      for (int64_t i = gtid; i < s.T; i += gstride) w.rhoP[i] = w.rfull[i] - srow(s, i, w.lam);
      SYNC_OR_EXIT();
      g0t(s, w.rhoP, w.V, gtid, gstride);
      SYNC_OR_EXIT();
      coarse_stage1(s, w, w.V, col);
      SYNC_OR_EXIT();
      coarse_stage2(s, w, w.Y, col);
      SYNC_OR_EXIT();
      // rho = rhoP - G0 Y ; zt = Minv rho
      {
        double r2 = 0.0;
        for (int64_t f = gtid; f < s.F; f += gstride) {
          double rl[8];
          for (int r = 0; r < fs; ++r) {
            const int64_t i = f * fs + r;
            rl[r] = w.rhoP[i] - g0_apply(s, i, w.Y);
            w.rho[i] = rl[r];
            r2 += rl[r] * rl[r];
          }
          for (int r = 0; r < fs; ++r) {
            double acc = 0.0;
            for (int c = 0; c < fs; ++c) acc = fma(w.minv[(size_t)f * fs * fs + r * fs + c], rl[c], acc);
            w.zt[f * fs + r] = acc;
          }
        }
        put_partial(w, 1, r2, red);
      }
      SYNC_OR_EXIT();
      const double r0 = sqrt(grid_total(w, 1, sh));
      g0t(s, w.zt, w.V, gtid, gstride);
      SYNC_OR_EXIT();
      coarse_stage1(s, w, w.V, col);
      SYNC_OR_EXIT();
      coarse_stage2(s, w, w.Y, col);
      SYNC_OR_EXIT();
      {
        double rz = 0.0;
        for (int64_t i = gtid; i < s.T; i += gstride) {
          const double zi = w.zt[i] - g0_apply(s, i, w.Y);
          w.z[i] = zi;
          w.p[i] = zi;
          rz += w.rho[i] * zi;
        }
        put_partial(w, 2, rz, red);
      }
      SYNC_OR_EXIT();
      double rz = grid_total(w, 2, sh);
      {
        double pq = 0.0;
        for (int64_t i = gtid; i < s.T; i += gstride) {
          const double qi = srow(s, i, w.p);
          w.q[i] = qi;
          pq += w.p[i] * qi;
        }
        put_partial(w, 3, pq, red);
      }
      SYNC_OR_EXIT();
      int k = 0;
      if (r0 > 0.0) {
        for (k = 0; k < P.max_inner; ++k) {
          const double pq = grid_total(w, 3, sh);
          if (!(pq > 0.0)) { status = MHM_SOLVE_BREAKDOWN; break; }
          const double alpha = rz / pq;
          for (int64_t i = gtid; i < s.T; i += gstride) {
            w.lam[i] = fma(alpha, w.p[i], w.lam[i]);
            w.rhoP[i] = fma(-alpha, w.q[i], w.rho[i]);
          }
          for (int64_t c = gtid; c < s.M; c += gstride) {
            double acc = 0.0;
            for (int a = 0; a < s.t; ++a) {
              const int64_t i = s.cell_dofs[(size_t)c * s.t + a];
              acc = fma(s.g0[(size_t)c * s.t + a], fma(-alpha, w.q[i], w.rho[i]), acc);
            }
            w.V[c] = acc;
          }
          SYNC_OR_EXIT();
          coarse_stage1(s, w, w.V, col);
          SYNC_OR_EXIT();
          coarse_stage2(s, w, w.Y, col);
          SYNC_OR_EXIT();
          {
            double r2 = 0.0;
            for (int64_t f = gtid; f < s.F; f += gstride) {
              double rl[8];
              for (int r = 0; r < fs; ++r) {
                const int64_t i = f * fs + r;
                rl[r] = w.rhoP[i] - g0_apply(s, i, w.Y);
                w.rho[i] = rl[r];
                r2 += rl[r] * rl[r];
              }
              for (int r = 0; r < fs; ++r) {
                double acc = 0.0;
                for (int c = 0; c < fs; ++c) acc = fma(w.minv[(size_t)f * fs * fs + r * fs + c], rl[c], acc);
                w.zt[f * fs + r] = acc;
              }
            }
            // V2 = G0^T (Minv rho), recomputed per cell from rhoP and Y (no extra barrier)
            for (int64_t c = gtid; c < s.M; c += gstride) {
              double acc = 0.0;
              for (int a = 0; a < s.t; a += fs) {
                const int64_t i0 = s.cell_dofs[(size_t)c * s.t + a];
                const int64_t f = i0 / fs;
                double rl[8];
                for (int r = 0; r < fs; ++r) rl[r] = w.rhoP[f * fs + r] - g0_apply(s, f * fs + r, w.Y);
                for (int r = 0; r < fs; ++r) {
                  double zr = 0.0;
                  for (int cc = 0; cc < fs; ++cc) zr = fma(w.minv[(size_t)f * fs * fs + r * fs + cc], rl[cc], zr);
                  acc = fma(s.g0[(size_t)c * s.t + a + r], zr, acc);
                }
              }
              w.V[c] = acc;  // V is free: stage 1 of this iteration already consumed it
            }
            put_partial(w, 1, r2, red);
          }
          SYNC_OR_EXIT();
          {
            const double rn = sqrt(grid_total(w, 1, sh));
            if (!isfinite(rn)) { status = MHM_SOLVE_NONFINITE; break; }
            if (rn <= itol * r0) { ++k; break; }
          }
          coarse_stage1(s, w, w.V, col);
          SYNC_OR_EXIT();
          coarse_stage2(s, w, w.Y, col);
          SYNC_OR_EXIT();
          {
            double rzn = 0.0;
            for (int64_t i = gtid; i < s.T; i += gstride) {
              const double zi = w.zt[i] - g0_apply(s, i, w.Y);
              w.z[i] = zi;
              rzn += w.rho[i] * zi;
            }
            put_partial(w, 2, rzn, red);
          }
          SYNC_OR_EXIT();
          {
            const double rzn = grid_total(w, 2, sh);
            const double beta = rzn / rz;
            rz = rzn;
            double pq = 0.0;
            for (int64_t i = gtid; i < s.T; i += gstride) {
              const double pi = fma(beta, w.p[i], w.z[i]);
              const double qi = fma(beta, w.q[i], srow(s, i, w.z));
              w.p[i] = pi;
              w.q[i] = qi;
              pq += pi * qi;
            }
            put_partial(w, 3, pq, red);
          }
          SYNC_OR_EXIT();
        }
        if (k >= P.max_inner && status == MHM_SOLVE_OK) status = MHM_SOLVE_NOT_CONVERGED;
      }
      total_inner += k;
      if (status != MHM_SOLVE_OK) goto finish;
      // c = C^-1 G0^T (S lam - r1)
      for (int64_t i = gtid; i < s.T; i += gstride) w.tmp[i] = srow(s, i, w.lam) - w.rfull[i];
      SYNC_OR_EXIT();
      g0t(s, w.tmp, w.V, gtid, gstride);
      SYNC_OR_EXIT();
      coarse_stage1(s, w, w.V, col);
      SYNC_OR_EXIT();
      coarse_stage2(s, w, w.Y, col);
      SYNC_OR_EXIT();
      for (int64_t i = gtid; i < s.T; i += gstride) P.x[i] += w.lam[i];
      for (int64_t c = gtid; c < s.M; c += gstride) P.x[s.T + c] += w.Y[c];
      SYNC_OR_EXIT();
    }
    if (outer >= P.max_outer) {
      // final residual after the last correction
      double r2 = 0.0;
      for (int64_t i = gtid; i < s.N; i += gstride) {
        const double v = P.rhs[i] - krow(s, i, P.x);
        r2 += v * v;
      }
      put_partial(w, 0, r2, red);
      SYNC_OR_EXIT();
      res = sqrt(grid_total(w, 0, sh)) / bnorm;
      if (!(res <= P.rtol) && status == MHM_SOLVE_OK) status = MHM_SOLVE_NOT_CONVERGED;
    }
  finish:
    // physical certificate (system.py:481-507): ||K x - b|| / max(||b||, ||load_scale||, || |K||x| ||)
    {
      double d2 = 0.0, a2 = 0.0, l2 = 0.0;
      for (int64_t i = gtid; i < s.N; i += gstride) {
        double acc = 0.0, aacc = 0.0;
        for (int64_t e = s.indptr[i]; e < s.indptr[i + 1]; ++e) {
          const double xv = P.x[s.indices[e]];
          acc = fma(s.values[e], xv, acc);
          aacc = fma(fabs(s.values[e]), fabs(xv), aacc);
        }
        const double d = acc - P.rhs[i];
        d2 += d * d;
        a2 += aacc * aacc;
        const double ls = P.load_scale ? P.load_scale[i] : 0.0;
        l2 += ls * ls;
      }
      put_partial(w, 0, d2, red);
      put_partial(w, 1, a2, red);
      put_partial(w, 2, l2, red);
      if (!grid_sync(w)) { status = MHM_SOLVE_BARRIER_TIMEOUT; goto done; }
      const double dn = sqrt(grid_total(w, 0, sh));
      const double an = sqrt(grid_total(w, 1, sh));
      const double ln = sqrt(grid_total(w, 2, sh));
      const double scale = fmax(fmax(bnorm, ln), fmax(an, 2.2250738585072014e-308));
      if (blockIdx.x == 0 && threadIdx.x == 0) {
        P.stats[0] = (bnorm > 0.0) ? dn / bnorm : 0.0;
        P.stats[1] = dn / scale;
      }
    }
  }
done:
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    P.info[0] = status;
    P.info[1] = total_inner;
    P.info[2] = outer;
    P.info[3] = atomicOr(w.err, 0);
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
  size_t lam, rho, rhoP, z, zt, p, q, tmp, rfull, V, W, Y, minv, part, bar, err, total;
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
  L.V = take(M * 8); L.W = take(M * 8); L.Y = take(M * 8);
  L.minv = take((size_t)s->faces * s->face_size * s->face_size * 8);
  L.part = take((size_t)grid * 4 * 8);
  L.bar = take(2 * sizeof(unsigned));
  L.err = take(sizeof(int));
  L.total = off;
  return L;
}

int resolve_grid(int grid, int ny_col) {
  int dev = 0, sms = 0, per_sm = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return -1;
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return -1;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, skeleton_pcg_kernel, kSolveThreads,
                                                    (size_t)ny_col * 8) != cudaSuccess)
    return -1;
  const int cap = sms * (per_sm > 0 ? per_sm : 1);
  if (grid <= 0) grid = sms;
  return grid < cap ? grid : cap;
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
  if (!s || s->face_size < 1 || s->face_size > 8) return -1;
  const int g = resolve_grid(grid, s->ny);
  if (g <= 0) return -1;
  return (int64_t)layout(s, g).total;
}

extern "C" int mhm_skeleton_solve(const mhm_skeleton_system* s, const double* rhs,
                                  const double* load_scale, double* x, double rtol,
                                  double inner_rtol, int32_t max_inner, int32_t max_outer,
                                  int32_t grid, void* workspace, int64_t workspace_bytes,
                                  int32_t* info, double* stats, void* stream) {
  if (!s || !rhs || !x || !workspace || !info || !stats) return MHM_ERR_ARGUMENT;
  if (s->size != s->trace_size + s->cells || s->face_size < 1 || s->face_size > 8 ||
      (int64_t)s->faces * s->face_size != s->trace_size || s->cell_width % s->face_size != 0 ||
      (int64_t)s->nx * s->ny != s->cells || max_inner < 1 || max_outer < 1 || !(rtol > 0) ||
      !(inner_rtol > 0))
    return MHM_ERR_ARGUMENT;
  const int g = resolve_grid(grid, s->ny);
  if (g <= 0) return MHM_ERR_LAUNCH;
  const Layout L = layout(s, g);
  if ((int64_t)L.total > workspace_bytes) return MHM_ERR_ARGUMENT;
  char* base = static_cast<char*>(workspace);
  Params P{};
  P.s = Sys{s->size, s->trace_size, s->indptr, s->indices, s->values, s->trace_end, s->faces,
            s->face_size, s->cells, s->cell_width, s->cell_dofs, s->cell_g0, s->dof_cells,
            s->dof_slot, s->nx, s->ny, s->qx, s->qy, s->coarse_eig};
  P.w.lam = (double*)(base + L.lam); P.w.rho = (double*)(base + L.rho);
  P.w.rhoP = (double*)(base + L.rhoP); P.w.z = (double*)(base + L.z);
  P.w.zt = (double*)(base + L.zt); P.w.p = (double*)(base + L.p); P.w.q = (double*)(base + L.q);
  P.w.tmp = (double*)(base + L.tmp); P.w.rfull = (double*)(base + L.rfull);
  P.w.V = (double*)(base + L.V); P.w.W = (double*)(base + L.W); P.w.Y = (double*)(base + L.Y);
  P.w.minv = (double*)(base + L.minv); P.w.part = (double*)(base + L.part);
  P.w.bar = (unsigned*)(base + L.bar); P.w.err = (int*)(base + L.err);
  P.rhs = rhs; P.load_scale = load_scale; P.x = x; P.rtol = rtol; P.inner_rtol = inner_rtol;
  P.max_inner = max_inner; P.max_outer = max_outer; P.info = info; P.stats = stats;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // barrier counters and error flag start at zero on every call
  if (cudaMemsetAsync(base + L.bar, 0, L.total - L.bar, st) != cudaSuccess) return MHM_ERR_LAUNCH;
  if (cudaMemsetAsync(stats, 0, 4 * sizeof(double), st) != cudaSuccess) return MHM_ERR_LAUNCH;
  void* args[] = {&P};
  const size_t smem = (size_t)s->ny * 8;
  cudaError_t e = cudaLaunchCooperativeKernel((const void*)skeleton_pcg_kernel, dim3(g),
                                              dim3(kSolveThreads), args, smem, st);
  return e == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}
