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
//   preconditioner P M^-1 P with M^-1 = block Jacobi over the skeleton faces;
//   c = Q G0^T (S lambda - r_lambda),  lambda = lambda0 + mu.
//
// One persistent cooperative launch does everything.  Vectors live in the caller's
// workspace; the trace-trace block S is read from the CSR rows (columns < T).  Every
// sum runs in a fixed order (per-CTA partials summed identically in every CTA), so
// results are bitwise reproducible.  Six grid barriers per CG iteration: the residual
// and the search direction are double-buffered so that values another CTA still reads
// are never overwritten in the same phase, and quantities a phase needs from other
// CTAs' DOFs (the updated residual in the cell sums, the preconditioned residual of
// a shared face) are recomputed where they are read, with the same arithmetic.  Every
// barrier is bounded: a CTA that waits too long sets the error flag, and all return.
#include <cmath>
#include <cstdint>

#include "mhm_common.cuh"

namespace mhm {
namespace {

constexpr int kGThreads = 512;
constexpr int kGWarps = kGThreads / 32;
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
  int32_t* dof_face;
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

// Totals of slots [0, n) over all CTAs, in CTA order (the same bits in every CTA).
__device__ void g_totals(const GWork& w, int n, double* out, double* sh) {
  if (threadIdx.x < 32) {
    for (int k = 0; k < n; ++k) {
      double a = 0.0;
      for (int i = threadIdx.x; i < (int)gridDim.x; i += 32) a += __ldcg(w.part + i * kSlots + k);
      a = warp_sum(a);
      if (threadIdx.x == 0) sh[k] = a;
    }
  }
  __syncthreads();
  for (int k = 0; k < n; ++k) out[k] = sh[k];
  __syncthreads();
}

// (G0 v)_i: the DOF's entries in its (at most two) cells, first cell then second.
__device__ __forceinline__ double g0_apply(const mhm_general_system& s, int64_t i, const double* v) {
  double acc = 0.0;
#pragma unroll
  for (int k = 0; k < 2; ++k) {
    const int c = s.dof_cells[2 * i + k];
    if (c >= 0) acc = fma(s.cell_g0[s.dof_entry[2 * i + k]], __ldcg(v + c), acc);
  }
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

// Projected, preconditioned residual entry of DOF i: r = rt - G0 v on its face, then
// z0_i = (M_f^-1 r_f)_i.  Also returns r_i.
__device__ __forceinline__ double dof_z0(const GParams& P, int64_t i, const double* rt, const double* v,
                                         double& ri) {
  const mhm_general_system& s = P.s;
  const int f = P.dof_face[i];
  const int64_t f0 = s.face_ptr[f];
  const int fs = (int)(s.face_ptr[f + 1] - f0);
  const double* inv = P.w.finv + (int64_t)f * kMaxFace * kMaxFace + (i - f0) * kMaxFace;
  double acc = 0.0;
  ri = 0.0;
  for (int j = 0; j < fs; ++j) {
    const double rj = __ldcg(rt + f0 + j) - g0_apply(s, f0 + j, v);
    if (f0 + j == i) ri = rj;
    acc = fma(inv[j], rj, acc);
  }
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
  double bnorm = 0.0, res = 0.0;
#define GSYNC()                                                              \
  do {                                                                       \
    if (!g_sync(w, epoch)) { status = MHM_SOLVE_BARRIER_TIMEOUT; goto done; } \
  } while (0)

  for (int64_t f = gtid; f < s.faces; f += gstride) face_inverse(s, (int)f, w.finv + f * kMaxFace * kMaxFace);
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
    // ---- outer residual rfull = b - K x over all rows ------------------------------
    {
      double r2 = 0.0;
      for (int64_t i = gtid; i < N; i += gstride) {
        double acc = P.rhs[i];
        for (int64_t k = s.indptr[i]; k < s.indptr[i + 1]; ++k)
          acc = fma(-s.values[k], __ldcg(P.x + s.indices[k]), acc);
        w.rfull[i] = acc;
        r2 = fma(acc, acc, r2);
      }
      g_partial(w, 0, r2, red);
    }
    GSYNC();
    g_totals(w, 1, tot, sh);
    res = sqrt(tot[0]) / bnorm;
    if (!isfinite(res)) { status = MHM_SOLVE_NONFINITE; goto done; }
    if (res <= P.rtol) break;
    if (outer >= P.max_outer || total_inner >= P.max_inner) { status = MHM_SOLVE_NOT_CONVERGED; goto done; }
    ++outer;
    // ---- lambda0 = G0 Q (-r_c) ---------------------------------------------------
    for (int64_t c = gtid; c < M; c += gstride) w.w[c] = -w.rfull[T + c];
    GSYNC();
    q_gemv(s, w.w, w.v);
    GSYNC();
    for (int64_t i = gtid; i < T; i += gstride) {
      w.lam0[i] = g0_apply(s, i, w.v);
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
    for (int64_t i = gtid; i < T; i += gstride) {
      double ri;
      w.z0[i] = dof_z0(P, i, w.rt[0], w.v, ri);
      w.r[i] = ri;
    }
    for (int64_t c = gtid; c < M; c += gstride) {
      double acc = 0.0;
      for (int64_t e = s.cell_ptr[c]; e < s.cell_ptr[c + 1]; ++e) {
        double ri;
        acc = fma(s.cell_g0[e], dof_z0(P, s.cell_dofs[e], w.rt[0], w.v, ri), acc);
      }
      w.w2[c] = acc;
    }
    GSYNC();
    q_gemv(s, w.w2, w.v2);
    GSYNC();
    double gamma, rr0;
    {
      double rz = 0.0, rr = 0.0;
      for (int64_t i = gtid; i < T; i += gstride) {
        const double zi = __ldcg(w.z0 + i) - g0_apply(s, i, w.v2);
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
      // stop at the inner tolerance, or once the inner residual is below half of what
      // the outer tolerance asks of the whole system
      const double floor_abs = 0.5 * P.rtol * bnorm;
      const double target = fmax(P.inner_rtol * sqrt(rr0), floor_abs);
      double beta = 0.0;
      int cur = 0;
      double rr = rr0;
      while (sqrt(rr) > target && total_inner < P.max_inner) {
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
        // P4: r = P rt, z0 = M^-1 r (face blocks); the cells' G0^T z0
        for (int64_t i = gtid; i < T; i += gstride) {
          double ri;
          w.z0[i] = dof_z0(P, i, w.rt[nxt], w.v, ri);
          w.r[i] = ri;
        }
        for (int64_t c = gtid; c < M; c += gstride) {
          double acc = 0.0;
          for (int64_t e = s.cell_ptr[c]; e < s.cell_ptr[c + 1]; ++e) {
            double ri;
            acc = fma(s.cell_g0[e], dof_z0(P, s.cell_dofs[e], w.rt[nxt], w.v, ri), acc);
          }
          w.w2[c] = acc;
        }
        GSYNC();
        // P5: v2 = Q G0^T z0
        q_gemv(s, w.w2, w.v2);
        GSYNC();
        // P6: z = P z0; (r, z) and (r, r)
        {
          double rz = 0.0, r2 = 0.0;
          for (int64_t i = gtid; i < T; i += gstride) {
            const double zi = __ldcg(w.z0 + i) - g0_apply(s, i, w.v2);
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
  }
#undef GSYNC
}

struct GLayout {
  size_t mu, rt0, rt1, p0, p1, q, r, z0, z, lam0, w, v, w2, v2, rfull, finv, dof_face, part, bar, err, total;
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
  L.dof_face = take(T * 4);
  L.part = take((size_t)grid * kSlots * 8);
  L.bar = take(2 * sizeof(unsigned));
  L.err = take(sizeof(int));
  L.total = off;
  return L;
}

__global__ void dof_face_kernel(int64_t faces, const int64_t* face_ptr, int32_t* dof_face) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t f = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; f < faces; f += stride)
    for (int64_t i = face_ptr[f]; i < face_ptr[f + 1]; ++i) dof_face[i] = (int32_t)f;
}

// The layout (everything but the matrix values, which change from solve to solve).
bool g_valid_layout(const mhm_general_system* s) {
  return s && s->trace_size >= 1 && s->cells >= 1 && s->size == s->trace_size + s->cells && s->faces >= 1 &&
         s->indptr && s->indices && s->face_ptr && s->cell_ptr && s->cell_dofs && s->cell_g0 && s->dof_cells &&
         s->dof_entry && s->coarse_inverse && s->max_face_size >= 1 && s->max_face_size <= kMaxFace &&
         s->trace_size <= INT32_MAX;
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
  P.w.part = d(L.part);
  P.w.bar = reinterpret_cast<unsigned*>(base + L.bar);
  P.w.err = reinterpret_cast<int*>(base + L.err);
  P.dof_face = reinterpret_cast<int32_t*>(base + L.dof_face);
  P.rhs = rhs;
  P.x = x;
  P.rtol = rtol;
  P.inner_rtol = inner_rtol;
  P.max_inner = max_inner;
  P.max_outer = max_outer;
  P.info = info;
  P.stats = stats;
  if (cudaMemsetAsync(base + L.bar, 0, L.total - L.bar, st) != cudaSuccess) return MHM_ERR_LAUNCH;
  int blocks = (int)((s->faces + 255) / 256);
  if (blocks > 4096) blocks = 4096;
  dof_face_kernel<<<blocks, 256, 0, st>>>(s->faces, s->face_ptr, P.dof_face);
  void* args[] = {&P};
  if (cudaLaunchCooperativeKernel((const void*)general_pcg_kernel, grid, kGThreads, args, 0, st) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}
