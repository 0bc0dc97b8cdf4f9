// Cartesian Q1 macrocells: fused assembly, constrained condensation and Schur block.
//
// One CTA owns one macrocell for its whole life: the fine-grid operator, the
// factor and the right-hand sides never leave shared memory; only the
// responses (needed later for reconstruction), the (t+1)^2 Schur block and
// its load are written to HBM.
//
// Reference algorithm (PyMHM 1.3.2, src/pymhm/):
//   operators        fem/scalar/quadrilateral.py:191-253 (Q1 Gram blocks, mass, load)
//   trace coupling   fem/scalar/quadrilateral.py:256-298
//   local contract   core/contracts.py:92-211 (Z = 1, C = M 1, retained action A Z)
//   augmented system core/condensation.py:125-174 (constraint scaling min(1, max|A|/max|C|))
//   checked solve    linalg/linear.py:132-152, 262-310 (columnwise residual criterion)
//   Schur block/load core/contributions.py:14-74, core/reconstruction.py:91-127
//
// B200 design: the augmented saddle [[A, c],[c^T, 0]] is never factored as a
// saddle.  A is a 9-point Neumann operator whose kernel is the constant; pinning
// the last node (A + a_pp e_p e_p^T) and scaling it symmetrically to unit
// diagonal gives an SPD matrix that is block tridiagonal over the lines of the
// local grid (nny blocks of nnx x nnx).  It is factored by block LDL^T with the
// explicit inverse of every Schur-complement block S_y = A_yy - B_y S_{y-1}^-1
// B_y^T (Gauss-Jordan, one barrier per pivot), so every refinement sweep is
// 2 nny dense block steps applied to all right-hand sides at once.  The exact
// augmented inverse is recovered by a rank-one kernel correction and FP64
// residual refinement against the original augmented operator, so the
// accepted result is the augmented system's solution to the requested
// tolerance, whatever arithmetic the factor used (binary64, or binary32 for
// MHM_PRECISION_MIXED).
#include <cmath>
#include <cstdio>

#include "mhm_common.cuh"

namespace mhm {
namespace {

constexpr int kThreads = 256;
constexpr int kMaxQuad = 8;

struct Q1Args {
  int nx, ny, rx, ry, nnx, nny, n, t, w, tfh, tfv, kmax, jmax;
  int NYf;
  double hx, hy, area;
  const double* table;
  const int8_t* sign;
  const int8_t* orient;
  int kmode;
  const double* kappa;
  double k0, k1, k2;
  int smode;
  const double* src;
  double s0;
  int qorder;
  double gpt[kMaxQuad], gwt[kMaxQuad];
  int max_refine;
  double tol;
  double* sol;
  double* blocks;
  double* loads;
  uint8_t* corrected;
  int32_t* status;
  int32_t* iters;
  // shared-memory carve-up (byte offsets)
  size_t off_sinv, off_gj, off_cpl, off_tmp, off_sten, off_vec, off_work, off_misc, smem;
};

// Closed form of the Q1 element Gram entry int grad(phi_a) . K grad(phi_c) on an
// hx-by-hy rectangle with constant K, nodes ordered x-fastest (a = ay*2 + ax).
// Equal to the reference's 4x4-point Gauss sum (exact for Q1) up to rounding.
__device__ __forceinline__ double elem_k(double kxx, double kxy, double kyy, double rxy,
                                         double ryx, int a, int c) {
  const int ax = a & 1, ay = a >> 1, cx = c & 1, cy = c >> 1;
  const double s1x = (ax == cx) ? 1.0 : -1.0, m1y = (ay == cy) ? 2.0 : 1.0;
  const double m1x = (ax == cx) ? 2.0 : 1.0, s1y = (ay == cy) ? 1.0 : -1.0;
  double v = (kxx * rxy * (s1x * m1y) + kyy * ryx * (m1x * s1y)) / 6.0;
  if (kxy != 0.0) {
    const double dax = ax ? 0.5 : -0.5, day = ay ? 0.5 : -0.5;
    const double dcx = cx ? 0.5 : -0.5, dcy = cy ? 0.5 : -0.5;
    v += kxy * (dax * dcy + dcx * day);
  }
  return v;
}

struct Side {
  int s, q;
};

// Trace column j -> (side, local face DOF).
__device__ __forceinline__ Side trace_side(const Q1Args& a, int j) {
  if (j < a.tfh) return {0, j};
  j -= a.tfh;
  if (j < a.tfv) return {1, j};
  j -= a.tfv;
  if (j < a.tfh) return {2, j};
  return {3, j - a.tfh};
}

__device__ __forceinline__ int side_len(const Q1Args& a, int s) { return (s & 1) ? a.nny : a.nnx; }

__device__ __forceinline__ int side_node(const Q1Args& a, int s, int k) {
  switch (s) {
    case 0: return k;
    case 1: return k * a.nnx + a.nnx - 1;
    case 2: return (a.nny - 1) * a.nnx + k;
    default: return k * a.nnx;
  }
}

__device__ __forceinline__ double coupling(const Q1Args& a, int cell, int s, int k, int q) {
  const int kind = s & 1;
  const int orient = a.orient[cell * 4 + s];
  const double v = a.table[((kind * 2 + orient) * a.kmax + k) * a.jmax + q];
  return a.sign[cell * 4 + s] * v;
}

// Entry i of right-hand-side column col: [f | B | A 1].
__device__ __forceinline__ double rhs_entry(const Q1Args& a, int cell, int col, int i,
                                            const double* fvec, const double* az) {
  if (i >= a.n) return 0.0;
  if (col == 0) return fvec[i];
  if (col == a.w - 1) return az[i];
  const Side sd = trace_side(a, col - 1);
  const int ix = i % a.nnx, iy = i / a.nnx;
  int k = -1;
  switch (sd.s) {
    case 0: k = (iy == 0) ? ix : -1; break;
    case 1: k = (ix == a.nnx - 1) ? iy : -1; break;
    case 2: k = (iy == a.nny - 1) ? ix : -1; break;
    default: k = (ix == 0) ? iy : -1; break;
  }
  return k < 0 ? 0.0 : coupling(a, cell, sd.s, k, sd.q);
}

// Lower 9-point stencil slots of node i: 0 diag, 1 (i-1), 2 (i-nnx+1), 3 (i-nnx), 4 (i-nnx-1).
__device__ __forceinline__ int stencil_offset(const Q1Args& a, int slot) {
  return slot == 0 ? 0 : slot == 1 ? 1 : slot == 2 ? a.nnx - 1 : slot == 3 ? a.nnx : a.nnx + 1;
}

// (A x)_i from the lower stencil of i and the lower stencils of its upper neighbours.
__device__ __forceinline__ double stencil_apply(const Q1Args& a, const double* sten, int i,
                                                const double* x) {
  const int ix = i % a.nnx, iy = i / a.nnx, nnx = a.nnx;
  const double* s = sten + 5 * i;
  double acc = s[0] * x[i];
  if (ix > 0) acc = fma(s[1], x[i - 1], acc);
  if (iy > 0 && ix < nnx - 1) acc = fma(s[2], x[i - nnx + 1], acc);
  if (iy > 0) acc = fma(s[3], x[i - nnx], acc);
  if (iy > 0 && ix > 0) acc = fma(s[4], x[i - nnx - 1], acc);
  if (ix < nnx - 1) acc = fma(sten[5 * (i + 1) + 1], x[i + 1], acc);
  if (iy < a.nny - 1) {
    if (ix > 0) acc = fma(sten[5 * (i + nnx - 1) + 2], x[i + nnx - 1], acc);
    acc = fma(sten[5 * (i + nnx) + 3], x[i + nnx], acc);
    if (ix < nnx - 1) acc = fma(sten[5 * (i + nnx + 1) + 4], x[i + nnx + 1], acc);
  }
  return acc;
}

// Minimum resident CTAs per SM for the factor precision (register budget).
template <typename T>
struct Occupancy {
  static constexpr int value = sizeof(T) == 8 ? 2 : 3;
};

template <typename T>
__global__ void __launch_bounds__(kThreads, Occupancy<T>::value) q1_condense_kernel(const Q1Args a) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int cell = blockIdx.x;
  const int tid = threadIdx.x;
  const int n = a.n, nnx = a.nnx, nny = a.nny, w = a.w, t = a.t;
  const int nb = nnx * nnx;
  T* sinv = reinterpret_cast<T*>(smem + a.off_sinv);  // nny blocks of nnx x nnx
  T* gj0 = reinterpret_cast<T*>(smem + a.off_gj);     // Gauss-Jordan ping-pong
  T* gj1 = gj0 + nb;
  T* cdn = reinterpret_cast<T*>(smem + a.off_cpl);    // (n, 3): to (y-1, x-1), (y-1, x), (y-1, x+1)
  T* dg = cdn + 3 * n;                                // (n): scaled diagonal
  T* dl = dg + n;                                     // (n): scaled coupling to (y, x-1)
  T* tmp = reinterpret_cast<T*>(smem + a.off_tmp);    // (nnx, w)
  double* sten = reinterpret_cast<double*>(smem + a.off_sten);
  double* fvec = reinterpret_cast<double*>(smem + a.off_vec);
  double* az = fvec + n;
  double* ctil = az + n;
  double* dsc = ctil + n;
  T* work = reinterpret_cast<T*>(smem + a.off_work);
  double* kel = reinterpret_cast<double*>(smem + a.off_work);  // aliases work during assembly
  double* fel = kel + 3 * a.rx * a.ry;
  double* red = reinterpret_cast<double*>(smem + a.off_misc);
  double* bnorm = red + 32;
  double* rnorm = bnorm + w;
  double* cmu = rnorm + w;
  double* cshift = cmu + w;
  int* conv = reinterpret_cast<int*>(cshift + w);
  int* flag = conv + w;

  const int cx = cell % a.nx, cy = cell / a.nx;
  const int ne = a.rx * a.ry;
  double* xg = a.sol + (size_t)cell * w * (n + 1);

  // ---- element coefficients and element loads --------------------------------
  for (int e = tid; e < ne; e += blockDim.x) {
    const int ex = e % a.rx, ey = e / a.rx;
    const size_t g = (size_t)(cx * a.rx + ex) * a.NYf + (cy * a.ry + ey);
    double kxx, kxy, kyy;
    if (a.kmode == 0) {
      kxx = a.k0; kxy = a.k1; kyy = a.k2;
    } else if (a.kmode == 1) {
      kxx = kyy = a.kappa[g]; kxy = 0.0;
    } else {
      kxx = a.kappa[3 * g]; kxy = a.kappa[3 * g + 1]; kyy = a.kappa[3 * g + 2];
    }
    kel[3 * e] = kxx; kel[3 * e + 1] = kxy; kel[3 * e + 2] = kyy;
    double fe[4];
    if (a.smode == 2) {
      const int Q = a.qorder;
      fe[0] = fe[1] = fe[2] = fe[3] = 0.0;
      for (int qy = 0; qy < Q; ++qy)
        for (int qx = 0; qx < Q; ++qx) {
          const double xi = a.gpt[qx], eta = a.gpt[qy];
          const double wq = a.gwt[qx] * a.gwt[qy];
          const double f = a.src[g * (size_t)(Q * Q) + qy * Q + qx];
          fe[0] += wq * ((1 - xi) * (1 - eta)) * f;
          fe[1] += wq * (xi * (1 - eta)) * f;
          fe[2] += wq * ((1 - xi) * eta) * f;
          fe[3] += wq * (xi * eta) * f;
        }
      for (int c = 0; c < 4; ++c) fe[c] *= a.area;
    } else {
      const double s = (a.smode == 0) ? a.s0 : a.src[g];
      fe[0] = fe[1] = fe[2] = fe[3] = a.area * (s * 0.25);
    }
    for (int c = 0; c < 4; ++c) fel[4 * e + c] = fe[c];
  }
  if (tid < w) { conv[tid] = 0; }
  if (tid == 0) flag[0] = 0;
  __syncthreads();

  // ---- node-wise gather of the lower stencil, load and constraint -------------
  const double rxy = a.hy / a.hx, ryx = a.hx / a.hy;
  double amax = 0.0, fro = 0.0, cmax = 0.0;
  for (int i = tid; i < n; i += blockDim.x) {
    const int ix = i % nnx, iy = i / nnx;
    double s[5] = {0, 0, 0, 0, 0};
    double f = 0.0;
    int count = 0;
    // candidate elements: E00 (ix-1,iy-1) local 3; E10 (ix,iy-1) local 2;
    //                     E01 (ix-1,iy) local 1;   E11 (ix,iy) local 0
    const bool l = ix > 0, r = ix < a.rx, d = iy > 0, u = iy < a.ry;
    if (l && d) {
      const int e = (iy - 1) * a.rx + ix - 1;
      const double* k = kel + 3 * e;
      s[0] += elem_k(k[0], k[1], k[2], rxy, ryx, 3, 3);
      s[1] += elem_k(k[0], k[1], k[2], rxy, ryx, 3, 2);
      s[3] += elem_k(k[0], k[1], k[2], rxy, ryx, 3, 1);
      s[4] += elem_k(k[0], k[1], k[2], rxy, ryx, 3, 0);
      f += fel[4 * e + 3];
      ++count;
    }
    if (r && d) {
      const int e = (iy - 1) * a.rx + ix;
      const double* k = kel + 3 * e;
      s[0] += elem_k(k[0], k[1], k[2], rxy, ryx, 2, 2);
      s[2] += elem_k(k[0], k[1], k[2], rxy, ryx, 2, 1);
      s[3] += elem_k(k[0], k[1], k[2], rxy, ryx, 2, 0);
      f += fel[4 * e + 2];
      ++count;
    }
    if (l && u) {
      const int e = iy * a.rx + ix - 1;
      const double* k = kel + 3 * e;
      s[0] += elem_k(k[0], k[1], k[2], rxy, ryx, 1, 1);
      s[1] += elem_k(k[0], k[1], k[2], rxy, ryx, 1, 0);
      f += fel[4 * e + 1];
      ++count;
    }
    if (r && u) {
      const int e = iy * a.rx + ix;
      const double* k = kel + 3 * e;
      s[0] += elem_k(k[0], k[1], k[2], rxy, ryx, 0, 0);
      f += fel[4 * e + 0];
      ++count;
    }
    for (int q = 0; q < 5; ++q) sten[5 * i + q] = s[q];
    fvec[i] = f;
    ctil[i] = count * (a.area * 0.25);
    amax = fmax(amax, fabs(s[0]));
    fro += s[0] * s[0];
    for (int q = 1; q < 5; ++q) {
      amax = fmax(amax, fabs(s[q]));
      fro += 2.0 * s[q] * s[q];
    }
    cmax = fmax(cmax, ctil[i]);
  }
  __syncthreads();
  // retained action A 1 (compensated row sums) and finiteness
  double az2 = 0.0;
  int nonzero = 0, nonfinite = 0;
  for (int i = tid; i < n; i += blockDim.x) {
    const int ix = i % nnx, iy = i / nnx;
    const double* s = sten + 5 * i;
    double hi = 0.0, lo = 0.0;
    dd_add(hi, lo, s[0]);
    if (ix > 0) dd_add(hi, lo, s[1]);
    if (iy > 0 && ix < nnx - 1) dd_add(hi, lo, s[2]);
    if (iy > 0) dd_add(hi, lo, s[3]);
    if (iy > 0 && ix > 0) dd_add(hi, lo, s[4]);
    if (ix < nnx - 1) dd_add(hi, lo, sten[5 * (i + 1) + 1]);
    if (iy < nny - 1) {
      if (ix > 0) dd_add(hi, lo, sten[5 * (i + nnx - 1) + 2]);
      dd_add(hi, lo, sten[5 * (i + nnx) + 3]);
      if (ix < nnx - 1) dd_add(hi, lo, sten[5 * (i + nnx + 1) + 4]);
    }
    const double v = hi + lo;
    az[i] = v;
    az2 += v * v;
    nonzero |= (v != 0.0);
    if (!isfinite(v) || !isfinite(fvec[i])) nonfinite = 1;
  }
  amax = block_max(amax, red);
  fro = block_sum(fro, red);
  cmax = block_max(cmax, red);
  az2 = block_sum(az2, red);
  const int any_nonzero = __syncthreads_or(nonzero);
  const int any_nonfinite = __syncthreads_or(nonfinite);
  int st = MHM_CELL_OK;
  if (any_nonfinite || !isfinite(amax)) st = MHM_CELL_NONFINITE;
  // declared-kernel test at the matrix scale (contracts.py:175-186)
  if (st == MHM_CELL_OK && amax > 0.0 &&
      sqrt(az2) / amax > 1e-10 * (sqrt(fro) / amax) * sqrt((double)n))
    st = MHM_CELL_KERNEL;
  // constraint scaling (condensation.py:160-166) and its kernel pairing
  const double scale = (amax > 0.0) ? amax : 1.0;
  const double cfac = fmin(1.0, scale / cmax);
  double zc_part = 0.0;
  for (int i = tid; i < n; i += blockDim.x) {
    ctil[i] *= cfac;
    zc_part += ctil[i];
  }
  const double zc = block_sum(zc_part, red);

  // ---- pinned, Jacobi-scaled operator in line-block form -----------------------
  const int pin = n - 1;
  for (int i = tid; i < n; i += blockDim.x) {
    const double dii = sten[5 * i] * (i == pin ? 2.0 : 1.0);
    dsc[i] = (dii > 0.0) ? rsqrt(dii) : 0.0;
  }
  __syncthreads();
  for (int i = tid; i < n; i += blockDim.x) {
    const int ix = i % nnx, iy = i / nnx;
    const double si = dsc[i];
    const double* s = sten + 5 * i;
    dg[i] = T(s[0] * (i == pin ? 2.0 : 1.0) * si * si);
    dl[i] = ix > 0 ? T(s[1] * si * dsc[i - 1]) : T(0);
    cdn[3 * i + 0] = (iy > 0 && ix > 0) ? T(s[4] * si * dsc[i - nnx - 1]) : T(0);
    cdn[3 * i + 1] = iy > 0 ? T(s[3] * si * dsc[i - nnx]) : T(0);
    cdn[3 * i + 2] = (iy > 0 && ix < nnx - 1) ? T(s[2] * si * dsc[i - nnx + 1]) : T(0);
    if (st == MHM_CELL_OK && !(si > 0.0)) flag[0] = MHM_CELL_SINGULAR_PIVOT;
  }
  __syncthreads();
  if (st == MHM_CELL_OK) st = flag[0];

  // ---- block LDL^T: S_y^-1 for every line y ------------------------------------
  // S_y[a][c] = Adiag_y[a][c] - sum_{b,d} B_y[a][b] S_{y-1}^-1[b][d] B_y[c][d], B_y the
  // (tridiagonal) coupling of line y to line y-1; inverted by Gauss-Jordan without
  // pivoting (SPD), whose pivots are those of the LDL^T of the whole matrix.
  double dmin = 1e300, dmax = 0.0;
  if (st == MHM_CELL_OK) {
    for (int y = 0; y < nny && st == MHM_CELL_OK; ++y) {
      const T* prev = sinv + (size_t)(y - 1) * nb;
      for (int e = tid; e < nb; e += blockDim.x) {
        const int r = e / nnx, c = e - r * nnx;
        const int ir = y * nnx + r, ic = y * nnx + c;
        T v = T(0);
        if (r == c) v = dg[ir];
        else if (c == r - 1) v = dl[ir];
        else if (r == c - 1) v = dl[ic];
        if (y > 0) {
          T acc = T(0);
#pragma unroll
          for (int p = 0; p < 3; ++p) {
            const int b = r - 1 + p;
            if (b < 0 || b >= nnx) continue;
            const T brb = cdn[3 * ir + p];
#pragma unroll
            for (int q = 0; q < 3; ++q) {
              const int d = c - 1 + q;
              if (d < 0 || d >= nnx) continue;
              acc += brb * prev[b * nnx + d] * cdn[3 * ic + q];
            }
          }
          v -= acc;
        }
        gj0[e] = v;
      }
      __syncthreads();
      T* cur = gj0;
      T* nxt = gj1;
      for (int k = 0; k < nnx; ++k) {
        const T d = cur[k * nnx + k];
        if (!(d > T(0))) { st = MHM_CELL_SINGULAR_PIVOT; break; }  // uniform: every thread reads d
        dmin = fmin(dmin, (double)d);
        dmax = fmax(dmax, (double)d);
        const T inv = T(1) / d;
        T* dst = (k == nnx - 1) ? sinv + (size_t)y * nb : nxt;
        for (int e = tid; e < nb; e += blockDim.x) {
          const int r = e / nnx, c = e - r * nnx;
          T v;
          if (r == k) v = (c == k) ? inv : cur[e] * inv;
          else if (c == k) v = -cur[r * nnx + k] * inv;
          else v = cur[e] - cur[r * nnx + k] * inv * cur[k * nnx + c];
          dst[e] = v;
        }
        __syncthreads();
        T* sw = cur; cur = nxt; nxt = sw;
      }
    }
  }
  if (st == MHM_CELL_OK) {
    const double eps = (sizeof(T) == 8) ? 2.220446049250313e-16 : 1.1920928955078125e-07;
    if (dmin <= eps * n * dmax) st = MHM_CELL_RANK_DEFICIENT;
  }
  __syncthreads();

  // ---- right-hand sides, refinement ------------------------------------------
  const int np1 = n + 1;
  const int lane = tid & 31, wid = tid >> 5, nwarps = blockDim.x >> 5;
  // b norms (warp per column, deterministic)
  for (int col = wid; col < w; col += nwarps) {
    double s2 = 0.0;
    for (int i = lane; i < n; i += 32) {
      const double v = rhs_entry(a, cell, col, i, fvec, az);
      s2 += v * v;
    }
    s2 = warp_sum(s2);
    if (lane == 0) { bnorm[col] = sqrt(s2); conv[col] = (s2 == 0.0); }
  }
  for (int idx = tid; idx < w * np1; idx += blockDim.x) {
    const int col = idx / np1, i = idx % np1;
    xg[idx] = 0.0;
    work[idx] = T(rhs_entry(a, cell, col, i, fvec, az));
  }
  __syncthreads();
  int it = 0;
  const int nrw = nnx * w;
  if (st == MHM_CELL_OK) {
    for (it = 0; it < a.max_refine; ++it) {
      // (1) approximate inverse of the augmented operator on every residual column:
      //     mu = sum(v) / zc; y = D Apin^-1 D (v - c mu); x = y + (v_n - c.y) / zc; x_n = mu
      for (int col = wid; col < w; col += nwarps) {
        const T* v = work + (size_t)col * np1;
        double sum = 0.0;
        for (int i = lane; i < n; i += 32) sum += (double)v[i];
        sum = warp_sum(sum);
        if (lane == 0) cmu[col] = sum / zc;
      }
      __syncthreads();
      for (int idx = tid; idx < w * n; idx += blockDim.x) {
        const int col = idx / n, i = idx - col * n;
        T* v = work + (size_t)col * np1 + i;
        *v = T(((double)*v - ctil[i] * cmu[col]) * dsc[i]);
      }
      __syncthreads();
      // block forward: z_y = S_y^-1 (v_y - B_y z_{y-1})
      for (int y = 0; y < nny; ++y) {
        for (int idx = tid; idx < nrw; idx += blockDim.x) {
          const int col = idx / nnx, r = idx - col * nnx;
          const int ir = y * nnx + r;
          const T* v = work + (size_t)col * np1;
          T acc = v[ir];
          if (y > 0) {
#pragma unroll
            for (int p = 0; p < 3; ++p) {
              const int b = r - 1 + p;
              if (b >= 0 && b < nnx) acc -= cdn[3 * ir + p] * v[ir - nnx - r + b];
            }
          }
          tmp[col * nnx + r] = acc;
        }
        __syncthreads();
        const T* S = sinv + (size_t)y * nb;
        for (int idx = tid; idx < nrw; idx += blockDim.x) {
          const int col = idx / nnx, r = idx - col * nnx;
          const T* tc = tmp + col * nnx;
          const T* sr = S + r * nnx;
          T acc0 = T(0), acc1 = T(0);
          int b = 0;
          for (; b + 1 < nnx; b += 2) {
            acc0 += sr[b] * tc[b];
            acc1 += sr[b + 1] * tc[b + 1];
          }
          if (b < nnx) acc0 += sr[b] * tc[b];
          work[(size_t)col * np1 + y * nnx + r] = acc0 + acc1;
        }
        __syncthreads();
      }
      // block backward: x_y = z_y - S_y^-1 B_{y+1}^T x_{y+1}
      for (int y = nny - 2; y >= 0; --y) {
        for (int idx = tid; idx < nrw; idx += blockDim.x) {
          const int col = idx / nnx, r = idx - col * nnx;
          const T* v = work + (size_t)col * np1 + (y + 1) * nnx;
          const int base = 3 * (y + 1) * nnx;
          T acc = T(0);
          // B_{y+1}[q][r] sits in the stencil row of node q = r+1, r, r-1 of line y+1
          if (r + 1 < nnx) acc += cdn[base + 3 * (r + 1) + 0] * v[r + 1];
          acc += cdn[base + 3 * r + 1] * v[r];
          if (r > 0) acc += cdn[base + 3 * (r - 1) + 2] * v[r - 1];
          tmp[col * nnx + r] = acc;
        }
        __syncthreads();
        const T* S = sinv + (size_t)y * nb;
        for (int idx = tid; idx < nrw; idx += blockDim.x) {
          const int col = idx / nnx, r = idx - col * nnx;
          const T* tc = tmp + col * nnx;
          const T* sr = S + r * nnx;
          T acc0 = T(0), acc1 = T(0);
          int b = 0;
          for (; b + 1 < nnx; b += 2) {
            acc0 += sr[b] * tc[b];
            acc1 += sr[b + 1] * tc[b + 1];
          }
          if (b < nnx) acc0 += sr[b] * tc[b];
          work[(size_t)col * np1 + y * nnx + r] -= acc0 + acc1;
        }
        __syncthreads();
      }
      // kernel shift per column
      for (int col = wid; col < w; col += nwarps) {
        const T* v = work + (size_t)col * np1;
        double cyv = 0.0;
        for (int i = lane; i < n; i += 32) cyv = fma(ctil[i], (double)v[i] * dsc[i], cyv);
        cyv = warp_sum(cyv);
        if (lane == 0) cshift[col] = ((double)v[n] - cyv) / zc;
      }
      __syncthreads();
      // (2) x += correction (FP64, global)
      for (int idx = tid; idx < w * np1; idx += blockDim.x) {
        const int col = idx / np1, i = idx - col * np1;
        if (!conv[col]) xg[idx] += (i < n) ? (double)work[idx] * dsc[i] + cshift[col] : cmu[col];
      }
      __syncthreads();
      // (3) residual r = b - K x in FP64, warp per column
      for (int col = wid; col < w; col += nwarps) {
        if (conv[col]) continue;
        const double* x = xg + (size_t)col * np1;
        T* v = work + (size_t)col * np1;
        const double xm = x[n];
        double s2 = 0.0, cr = 0.0;
        for (int i = lane; i < n; i += 32) {
          const double r = rhs_entry(a, cell, col, i, fvec, az) - stencil_apply(a, sten, i, x) -
                           ctil[i] * xm;
          v[i] = T(r);
          s2 += r * r;
          cr = fma(ctil[i], x[i], cr);
        }
        s2 = warp_sum(s2);
        cr = warp_sum(cr);
        if (lane == 0) {
          const double rn = -cr;
          v[n] = T(rn);
          s2 += rn * rn;
          rnorm[col] = sqrt(s2);
        }
      }
      __syncthreads();
      int all = 1;
      for (int col = 0; col < w; ++col) {
        if (!conv[col] && !(rnorm[col] <= a.tol * bnorm[col])) all = 0;
      }
      __syncthreads();
      if (tid < w && !conv[tid] && rnorm[tid] <= a.tol * bnorm[tid]) conv[tid] = 1;
      __syncthreads();
      if (all) { ++it; break; }
    }
    int ok = 1;
    for (int col = 0; col < w; ++col) ok &= conv[col];
    if (!ok) st = MHM_CELL_RESIDUAL;
    for (int col = 0; col < w; ++col)
      if (!isfinite(rnorm[col]) && !conv[col]) st = MHM_CELL_NONFINITE;
  }
  __syncthreads();

  // ---- Schur block and reduced load (contributions.py:40-47) ----------------
  const int t1 = t + 1;
  const int nout = t1 * t1 + t1;
  const double* x0 = xg;                           // R f
  const double* xr = xg + (size_t)(w - 1) * np1;   // R (A 1)
  for (int e = wid; e < nout; e += nwarps) {
    double acc = 0.0;
    if (e < t1 * t1) {
      const int r = e / t1, c = e % t1;
      if (r < t) {
        const Side sd = trace_side(a, r);
        const int len = side_len(a, sd.s);
        for (int k = lane; k < len; k += 32) {
          const int node = side_node(a, sd.s, k);
          const double bv = coupling(a, cell, sd.s, k, sd.q);
          const double v = (c < t) ? xg[(size_t)(1 + c) * np1 + node] : (1.0 - xr[node]);
          acc = fma(bv, v, acc);
        }
        acc = warp_sum(acc);
        if (c == t) acc = -acc;
      } else if (c < t) {
        const Side sd = trace_side(a, c);
        const int len = side_len(a, sd.s);
        double zb = 0.0;
        for (int k = lane; k < len; k += 32) zb += coupling(a, cell, sd.s, k, sd.q);
        double al = 0.0;
        for (int i = lane; i < n; i += 32) al = fma(az[i], xg[(size_t)(1 + c) * np1 + i], al);
        acc = -(warp_sum(zb) - warp_sum(al));
      } else {
        for (int i = lane; i < n; i += 32) acc = fma(az[i], 1.0 - xr[i], acc);
        acc = -warp_sum(acc);
      }
      if (lane == 0) a.blocks[(size_t)cell * t1 * t1 + e] = acc;
    } else {
      const int r = e - t1 * t1;
      if (r < t) {
        const Side sd = trace_side(a, r);
        const int len = side_len(a, sd.s);
        for (int k = lane; k < len; k += 32)
          acc = fma(coupling(a, cell, sd.s, k, sd.q), x0[side_node(a, sd.s, k)], acc);
        acc = warp_sum(acc);
      } else {
        double al = 0.0, fz = 0.0;
        for (int i = lane; i < n; i += 32) {
          al = fma(az[i], x0[i], al);
          fz += fvec[i];
        }
        acc = warp_sum(al) - warp_sum(fz);
      }
      if (lane == 0) a.loads[(size_t)cell * t1 + r] = acc;
    }
  }
  if (tid == 0) {
    a.status[cell] = st;
    a.iters[cell] = it;
    a.corrected[cell] = any_nonzero ? 1 : 0;
  }
}

// Reconstruction u = R f - (R B) lambda_K + (1 - R A 1) c_K and flux -K grad u at
// fine-cell centres (reconstruction.py:130-141, solutions.py:278-324).
__global__ void __launch_bounds__(kThreads) q1_reconstruct_kernel(
    const Q1Args a, const int64_t* cell_dofs, int64_t trace_size, const double* x, double* fields,
    double* flux) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* lam = reinterpret_cast<double*>(smem);
  double* u = lam + a.t;
  const int cell = blockIdx.x, tid = threadIdx.x;
  const int n = a.n, w = a.w, np1 = n + 1;
  const double* xs = a.sol + (size_t)cell * w * np1;
  for (int j = tid; j < a.t; j += blockDim.x) lam[j] = x[cell_dofs[(size_t)cell * a.t + j]];
  __syncthreads();
  const double c = x[trace_size + cell];
  for (int i = tid; i < n; i += blockDim.x) {
    double v = xs[i];
    for (int j = 0; j < a.t; ++j) v = fma(-xs[(size_t)(1 + j) * np1 + i], lam[j], v);
    v = fma(1.0 - xs[(size_t)(w - 1) * np1 + i], c, v);
    u[i] = v;
    fields[(size_t)cell * n + i] = v;
  }
  __syncthreads();
  if (flux == nullptr) return;
  const int cx = cell % a.nx, cy = cell / a.nx;
  const int ne = a.rx * a.ry;
  for (int e = tid; e < ne; e += blockDim.x) {
    const int ex = e % a.rx, ey = e / a.rx;
    const int n0 = ey * a.nnx + ex;
    const double u0 = u[n0], u1 = u[n0 + 1], u2 = u[n0 + a.nnx], u3 = u[n0 + a.nnx + 1];
    const double gx = (-u0 + u1 - u2 + u3) * (0.5 / a.hx);
    const double gy = (-u0 - u1 + u2 + u3) * (0.5 / a.hy);
    const size_t g = (size_t)(cx * a.rx + ex) * a.NYf + (cy * a.ry + ey);
    double kxx, kxy, kyy;
    if (a.kmode == 0) {
      kxx = a.k0; kxy = a.k1; kyy = a.k2;
    } else if (a.kmode == 1) {
      kxx = kyy = a.kappa[g]; kxy = 0.0;
    } else {
      kxx = a.kappa[3 * g]; kxy = a.kappa[3 * g + 1]; kyy = a.kappa[3 * g + 2];
    }
    double* out = flux + ((size_t)cell * ne + e) * 2;
    out[0] = -(kxx * gx + kxy * gy);
    out[1] = -(kxy * gx + kyy * gy);
  }
}

// Gauss-Legendre nodes/weights on [0,1] by Newton iteration on P_m (host).
void gauss01(int m, double* x, double* wts) {
  for (int i = 0; i < m; ++i) {
    double z = cos(M_PI * (i + 0.75) / (m + 0.5));
    for (int iter = 0; iter < 100; ++iter) {
      double p0 = 1.0, p1 = z;
      for (int k = 2; k <= m; ++k) {
        const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      if (m == 1) { p0 = 1.0; p1 = z; }
      const double dp = m * (z * p1 - p0) / (z * z - 1.0);
      const double dz = p1 / dp;
      z -= dz;
      if (fabs(dz) < 1e-16) break;
    }
    double p0 = 1.0, p1 = z;
    for (int k = 2; k <= m; ++k) {
      const double p2 = ((2.0 * k - 1.0) * z * p1 - (k - 1.0) * p0) / k;
      p0 = p1;
      p1 = p2;
    }
    const double dp = m * (z * p1 - p0) / (z * z - 1.0);
    // node in ascending order on [0,1]
    x[m - 1 - i] = (z + 1.0) / 2.0;
    wts[m - 1 - i] = 1.0 / ((1.0 - z * z) * dp * dp);
  }
}

int fill_args(const mhm_q1_problem* p, int precision, Q1Args& a) {
  if (!p || p->macro_nx < 1 || p->macro_ny < 1 || p->rx < 1 || p->ry < 1) return MHM_ERR_ARGUMENT;
  if (!(p->hx > 0) || !(p->hy > 0) || p->tf_h < 1 || p->tf_v < 1) return MHM_ERR_ARGUMENT;
  if (p->kappa_mode < 0 || p->kappa_mode > 2 || p->source_mode < 0 || p->source_mode > 2)
    return MHM_ERR_ARGUMENT;
  if ((p->kappa_mode && !p->kappa) || (p->source_mode && !p->source)) return MHM_ERR_ARGUMENT;
  if (p->source_mode == 2 && (p->quad_order < 1 || p->quad_order > kMaxQuad)) return MHM_ERR_ARGUMENT;
  if (!p->coupling_table || !p->side_sign || !p->side_orient) return MHM_ERR_ARGUMENT;
  a = Q1Args{};
  a.nx = p->macro_nx; a.ny = p->macro_ny; a.rx = p->rx; a.ry = p->ry;
  a.nnx = a.rx + 1; a.nny = a.ry + 1; a.n = a.nnx * a.nny;
  a.tfh = p->tf_h; a.tfv = p->tf_v; a.t = 2 * (a.tfh + a.tfv); a.w = a.t + 2;
  a.kmax = (a.rx > a.ry ? a.rx : a.ry) + 1;
  a.jmax = a.tfh > a.tfv ? a.tfh : a.tfv;
  if (a.w > 32 * (kThreads / 32)) return MHM_ERR_UNSUPPORTED;
  a.NYf = a.ny * a.ry;
  a.hx = p->hx; a.hy = p->hy; a.area = p->hx * p->hy;
  a.table = p->coupling_table; a.sign = p->side_sign; a.orient = p->side_orient;
  a.kmode = p->kappa_mode; a.kappa = p->kappa;
  a.k0 = p->kappa_const[0]; a.k1 = p->kappa_const[1]; a.k2 = p->kappa_const[2];
  a.smode = p->source_mode; a.src = p->source; a.s0 = p->source_const;
  a.qorder = p->quad_order > 0 ? p->quad_order : 1;
  gauss01(a.qorder, a.gpt, a.gwt);
  const size_t tsz = precision == MHM_PRECISION_FP64 ? 8 : 4;
  size_t off = 0;
  const size_t nb = (size_t)a.nnx * a.nnx;
  a.off_sinv = off; off = align16(off + (size_t)a.nny * nb * tsz);
  a.off_gj = off; off = align16(off + 2 * nb * tsz);
  a.off_cpl = off; off = align16(off + (size_t)5 * a.n * tsz);
  a.off_tmp = off; off = align16(off + (size_t)a.nnx * a.w * tsz);
  a.off_sten = off; off = align16(off + (size_t)5 * a.n * 8);
  a.off_vec = off; off = align16(off + (size_t)4 * a.n * 8);
  a.off_work = off;
  const size_t work = (size_t)a.w * (a.n + 1) * tsz;
  const size_t asm_tmp = (size_t)7 * a.rx * a.ry * 8;
  off = align16(off + (work > asm_tmp ? work : asm_tmp));
  a.off_misc = off; off = align16(off + (32 + 4 * (size_t)a.w) * 8 + ((size_t)a.w + 1) * 4);
  a.smem = off;
  return MHM_OK;
}

}  // namespace
}  // namespace mhm

using namespace mhm;

extern "C" int32_t mhm_q1_rhs_width(const mhm_q1_problem* p) {
  if (!p) return 0;
  return 2 * (p->tf_h + p->tf_v) + 2;
}

extern "C" int64_t mhm_q1_condense_smem_bytes(const mhm_q1_problem* p, int32_t precision) {
  Q1Args a;
  if (fill_args(p, precision, a) != MHM_OK) return 0;
  if (a.smem > 227 * 1024) return 0;
  return (int64_t)a.smem;
}

extern "C" int mhm_q1_condense(const mhm_q1_problem* p, int32_t precision, int32_t max_refine,
                               double tol, double* solution, double* blocks, double* loads,
                               uint8_t* corrected, int32_t* cell_status, int32_t* cell_iters,
                               void* stream) {
  if (precision != MHM_PRECISION_FP64 && precision != MHM_PRECISION_MIXED) return MHM_ERR_ARGUMENT;
  Q1Args a;
  int rc = fill_args(p, precision, a);
  if (rc != MHM_OK) return rc;
  if (!solution || !blocks || !loads || !corrected || !cell_status || !cell_iters || max_refine < 1 ||
      !(tol > 0))
    return MHM_ERR_ARGUMENT;
  if (a.smem > 227 * 1024) return MHM_ERR_UNSUPPORTED;
  a.max_refine = max_refine; a.tol = tol;
  a.sol = solution; a.blocks = blocks; a.loads = loads; a.corrected = corrected;
  a.status = cell_status; a.iters = cell_iters;
  const int cells = a.nx * a.ny;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  cudaError_t e;
  if (precision == MHM_PRECISION_FP64) {
    e = cudaFuncSetAttribute(q1_condense_kernel<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)a.smem);
    if (e != cudaSuccess) return MHM_ERR_LAUNCH;
    q1_condense_kernel<double><<<cells, kThreads, a.smem, s>>>(a);
  } else {
    e = cudaFuncSetAttribute(q1_condense_kernel<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)a.smem);
    if (e != cudaSuccess) return MHM_ERR_LAUNCH;
    q1_condense_kernel<float><<<cells, kThreads, a.smem, s>>>(a);
  }
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_q1_reconstruct(const mhm_q1_problem* p, const double* solution,
                                  const int64_t* cell_dofs, int64_t trace_size, const double* x,
                                  double* fields, double* flux, void* stream) {
  Q1Args a;
  int rc = fill_args(p, MHM_PRECISION_FP64, a);
  if (rc != MHM_OK) return rc;
  if (!solution || !cell_dofs || !x || !fields) return MHM_ERR_ARGUMENT;
  a.sol = const_cast<double*>(solution);
  const size_t smem = ((size_t)a.t + a.n) * 8;
  if (smem > 227 * 1024) return MHM_ERR_UNSUPPORTED;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(q1_reconstruct_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  q1_reconstruct_kernel<<<a.nx * a.ny, kThreads, smem, static_cast<cudaStream_t>(stream)>>>(
      a, cell_dofs, trace_size, x, fields, flux);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}
