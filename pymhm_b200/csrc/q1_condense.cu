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

// 7 warps: the 14 right-hand-side columns of P2 traces in two passes, and room for
// two (FP64) or three (binary32 factor) macrocells per SM.
constexpr int kThreads = 224;
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
  // kmode 3/4: pixel field [px][py][comp] whose lines may cut the fine cells; a
  // pre-pass writes the lower triangle of every fine cell's element matrix to cut,
  // entry-major ([entry][gx][gy], entry (r, c), r >= c, at r (r + 1) / 2 + c, stride
  // cut_stride = fine cells), which the node gather reads in place of the tensor
  bool cut_mode;
  int64_t cut_stride;
  double x0, y0;
  double px0, py0, psx, psy;
  int pnx, pny;
  double* cut;
  int smode;
  const double* src;
  double s0;
  int qorder;
  double gpt[kMaxQuad], gwt[kMaxQuad];
  int max_refine;
  // 0: condense; 1: condense and store each cell's line-block inverses in factors;
  // 2: source response only, with the stored factors (columns 0 only, no Schur block);
  // 3: source response only, with a fresh factorization
  int mode;
  void* factors;
  double tol;
  double* sol;
  double* blocks;
  double* loads;
  uint8_t* corrected;
  int32_t* status;
  int32_t* iters;
  // shared-memory carve-up (byte offsets)
  size_t off_sinv, off_gj, off_cpl, off_cb, off_sten, off_vec, off_warp, off_misc, smem;
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

// Pixel columns [first, last] that the interval [lo, lo + h) overlaps, in the
// reference's snapped pixel coordinates (quadrilateral.py:152-170): a coordinate
// within 64 eps * count of an integer is that integer.  Clamped to the field.
__device__ __forceinline__ void pixel_span(double lo, double h, double origin, double spacing, int count,
                                           int& first, int& last) {
  const double tol = 64.0 * 2.220446049250313e-16 * count;
  double u0 = (lo - origin) / spacing, u1 = (lo + h - origin) / spacing;
  const double r0 = rint(u0), r1 = rint(u1);
  if (fabs(u0 - r0) <= tol) u0 = r0;
  if (fabs(u1 - r1) <= tol) u1 = r1;
  first = (int)floor(u0);
  last = (int)ceil(u1) - 1;
  if (first < 0) first = 0;
  if (last > count - 1) last = count - 1;
}

// Reference-coordinate segment of pixel column i inside [lo, lo + h]: midpoint m
// and width w (both in units of h), as rectangle_intersection_quadrature clips it.
__device__ __forceinline__ void pixel_segment(double lo, double h, double origin, double spacing, int i,
                                              double& m, double& w) {
  const double end = lo + h;
  const double plo = fmin(fmax(origin + i * spacing, lo), end);
  const double phi = fmax(fmin(origin + (i + 1) * spacing, end), plo);
  const double a = fmin(fmax((plo - lo) / h, 0.0), 1.0);
  w = fmin((phi - plo) / h, 1.0 - a);
  m = a + 0.5 * w;
}

// Lower triangle of the element matrix of a fine cell cut by pixel lines (kappa_mode
// 3/4, entry (a, c) with a >= c at a (a + 1) / 2 + c): the sum over
// its pixel intersections [a,b] x [c,d] (reference coordinates) of the exact Q1
// integrals with that pixel's constant tensor.  With X_0 = 1 - xi, X_1 = xi,
// slopes s_0 = -1, s_1 = 1, midpoints m and widths w, every product of two linear
// factors integrates exactly as w (f(m) g(m) + f' g' w^2 / 12):
//   K_ac += kxx (hy/hx) s_ax s_cx wx IY(ay,cy) + kyy (hx/hy) s_ay s_cy wy IX(ax,cx)
//         + kxy (s_ax s_cy JX(cx) JY(ay) + s_ay s_cx JX(ax) JY(cy)),
// IX(i,j) = wx (X_i X_j (mx) + s_i s_j wx^2/12), JX(i) = wx X_i(mx), likewise in y.
// This is the reference's per-intersection Gauss sum (exact for these integrands)
// up to rounding (quadrilateral.py:215-234).
__device__ __forceinline__ void cut_element(const Q1Args& a, double ex0, double ey0, double (&km)[10]) {
  const double rxy = a.hy / a.hx, ryx = a.hx / a.hy;
#pragma unroll
  for (int q = 0; q < 10; ++q) km[q] = 0.0;
  int fx, lx, fy, ly;
  pixel_span(ex0, a.hx, a.px0, a.psx, a.pnx, fx, lx);
  pixel_span(ey0, a.hy, a.py0, a.psy, a.pny, fy, ly);
  for (int iy = fy; iy <= ly; ++iy) {
    double my, wy;
    pixel_segment(ey0, a.hy, a.py0, a.psy, iy, my, wy);
    if (!(wy > 0.0)) continue;
    const double Y[2] = {1.0 - my, my};
    for (int ix = fx; ix <= lx; ++ix) {
      double mx, wx;
      pixel_segment(ex0, a.hx, a.px0, a.psx, ix, mx, wx);
      if (!(wx > 0.0)) continue;
      const double X[2] = {1.0 - mx, mx};
      const size_t g = (size_t)ix * a.pny + iy;
      double kxx, kxy, kyy;
      if (a.kmode == 3) {
        kxx = kyy = a.kappa[g]; kxy = 0.0;
      } else {
        kxx = a.kappa[3 * g]; kxy = a.kappa[3 * g + 1]; kyy = a.kappa[3 * g + 2];
      }
      const double cx2 = wx * wx / 12.0, cy2 = wy * wy / 12.0;
#pragma unroll
      for (int A = 0; A < 4; ++A) {
        const int ax = A & 1, ay = A >> 1;
        const double sax = ax ? 1.0 : -1.0, say = ay ? 1.0 : -1.0;
#pragma unroll
        for (int Cc = 0; Cc <= A; ++Cc) {
          const int cx = Cc & 1, cy = Cc >> 1;
          const double scx = cx ? 1.0 : -1.0, scy = cy ? 1.0 : -1.0;
          const double iy2 = wy * (Y[ay] * Y[cy] + say * scy * cy2);
          const double ix2 = wx * (X[ax] * X[cx] + sax * scx * cx2);
          double v = kxx * rxy * (sax * scx) * wx * iy2 + kyy * ryx * (say * scy) * wy * ix2;
          if (kxy != 0.0)
            v += kxy * (sax * scy * (wx * X[cx]) * (wy * Y[ay]) + say * scx * (wx * X[ax]) * (wy * Y[cy]));
          km[A * (A + 1) / 2 + Cc] += v;
        }
      }
    }
  }
}

// Pre-pass of the cut-cell modes: thread per global fine cell g = gx * NYf + gy.
// Pre-pass of the quadrature modes (kappa_mode 5/6, a permeability that varies inside
// the fine cells, given at the Gauss points): thread per global fine cell, the lower
// triangle of sum_q w_q area grad(phi_a) . K_q grad(phi_c), the reference's tensor
// Gauss rule (quadrilateral.py:191-253, _integration.py:43-88), in the cut-cell
// layout.  kappa: [gx][gy][Q*Q + 1][comp], point q = qy Q + qx, the last one the centre.
__global__ void __launch_bounds__(256) quad_element_kernel(const Q1Args a) {
  const int64_t total = (int64_t)a.nx * a.rx * a.NYf;
  const int Q = a.qorder, qq = Q * Q;
  const int comp = a.kmode == 5 ? 1 : 3;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    double km[10];
#pragma unroll
    for (int q = 0; q < 10; ++q) km[q] = 0.0;
    const double* kg = a.kappa + (size_t)g * (qq + 1) * comp;
    for (int qy = 0; qy < Q; ++qy)
      for (int qx = 0; qx < Q; ++qx) {
        const double xi = a.gpt[qx], eta = a.gpt[qy], wq = a.gwt[qx] * a.gwt[qy] * a.area;
        const double* k = kg + (size_t)(qy * Q + qx) * comp;
        const double kxx = k[0], kxy = comp == 3 ? k[1] : 0.0, kyy = comp == 3 ? k[2] : k[0];
        const double X[2] = {1.0 - xi, xi}, Y[2] = {1.0 - eta, eta};
        double gxv[4], gyv[4];
#pragma unroll
        for (int A = 0; A < 4; ++A) {
          const int ax = A & 1, ay = A >> 1;
          gxv[A] = (ax ? 1.0 : -1.0) * Y[ay] / a.hx;
          gyv[A] = X[ax] * (ay ? 1.0 : -1.0) / a.hy;
        }
#pragma unroll
        for (int A = 0; A < 4; ++A)
#pragma unroll
          for (int C = 0; C <= A; ++C) {
            const double kc_x = kxx * gxv[C] + kxy * gyv[C], kc_y = kxy * gxv[C] + kyy * gyv[C];
            km[A * (A + 1) / 2 + C] += wq * (gxv[A] * kc_x + gyv[A] * kc_y);
          }
      }
#pragma unroll
    for (int q = 0; q < 10; ++q) a.cut[q * a.cut_stride + g] = km[q];
  }
}

__global__ void __launch_bounds__(256) cut_element_kernel(const Q1Args a) {
  const int64_t total = (int64_t)a.nx * a.rx * a.NYf;
  for (int64_t g = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; g < total;
       g += (int64_t)gridDim.x * blockDim.x) {
    const int gx = (int)(g / a.NYf), gy = (int)(g - (int64_t)gx * a.NYf);
    double km[10];
    cut_element(a, a.x0 + (double)gx * a.hx, a.y0 + (double)gy * a.hy, km);
    // entry-major: consecutive threads store consecutive fine cells of one entry
#pragma unroll
    for (int q = 0; q < 10; ++q) a.cut[q * a.cut_stride + g] = km[q];
  }
}

// Entry (r, c), r >= c, of an element stiffness: k points at the element's first
// cut-cell entry from the pre-pass (entries cut_stride apart), or at its tensor
// (kxx, kxy, kyy) for the closed form.
__device__ __forceinline__ double elem_entry(const Q1Args& a, bool cut, const double* k, double rxy, double ryx,
                                             int r, int c) {
  if (cut) return __ldg(k + (r * (r + 1) / 2 + c) * a.cut_stride);
  return elem_k(k[0], k[1], k[2], rxy, ryx, r, c);
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

// Entry i of right-hand-side column col: [f | B | A 1]; cb[j][k] holds the coupling
// of trace column j at node k of its side.
__device__ __forceinline__ double rhs_value(const Q1Args& a, int col, int i, const double* fvec,
                                            const double* az, const double* cb) {
  if (col == 0) return fvec[i];
  if (col == a.w - 1) return az[i];
  const int j = col - 1;
  const Side sd = trace_side(a, j);
  const int ix = i % a.nnx, iy = i / a.nnx;
  int k;
  switch (sd.s) {
    case 0: k = (iy == 0) ? ix : -1; break;
    case 1: k = (ix == a.nnx - 1) ? iy : -1; break;
    case 2: k = (iy == a.nny - 1) ? ix : -1; break;
    default: k = (ix == 0) ? iy : -1; break;
  }
  return k < 0 ? 0.0 : cb[j * a.kmax + k];
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

// Reciprocal of a pivot of the unit-diagonal scaled operator (a value in (0, 2]):
// the single-precision reciprocal, refined for binary64 by two Newton steps
// r <- r + r (1 - d r), each doubling the number of correct bits.
__device__ __forceinline__ float pivot_reciprocal(float d) { return __frcp_rn(d); }
__device__ __forceinline__ double pivot_reciprocal(double d) {
  double r = (double)__frcp_rn((float)d);
  r = fma(r, fma(-d, r, 1.0), r);
  r = fma(r, fma(-d, r, 1.0), r);
  return r;
}

// Register-resident line blocks: lane c of a warp holds column c of an NNX x NNX
// block (idle lanes mirror the last column).  Couplings: node (y, a) to line y-1
// sits in cdn[3 (y nnx + a) + (b - a + 1)] for the node (y-1, b).
template <typename T, int NNX>
__device__ __forceinline__ void block_diag(T (&col)[NNX], int c, int y, const T* dg, const T* dl) {
  const int base = y * NNX;
#pragma unroll
  for (int r = 0; r < NNX; ++r)
    col[r] = (r == c) ? dg[base + r] : (c == r - 1) ? dl[base + r] : (r == c - 1) ? dl[base + c] : T(0);
}

// col -= B_y X B_y^T (X: the block above... i.e. of line y-1, held like col).
template <typename T, int NNX>
__device__ __forceinline__ void sub_from_below(T (&col)[NNX], const T (&X)[NNX], int c, int y, const T* cdn) {
  const int base = y * NNX;
  const T bcm = c > 0 ? cdn[3 * (base + c) + 0] : T(0);
  const T bc0 = cdn[3 * (base + c) + 1];
  const T bcp = c < NNX - 1 ? cdn[3 * (base + c) + 2] : T(0);
  T wv[NNX];
#pragma unroll
  for (int b = 0; b < NNX; ++b) {
    const T lft = __shfl_up_sync(0xffffffffu, X[b], 1);
    const T rgt = __shfl_down_sync(0xffffffffu, X[b], 1);
    wv[b] = lft * bcm + X[b] * bc0 + rgt * bcp;
  }
#pragma unroll
  for (int r = 0; r < NNX; ++r) {
    T acc = cdn[3 * (base + r) + 1] * wv[r];
    if (r > 0) acc += cdn[3 * (base + r) + 0] * wv[r - 1];
    if (r < NNX - 1) acc += cdn[3 * (base + r) + 2] * wv[r + 1];
    col[r] -= acc;
  }
}

// col -= B_{y+1}^T X B_{y+1} (X: the block of line y+1, held like col).
template <typename T, int NNX>
__device__ __forceinline__ void sub_from_above(T (&col)[NNX], const T (&X)[NNX], int c, int y, const T* cdn) {
  const int base = (y + 1) * NNX;
  // B[p][q]: node (y+1, p) to node (y, q); lane c needs B[c-1][c], B[c][c], B[c+1][c]
  const T bcm = c > 0 ? cdn[3 * (base + c - 1) + 2] : T(0);
  const T bc0 = cdn[3 * (base + c) + 1];
  const T bcp = c < NNX - 1 ? cdn[3 * (base + c + 1) + 0] : T(0);
  T wv[NNX];
#pragma unroll
  for (int p = 0; p < NNX; ++p) {
    const T lft = __shfl_up_sync(0xffffffffu, X[p], 1);
    const T rgt = __shfl_down_sync(0xffffffffu, X[p], 1);
    wv[p] = lft * bcm + X[p] * bc0 + rgt * bcp;
  }
#pragma unroll
  for (int r = 0; r < NNX; ++r) {
    T acc = cdn[3 * (base + r) + 1] * wv[r];
    if (r > 0) acc += cdn[3 * (base + r - 1) + 2] * wv[r - 1];
    if (r < NNX - 1) acc += cdn[3 * (base + r + 1) + 0] * wv[r + 1];
    col[r] -= acc;
  }
}

// In-place Gauss-Jordan inverse of the register block (SPD, no pivoting); the pivot
// column goes through shared memory pb (one store per entry, broadcast loads).
template <typename T, int NNX>
__device__ __forceinline__ void block_invert(T (&col)[NNX], int c, T* pb, double& dmin, double& dmax, int& bad) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int k = 0; k < NNX; ++k) {
    if (lane == k) {
#pragma unroll
      for (int i = 0; i < NNX; ++i) pb[i] = col[i];
    }
    __syncwarp();
    const T d = pb[k];
    if (!(d > T(0))) bad = 1;
    dmin = fmin(dmin, (double)d);
    dmax = fmax(dmax, (double)d);
    const T inv = pivot_reciprocal(d);
    const T f = col[k] * inv;
#pragma unroll
    for (int i = 0; i < NNX; ++i) {
      const T pk = pb[i];
      if (i == k) col[i] = (c == k) ? inv : f;
      else col[i] = (c == k) ? -pk * inv : col[i] - pk * f;
    }
    __syncwarp();
  }
}

template <typename T, int NNX>
__device__ __forceinline__ void block_store(const T (&col)[NNX], int c, T* dst) {
  if ((threadIdx.x & 31) < NNX) {
#pragma unroll
    for (int r = 0; r < NNX; ++r) dst[r * NNX + c] = col[r];
  }
}

// Twisted block LDL^T of the line-block operator (lines 0..nny-1, middle line
// m = (nny-1)/2): warp 0 eliminates lines 0..m-1 top-down (S_y = A_yy - B_y S_{y-1}^-1
// B_y^T), warp 1 lines nny-1..m+1 bottom-up (T_y = A_yy - B_{y+1}^T T_{y+1}^-1
// B_{y+1}), then warp 0 the middle line M = A_mm - B_m S_{m-1}^-1 B_m^T -
// B_{m+1}^T T_{m+1}^-1 B_{m+1}.  The inverses of all blocks land in sinv (row-major,
// block y at y nnx^2).  Pivot statistics of both warps are merged into stat.
template <typename T, int NNX>
__device__ void factor_twisted(int nny, const T* dg, const T* dl, const T* cdn, T* sinv, T* pb, double* stat) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int c = lane < NNX ? lane : NNX - 1;
  const int m = (nny - 1) / 2;
  constexpr int nb = NNX * NNX;
  double dmin = 1e300, dmax = 0.0;
  int bad = 0;
  T col[NNX], prev[NNX];
  if (wid == 0) {
    for (int y = 0; y < m; ++y) {
      block_diag<T, NNX>(col, c, y, dg, dl);
      if (y > 0) sub_from_below<T, NNX>(col, prev, c, y, cdn);
      block_invert<T, NNX>(col, c, pb, dmin, dmax, bad);
      block_store<T, NNX>(col, c, sinv + (size_t)y * nb);
#pragma unroll
      for (int r = 0; r < NNX; ++r) prev[r] = col[r];
    }
  } else if (wid == 1) {
    for (int y = nny - 1; y > m; --y) {
      block_diag<T, NNX>(col, c, y, dg, dl);
      if (y < nny - 1) sub_from_above<T, NNX>(col, prev, c, y, cdn);
      block_invert<T, NNX>(col, c, pb, dmin, dmax, bad);
      block_store<T, NNX>(col, c, sinv + (size_t)y * nb);
#pragma unroll
      for (int r = 0; r < NNX; ++r) prev[r] = col[r];
    }
    if (lane == 0) {
      stat[0] = dmin;
      stat[1] = dmax;
      stat[2] = bad;
    }
  }
  __syncthreads();
  if (wid == 0) {
    block_diag<T, NNX>(col, c, m, dg, dl);
    if (m > 0) sub_from_below<T, NNX>(col, prev, c, m, cdn);
    if (m + 1 < nny) {
      T up[NNX];
#pragma unroll
      for (int r = 0; r < NNX; ++r) up[r] = sinv[(size_t)(m + 1) * nb + r * NNX + c];
      sub_from_above<T, NNX>(col, up, c, m, cdn);
    }
    block_invert<T, NNX>(col, c, pb, dmin, dmax, bad);
    block_store<T, NNX>(col, c, sinv + (size_t)m * nb);
    if (lane == 0) {
      stat[0] = fmin(dmin, stat[0]);
      stat[1] = fmax(dmax, stat[1]);
      stat[2] = (bad || stat[2] != 0.0) ? 1.0 : 0.0;
    }
  }
  __syncthreads();
}

// The same factorization by the whole block in shared memory (any line length):
// one barrier per Gauss-Jordan pivot, ping-pong buffers gj0 / gj1.
template <typename T>
__device__ void factor_lines_block(int nnx, int nny, const T* dg, const T* dl, const T* cdn, T* sinv, T* gj0,
                                   T* gj1, double& dmin, double& dmax, int& bad) {
  const int nb = nnx * nnx;
  dmin = 1e300;
  dmax = 0.0;
  bad = 0;
  for (int y = 0; y < nny && !bad; ++y) {
    const T* prev = sinv + (size_t)(y - 1) * nb;
    for (int e = threadIdx.x; e < nb; e += blockDim.x) {
      const int r = e / nnx, c = e - r * nnx;
      const int ir = y * nnx + r, ic = y * nnx + c;
      T v = (r == c) ? dg[ir] : (c == r - 1) ? dl[ir] : (r == c - 1) ? dl[ic] : T(0);
      if (y > 0) {
        T acc = T(0);
        for (int p = 0; p < 3; ++p) {
          const int b = r - 1 + p;
          if (b < 0 || b >= nnx) continue;
          const T brb = cdn[3 * ir + p];
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
      if (!(d > T(0))) { bad = 1; break; }  // uniform: every thread reads d
      dmin = fmin(dmin, (double)d);
      dmax = fmax(dmax, (double)d);
      const T inv = T(1) / d;
      T* dst = (k == nnx - 1) ? sinv + (size_t)y * nb : nxt;
      for (int e = threadIdx.x; e < nb; e += blockDim.x) {
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

// Minimum resident CTAs per SM for the factor precision (register budget).
template <typename T>
struct Occupancy {
  static constexpr int value = sizeof(T) == 8 ? 2 : 3;
};

// NNX > 0: the factorization runs in one warp's registers for lines of NNX nodes;
// NNX = 0: any line length, factorization in shared memory by the whole block.
// Local assembly of one macrocell (quadrilateral.py:191-253, cartesian.py:69-83):
// element coefficients kel (3 ne) and loads fel (4 ne), the trace coupling of every
// boundary node cb (t kmax) and its column sums zb (t), and node-wise the lower
// stencil of A sten (5 n), the load f (n) and the constraint c = M 1 (n).  Each
// thread returns its part of max|A|, ||A||_F^2 and max c.
// CUT: the cut-cell modes (kappa_mode 3/4), a compile-time switch so that the
// aligned modes' kernels carry no trace of the cut path.
template <bool CUT>
__device__ __forceinline__ void assemble_cell(const Q1Args& a, int cell, double* kel, double* fel, double* cb,
                                              double* zb, double* sten, double* fvec, double* ctil, double& amax,
                                              double& fro, double& cmax) {
  const int tid = threadIdx.x, n = a.n, t = a.t, nnx = a.nnx;
  const int cx = cell % a.nx, cy = cell / a.nx;
  const int ne = a.rx * a.ry;
  // element coefficients and element loads; boundary coupling table ---------
  for (int e = tid; e < ne; e += blockDim.x) {
    const int ex = e % a.rx, ey = e / a.rx;
    const size_t g = (size_t)(cx * a.rx + ex) * a.NYf + (cy * a.ry + ey);
    if (!CUT) {
      double kxx, kxy, kyy;
      if (a.kmode == 0) {
        kxx = a.k0; kxy = a.k1; kyy = a.k2;
      } else if (a.kmode == 1) {
        kxx = kyy = a.kappa[g]; kxy = 0.0;
      } else {
        kxx = a.kappa[3 * g]; kxy = a.kappa[3 * g + 1]; kyy = a.kappa[3 * g + 2];
      }
      kel[3 * e] = kxx; kel[3 * e + 1] = kxy; kel[3 * e + 2] = kyy;
    }
    double fe[4];
    if (a.smode == 3) {
      fe[0] = fe[1] = fe[2] = fe[3] = 0.0;  // nodal loads are given, see the gather
    } else if (a.smode == 2) {
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
  for (int idx = tid; idx < t * a.kmax; idx += blockDim.x) {
    const int j = idx / a.kmax, k = idx - j * a.kmax;
    const Side sd = trace_side(a, j);
    cb[idx] = k < side_len(a, sd.s) ? coupling(a, cell, sd.s, k, sd.q) : 0.0;
  }
  __syncthreads();
  for (int j = tid; j < t; j += blockDim.x) {
    double acc = 0.0;
    const int len = side_len(a, trace_side(a, j).s);
    for (int k = 0; k < len; ++k) acc += cb[j * a.kmax + k];
    zb[j] = acc;
  }

  // node-wise gather of the lower stencil, load and constraint -------------
  const double rxy = a.hy / a.hx, ryx = a.hx / a.hy;
  amax = fro = cmax = 0.0;
  for (int i = tid; i < n; i += blockDim.x) {
    const int ix = i % nnx, iy = i / nnx;
    double sv[5] = {0, 0, 0, 0, 0};
    double f = 0.0;
    int count = 0;
    // candidate elements: E00 (ix-1,iy-1) local 3; E10 (ix,iy-1) local 2;
    //                     E01 (ix-1,iy) local 1;   E11 (ix,iy) local 0
    const bool l = ix > 0, r = ix < a.rx, d = iy > 0, u = iy < a.ry;
    // global fine cell above-right of the node (element E11); used in cut mode only
    const size_t g11 = (size_t)(cx * a.rx + ix) * a.NYf + (cy * a.ry + iy);
    if (l && d) {
      const int e = (iy - 1) * a.rx + ix - 1;
      const double* k = CUT ? a.cut + (g11 - a.NYf - 1) : kel + 3 * e;
      sv[0] += elem_entry(a, CUT, k, rxy, ryx, 3, 3);
      sv[1] += elem_entry(a, CUT, k, rxy, ryx, 3, 2);
      sv[3] += elem_entry(a, CUT, k, rxy, ryx, 3, 1);
      sv[4] += elem_entry(a, CUT, k, rxy, ryx, 3, 0);
      f += fel[4 * e + 3];
      ++count;
    }
    if (r && d) {
      const int e = (iy - 1) * a.rx + ix;
      const double* k = CUT ? a.cut + (g11 - 1) : kel + 3 * e;
      sv[0] += elem_entry(a, CUT, k, rxy, ryx, 2, 2);
      sv[2] += elem_entry(a, CUT, k, rxy, ryx, 2, 1);
      sv[3] += elem_entry(a, CUT, k, rxy, ryx, 2, 0);
      f += fel[4 * e + 2];
      ++count;
    }
    if (l && u) {
      const int e = iy * a.rx + ix - 1;
      const double* k = CUT ? a.cut + (g11 - a.NYf) : kel + 3 * e;
      sv[0] += elem_entry(a, CUT, k, rxy, ryx, 1, 1);
      sv[1] += elem_entry(a, CUT, k, rxy, ryx, 1, 0);
      f += fel[4 * e + 1];
      ++count;
    }
    if (r && u) {
      const int e = iy * a.rx + ix;
      const double* k = CUT ? a.cut + (g11) : kel + 3 * e;
      sv[0] += elem_entry(a, CUT, k, rxy, ryx, 0, 0);
      f += fel[4 * e + 0];
      ++count;
    }
    for (int q = 0; q < 5; ++q) sten[5 * i + q] = sv[q];
    fvec[i] = a.smode == 3 ? a.src[(size_t)cell * n + i] : f;
    ctil[i] = count * (a.area * 0.25);
    amax = fmax(amax, fabs(sv[0]));
    fro += sv[0] * sv[0];
    for (int q = 1; q < 5; ++q) {
      amax = fmax(amax, fabs(sv[q]));
      fro += 2.0 * sv[q] * sv[q];
    }
    cmax = fmax(cmax, ctil[i]);
  }
  __syncthreads();
}

// One macrocell's local stage (the body of q1_condense_kernel and of its batched
// form): `a` describes the cell's problem, `cell` its index within that problem.
template <typename T, int NNX, bool CUT>
__device__ __forceinline__ void condense_cell(const Q1Args& a, const int cell) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int tid = threadIdx.x;
  const int n = a.n, nnx = NNX > 0 ? NNX : a.nnx, nny = a.nny, w = a.w, t = a.t;
  const int nb = nnx * nnx, np1 = n + 1;
  const int lane = tid & 31, wid = tid >> 5, nwarps = blockDim.x >> 5;
  T* sinv = reinterpret_cast<T*>(smem + a.off_sinv);  // nny blocks of nnx x nnx, row-major
  T* gj0 = reinterpret_cast<T*>(smem + a.off_gj);     // Gauss-Jordan ping-pong (NNX = 0)
  T* gj1 = gj0 + nb;
  T* cdn = reinterpret_cast<T*>(smem + a.off_cpl);    // (n, 3): to (y-1, x-1), (y-1, x), (y-1, x+1)
  T* dg = cdn + 3 * n;                                // (n): scaled diagonal
  T* dl = dg + n;                                     // (n): scaled coupling to (y, x-1)
  double* cb = reinterpret_cast<double*>(smem + a.off_cb);  // (t, kmax) boundary couplings
  double* zb = cb + (size_t)t * a.kmax;                     // (t): sum of each column's couplings
  double* sten = reinterpret_cast<double*>(smem + a.off_sten);
  double* fvec = reinterpret_cast<double*>(smem + a.off_vec);
  double* az = fvec + n;
  double* ctil = az + n;
  double* dsc = ctil + n;
  // per-warp column buffers: x (n+1 doubles) and residual / solve vector (n+1 T)
  const size_t wstride = align16((size_t)np1 * 8) + align16((size_t)np1 * sizeof(T)) + 64 * sizeof(T);
  double* xw = reinterpret_cast<double*>(smem + a.off_warp + wid * wstride);
  T* rw = reinterpret_cast<T*>(smem + a.off_warp + wid * wstride + align16((size_t)np1 * 8));
  T* tb = reinterpret_cast<T*>(smem + a.off_warp + wid * wstride + align16((size_t)np1 * 8) +
                               align16((size_t)np1 * sizeof(T)));  // 2 x 32 T: broadcast buffers
  double* kel = reinterpret_cast<double*>(smem + a.off_warp);  // aliases the warp buffers
  double* fel = kel + 3 * a.rx * a.ry;
  double* red = reinterpret_cast<double*>(smem + a.off_misc);
  double* rnorm = red + 32;
  int* cstat = reinterpret_cast<int*>(rnorm + w);  // per column: 1 converged, 2 non-finite
  int* citer = cstat + w;
  int* flag = citer + w;

  double* xg = a.sol + (size_t)cell * w * np1;

  if (tid == 0) flag[0] = 0;
  double amax, fro, cmax;
  assemble_cell<CUT>(a, cell, kel, fel, cb, zb, sten, fvec, ctil, amax, fro, cmax);
  // retained action A 1 (compensated row sums) and finiteness
  double az2 = 0.0;
  int nonzero = 0, nonfinite = 0;
  for (int i = tid; i < n; i += blockDim.x) {
    const int ix = i % nnx, iy = i / nnx;
    const double* sv = sten + 5 * i;
    double hi = 0.0, lo = 0.0;
    dd_add(hi, lo, sv[0]);
    if (ix > 0) dd_add(hi, lo, sv[1]);
    if (iy > 0 && ix < nnx - 1) dd_add(hi, lo, sv[2]);
    if (iy > 0) dd_add(hi, lo, sv[3]);
    if (iy > 0 && ix > 0) dd_add(hi, lo, sv[4]);
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
    const double* sv = sten + 5 * i;
    dg[i] = T(sv[0] * (i == pin ? 2.0 : 1.0) * si * si);
    dl[i] = ix > 0 ? T(sv[1] * si * dsc[i - 1]) : T(0);
    cdn[3 * i + 0] = (iy > 0 && ix > 0) ? T(sv[4] * si * dsc[i - nnx - 1]) : T(0);
    cdn[3 * i + 1] = iy > 0 ? T(sv[3] * si * dsc[i - nnx]) : T(0);
    cdn[3 * i + 2] = (iy > 0 && ix < nnx - 1) ? T(sv[2] * si * dsc[i - nnx + 1]) : T(0);
    if (st == MHM_CELL_OK && !(si > 0.0)) flag[0] = MHM_CELL_SINGULAR_PIVOT;
  }
  __syncthreads();
  if (st == MHM_CELL_OK) st = flag[0];

  // ---- block LDL^T of the line blocks ------------------------------------------
  if (st == MHM_CELL_OK && a.mode == 2) {
    // the factor of an earlier condensation of the same operator (offline / online)
    const T* src = static_cast<const T*>(a.factors) + (size_t)cell * nny * nb;
    for (int e = tid; e < nny * nb; e += blockDim.x) sinv[e] = src[e];
    __syncthreads();
  } else if (st == MHM_CELL_OK) {
    double dmin, dmax;
    int bad;
    if constexpr (NNX > 0) {
      factor_twisted<T, NNX>(nny, dg, dl, cdn, sinv, tb, red);
      const double eps = (sizeof(T) == 8) ? 2.220446049250313e-16 : 1.1920928955078125e-07;
      dmin = red[0];
      dmax = red[1];
      if (red[2] != 0.0) st = MHM_CELL_SINGULAR_PIVOT;
      else if (dmin <= eps * n * dmax) st = MHM_CELL_RANK_DEFICIENT;
      __syncthreads();
    } else {
      factor_lines_block<T>(nnx, nny, dg, dl, cdn, sinv, gj0, gj1, dmin, dmax, bad);
      const double eps = (sizeof(T) == 8) ? 2.220446049250313e-16 : 1.1920928955078125e-07;
      if (bad) st = MHM_CELL_SINGULAR_PIVOT;
      else if (dmin <= eps * n * dmax) st = MHM_CELL_RANK_DEFICIENT;
      __syncthreads();
    }
    if (a.mode == 1 && st == MHM_CELL_OK) {
      T* dst = static_cast<T*>(a.factors) + (size_t)cell * nny * nb;
      for (int e = tid; e < nny * nb; e += blockDim.x) dst[e] = sinv[e];
    }
  }

  // ---- refinement, one warp per right-hand-side column ---------------------------
  // x += y + (r_n - c.y) / zc, x_n += mu with mu = sum(r) / zc and y = D Apin^-1 D
  // (r - c mu), until ||b - K x|| <= tol ||b|| (columnwise, FP64 residual).
  // middle line of the twisted factorization (plain top-down for the shared-memory one)
  const int mid = NNX > 0 ? (nny - 1) / 2 : nny - 1;
  double fz = 0.0;
  for (int i = lane; i < n; i += 32) fz += fvec[i];
  fz = warp_sum(fz);
  const int t1 = t + 1;
  const int ncol = a.mode >= 2 ? 1 : w;  // a source response refines the source column only
  for (int col = wid; col < ncol; col += nwarps) {
    double s2 = 0.0;
    for (int i = lane; i < n; i += 32) {
      const double bv = rhs_value(a, col, i, fvec, az, cb);
      rw[i] = T(bv);
      xw[i] = 0.0;
      s2 += bv * bv;
    }
    if (lane == 0) { rw[n] = T(0); xw[n] = 0.0; }
    s2 = warp_sum(s2);
    const double bn = sqrt(s2);
    int done = (s2 == 0.0) ? 1 : 0;
    double rn = bn;
    int sweeps = 0;
    __syncwarp();
    while (st == MHM_CELL_OK && !done && sweeps < a.max_refine) {
      double sum = 0.0;
      for (int i = lane; i < n; i += 32) sum += (double)rw[i];
      const double mu = warp_sum(sum) / zc;
      const double rmu = (double)rw[n];
      // Twisted block solve, lane = node of a line; the lines' values are broadcast
      // through tb, neighbouring lines are read back from rw.  Lines 0..m-1 go forward
      // top-down, lines nny-1..m+1 bottom-up (interleaved), line m closes, and the
      // back-substitution runs outward from m.  (m = nny-1: plain top-down.)
      const int la = lane < nnx ? lane : 0;
      const int ntop = mid, nbot = nny - 1 - mid, nstep = ntop > nbot ? ntop : nbot;
      T* tbt = tb;
      T* tbb = tb + 32;
      for (int sidx = 0; sidx < nstep; ++sidx) {
        const bool dt = sidx < ntop, db = sidx < nbot;
        const int yt = sidx, yb = nny - 1 - sidx;
        if (lane < nnx) {
          if (dt) {
            const int i = yt * nnx + la;
            T tv = T(((double)rw[i] - ctil[i] * mu) * dsc[i]);
            if (yt > 0) {
              const T* zp = rw + (yt - 1) * nnx;
              tv -= cdn[3 * i + 1] * zp[la];
              if (la > 0) tv -= cdn[3 * i + 0] * zp[la - 1];
              if (la < nnx - 1) tv -= cdn[3 * i + 2] * zp[la + 1];
            }
            tbt[la] = tv;
          }
          if (db) {
            const int i = yb * nnx + la;
            T tv = T(((double)rw[i] - ctil[i] * mu) * dsc[i]);
            if (yb < nny - 1) {
              const T* zp = rw + (yb + 1) * nnx;
              const int base = 3 * (yb + 1) * nnx;
              tv -= cdn[base + 3 * la + 1] * zp[la];
              if (la + 1 < nnx) tv -= cdn[base + 3 * (la + 1) + 0] * zp[la + 1];
              if (la > 0) tv -= cdn[base + 3 * (la - 1) + 2] * zp[la - 1];
            }
            tbb[la] = tv;
          }
        }
        __syncwarp();
        const T* St = sinv + (size_t)yt * nb + la * nnx;
        const T* Sb = sinv + (size_t)yb * nb + la * nnx;
        T at = T(0), ab = T(0);
#pragma unroll 4
        for (int b = 0; b < nnx; ++b) {
          if (dt) at += St[b] * tbt[b];
          if (db) ab += Sb[b] * tbb[b];
        }
        __syncwarp();
        if (lane < nnx) {
          if (dt) rw[yt * nnx + la] = at;
          if (db) rw[yb * nnx + la] = ab;
        }
        __syncwarp();
      }
      {
        const int i = mid * nnx + la;
        if (lane < nnx) {
          T tv = T(((double)rw[i] - ctil[i] * mu) * dsc[i]);
          if (mid > 0) {
            const T* zp = rw + (mid - 1) * nnx;
            tv -= cdn[3 * i + 1] * zp[la];
            if (la > 0) tv -= cdn[3 * i + 0] * zp[la - 1];
            if (la < nnx - 1) tv -= cdn[3 * i + 2] * zp[la + 1];
          }
          if (mid + 1 < nny) {
            const T* zp = rw + (mid + 1) * nnx;
            const int base = 3 * (mid + 1) * nnx;
            tv -= cdn[base + 3 * la + 1] * zp[la];
            if (la + 1 < nnx) tv -= cdn[base + 3 * (la + 1) + 0] * zp[la + 1];
            if (la > 0) tv -= cdn[base + 3 * (la - 1) + 2] * zp[la - 1];
          }
          tbt[la] = tv;
        }
        __syncwarp();
        const T* Sm = sinv + (size_t)mid * nb + la * nnx;
        T acc = T(0);
#pragma unroll 4
        for (int b = 0; b < nnx; ++b) acc += Sm[b] * tbt[b];
        __syncwarp();
        if (lane < nnx) rw[i] = acc;
        __syncwarp();
      }
      for (int sidx = 0; sidx < nstep; ++sidx) {
        const bool dt = sidx < ntop, db = sidx < nbot;
        const int yt = mid - 1 - sidx, yb = mid + 1 + sidx;
        if (lane < nnx) {
          if (dt) {  // B_{yt+1}^T x_{yt+1}
            const T* xn = rw + (yt + 1) * nnx;
            const int base = 3 * (yt + 1) * nnx;
            T u = cdn[base + 3 * la + 1] * xn[la];
            if (la + 1 < nnx) u += cdn[base + 3 * (la + 1) + 0] * xn[la + 1];
            if (la > 0) u += cdn[base + 3 * (la - 1) + 2] * xn[la - 1];
            tbt[la] = u;
          }
          if (db) {  // B_yb x_{yb-1}
            const T* xp = rw + (yb - 1) * nnx;
            const int i = yb * nnx + la;
            T u = cdn[3 * i + 1] * xp[la];
            if (la > 0) u += cdn[3 * i + 0] * xp[la - 1];
            if (la < nnx - 1) u += cdn[3 * i + 2] * xp[la + 1];
            tbb[la] = u;
          }
        }
        __syncwarp();
        const T* St = sinv + (size_t)(dt ? yt : 0) * nb + la * nnx;
        const T* Sb = sinv + (size_t)(db ? yb : 0) * nb + la * nnx;
        T at = T(0), ab = T(0);
#pragma unroll 4
        for (int b = 0; b < nnx; ++b) {
          if (dt) at += St[b] * tbt[b];
          if (db) ab += Sb[b] * tbb[b];
        }
        __syncwarp();
        if (lane < nnx) {
          if (dt) rw[yt * nnx + la] -= at;
          if (db) rw[yb * nnx + la] -= ab;
        }
        __syncwarp();
      }
      __syncwarp();
      // kernel shift and update
      double cyv = 0.0;
      for (int i = lane; i < n; i += 32) cyv = fma(ctil[i], (double)rw[i] * dsc[i], cyv);
      const double shift = (rmu - warp_sum(cyv)) / zc;
      for (int i = lane; i < n; i += 32) xw[i] += (double)rw[i] * dsc[i] + shift;
      if (lane == 0) xw[n] += mu;
      __syncwarp();
      // FP64 residual of the augmented system
      double r2 = 0.0, cr = 0.0;
      const double xm = xw[n];
      for (int i = lane; i < n; i += 32) {
        const double rv = rhs_value(a, col, i, fvec, az, cb) - stencil_apply(a, sten, i, xw) - ctil[i] * xm;
        rw[i] = T(rv);
        r2 += rv * rv;
        cr = fma(ctil[i], xw[i], cr);
      }
      r2 = warp_sum(r2);
      const double rlast = -warp_sum(cr);
      if (lane == 0) rw[n] = T(rlast);
      rn = sqrt(r2 + rlast * rlast);
      ++sweeps;
      __syncwarp();
      if (rn <= a.tol * bn) done = 1;
      if (!isfinite(rn)) break;
    }
    if (lane == 0) {
      rnorm[col] = rn;
      cstat[col] = done ? 1 : (isfinite(rn) ? 0 : 2);
      citer[col] = sweeps;
    }
    // the column to HBM and its entries of the Schur block / load (contributions.py:40-47)
    for (int i = lane; i < np1; i += 32) xg[(size_t)col * np1 + i] = xw[i];
    double al = 0.0;
    for (int i = lane; i < n; i += 32) {
      const double xv = (col == w - 1) ? 1.0 - xw[i] : xw[i];
      al = fma(az[i], xv, al);
    }
    al = warp_sum(al);
    if (lane < t) {
      const Side sd = trace_side(a, lane);
      const int len = side_len(a, sd.s);
      double acc = 0.0;
      for (int k = 0; k < len; ++k) {
        const double xv = xw[side_node(a, sd.s, k)];
        acc = fma(cb[lane * a.kmax + k], (col == w - 1) ? 1.0 - xv : xv, acc);
      }
      if (col == 0) a.loads[(size_t)cell * t1 + lane] = acc;
      else if (col == w - 1) a.blocks[(size_t)cell * t1 * t1 + lane * t1 + t] = -acc;
      else a.blocks[(size_t)cell * t1 * t1 + lane * t1 + (col - 1)] = acc;
    }
    if (lane == 0) {
      if (col == 0) a.loads[(size_t)cell * t1 + t] = al - fz;
      else if (col == w - 1) a.blocks[(size_t)cell * t1 * t1 + t * t1 + t] = -al;
      else a.blocks[(size_t)cell * t1 * t1 + t * t1 + (col - 1)] = -(zb[col - 1] - al);
    }
    __syncwarp();
  }
  __syncthreads();
  if (tid == 0) {
    int it = 0, ok = 1, nf = 0;
    for (int col = 0; col < ncol; ++col) {
      it = citer[col] > it ? citer[col] : it;
      ok &= (cstat[col] == 1);
      nf |= (cstat[col] == 2);
    }
    if (st == MHM_CELL_OK && !ok) st = nf ? MHM_CELL_NONFINITE : MHM_CELL_RESIDUAL;
    a.status[cell] = st;
    a.iters[cell] = it;
    a.corrected[cell] = any_nonzero ? 1 : 0;
  }
}

template <typename T, int NNX, bool CUT>
__global__ void __launch_bounds__(kThreads, Occupancy<T>::value) q1_condense_kernel(const __grid_constant__ Q1Args a) {
  condense_cell<T, NNX, CUT>(a, blockIdx.x);
}

// Several problems of one shape in one launch: blockIdx.y selects the problem (its
// own permeability, source and output buffers), blockIdx.x the macrocell.
constexpr int kMaxBatch = 16;
struct Q1Batch {
  Q1Args a[kMaxBatch];
};

template <typename T, int NNX>
__global__ void __launch_bounds__(kThreads, Occupancy<T>::value) q1_condense_batch_kernel(
    const __grid_constant__ Q1Batch b) {
  condense_cell<T, NNX, false>(b.a[blockIdx.y], blockIdx.x);
}

// Pixel that holds the centre of global fine cell (gx, gy): points on a pixel line
// (to 4 eps of the coordinate) take the pixel on the positive side, clipped at the
// field's upper edge (materials/cartesian.py:40-72).
__device__ __forceinline__ size_t centre_pixel(const Q1Args& a, int gx, int gy) {
  const double eps = 2.220446049250313e-16;
  double u = ((a.x0 + (double)gx * a.hx + 0.5 * a.hx) - a.px0) / a.psx;
  double v = ((a.y0 + (double)gy * a.hy + 0.5 * a.hy) - a.py0) / a.psy;
  const double ru = rint(u), rv = rint(v);
  if (fabs(u - ru) <= 4.0 * eps * fmax(1.0, fabs(u))) u = ru;
  if (fabs(v - rv) <= 4.0 * eps * fmax(1.0, fabs(v))) v = rv;
  int ix = (int)fmax(u, 0.0), iy = (int)fmax(v, 0.0);
  if (ix > a.pnx - 1) ix = a.pnx - 1;
  if (iy > a.pny - 1) iy = a.pny - 1;
  return (size_t)ix * a.pny + iy;
}

// Flux -K grad u at the fine-cell centres of one macrocell from its nodal values u
// (shared memory), postprocessing/solutions.py:278-324.
__device__ __forceinline__ void cell_flux(const Q1Args& a, int cell, const double* u, double* flux) {
  const int tid = threadIdx.x;
  const int cx = cell % a.nx, cy = cell / a.nx;
  const int ne = a.rx * a.ry;
  for (int e = tid; e < ne; e += blockDim.x) {
    const int ex = e % a.rx, ey = e / a.rx;
    const int n0 = ey * a.nnx + ex;
    const double u0 = u[n0], u1 = u[n0 + 1], u2 = u[n0 + a.nnx], u3 = u[n0 + a.nnx + 1];
    const double gx = (-u0 + u1 - u2 + u3) * (0.5 / a.hx);
    const double gy = (-u0 - u1 + u2 + u3) * (0.5 / a.hy);
    size_t g = (size_t)(cx * a.rx + ex) * a.NYf + (cy * a.ry + ey);
    if (a.kmode >= 5)  // quadrature modes: the value stored after the Gauss points
      g = g * (size_t)(a.qorder * a.qorder + 1) + (size_t)(a.qorder * a.qorder);
    else if (a.cut_mode)
      g = centre_pixel(a, cx * a.rx + ex, cy * a.ry + ey);
    double kxx, kxy, kyy;
    if (a.kmode == 0) {
      kxx = a.k0; kxy = a.k1; kyy = a.k2;
    } else if (a.kmode == 1 || a.kmode == 3 || a.kmode == 5) {
      kxx = kyy = a.kappa[g]; kxy = 0.0;
    } else {
      kxx = a.kappa[3 * g]; kxy = a.kappa[3 * g + 1]; kyy = a.kappa[3 * g + 2];
    }
    double* out = flux + ((size_t)cell * ne + e) * 2;
    out[0] = -(kxx * gx + kxy * gy);
    out[1] = -(kxy * gx + kyy * gy);
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
  cell_flux(a, cell, u, flux);
}

// Flux of given nodal fields (one CTA per macrocell).
__global__ void __launch_bounds__(kThreads) q1_flux_kernel(const Q1Args a, const double* fields, double* flux) {
  extern __shared__ __align__(16) unsigned char smem[];
  double* u = reinterpret_cast<double*>(smem);
  const int cell = blockIdx.x;
  for (int i = threadIdx.x; i < a.n; i += blockDim.x) u[i] = fields[(size_t)cell * a.n + i];
  __syncthreads();
  cell_flux(a, cell, u, flux);
}

// Original (uncondensed) equations of every cell at a hybrid solution
// (refinement.py:718-738): the local defect d = f - B lambda - A u per node, each
// row accumulated in double-double arithmetic as the reference's accurate residual
// does in extended precision (linalg/linear.py:98-126); the cell's weak-trace terms
// B^T u per trace slot, also accumulated in double-double; and per cell the sums
// [d.d, f.f, 1.d].
// x_lo / fields_lo (nullable): low parts of a double-double solution (extended
// refinement storage); their terms enter the same double-double sums.
__global__ void __launch_bounds__(kThreads) q1_defect_kernel(const Q1Args a, const int64_t* cell_dofs,
                                                             const uint8_t* fixed, const double* x,
                                                             const double* x_lo, const double* fields,
                                                             const double* fields_lo, double* defect,
                                                             double* slot_terms, double* partial) {
  extern __shared__ __align__(16) unsigned char smem[];
  const int n = a.n, t = a.t, nnx = a.nnx, ne = a.rx * a.ry, cell = blockIdx.x, tid = threadIdx.x;
  double* kel = reinterpret_cast<double*>(smem);
  double* fel = kel + 3 * ne;
  double* cb = fel + 4 * ne;
  double* zb = cb + (size_t)t * a.kmax;
  double* sten = zb + t;
  double* fvec = sten + 5 * n;
  double* ctil = fvec + n;
  double* u = ctil + n;
  double* lam = u + n;
  double* lamf = lam + t;  // lambda on the fixed trace slots, 0 elsewhere
  double* ulo = lamf + t;  // low parts (zero without them)
  double* lamlo = ulo + n;
  double* red = lamlo + t;
  double amax, fro, cmax;
  if (a.cut_mode)
    assemble_cell<true>(a, cell, kel, fel, cb, zb, sten, fvec, ctil, amax, fro, cmax);
  else
    assemble_cell<false>(a, cell, kel, fel, cb, zb, sten, fvec, ctil, amax, fro, cmax);
  const bool has_lo = x_lo && fields_lo;
  for (int i = tid; i < n; i += blockDim.x) {
    u[i] = fields[(size_t)cell * n + i];
    ulo[i] = has_lo ? fields_lo[(size_t)cell * n + i] : 0.0;
  }
  for (int j = tid; j < t; j += blockDim.x) {
    const int64_t dof = cell_dofs[(size_t)cell * t + j];
    lam[j] = x[dof];
    lamlo[j] = has_lo ? x_lo[dof] : 0.0;
    lamf[j] = (fixed && fixed[dof]) ? x[dof] : 0.0;
  }
  __syncthreads();
  double d2 = 0.0, f2 = 0.0, d1 = 0.0;
  for (int i = tid; i < n; i += blockDim.x) {
    const int ix = i % nnx, iy = i / nnx;
    double hi = fvec[i], lo = 0.0;
    double fb = fvec[i];  // the load less the prescribed traces' coupling (refinement.py:704-709)
    for (int j = 0; j < t; ++j) {
      const double bij = rhs_value(a, 1 + j, i, fvec, nullptr, cb);
      if (bij != 0.0) {
        dd_fma(hi, lo, -bij, lam[j]);
        if (has_lo) dd_fma(hi, lo, -bij, lamlo[j]);
        fb = fma(-bij, lamf[j], fb);
      }
    }
    const double* sv = sten + 5 * i;
    for (int part = 0; part < (has_lo ? 2 : 1); ++part) {
      const double* v = part ? ulo : u;
      dd_fma(hi, lo, -sv[0], v[i]);
      if (ix > 0) dd_fma(hi, lo, -sv[1], v[i - 1]);
      if (iy > 0 && ix < nnx - 1) dd_fma(hi, lo, -sv[2], v[i - nnx + 1]);
      if (iy > 0) dd_fma(hi, lo, -sv[3], v[i - nnx]);
      if (iy > 0 && ix > 0) dd_fma(hi, lo, -sv[4], v[i - nnx - 1]);
      if (ix < nnx - 1) dd_fma(hi, lo, -sten[5 * (i + 1) + 1], v[i + 1]);
      if (iy < a.nny - 1) {
        if (ix > 0) dd_fma(hi, lo, -sten[5 * (i + nnx - 1) + 2], v[i + nnx - 1]);
        dd_fma(hi, lo, -sten[5 * (i + nnx) + 3], v[i + nnx]);
        if (ix < nnx - 1) dd_fma(hi, lo, -sten[5 * (i + nnx + 1) + 4], v[i + nnx + 1]);
      }
    }
    const double d = hi + lo;
    defect[(size_t)cell * n + i] = d;
    d2 = fma(d, d, d2);
    f2 = fma(fb, fb, f2);
    d1 += d;
  }
  for (int j = tid; j < t; j += blockDim.x) {
    const Side sd = trace_side(a, j);
    const int len = side_len(a, sd.s);
    double hi = 0.0, lo = 0.0;
    for (int k = 0; k < len; ++k) dd_fma(hi, lo, cb[j * a.kmax + k], u[side_node(a, sd.s, k)]);
    if (has_lo)
      for (int k = 0; k < len; ++k) dd_fma(hi, lo, cb[j * a.kmax + k], ulo[side_node(a, sd.s, k)]);
    slot_terms[(size_t)cell * t + j] = hi + lo;
  }
  d2 = block_sum(d2, red);
  f2 = block_sum(f2, red);
  d1 = block_sum(d1, red);
  if (tid == 0) {
    partial[3 * (size_t)cell] = d2;
    partial[3 * (size_t)cell + 1] = f2;
    partial[3 * (size_t)cell + 2] = d1;
  }
}

// Weak-trace residual of the original equations (refinement.py:729-731):
// weak_i = boundary_i - sum over the DOF's cells (first, then second) of B^T u.
__global__ void weak_residual_kernel(int64_t trace_size, int t, const int32_t* dof_cells,
                                     const int32_t* dof_slot, const double* slot_terms,
                                     const double* boundary, double* weak) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < trace_size;
       i += (int64_t)gridDim.x * blockDim.x) {
    double hi = boundary ? boundary[i] : 0.0, lo = 0.0;
    for (int k = 0; k < 2; ++k) {
      const int c = dof_cells[2 * i + k];
      if (c >= 0) dd_add(hi, lo, -slot_terms[(size_t)c * t + dof_slot[2 * i + k]]);
    }
    weak[i] = hi + lo;
  }
}

// Norms of a refinement step: out[0] = ||[d; weak]||^2 (original residual),
// out[1] = ||[f; boundary]||^2 (its scale), out[2] = ||[weak; 1.d per cell]||^2
// (reduced residual), out[3] = ||rhs||^2 and out[4] = || |K| |x| ||^2 of the
// assembled system.  Block b of kNormBlocks sums fixed index ranges of the cells,
// trace DOFs and rows into partial[b][5]; refine_norms_final adds the partials in
// block order, so every sum has a fixed order.
constexpr int kNormBlocks = 256;

__device__ __forceinline__ void block_range(int64_t n, int64_t& lo, int64_t& hi) {
  lo = n * blockIdx.x / gridDim.x;
  hi = n * (blockIdx.x + 1) / gridDim.x;
}

__global__ void __launch_bounds__(256) refine_norms_partial(int cells, const double* partial, int64_t trace_size,
                                                            const uint8_t* fixed, const double* weak,
                                                            const double* boundary, int64_t size,
                                                            const int64_t* indptr, const int32_t* indices,
                                                            const double* values, const double* x,
                                                            const double* rhs, double* blocks) {
  __shared__ double red[32];
  double v[5] = {0.0, 0.0, 0.0, 0.0, 0.0};
  int64_t lo, hi;
  block_range(cells, lo, hi);
  for (int64_t c = lo + threadIdx.x; c < hi; c += blockDim.x) {
    v[0] += partial[3 * c];
    v[1] += partial[3 * c + 1];
    v[2] += partial[3 * c + 2] * partial[3 * c + 2];
  }
  block_range(trace_size, lo, hi);
  for (int64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
    if (fixed && fixed[i]) continue;  // the free trace DOFs' weak equations only
    const double w2 = weak[i] * weak[i];
    v[0] += w2;
    v[2] += w2;
    const double b = boundary ? boundary[i] : 0.0;
    v[1] += b * b;
  }
  if (indptr) {
    block_range(size, lo, hi);
    for (int64_t r = lo + threadIdx.x; r < hi; r += blockDim.x) {
      if (fixed && r < trace_size && fixed[r]) continue;  // active rows
      double acc = 0.0;
      for (int64_t e = indptr[r]; e < indptr[r + 1]; ++e) acc = fma(fabs(values[e]), fabs(x[indices[e]]), acc);
      v[4] = fma(acc, acc, v[4]);
      v[3] = fma(rhs[r], rhs[r], v[3]);
    }
  }
  for (int k = 0; k < 5; ++k) {
    const double tot = block_sum(v[k], red);
    if (threadIdx.x == 0) blocks[blockIdx.x * 5 + k] = tot;
  }
}

// Warp k adds the partials of result k (lane-strided, then a fixed shuffle tree).
__global__ void refine_norms_final(int nblocks, const double* blocks, double* out) {
  const int k = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (k >= 5) return;
  double t = 0.0;
  for (int b = lane; b < nblocks; b += 32) t += blocks[b * 5 + k];
  t = warp_sum(t);
  if (lane == 0) out[k] = t;
}

__global__ void accumulate_kernel(int64_t n, double* dst, const double* src) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    dst[i] += src[i];
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
  if (p->kappa_mode < 0 || p->kappa_mode > 6 || p->source_mode < 0 || p->source_mode > 3)
    return MHM_ERR_ARGUMENT;
  if (p->kappa_mode >= 5 && (p->quad_order < 1 || p->quad_order > kMaxQuad || !p->cut_elements))
    return MHM_ERR_ARGUMENT;
  if ((p->kappa_mode == 3 || p->kappa_mode == 4) &&
      (p->pixel_nx < 1 || p->pixel_ny < 1 || !(p->pixel_spacing[0] > 0) || !(p->pixel_spacing[1] > 0) ||
       !std::isfinite(p->pixel_origin[0]) || !std::isfinite(p->pixel_origin[1]) || !p->cut_elements))
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
  if (a.nnx > 32) return MHM_ERR_UNSUPPORTED;  // one lane per node of a line
  a.NYf = a.ny * a.ry;
  a.hx = p->hx; a.hy = p->hy; a.area = p->hx * p->hy;
  a.table = p->coupling_table; a.sign = p->side_sign; a.orient = p->side_orient;
  a.kmode = p->kappa_mode; a.kappa = p->kappa;
  a.k0 = p->kappa_const[0]; a.k1 = p->kappa_const[1]; a.k2 = p->kappa_const[2];
  a.cut_mode = a.kmode >= 3;
  a.x0 = p->x0; a.y0 = p->y0;
  if (a.kmode >= 3) {
    if (a.kmode <= 4) {
      a.px0 = p->pixel_origin[0]; a.py0 = p->pixel_origin[1];
      a.psx = p->pixel_spacing[0]; a.psy = p->pixel_spacing[1];
      a.pnx = p->pixel_nx; a.pny = p->pixel_ny;
    }
    a.cut = p->cut_elements;
    a.cut_stride = (int64_t)a.nx * a.rx * a.NYf;
  }
  a.smode = p->source_mode; a.src = p->source; a.s0 = p->source_const;
  a.qorder = p->quad_order > 0 ? p->quad_order : 1;
  gauss01(a.qorder, a.gpt, a.gwt);
  const size_t tsz = precision == MHM_PRECISION_FP64 ? 8 : 4;
  size_t off = 0;
  const size_t nb = (size_t)a.nnx * a.nnx, np1 = (size_t)a.n + 1;
  a.off_sinv = off; off = align16(off + (size_t)a.nny * nb * tsz);
  const bool reg_factor = a.nnx == 5 || a.nnx == 9 || a.nnx == 17;  // see launch_condense
  a.off_gj = off; off = align16(off + (reg_factor ? 0 : 2 * nb * tsz));
  a.off_cpl = off; off = align16(off + (size_t)5 * a.n * tsz);
  a.off_cb = off; off = align16(off + ((size_t)a.t * a.kmax + a.t) * 8);
  a.off_sten = off; off = align16(off + (size_t)5 * a.n * 8);
  a.off_vec = off; off = align16(off + (size_t)4 * a.n * 8);
  a.off_warp = off;
  const size_t warps = (size_t)(kThreads / 32) * (align16(np1 * 8) + align16(np1 * tsz) + 64 * tsz);
  const size_t asm_tmp = (size_t)7 * a.rx * a.ry * 8;
  off = align16(off + (warps > asm_tmp ? warps : asm_tmp));
  a.off_misc = off; off = align16(off + (32 + (size_t)a.w) * 8 + (2 * (size_t)a.w + 1) * 4);
  a.smem = off;
  return MHM_OK;
}

template <typename T, int NNX, bool CUT>
int launch_variant(const Q1Args& a, int cells, cudaStream_t s) {
  if (cudaFuncSetAttribute(q1_condense_kernel<T, NNX, CUT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)a.smem) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  q1_condense_kernel<T, NNX, CUT><<<cells, kThreads, a.smem, s>>>(a);
  return MHM_OK;
}

template <typename T, int NNX>
int launch_one(const Q1Args& a, int cells, cudaStream_t s) {
  return a.cut_mode ? launch_variant<T, NNX, true>(a, cells, s) : launch_variant<T, NNX, false>(a, cells, s);
}

// Register-resident factorization for the common line lengths (4, 8 and 16 fine
// cells per macrocell side); other lengths use the shared-memory one.
template <typename T>
int launch_condense(const Q1Args& a, int cells, cudaStream_t s) {
  switch (a.nnx) {
    case 5: return launch_one<T, 5>(a, cells, s);
    case 9: return launch_one<T, 9>(a, cells, s);
    case 17: return launch_one<T, 17>(a, cells, s);
    default: return launch_one<T, 0>(a, cells, s);
  }
}

template <typename T, int NNX>
int launch_batch_variant(const Q1Batch& b, int count, int cells, size_t smem, cudaStream_t s) {
  if (cudaFuncSetAttribute(q1_condense_batch_kernel<T, NNX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)smem) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  q1_condense_batch_kernel<T, NNX><<<dim3(cells, count), kThreads, smem, s>>>(b);
  return MHM_OK;
}

template <typename T>
int launch_batch(const Q1Batch& b, int count, int cells, int nnx, size_t smem, cudaStream_t s) {
  switch (nnx) {
    case 5: return launch_batch_variant<T, 5>(b, count, cells, smem, s);
    case 9: return launch_batch_variant<T, 9>(b, count, cells, smem, s);
    case 17: return launch_batch_variant<T, 17>(b, count, cells, smem, s);
    default: return launch_batch_variant<T, 0>(b, count, cells, smem, s);
  }
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

namespace {
// Cut-cell modes: fill the element-matrix buffer before a local kernel reads it.
void launch_cut_elements(const Q1Args& a, cudaStream_t s) {
  if (!a.cut_mode) return;
  const int64_t total = (int64_t)a.nx * a.rx * a.NYf;
  int64_t grid = (total + 255) / 256;
  if (grid > 148 * 16) grid = 148 * 16;
  if (a.kmode >= 5)
    quad_element_kernel<<<(int)grid, 256, 0, s>>>(a);
  else
    cut_element_kernel<<<(int)grid, 256, 0, s>>>(a);
}

int run_condense(const mhm_q1_problem* p, int32_t precision, int32_t max_refine, double tol, double* solution,
                 double* blocks, double* loads, uint8_t* corrected, int32_t* cell_status, int32_t* cell_iters,
                 int mode, void* factors, void* stream) {
  if (precision != MHM_PRECISION_FP64 && precision != MHM_PRECISION_MIXED) return MHM_ERR_ARGUMENT;
  Q1Args a;
  int rc = fill_args(p, precision, a);
  if (rc != MHM_OK) return rc;
  if (!solution || (!blocks && mode < 2) || !loads || !corrected || !cell_status || !cell_iters ||
      max_refine < 1 || !(tol > 0) || ((mode == 1 || mode == 2) && !factors))
    return MHM_ERR_ARGUMENT;
  if (a.smem > 227 * 1024) return MHM_ERR_UNSUPPORTED;
  a.max_refine = max_refine; a.tol = tol;
  a.sol = solution; a.blocks = blocks; a.loads = loads; a.corrected = corrected;
  a.status = cell_status; a.iters = cell_iters;
  a.mode = mode; a.factors = factors;
  const int cells = a.nx * a.ny;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  launch_cut_elements(a, s);
  const int rc2 = precision == MHM_PRECISION_FP64 ? launch_condense<double>(a, cells, s)
                                                  : launch_condense<float>(a, cells, s);
  if (rc2 != MHM_OK) return rc2;
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}
}  // namespace

extern "C" int mhm_q1_condense(const mhm_q1_problem* p, int32_t precision, int32_t max_refine,
                               double tol, double* solution, double* blocks, double* loads,
                               uint8_t* corrected, int32_t* cell_status, int32_t* cell_iters,
                               void* stream) {
  return run_condense(p, precision, max_refine, tol, solution, blocks, loads, corrected, cell_status,
                      cell_iters, 0, nullptr, stream);
}

extern "C" int64_t mhm_q1_factor_bytes(const mhm_q1_problem* p, int32_t precision) {
  if (precision != MHM_PRECISION_FP64 && precision != MHM_PRECISION_MIXED) return -1;
  Q1Args a;
  if (fill_args(p, precision, a) != MHM_OK) return -1;
  const int64_t tsz = precision == MHM_PRECISION_FP64 ? 8 : 4;
  return (int64_t)a.nx * a.ny * a.nny * a.nnx * a.nnx * tsz;
}

extern "C" int mhm_q1_condense_offline(const mhm_q1_problem* p, int32_t precision, int32_t max_refine,
                                       double tol, double* solution, double* blocks, double* loads,
                                       uint8_t* corrected, int32_t* cell_status, int32_t* cell_iters,
                                       void* factors, void* stream) {
  return run_condense(p, precision, max_refine, tol, solution, blocks, loads, corrected, cell_status,
                      cell_iters, 1, factors, stream);
}

extern "C" int mhm_q1_condense_batch(int32_t count, const mhm_q1_problem* problems, int32_t precision,
                                     int32_t max_refine, double tol, double* const* solution, double* const* blocks,
                                     double* const* loads, uint8_t* const* corrected, int32_t* const* cell_status,
                                     int32_t* const* cell_iters, void* const* factors, void* stream) {
  if (count < 1 || count > kMaxBatch || !problems || !solution || !blocks || !loads || !corrected ||
      !cell_status || !cell_iters || max_refine < 1 || !(tol > 0))
    return MHM_ERR_ARGUMENT;
  if (precision != MHM_PRECISION_FP64 && precision != MHM_PRECISION_MIXED) return MHM_ERR_ARGUMENT;
  Q1Batch b;
  for (int k = 0; k < count; ++k) {
    Q1Args& a = b.a[k];
    const int rc = fill_args(&problems[k], precision, a);
    if (rc != MHM_OK) return rc;
    if (!solution[k] || !blocks[k] || !loads[k] || !corrected[k] || !cell_status[k] || !cell_iters[k])
      return MHM_ERR_ARGUMENT;
    // one shape per launch (shared-memory layout and kernel variant), and no
    // permeability pre-pass (pixel fields that cut the fine cells, Gauss-point fields)
    if (a.cut_mode || a.kmode >= 3) return MHM_ERR_UNSUPPORTED;
    const Q1Args& a0 = b.a[0];
    if (a.nx != a0.nx || a.ny != a0.ny || a.rx != a0.rx || a.ry != a0.ry || a.t != a0.t || a.w != a0.w ||
        a.smem != a0.smem)
      return MHM_ERR_ARGUMENT;
    if (a.smem > 227 * 1024) return MHM_ERR_UNSUPPORTED;
    a.max_refine = max_refine;
    a.tol = tol;
    a.sol = solution[k];
    a.blocks = blocks[k];
    a.loads = loads[k];
    a.corrected = corrected[k];
    a.status = cell_status[k];
    a.iters = cell_iters[k];
    a.mode = (factors && factors[k]) ? 1 : 0;
    a.factors = (factors && factors[k]) ? factors[k] : nullptr;
  }
  const int cells = b.a[0].nx * b.a[0].ny;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int rc = precision == MHM_PRECISION_FP64 ? launch_batch<double>(b, count, cells, b.a[0].nnx, b.a[0].smem, s)
                                                 : launch_batch<float>(b, count, cells, b.a[0].nnx, b.a[0].smem, s);
  if (rc != MHM_OK) return rc;
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_q1_source_response(const mhm_q1_problem* p, int32_t precision, int32_t max_refine,
                                      double tol, const void* factors, double* solution, double* loads,
                                      uint8_t* corrected, int32_t* cell_status, int32_t* cell_iters,
                                      void* stream) {
  return run_condense(p, precision, max_refine, tol, solution, nullptr, loads, corrected, cell_status,
                      cell_iters, 2, const_cast<void*>(factors), stream);
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

extern "C" int mhm_q1_correction_response(const mhm_q1_problem* p, int32_t precision, int32_t max_refine,
                                          double tol, const void* factors, double* solution, double* loads,
                                          uint8_t* corrected, int32_t* cell_status, int32_t* cell_iters,
                                          void* stream) {
  return run_condense(p, precision, max_refine, tol, solution, nullptr, loads, corrected, cell_status,
                      cell_iters, factors ? 2 : 3, const_cast<void*>(factors), stream);
}

namespace mhm {
namespace {
int original_defect(const mhm_q1_problem* p, const int64_t* cell_dofs, int64_t trace_size, const int32_t* dof_cells,
                    const int32_t* dof_slot, const uint8_t* fixed, const double* x, const double* x_lo,
                    const double* fields, const double* fields_lo, const double* boundary, double* defect,
                    double* slot_terms, double* weak, double* partial, void* stream) {
  Q1Args a;
  int rc = fill_args(p, MHM_PRECISION_FP64, a);
  if (rc != MHM_OK) return rc;
  if (!cell_dofs || trace_size < 1 || !dof_cells || !dof_slot || !x || !fields || !defect || !slot_terms ||
      !weak || !partial || (!x_lo) != (!fields_lo))
    return MHM_ERR_ARGUMENT;
  const int ne = a.rx * a.ry;
  const size_t smem = ((size_t)7 * ne + (size_t)a.t * a.kmax + a.t + 9 * (size_t)a.n + 3 * a.t + 32) * 8;
  if (smem > 227 * 1024) return MHM_ERR_UNSUPPORTED;
  if (smem > 48 * 1024 &&
      cudaFuncSetAttribute(q1_defect_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
          cudaSuccess)
    return MHM_ERR_LAUNCH;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  launch_cut_elements(a, st);
  q1_defect_kernel<<<a.nx * a.ny, kThreads, smem, st>>>(a, cell_dofs, fixed, x, x_lo, fields, fields_lo, defect,
                                                        slot_terms, partial);
  int blocks = (int)((trace_size + 255) / 256);
  if (blocks > 4096) blocks = 4096;
  weak_residual_kernel<<<blocks, 256, 0, st>>>(trace_size, a.t, dof_cells, dof_slot, slot_terms, boundary, weak);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

// (hi, lo) += src elementwise in double-double (two-sum, then renormalised).
__global__ void accumulate_dd_kernel(int64_t n, double* hi, double* lo, const double* src) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
    double s, e;
    two_sum(hi[i], src[i], s, e);
    e += lo[i];
    double h, l;
    two_sum(s, e, h, l);
    hi[i] = h;
    lo[i] = l;
  }
}
}  // namespace
}  // namespace mhm

extern "C" int mhm_q1_original_defect(const mhm_q1_problem* p, const int64_t* cell_dofs, int64_t trace_size,
                                      const int32_t* dof_cells, const int32_t* dof_slot, const uint8_t* fixed,
                                      const double* x, const double* fields, const double* boundary,
                                      double* defect, double* slot_terms, double* weak, double* partial,
                                      void* stream) {
  return original_defect(p, cell_dofs, trace_size, dof_cells, dof_slot, fixed, x, nullptr, fields, nullptr,
                         boundary, defect, slot_terms, weak, partial, stream);
}

extern "C" int mhm_q1_original_defect_dd(const mhm_q1_problem* p, const int64_t* cell_dofs, int64_t trace_size,
                                         const int32_t* dof_cells, const int32_t* dof_slot, const uint8_t* fixed,
                                         const double* x, const double* x_lo, const double* fields,
                                         const double* fields_lo, const double* boundary, double* defect,
                                         double* slot_terms, double* weak, double* partial, void* stream) {
  if (!x_lo || !fields_lo) return MHM_ERR_ARGUMENT;
  return original_defect(p, cell_dofs, trace_size, dof_cells, dof_slot, fixed, x, x_lo, fields, fields_lo,
                         boundary, defect, slot_terms, weak, partial, stream);
}

extern "C" int mhm_vector_accumulate_dd(int64_t n, double* hi, double* lo, const double* src, void* stream) {
  if (n < 0 || (n > 0 && (!hi || !lo || !src))) return MHM_ERR_ARGUMENT;
  if (n == 0) return MHM_OK;
  int blocks = (int)((n + 255) / 256);
  if (blocks > 4096) blocks = 4096;
  accumulate_dd_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(n, hi, lo, src);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_refine_norms(int32_t cells, const double* partial, int64_t trace_size, const uint8_t* fixed,
                                const double* weak, const double* boundary, int64_t size, const int64_t* indptr,
                                const int32_t* indices, const double* values, const double* x,
                                const double* rhs, double* out, void* stream) {
  if (cells < 1 || !partial || trace_size < 0 || (trace_size > 0 && !weak) || !out) return MHM_ERR_ARGUMENT;
  if (indptr && (size < 1 || !indices || !values || !x || !rhs)) return MHM_ERR_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* blocks = out + 5;
  refine_norms_partial<<<kNormBlocks, 256, 0, st>>>(cells, partial, trace_size, fixed, weak, boundary, size, indptr,
                                                    indices, values, x, rhs, blocks);
  refine_norms_final<<<1, 160, 0, st>>>(kNormBlocks, blocks, out);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_vector_accumulate(int64_t n, double* dst, const double* src, void* stream) {
  if (n < 0 || (n > 0 && (!dst || !src))) return MHM_ERR_ARGUMENT;
  if (n == 0) return MHM_OK;
  int blocks = (int)((n + 255) / 256);
  if (blocks > 4096) blocks = 4096;
  accumulate_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(n, dst, src);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

namespace mhm {
namespace {
// Mean-pressure gauge of a pure-Neumann solve (hybrid_mean_constraint,
// core/system.py:531-566, with the weights C = M 1 of every cell): per cell
// s1 = C . u and s2 = C . (1 - R A1), C_i = area / 4 times the elements at node i.
__global__ void __launch_bounds__(kThreads) gauge_partial_kernel(const Q1Args a, const double* fields,
                                                                 double* partial) {
  __shared__ double red[32];
  const int cell = blockIdx.x, n = a.n, np1 = n + 1;
  const double* ra1 = a.sol + ((size_t)cell * a.w + (a.w - 1)) * np1;
  double s1 = 0.0, s2 = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const int ix = i % a.nnx, iy = i / a.nnx;
    const double c = ((ix == 0 || ix == a.rx) ? 1.0 : 2.0) * ((iy == 0 || iy == a.ry) ? 1.0 : 2.0) * (a.area * 0.25);
    s1 = fma(c, fields[(size_t)cell * n + i], s1);
    s2 = fma(c, 1.0 - ra1[i], s2);
  }
  s1 = block_sum(s1, red);
  s2 = block_sum(s2, red);
  if (threadIdx.x == 0) {
    partial[2 * (size_t)cell] = s1;
    partial[2 * (size_t)cell + 1] = s2;
  }
}

// One block: alpha = (value - sum s1) / sum s2 (fixed-order sums), then every coarse
// unknown += alpha, so that sum_cells C . u = value once the fields are reconstructed.
__global__ void __launch_bounds__(256) gauge_apply_kernel(int cells, const double* partial, double value,
                                                         int64_t trace_size, double* x, double* alpha_out) {
  __shared__ double red[32];
  double s1 = 0.0, s2 = 0.0;
  for (int c = threadIdx.x; c < cells; c += blockDim.x) {
    s1 += partial[2 * (size_t)c];
    s2 += partial[2 * (size_t)c + 1];
  }
  s1 = block_sum(s1, red);
  s2 = block_sum(s2, red);
  const double alpha = (value - s1) / s2;
  if (threadIdx.x == 0) alpha_out[0] = alpha;
  for (int c = threadIdx.x; c < cells; c += blockDim.x) x[trace_size + c] += alpha;
}
}  // namespace
}  // namespace mhm

extern "C" int mhm_q1_mean_gauge(const mhm_q1_problem* p, const double* solution, const double* fields,
                                 double value, int64_t trace_size, double* x, double* partial, void* stream) {
  Q1Args a;
  int rc = fill_args(p, MHM_PRECISION_FP64, a);
  if (rc != MHM_OK) return rc;
  if (!solution || !fields || trace_size < 0 || !x || !partial || !std::isfinite(value)) return MHM_ERR_ARGUMENT;
  a.sol = const_cast<double*>(solution);
  const int cells = a.nx * a.ny;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  gauge_partial_kernel<<<cells, kThreads, 0, st>>>(a, fields, partial);
  gauge_apply_kernel<<<1, 256, 0, st>>>(cells, partial, value, trace_size, x, partial + 2 * (size_t)cells);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_q1_flux(const mhm_q1_problem* p, const double* fields, double* flux, void* stream) {
  Q1Args a;
  int rc = fill_args(p, MHM_PRECISION_FP64, a);
  if (rc != MHM_OK) return rc;
  if (!fields || !flux) return MHM_ERR_ARGUMENT;
  const size_t smem = (size_t)a.n * 8;
  if (smem > 48 * 1024) return MHM_ERR_UNSUPPORTED;
  q1_flux_kernel<<<a.nx * a.ny, kThreads, smem, static_cast<cudaStream_t>(stream)>>>(a, fields, flux);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}
