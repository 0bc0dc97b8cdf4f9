// P2 triangle local operators of polygonal macrocells (config 3), dense per cell, and
// the mixed RT0 / P0 local saddles of the same cells (rt0_element_kernel).
//
// Reference (PyMHM 1.3.2, src/pymhm/): scalar_operators (fem/scalar/triangle.py:
// 208-257) with the Duffy rule triangle_quadrature (fem/scalar/operators.py:63-69),
// the material sampled at the rule's points (material_triangle_quadrature,
// fem/quadrature/material.py:154-199, ordinary coefficients), P2 nodes in the order of
// multiindices (triangle.py:14-24): vertices, then the edges (0,1), (1,2), (2,0).
//
// Two passes, both deterministic:
//   p2_element_kernel  one thread per fine triangle of every cell: the 6 x 6 stiffness
//                      sum_q w_q area kappa(x_q) grad(phi_i).grad(phi_j), mass and load;
//   p2_dense_kernel    one warp per (cell, node): the node's rows of the dense
//                      stiffness and mass and its load, summing its elements in
//                      ascending element order (the reference sums COO duplicates).
// kappa(x) is a union of discs (value `inside`, else `outside`); a point is inside when
// (x - cx)^2 + (y - cy)^2 <= r^2 with each square and the sum rounded separately, and
// the quadrature points are ((b0 p0 + b1 p1) + b2 p2), NumPy's einsum order, so points
// near a disc boundary fall on the same side as in the reference's evaluation.  A
// uniform grid of disc lists (built on the host, conservative) limits the tests.
#include <cstdint>

#include "mhm_common.cuh"

namespace mhm {
namespace {

constexpr int kElemStride = 78;  // 36 stiffness + 36 mass + 6 load

__device__ __forceinline__ double disc_value(double x, double y, int grid, const int32_t* __restrict__ gptr,
                                             const int32_t* __restrict__ glist, const double* __restrict__ centres,
                                             const double* __restrict__ r2, double inside, double outside) {
  if (grid <= 0) return outside;
  const double cx = fmin(fmax(x, 0.0), 1.0), cy = fmin(fmax(y, 0.0), 1.0);
  int gx = (int)(cx * grid), gy = (int)(cy * grid);
  if (gx > grid - 1) gx = grid - 1;
  if (gy > grid - 1) gy = grid - 1;
  const int g = gx * grid + gy;
  for (int k = gptr[g]; k < gptr[g + 1]; ++k) {
    const int d = glist[k];
    const double dx = __dadd_rn(x, -centres[2 * d]);
    const double dy = __dadd_rn(y, -centres[2 * d + 1]);
    if (__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)) <= r2[d]) return inside;
  }
  return outside;
}

__global__ void p2_element_kernel(int64_t elements, const double* __restrict__ points,
                                  const int64_t* __restrict__ tri, int nquad, const double* __restrict__ qbary,
                                  const double* __restrict__ qw, int grid, const int32_t* __restrict__ gptr,
                                  const int32_t* __restrict__ glist, const double* __restrict__ centres,
                                  const double* __restrict__ r2, double inside, double outside, double source,
                                  double* __restrict__ elem) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < elements; e += stride) {
    double p[3][2];
    for (int v = 0; v < 3; ++v) {
      const int64_t id = tri[3 * e + v];
      p[v][0] = points[2 * id];
      p[v][1] = points[2 * id + 1];
    }
    const double j00 = p[1][0] - p[0][0], j01 = p[2][0] - p[0][0];
    const double j10 = p[1][1] - p[0][1], j11 = p[2][1] - p[0][1];
    const double det = j00 * j11 - j01 * j10;
    const double area = 0.5 * fabs(det);
    double gl[3][2];  // barycentric gradients
    gl[1][0] = j11 / det;
    gl[1][1] = -j01 / det;
    gl[2][0] = -j10 / det;
    gl[2][1] = j00 / det;
    gl[0][0] = -gl[1][0] - gl[2][0];
    gl[0][1] = -gl[1][1] - gl[2][1];
    double K[21] = {0}, Mm[21] = {0}, F[6] = {0};
    for (int q = 0; q < nquad; ++q) {
      const double l0 = qbary[3 * q], l1 = qbary[3 * q + 1], l2 = qbary[3 * q + 2];
      double xq[2];
      for (int j = 0; j < 2; ++j)
        xq[j] = __dadd_rn(__dadd_rn(__dmul_rn(l0, p[0][j]), __dmul_rn(l1, p[1][j])), __dmul_rn(l2, p[2][j]));
      const double kap = disc_value(xq[0], xq[1], grid, gptr, glist, centres, r2, inside, outside);
      const double phi[6] = {l0 * (2 * l0 - 1), l1 * (2 * l1 - 1), l2 * (2 * l2 - 1),
                             4 * l0 * l1,       4 * l1 * l2,       4 * l2 * l0};
      // d phi / d lambda_a, then the physical gradients
      const double dl[6][3] = {{4 * l0 - 1, 0, 0}, {0, 4 * l1 - 1, 0}, {0, 0, 4 * l2 - 1},
                               {4 * l1, 4 * l0, 0}, {0, 4 * l2, 4 * l1}, {4 * l2, 0, 4 * l0}};
      double g[6][2];
      for (int i = 0; i < 6; ++i)
        for (int d = 0; d < 2; ++d) g[i][d] = dl[i][0] * gl[0][d] + dl[i][1] * gl[1][d] + dl[i][2] * gl[2][d];
      const double wk = qw[q] * area;
      int k = 0;
      for (int i = 0; i < 6; ++i) {
        for (int j = 0; j <= i; ++j, ++k) {
          K[k] = fma(wk * kap, g[i][0] * g[j][0] + g[i][1] * g[j][1], K[k]);
          Mm[k] = fma(wk, phi[i] * phi[j], Mm[k]);
        }
        F[i] = fma(wk * source, phi[i], F[i]);
      }
    }
    double* out = elem + e * kElemStride;
    int k = 0;
    for (int i = 0; i < 6; ++i)
      for (int j = 0; j <= i; ++j, ++k) {
        out[i * 6 + j] = out[j * 6 + i] = K[k];
        out[36 + i * 6 + j] = out[36 + j * 6 + i] = Mm[k];
      }
    for (int i = 0; i < 6; ++i) out[72 + i] = F[i];
  }
}

// Mixed RT0 / P0 elements (rt0_operators, fem/scalar/operators.py:324-364, and the
// saddle of normal_flux_blocks, fem/hdiv/mixed.py:77-112), one thread per fine
// triangle, written in the P2 element layout so that p2_dense_kernel builds the dense
// rows: local slots (face 0, face 1, face 2, cell pressure, boundary multiplier a,
// boundary multiplier b).  The face basis is sign_s (x - v_(s+2)%3) / (2 area) (the
// triangle's vertices counter-clockwise, face s from vertex s to s + 1); the first 36
// entries hold [[M, -s, S], [-s^T, 0, 0], [S^T, 0, 0]] with
// M_ab = sum_q w_q area kappa(x_q)^-1 phi_a(x_q).phi_b(x_q) and S the 0/1 selector of
// the faces that info[3], info[4] name (-1: a padding slot, all zero); the next 36 the
// pressure mass (the area on the pressure slot) and the last 6 the load, -area sum_q
// w_q f on the pressure slot.  info (elements, 5): the three signs, the two selected
// local faces.
__global__ void rt0_element_kernel(int64_t elements, const double* __restrict__ points,
                                   const int64_t* __restrict__ tri, const int32_t* __restrict__ info, int nquad,
                                   const double* __restrict__ qbary, const double* __restrict__ qw, int grid,
                                   const int32_t* __restrict__ gptr, const int32_t* __restrict__ glist,
                                   const double* __restrict__ centres, const double* __restrict__ r2, double inside,
                                   double outside, double source, double* __restrict__ elem) {
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; e < elements; e += stride) {
    double p[3][2];
    for (int v = 0; v < 3; ++v) {
      const int64_t id = tri[3 * e + v];
      p[v][0] = points[2 * id];
      p[v][1] = points[2 * id + 1];
    }
    const double a0 = p[1][0] - p[0][0], a1 = p[1][1] - p[0][1];
    const double b0 = p[2][0] - p[0][0], b1 = p[2][1] - p[0][1];
    const double area = __dmul_rn(__dadd_rn(__dmul_rn(a0, b1), -__dmul_rn(a1, b0)), 0.5);
    const int32_t* in = info + 5 * e;
    const double sg[3] = {(double)in[0], (double)in[1], (double)in[2]};
    const double inv2a = 1.0 / (2.0 * area);
    double Mf[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};  // (0,0) (1,0) (1,1) (2,0) (2,1) (2,2)
    double fsum = 0.0;
    for (int q = 0; q < nquad; ++q) {
      const double l0 = qbary[3 * q], l1 = qbary[3 * q + 1], l2 = qbary[3 * q + 2];
      double xq[2];
      for (int j = 0; j < 2; ++j)
        xq[j] = __dadd_rn(__dadd_rn(__dmul_rn(l0, p[0][j]), __dmul_rn(l1, p[1][j])), __dmul_rn(l2, p[2][j]));
      const double kap = disc_value(xq[0], xq[1], grid, gptr, glist, centres, r2, inside, outside);
      double phi[3][2];
      for (int f = 0; f < 3; ++f) {
        const int opp = (f + 2) % 3;
        phi[f][0] = sg[f] * (xq[0] - p[opp][0]) * inv2a;
        phi[f][1] = sg[f] * (xq[1] - p[opp][1]) * inv2a;
      }
      const double wk = qw[q] * area / kap;
      int k = 0;
      for (int i = 0; i < 3; ++i)
        for (int j = 0; j <= i; ++j, ++k) Mf[k] = fma(wk, phi[i][0] * phi[j][0] + phi[i][1] * phi[j][1], Mf[k]);
      fsum = fma(source, qw[q], fsum);
    }
    double* out = elem + e * kElemStride;
    for (int k = 0; k < kElemStride; ++k) out[k] = 0.0;
    int k = 0;
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j <= i; ++j, ++k) out[i * 6 + j] = out[j * 6 + i] = Mf[k];
    for (int f = 0; f < 3; ++f) {
      out[f * 6 + 3] = out[3 * 6 + f] = -sg[f];
      for (int m = 0; m < 2; ++m)
        if (in[3 + m] == f) out[f * 6 + 4 + m] = out[(4 + m) * 6 + f] = 1.0;
    }
    out[36 + 3 * 6 + 3] = area;
    out[72 + 3] = -(fsum * area);
  }
}

// Node rows: node g (of all cells) is row node_row[g] of cell node_cell[g], whose dense
// stiffness / mass start at dense_off[cell] with row length ld_of[cell] and whose load
// starts at load_off[cell]; inc[inc_ptr[g] .. inc_ptr[g+1]) lists element * 6 + local
// index in ascending order; elem_dofs (elements, 6) are the cell-local P2 DOFs.
// A warp per node: the two rows are built in shared memory (rows up to kMaxRow; longer
// rows directly in global memory), element by element in ascending order, lanes 0..5
// adding one element's six (distinct) columns, then written out coalesced.
constexpr int kDenseWarps = 8;
constexpr int kMaxRow = 640;

__global__ void __launch_bounds__(kDenseWarps * 32) p2_dense_kernel(
    int64_t nodes, const int32_t* __restrict__ node_cell, const int32_t* __restrict__ node_row,
    const int64_t* __restrict__ inc_ptr, const int64_t* __restrict__ inc, const int32_t* __restrict__ elem_dofs,
    const double* __restrict__ elem, const int64_t* __restrict__ dense_off, const int32_t* __restrict__ ld_of,
    const int64_t* __restrict__ load_off, double* __restrict__ stiffness, double* __restrict__ mass,
    double* __restrict__ load) {
  extern __shared__ double rows_smem[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double* sA = rows_smem + (size_t)wid * 2 * kMaxRow;
  double* sM = sA + kMaxRow;
  const int64_t nwarps = (int64_t)gridDim.x * kDenseWarps;
  for (int64_t g = (int64_t)blockIdx.x * kDenseWarps + wid; g < nodes; g += nwarps) {
    const int c = node_cell[g], i = node_row[g], ld = ld_of[c];
    double* gA = stiffness + dense_off[c] + (int64_t)i * ld;
    double* gM = mass + dense_off[c] + (int64_t)i * ld;
    const bool staged = ld <= kMaxRow;
    double* A = staged ? sA : gA;
    double* Mm = staged ? sM : gM;
    for (int j = lane; j < ld; j += 32) {
      A[j] = 0.0;
      Mm[j] = 0.0;
    }
    __syncwarp();
    double f = 0.0;
    for (int64_t k = inc_ptr[g]; k < inc_ptr[g + 1]; ++k) {
      const int64_t e = inc[k] / 6;
      const int a = (int)(inc[k] - e * 6);
      const double* el = elem + e * kElemStride;
      if (lane < 6) {
        const int j = elem_dofs[6 * e + lane];
        A[j] += el[a * 6 + lane];
        Mm[j] += el[36 + a * 6 + lane];
      }
      f += el[72 + a];
      __syncwarp();
    }
    if (staged)
      for (int j = lane; j < ld; j += 32) {
        gA[j] = sA[j];
        gM[j] = sM[j];
      }
    if (lane == 0) load[load_off[c] + i] = f;
    __syncwarp();
  }
}

int blocks_for(int64_t work) {
  int64_t b = (work + 255) / 256;
  if (b > 65535) b = 65535;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace
}  // namespace mhm

using namespace mhm;

extern "C" int64_t mhm_p2_element_bytes(int64_t elements) {
  return elements < 1 ? -1 : elements * kElemStride * (int64_t)sizeof(double);
}

extern "C" int mhm_p2_assemble(int64_t elements, const double* points, const int64_t* triangles, int32_t nquad,
                               const double* quad_bary, const double* quad_weights, int32_t grid,
                               const int32_t* grid_ptr, const int32_t* grid_discs, const double* centres,
                               const double* radii2, double inside, double outside, double source,
                               double* element_scratch, int64_t nodes, const int32_t* node_cell,
                               const int32_t* node_row, const int64_t* inc_ptr, const int64_t* inc,
                               const int32_t* elem_dofs, const int64_t* dense_off, const int32_t* ld_of,
                               const int64_t* load_off, double* stiffness, double* mass, double* load,
                               void* stream) {
  if (elements < 1 || nodes < 1 || nquad < 1 || grid < 0 || !points || !triangles || !quad_bary ||
      !quad_weights || (grid > 0 && (!grid_ptr || !grid_discs || !centres || !radii2)) || !element_scratch ||
      !node_cell || !node_row || !inc_ptr || !inc || !elem_dofs || !dense_off || !ld_of || !load_off ||
      !stiffness || !mass || !load)
    return MHM_ERR_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  p2_element_kernel<<<blocks_for(elements), 256, 0, st>>>(elements, points, triangles, nquad, quad_bary,
                                                          quad_weights, grid, grid_ptr, grid_discs, centres, radii2,
                                                          inside, outside, source, element_scratch);
  const size_t smem = (size_t)kDenseWarps * 2 * kMaxRow * sizeof(double);
  if (cudaFuncSetAttribute(p2_dense_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  int64_t dblocks = (nodes + kDenseWarps - 1) / kDenseWarps;
  if (dblocks > 148 * 16) dblocks = 148 * 16;
  p2_dense_kernel<<<(unsigned)dblocks, kDenseWarps * 32, smem, st>>>(nodes, node_cell, node_row, inc_ptr, inc,
                                                                     elem_dofs, element_scratch, dense_off, ld_of,
                                                                     load_off, stiffness, mass, load);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

// The two passes of mhm_p2_assemble as separate calls, for callers that assemble the
// node rows in several parts (local matrices too large to hold at once): the element
// pass over every fine triangle once, then the row pass over any contiguous range of
// nodes (pointer offsets into node_cell, node_row and inc_ptr).
extern "C" int mhm_p2_elements(int64_t elements, const double* points, const int64_t* triangles, int32_t nquad,
                               const double* quad_bary, const double* quad_weights, int32_t grid,
                               const int32_t* grid_ptr, const int32_t* grid_discs, const double* centres,
                               const double* radii2, double inside, double outside, double source,
                               double* element_scratch, void* stream) {
  if (elements < 1 || nquad < 1 || grid < 0 || !points || !triangles || !quad_bary || !quad_weights ||
      (grid > 0 && (!grid_ptr || !grid_discs || !centres || !radii2)) || !element_scratch)
    return MHM_ERR_ARGUMENT;
  p2_element_kernel<<<blocks_for(elements), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      elements, points, triangles, nquad, quad_bary, quad_weights, grid, grid_ptr, grid_discs, centres, radii2,
      inside, outside, source, element_scratch);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_p2_assemble_rows(int64_t nodes, const int32_t* node_cell, const int32_t* node_row,
                                    const int64_t* inc_ptr, const int64_t* inc, const int32_t* elem_dofs,
                                    const double* element_scratch, const int64_t* dense_off, const int32_t* ld_of,
                                    const int64_t* load_off, double* stiffness, double* mass, double* load,
                                    void* stream) {
  if (nodes < 1 || !node_cell || !node_row || !inc_ptr || !inc || !elem_dofs || !element_scratch || !dense_off ||
      !ld_of || !load_off || !stiffness || !mass || !load)
    return MHM_ERR_ARGUMENT;
  const size_t smem = (size_t)kDenseWarps * 2 * kMaxRow * sizeof(double);
  if (cudaFuncSetAttribute(p2_dense_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  int64_t dblocks = (nodes + kDenseWarps - 1) / kDenseWarps;
  if (dblocks > 148 * 16) dblocks = 148 * 16;
  p2_dense_kernel<<<(unsigned)dblocks, kDenseWarps * 32, smem, static_cast<cudaStream_t>(stream)>>>(
      nodes, node_cell, node_row, inc_ptr, inc, elem_dofs, element_scratch, dense_off, ld_of, load_off, stiffness,
      mass, load);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_rt0_elements(int64_t elements, const double* points, const int64_t* triangles,
                                const int32_t* info, int32_t nquad, const double* quad_bary,
                                const double* quad_weights, int32_t grid, const int32_t* grid_ptr,
                                const int32_t* grid_discs, const double* centres, const double* radii2, double inside,
                                double outside, double source, double* element_scratch, void* stream) {
  if (elements < 1 || nquad < 1 || grid < 0 || !points || !triangles || !info || !quad_bary || !quad_weights ||
      (grid > 0 && (!grid_ptr || !grid_discs || !centres || !radii2)) || !element_scratch || !(inside > 0) ||
      !(outside > 0))
    return MHM_ERR_ARGUMENT;
  rt0_element_kernel<<<blocks_for(elements), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      elements, points, triangles, info, nquad, quad_bary, quad_weights, grid, grid_ptr, grid_discs, centres, radii2,
      inside, outside, source, element_scratch);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}
