// Dense batched P1 simplex assembly (triangles and tetrahedra sharing one
// connectivity), the device counterpart of assemble_p1_batch
// (execution/cuda.py:27-105).
//
// Two passes over HBM-resident data.  p1_element_kernel (thread per batch item
// and element) forms the affine geometry, the barycentric gradients and the
// element stiffness vol G K G^T, and flags non-finite points, degenerate
// simplices and invalid coefficients.  p1_row_kernel (thread per batch item and
// node) sums the element blocks of its row in ascending element order, so the
// dense result does not depend on scheduling (the reference scatters with
// atomic adds).  The dense outputs are zeroed by the host first.
#include <cmath>

#include "mhm_common.cuh"

namespace mhm {
namespace {

constexpr int kP1Threads = 256;

struct P1Args {
  int64_t batch;
  int npoints, dim, ncells;
  const double* points;
  const int32_t* cells;
  const double* diffusion;
  int64_t kb, kc;  // tensor strides (in tensors of dim*dim) over batch items / cells
  const double* source;
  int64_t sb, sc;  // value strides over batch items / cells
  const int64_t* node_ptr;
  const int32_t* node_contrib;  // element * (dim + 1) + local node, ascending element
  double* scratch;              // per (batch, element): stiffness (dim+1)^2, volume, volume * source
  double* stiffness;
  double* mass;
  double* load;
  int32_t* status;              // 0 points, 1 degenerate, 2 diffusion, 3 source
};

template <int D>
__device__ void element(const P1Args& a, int64_t b, int e) {
  constexpr int NV = D + 1;
  const double* pts = a.points + (size_t)b * a.npoints * D;
  const int32_t* c = a.cells + (size_t)e * NV;
  double v[NV][D];
  bool finite = true;
#pragma unroll
  for (int k = 0; k < NV; ++k)
#pragma unroll
    for (int d = 0; d < D; ++d) {
      v[k][d] = pts[(size_t)c[k] * D + d];
      finite &= isfinite(v[k][d]);
    }
  if (!finite) atomicOr(a.status + 0, 1);
  // J[r][k] = (v_{k+1} - v_0)_r; bound = product of the column norms
  double J[D][D];
  double bound = 1.0;
#pragma unroll
  for (int k = 0; k < D; ++k) {
    double n2 = 0.0;
#pragma unroll
    for (int r = 0; r < D; ++r) {
      J[r][k] = v[k + 1][r] - v[0][r];
      n2 = fma(J[r][k], J[r][k], n2);
    }
    bound *= sqrt(n2);
  }
  double det, inv[D][D];  // inv = J^-1 by the adjugate
  if constexpr (D == 2) {
    det = J[0][0] * J[1][1] - J[0][1] * J[1][0];
    inv[0][0] = J[1][1] / det; inv[0][1] = -J[0][1] / det;
    inv[1][0] = -J[1][0] / det; inv[1][1] = J[0][0] / det;
  } else {
    const double c00 = J[1][1] * J[2][2] - J[1][2] * J[2][1];
    const double c01 = J[1][2] * J[2][0] - J[1][0] * J[2][2];
    const double c02 = J[1][0] * J[2][1] - J[1][1] * J[2][0];
    det = J[0][0] * c00 + J[0][1] * c01 + J[0][2] * c02;
    inv[0][0] = c00 / det;
    inv[1][0] = c01 / det;
    inv[2][0] = c02 / det;
    inv[0][1] = (J[0][2] * J[2][1] - J[0][1] * J[2][2]) / det;
    inv[1][1] = (J[0][0] * J[2][2] - J[0][2] * J[2][0]) / det;
    inv[2][1] = (J[0][1] * J[2][0] - J[0][0] * J[2][1]) / det;
    inv[0][2] = (J[0][1] * J[1][2] - J[0][2] * J[1][1]) / det;
    inv[1][2] = (J[0][2] * J[1][0] - J[0][0] * J[1][2]) / det;
    inv[2][2] = (J[0][0] * J[1][1] - J[0][1] * J[1][0]) / det;
  }
  if (!(fabs(det) > 2.220446049250313e-16 * bound)) atomicOr(a.status + 1, 1);
  const double vol = fabs(det) / (D == 2 ? 2.0 : 6.0);
  // barycentric gradients: g_0 = -sum of the rows of J^-1, g_{k+1} = row k
  double g[NV][D];
#pragma unroll
  for (int d = 0; d < D; ++d) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < D; ++k) {
      g[k + 1][d] = inv[k][d];
      s += inv[k][d];
    }
    g[0][d] = -s;
  }
  // coefficient: finite, symmetric to 1e-12 relative, positive definite (leading minors)
  const double* K = a.diffusion + ((size_t)b * a.kb + (size_t)e * a.kc) * D * D;
  double T[D][D];
  bool ok = true;
#pragma unroll
  for (int r = 0; r < D; ++r)
#pragma unroll
    for (int s = 0; s < D; ++s) {
      T[r][s] = K[r * D + s];
      ok &= isfinite(T[r][s]);
    }
#pragma unroll
  for (int r = 0; r < D; ++r)
#pragma unroll
    for (int s = 0; s < D; ++s) ok &= fabs(T[r][s] - T[s][r]) <= 1e-12 * fabs(T[s][r]);
  if (ok) {
    // Sylvester's criterion on the lower triangle (what a symmetric eigensolver reads)
    const double m1 = T[0][0];
    const double m2 = T[0][0] * T[1][1] - T[1][0] * T[1][0];
    bool pd = m1 > 0.0 && m2 > 0.0;
    if constexpr (D == 3) {
      const double m3 = T[0][0] * (T[1][1] * T[2][2] - T[2][1] * T[2][1]) -
                        T[1][0] * (T[1][0] * T[2][2] - T[2][1] * T[2][0]) +
                        T[2][0] * (T[1][0] * T[2][1] - T[1][1] * T[2][0]);
      pd = pd && m3 > 0.0;
    }
    ok = pd;
  }
  if (!ok) atomicOr(a.status + 2, 1);
  const double f = a.source[(size_t)b * a.sb + (size_t)e * a.sc];
  if (!isfinite(f)) atomicOr(a.status + 3, 1);
  double* out = a.scratch + ((size_t)b * a.ncells + e) * (NV * NV + 2);
#pragma unroll
  for (int i = 0; i < NV; ++i)
#pragma unroll
    for (int j = 0; j < NV; ++j) {
      double acc = 0.0;
#pragma unroll
      for (int p = 0; p < D; ++p) {
        double tg = 0.0;
#pragma unroll
        for (int q = 0; q < D; ++q) tg = fma(T[p][q], g[j][q], tg);
        acc = fma(g[i][p], tg, acc);
      }
      out[i * NV + j] = vol * acc;
    }
  out[NV * NV] = vol;
  out[NV * NV + 1] = vol * f;
}

__global__ void __launch_bounds__(kP1Threads) p1_element_kernel(const P1Args a) {
  const int64_t total = a.batch * a.ncells;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += stride) {
    const int64_t b = idx / a.ncells;
    const int e = (int)(idx - b * a.ncells);
    if (a.dim == 2) element<2>(a, b, e);
    else element<3>(a, b, e);
  }
  // every point, referenced or not, must be finite
  const int64_t coords = a.batch * a.npoints * a.dim;
  bool finite = true;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < coords; i += stride)
    finite &= isfinite(a.points[i]);
  if (!finite) atomicOr(a.status + 0, 1);
}

// Row i of batch item b: stiffness and mass entries and the load, summed over the
// node's elements in ascending element order (mass = vol (1 + delta_ij) /
// ((d+1)(d+2)), load = vol f / (d+1)).
__global__ void __launch_bounds__(kP1Threads) p1_row_kernel(const P1Args a) {
  const int NV = a.dim + 1;
  const double mdiv = 1.0 / ((double)NV * (NV + 1));
  const int64_t total = a.batch * a.npoints;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < total; idx += stride) {
    const int64_t b = idx / a.npoints;
    const int i = (int)(idx - b * a.npoints);
    double* srow = a.stiffness + ((size_t)b * a.npoints + i) * a.npoints;
    double* mrow = a.mass + ((size_t)b * a.npoints + i) * a.npoints;
    double f = 0.0;
    for (int64_t q = a.node_ptr[i]; q < a.node_ptr[i + 1]; ++q) {
      const int code = a.node_contrib[q];
      const int e = code / NV, li = code - e * NV;
      const double* el = a.scratch + ((size_t)b * a.ncells + e) * (NV * NV + 2);
      const int32_t* c = a.cells + (size_t)e * NV;
      const double vol = el[NV * NV];
      for (int lj = 0; lj < NV; ++lj) {
        const int j = c[lj];
        srow[j] += el[li * NV + lj];
        mrow[j] += vol * ((li == lj ? 2.0 : 1.0) * mdiv);
      }
      f += el[NV * NV + 1] / NV;
    }
    a.load[(size_t)b * a.npoints + i] = f;
  }
}

int grid_for(int64_t work) {
  int64_t g = (work + kP1Threads - 1) / kP1Threads;
  if (g > 148 * 32) g = 148 * 32;
  return g < 1 ? 1 : (int)g;
}

}  // namespace
}  // namespace mhm

using namespace mhm;

extern "C" int mhm_p1_batch_assemble(int64_t batch, int32_t npoints, int32_t dim, const double* points,
                                     int32_t ncells, const int32_t* cells, const double* diffusion,
                                     int64_t diffusion_batch_stride, int64_t diffusion_cell_stride,
                                     const double* source, int64_t source_batch_stride,
                                     int64_t source_cell_stride, const int64_t* node_ptr,
                                     const int32_t* node_contrib, double* scratch, double* stiffness,
                                     double* mass, double* load, int32_t* status, void* stream) {
  if (batch < 1 || npoints < 1 || (dim != 2 && dim != 3) || ncells < 1 || !points || !cells || !diffusion ||
      !source || !node_ptr || !node_contrib || !scratch || !stiffness || !mass || !load || !status ||
      diffusion_batch_stride < 0 || diffusion_cell_stride < 0 || source_batch_stride < 0 ||
      source_cell_stride < 0)
    return MHM_ERR_ARGUMENT;
  P1Args a{batch, npoints, dim, ncells, points, cells, diffusion, diffusion_batch_stride, diffusion_cell_stride,
           source, source_batch_stride, source_cell_stride, node_ptr, node_contrib, scratch, stiffness, mass,
           load, status};
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const size_t dense = (size_t)batch * npoints * npoints * sizeof(double);
  if (cudaMemsetAsync(stiffness, 0, dense, st) != cudaSuccess || cudaMemsetAsync(mass, 0, dense, st) != cudaSuccess ||
      cudaMemsetAsync(status, 0, 4 * sizeof(int32_t), st) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  p1_element_kernel<<<grid_for(batch * ncells), kP1Threads, 0, st>>>(a);
  p1_row_kernel<<<grid_for(batch * npoints), kP1Threads, 0, st>>>(a);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int64_t mhm_p1_batch_scratch_bytes(int64_t batch, int32_t dim, int32_t ncells) {
  if (batch < 1 || (dim != 2 && dim != 3) || ncells < 1) return -1;
  return batch * ncells * ((int64_t)(dim + 1) * (dim + 1) + 2) * (int64_t)sizeof(double);
}
