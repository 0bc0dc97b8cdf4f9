// Local stage of macro meshes whose local problems are stored dense (tetrahedra and
// other unstructured local meshes): the material pre-pass of the layered permeability,
// the local contract and augmented systems, the condensation products on the tensor
// cores, and the reconstruction.  The factorization and solves in between are the
// batched equilibrated LU (batched_lu.cu).
//
// Reference (PyMHM 1.3.2, src/pymhm/):
//   material quadrature  fem/scalar/tetrahedron.py:41-52, 157-190 (Duffy rule, points
//                        einsum("qi,tij->tqj", bary, vertices))
//   local contract       core/contracts.py:92-211 (kernel 1, constraint M 1, the
//                        retained and test actions A 1 and A^T 1, corrected flag)
//   augmented system     core/condensation.py:125-174 (scaling min(1, max|A|/max|C|))
//   contributions        core/contributions.py:14-74, core/reconstruction.py:91-127
//   reconstruction       core/reconstruction.py:130-141
#include <cmath>
#include <cstdint>

#include "mhm_common.cuh"

namespace mhm {
namespace {

// ---------------------------------------------------------------------------------
// Material pre-pass: for every (macrocell, fine tetrahedron) the Duffy-rule average
// sum_q w_q kappa(x_q) of a layered voxel field, written as the isotropic tensor the
// P1 assembly reads.  The fine vertices come from the host, computed as the
// reference's submesh computes them; each quadrature point is
// ((b0 p0 + b1 p1) + b2 p2) + b3 p3 with separate roundings, the order NumPy's einsum
// uses, so that points on either side of a voxel face select the same voxel as the
// reference's evaluation.
// ---------------------------------------------------------------------------------
__global__ void tet_kappa_kernel(int64_t cells, const double* __restrict__ points, int npoints, int nfine,
                                 const int32_t* __restrict__ fine_cells, int nquad, const double* __restrict__ qbary,
                                 const double* __restrict__ qw, int layers, int px, int py,
                                 const double* __restrict__ voxels, double* __restrict__ diffusion) {
  const int64_t total = cells * (int64_t)nfine;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < total; id += stride) {
    const int64_t cell = id / nfine;
    const int e = (int)(id - cell * nfine);
    const double* X = points + cell * (int64_t)npoints * 3;
    double p[4][3];
    for (int v = 0; v < 4; ++v)
      for (int j = 0; j < 3; ++j) p[v][j] = X[(int64_t)fine_cells[4 * e + v] * 3 + j];
    double kbar = 0.0;
    for (int q = 0; q < nquad; ++q) {
      const double* b = qbary + 4 * q;
      double x[3];
      for (int j = 0; j < 3; ++j) {
        double acc = __dmul_rn(b[0], p[0][j]);
        acc = __dadd_rn(acc, __dmul_rn(b[1], p[1][j]));
        acc = __dadd_rn(acc, __dmul_rn(b[2], p[2][j]));
        x[j] = __dadd_rn(acc, __dmul_rn(b[3], p[3][j]));
      }
      const double cx = fmin(fmax(x[0], 0.0), 1.0), cy = fmin(fmax(x[1], 0.0), 1.0),
                   cz = fmin(fmax(x[2], 0.0), 1.0);
      long long k = (long long)(cz * layers), i = (long long)(cx * px), j = (long long)(cy * py);
      if (k > layers - 1) k = layers - 1;
      if (i > px - 1) i = px - 1;
      if (j > py - 1) j = py - 1;
      kbar = fma(qw[q], __ldg(voxels + (k * px + i) * py + j), kbar);
    }
    double* D = diffusion + id * 9;
    for (int a = 0; a < 9; ++a) D[a] = (a % 4 == 0) ? kbar : 0.0;
  }
}

// ---------------------------------------------------------------------------------
// Local contract and augmented systems, one CTA per cell.  Cells of one launch share
// the storage strides but may differ in size: cell k has n = n_of[k] unknowns and
// t = t_of[k] trace columns; its stiffness, mass (rows of lds), load (lds) and
// coupling (lds x tld) sit at k times their strides; its augmented matrix is nb x nb
// (nb >= n + 1) and its right-hand sides nb x w (w >= t + 2).  Rows and columns past
// n + 1 are an identity block with zero right-hand sides (solution zero there).  The
// declared kernel Z is the ones vector, or with kvec a 0/1 vector per cell in the
// load's layout (the mixed RT0 problems: zero on the fluxes, one on the cell and
// boundary pressures); the constraint is M Z.
// ---------------------------------------------------------------------------------
constexpr int kDThreads = 256;
constexpr int kTileStride = 33;  // odd: a thread's row of a staged tile spans distinct banks
constexpr size_t kSystemSmem = (size_t)kDThreads * kTileStride * sizeof(double);  // a 32 x 33 tile per warp

// With desc (ragged launches), CTA k builds the system desc[k] describes: order nb =
// desc.n (= lds), w = desc.nrhs columns, its matrices at mat_off (stiffness, mass and
// augmented matrix alike), load at vec_off, actions at 3 vec_off, right-hand sides at
// rhs_off, coupling at cpl_off[k] with tld_of[k] columns, and the cell's sizes, flag
// and status at slot.
template <bool kKernel>
__global__ void __launch_bounds__(kDThreads, 2) dense_system_kernel(
    int lds, int tld, int nb, int w, int normalize, const int32_t* __restrict__ n_of,
    const int32_t* __restrict__ t_of,
    const double* __restrict__ stiffness, const double* __restrict__ mass, const double* __restrict__ load,
    const double* __restrict__ coupling, double* __restrict__ aug, double* __restrict__ rhs,
    double* __restrict__ action, uint8_t* __restrict__ corrected, int32_t* __restrict__ status,
    const mhm_ragged_matrix* __restrict__ desc, const int64_t* __restrict__ cpl_off,
    const int32_t* __restrict__ tld_of, const double* __restrict__ kvec) {
  extern __shared__ __align__(16) double tiles[];
  __shared__ double red[32];
  __shared__ int nonzero;
  int64_t cell = blockIdx.x;
  const int tid = threadIdx.x;
  int64_t moff = cell * (int64_t)lds * lds, koff = cell * (int64_t)nb * nb, roff = cell * (int64_t)nb * w,
          aoff = cell * 3 * (int64_t)nb, loff = cell * (int64_t)lds, coff = cell * (int64_t)lds * tld;
  if (desc) {
    const mhm_ragged_matrix d = desc[blockIdx.x];
    cell = d.slot;
    nb = lds = d.n;
    w = d.nrhs;
    tld = tld_of[blockIdx.x];
    moff = koff = d.mat_off;
    roff = d.rhs_off;
    aoff = 3 * d.vec_off;
    loff = d.vec_off;
    coff = cpl_off[blockIdx.x];
  }
  const int n = n_of[cell], t = t_of[cell];
  const double* A = stiffness + moff;
  const double* Mm = mass + moff;
  double* K = aug + koff;
  double* R = rhs + roff;
  double* act = action + aoff;  // rows: A 1, A^T 1, the constraint
  const double* ldv = load + loff;
  const double* cpl = coupling + coff;
  const double* zk = kKernel ? kvec + loff : nullptr;  // the declared kernel Z (kKernel false: ones)
  if (tid == 0) nonzero = 0;
  // max |A| and ||A||_F^2, the retained action A 1 and the test action A^T 1 (double-double
  // sums, the reference's extended-precision _matrix_action), the plain products A 1
  // that the kernel check reads, and the constraint C = M 1
  double amax = 0.0, fro = 0.0, r2 = 0.0, l2 = 0.0, cmax = 0.0, csum = 0.0, zsum = 0.0;
  __syncthreads();
  // Thread t owns rows t, t + blockDim, ... and walks each row's columns in ascending
  // order (every sum below keeps that order).  Each warp works alone on 32 of those
  // rows at a time (lane l on row r0 + l): per chunk of 32 columns its lanes load the
  // rows' entries into the warp's shared-memory tile (a row per step, coalesced) and
  // the column entries A[j][r0 + l] into registers, all 64 loads in flight at once;
  // then each lane sums its row from the tile and its column from the registers.
  double* tile = tiles + (size_t)(tid >> 5) * 32 * kTileStride;  // this warp's (32, 33)
  const int lane0 = tid & 31;
  for (int r0 = tid - lane0; r0 < n; r0 += blockDim.x) {
    const int i = r0 + lane0;
    double hi = 0.0, lo = 0.0, plain = 0.0, chi = 0.0, clo = 0.0, cplain = 0.0, c = 0.0;
    for (int c0 = 0; c0 < n; c0 += 32) {
      const int jn = min(32, n - c0);
      double colv[32];
#pragma unroll
      for (int q = 0; q < 32; ++q) {
        tile[q * kTileStride + lane0] = (r0 + q < n && c0 + lane0 < n) ? A[(int64_t)(r0 + q) * lds + c0 + lane0] : 0.0;
        colv[q] = (q < jn && i < n) ? A[(int64_t)(c0 + q) * lds + i] : 0.0;
      }
      __syncwarp();
      if (i < n) {
#pragma unroll
        for (int q = 0; q < 32; ++q) {
          if (q < jn) {
            const double a = tile[lane0 * kTileStride + q];
            amax = fmax(amax, fabs(a));
            fro = fma(a, a, fro);
            if (kKernel) {
              const double zq = zk[c0 + q];  // 0 or 1: the products are exact
              dd_add(hi, lo, a * zq);
              plain += a * zq;
              dd_add(chi, clo, colv[q] * zq);
              cplain += colv[q] * zq;
            } else {
              dd_add(hi, lo, a);
              plain += a;
              dd_add(chi, clo, colv[q]);
              cplain += colv[q];
            }
          }
        }
      }
      __syncwarp();
#pragma unroll
      for (int q = 0; q < 32; ++q)
        tile[q * kTileStride + lane0] = (r0 + q < n && c0 + lane0 < n) ? Mm[(int64_t)(r0 + q) * lds + c0 + lane0] : 0.0;
      __syncwarp();
      if (i < n)
        for (int q = 0; q < jn; ++q) {
          const double m = tile[lane0 * kTileStride + q];
          c += kKernel ? m * zk[c0 + q] : m;
        }
      __syncwarp();
    }
    if (i < n) {
      const double ai = hi + lo, ti = chi + clo;
      act[i] = ai;
      act[nb + i] = ti;
      if (ai != 0.0 || ti != 0.0) nonzero = 1;
      r2 = fma(plain, plain, r2);
      l2 = fma(cplain, cplain, l2);
      act[2 * nb + i] = c;
      if (kKernel) {
        csum += zk[i] * c;
        zsum += zk[i] * zk[i];
      } else {
        csum += c;
      }
    }
  }
  amax = block_max(amax, red);
  fro = block_sum(fro, red);
  r2 = block_sum(r2, red);
  l2 = block_sum(l2, red);
  csum = block_sum(csum, red);
  zsum = kKernel ? block_sum(zsum, red) : (double)n;
  // the 2D drivers divide the constraint M Z by Z^T M Z, the cell's area (primal.py:
  // 69-71, 99-100); the 3D driver keeps M 1 (primal_3d.py:58-65)
  const double cdiv = normalize ? csum : 1.0;
  for (int i = tid; i < n; i += blockDim.x) cmax = fmax(cmax, fabs(act[2 * nb + i] / cdiv));
  cmax = block_max(cmax, red);
  __syncthreads();
  const int corr = nonzero;
  // declared kernel: ||A Z|| and ||A^T Z|| <= 1e-10 ||A||_F ||Z|| (both scaled by max|A|)
  int st = MHM_CELL_OK;
  if (amax > 0.0 && (sqrt(r2) > 1e-10 * sqrt(fro) * sqrt(zsum) || sqrt(l2) > 1e-10 * sqrt(fro) * sqrt(zsum)))
    st = MHM_CELL_KERNEL;
  const double scale = (cmax > 0.0) ? fmin(1.0, (amax > 0.0 ? amax : 1.0) / cmax) : 1.0;
  // the augmented matrix and the right-hand sides, a warp per row (no index division)
  const int lane = tid & 31, wid = tid >> 5, nw = blockDim.x >> 5;
  for (int i = wid; i < nb; i += nw) {
    double* Ki = K + (int64_t)i * nb;
    if (i < n) {
      const double* Ai = A + (int64_t)i * lds;
      const double ci = (act[2 * nb + i] / cdiv) * scale;
      for (int j = lane; j < nb; j += 32) Ki[j] = j < n ? Ai[j] : (j == n ? ci : 0.0);
    } else if (i == n) {
      for (int j = lane; j < nb; j += 32) Ki[j] = j < n ? (act[2 * nb + j] / cdiv) * scale : 0.0;
    } else {
      for (int j = lane; j < nb; j += 32) Ki[j] = (i == j) ? 1.0 : 0.0;
    }
    double* Ri = R + (int64_t)i * w;
    for (int col = lane; col < w; col += 32) {
      double v = 0.0;
      if (i < n) {
        if (col == 0) v = ldv[i];
        else if (col <= t) v = cpl[(int64_t)i * tld + (col - 1)];
        else if (col == t + 1) v = corr ? act[i] : 0.0;
      }
      Ri[col] = v;
    }
  }
  if (tid == 0) {
    corrected[cell] = (uint8_t)corr;
    status[cell] = st;
  }
}

// ---------------------------------------------------------------------------------
// Condensation products on the tensor cores.  Per cell one GEMM P = L^T X with
//   L = [B | A^T Z | Z]          (n x (t+2): the t trace columns, the test action, Z)
//   X = [R f | R B | E | Z | f]  (n x (t+4), E = Z - R (A Z))
// (Z the ones vector, or kvec in the load's layout as for the systems)
// in FP64 mma.sync m8n8k4 tiles over a TILE x TILE output (t + 4 <= TILE), one warp
// per 8 x 8 output tile over k-steps of 4 rows, operands staged in shared memory.  Then
//   block[a][b] = P[a][1+b],  block[a][t] = -P[a][t+1]              (B^T lifts, -B^T E)
//   block[t][b] = -(P[b][t+2] - P[t][1+b]),  block[t][t] = -P[t][t+1]
//   load[a] = P[a][0],  load[t] = P[t][0] - P[t+1][t+3]
// (contributions.py:40-47, reconstruction.py:91-127, corrected branch; with A Z = 0
// the test action is zero, E = Z and these are the uncorrected formulas).  The block
// and load of cell k, times sgn (1, or -1 for the mixed problems, whose blocks are
// negative semi-definite), go to blocks + block_off[k] and loads + load_off[k].
// ---------------------------------------------------------------------------------
constexpr int kKChunk = 32;

__device__ __forceinline__ void dmma_8x8x4(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

template <int TILE>
__global__ void __launch_bounds__(TILE * TILE / 2) dense_contrib_kernel(
    int lds, int tld, int nb, int w, const int32_t* __restrict__ n_of, const int32_t* __restrict__ t_of,
    const double* __restrict__ solution, const double* __restrict__ coupling, const double* __restrict__ action,
    const double* __restrict__ load, const int64_t* __restrict__ block_off, const int64_t* __restrict__ load_off,
    double* __restrict__ blocks, double* __restrict__ loads, const double* __restrict__ kvec, double sgn) {
  constexpr int kTilesPerSide = TILE / 8;
  __shared__ double Ls[kKChunk][TILE + 1];  // L rows (k) x columns (m)
  __shared__ double Xs[kKChunk][TILE + 1];  // X rows (k) x columns (n)
  __shared__ double Ps[TILE][TILE + 1];
  const int64_t cell = blockIdx.x;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int n = n_of[cell], t = t_of[cell];
  const double* X = solution + cell * (int64_t)nb * w;
  const double* Bm = coupling + cell * (int64_t)lds * tld;
  const double* tact = action + cell * 3 * (int64_t)nb + nb;
  const double* f = load + cell * (int64_t)lds;
  const double* zk = kvec ? kvec + cell * (int64_t)lds : nullptr;
  const int tm = warp / kTilesPerSide, tn = warp % kTilesPerSide;  // this warp's 8 x 8 output tile
  double d0 = 0.0, d1 = 0.0;
  for (int k0 = 0; k0 < n; k0 += kKChunk) {
    __syncthreads();
    for (int e = tid; e < kKChunk * TILE; e += blockDim.x) {
      const int k = e / TILE, c = e - k * TILE;
      const int i = k0 + k;
      double lv = 0.0, xv = 0.0;
      if (i < n) {
        const double zi = zk ? zk[i] : 1.0;
        if (c < t) lv = Bm[(int64_t)i * tld + c];
        else if (c == t) lv = tact[i];
        else if (c == t + 1) lv = zi;
        const double* xr = X + (int64_t)i * w;
        if (c == 0) xv = xr[0];
        else if (c <= t) xv = xr[c];
        else if (c == t + 1) xv = zi - xr[t + 1];
        else if (c == t + 2) xv = zi;
        else if (c == t + 3) xv = f[i];
      }
      Ls[k][c] = lv;
      Xs[k][c] = xv;
    }
    __syncthreads();
    const int kend = (n - k0 < kKChunk) ? (n - k0) : kKChunk;
    for (int k = 0; k < kend; k += 4) {
      // A fragment (row-major 8 x 4): row = lane / 4, col = lane % 4 -> L^T[m][k] = L[k][m]
      const double a = Ls[k + (lane & 3)][tm * 8 + (lane >> 2)];
      // B fragment (col-major 4 x 8): row = lane % 4, col = lane / 4 -> X[k][n]
      const double b = Xs[k + (lane & 3)][tn * 8 + (lane >> 2)];
      dmma_8x8x4(d0, d1, a, b);
    }
  }
  // C fragment: row = lane / 4, columns 2 (lane % 4) and 2 (lane % 4) + 1
  {
    const int r = tm * 8 + (lane >> 2), c = tn * 8 + 2 * (lane & 3);
    Ps[r][c] = d0;
    Ps[r][c + 1] = d1;
  }
  __syncthreads();
  const int t1 = t + 1;
  double* blk = blocks + block_off[cell];
  double* ld = loads + load_off[cell];
  for (int e = tid; e < t1 * t1; e += blockDim.x) {
    const int a = e / t1, b = e - a * t1;
    double v;
    if (a < t && b < t) v = Ps[a][1 + b];
    else if (a < t) v = -Ps[a][t + 1];
    else if (b < t) v = -(Ps[b][t + 2] - Ps[t][1 + b]);
    else v = -Ps[t][t + 1];
    blk[e] = sgn * v;
  }
  for (int a = tid; a < t1; a += blockDim.x) ld[a] = sgn * ((a < t) ? Ps[a][0] : Ps[t][0] - Ps[t + 1][t + 3]);
}

// u = R f - (R B) lambda_K + E c_K, thread per (cell, node i < tile of rows); fields of
// cell k at fields + field_off[k], its trace DOFs at cell_dofs + dof_off[k], its coarse
// unknown x[trace_size + cell_id[k]]; E = Z - R (A Z), Z the ones vector or kfield in
// the fields' layout.
__global__ void dense_reconstruct_kernel(int64_t cells, int nb, int w, const int32_t* __restrict__ n_of,
                                         const int32_t* __restrict__ t_of, const double* __restrict__ solution,
                                         const int64_t* __restrict__ cell_dofs, const int64_t* __restrict__ dof_off,
                                         const int32_t* __restrict__ cell_id, int64_t trace_size,
                                         const double* __restrict__ x, const int64_t* __restrict__ field_off,
                                         double* __restrict__ fields, const double* __restrict__ kfield) {
  const int64_t total = cells * (int64_t)nb;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t id = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; id < total; id += stride) {
    const int64_t cell = id / nb;
    const int i = (int)(id - cell * nb);
    const int n = n_of[cell], t = t_of[cell];
    if (i >= n) continue;
    const double* xr = solution + (cell * nb + i) * w;
    const int64_t* dofs = cell_dofs + dof_off[cell];
    double u = xr[0];
    for (int b = 0; b < t; ++b) u = fma(-xr[1 + b], x[dofs[b]], u);
    const double zi = kfield ? kfield[field_off[cell] + i] : 1.0;
    u = fma(zi - xr[t + 1], x[trace_size + cell_id[cell]], u);
    fields[field_off[cell] + i] = u;
  }
}

int grid_for(int64_t work) {
  int64_t b = (work + 255) / 256;
  if (b > 65535) b = 65535;
  return (int)(b < 1 ? 1 : b);
}

}  // namespace
}  // namespace mhm

using namespace mhm;

extern "C" int mhm_tet_kappa(int64_t cells, const double* points, int32_t npoints, int32_t nfine,
                             const int32_t* fine_cells, int32_t nquad, const double* quad_bary,
                             const double* quad_weights, int32_t layers, int32_t px, int32_t py,
                             const double* voxels, double* diffusion, void* stream) {
  if (cells < 1 || npoints < 4 || nfine < 1 || nquad < 1 || layers < 1 || px < 1 || py < 1 || !points ||
      !fine_cells || !quad_bary || !quad_weights || !voxels || !diffusion)
    return MHM_ERR_ARGUMENT;
  tet_kappa_kernel<<<grid_for(cells * nfine), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      cells, points, npoints, nfine, fine_cells, nquad, quad_bary, quad_weights, layers, px, py, voxels, diffusion);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

namespace {
int launch_systems(int64_t count, int32_t lds, int32_t tld, int32_t nb, int32_t w, int32_t normalize,
                   const int32_t* n_of, const int32_t* t_of, const double* stiffness, const double* mass,
                   const double* load, const double* coupling, const double* kvec, double* aug, double* rhs,
                   double* action, uint8_t* corrected, int32_t* status, void* stream) {
  if (count < 1 || count > INT32_MAX || lds < 1 || tld < 1 || nb < 2 || nb > lds + 64 || w < 3 || !n_of ||
      !t_of || !stiffness || !mass || !load || !coupling || !aug || !rhs || !action || !corrected || !status)
    return MHM_ERR_ARGUMENT;
  auto kernel = kvec ? dense_system_kernel<true> : dense_system_kernel<false>;
  if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSystemSmem) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  kernel<<<(unsigned)count, kDThreads, kSystemSmem, static_cast<cudaStream_t>(stream)>>>(
      lds, tld, nb, w, normalize, n_of, t_of, stiffness, mass, load, coupling, aug, rhs, action, corrected,
      status, nullptr, nullptr, nullptr, kvec);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

int launch_contributions(int64_t count, int32_t lds, int32_t tld, int32_t nb, int32_t w, int32_t max_t,
                         const int32_t* n_of, const int32_t* t_of, const double* solution, const double* coupling,
                         const double* action, const double* load, const double* kvec, double sgn,
                         const int64_t* block_off, const int64_t* load_off, double* blocks, double* loads,
                         void* stream) {
  if (count < 1 || count > INT32_MAX || lds < 1 || tld < 1 || nb < 2 || w < 3 || max_t < 1 || max_t > 28 ||
      !n_of || !t_of || !solution || !coupling || !action || !load || !block_off || !load_off || !blocks ||
      !loads)
    return MHM_ERR_ARGUMENT;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (max_t + 4 <= 16)
    dense_contrib_kernel<16><<<(unsigned)count, 128, 0, st>>>(lds, tld, nb, w, n_of, t_of, solution, coupling,
                                                               action, load, block_off, load_off, blocks, loads,
                                                               kvec, sgn);
  else
    dense_contrib_kernel<32><<<(unsigned)count, 512, 0, st>>>(lds, tld, nb, w, n_of, t_of, solution, coupling,
                                                               action, load, block_off, load_off, blocks, loads,
                                                               kvec, sgn);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

int launch_reconstruct(int64_t count, int32_t nb, int32_t w, const int32_t* n_of, const int32_t* t_of,
                       const double* solution, const int64_t* cell_dofs, const int64_t* dof_off,
                       const int32_t* cell_id, int64_t trace_size, const double* x, const int64_t* field_off,
                       const double* kfield, double* fields, void* stream) {
  if (count < 1 || nb < 2 || w < 3 || trace_size < 1 || !n_of || !t_of || !solution || !cell_dofs || !dof_off ||
      !cell_id || !x || !field_off || !fields)
    return MHM_ERR_ARGUMENT;
  dense_reconstruct_kernel<<<grid_for(count * nb), 256, 0, static_cast<cudaStream_t>(stream)>>>(
      count, nb, w, n_of, t_of, solution, cell_dofs, dof_off, cell_id, trace_size, x, field_off, fields, kfield);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}
}  // namespace

extern "C" int mhm_dense_systems(int64_t count, int32_t lds, int32_t tld, int32_t nb, int32_t w,
                                 int32_t normalize, const int32_t* n_of, const int32_t* t_of, const double* stiffness,
                                 const double* mass, const double* load, const double* coupling, double* aug,
                                 double* rhs, double* action, uint8_t* corrected, int32_t* status, void* stream) {
  return launch_systems(count, lds, tld, nb, w, normalize, n_of, t_of, stiffness, mass, load, coupling, nullptr,
                        aug, rhs, action, corrected, status, stream);
}

extern "C" int mhm_mixed_systems(int64_t count, int32_t lds, int32_t tld, int32_t nb, int32_t w,
                                 const int32_t* n_of, const int32_t* t_of, const double* matrix, const double* mass,
                                 const double* load, const double* coupling, const double* kernel, double* aug,
                                 double* rhs, double* action, uint8_t* corrected, int32_t* status, void* stream) {
  if (!kernel) return MHM_ERR_ARGUMENT;
  return launch_systems(count, lds, tld, nb, w, 1, n_of, t_of, matrix, mass, load, coupling, kernel, aug, rhs,
                        action, corrected, status, stream);
}

extern "C" int mhm_dense_systems_ragged(int64_t count, const mhm_ragged_matrix* desc, const int64_t* cpl_off,
                                        const int32_t* tld_of, int32_t normalize, const int32_t* n_of,
                                        const int32_t* t_of, const double* stiffness, const double* mass,
                                        const double* load, const double* coupling, double* aug, double* rhs,
                                        double* action, uint8_t* corrected, int32_t* status, void* stream) {
  if (count < 1 || count > INT32_MAX || !desc || !cpl_off || !tld_of || !n_of || !t_of || !stiffness || !mass ||
      !load || !coupling || !aug || !rhs || !action || !corrected || !status)
    return MHM_ERR_ARGUMENT;
  if (cudaFuncSetAttribute(dense_system_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                           (int)kSystemSmem) != cudaSuccess)
    return MHM_ERR_LAUNCH;
  dense_system_kernel<false><<<(unsigned)count, kDThreads, kSystemSmem, static_cast<cudaStream_t>(stream)>>>(
      0, 0, 0, 0, normalize, n_of, t_of, stiffness, mass, load, coupling, aug, rhs, action, corrected, status, desc,
      cpl_off, tld_of, nullptr);
  return cudaGetLastError() == cudaSuccess ? MHM_OK : MHM_ERR_LAUNCH;
}

extern "C" int mhm_dense_contributions(int64_t count, int32_t lds, int32_t tld, int32_t nb, int32_t w,
                                       int32_t max_t, const int32_t* n_of, const int32_t* t_of,
                                       const double* solution, const double* coupling, const double* action,
                                       const double* load, const int64_t* block_off, const int64_t* load_off,
                                       double* blocks, double* loads, void* stream) {
  return launch_contributions(count, lds, tld, nb, w, max_t, n_of, t_of, solution, coupling, action, load, nullptr,
                              1.0, block_off, load_off, blocks, loads, stream);
}

extern "C" int mhm_mixed_contributions(int64_t count, int32_t lds, int32_t tld, int32_t nb, int32_t w,
                                       int32_t max_t, const int32_t* n_of, const int32_t* t_of,
                                       const double* solution, const double* coupling, const double* action,
                                       const double* load, const double* kernel, const int64_t* block_off,
                                       const int64_t* load_off, double* blocks, double* loads, void* stream) {
  if (!kernel) return MHM_ERR_ARGUMENT;
  return launch_contributions(count, lds, tld, nb, w, max_t, n_of, t_of, solution, coupling, action, load, kernel,
                              -1.0, block_off, load_off, blocks, loads, stream);
}

extern "C" int mhm_dense_reconstruct(int64_t count, int32_t nb, int32_t w, const int32_t* n_of,
                                     const int32_t* t_of, const double* solution, const int64_t* cell_dofs,
                                     const int64_t* dof_off, const int32_t* cell_id, int64_t trace_size,
                                     const double* x, const int64_t* field_off, double* fields, void* stream) {
  return launch_reconstruct(count, nb, w, n_of, t_of, solution, cell_dofs, dof_off, cell_id, trace_size, x,
                            field_off, nullptr, fields, stream);
}

extern "C" int mhm_mixed_reconstruct(int64_t count, int32_t nb, int32_t w, const int32_t* n_of,
                                     const int32_t* t_of, const double* solution, const int64_t* cell_dofs,
                                     const int64_t* dof_off, const int32_t* cell_id, int64_t trace_size,
                                     const double* x, const int64_t* field_off, const double* kernel_fields,
                                     double* fields, void* stream) {
  if (!kernel_fields) return MHM_ERR_ARGUMENT;
  return launch_reconstruct(count, nb, w, n_of, t_of, solution, cell_dofs, dof_off, cell_id, trace_size, x,
                            field_off, kernel_fields, fields, stream);
}
