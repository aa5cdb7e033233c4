// Coarsest multigrid level: dense FP64 matrix over the kept dofs, explicit inverse by a blocked
// Gauss-Jordan sweep (symmetric positive definite, no pivoting), applied as a GEMV in every V-cycle.
// The reference factorises the same matrix (SciPy splu, fe/gmg.py:102; cuSOLVER Cholesky,
// rb/gpusolve.py:138-161); an explicit inverse turns the per-V-cycle solve into one coalesced GEMV.
#include "dense.cuh"

namespace feb {

namespace {

constexpr int GJ_B = 32;      // pivot block
constexpr int GJ_T = 64;      // update tile

__global__ void k_dense_from_stencil(const double* __restrict__ A, int nx, int ny, int nz,
                                     const int* __restrict__ cmap, double* __restrict__ M, int nd) {
  const int o = threadIdx.x;
  const int64_t n = (int64_t)nx * ny * nz;
  const int64_t J = blockIdx.x * (int64_t)blockDim.y + threadIdx.y;
  if (J >= n) return;
  int cj = cmap[J];
  if (cj < 0) return;
  int i = int(J % nx), j = int((J / nx) % ny), k = int(J / ((int64_t)nx * ny));
  int dx = o % 3 - 1, dy = (o / 3) % 3 - 1, dz = o / 9 - 1;
  if (i + dx < 0 || i + dx >= nx || j + dy < 0 || j + dy >= ny || k + dz < 0 || k + dz >= nz) return;
  int64_t K = J + dx + (int64_t)nx * (dy + (int64_t)ny * dz);
  int ck = cmap[K];
  if (ck < 0) return;
  for (int r = 0; r < 3; ++r)
    for (int c = 0; c < 3; ++c)
      M[(size_t)(3 * cj + r) * nd + 3 * ck + c] += A[(size_t)(o * 9 + 3 * r + c) * n + J];
}

__global__ void k_dense_add_entries(int nent, const int* __restrict__ rdof, const int* __restrict__ cdof,
                                    const double* __restrict__ val, const int* __restrict__ cmap,
                                    double* __restrict__ M, int nd) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nent) return;
  int cr = cmap[rdof[e] / 3], cc = cmap[cdof[e] / 3];
  if (cr < 0 || cc < 0) return;
  atomicAdd(M + (size_t)(3 * cr + rdof[e] % 3) * nd + 3 * cc + cdof[e] % 3, val[e]);
}

__global__ void k_symmetrize(double* __restrict__ M, int nd) {
  int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int64_t i = t / nd, j = t % nd;
  if (i >= nd || j <= i) return;
  double v = 0.5 * (M[i * nd + j] + M[j * nd + i]);
  M[i * nd + j] = v;
  M[j * nd + i] = v;
}

// Invert the pivot block in shared memory (scalar Gauss-Jordan, SPD so no pivoting), one thread per element:
// each sweep step p reads a_ip, a_pj, a_pp, then every thread rewrites its own element
// (a_ij -= a_ip a_pj / a_pp; a_pj /= a_pp; a_ip = -a_ip / a_pp; a_pp = 1 / a_pp).
__global__ void __launch_bounds__(GJ_B * GJ_B)
k_gj_pivot(double* __restrict__ M, int nd, int k0, int bs, double* __restrict__ Dinv, int* __restrict__ status) {
  __shared__ double a[GJ_B][GJ_B + 1];
  const int i = threadIdx.y, j = threadIdx.x;
  const bool in = i < bs && j < bs;
  if (in) a[i][j] = M[(size_t)(k0 + i) * nd + k0 + j];
  __syncthreads();
  for (int p = 0; p < bs; ++p) {
    double piv = a[p][p];
    const double aip = in ? a[i][p] : 0.0, apj = in ? a[p][j] : 0.0, aij = in ? a[i][j] : 0.0;
    __syncthreads();
    if (!(piv > 0.0) || !isfinite(piv)) {
      if (i == 0 && j == 0) atomicExch(status, FEB_ERR_COARSE);
      piv = 1.0;
    }
    const double ip = 1.0 / piv;
    if (in) {
      if (i != p && j != p) a[i][j] = aij - aip * apj * ip;
      else if (i == p && j != p) a[p][j] = apj * ip;
      else if (j == p && i != p) a[i][p] = -aip * ip;
      else a[p][p] = ip;
    }
    __syncthreads();
  }
  if (in) Dinv[i * bs + j] = a[i][j];
}

// Trow[r][j] = sum_q Dinv[r][q] M[k0+q][j] for all j (pivot-block rows of the sweep)
__global__ void k_gj_row(const double* __restrict__ M, int nd, int k0, int bs, const double* __restrict__ Dinv,
                         double* __restrict__ Trow) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (j >= nd || r >= bs) return;
  double s = 0.0;
  for (int q = 0; q < bs; ++q) s += Dinv[r * bs + q] * M[(size_t)(k0 + q) * nd + j];
  Trow[(size_t)r * nd + j] = s;
}

// Tcol[i][q] = M[i][k0+q]: the pivot-block columns before the sweep changes them
__global__ void k_gj_colcopy(const double* __restrict__ M, int nd, int k0, int bs, double* __restrict__ Tcol) {
  int i = blockIdx.x * blockDim.x + threadIdx.x;
  int q = blockIdx.y;
  if (i >= nd || q >= bs) return;
  Tcol[(size_t)i * GJ_B + q] = M[(size_t)i * nd + k0 + q];
}

// M[i][j] -= Tcol[i][:] Trow[:, j] for i, j outside the pivot block (64x64 tiles, 4x4 per thread)
__global__ void __launch_bounds__(256)
k_gj_update(double* __restrict__ M, int nd, int k0, int bs, const double* __restrict__ Tcol,
            const double* __restrict__ Trow) {
  __shared__ double As[GJ_T][GJ_B + 1];
  __shared__ double Bs[GJ_B][GJ_T + 1];
  const int i0 = blockIdx.y * GJ_T, j0 = blockIdx.x * GJ_T;
  const int t = threadIdx.x;
  for (int e = t; e < GJ_T * GJ_B; e += 256) {
    int ii = e / GJ_B, q = e % GJ_B;
    As[ii][q] = (i0 + ii < nd && q < bs) ? Tcol[(size_t)(i0 + ii) * GJ_B + q] : 0.0;
    int q2 = e / GJ_T, jj = e % GJ_T;
    Bs[q2][jj] = (j0 + jj < nd && q2 < bs) ? Trow[(size_t)q2 * nd + j0 + jj] : 0.0;
  }
  __syncthreads();
  const int ty = t / 16, tx = t % 16;
  double acc[4][4] = {};
  for (int q = 0; q < bs; ++q) {
    double av[4], bv[4];
#pragma unroll
    for (int u = 0; u < 4; ++u) { av[u] = As[ty + 16 * u][q]; bv[u] = Bs[q][tx + 16 * u]; }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v) acc[u][v] += av[u] * bv[v];
  }
#pragma unroll
  for (int u = 0; u < 4; ++u) {
    int i = i0 + ty + 16 * u;
    if (i >= nd || (i >= k0 && i < k0 + bs)) continue;
#pragma unroll
    for (int v = 0; v < 4; ++v) {
      int j = j0 + tx + 16 * v;
      if (j >= nd || (j >= k0 && j < k0 + bs)) continue;
      M[(size_t)i * nd + j] -= acc[u][v];
    }
  }
}

// pivot rows: M[k-block][j] <- Trow (j outside the block); pivot columns: M[i][k-block] <- -Tcol[i] Dinv
// (i outside), M[kk] <- Dinv.  One thread per element of the pivot rows and of the pivot columns.
__global__ void k_gj_finish(double* __restrict__ M, int nd, int k0, int bs, const double* __restrict__ Dinv,
                            const double* __restrict__ Trow, const double* __restrict__ Tcol) {
  int j = blockIdx.x * blockDim.x + threadIdx.x;
  int r = blockIdx.y;
  if (j >= nd || r >= bs) return;
  // element (k0 + r, j) of the pivot rows
  if (j >= k0 && j < k0 + bs) M[(size_t)(k0 + r) * nd + j] = Dinv[r * bs + (j - k0)];
  else M[(size_t)(k0 + r) * nd + j] = Trow[(size_t)r * nd + j];
  // element (j, k0 + r) of the pivot columns (row j outside the block)
  if (j < k0 || j >= k0 + bs) {
    double s = 0.0;
    for (int q = 0; q < bs; ++q) s += Tcol[(size_t)j * GJ_B + q] * Dinv[q * bs + r];
    M[(size_t)j * nd + k0 + r] = -s;
  }
}

// x = Minv b on the coarsest level in one launch: blocks [0, brows) take 8 rows each (warp per row, b gathered
// through klist on the fly, the row's result written straight to its node); the remaining blocks zero the
// entries of nodes outside the dense system (cmap < 0), a disjoint set.
template <typename T>
__global__ void k_dense_solve(const double* __restrict__ Minv, int nd, const int* __restrict__ klist,
                              const int* __restrict__ cmap, int64_t n, const T* __restrict__ b, T* __restrict__ x,
                              int brows, const int* __restrict__ skip) {
  if (skip && *skip) return;
  if ((int)blockIdx.x < brows) {
    const int row = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
    if (row >= nd) return;
    const double* m = Minv + (size_t)row * nd;
    double acc = 0.0;
    for (int j = lane; j < nd; j += 32) acc += m[j] * double(b[3 * (int64_t)klist[j / 3] + j % 3]);
    acc = warp_sum(acc);
    if (lane == 0) x[3 * (int64_t)klist[row / 3] + row % 3] = T(acc);
    return;
  }
  const int64_t e = (int64_t)(blockIdx.x - brows) * blockDim.x + threadIdx.x;
  if (e < 3 * n && cmap[e / 3] < 0) x[e] = T(0);
}

}  // namespace

void launch_dense_from_stencil(const double* A, int nx, int ny, int nz, const int* cmap, double* M, int nd,
                               cudaStream_t s) {
  int64_t n = (int64_t)nx * ny * nz;
  dim3 blk(27, 8);
  k_dense_from_stencil<<<div_up(n, 8), blk, 0, s>>>(A, nx, ny, nz, cmap, M, nd); note_launch();
}

// M += lam_t v_t v_t^T of every term (one block per term; entries on dropped nodes are skipped)
__global__ void k_dense_add_terms(const int* __restrict__ t_ptr, const int* __restrict__ t_dof,
                                  const double* __restrict__ t_val, const double* __restrict__ t_lam,
                                  const int* __restrict__ cmap, double* __restrict__ M, int nd) {
  const int t = blockIdx.x, eb = t_ptr[t], ne = t_ptr[t + 1] - eb;
  const double lam = t_lam[t];
  for (int q = threadIdx.x; q < ne * ne; q += blockDim.x) {
    const int a = eb + q / ne, b = eb + q % ne;
    const int ca = cmap[t_dof[a] / 3], cb = cmap[t_dof[b] / 3];
    if (ca < 0 || cb < 0) continue;
    atomicAdd(M + (size_t)(3 * ca + t_dof[a] % 3) * nd + 3 * cb + t_dof[b] % 3, lam * t_val[a] * t_val[b]);
  }
}

void launch_dense_add_terms(int nterms, const int* t_ptr, const int* t_dof, const double* t_val, const double* t_lam,
                            const int* cmap, double* M, int nd, cudaStream_t s) {
  if (nterms > 0) k_dense_add_terms<<<nterms, kThreads, 0, s>>>(t_ptr, t_dof, t_val, t_lam, cmap, M, nd); note_launch();
}

void launch_dense_add_entries(int nent, const int* rdof, const int* cdof, const double* val, const int* cmap,
                              double* M, int nd, cudaStream_t s) {
  if (nent > 0) k_dense_add_entries<<<div_up(nent, kThreads), kThreads, 0, s>>>(nent, rdof, cdof, val, cmap, M, nd); note_launch();
}

void launch_dense_invert(double* M, int nd, double* scratch, int* status, cudaStream_t s) {
  k_symmetrize<<<div_up((int64_t)nd * nd, kThreads), kThreads, 0, s>>>(M, nd); note_launch();
  double* Dinv = scratch;
  double* Trow = scratch + GJ_B * GJ_B;
  double* Tcol = Trow + (size_t)GJ_B * nd;
  for (int k0 = 0; k0 < nd; k0 += GJ_B) {
    int bs = std::min(GJ_B, nd - k0);
    k_gj_pivot<<<1, dim3(GJ_B, GJ_B), 0, s>>>(M, nd, k0, bs, Dinv, status); note_launch();
    dim3 g1(div_up(nd, 128), bs);
    k_gj_row<<<g1, 128, 0, s>>>(M, nd, k0, bs, Dinv, Trow); note_launch();
    k_gj_colcopy<<<g1, 128, 0, s>>>(M, nd, k0, bs, Tcol); note_launch();
    dim3 g2(div_up(nd, GJ_T), div_up(nd, GJ_T));
    k_gj_update<<<g2, 256, 0, s>>>(M, nd, k0, bs, Tcol, Trow); note_launch();
    k_gj_finish<<<g1, 128, 0, s>>>(M, nd, k0, bs, Dinv, Trow, Tcol); note_launch();
  }
}

size_t dense_scratch_doubles(int nd) { return (size_t)GJ_B * GJ_B + 2 * (size_t)GJ_B * nd; }

template <typename T>
void launch_dense_solve(const double* Minv, int nd, const int* klist, const int* cmap, int64_t n, const T* b, T* x,
                        const int* skip, cudaStream_t s) {
  const int brows = div_up(nd, 8);
  k_dense_solve<T><<<brows + (int)div_up(3 * n, 256), 256, 0, s>>>(Minv, nd, klist, cmap, n, b, x, brows, skip);
  note_launch();
}

template void launch_dense_solve<float>(const double*, int, const int*, const int*, int64_t, const float*, float*,
                                        const int*, cudaStream_t);
template void launch_dense_solve<double>(const double*, int, const int*, const int*, int64_t, const double*, double*,
                                         const int*, cudaStream_t);

}  // namespace feb
