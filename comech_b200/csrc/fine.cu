// Level-0 operator kernels: structured matrix-free K.u, sparse pass, diagonal blocks.
#include "fine.cuh"

namespace feb {

namespace {

constexpr int TX = 32;        // cells per tile along x (one warp)
constexpr int TY = 8;         // cells per tile along y (warps)
constexpr int PX = TX + 1;    // node columns staged per plane
constexpr int PY = TY + 1;

template <typename T, int W>
__device__ __forceinline__ bool load_material(const T* __restrict__ p, T (&m)[W]) {
  bool nz = false;
#pragma unroll
  for (int q = 0; q < W; ++q) {
    m[q] = p[q];
    nz |= (m[q] != T(0));
  }
  return nz;
}

// Matrix-free K.u over the regular cells.  A CTA owns a (TX-1) x (TY-1) column of grid nodes over
// `zchunk` node planes.  It computes the TX x TY cells touching those nodes (the first row/column of
// cells is shared with the neighbouring CTAs and recomputed there), marching upward one cell layer
// at a time:
//   * the node plane above the layer is staged in shared memory (two-plane ring);
//   * every thread computes one cell's 24 nodal forces in registers (modal hex8 operator);
//   * forces of the x-neighbour arrive by warp shuffle, those of the y-neighbour row through shared
//     memory; each owned node sums its 4 cells of the layer below (kept in registers from the
//     previous step) and the 4 cells of the layer above, then stores its 3 components once.
// No global atomics: every output is written by exactly one thread.
template <typename T, int MODE>
__global__ void __launch_bounds__(TX * TY)
k_fine_struct(FineView<T> F, const T* __restrict__ u, T* __restrict__ y, const int* __restrict__ skip, int zchunk) {
  if (skip && *skip) return;
  constexpr int W = MatWidth<MODE>::value;
  __shared__ T plane[2][PY * PX * 3];
  __shared__ T rowp[TY][TX][6];
  const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
  const int pi0 = blockIdx.x * (TX - 1) - 1;
  const int pj0 = blockIdx.y * (TY - 1) - 1;
  const int ci = pi0 + tx, cj = pj0 + ty;       // this thread's cell, and the node it owns
  const int K0 = blockIdx.z * zchunk;
  const int K1 = min(K0 + zchunk, F.nzn);
  const bool cell_xy = (ci >= 0) && (ci < F.nx) && (cj >= 0) && (cj < F.ny);
  const bool owner = (tx >= 1) && (ty >= 1) && (ci < F.nxn) && (cj < F.nyn);
  T a = T(1), b = T(1), ia = T(1), ib = T(1);
  if (cell_xy) { a = F.dx[ci]; ia = F.idx[ci]; b = F.dy[cj]; ib = F.idy[cj]; }

  auto stage = [&](int k, int slot) {
    T* dst = plane[slot];
    const bool kin = (k >= 0) && (k < F.nzn);
    for (int e = tid; e < PY * PX * 3; e += TX * TY) {
      int row = e / (PX * 3), w = e - row * (PX * 3);
      int ni = pi0 + w / 3, nj = pj0 + row;
      T v = T(0);
      if (kin && ni >= 0 && ni < F.nxn && nj >= 0 && nj < F.nyn)
        v = u[3 * ((int64_t)ni + (int64_t)F.nxn * (nj + (int64_t)F.nyn * k)) + (w % 3)];
      dst[e] = v;
    }
  };

  T acc[3] = {T(0), T(0), T(0)};
  stage(K0 - 1, (K0 - 1) & 1);
  for (int k = K0 - 1; k < K1; ++k) {
    stage(k + 1, (k + 1) & 1);
    T m[W];
    bool act = false;
    if (cell_xy && k >= 0 && k < F.nz)
      act = load_material<T, W>(F.mat + (size_t)W * ((int64_t)ci + (int64_t)F.nx * (cj + (int64_t)F.ny * k)), m);
    __syncthreads();
    T f[3][8];
    if (act) {
      T uc[3][8];
#pragma unroll
      for (int l = 0; l < 8; ++l) {
        const T* src = plane[(k + ((l >> 2) & 1)) & 1] + ((ty + ((l >> 1) & 1)) * PX + tx + (l & 1)) * 3;
#pragma unroll
        for (int c = 0; c < 3; ++c) uc[c][l] = src[c];
      }
      T cz = F.dz[k], icz = F.idz[k];
      Material<T> mat = make_material<T, MODE>(m);
      hex8_apply(uc, a, b, cz, ia, ib, icz, mat, f);
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int l = 0; l < 8; ++l) f[c][l] = T(0);
    }
    T own[2][3];
#pragma unroll
    for (int zl = 0; zl < 2; ++zl) {
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        T left_own = __shfl_up_sync(0xffffffffu, f[c][1 + 4 * zl], 1);
        T left_row = __shfl_up_sync(0xffffffffu, f[c][3 + 4 * zl], 1);
        own[zl][c] = f[c][4 * zl] + (tx ? left_own : T(0));
        rowp[ty][tx][3 * zl + c] = f[c][2 + 4 * zl] + (tx ? left_row : T(0));
      }
    }
    __syncthreads();
    if (ty >= 1) {
#pragma unroll
      for (int zl = 0; zl < 2; ++zl)
#pragma unroll
        for (int c = 0; c < 3; ++c) own[zl][c] += rowp[ty - 1][tx][3 * zl + c];
    }
    if (k >= K0 && owner) {
      T* dst = y + 3 * ((int64_t)ci + (int64_t)F.nxn * (cj + (int64_t)F.nyn * k));
#pragma unroll
      for (int c = 0; c < 3; ++c) dst[c] = acc[c] + own[0][c];
    }
#pragma unroll
    for (int c = 0; c < 3; ++c) acc[c] = own[1][c];
  }
}

// Sparse part of the level-0 operator, accumulated into y with atomics after k_fine_struct:
//   blocks [0, b_irr)            irregular cells (cells touching split copies), one thread per cell
//   blocks [b_irr, b_irr+b_pen)  diagonal penalties, one thread per node
//   remaining blocks             rows of the extra matrix, one thread per row
template <typename T, int MODE>
__global__ void __launch_bounds__(kThreads)
k_fine_sparse(FineView<T> F, const T* __restrict__ u, T* __restrict__ y, const int* __restrict__ skip, int b_irr,
              int b_pen) {
  if (skip && *skip) return;
  constexpr int W = MatWidth<MODE>::value;
  const int bid = blockIdx.x;
  if (bid < b_irr) {
    int e = bid * kThreads + threadIdx.x;
    if (e >= F.nirr) return;
    int cell = F.irr_cell[e];
    int i = cell % F.nx, j = (cell / F.nx) % F.ny, k = cell / (F.nx * F.ny);
    int nodes[8];
    T uc[3][8];
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      nodes[l] = F.irr_nodes[8 * e + l];
#pragma unroll
      for (int c = 0; c < 3; ++c) uc[c][l] = u[3 * (int64_t)nodes[l] + c];
    }
    T m[W];
#pragma unroll
    for (int q = 0; q < W; ++q) m[q] = F.irr_mat[(size_t)W * e + q];
    Material<T> mat = make_material<T, MODE>(m);
    T f[3][8];
    hex8_apply(uc, F.dx[i], F.dy[j], F.dz[k], F.idx[i], F.idy[j], F.idz[k], mat, f);
#pragma unroll
    for (int l = 0; l < 8; ++l)
#pragma unroll
      for (int c = 0; c < 3; ++c) atomic_add(y + 3 * (int64_t)nodes[l] + c, f[c][l]);
  } else if (bid < b_irr + b_pen) {
    int e = (bid - b_irr) * kThreads + threadIdx.x;
    if (e >= F.npen) return;
    int64_t n = F.pen_node[e];
#pragma unroll
    for (int c = 0; c < 3; ++c) atomic_add(y + 3 * n + c, F.pen_k[3 * e + c] * u[3 * n + c]);
  } else {
    int e = (bid - b_irr - b_pen) * kThreads + threadIdx.x;
    if (e >= F.nrow) return;
    T s = T(0);
    for (int q = F.row_ptr[e]; q < F.row_ptr[e + 1]; ++q) s += F.val[q] * u[F.col[q]];
    atomic_add(y + F.row_dof[e], s);
  }
}

// Copies (ids >= nnode) receive no structured contribution: clear them before the sparse pass.
template <typename T>
__global__ void k_zero_tail(T* __restrict__ y, int64_t from, int64_t to, const int* __restrict__ skip) {
  if (skip && *skip) return;
  int64_t i = from + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i < to) y[i] = T(0);
}

// Diagonal 3x3 block contributed by one cell at corner l (closed form of the 2x2x2 Gauss integrals:
// int Nx^2 = bc/(9a), int Nx Ny = sx sy c/12, ...; centre lambda: vol (sx/4a)(sy/4b) ...).
template <int MODE>
__device__ __forceinline__ void corner_diag(int l, double a, double b, double c, const double* p, double (&D)[9]) {
  Material<double> m = make_material<double, MODE>(p);
  const double sx = (l & 1) ? 1.0 : -1.0, sy = (l & 2) ? 1.0 : -1.0, sz = (l & 4) ? 1.0 : -1.0;
  const double Ixx = b * c / (9.0 * a), Iyy = a * c / (9.0 * b), Izz = a * b / (9.0 * c);
  const double Ixy = sx * sy * c / 12.0, Ixz = sx * sz * b / 12.0, Iyz = sy * sz * a / 12.0;
  D[0] += m.c0 * Ixx + m.c4 * Iyy + m.c5 * Izz;
  D[4] += m.c4 * Ixx + m.c0 * Iyy + m.c5 * Izz;
  D[8] += m.c5 * Ixx + m.c5 * Iyy + m.c3 * Izz;
  D[1] += (m.c1 + m.c4) * Ixy; D[3] += (m.c1 + m.c4) * Ixy;
  D[2] += (m.c2 + m.c5) * Ixz; D[6] += (m.c2 + m.c5) * Ixz;
  D[5] += (m.c2 + m.c5) * Iyz; D[7] += (m.c2 + m.c5) * Iyz;
  if (m.lamc != 0.0) {
    const double v = a * b * c, gx = sx / (4.0 * a), gy = sy / (4.0 * b), gz = sz / (4.0 * c);
    const double g[3] = {gx, gy, gz};
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
      for (int q = 0; q < 3; ++q) D[3 * r + q] += m.lamc * v * g[r] * g[q];
  }
}

template <int MODE>
__global__ void k_fine_diag_grid(FineView<double> F, double* __restrict__ D) {
  constexpr int W = MatWidth<MODE>::value;
  int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= F.ntotal) return;
  double d[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  if (n < F.nnode) {
    int i = int(n % F.nxn), j = int((n / F.nxn) % F.nyn), k = int(n / ((int64_t)F.nxn * F.nyn));
#pragma unroll
    for (int l = 0; l < 8; ++l) {          // cell whose corner l is this node
      int ci = i - (l & 1), cj = j - ((l >> 1) & 1), ck = k - ((l >> 2) & 1);
      if (ci < 0 || cj < 0 || ck < 0 || ci >= F.nx || cj >= F.ny || ck >= F.nz) continue;
      const double* p = F.mat + (size_t)W * (ci + (int64_t)F.nx * (cj + (int64_t)F.ny * ck));
      bool nz = false;
#pragma unroll
      for (int q = 0; q < W; ++q) nz |= (p[q] != 0.0);
      if (nz) corner_diag<MODE>(l, F.dx[ci], F.dy[cj], F.dz[ck], p, d);
    }
  }
#pragma unroll
  for (int q = 0; q < 9; ++q) D[9 * n + q] = d[q];
}

template <int MODE>
__global__ void k_fine_diag_sparse(FineView<double> F, double* __restrict__ D) {
  constexpr int W = MatWidth<MODE>::value;
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < F.nirr) {
    int cell = F.irr_cell[e];
    int i = cell % F.nx, j = (cell / F.nx) % F.ny, k = cell / (F.nx * F.ny);
    for (int l = 0; l < 8; ++l) {
      double d[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
      corner_diag<MODE>(l, F.dx[i], F.dy[j], F.dz[k], F.irr_mat + (size_t)W * e, d);
      int64_t n = F.irr_nodes[8 * e + l];
      for (int q = 0; q < 9; ++q) atomicAdd(D + 9 * n + q, d[q]);
    }
  }
  if (e < F.npen) {
    int64_t n = F.pen_node[e];
    for (int c = 0; c < 3; ++c) atomicAdd(D + 9 * n + 4 * c, F.pen_k[3 * e + c]);
  }
  if (e < F.nrow) {
    int rd = F.row_dof[e];
    int64_t n = rd / 3;
    int r = rd % 3;
    for (int q = F.row_ptr[e]; q < F.row_ptr[e + 1]; ++q) {
      int cd = F.col[q];
      if (cd / 3 == n) atomicAdd(D + 9 * n + 3 * r + cd % 3, F.val[q]);
    }
  }
}

// column q of K_e for every regular / irregular cell, scattered into the dense matrix
template <int MODE>
__global__ void k_dense_from_fine(FineView<double> F, const int* __restrict__ cmap, double* __restrict__ M, int nd) {
  constexpr int W = MatWidth<MODE>::value;
  const int q = threadIdx.x;     // 0..23
  const int64_t ncell = (int64_t)F.nx * F.ny * F.nz;
  const int64_t e = blockIdx.x * (int64_t)blockDim.y + threadIdx.y;
  if (e >= ncell + F.nirr) return;
  int i, j, k;
  int64_t nodes[8];
  double m[W];
  if (e < ncell) {
    i = int(e % F.nx); j = int((e / F.nx) % F.ny); k = int(e / ((int64_t)F.nx * F.ny));
    bool nz = false;
    for (int t = 0; t < W; ++t) { m[t] = F.mat[(size_t)W * e + t]; nz |= (m[t] != 0.0); }
    if (!nz) return;
    for (int l = 0; l < 8; ++l)
      nodes[l] = (i + (l & 1)) + (int64_t)F.nxn * ((j + ((l >> 1) & 1)) + (int64_t)F.nyn * (k + ((l >> 2) & 1)));
  } else {
    int r = int(e - ncell);
    int cell = F.irr_cell[r];
    i = cell % F.nx; j = (cell / F.nx) % F.ny; k = cell / (F.nx * F.ny);
    for (int t = 0; t < W; ++t) m[t] = F.irr_mat[(size_t)W * r + t];
    for (int l = 0; l < 8; ++l) nodes[l] = F.irr_nodes[8 * r + l];
  }
  double u[3][8], f[3][8];
  for (int l = 0; l < 8; ++l)
    for (int c = 0; c < 3; ++c) u[c][l] = (3 * l + c == q) ? 1.0 : 0.0;
  Material<double> mt = make_material<double, MODE>(m);
  hex8_apply(u, F.dx[i], F.dy[j], F.dz[k], F.idx[i], F.idy[j], F.idz[k], mt, f);
  const int cq = cmap[nodes[q / 3]];
  if (cq < 0) return;
  for (int l = 0; l < 8; ++l) {
    int cl = cmap[nodes[l]];
    if (cl < 0) continue;
    for (int r = 0; r < 3; ++r) atomicAdd(M + (size_t)(3 * cl + r) * nd + 3 * cq + q % 3, f[r][l]);
  }
}

__global__ void k_dense_penalty(FineView<double> F, const int* __restrict__ cmap, double* __restrict__ M, int nd) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= F.npen) return;
  int c = cmap[F.pen_node[e]];
  if (c < 0) return;
  for (int q = 0; q < 3; ++q) atomicAdd(M + (size_t)(3 * c + q) * nd + 3 * c + q, F.pen_k[3 * e + q]);
}

__global__ void k_dense_csr(FineView<double> F, const int* __restrict__ cmap, double* __restrict__ M, int nd) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= F.nrow) return;
  int rd = F.row_dof[e];
  int cr = cmap[rd / 3];
  if (cr < 0) return;
  for (int q = F.row_ptr[e]; q < F.row_ptr[e + 1]; ++q) {
    int cc = cmap[F.col[q] / 3];
    if (cc >= 0) atomicAdd(M + (size_t)(3 * cr + rd % 3) * nd + 3 * cc + F.col[q] % 3, F.val[q]);
  }
}

}  // namespace

template <int MODE>
void launch_dense_from_fine(const FineView<double>& F, const int* cmap, double* M, int nd, cudaStream_t s) {
  int64_t n = (int64_t)F.nx * F.ny * F.nz + F.nirr;
  dim3 blk(24, 8);
  k_dense_from_fine<MODE><<<div_up(n, 8), blk, 0, s>>>(F, cmap, M, nd); note_launch();
  if (F.npen) k_dense_penalty<<<div_up(F.npen, kThreads), kThreads, 0, s>>>(F, cmap, M, nd); note_launch();
  if (F.nrow) k_dense_csr<<<div_up(F.nrow, kThreads), kThreads, 0, s>>>(F, cmap, M, nd); note_launch();
}
template void launch_dense_from_fine<MAT_ISO_SRI>(const FineView<double>&, const int*, double*, int, cudaStream_t);
template void launch_dense_from_fine<MAT_ISO_FULL>(const FineView<double>&, const int*, double*, int, cudaStream_t);
template void launch_dense_from_fine<MAT_ORTHO>(const FineView<double>&, const int*, double*, int, cudaStream_t);

template <typename T, int MODE>
void launch_fine_apply(const FineView<T>& F, const T* u, T* y, const int* skip, int zchunk, cudaStream_t s) {
  dim3 block(TX, TY);
  dim3 grid(div_up(F.nxn, TX - 1), div_up(F.nyn, TY - 1), div_up(F.nzn, zchunk));
  k_fine_struct<T, MODE><<<grid, block, 0, s>>>(F, u, y, skip, zchunk); note_launch();
  if (F.ntotal > F.nnode) {
    int64_t n = 3 * (F.ntotal - F.nnode);
    k_zero_tail<T><<<div_up(n, kThreads), kThreads, 0, s>>>(y, 3 * F.nnode, 3 * F.ntotal, skip); note_launch();
  }
  int b_irr = div_up(F.nirr, kThreads), b_pen = div_up(F.npen, kThreads), b_row = div_up(F.nrow, kThreads);
  if (b_irr + b_pen + b_row > 0)
    k_fine_sparse<T, MODE><<<b_irr + b_pen + b_row, kThreads, 0, s>>>(F, u, y, skip, b_irr, b_pen); note_launch();
}

template <int MODE>
void launch_fine_diag(const FineView<double>& F, double* D, cudaStream_t s) {
  k_fine_diag_grid<MODE><<<div_up(F.ntotal, kThreads), kThreads, 0, s>>>(F, D); note_launch();
  int n = max(F.nirr, max(F.npen, F.nrow));
  if (n > 0) k_fine_diag_sparse<MODE><<<div_up(n, kThreads), kThreads, 0, s>>>(F, D); note_launch();
}

#define INST(T, M) template void launch_fine_apply<T, M>(const FineView<T>&, const T*, T*, const int*, int, cudaStream_t);
INST(float, MAT_ISO_SRI) INST(float, MAT_ISO_FULL) INST(float, MAT_ORTHO)
INST(double, MAT_ISO_SRI) INST(double, MAT_ISO_FULL) INST(double, MAT_ORTHO)
#undef INST
template void launch_fine_diag<MAT_ISO_SRI>(const FineView<double>&, double*, cudaStream_t);
template void launch_fine_diag<MAT_ISO_FULL>(const FineView<double>&, double*, cudaStream_t);
template void launch_fine_diag<MAT_ORTHO>(const FineView<double>&, double*, cudaStream_t);

}  // namespace feb
