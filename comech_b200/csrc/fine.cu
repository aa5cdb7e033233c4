// Level-0 operator kernels: structured matrix-free K.u, sparse pass, diagonal blocks.
#include <algorithm>

#include "fine.cuh"

namespace feb {

namespace {

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

// Matrix-free K.u over the regular cells, sum-factorised across cells.
//
// A CTA of 32 x TY threads owns a 30 x (TY-2) column of grid nodes over `zchunk` node planes and computes
// the 31 x (TY-1) cells touching them (the outermost row / column of cells is shared with the neighbouring
// CTAs).  Thread (tx, ty) holds node (tx, ty) of the node planes, prefetched two planes ahead, and works
// on the xy-face and x-edge that start at its node:
//   forward   x-edge butterfly of its node and its +x neighbour (warp shuffle), xy-face butterfly with the
//             edge of the row above (shared memory) -- once per plane, shared by the two cells above and
//             below the face; the z butterfly between the faces of planes k and k+1 completes the modal
//             transform of cell layer k;
//   core      the element operator in the modal basis (hex8_modal);
//   backward  the transposed butterflies in reverse: z (into the faces of planes k and k+1, the upper one
//             carried in registers to the next layer), y (into the edge of this row and, through shared
//             memory, of the row above), x (into this node and, by shuffle, its +x neighbour).
// Each owned node therefore sums its 8 cells with no global atomics and stores its 3 components once.
// One barrier per cell layer: both shared-memory exchanges are double-buffered.
template <typename T, int MODE, int TY>
__global__ void __launch_bounds__(32 * TY)
k_fine_struct(FineView<T> F, const T* __restrict__ u, T* __restrict__ y, const int* __restrict__ skip, int zchunk) {
  if (skip && *skip) return;
  constexpr int W = MatWidth<MODE>::value;
  constexpr bool HAS12 = (MODE != MAT_ISO_SRI);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T (*sE)[TY][32][6] = reinterpret_cast<T (*)[TY][32][6]>(smem_raw);                               // [2]
  T (*sB)[TY][32][6] = reinterpret_cast<T (*)[TY][32][6]>(smem_raw + sizeof(T) * 2 * TY * 32 * 6);  // [2]
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int ni = blockIdx.x * 30 - 1 + tx;
  const int nj = blockIdx.y * (TY - 2) - 1 + ty;
  const int K0 = blockIdx.z * zchunk;
  const int K1 = min(K0 + zchunk, F.nzn);
  const bool node_in = ni >= 0 && ni < F.nxn && nj >= 0 && nj < F.nyn;
  const bool cell_xy = tx < 31 && ty < TY - 1 && ni >= 0 && ni < F.nx && nj >= 0 && nj < F.ny;
  const bool owner = tx >= 1 && tx <= 30 && ty >= 1 && ty <= TY - 2 && ni < F.nxn && nj < F.nyn;
  const bool has_above = ty + 1 < TY;
  const int64_t plane = (int64_t)F.nxn * F.nyn;
  const int64_t nbase = node_in ? (ni + (int64_t)F.nxn * nj) : 0;
  const int64_t cplane = (int64_t)F.nx * F.ny;
  const int64_t cbase = cell_xy ? (ni + (int64_t)F.nx * nj) : 0;
  T a = T(1), b = T(1), ia = T(1), ib = T(1);
  if (cell_xy) { a = F.dx[ni]; ia = F.idx[ni]; b = F.dy[nj]; ib = F.idy[nj]; }

  auto load_node = [&](int k, T (&v)[3]) {
    if (node_in && k >= 0 && k < F.nzn) {
      const T* p = u + 3 * (nbase + plane * k);
      v[0] = p[0]; v[1] = p[1]; v[2] = p[2];
    } else {
      v[0] = v[1] = v[2] = T(0);
    }
  };
  auto load_mat = [&](int k, T (&m)[W]) {
    if (cell_xy && k >= 0 && k < F.nz) {
      const T* p = F.mat + (size_t)W * (cbase + cplane * k);
#pragma unroll
      for (int q = 0; q < W; ++q) m[q] = p[q];
    } else {
#pragma unroll
      for (int q = 0; q < W; ++q) m[q] = T(0);
    }
  };
  // x-edge butterfly of this node and its +x neighbour: E[c] = (sum, difference)
  auto edge = [&](const T (&v)[3], T (&E)[3][2]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T w = __shfl_down_sync(0xffffffffu, v[c], 1);
      E[c][0] = v[c] + w;
      E[c][1] = w - v[c];
    }
  };
  auto put6 = [&](T* d, const T (&E)[3][2]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) { d[2 * c] = E[c][0]; d[2 * c + 1] = E[c][1]; }
  };
  auto get6 = [&](const T* s, T (&E)[3][2]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) { E[c][0] = s[2 * c]; E[c][1] = s[2 * c + 1]; }
  };
  auto slot = [](int p) { return (p + 2) & 1; };

  T vn[3], vp[3], vq[3], mc[W], mn[W];
  T Fk[3][4], topc[3][4], plo[3][2];
  // prologue: face of plane K0-1
  {
    T v0[3], E[3][2], A[3][2] = {};
    load_node(K0 - 1, v0);
    load_node(K0, vn);
    load_node(K0 + 1, vp);
    load_mat(K0 - 1, mc);
    edge(v0, E);
    put6(sE[slot(K0 - 1)][ty][tx], E);
    __syncthreads();
    if (has_above) get6(sE[slot(K0 - 1)][ty + 1][tx], A);
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int ax = 0; ax < 2; ++ax) {
        Fk[c][ax] = E[c][ax] + A[c][ax];
        Fk[c][ax + 2] = A[c][ax] - E[c][ax];
        topc[c][ax] = topc[c][ax + 2] = T(0);
      }
#pragma unroll
    for (int c = 0; c < 3; ++c) plo[c][0] = plo[c][1] = T(0);
  }
  for (int k = K0 - 1; k < K1; ++k) {
    // (a) x-edge of plane k+1; prefetch plane k+3 and the material of layer k+1
    T E[3][2];
    edge(vn, E);
    put6(sE[slot(k + 1)][ty][tx], E);
    load_node(k + 3, vq);
    load_mat(k + 1, mn);
    __syncthreads();
    // (c) finish plane k-1: edge = this face's lower share + the row below's upper share; x back-transform
    if (k > K0 - 1) {
      T up[3][2] = {};
      if (ty >= 1) get6(sB[slot(k - 1)][ty - 1][tx], up);
      T out[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const T m = plo[c][0] + up[c][0], d = plo[c][1] + up[c][1];
        const T left = __shfl_up_sync(0xffffffffu, m + d, 1);
        out[c] = (m - d) + (tx ? left : T(0));
      }
      if (owner && k - 1 >= K0) {
        T* dst = y + 3 * (nbase + plane * (k - 1));
        dst[0] = out[0]; dst[1] = out[1]; dst[2] = out[2];
      }
    }
    // (d) xy-face of plane k+1, (e) z butterfly -> modal coefficients of cell layer k
    T A[3][2] = {};
    if (has_above) get6(sE[slot(k + 1)][ty + 1][tx], A);
    T Fk1[3][4];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int ax = 0; ax < 2; ++ax) {
        Fk1[c][ax] = E[c][ax] + A[c][ax];
        Fk1[c][ax + 2] = A[c][ax] - E[c][ax];
      }
    bool act = false;
#pragma unroll
    for (int q = 0; q < W; ++q) act |= (mc[q] != T(0));
    T G[3][4];
    if (act) {
      T X[8], Y[8], Z[8];
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        X[l] = Fk[0][l] + Fk1[0][l]; X[l + 4] = Fk1[0][l] - Fk[0][l];
        Y[l] = Fk[1][l] + Fk1[1][l]; Y[l + 4] = Fk1[1][l] - Fk[1][l];
        Z[l] = Fk[2][l] + Fk1[2][l]; Z[l + 4] = Fk1[2][l] - Fk[2][l];
      }
      Material<T> mt = make_material<T, MODE>(mc);
      const T cz = F.dz[k], icz = F.idz[k];
      T FX[8], FY[8], FZ[8];
      hex8_modal<T, HAS12>(X, Y, Z, make_coef(a, b, cz, ia, ib, icz, mt), FX, FY, FZ);
      // (g, h) z back-transform: bottom share completes the face of plane k, top share carries to plane k+1
#pragma unroll
      for (int l = 0; l < 4; ++l) {
        G[0][l] = topc[0][l] + (FX[l] - FX[l + 4]); topc[0][l] = FX[l] + FX[l + 4];
        G[1][l] = topc[1][l] + (FY[l] - FY[l + 4]); topc[1][l] = FY[l] + FY[l + 4];
        G[2][l] = topc[2][l] + (FZ[l] - FZ[l + 4]); topc[2][l] = FZ[l] + FZ[l + 4];
      }
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int l = 0; l < 4; ++l) { G[c][l] = topc[c][l]; topc[c][l] = T(0); }
    }
    // (i) y back-transform of the face of plane k: lower share stays, upper share goes to the row above
    T hi[3][2];
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int ax = 0; ax < 2; ++ax) {
        plo[c][ax] = G[c][ax] - G[c][ax + 2];
        hi[c][ax] = G[c][ax] + G[c][ax + 2];
      }
    put6(sB[slot(k)][ty][tx], hi);
    // (j) advance
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int l = 0; l < 4; ++l) Fk[c][l] = Fk1[c][l];
      vn[c] = vp[c]; vp[c] = vq[c];
    }
#pragma unroll
    for (int q = 0; q < W; ++q) mc[q] = mn[q];
  }
  __syncthreads();
  {
    T up[3][2] = {};
    if (ty >= 1) get6(sB[slot(K1 - 1)][ty - 1][tx], up);
    T out[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const T m = plo[c][0] + up[c][0], d = plo[c][1] + up[c][1];
      const T left = __shfl_up_sync(0xffffffffu, m + d, 1);
      out[c] = (m - d) + (tx ? left : T(0));
    }
    if (owner && K1 - 1 >= K0) {
      T* dst = y + 3 * (nbase + plane * (K1 - 1));
      dst[0] = out[0]; dst[1] = out[1]; dst[2] = out[2];
    }
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

// A failed attribute call leaves its message in the last error and the launch then fails; the caller's
// next status check reports it.
template <typename T, int MODE, int TY>
void launch_struct(dim3 grid, size_t smem, const FineView<T>& F, const T* u, T* y, const int* skip, int zc,
                   cudaStream_t s) {
  if (set_dyn_smem((const void*)k_fine_struct<T, MODE, TY>, (int)smem) != FEB_OK) return;
  k_fine_struct<T, MODE, TY><<<grid, dim3(32, TY), smem, s>>>(F, u, y, skip, zc); note_launch();
}

template <typename T, int MODE>
void launch_fine_sparse_into(const FineView<T>& F, const T* u, T* acc, const int* skip, cudaStream_t s) {
  int b_irr = div_up(F.nirr, kThreads), b_pen = div_up(F.npen, kThreads), b_row = div_up(F.nrow, kThreads);
  if (b_irr + b_pen + b_row > 0) {
    k_fine_sparse<T, MODE><<<b_irr + b_pen + b_row, kThreads, 0, s>>>(F, u, acc, skip, b_irr, b_pen); note_launch();
  }
}

template <typename T, int MODE>
void launch_fine_apply(const FineView<T>& F, const T* u, T* y, const int* skip, KuConfig cfg, cudaStream_t s) {
  const int ty = cfg.ty == 8 ? 8 : (cfg.ty == 12 ? 12 : 16);
  const int zc = std::max(1, cfg.zchunk);
  dim3 grid(div_up(F.nxn, 30), div_up(F.nyn, ty - 2), div_up(F.nzn, zc));
  const size_t smem = sizeof(T) * (size_t)ty * 32 * 24;
  bool tc_done = false;
  if constexpr (std::is_same<T, float>::value && MODE != MAT_ORTHO) {
    if (cfg.tc) {
      launch_fine_struct_tc<MODE>(F, u, y, skip, zc, s);
      tc_done = true;
    }
  }
  if (tc_done) {
  } else if (ty == 8) {
    launch_struct<T, MODE, 8>(grid, smem, F, u, y, skip, zc, s);
  } else if (ty == 12) {
    launch_struct<T, MODE, 12>(grid, smem, F, u, y, skip, zc, s);
  } else {
    launch_struct<T, MODE, 16>(grid, smem, F, u, y, skip, zc, s);
  }
  if (F.ntotal > F.nnode) {
    int64_t n = 3 * (F.ntotal - F.nnode);
    k_zero_tail<T><<<div_up(n, kThreads), kThreads, 0, s>>>(y, 3 * F.nnode, 3 * F.ntotal, skip); note_launch();
  }
  int b_irr = div_up(F.nirr, kThreads), b_pen = div_up(F.npen, kThreads), b_row = div_up(F.nrow, kThreads);
  if (b_irr + b_pen + b_row > 0) {
    k_fine_sparse<T, MODE><<<b_irr + b_pen + b_row, kThreads, 0, s>>>(F, u, y, skip, b_irr, b_pen); note_launch();
  }
}

template <int MODE>
void launch_fine_diag(const FineView<double>& F, double* D, cudaStream_t s) {
  k_fine_diag_grid<MODE><<<div_up(F.ntotal, kThreads), kThreads, 0, s>>>(F, D); note_launch();
  int n = max(F.nirr, max(F.npen, F.nrow));
  if (n > 0) k_fine_diag_sparse<MODE><<<div_up(n, kThreads), kThreads, 0, s>>>(F, D); note_launch();
}

#define INST(T, M) template void launch_fine_apply<T, M>(const FineView<T>&, const T*, T*, const int*, KuConfig, cudaStream_t); \
  template void launch_fine_sparse_into<T, M>(const FineView<T>&, const T*, T*, const int*, cudaStream_t);
INST(float, MAT_ISO_SRI) INST(float, MAT_ISO_FULL) INST(float, MAT_ORTHO)
INST(double, MAT_ISO_SRI) INST(double, MAT_ISO_FULL) INST(double, MAT_ORTHO)
#undef INST
template void launch_fine_diag<MAT_ISO_SRI>(const FineView<double>&, double*, cudaStream_t);
template void launch_fine_diag<MAT_ISO_FULL>(const FineView<double>&, double*, cudaStream_t);
template void launch_fine_diag<MAT_ORTHO>(const FineView<double>&, double*, cudaStream_t);

}  // namespace feb
