// Coarse-level kernels: stencil products, structured restriction / prolongation, Galerkin on the device.
#include <algorithm>

#include "coarse.cuh"
#include "vec.cuh"

namespace feb {

namespace {

__device__ __forceinline__ double axis_w(const AxisDev& A, int i, int J) {
  double w = 0.0;
  if (A.ca[i] == J) w += A.wa[i];
  if (A.cb[i] == J) w += A.wb[i];
  return w;
}

// coarse support of fine node i along one axis: up to 2 (index, weight) pairs
__device__ __forceinline__ int axis_support(const AxisDev& A, int i, int (&J)[2], double (&w)[2]) {
  int n = 0;
  if (A.wa[i] != 0.0) { J[n] = A.ca[i]; w[n] = A.wa[i]; ++n; }
  if (A.cb[i] != A.ca[i] && A.wb[i] != 0.0) { J[n] = A.cb[i]; w[n] = A.wb[i]; ++n; }
  return n;
}

// fine nodes interpolating from coarse node J along one axis: up to 3 (index, weight) pairs
__device__ __forceinline__ int axis_fan(const AxisDev& A, int J, int (&I)[3], double (&w)[3]) {
  int n = 0, f = A.cidx[J];
  for (int i = f - 1; i <= f + 1; ++i) {
    if (i < 0 || i >= A.nf) continue;
    double x = axis_w(A, i, J);
    if (x != 0.0) { I[n] = i; w[n] = x; ++n; }
  }
  return n;
}

template <typename T>
__global__ void __launch_bounds__(kThreads)
k_stencil_apply(StencilView<T> L, const T* __restrict__ u, T* __restrict__ y, const int* __restrict__ skip) {
  if (skip && *skip) return;
  int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= L.n) return;
  int i = int(n % L.nx), j = int((n / L.nx) % L.ny), k = int(n / ((int64_t)L.nx * L.ny));
  T acc0 = 0, acc1 = 0, acc2 = 0;
#pragma unroll
  for (int o = 0; o < 27; ++o) {
    const int dx = o % 3 - 1, dy = (o / 3) % 3 - 1, dz = o / 9 - 1;
    const int ii = i + dx, jj = j + dy, kk = k + dz;
    if (ii < 0 || jj < 0 || kk < 0 || ii >= L.nx || jj >= L.ny || kk >= L.nz) continue;
    const int64_t m = n + dx + (int64_t)L.nx * (dy + (int64_t)L.ny * dz);
    const T u0 = u[3 * m], u1 = u[3 * m + 1], u2 = u[3 * m + 2];
    const T* a = L.A + (size_t)(o * 9) * L.n + n;
    acc0 += a[0] * u0 + a[L.n] * u1 + a[2 * L.n] * u2;
    acc1 += a[3 * L.n] * u0 + a[4 * L.n] * u1 + a[5 * L.n] * u2;
    acc2 += a[6 * L.n] * u0 + a[7 * L.n] * u1 + a[8 * L.n] * u2;
  }
  y[3 * n] = acc0; y[3 * n + 1] = acc1; y[3 * n + 2] = acc2;
}

template <typename T>
__global__ void k_csr_add(int nrow, const int* __restrict__ row_dof, const int* __restrict__ row_ptr,
                          const int* __restrict__ col, const T* __restrict__ val, const T* __restrict__ u,
                          T* __restrict__ y, const int* __restrict__ skip) {
  if (skip && *skip) return;
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nrow) return;
  T s = 0;
  for (int q = row_ptr[e]; q < row_ptr[e + 1]; ++q) s += val[q] * u[col[q]];
  atomic_add(y + row_dof[e], s);
}

template <typename T>
__global__ void k_restrict_grid(TransferDev P, int fnx, int fny, const T* __restrict__ rf, T* __restrict__ rc,
                                const int* __restrict__ skip, T* __restrict__ zero, int nzero) {
  if (skip && *skip) return;
  if (nzero && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0)
    for (int e = threadIdx.x; e < nzero; e += blockDim.x) zero[e] = T(0);
  const int cnx = P.ax[0].nc, cny = P.ax[1].nc;
  const int jx = blockIdx.x * blockDim.x + threadIdx.x, jy = blockIdx.y, jz = blockIdx.z;
  if (jx >= cnx) return;
  const int64_t J = jx + (int64_t)cnx * (jy + (int64_t)cny * jz);
  int Ix[3], Iy[3], Iz[3];
  double wx[3], wy[3], wz[3];
  int nxs = axis_fan(P.ax[0], jx, Ix, wx), nys = axis_fan(P.ax[1], jy, Iy, wy), nzs = axis_fan(P.ax[2], jz, Iz, wz);
  T s0 = 0, s1 = 0, s2 = 0;
  for (int c = 0; c < nzs; ++c)
    for (int b = 0; b < nys; ++b)
      for (int a = 0; a < nxs; ++a) {
        int64_t f = Ix[a] + (int64_t)fnx * (Iy[b] + (int64_t)fny * Iz[c]);
        T w = T(wx[a] * wy[b] * wz[c]);
        s0 += w * rf[3 * f]; s1 += w * rf[3 * f + 1]; s2 += w * rf[3 * f + 2];
      }
  rc[3 * J] = s0; rc[3 * J + 1] = s1; rc[3 * J + 2] = s2;
}

// r_c = P^T r_f for even coarsening: coarse node J gathers fine nodes 2 J + a, a in {-1, 0, 1} per axis, with
// weight 1 (a = 0) or 1/2 (a = +-1)
template <typename T>
__global__ void k_restrict_even(int cnx, int cny, int fnx, int fny, int fnz, const T* __restrict__ rf,
                                T* __restrict__ rc, const int* __restrict__ skip, T* __restrict__ zero, int nzero,
                                const int* __restrict__ cp_ptr, const int* __restrict__ cp_copy,
                                const double* __restrict__ cp_w, int64_t fnnode) {
  if (skip && *skip) return;
  if (nzero && blockIdx.x == 0 && blockIdx.y == 0 && blockIdx.z == 0)
    for (int e = threadIdx.x; e < nzero; e += blockDim.x) zero[e] = T(0);
  const int jx = blockIdx.x * blockDim.x + threadIdx.x, jy = blockIdx.y, jz = blockIdx.z;
  if (jx >= cnx) return;
  T s0 = 0, s1 = 0, s2 = 0;
#pragma unroll
  for (int c = -1; c <= 1; ++c) {
    const int fk = 2 * jz + c;
    if (fk < 0 || fk >= fnz) continue;
#pragma unroll
    for (int b = -1; b <= 1; ++b) {
      const int fj = 2 * jy + b;
      if (fj < 0 || fj >= fny) continue;
#pragma unroll
      for (int a = -1; a <= 1; ++a) {
        const int fi = 2 * jx + a;
        if (fi < 0 || fi >= fnx) continue;
        const T w = T((a ? 0.5 : 1.0) * (b ? 0.5 : 1.0) * (c ? 0.5 : 1.0));
        const int64_t f = fi + (int64_t)fnx * (fj + (int64_t)fny * fk);
        s0 += w * rf[3 * f]; s1 += w * rf[3 * f + 1]; s2 += w * rf[3 * f + 2];
      }
    }
  }
  const int64_t J = jx + (int64_t)cnx * (jy + (int64_t)cny * jz);
  if (cp_ptr) {   // split copies restricting into J, in ascending copy order
    for (int e = cp_ptr[J]; e < cp_ptr[J + 1]; ++e) {
      const int64_t f = fnnode + cp_copy[e];
      const T w = T(cp_w[e]);
      s0 += w * rf[3 * f]; s1 += w * rf[3 * f + 1]; s2 += w * rf[3 * f + 2];
    }
  }
  rc[3 * J] = s0; rc[3 * J + 1] = s1; rc[3 * J + 2] = s2;
}

// x_f += P x_c on used fine nodes for even coarsening: per axis an even fine node takes its coarse node, an odd
// one the mean of its two neighbours
// even coarsening: the interpolated coarse value at fine grid position (pi, pj, pk)
template <typename T>
__device__ __forceinline__ void even_interp(int cnx, int cny, int pi, int pj, int pk, const T* __restrict__ xc,
                                            T& s0, T& s1, T& s2) {
  const int ni = (pi & 1) + 1, nj = (pj & 1) + 1, nk = (pk & 1) + 1;
  const T wi = T(ni == 2 ? 0.5 : 1.0), wj = T(nj == 2 ? 0.5 : 1.0), wk = T(nk == 2 ? 0.5 : 1.0);
  s0 = 0; s1 = 0; s2 = 0;
  for (int c = 0; c < nk; ++c)
    for (int b = 0; b < nj; ++b)
      for (int a = 0; a < ni; ++a) {
        const int64_t K = (pi >> 1) + a + (int64_t)cnx * ((pj >> 1) + b + (int64_t)cny * ((pk >> 1) + c));
        const T w = wi * wj * wk;
        s0 += w * xc[3 * K]; s1 += w * xc[3 * K + 1]; s2 += w * xc[3 * K + 2];
      }
}

// x_f += P x_c for even coarsening; grid (x blocks of 64, fny, fnz + extra): the z layers past fnz take the
// split copies (ids fnnode .. fnnode + ncopy), which receive their grid position's value
template <typename T>
__global__ void k_prolong_even(int cnx, int cny, int fnx, int fny, int fnz, const uint8_t* __restrict__ used,
                               const T* __restrict__ xc, T* __restrict__ xf, const int* __restrict__ skip,
                               TermAcc<T> acc, int64_t fnnode, int64_t ncopy, const int* __restrict__ orig_copy) {
  if (skip && *skip) return;
  if ((int)blockIdx.z >= fnz) {
    const int64_t c = ((int64_t)(blockIdx.z - fnz) * gridDim.y + blockIdx.y) * ((int64_t)gridDim.x * blockDim.x) +
                      blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (c >= ncopy) return;
    const int o = orig_copy[c];
    const int pi = o % fnx, pj = (o / fnx) % fny, pk = o / (fnx * fny);
    T s0, s1, s2;
    even_interp(cnx, cny, pi, pj, pk, xc, s0, s1, s2);
    const int64_t n = fnnode + c;
    xf[3 * n] += s0; xf[3 * n + 1] += s1; xf[3 * n + 2] += s2;
    return;
  }
  const int pi = blockIdx.x * blockDim.x + threadIdx.x, pj = blockIdx.y, pk = blockIdx.z;
  if (pi >= fnx) return;
  const int64_t n = pi + (int64_t)fnx * (pj + (int64_t)fny * pk);
  if (!used[n]) return;
  T s0, s1, s2;
  even_interp(cnx, cny, pi, pj, pk, xc, s0, s1, s2);
  xf[3 * n] += s0; xf[3 * n + 1] += s1; xf[3 * n + 2] += s2;
  term_acc(acc, n, s0, s1, s2);
}

template <typename T>
__global__ void k_restrict_copies(TransferDev P, int fnx, int fny, int64_t fnnode, int64_t fntotal,
                                  const int* __restrict__ orig_copy, const T* __restrict__ rf, T* __restrict__ rc,
                                  const int* __restrict__ skip) {
  if (skip && *skip) return;
  int64_t e = fnnode + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= fntotal) return;
  const int o = orig_copy[e - fnnode];
  const int pi = o % fnx, pj = (o / fnx) % fny, pk = o / (fnx * fny);
  int Jx[2], Jy[2], Jz[2];
  double wx[2], wy[2], wz[2];
  int nxs = axis_support(P.ax[0], pi, Jx, wx), nys = axis_support(P.ax[1], pj, Jy, wy),
      nzs = axis_support(P.ax[2], pk, Jz, wz);
  const int cnx = P.ax[0].nc, cny = P.ax[1].nc;
  for (int c = 0; c < nzs; ++c)
    for (int b = 0; b < nys; ++b)
      for (int a = 0; a < nxs; ++a) {
        int64_t K = Jx[a] + (int64_t)cnx * (Jy[b] + (int64_t)cny * Jz[c]);
        T w = T(wx[a] * wy[b] * wz[c]);
        for (int q = 0; q < 3; ++q) atomic_add(rc + 3 * K + q, w * rf[3 * e + q]);
      }
}

template <typename T>
__device__ __forceinline__ void prolong_at(const TransferDev& P, int pi, int pj, int pk, const T* __restrict__ xc,
                                           T& s0, T& s1, T& s2) {
  int Jx[2], Jy[2], Jz[2];
  double wx[2], wy[2], wz[2];
  int nxs = axis_support(P.ax[0], pi, Jx, wx), nys = axis_support(P.ax[1], pj, Jy, wy),
      nzs = axis_support(P.ax[2], pk, Jz, wz);
  const int cnx = P.ax[0].nc, cny = P.ax[1].nc;
  s0 = s1 = s2 = T(0);
  for (int c = 0; c < nzs; ++c)
    for (int b = 0; b < nys; ++b)
      for (int a = 0; a < nxs; ++a) {
        int64_t K = Jx[a] + (int64_t)cnx * (Jy[b] + (int64_t)cny * Jz[c]);
        T w = T(wx[a] * wy[b] * wz[c]);
        s0 += w * xc[3 * K]; s1 += w * xc[3 * K + 1]; s2 += w * xc[3 * K + 2];
      }
}

template <typename T>
__global__ void k_prolong_grid(TransferDev P, int fnx, int fny, const uint8_t* __restrict__ used,
                               const T* __restrict__ xc, T* __restrict__ xf, const int* __restrict__ skip,
                               TermAcc<T> acc) {
  if (skip && *skip) return;
  const int pi = blockIdx.x * blockDim.x + threadIdx.x, pj = blockIdx.y, pk = blockIdx.z;
  if (pi >= fnx) return;
  const int64_t n = pi + (int64_t)fnx * (pj + (int64_t)fny * pk);
  if (!used[n]) return;
  T s0, s1, s2;
  prolong_at(P, pi, pj, pk, xc, s0, s1, s2);
  xf[3 * n] += s0; xf[3 * n + 1] += s1; xf[3 * n + 2] += s2;
  term_acc(acc, n, s0, s1, s2);
}

template <typename T>
__global__ void k_prolong_copies(TransferDev P, int fnx, int fny, int64_t fnnode, int64_t fntotal,
                                 const int* __restrict__ orig_copy, const T* __restrict__ xc, T* __restrict__ xf,
                                 const int* __restrict__ skip) {
  if (skip && *skip) return;
  int64_t n = fnnode + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= fntotal) return;
  const int o = orig_copy[n - fnnode];
  const int pi = o % fnx, pj = (o / fnx) % fny, pk = o / (fnx * fny);
  T s0, s1, s2;
  prolong_at(P, pi, pj, pk, xc, s0, s1, s2);
  xf[3 * n] += s0; xf[3 * n + 1] += s1; xf[3 * n + 2] += s2;
}

__global__ void k_kept_mask(TransferDev P, const uint8_t* __restrict__ used_f, uint8_t* __restrict__ kept_c) {
  const int cnx = P.ax[0].nc, cny = P.ax[1].nc, cnz = P.ax[2].nc;
  const int fnx = P.ax[0].nf, fny = P.ax[1].nf;
  int64_t J = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (J >= (int64_t)cnx * cny * cnz) return;
  int jx = int(J % cnx), jy = int((J / cnx) % cny), jz = int(J / ((int64_t)cnx * cny));
  int Ix[3], Iy[3], Iz[3];
  double wx[3], wy[3], wz[3];
  int nxs = axis_fan(P.ax[0], jx, Ix, wx), nys = axis_fan(P.ax[1], jy, Iy, wy), nzs = axis_fan(P.ax[2], jz, Iz, wz);
  uint8_t k = 0;
  for (int c = 0; c < nzs && !k; ++c)
    for (int b = 0; b < nys && !k; ++b)
      for (int a = 0; a < nxs && !k; ++a) k = used_f[Ix[a] + (int64_t)fnx * (Iy[b] + (int64_t)fny * Iz[c])];
  kept_c[J] = k ? 1 : 0;
}

// Column q = (corner a, component s) of the coarse-cell matrix sum_{fine cells} P_c^T K_c P_c, obtained by
// applying the fine element operator to the prolonged unit vector and restricting the result.
template <int MODE>
__global__ void __launch_bounds__(192)
k_galerkin_cells(FineView<double> F, const double* __restrict__ mat_all, TransferDev P, double* __restrict__ KeC,
                 int ncx, int ncy, int ncz) {
  constexpr int W = MatWidth<MODE>::value;
  const int q = threadIdx.x;                     // 0..23
  const int64_t C = blockIdx.x * (int64_t)blockDim.y + threadIdx.y;
  if (C >= (int64_t)ncx * ncy * ncz) return;
  const int CI = int(C % ncx), CJ = int((C / ncx) % ncy), CK = int(C / ((int64_t)ncx * ncy));
  const int a = q / 3, s = q % 3;
  const int ax = a & 1, ay = (a >> 1) & 1, az = (a >> 2) & 1;
  double acc[24];
#pragma unroll
  for (int t = 0; t < 24; ++t) acc[t] = 0.0;
  const AxisDev &X = P.ax[0], &Y = P.ax[1], &Z = P.ax[2];
  for (int fk = Z.iv_first[CK]; fk < Z.iv_first[CK] + Z.iv_count[CK]; ++fk)
    for (int fj = Y.iv_first[CJ]; fj < Y.iv_first[CJ] + Y.iv_count[CJ]; ++fj)
      for (int fi = X.iv_first[CI]; fi < X.iv_first[CI] + X.iv_count[CI]; ++fi) {
        const double* p = mat_all + (size_t)W * (fi + (int64_t)F.nx * (fj + (int64_t)F.ny * fk));
        double m[W];
        bool nz = false;
#pragma unroll
        for (int t = 0; t < W; ++t) { m[t] = p[t]; nz |= (m[t] != 0.0); }
        if (!nz) continue;
        // weights of the fine corners (2 per axis) toward the coarse corners (2 per axis)
        double wxt[2][2], wyt[2][2], wzt[2][2];
#pragma unroll
        for (int f = 0; f < 2; ++f)
#pragma unroll
          for (int c = 0; c < 2; ++c) {
            wxt[f][c] = axis_w(X, fi + f, CI + c);
            wyt[f][c] = axis_w(Y, fj + f, CJ + c);
            wzt[f][c] = axis_w(Z, fk + f, CK + c);
          }
        double u[3][8], f[3][8];
#pragma unroll
        for (int l = 0; l < 8; ++l) {
          double v = wxt[l & 1][ax] * wyt[(l >> 1) & 1][ay] * wzt[(l >> 2) & 1][az];
          u[0][l] = s == 0 ? v : 0.0;
          u[1][l] = s == 1 ? v : 0.0;
          u[2][l] = s == 2 ? v : 0.0;
        }
        Material<double> mt = make_material<double, MODE>(m);
        hex8_apply(u, F.dx[fi], F.dy[fj], F.dz[fk], F.idx[fi], F.idy[fj], F.idz[fk], mt, f);
#pragma unroll
        for (int b = 0; b < 8; ++b) {
#pragma unroll
          for (int l = 0; l < 8; ++l) {
            double w = wxt[l & 1][b & 1] * wyt[(l >> 1) & 1][(b >> 1) & 1] * wzt[(l >> 2) & 1][(b >> 2) & 1];
#pragma unroll
            for (int r = 0; r < 3; ++r) acc[3 * b + r] += w * f[r][l];
          }
        }
      }
  double* dst = KeC + (size_t)C * 576 + q;
#pragma unroll
  for (int t = 0; t < 24; ++t) dst[24 * t] = acc[t];
}

// Node stencil of level 1 from the coarse-cell matrices: A1[J][o] = sum over coarse cells holding J and J+o.
__global__ void k_cells_to_stencil(const double* __restrict__ KeC, double* __restrict__ A, int cnx, int cny, int cnz) {
  const int o = threadIdx.x;          // 0..26
  const int64_t n = (int64_t)cnx * cny * cnz;
  const int64_t J = blockIdx.x * (int64_t)blockDim.y + threadIdx.y;
  if (J >= n) return;
  const int jx = int(J % cnx), jy = int((J / cnx) % cny), jz = int(J / ((int64_t)cnx * cny));
  const int od[3] = {o % 3 - 1, (o / 3) % 3 - 1, o / 9 - 1};
  const int jc[3] = {jx, jy, jz}, nn[3] = {cnx, cny, cnz};
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  int I[3][2], aJ[3][2], aK[3][2], cnt[3];
  bool ok = true;
  for (int d = 0; d < 3; ++d) {
    cnt[d] = 0;
    int K = jc[d] + od[d];
    if (K < 0 || K >= nn[d]) { ok = false; break; }
    for (int iv = jc[d] - 1; iv <= jc[d]; ++iv) {
      if (iv < 0 || iv >= nn[d] - 1) continue;
      if (K < iv || K > iv + 1) continue;
      I[d][cnt[d]] = iv; aJ[d][cnt[d]] = jc[d] - iv; aK[d][cnt[d]] = K - iv; ++cnt[d];
    }
  }
  if (ok) {
    for (int c = 0; c < cnt[2]; ++c)
      for (int b = 0; b < cnt[1]; ++b)
        for (int a = 0; a < cnt[0]; ++a) {
          int64_t C = I[0][a] + (int64_t)(cnx - 1) * (I[1][b] + (int64_t)(cny - 1) * I[2][c]);
          int la = aJ[0][a] + 2 * aJ[1][b] + 4 * aJ[2][c];
          int lb = aK[0][a] + 2 * aK[1][b] + 4 * aK[2][c];
          const double* src = KeC + (size_t)C * 576;
          for (int r = 0; r < 3; ++r)
            for (int q = 0; q < 3; ++q) acc[3 * r + q] += src[(3 * la + r) * 24 + 3 * lb + q];
        }
  }
  for (int t = 0; t < 9; ++t) A[(size_t)(o * 9 + t) * n + J] = acc[t];
}

// Galerkin basis of a coarse cell on a uniform fine grid with even cell counts: every coarse cell holds 2 x 2 x 2
// fine cells of equal widths (a, b, c), and its prolongation weights are the same (1, 1/2, 0 per axis).  Hence
// P_f^T K_f P_f of the fine cell at sub-position f is lam_f BL[f] + mu_f BM[f] with 16 constant 24 x 24
// matrices (isotropic models), computed here once: out[(2 f + m) * 576 + 24 row + col], m = 0 (lam), 1 (mu).
template <int MODE>
__global__ void k_galerkin_basis(double a, double b, double c, double* __restrict__ out) {
  const int f = blockIdx.x >> 1, m = blockIdx.x & 1;   // sub-position, material part
  const int q = threadIdx.x;                              // column: coarse corner q / 3, component q % 3
  if (q >= 24) return;
  const int fx = f & 1, fy = (f >> 1) & 1, fz = (f >> 2) & 1;
  const int ca = q / 3, s = q % 3;
  auto w = [](int p, int corner) { return p == 1 ? 0.5 : ((p == 0) == (corner == 0) ? 1.0 : 0.0); };
  double u[3][8], fo[3][8];
  for (int l = 0; l < 8; ++l) {
    const double v = w(fx + (l & 1), ca & 1) * w(fy + ((l >> 1) & 1), (ca >> 1) & 1) * w(fz + ((l >> 2) & 1), (ca >> 2) & 1);
    for (int r = 0; r < 3; ++r) u[r][l] = (r == s) ? v : 0.0;
  }
  double mat[2] = {m == 0 ? 1.0 : 0.0, m == 1 ? 1.0 : 0.0};
  Material<double> mt = make_material<double, MODE>(mat);
  hex8_apply(u, a, b, c, 1.0 / a, 1.0 / b, 1.0 / c, mt, fo);
  for (int cb = 0; cb < 8; ++cb)
    for (int r = 0; r < 3; ++r) {
      double acc = 0.0;
      for (int l = 0; l < 8; ++l)
        acc += w(fx + (l & 1), cb & 1) * w(fy + ((l >> 1) & 1), (cb >> 1) & 1) * w(fz + ((l >> 2) & 1), (cb >> 2) & 1) *
               fo[r][l];
      out[(size_t)blockIdx.x * 576 + (3 * cb + r) * 24 + q] = acc;
    }
}

// Level-1 stencil A1[J][o] (27 blocks of 3 x 3) summed directly over the coarse cells holding J and J + o and
// their 8 fine cells: sum_C sum_f lam_f BL[f][la][lb] + mu_f BM[f][la][lb] (same sums as k_galerkin_cells +
// k_cells_to_stencil, without the 576-value coarse-cell matrices in memory).
__global__ void __launch_bounds__(27 * 8)
k_galerkin_direct(const double* __restrict__ mat_all, int fnx, int fny, const double* __restrict__ basis,
                  double* __restrict__ A, int cnx, int cny, int cnz) {
  extern __shared__ double sbasis[];   // 16 x 576
  for (int t = threadIdx.y * 27 + threadIdx.x; t < 16 * 576; t += 27 * 8) sbasis[t] = basis[t];
  __syncthreads();
  const int o = threadIdx.x;
  const int64_t n = (int64_t)cnx * cny * cnz;
  const int64_t J = blockIdx.x * (int64_t)8 + threadIdx.y;
  if (J >= n) return;
  const int jx = int(J % cnx), jy = int((J / cnx) % cny), jz = int(J / ((int64_t)cnx * cny));
  const int od[3] = {o % 3 - 1, (o / 3) % 3 - 1, o / 9 - 1};
  const int jc[3] = {jx, jy, jz}, nn[3] = {cnx, cny, cnz};
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  int I[3][2], aJ[3][2], aK[3][2], cnt[3];
  bool ok = true;
  for (int d = 0; d < 3; ++d) {
    cnt[d] = 0;
    const int K = jc[d] + od[d];
    if (K < 0 || K >= nn[d]) { ok = false; break; }
    for (int iv = jc[d] - 1; iv <= jc[d]; ++iv) {
      if (iv < 0 || iv >= nn[d] - 1) continue;
      if (K < iv || K > iv + 1) continue;
      I[d][cnt[d]] = iv; aJ[d][cnt[d]] = jc[d] - iv; aK[d][cnt[d]] = K - iv; ++cnt[d];
    }
  }
  if (ok) {
    for (int cz = 0; cz < cnt[2]; ++cz)
      for (int cy = 0; cy < cnt[1]; ++cy)
        for (int cx = 0; cx < cnt[0]; ++cx) {
          const int la = aJ[0][cx] + 2 * aJ[1][cy] + 4 * aJ[2][cz];
          const int lb = aK[0][cx] + 2 * aK[1][cy] + 4 * aK[2][cz];
          for (int f = 0; f < 8; ++f) {
            const int fi = 2 * I[0][cx] + (f & 1), fj = 2 * I[1][cy] + ((f >> 1) & 1), fk = 2 * I[2][cz] + ((f >> 2) & 1);
            const double* p = mat_all + 2 * (fi + (int64_t)fnx * (fj + (int64_t)fny * fk));
            const double lam = p[0], mu = p[1];
            if (lam == 0.0 && mu == 0.0) continue;
            const double* BL = sbasis + (2 * f) * 576 + (3 * la) * 24 + 3 * lb;
            const double* BM = BL + 576;
#pragma unroll
            for (int r = 0; r < 3; ++r)
#pragma unroll
              for (int qq = 0; qq < 3; ++qq) acc[3 * r + qq] += lam * BL[24 * r + qq] + mu * BM[24 * r + qq];
          }
        }
  }
  for (int t = 0; t < 9; ++t) A[(size_t)(o * 9 + t) * n + J] = acc[t];
}

// Interior patterns: for the offsets o = 13..26 the blocks summed over the coarse cells holding J and J + o and
// all 8 fine cells of each (one thread per (m, o, entry)).
__global__ void k_sym_pattern(const double* __restrict__ basis, double* __restrict__ pat) {
  const int t = threadIdx.x;   // 0..251
  if (t >= 252) return;
  const int m = t / 126, e = t % 126, q = e / 9, rc = e % 9, r = rc / 3, cc = rc % 3;
  const int o = 13 + q;
  const int od[3] = {o % 3 - 1, (o / 3) % 3 - 1, o / 9 - 1};
  int la_ax[3][2], lb_ax[3][2], cnt[3];
  for (int d = 0; d < 3; ++d) {
    cnt[d] = 0;
    for (int iv = -1; iv <= 0; ++iv) {   // cells [jc + iv, jc + iv + 1] holding jc and jc + od
      const int la = -iv, lb = od[d] - iv;
      if (lb < 0 || lb > 1) continue;
      la_ax[d][cnt[d]] = la; lb_ax[d][cnt[d]] = lb; ++cnt[d];
    }
  }
  double acc = 0.0;
  for (int cz = 0; cz < cnt[2]; ++cz)
    for (int cy = 0; cy < cnt[1]; ++cy)
      for (int cx = 0; cx < cnt[0]; ++cx) {
        const int la = la_ax[0][cx] + 2 * la_ax[1][cy] + 4 * la_ax[2][cz];
        const int lb = lb_ax[0][cx] + 2 * lb_ax[1][cy] + 4 * lb_ax[2][cz];
        for (int f = 0; f < 8; ++f) acc += basis[(2 * f + m) * 576 + (3 * la + r) * 24 + 3 * lb + cc];
      }
  pat[t] = acc;
}

__global__ void k_sym_tags(const double* __restrict__ S64, int cnx, int cny, int cnz,
                           const uint16_t* __restrict__ cellpair, int fnxn, int mp, const double* __restrict__ mtab,
                           const double* __restrict__ pat, uint8_t* __restrict__ tag) {
  const int64_t n = (int64_t)cnx * cny * cnz;
  const int64_t J = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (J >= n) return;
  const int jx = int(J % cnx), jy = int((J / cnx) % cny), jz = int(J / ((int64_t)cnx * cny));
  const int64_t np = sym_np(cnx, cny, cnz), P = jx + (int64_t)sym_nxp(cnx) * (jy + (int64_t)cny * jz);
  // fine cell (2 jx, 2 jy, 2 jz): row 2 jy is the upper byte of row pair m = jy
  uint32_t id = 0;
  if (jy < mp) id = (cellpair[2 * jx + (int64_t)fnxn * (jy + (int64_t)mp * (2 * jz))] >> 8) & 0x7fu;
  uint8_t t = 0;
  if (id > 0) {
    const double lam = mtab[2 * id], mu = mtab[2 * id + 1];
    double scale = 0.0;
    for (int e = 0; e < 126; ++e) scale = fmax(scale, fabs(lam * pat[e]) + fabs(mu * pat[126 + e]));
    bool same = scale > 0.0;
    for (int e = 0; e < 126 && same; ++e)
      same = fabs(S64[(size_t)e * np + P] - (lam * pat[e] + mu * pat[126 + e])) <= 1e-12 * scale;
    t = same ? (uint8_t)id : 0;
  }
  tag[J] = t;
}

__device__ __forceinline__ int64_t grid_pos(int64_t node, int64_t fnnode, const int* orig_copy) {
  return node < fnnode ? node : (int64_t)orig_copy[node - fnnode];
}

__global__ void k_galerkin_penalty(TransferDev P, int fnx, int fny, int64_t fnnode, const int* __restrict__ orig_copy,
                                   int npen, const int* __restrict__ pen_node, const double* __restrict__ pen_k,
                                   double* __restrict__ A, int cnx, int cny, int64_t cn) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= npen) return;
  int64_t o = grid_pos(pen_node[e], fnnode, orig_copy);
  int p[3] = {int(o % fnx), int((o / fnx) % fny), int(o / ((int64_t)fnx * fny))};
  int J[3][2], ns[3];
  double w[3][2];
  for (int d = 0; d < 3; ++d) ns[d] = axis_support(P.ax[d], p[d], J[d], w[d]);
  for (int c1 = 0; c1 < ns[2]; ++c1) for (int b1 = 0; b1 < ns[1]; ++b1) for (int a1 = 0; a1 < ns[0]; ++a1) {
    int64_t Jn = J[0][a1] + (int64_t)cnx * (J[1][b1] + (int64_t)cny * J[2][c1]);
    double wJ = w[0][a1] * w[1][b1] * w[2][c1];
    for (int c2 = 0; c2 < ns[2]; ++c2) for (int b2 = 0; b2 < ns[1]; ++b2) for (int a2 = 0; a2 < ns[0]; ++a2) {
      int oo = (J[0][a2] - J[0][a1] + 1) + 3 * (J[1][b2] - J[1][b1] + 1) + 9 * (J[2][c2] - J[2][c1] + 1);
      double wK = w[0][a2] * w[1][b2] * w[2][c2];
      for (int c = 0; c < 3; ++c) atomicAdd(A + (size_t)(oo * 9 + 4 * c) * cn + Jn, wJ * wK * pen_k[3 * e + c]);
    }
  }
}

__global__ void k_galerkin_local(TransferDev P, int fnx, int fny, int64_t fnnode, const int* __restrict__ orig_copy,
                                 int nent, const int* __restrict__ rdof, const int* __restrict__ cdof,
                                 const double* __restrict__ val, double* __restrict__ A, int cnx, int cny, int64_t cn) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nent) return;
  int64_t orow = grid_pos(rdof[e] / 3, fnnode, orig_copy), ocol = grid_pos(cdof[e] / 3, fnnode, orig_copy);
  int r = rdof[e] % 3, c = cdof[e] % 3;
  int pr[3] = {int(orow % fnx), int((orow / fnx) % fny), int(orow / ((int64_t)fnx * fny))};
  int pc[3] = {int(ocol % fnx), int((ocol / fnx) % fny), int(ocol / ((int64_t)fnx * fny))};
  int Jr[3][2], Jc[3][2], nr[3], nc[3];
  double wr[3][2], wc[3][2];
  for (int d = 0; d < 3; ++d) {
    nr[d] = axis_support(P.ax[d], pr[d], Jr[d], wr[d]);
    nc[d] = axis_support(P.ax[d], pc[d], Jc[d], wc[d]);
  }
  for (int c1 = 0; c1 < nr[2]; ++c1) for (int b1 = 0; b1 < nr[1]; ++b1) for (int a1 = 0; a1 < nr[0]; ++a1) {
    int64_t Jn = Jr[0][a1] + (int64_t)cnx * (Jr[1][b1] + (int64_t)cny * Jr[2][c1]);
    double wJ = wr[0][a1] * wr[1][b1] * wr[2][c1];
    for (int c2 = 0; c2 < nc[2]; ++c2) for (int b2 = 0; b2 < nc[1]; ++b2) for (int a2 = 0; a2 < nc[0]; ++a2) {
      int dx = Jc[0][a2] - Jr[0][a1], dy = Jc[1][b2] - Jr[1][b1], dz = Jc[2][c2] - Jr[2][c1];
      if (dx < -1 || dx > 1 || dy < -1 || dy > 1 || dz < -1 || dz > 1) continue;   // not local: excluded on the host
      int oo = (dx + 1) + 3 * (dy + 1) + 9 * (dz + 1);
      double wK = wc[0][a2] * wc[1][b2] * wc[2][c2];
      atomicAdd(A + (size_t)(oo * 9 + 3 * r + c) * cn + Jn, wJ * wK * val[e]);
    }
  }
}

// One axis of the Galerkin product P^T A P of a 27-point 3x3-block stencil.  P = Px (x) Py (x) Pz (x) I3 is
// separable, so the product is three passes, each coarsening one axis d: the output grid is the input grid
// with axis d coarsened and the stencil stays 27-point (coarse nodes J, J' couple only through fine nodes
// at most one apart).  Thread per output node (x fastest, coalesced), block row per offset.
__global__ void __launch_bounds__(128)
k_galerkin_axis(AxisDev ax, int d, const double* __restrict__ Ain, int inx, int iny, int inz,
                double* __restrict__ Aout, int onx, int ony, int onz) {
  const int o = blockIdx.y;
  const int64_t no = (int64_t)onx * ony * onz, ni = (int64_t)inx * iny * inz;
  const int64_t J = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (J >= no) return;
  const int jc[3] = {int(J % onx), int((J / onx) % ony), int(J / ((int64_t)onx * ony))};
  const int od[3] = {o % 3 - 1, (o / 3) % 3 - 1, o / 9 - 1};
  const int on[3] = {onx, ony, onz};
  double acc[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  bool ok = true;
  for (int e = 0; e < 3; ++e) {
    const int K = jc[e] + od[e];
    if (K < 0 || K >= on[e]) ok = false;
  }
  if (ok) {
    int I[3];
    double w[3];
    const int nI = axis_fan(ax, jc[d], I, w);
    const int K = jc[d] + od[d];
    for (int a = 0; a < nI; ++a)
      for (int dd = -1; dd <= 1; ++dd) {
        const int i2 = I[a] + dd;
        if (i2 < 0 || i2 >= ax.nf) continue;
        const double w2 = axis_w(ax, i2, K);
        if (w2 == 0.0) continue;
        int p[3] = {jc[0], jc[1], jc[2]}, q[3] = {od[0], od[1], od[2]};
        p[d] = I[a];
        q[d] = dd;
        const int64_t f = p[0] + (int64_t)inx * (p[1] + (int64_t)iny * p[2]);
        const int oi = (q[0] + 1) + 3 * (q[1] + 1) + 9 * (q[2] + 1);
        const double ww = w[a] * w2;
        const double* src = Ain + (size_t)(oi * 9) * ni + f;
#pragma unroll
        for (int t = 0; t < 9; ++t) acc[t] += ww * src[(size_t)t * ni];
      }
  }
#pragma unroll
  for (int t = 0; t < 9; ++t) Aout[(size_t)(o * 9 + t) * no + J] = acc[t];
}

__global__ void k_stencil_diag(const double* __restrict__ A, int64_t n, double* __restrict__ D) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  for (int t = 0; t < 9; ++t) D[9 * i + t] = A[(size_t)(13 * 9 + t) * n + i];
}

__global__ void k_add_diag_entries(int nent, const int* __restrict__ rdof, const int* __restrict__ cdof,
                                   const double* __restrict__ val, double* __restrict__ D) {
  int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nent) return;
  int64_t n = rdof[e] / 3;
  atomicAdd(D + 9 * n + 3 * (rdof[e] % 3) + cdof[e] % 3, val[e]);
}

__global__ void k_block_inverse(const double* __restrict__ D, int64_t n, double* __restrict__ Di64,
                                float* __restrict__ Di32) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  double a[9];
  for (int t = 0; t < 9; ++t) a[t] = D[9 * i + t];
  double c00 = a[4] * a[8] - a[5] * a[7], c01 = a[5] * a[6] - a[3] * a[8], c02 = a[3] * a[7] - a[4] * a[6];
  double det = a[0] * c00 + a[1] * c01 + a[2] * c02;
  double inv[9];
  if (fabs(det) < 1e-30) {
    for (int t = 0; t < 9; ++t) inv[t] = (t % 4 == 0) ? 1.0 : 0.0;
  } else {
    double id = 1.0 / det;
    inv[0] = c00 * id;
    inv[1] = (a[2] * a[7] - a[1] * a[8]) * id;
    inv[2] = (a[1] * a[5] - a[2] * a[4]) * id;
    inv[3] = c01 * id;
    inv[4] = (a[0] * a[8] - a[2] * a[6]) * id;
    inv[5] = (a[2] * a[3] - a[0] * a[5]) * id;
    inv[6] = c02 * id;
    inv[7] = (a[1] * a[6] - a[0] * a[7]) * id;
    inv[8] = (a[0] * a[4] - a[1] * a[3]) * id;
  }
  for (int t = 0; t < 9; ++t) {
    Di64[(size_t)t * n + i] = inv[t];
    if (Di32) Di32[(size_t)t * n + i] = float(inv[t]);
  }
}

// one thread per padded position p; padding positions (i >= nx) are written zero
template <typename T>
__global__ void k_stencil_to_sym(const double* __restrict__ A, int nx, int nxp, int64_t n, int64_t np,
                                 T* __restrict__ S) {
  const int64_t p = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (p >= np) return;
  const int64_t row = p / nxp;
  const int i = int(p - row * nxp);
  const int64_t m = row * nx + i;
  for (int q = 0; q < 14; ++q)
    for (int t = 0; t < 9; ++t)
      S[(size_t)(q * 9 + t) * np + p] = i < nx ? T(A[(size_t)((q + 13) * 9 + t) * n + m]) : T(0);
}

// largest |entry| of the FP64 half storage into *amax (float bits; non-negative floats order as unsigned ints)
__global__ void k_sym_absmax(const double* __restrict__ S, int64_t m, unsigned* __restrict__ amax) {
  float v = 0.f;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < m; e += (int64_t)gridDim.x * blockDim.x)
    v = fmaxf(v, (float)fabs(S[e]));
  for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
  if ((threadIdx.x & 31) == 0) atomicMax(amax, __float_as_uint(v));
}

// Sh = S / 2^e as FP16 with 2^e the smallest power of two above amax / 2^15 (so |Sh| < 2^15 < 65504); the
// scale itself goes to hscale[0]
__global__ void k_sym_to_half(const double* __restrict__ S, int64_t m, const unsigned* __restrict__ amax,
                              float* __restrict__ hscale, __half* __restrict__ Sh) {
  int e = 0;
  frexpf(__uint_as_float(*amax), &e);            // amax < 2^e
  const double inv = ldexp(1.0, 15 - e);
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i == 0) *hscale = ldexpf(1.f, e - 15);
  if (i < m) Sh[i] = __float2half_rn((float)(S[i] * inv));
}

// Stencil product of a symmetric half-stored level with a fused epilogue.
//
// A CTA of 32 x 4 threads takes 32 consecutive nodes of one x-row.  The 14 stored block slots
// q = 0..13 (self and the 13 forward offsets o = 13 + q) are split over the 4 warps, q = w, w+4, w+8,
// w+12: every warp reads, for its 32 nodes, the forward block of slot q at the node and the backward
// block (the transpose of the forward block stored at the neighbour n - off).  Out-of-range neighbours are
// clamped to the node itself and their u zeroed, so the loads carry no branches and a warp keeps all of
// its slots' loads in flight together.  Partial sums meet in shared memory; warps 0..2 then each finish
// one component of the 32 nodes.  Entries the stencil cannot hold (per-node CSR) are summed by the warps
// cooperatively: warp w takes the nodes of its 32 with entries whose lane is w mod 4.
// lam_t v_t.u of every rank-1 term, one warp per term (lanes over its entries)
template <typename T>
__global__ void k_term_dots(SymView<T> L, int nterms, const T* __restrict__ u, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int t = blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32, lane = threadIdx.x & 31;
  if (t >= nterms) return;
  T d = 0;
  for (int e = L.t_ptr[t] + lane; e < L.t_ptr[t + 1]; e += 32) d += L.t_val[e] * u[L.t_dof[e]];
  d = warp_sum(d);
  if (lane == 0) L.tdot[t] = L.t_lam[t] * d;
}

// Slot Q (offset o = 13 + Q) of one node: the forward block stored at the node times u at n + off, and, for
// Q > 0, the forward block stored at n - off, transposed, times u there.  Out-of-range neighbours are clamped
// to the node itself and their u zeroed, so the loads carry no branches.  Q is a compile-time constant: the
// offsets, the bounds tests and the plane offsets fold.  CMP: blocks of tagged (single-material) nodes are
// formed from the patterns sp[2][126] and the material table sm[128][2] (shared memory) instead of read.
// sym_load gathers a slot's operands, sym_acc applies them.
template <typename T>
struct SlotVals {
  T f[9], g[9], uf[3], ub[3];
};

template <typename T, bool CMP, bool H, int Q>
__device__ __forceinline__ void sym_load(const SymView<T>& L, const T* __restrict__ u, int n, int pn, int ic, int j,
                                         int k, int tn, const T* sp, const T* sm, SlotVals<T>& v) {
  constexpr int o = 13 + Q;
  constexpr int dx = o % 3 - 1, dy = (o / 3) % 3 - 1, dz = o / 9 - 1;
  const int nx = L.nx, ny = L.ny, nz = L.nz, nxp = L.nxp, NP = (int)L.np;
  const int off = dx + nx * (dy + ny * dz), offp = dx + nxp * (dy + ny * dz);
  const T* __restrict__ B = L.S + (size_t)Q * 9 * NP;
  bool vf = true, vb = Q > 0;
  if constexpr (dx > 0) { vf = vf && ic + 1 < nx; vb = vb && ic >= 1; }
  if constexpr (dx < 0) { vf = vf && ic >= 1; vb = vb && ic + 1 < nx; }
  if constexpr (dy > 0) { vf = vf && j + 1 < ny; vb = vb && j >= 1; }
  if constexpr (dy < 0) { vf = vf && j >= 1; vb = vb && j + 1 < ny; }
  if constexpr (dz > 0) { vf = vf && k + 1 < nz; vb = vb && k >= 1; }
  const int mf = vf ? n + off : n;
#pragma unroll
  for (int c = 0; c < 3; ++c) v.uf[c] = u[3 * mf + c];
  if (!vf) { v.uf[0] = 0; v.uf[1] = 0; v.uf[2] = 0; }
  auto stored = [&](int m, T (&w)[9]) {     // m: padded position
    if constexpr (H) {
      const __half* __restrict__ Bh = L.Sh + (size_t)Q * 9 * NP;
#pragma unroll
      for (int t = 0; t < 9; ++t) w[t] = T(__half2float(Bh[(size_t)t * NP + m]));
    } else {
#pragma unroll
      for (int t = 0; t < 9; ++t) w[t] = B[(size_t)t * NP + m];
    }
  };
  auto formed = [&](int tg, T (&w)[9]) {
    const T lam = sm[2 * tg], mu = sm[2 * tg + 1];
#pragma unroll
    for (int t = 0; t < 9; ++t) w[t] = lam * sp[9 * Q + t] + mu * sp[126 + 9 * Q + t];
  };
  if constexpr (CMP) { if (tn) formed(tn, v.f); else stored(pn, v.f); }
  else stored(pn, v.f);
  if constexpr (Q > 0) {
    const int mb = vb ? n - off : n, pb = vb ? pn - offp : pn;
#pragma unroll
    for (int c = 0; c < 3; ++c) v.ub[c] = u[3 * mb + c];
    if (!vb) { v.ub[0] = 0; v.ub[1] = 0; v.ub[2] = 0; }
    if constexpr (CMP) { const int tm = L.tag[mb]; if (tm) formed(tm, v.g); else stored(pb, v.g); }
    else stored(pb, v.g);
  }
}

template <typename T, int Q>
__device__ __forceinline__ void sym_acc(const SlotVals<T>& v, T& a0, T& a1, T& a2) {
  a0 += v.f[0] * v.uf[0] + v.f[1] * v.uf[1] + v.f[2] * v.uf[2];
  a1 += v.f[3] * v.uf[0] + v.f[4] * v.uf[1] + v.f[5] * v.uf[2];
  a2 += v.f[6] * v.uf[0] + v.f[7] * v.uf[1] + v.f[8] * v.uf[2];
  if constexpr (Q > 0) {
    a0 += v.g[0] * v.ub[0] + v.g[3] * v.ub[1] + v.g[6] * v.ub[2];
    a1 += v.g[1] * v.ub[0] + v.g[4] * v.ub[1] + v.g[7] * v.ub[2];
    a2 += v.g[2] * v.ub[0] + v.g[5] * v.ub[1] + v.g[8] * v.ub[2];
  }
}

template <typename T, bool CMP, bool H, int Q>
__device__ __forceinline__ void sym_slot(const SymView<T>& L, const T* __restrict__ u, int n, int pn, int ic, int j,
                                         int k, int tn, const T* sp, const T* sm, T& a0, T& a1, T& a2) {
  SlotVals<T> v;
  sym_load<T, CMP, H, Q>(L, u, n, pn, ic, j, k, tn, sp, sm, v);
  sym_acc<T, Q>(v, a0, a1, a2);
}

// CMP: the level carries the compressed single-material blocks (tags); without them the pattern code is not
// compiled into the kernel at all.  Offsets within the stencil planes are 32-bit (126 x the padded node count
// < 2^31 is checked at launch).  H (with CT, FP32): the stored blocks are read from the 16-bit copy Sh and the
// slot sums scaled by hscale before the entries and terms are added.
template <typename T, int EPI, bool CMP, bool CT, bool H>
__global__ void __launch_bounds__(128)
k_sym(SymView<T> L, const T* __restrict__ u, T* __restrict__ y, const T* __restrict__ b, T* __restrict__ r,
      T* __restrict__ d_out, T* __restrict__ x, const LevelParams* __restrict__ lp, int kstep,
      const int* __restrict__ skip, TermAcc<T> acc) {
  if (skip && *skip) return;
  __shared__ T red[4][3][32];
  __shared__ T spat[2][CMP ? 126 : 1];
  __shared__ T smat[CMP ? 128 : 1][2];
  const int lane = threadIdx.x, w = threadIdx.y;
  if constexpr (CMP) {
    const int tid = w * 32 + lane;
    for (int e = tid; e < 252; e += 128) spat[e / 126][e % 126] = L.pat[e];
    for (int e = tid; e < 256; e += 128) smat[e / 2][e % 2] = L.tmat[e];
    __syncthreads();
  }
  const int i = blockIdx.x * 32 + lane, j = blockIdx.y, k = blockIdx.z;
  const int nx = L.nx, ny = L.ny, nz = L.nz;
  const bool valid = i < nx;
  const int ic = valid ? i : nx - 1;
  const int n = ic + nx * (j + ny * k);
  const int N = (int)L.n;
  const int nxp = L.nxp, NP = (int)L.np;          // row-padded stencil planes
  const int pn = ic + nxp * (j + ny * k);
  int tn = 0;
  if constexpr (CMP) tn = L.tag[n];
  T a0 = 0, a1 = 0, a2 = 0;
  const T* sp = CMP ? &spat[0][0] : nullptr;
  const T* sm = CMP ? &smat[0][0] : nullptr;
  if constexpr (CT) {
    // the 14 slots over the 4 warps (warp-uniform switch): 0 4 8 12 | 1 5 9 13 | 2 6 10 | 3 7 11
#define FEB_SLOT(Q) sym_slot<T, CMP, H, Q>(L, u, n, pn, ic, j, k, tn, sp, sm, a0, a1, a2)
    switch (w) {
      case 0: FEB_SLOT(0); FEB_SLOT(4); FEB_SLOT(8); FEB_SLOT(12); break;
      case 1: FEB_SLOT(1); FEB_SLOT(5); FEB_SLOT(9); FEB_SLOT(13); break;
      case 2: FEB_SLOT(2); FEB_SLOT(6); FEB_SLOT(10); break;
      default: FEB_SLOT(3); FEB_SLOT(7); FEB_SLOT(11); break;
    }
#undef FEB_SLOT
    if constexpr (H) {
      const T sc = T(*L.hscale);
      a0 *= sc; a1 *= sc; a2 *= sc;
    }
  } else {
    // the same slots with the slot index a run-time value (the loop keeps every slot's loads in flight together)
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int q = w + 4 * t;
      if (q > 13) break;                                     // warp-uniform (t == 3, w >= 2)
      const int o = 13 + q;
      const int dx = o % 3 - 1, dy = (o / 3) % 3 - 1, dz = o / 9 - 1;
      const int off = dx + nx * (dy + ny * dz), offp = dx + nxp * (dy + ny * dz);
      const T* __restrict__ B = L.S + q * 9 * NP;
      const bool vf = ic + dx >= 0 && ic + dx < nx && j + dy >= 0 && j + dy < ny && k + dz < nz;
      const bool vb = q > 0 && ic - dx >= 0 && ic - dx < nx && j - dy >= 0 && j - dy < ny && k - dz >= 0;
      const int mf = vf ? n + off : n, mb = vb ? n - off : n, pb = vb ? pn - offp : pn;
      T uf0 = u[3 * mf], uf1 = u[3 * mf + 1], uf2 = u[3 * mf + 2];
      T ub0 = u[3 * mb], ub1 = u[3 * mb + 1], ub2 = u[3 * mb + 2];
      T fv[9], gv[9];
      auto stored = [&](int m, T (&v)[9]) {     // m: padded position
#pragma unroll
        for (int tt = 0; tt < 9; ++tt) v[tt] = B[tt * NP + m];
      };
      if constexpr (CMP) {
        auto formed = [&](int tg, T (&v)[9]) {
          const T lam = sm[2 * tg], mu = sm[2 * tg + 1];
#pragma unroll
          for (int tt = 0; tt < 9; ++tt) v[tt] = lam * sp[9 * q + tt] + mu * sp[126 + 9 * q + tt];
        };
        const int tm = L.tag[mb];
        if (tn) formed(tn, fv); else stored(pn, fv);
        if (tm) formed(tm, gv); else stored(pb, gv);
      } else {
        stored(pn, fv);
        stored(pb, gv);
      }
      if (!vf) { uf0 = 0; uf1 = 0; uf2 = 0; }
      if (!vb) { ub0 = 0; ub1 = 0; ub2 = 0; }
      a0 += fv[0] * uf0 + fv[1] * uf1 + fv[2] * uf2 + gv[0] * ub0 + gv[3] * ub1 + gv[6] * ub2;
      a1 += fv[3] * uf0 + fv[4] * uf1 + fv[5] * uf2 + gv[1] * ub0 + gv[4] * ub1 + gv[7] * ub2;
      a2 += fv[6] * uf0 + fv[7] * uf1 + fv[8] * uf2 + gv[2] * ub0 + gv[5] * ub1 + gv[8] * ub2;
    }
  }
  if (L.node_ptr) {
    int beg = 0, end = 0;
    if (valid) { beg = L.node_ptr[n]; end = L.node_ptr[n + 1]; }
    unsigned todo = __ballot_sync(0xffffffffu, end > beg) & (0x11111111u << w);
    while (todo) {
      const int src = __ffs(todo) - 1;
      todo &= todo - 1;
      const int b0 = __shfl_sync(0xffffffffu, beg, src), b1 = __shfl_sync(0xffffffffu, end, src);
      T s0 = 0, s1 = 0, s2 = 0;
      for (int e = b0 + lane; e < b1; e += 32) {
        const T v = L.ent_v[e] * u[L.ent_col[e]];
        const int rr = L.ent_r[e];
        s0 += rr == 0 ? v : T(0);
        s1 += rr == 1 ? v : T(0);
        s2 += rr == 2 ? v : T(0);
      }
      s0 = warp_sum(s0); s1 = warp_sum(s1); s2 = warp_sum(s2);
      if (lane == src) { a0 += s0; a1 += s1; a2 += s2; }
    }
  }
  if (L.tn_ptr && valid) {   // rank-1 terms: the term's dot lam_t v_t.u comes from k_term_dots; the node's
                             // pairs are split over the 4 warps
    const int pe = L.tn_ptr[n + 1];
    for (int p = L.tn_ptr[n] + w; p < pe; p += 4) {
      const T dot = L.tdot[L.tn_term[p]];
      a0 += dot * L.tn_coef[3 * p];
      a1 += dot * L.tn_coef[3 * p + 1];
      a2 += dot * L.tn_coef[3 * p + 2];
    }
  }
  red[w][0][lane] = a0; red[w][1][lane] = a1; red[w][2][lane] = a2;
  // epilogue operands that do not depend on the product, read before the barrier (r is rewritten after it)
  const int c = w;
  T rold0 = 0, rold1 = 0, rold2 = 0, bc = 0, uc = 0, xc = 0, D0 = 0, D1 = 0, D2 = 0;
  if (c < 3 && valid) {
    if constexpr (EPI == EPI_RESID) bc = b[3 * n + c];
    if constexpr (EPI == EPI_CHEB) {
      rold0 = r[3 * n]; rold1 = r[3 * n + 1]; rold2 = r[3 * n + 2];
      uc = u[3 * n + c]; xc = x[3 * n + c];
      D0 = L.Dinv[(3 * c) * N + n]; D1 = L.Dinv[(3 * c + 1) * N + n]; D2 = L.Dinv[(3 * c + 2) * N + n];   // 9 N < 2^31
    }
  }
  __syncthreads();
  if (c >= 3 || !valid) return;
  if constexpr (EPI == EPI_APPLY) {
    y[3 * n + c] = red[0][c][lane] + red[1][c][lane] + red[2][c][lane] + red[3][c][lane];
  } else if constexpr (EPI == EPI_RESID) {
    r[3 * n + c] = bc - (red[0][c][lane] + red[1][c][lane] + red[2][c][lane] + red[3][c][lane]);
  } else {
    const T A0 = red[0][0][lane] + red[1][0][lane] + red[2][0][lane] + red[3][0][lane];
    const T A1 = red[0][1][lane] + red[1][1][lane] + red[2][1][lane] + red[3][1][lane];
    const T A2 = red[0][2][lane] + red[1][2][lane] + red[2][2][lane] + red[3][2][lane];
    const T r0 = rold0 - A0, r1 = rold1 - A1, r2 = rold2 - A2;
    const T rc = c == 0 ? r0 : (c == 1 ? r1 : r2);
    const T c1 = T(lp->a1[kstep]), c2 = T(lp->a2[kstep]);
    const T z = D0 * r0 + D1 * r1 + D2 * r2;
    const T e = c1 * uc + c2 * z;
    r[3 * n + c] = rc;
    d_out[3 * n + c] = e;
    x[3 * n + c] = xc + e;
    term_acc1(acc, n, c, e);
  }
}

}  // namespace

template <typename T>
void launch_sym(const SymView<T>& L0, int epi, const T* u, T* y, const T* b, T* r, T* d_out, T* x,
                const LevelParams* lp, int k, const int* skip, cudaStream_t s, const T* tdot_in,
                const TermAcc<T>& acc) {
  const dim3 g(div_up(L0.nx, 32), L0.ny, L0.nz), blk(32, 4);
  SymView<T> L = L0;
  if (L.tn_ptr && L.nterms > 0) {
    if (tdot_in) {
      L.tdot = const_cast<T*>(tdot_in);
    } else {
      k_term_dots<T><<<div_up(L.nterms, 8), 256, 0, s>>>(L, L.nterms, u, skip); note_launch();
    }
  }
  if (126 * L.np >= (int64_t)INT32_MAX) {  // stencil-plane offsets are 32-bit; never reached by a coarse level
    fprintf(stderr, "launch_sym: level of %lld nodes exceeds the 32-bit stencil offsets\n", (long long)L.n);
    return;
  }
  const bool cmp = L.tag != nullptr;
  const bool ct = L.slots == 2 || (L.slots == 0 && std::is_same<T, float>::value);
#define FEB_SYM(E, C, CT_) k_sym<T, E, C, CT_, false><<<g, blk, 0, s>>>(L, u, y, b, r, d_out, x, lp, k, skip, acc)
#define FEB_SYM2(E, C) do { if (ct) FEB_SYM(E, C, true); else FEB_SYM(E, C, false); } while (0)
  if constexpr (std::is_same<T, float>::value) {
    if (L.Sh) {   // 16-bit storage: uncompressed levels, compile-time slots (the builder sets it only then)
#define FEB_SYMH(E) k_sym<T, E, false, true, true><<<g, blk, 0, s>>>(L, u, y, b, r, d_out, x, lp, k, skip, acc)
      if (epi == EPI_APPLY) FEB_SYMH(EPI_APPLY);
      else if (epi == EPI_RESID) FEB_SYMH(EPI_RESID);
      else FEB_SYMH(EPI_CHEB);
#undef FEB_SYMH
      note_launch();
      return;
    }
  }
  if (epi == EPI_APPLY) {
    if (cmp) FEB_SYM2(EPI_APPLY, true); else FEB_SYM2(EPI_APPLY, false);
  } else if (epi == EPI_RESID) {
    if (cmp) FEB_SYM2(EPI_RESID, true); else FEB_SYM2(EPI_RESID, false);
  } else {
    if (cmp) FEB_SYM2(EPI_CHEB, true); else FEB_SYM2(EPI_CHEB, false);
  }
#undef FEB_SYM2
#undef FEB_SYM
  note_launch();
}

void launch_sym_to_half(const double* S64, int nx, int ny, int nz, unsigned* amax, float* hscale, __half* Sh,
                        cudaStream_t s) {
  const int64_t m = 126 * sym_np(nx, ny, nz);
  cudaMemsetAsync(amax, 0, sizeof(unsigned), s);
  k_sym_absmax<<<std::min<int64_t>(div_up(m, kThreads), 4 * 148), kThreads, 0, s>>>(S64, m, amax); note_launch();
  k_sym_to_half<<<div_up(m, kThreads), kThreads, 0, s>>>(S64, m, amax, hscale, Sh); note_launch();
}

template <typename T>
void launch_stencil_to_sym(const double* A, int nx, int ny, int nz, T* S, cudaStream_t s) {
  const int64_t n = (int64_t)nx * ny * nz, np = sym_np(nx, ny, nz);
  k_stencil_to_sym<T><<<div_up(np, kThreads), kThreads, 0, s>>>(A, nx, sym_nxp(nx), n, np, S); note_launch();
}

template void launch_sym<float>(const SymView<float>&, int, const float*, float*, const float*, float*, float*,
                                float*, const LevelParams*, int, const int*, cudaStream_t, const float*,
                                const TermAcc<float>&);
template void launch_sym<double>(const SymView<double>&, int, const double*, double*, const double*, double*,
                                 double*, double*, const LevelParams*, int, const int*, cudaStream_t, const double*,
                                 const TermAcc<double>&);
void launch_galerkin_axis(const AxisDev& ax, int d, const double* Ain, int inx, int iny, int inz, double* Aout,
                          int onx, int ony, int onz, cudaStream_t s) {
  const int64_t no = (int64_t)onx * ony * onz;
  k_galerkin_axis<<<dim3(div_up(no, 128), 27), 128, 0, s>>>(ax, d, Ain, inx, iny, inz, Aout, onx, ony, onz);
  note_launch();
}

template void launch_stencil_to_sym<float>(const double*, int, int, int, float*, cudaStream_t);
template void launch_stencil_to_sym<double>(const double*, int, int, int, double*, cudaStream_t);

template <typename T>
void launch_stencil_apply(const StencilView<T>& L, const T* u, T* y, const int* skip, cudaStream_t s) {
  k_stencil_apply<T><<<div_up(L.n, kThreads), kThreads, 0, s>>>(L, u, y, skip); note_launch();
  if (L.nrow > 0) launch_csr_add<T>(L.nrow, L.row_dof, L.row_ptr, L.col, L.val, u, y, skip, s);
}

template <typename T>
void launch_csr_add(int nrow, const int* row_dof, const int* row_ptr, const int* col, const T* val, const T* u, T* y,
                    const int* skip, cudaStream_t s) {
  if (nrow <= 0) return;
  k_csr_add<T><<<div_up(nrow, kThreads), kThreads, 0, s>>>(nrow, row_dof, row_ptr, col, val, u, y, skip); note_launch();
}

template <typename T>
void launch_restrict(const TransferDev& P, int fnx, int fny, int fnz, int64_t fnnode, int64_t fntotal,
                     const int* orig_copy, const T* rf, T* rc, const int* skip, cudaStream_t s, T* zero, int nzero) {
  if (!zero) nzero = 0;
  if (P.even) {
    k_restrict_even<T><<<dim3(div_up(P.ax[0].nc, 64), P.ax[1].nc, P.ax[2].nc), 64, 0, s>>>(
        P.ax[0].nc, P.ax[1].nc, fnx, fny, fnz, rf, rc, skip, zero, nzero, P.cp_ptr, P.cp_copy, P.cp_w, fnnode);
    note_launch();
    if (P.cp_ptr) return;   // the copies were gathered
  } else {
    k_restrict_grid<T><<<dim3(div_up(P.ax[0].nc, 64), P.ax[1].nc, P.ax[2].nc), 64, 0, s>>>(P, fnx, fny, rf, rc, skip,
                                                                                         zero, nzero); note_launch();
  }
  if (fntotal > fnnode)
    k_restrict_copies<T><<<div_up(fntotal - fnnode, kThreads), kThreads, 0, s>>>(P, fnx, fny, fnnode, fntotal,
                                                                                 orig_copy, rf, rc, skip); note_launch();
  (void)fnz;
}

template <typename T>
void launch_prolong_add(const TransferDev& P, int fnx, int fny, int fnz, int64_t fnnode, int64_t fntotal,
                        const int* orig_copy, const uint8_t* used, const T* xc, T* xf, const int* skip,
                        cudaStream_t s, const TermAcc<T>& acc) {
  if (P.even) {   // the copies ride in extra z layers of the same launch
    const int64_t ncopy = fntotal - fnnode, layer = (int64_t)div_up(fnx, 64) * 64 * fny;
    const int extra = (int)((ncopy + layer - 1) / layer);
    k_prolong_even<T><<<dim3(div_up(fnx, 64), fny, fnz + extra), 64, 0, s>>>(
        P.ax[0].nc, P.ax[1].nc, fnx, fny, fnz, used, xc, xf, skip, acc, fnnode, ncopy, orig_copy); note_launch();
    return;
  } else {
    k_prolong_grid<T><<<dim3(div_up(fnx, 64), fny, fnz), 64, 0, s>>>(P, fnx, fny, used, xc, xf, skip, acc); note_launch();
  }
  if (fntotal > fnnode) {
    k_prolong_copies<T><<<div_up(fntotal - fnnode, kThreads), kThreads, 0, s>>>(P, fnx, fny, fnnode, fntotal,
                                                                               orig_copy, xc, xf, skip); note_launch();
  }
}

void launch_kept_mask(const TransferDev& P, const uint8_t* used_f, uint8_t* kept_c, cudaStream_t s) {
  int64_t nc = (int64_t)P.ax[0].nc * P.ax[1].nc * P.ax[2].nc;
  k_kept_mask<<<div_up(nc, kThreads), kThreads, 0, s>>>(P, used_f, kept_c); note_launch();
}

template <int MODE>
void launch_galerkin_cells(const FineView<double>& F, const double* mat_all, const TransferDev& P, double* KeC,
                           double* A1, int cnx, int cny, int cnz, cudaStream_t s) {
  int ncx = cnx - 1, ncy = cny - 1, ncz = cnz - 1;
  int64_t ncell = (int64_t)ncx * ncy * ncz;
  dim3 blk(24, 8);
  k_galerkin_cells<MODE><<<div_up(ncell, 8), blk, 0, s>>>(F, mat_all, P, KeC, ncx, ncy, ncz); note_launch();
  int64_t n = (int64_t)cnx * cny * cnz;
  dim3 blk2(27, 8);
  k_cells_to_stencil<<<div_up(n, 8), blk2, 0, s>>>(KeC, A1, cnx, cny, cnz); note_launch();
}

template <int MODE>
int launch_galerkin_direct(const double* mat_all, int fnx, int fny, double a, double b, double c, double* basis,
                           double* A1, int cnx, int cny, int cnz, cudaStream_t s) {
  if (MODE == MAT_ORTHO) return FEB_ERR_ARG;
  k_galerkin_basis<MODE><<<16, 32, 0, s>>>(a, b, c, basis); note_launch();
  const int smem = 16 * 576 * sizeof(double);
  FEB_TRY(set_dyn_smem((const void*)k_galerkin_direct, smem));
  const int64_t n = (int64_t)cnx * cny * cnz;
  k_galerkin_direct<<<div_up(n, 8), dim3(27, 8), smem, s>>>(mat_all, fnx, fny, basis, A1, cnx, cny, cnz); note_launch();
  return FEB_OK;
}
template int launch_galerkin_direct<MAT_ISO_SRI>(const double*, int, int, double, double, double, double*, double*, int,
                                                 int, int, cudaStream_t);
template int launch_galerkin_direct<MAT_ISO_FULL>(const double*, int, int, double, double, double, double*, double*, int,
                                                  int, int, cudaStream_t);

void launch_sym_pattern(const double* basis, double* pat, cudaStream_t s) {
  k_sym_pattern<<<1, 256, 0, s>>>(basis, pat); note_launch();
}
void launch_sym_tags(const double* S64, int cnx, int cny, int cnz, const uint16_t* cellpair, int fnxn, int mp,
                     const double* mtab, const double* pat, uint8_t* tag, cudaStream_t s) {
  const int64_t n = (int64_t)cnx * cny * cnz;
  k_sym_tags<<<div_up(n, kThreads), kThreads, 0, s>>>(S64, cnx, cny, cnz, cellpair, fnxn, mp, mtab, pat, tag);
  note_launch();
}

void launch_galerkin_penalty(const TransferDev& P, int fnx, int fny, int64_t fnnode, const int* orig_copy, int npen,
                             const int* pen_node, const double* pen_k, double* A1, int cnx, int cny, int cnz,
                             int64_t cn, cudaStream_t s) {
  if (npen <= 0) return;
  k_galerkin_penalty<<<div_up(npen, kThreads), kThreads, 0, s>>>(P, fnx, fny, fnnode, orig_copy, npen, pen_node,
                                                                  pen_k, A1, cnx, cny, cn); note_launch();
  (void)cnz;
}

void launch_galerkin_local(const TransferDev& P, int fnx, int fny, int64_t fnnode, const int* orig_copy, int nent,
                           const int* rdof, const int* cdof, const double* val, double* A1, int cnx, int cny, int cnz,
                           int64_t cn, cudaStream_t s) {
  if (nent <= 0) return;
  k_galerkin_local<<<div_up(nent, kThreads), kThreads, 0, s>>>(P, fnx, fny, fnnode, orig_copy, nent, rdof, cdof, val,
                                                                A1, cnx, cny, cn); note_launch();
  (void)cnz;
}

void launch_stencil_diag(const double* A, int64_t n, double* D, cudaStream_t s) {
  k_stencil_diag<<<div_up(n, kThreads), kThreads, 0, s>>>(A, n, D); note_launch();
}

void launch_add_diag_entries(int nent, const int* rdof, const int* cdof, const double* val, double* D, cudaStream_t s) {
  if (nent <= 0) return;
  k_add_diag_entries<<<div_up(nent, kThreads), kThreads, 0, s>>>(nent, rdof, cdof, val, D); note_launch();
}

void launch_block_inverse(const double* D, int64_t n, double* Dinv64, float* Dinv32, cudaStream_t s) {
  k_block_inverse<<<div_up(n, kThreads), kThreads, 0, s>>>(D, n, Dinv64, Dinv32); note_launch();
}

template void launch_stencil_apply<float>(const StencilView<float>&, const float*, float*, const int*, cudaStream_t);
template void launch_stencil_apply<double>(const StencilView<double>&, const double*, double*, const int*, cudaStream_t);
template void launch_csr_add<float>(int, const int*, const int*, const int*, const float*, const float*, float*,
                                    const int*, cudaStream_t);
template void launch_csr_add<double>(int, const int*, const int*, const int*, const double*, const double*, double*,
                                     const int*, cudaStream_t);
template void launch_restrict<float>(const TransferDev&, int, int, int, int64_t, int64_t, const int*, const float*,
                                     float*, const int*, cudaStream_t, float*, int);
template void launch_restrict<double>(const TransferDev&, int, int, int, int64_t, int64_t, const int*, const double*,
                                      double*, const int*, cudaStream_t, double*, int);
template void launch_prolong_add<float>(const TransferDev&, int, int, int, int64_t, int64_t, const int*,
                                        const uint8_t*, const float*, float*, const int*, cudaStream_t,
                                        const TermAcc<float>&);
template void launch_prolong_add<double>(const TransferDev&, int, int, int, int64_t, int64_t, const int*,
                                         const uint8_t*, const double*, double*, const int*, cudaStream_t,
                                         const TermAcc<double>&);
template void launch_galerkin_cells<MAT_ISO_SRI>(const FineView<double>&, const double*, const TransferDev&, double*,
                                                 double*, int, int, int, cudaStream_t);
template void launch_galerkin_cells<MAT_ISO_FULL>(const FineView<double>&, const double*, const TransferDev&, double*,
                                                  double*, int, int, int, cudaStream_t);
template void launch_galerkin_cells<MAT_ORTHO>(const FineView<double>&, const double*, const TransferDev&, double*,
                                               double*, int, int, int, cudaStream_t);

}  // namespace feb
