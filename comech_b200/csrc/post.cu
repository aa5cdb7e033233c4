// Post-processing of a solution on the device: forces between regions (rb/rbfe.py:194-219), rigid fit of a
// node set and displacement relative to it (rb/rbsim.py:99-107, 183-186), and resampling of the fields on
// an analysis grid (rb/rbsim.py:110-161).
#include <vector>

#include "element.cuh"

namespace feb {

namespace {

struct Geom {
  int nx, ny, nz;
  const double* xe; const double* ye; const double* ze;   // edges (nx+1, ny+1, nz+1)
};

// cell id (z fastest) -> (i, j, k) and its 8 node ids (split connectivity or grid connectivity)
__device__ __forceinline__ void cell_of(const Geom& G, int64_t cell, const int64_t* cn, int64_t (&nd)[8], int& i,
                                        int& j, int& k) {
  k = int(cell % G.nz);
  j = int((cell / G.nz) % G.ny);
  i = int(cell / ((int64_t)G.nz * G.ny));
  const int64_t nx1 = G.nx + 1, ny1 = G.ny + 1;
#pragma unroll
  for (int l = 0; l < 8; ++l)
    nd[l] = cn ? cn[8 * cell + l] : (i + (l & 1)) + nx1 * ((j + ((l >> 1) & 1)) + ny1 * (k + ((l >> 2) & 1)));
}

// coordinates of node id n (copies sit at their grid node, orig)
__device__ __forceinline__ void node_xyz(const Geom& G, const int64_t* orig, int64_t nnode, int64_t n, double (&x)[3]) {
  const int64_t p = (n < nnode || !orig) ? n : orig[n];
  const int64_t nx1 = G.nx + 1, ny1 = G.ny + 1;
  x[0] = G.xe[p % nx1];
  x[1] = G.ye[(p / nx1) % ny1];
  x[2] = G.ze[p / (nx1 * ny1)];
}

__global__ void k_mark_part_nodes(Geom G, int64_t ncell, const int64_t* __restrict__ cn,
                                  const uint8_t* __restrict__ active, const int32_t* __restrict__ part, int32_t target,
                                  uint8_t* __restrict__ mark) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ncell || !active[c] || part[c] != target) return;
  int64_t nd[8];
  int i, j, k;
  cell_of(G, c, cn, nd, i, j, k);
#pragma unroll
  for (int l = 0; l < 8; ++l) mark[nd[l]] = 1;
}

// Forces exerted on the marked nodes by every active cell outside the target part: minus the cell's nodal
// forces K_e u_e at its marked corners, summed per cell label (block sums in shared memory, then one atomic
// per label and component per block).
constexpr int kMaxLabels = 64;
__global__ void __launch_bounds__(256)
k_region_forces(Geom G, int64_t ncell, const double* __restrict__ mat, const double* __restrict__ U,
                const int64_t* __restrict__ cn, const uint8_t* __restrict__ active, const int32_t* __restrict__ part,
                int32_t target, const int32_t* __restrict__ lab, int nlab, const uint8_t* __restrict__ mark,
                double* __restrict__ out, int* __restrict__ present) {
  __shared__ double acc[kMaxLabels * 3];
  __shared__ int seen[kMaxLabels];
  for (int e = threadIdx.x; e < nlab * 3; e += blockDim.x) acc[e] = 0.0;
  for (int e = threadIdx.x; e < nlab; e += blockDim.x) seen[e] = 0;
  __syncthreads();
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c < ncell && active[c] && part[c] != target) {
    int64_t nd[8];
    int i, j, k;
    cell_of(G, c, cn, nd, i, j, k);
    bool touch = false;
#pragma unroll
    for (int l = 0; l < 8; ++l) touch |= mark[nd[l]] != 0;
    const int L = lab[c];
    if (touch && L >= 0 && L < nlab) {
      double u[3][8], f[3][8];
#pragma unroll
      for (int l = 0; l < 8; ++l)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          const double v = U[3 * nd[l] + q];
          u[q][l] = isnan(v) ? 0.0 : v;
        }
      const double p[2] = {mat[c], mat[ncell + c]};
      const Material<double> m = make_material<double, MAT_ISO_SRI>(p);
      const double a = G.xe[i + 1] - G.xe[i], b = G.ye[j + 1] - G.ye[j], cc = G.ze[k + 1] - G.ze[k];
      hex8_apply(u, a, b, cc, 1.0 / a, 1.0 / b, 1.0 / cc, m, f);
      double s[3] = {0.0, 0.0, 0.0};
#pragma unroll
      for (int l = 0; l < 8; ++l)
        if (mark[nd[l]])
#pragma unroll
          for (int q = 0; q < 3; ++q) s[q] += f[q][l];
#pragma unroll
      for (int q = 0; q < 3; ++q) atomicAdd(&acc[3 * L + q], -s[q]);
      seen[L] = 1;
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nlab * 3; e += blockDim.x)
    if (seen[e / 3]) atomicAdd(out + e, acc[e]);
  for (int e = threadIdx.x; e < nlab; e += blockDim.x)
    if (seen[e]) present[e] = 1;
}

// Rigid fit, pass 1: sum of the point coordinates (per-block partials)
__global__ void k_fit_centroid(const double* __restrict__ X, int64_t n, double* __restrict__ part) {
  double s[3] = {0.0, 0.0, 0.0};
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    s[0] += X[3 * e]; s[1] += X[3 * e + 1]; s[2] += X[3 * e + 2];
  }
  for (int q = 0; q < 3; ++q) {
    const double t = block_sum(s[q]);
    if (threadIdx.x == 0) part[3 * blockIdx.x + q] = t;
    __syncthreads();
  }
}

// Rigid fit, pass 2: normal equations A^T A (21 upper entries) and A^T u (6) of the 3n x 6 system of
// rb/rbsim.py:99-107 (rows x: 1 0 0 0 rz -ry; y: 0 1 0 -rz 0 rx; z: 0 0 1 ry -rx 0; r = X - c)
__global__ void k_fit_normal(const double* __restrict__ X, int64_t n, const double* __restrict__ U,
                             const double* __restrict__ cen, double* __restrict__ part) {
  double s[27];
#pragma unroll
  for (int q = 0; q < 27; ++q) s[q] = 0.0;
  for (int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; e < n; e += (int64_t)gridDim.x * blockDim.x) {
    const double rx = X[3 * e] - cen[0], ry = X[3 * e + 1] - cen[1], rz = X[3 * e + 2] - cen[2];
    const double u[3] = {U[3 * e], U[3 * e + 1], U[3 * e + 2]};
    const double A[3][6] = {{1, 0, 0, 0, rz, -ry}, {0, 1, 0, -rz, 0, rx}, {0, 0, 1, ry, -rx, 0}};
    int t = 0;
#pragma unroll
    for (int a = 0; a < 6; ++a)
#pragma unroll
      for (int b = a; b < 6; ++b) s[t++] += A[0][a] * A[0][b] + A[1][a] * A[1][b] + A[2][a] * A[2][b];
#pragma unroll
    for (int a = 0; a < 6; ++a) s[21 + a] += A[0][a] * u[0] + A[1][a] * u[1] + A[2][a] * u[2];
  }
  for (int q = 0; q < 27; ++q) {
    const double t = block_sum(s[q]);
    if (threadIdx.x == 0) part[27 * blockIdx.x + q] = t;
    __syncthreads();
  }
}

// Urel = nan_to_num(U) - (t + w x (X - c)) at every node (rb/rbsim.py:184)
__global__ void k_relative(Geom G, const int64_t* __restrict__ orig, int64_t nnode, int64_t ntotal,
                           const double* __restrict__ U, const double* __restrict__ fit, double* __restrict__ out) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= ntotal) return;
  double x[3];
  node_xyz(G, orig, nnode, n, x);
  const double t0 = fit[0], t1 = fit[1], t2 = fit[2], w0 = fit[3], w1 = fit[4], w2 = fit[5];
  const double r0 = x[0] - fit[6], r1 = x[1] - fit[7], r2 = x[2] - fit[8];
  const double rot[3] = {w1 * r2 - w2 * r1, w2 * r0 - w0 * r2, w0 * r1 - w1 * r0};
  const double tt[3] = {t0, t1, t2};
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const double v = U[3 * n + q];
    out[3 * n + q] = (isnan(v) ? 0.0 : v) - (tt[q] + rot[q]);
  }
}

// One analysis cell per thread: sub^3 sample points (per-axis FE index, local coordinate and inside flag
// precomputed), trilinear relative displacement in the FE cell, von Mises and stress of the FE cell,
// averaged over the points that fall in active FE cells (rb/rbsim.py:110-138).
__global__ void k_sample_cells(Geom G, int mx, int my, int mz, int sub, const int32_t* __restrict__ ix,
                               const double* __restrict__ tx, const uint8_t* __restrict__ inx,
                               const int32_t* __restrict__ iy, const double* __restrict__ ty,
                               const uint8_t* __restrict__ iny, const int32_t* __restrict__ iz,
                               const double* __restrict__ tz, const uint8_t* __restrict__ inz,
                               const int64_t* __restrict__ cn, const uint8_t* __restrict__ active,
                               const double* __restrict__ Urel, const float* __restrict__ VM,
                               const float* __restrict__ SIG, float* __restrict__ vm_out, float* __restrict__ u_out,
                               float* __restrict__ frac_out, float* __restrict__ sig_out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)mx * my * mz) return;
  const int ck = int(e % mz), cj = int((e / mz) % my), ci = int(e / ((int64_t)mz * my));
  double su[3] = {0.0, 0.0, 0.0}, svm = 0.0, ssg[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  int okc = 0;
  for (int a = 0; a < sub; ++a)
    for (int b = 0; b < sub; ++b)
      for (int c = 0; c < sub; ++c) {
        const int px = ci * sub + a, py = cj * sub + b, pz = ck * sub + c;
        const int64_t cell = ((int64_t)ix[px] * G.ny + iy[py]) * G.nz + iz[pz];
        if (!(inx[px] && iny[py] && inz[pz] && active[cell])) continue;
        ++okc;
        int64_t nd[8];
        int i, j, k;
        cell_of(G, cell, cn, nd, i, j, k);
        const double TX = tx[px], TY = ty[py], TZ = tz[pz];
#pragma unroll
        for (int l = 0; l < 8; ++l) {
          const double w = ((l & 1) ? TX : 1.0 - TX) * (((l >> 1) & 1) ? TY : 1.0 - TY) * (((l >> 2) & 1) ? TZ : 1.0 - TZ);
#pragma unroll
          for (int q = 0; q < 3; ++q) {
            const double v = Urel[3 * nd[l] + q];
            su[q] += w * (isnan(v) ? 0.0 : v);
          }
        }
        svm += (double)VM[cell];
#pragma unroll
        for (int q = 0; q < 6; ++q) ssg[q] += (double)SIG[6 * cell + q];
      }
  const double d = okc > 0 ? (double)okc : 1.0;
  vm_out[e] = float(svm / d);
#pragma unroll
  for (int q = 0; q < 3; ++q) u_out[3 * e + q] = float(su[q] / d);
#pragma unroll
  for (int q = 0; q < 6; ++q) sig_out[6 * e + q] = float(ssg[q] / d);
  frac_out[e] = float((double)okc / ((double)sub * sub * sub));
}

// Exact Euclidean feature transform over cell indices (nearest active cell of every cell), separable in the
// manner of Maurer, Qi and Raghavan (2003): one pass per axis in the order x, y, z.  Along each line the lower
// envelope of the parabolas g_s + (p - s)^2 of the candidate sites s is built on a stack (a site is dropped when
// the envelope test is positive), then every position takes the first site of minimal distance: ties go to the
// lower index, as scipy.ndimage.distance_transform_edt resolves them.  One thread per line; the stack (site
// position, partial distance and the site's feature coordinates) lives in global scratch, one slot per cell.
//   pass 0 (x lines, fixed j k): FI = i of the nearest active cell on the line
//   pass 1 (y lines, fixed i k): FI, FJ of the nearest active cell in the x-y plane, g = (FI - i)^2
//   pass 2 (z lines, fixed i j): ft = cell id of the nearest active cell, g = (FI - i)^2 + (FJ - j)^2
// "none" is -1 throughout (a grid without active cells gives ft = -1 everywhere).
__global__ void k_ft_pass(int pass, int nx, int ny, int nz, const uint8_t* __restrict__ active,
                          int32_t* __restrict__ FI, int32_t* __restrict__ FJ, int32_t* __restrict__ ft,
                          int32_t* __restrict__ sp, int64_t* __restrict__ sg, int32_t* __restrict__ sa,
                          int32_t* __restrict__ sb) {
  const int64_t line = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int n = pass == 0 ? nx : (pass == 1 ? ny : nz);
  const int64_t nlines = pass == 0 ? (int64_t)ny * nz : (pass == 1 ? (int64_t)nx * nz : (int64_t)nx * ny);
  if (line >= nlines) return;
  const int a = int(pass == 2 ? line / ny : line / nz);   // pass 0: j; pass 1: i; pass 2: i
  const int b = int(pass == 2 ? line % ny : line % nz);   // pass 0: k; pass 1: k; pass 2: j
  auto cell = [&](int p) -> int64_t {
    if (pass == 0) return ((int64_t)p * ny + a) * nz + b;
    if (pass == 1) return ((int64_t)a * ny + p) * nz + b;
    return ((int64_t)a * ny + b) * nz + p;
  };
  int32_t* S = sp + line * n;
  int64_t* G = sg + line * n;
  int32_t* A = sa + line * n;
  int32_t* B = sb + line * n;
  int top = 0;
  for (int p = 0; p < n; ++p) {
    const int64_t c = cell(p);
    int32_t fa = p, fb = 0;
    int64_t gp = 0;
    if (pass == 0) {
      if (!active[c]) continue;
    } else {
      if (FI[c] < 0) continue;
      fa = FI[c];
      const int64_t di = fa - a;
      gp = di * di;
      if (pass == 2) {
        fb = FJ[c];
        const int64_t dj = fb - b;
        gp += dj * dj;
      }
    }
    while (top >= 2) {
      const int64_t u = S[top - 2], v = S[top - 1], w = p;
      const int64_t x = v - u, y = w - v, z = w - u;
      if (z * G[top - 1] - y * G[top - 2] - x * gp - x * y * z > 0) --top;
      else break;
    }
    S[top] = p; G[top] = gp; A[top] = fa; B[top] = fb;
    ++top;
  }
  int l = 0;
  for (int p = 0; p < n; ++p) {
    const int64_t c = cell(p);
    if (top == 0) {
      if (pass == 0) FI[c] = -1;
      else if (pass == 1) { FI[c] = -1; FJ[c] = -1; }
      else ft[c] = -1;
      continue;
    }
    while (l < top - 1) {
      const int64_t d0 = G[l] + (int64_t)(S[l] - p) * (S[l] - p);
      const int64_t d1 = G[l + 1] + (int64_t)(S[l + 1] - p) * (S[l + 1] - p);
      if (d0 > d1) ++l;
      else break;
    }
    if (pass == 0) FI[c] = S[l];
    else if (pass == 1) { FI[c] = A[l]; FJ[c] = S[l]; }
    else ft[c] = (int32_t)(((int64_t)A[l] * ny + B[l]) * nz + S[l]);
  }
}

// Relative displacement at analysis-grid nodes (x fastest): the node's FE cell from per-axis indices, replaced
// by its nearest active cell (ft); local coordinates clamped to [0, 1]; trilinear in that cell
// (rb/rbsim.py:141-161).
__global__ void k_sample_nodes(Geom G, int mx1, int my1, int mz1, const int32_t* __restrict__ ix,
                               const double* __restrict__ px, const int32_t* __restrict__ iy,
                               const double* __restrict__ py, const int32_t* __restrict__ iz,
                               const double* __restrict__ pz, const int32_t* __restrict__ ft,
                               const int64_t* __restrict__ cn, const double* __restrict__ Urel, float* __restrict__ out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= (int64_t)mx1 * my1 * mz1) return;
  const int a = int(e % mx1), b = int((e / mx1) % my1), c = int(e / ((int64_t)mx1 * my1));
  const int64_t near = ft[((int64_t)ix[a] * G.ny + iy[b]) * G.nz + iz[c]];
  if (near < 0) {
    out[3 * e] = out[3 * e + 1] = out[3 * e + 2] = 0.f;
    return;
  }
  int64_t nd[8];
  int ci, cj, ck;
  cell_of(G, near, cn, nd, ci, cj, ck);
  const double tx = fmin(fmax((px[a] - G.xe[ci]) / (G.xe[ci + 1] - G.xe[ci]), 0.0), 1.0);
  const double ty = fmin(fmax((py[b] - G.ye[cj]) / (G.ye[cj + 1] - G.ye[cj]), 0.0), 1.0);
  const double tz = fmin(fmax((pz[c] - G.ze[ck]) / (G.ze[ck + 1] - G.ze[ck]), 0.0), 1.0);
  double u[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int l = 0; l < 8; ++l) {
    const double w = ((l & 1) ? tx : 1.0 - tx) * (((l >> 1) & 1) ? ty : 1.0 - ty) * (((l >> 2) & 1) ? tz : 1.0 - tz);
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const double v = Urel[3 * nd[l] + q];
      u[q] += w * (isnan(v) ? 0.0 : v);
    }
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) out[3 * e + q] = float(u[q]);
}

struct DevGeom {
  Geom G{};
  double* buf = nullptr;
};

int make_dev_geom(const FebGrid* grid, DevGeom& D, cudaStream_t s) {
  D.G.nx = grid->nx; D.G.ny = grid->ny; D.G.nz = grid->nz;
  const size_t n = (size_t)grid->nx + grid->ny + grid->nz + 3;
  FEB_CUDA(cudaMallocAsync((void**)&D.buf, n * sizeof(double), s));
  FEB_CUDA(cudaMemcpyAsync(D.buf, grid->xe, (grid->nx + 1) * sizeof(double), cudaMemcpyHostToDevice, s));
  FEB_CUDA(cudaMemcpyAsync(D.buf + grid->nx + 1, grid->ye, (grid->ny + 1) * sizeof(double), cudaMemcpyHostToDevice, s));
  FEB_CUDA(cudaMemcpyAsync(D.buf + grid->nx + grid->ny + 2, grid->ze, (grid->nz + 1) * sizeof(double),
                           cudaMemcpyHostToDevice, s));
  D.G.xe = D.buf;
  D.G.ye = D.buf + grid->nx + 1;
  D.G.ze = D.buf + grid->nx + grid->ny + 2;
  return FEB_OK;
}

constexpr int kFitBlocks = 148;

}  // namespace
}  // namespace feb

using namespace feb;

extern "C" int feb_region_forces(const FebGrid* grid, const double* mat, const double* U, const int64_t* cn,
                                 const uint8_t* active, const int32_t* part, const int32_t* lab, int32_t nlab,
                                 int32_t target, int64_t nnode_total, double* out, int32_t* present, void* stream) {
  if (!grid || !mat || !U || !active || !part || !lab || !out || !present || nlab < 1 || nlab > kMaxLabels ||
      nnode_total < 1) {
    set_last_error("feb_region_forces: bad argument (nlab 1..%d)", kMaxLabels);
    return FEB_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t ncell = (int64_t)grid->nx * grid->ny * grid->nz;
  DevGeom D;
  FEB_TRY(make_dev_geom(grid, D, s));
  uint8_t* mark = nullptr;
  FEB_CUDA(cudaMallocAsync((void**)&mark, (size_t)nnode_total, s));
  FEB_CUDA(cudaMemsetAsync(mark, 0, (size_t)nnode_total, s));
  FEB_CUDA(cudaMemsetAsync(out, 0, 3 * (size_t)nlab * sizeof(double), s));
  FEB_CUDA(cudaMemsetAsync(present, 0, (size_t)nlab * sizeof(int32_t), s));
  k_mark_part_nodes<<<div_up(ncell, kThreads), kThreads, 0, s>>>(D.G, ncell, cn, active, part, target, mark); note_launch();
  k_region_forces<<<div_up(ncell, 256), 256, 0, s>>>(D.G, ncell, mat, U, cn, active, part, target, lab, nlab, mark, out,
                                                    present); note_launch();
  FEB_CUDA(cudaGetLastError());
  FEB_CUDA(cudaFreeAsync(mark, s));
  FEB_CUDA(cudaFreeAsync(D.buf, s));
  return FEB_OK;
}

extern "C" int feb_rigid_fit(const double* X, const double* U, int64_t n, double* fit, void* stream) {
  if (!X || !U || !fit || n < 1) {
    set_last_error("feb_rigid_fit: bad argument");
    return FEB_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  double *part = nullptr, *cen = nullptr;
  FEB_CUDA(cudaMallocAsync((void**)&part, 27 * kFitBlocks * sizeof(double), s));
  FEB_CUDA(cudaMallocAsync((void**)&cen, 3 * sizeof(double), s));
  k_fit_centroid<<<kFitBlocks, kThreads, 0, s>>>(X, n, part); note_launch();
  std::vector<double> h(27 * kFitBlocks);
  FEB_CUDA(cudaMemcpyAsync(h.data(), part, 3 * kFitBlocks * sizeof(double), cudaMemcpyDeviceToHost, s));
  FEB_CUDA(cudaStreamSynchronize(s));
  double c[3] = {0.0, 0.0, 0.0};
  for (int b = 0; b < kFitBlocks; ++b)
    for (int q = 0; q < 3; ++q) c[q] += h[3 * b + q];
  for (int q = 0; q < 3; ++q) c[q] /= (double)n;
  FEB_CUDA(cudaMemcpyAsync(cen, c, 3 * sizeof(double), cudaMemcpyHostToDevice, s));
  k_fit_normal<<<kFitBlocks, kThreads, 0, s>>>(X, n, U, cen, part); note_launch();
  FEB_CUDA(cudaMemcpyAsync(h.data(), part, 27 * kFitBlocks * sizeof(double), cudaMemcpyDeviceToHost, s));
  FEB_CUDA(cudaStreamSynchronize(s));
  double S[27] = {0};
  for (int b = 0; b < kFitBlocks; ++b)
    for (int q = 0; q < 27; ++q) S[q] += h[27 * b + q];
  std::vector<double> AtA(36);
  int t = 0;
  for (int a = 0; a < 6; ++a)
    for (int b = a; b < 6; ++b) { AtA[a * 6 + b] = AtA[b * 6 + a] = S[t++]; }
  // least squares with the minimum-norm convention of numpy.linalg.lstsq: x = pinv(A^T A) A^T u
  std::vector<double> Pi = sym_pinv(AtA, 6);
  double x[6];
  for (int a = 0; a < 6; ++a) {
    x[a] = 0.0;
    for (int b = 0; b < 6; ++b) x[a] += Pi[a * 6 + b] * S[21 + b];
  }
  for (int q = 0; q < 6; ++q) fit[q] = x[q];
  for (int q = 0; q < 3; ++q) fit[6 + q] = c[q];
  FEB_CUDA(cudaFreeAsync(part, s));
  FEB_CUDA(cudaFreeAsync(cen, s));
  return FEB_OK;
}

extern "C" int feb_relative_displacement(const FebGrid* grid, const int64_t* orig, int64_t nnode_total, const double* U,
                                         const double* fit, double* out, void* stream) {
  if (!grid || !U || !fit || !out) {
    set_last_error("feb_relative_displacement: null argument");
    return FEB_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t nnode = (int64_t)(grid->nx + 1) * (grid->ny + 1) * (grid->nz + 1);
  if (nnode_total < nnode || (nnode_total > nnode && !orig)) {
    set_last_error("feb_relative_displacement: nnode_total below the grid nodes, or copies without orig");
    return FEB_ERR_ARG;
  }
  DevGeom D;
  FEB_TRY(make_dev_geom(grid, D, s));
  double* f = nullptr;
  FEB_CUDA(cudaMallocAsync((void**)&f, 9 * sizeof(double), s));
  FEB_CUDA(cudaMemcpyAsync(f, fit, 9 * sizeof(double), cudaMemcpyHostToDevice, s));
  k_relative<<<div_up(nnode_total, kThreads), kThreads, 0, s>>>(D.G, orig, nnode, nnode_total, U, f, out); note_launch();
  FEB_CUDA(cudaGetLastError());
  FEB_CUDA(cudaFreeAsync(f, s));
  FEB_CUDA(cudaFreeAsync(D.buf, s));
  FEB_CUDA(cudaStreamSynchronize(s));   // fit (host) may be released by the caller after return
  return FEB_OK;
}

extern "C" int feb_sample_cells(const FebGrid* grid, int32_t mx, int32_t my, int32_t mz, int32_t sub,
                                const int32_t* ix, const double* tx, const uint8_t* inx, const int32_t* iy,
                                const double* ty, const uint8_t* iny, const int32_t* iz, const double* tz,
                                const uint8_t* inz, const int64_t* cn, const uint8_t* active, const double* Urel,
                                const float* VM, const float* SIG, float* vm_out, float* u_out, float* frac_out,
                                float* sig_out, void* stream) {
  if (!grid || mx < 1 || my < 1 || mz < 1 || sub < 1 || !ix || !tx || !inx || !iy || !ty || !iny || !iz || !tz ||
      !inz || !active || !Urel || !VM || !SIG || !vm_out || !u_out || !frac_out || !sig_out) {
    set_last_error("feb_sample_cells: bad argument");
    return FEB_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  DevGeom D;
  FEB_TRY(make_dev_geom(grid, D, s));
  const int64_t n = (int64_t)mx * my * mz;
  k_sample_cells<<<div_up(n, kThreads), kThreads, 0, s>>>(D.G, mx, my, mz, sub, ix, tx, inx, iy, ty, iny, iz, tz, inz,
                                                         cn, active, Urel, VM, SIG, vm_out, u_out, frac_out, sig_out);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  FEB_CUDA(cudaFreeAsync(D.buf, s));
  return FEB_OK;
}

extern "C" int feb_nearest_active(const FebGrid* grid, const uint8_t* active, int32_t* ft, void* stream) {
  if (!grid || !active || !ft || grid->nx < 1 || grid->ny < 1 || grid->nz < 1) {
    set_last_error("feb_nearest_active: bad argument");
    return FEB_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int nx = grid->nx, ny = grid->ny, nz = grid->nz;
  const int64_t ncell = (int64_t)nx * ny * nz;
  int32_t *FI = nullptr, *FJ = nullptr, *sp = nullptr, *sa = nullptr, *sb = nullptr;
  int64_t* sg = nullptr;
  FEB_CUDA(cudaMallocAsync((void**)&FI, ncell * sizeof(int32_t), s));
  FEB_CUDA(cudaMallocAsync((void**)&FJ, ncell * sizeof(int32_t), s));
  FEB_CUDA(cudaMallocAsync((void**)&sp, ncell * sizeof(int32_t), s));
  FEB_CUDA(cudaMallocAsync((void**)&sa, ncell * sizeof(int32_t), s));
  FEB_CUDA(cudaMallocAsync((void**)&sb, ncell * sizeof(int32_t), s));
  FEB_CUDA(cudaMallocAsync((void**)&sg, ncell * sizeof(int64_t), s));
  const int64_t lines[3] = {(int64_t)ny * nz, (int64_t)nx * nz, (int64_t)nx * ny};
  for (int pass = 0; pass < 3; ++pass) {
    k_ft_pass<<<div_up(lines[pass], 128), 128, 0, s>>>(pass, nx, ny, nz, active, FI, FJ, ft, sp, sg, sa, sb);
    note_launch();
  }
  FEB_CUDA(cudaGetLastError());
  for (void* p : {(void*)FI, (void*)FJ, (void*)sp, (void*)sa, (void*)sb, (void*)sg}) FEB_CUDA(cudaFreeAsync(p, s));
  return FEB_OK;
}

extern "C" int feb_sample_nodes(const FebGrid* grid, int32_t mx1, int32_t my1, int32_t mz1, const int32_t* ix,
                                const double* px, const int32_t* iy, const double* py, const int32_t* iz,
                                const double* pz, const int32_t* ft, const int64_t* cn, const double* Urel, float* out,
                                void* stream) {
  if (!grid || mx1 < 1 || my1 < 1 || mz1 < 1 || !ix || !px || !iy || !py || !iz || !pz || !ft || !Urel || !out) {
    set_last_error("feb_sample_nodes: bad argument");
    return FEB_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  DevGeom D;
  FEB_TRY(make_dev_geom(grid, D, s));
  const int64_t n = (int64_t)mx1 * my1 * mz1;
  k_sample_nodes<<<div_up(n, kThreads), kThreads, 0, s>>>(D.G, mx1, my1, mz1, ix, px, iy, py, iz, pz, ft, cn, Urel, out);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  FEB_CUDA(cudaFreeAsync(D.buf, s));
  return FEB_OK;
}
