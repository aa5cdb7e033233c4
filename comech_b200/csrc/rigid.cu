// Additive rigid-body-mode correction z += Z pinv(Z^T K Z) Z^T r (fe/gmg.py:127-135, rb/gpusolve.py:216-228).
// Z has 6 columns per node group (3 translations, rotations about x, y, z with r = (X - mean X) / 20,
// rb/splitfe.py:105-120); its entries are recomputed from the grid coordinates, never stored.
#include "rigid.cuh"

namespace feb {

namespace {

__device__ __forceinline__ void node_xyz(const RigidView& Z, int64_t node, double& x, double& y, double& z) {
  int64_t o = node < Z.nnode ? node : (int64_t)Z.orig_copy[node - Z.nnode];
  int i = int(o % Z.nxn), j = int((o / Z.nxn) % Z.nyn), k = int(o / ((int64_t)Z.nxn * Z.nyn));
  x = Z.xe[i]; y = Z.ye[j]; z = Z.ze[k];
}

// mode m of a node with offset rho = (X - c) / 20: translations e_m, rotations (0,-rz,ry) (rz,0,-rx) (-ry,rx,0)
__device__ __forceinline__ void mode_vec(int m, double rx, double ry, double rz, double (&v)[3]) {
  v[0] = v[1] = v[2] = 0.0;
  switch (m) {
    case 0: v[0] = 1.0; break;
    case 1: v[1] = 1.0; break;
    case 2: v[2] = 1.0; break;
    case 3: v[1] = -rz; v[2] = ry; break;
    case 4: v[0] = rz; v[2] = -rx; break;
    default: v[0] = -ry; v[1] = rx; break;
  }
}

__global__ void k_centroids(RigidView Z, double* __restrict__ cen) {
  const int g = blockIdx.x;
  double sx = 0, sy = 0, sz = 0;
  for (int e = Z.off[g] + threadIdx.x; e < Z.off[g + 1]; e += blockDim.x) {
    double x, y, z;
    node_xyz(Z, Z.nodes[e], x, y, z);
    sx += x; sy += y; sz += z;
  }
  sx = block_sum(sx);
  __syncthreads();
  sy = block_sum(sy);
  __syncthreads();
  sz = block_sum(sz);
  if (threadIdx.x == 0) {
    double n = double(Z.off[g + 1] - Z.off[g]);
    cen[3 * g] = sx / n; cen[3 * g + 1] = sy / n; cen[3 * g + 2] = sz / n;
  }
}

// partial Z^T r: grid (blocks per group, groups); out[g][blk][6]
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_ztr_partial(RigidView Z, const T* __restrict__ r, double* __restrict__ part, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int g = blockIdx.y;
  double s[6] = {0, 0, 0, 0, 0, 0};
  const double cx = Z.cen[3 * g], cy = Z.cen[3 * g + 1], cz = Z.cen[3 * g + 2];
  for (int e = Z.off[g] + blockIdx.x * kThreads + threadIdx.x; e < Z.off[g + 1]; e += gridDim.x * kThreads) {
    int64_t n = Z.nodes[e];
    double x, y, z;
    node_xyz(Z, n, x, y, z);
    double rx = (x - cx) / 20.0, ry = (y - cy) / 20.0, rz = (z - cz) / 20.0;
    double r0 = double(r[3 * n]), r1 = double(r[3 * n + 1]), r2 = double(r[3 * n + 2]);
    s[0] += r0; s[1] += r1; s[2] += r2;
    s[3] += -rz * r1 + ry * r2;
    s[4] += rz * r0 - rx * r2;
    s[5] += -ry * r0 + rx * r1;
  }
  for (int m = 0; m < 6; ++m) {
    double v = block_sum(s[m]);
    if (threadIdx.x == 0) part[((size_t)g * gridDim.x + blockIdx.x) * 6 + m] = v;
    __syncthreads();
  }
}

// coef = Einv (Z^T r); one block
__global__ void k_ztr_finish(RigidView Z, int nblk, const double* __restrict__ part, const double* __restrict__ Einv,
                             double* __restrict__ zr, double* __restrict__ coef, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int nc = 6 * Z.ngroups;
  for (int t = threadIdx.x; t < nc; t += blockDim.x) {
    int g = t / 6, m = t % 6;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += part[((size_t)g * nblk + b) * 6 + m];
    zr[t] = s;
  }
  __syncthreads();
  if (Einv == nullptr) return;
  for (int t = threadIdx.x; t < nc; t += blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < nc; ++q) s += Einv[(size_t)t * nc + q] * zr[q];
    coef[t] = s;
  }
}

// z += Z coef
template <typename T>
__global__ void k_z_scatter(RigidView Z, const double* __restrict__ coef, T* __restrict__ z,
                            const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int g = blockIdx.y;
  const double cx = Z.cen[3 * g], cy = Z.cen[3 * g + 1], cz = Z.cen[3 * g + 2];
  const double* c = coef + 6 * g;
  for (int e = Z.off[g] + blockIdx.x * blockDim.x + threadIdx.x; e < Z.off[g + 1]; e += gridDim.x * blockDim.x) {
    int64_t n = Z.nodes[e];
    double x, y, zz;
    node_xyz(Z, n, x, y, zz);
    double rx = (x - cx) / 20.0, ry = (y - cy) / 20.0, rz = (zz - cz) / 20.0;
    double v0 = c[0] + c[4] * rz - c[5] * ry;
    double v1 = c[1] - c[3] * rz + c[5] * rx;
    double v2 = c[2] + c[3] * ry - c[4] * rx;
    atomic_add(z + 3 * n, T(v0));
    atomic_add(z + 3 * n + 1, T(v1));
    atomic_add(z + 3 * n + 2, T(v2));
  }
}

// column `col` of Z as a full-layout vector (zeroed beforehand)
__global__ void k_z_column(RigidView Z, int col, double* __restrict__ v) {
  const int g = col / 6, m = col % 6;
  const double cx = Z.cen[3 * g], cy = Z.cen[3 * g + 1], cz = Z.cen[3 * g + 2];
  for (int e = Z.off[g] + blockIdx.x * blockDim.x + threadIdx.x; e < Z.off[g + 1]; e += gridDim.x * blockDim.x) {
    int64_t n = Z.nodes[e];
    double x, y, z;
    node_xyz(Z, n, x, y, z);
    double w[3];
    mode_vec(m, (x - cx) / 20.0, (y - cy) / 20.0, (z - cz) / 20.0, w);
    v[3 * n] += w[0]; v[3 * n + 1] += w[1]; v[3 * n + 2] += w[2];
  }
}

}  // namespace

int rigid_blocks(const RigidView& Z) { (void)Z; return 2 * kSmCount / 4; }

void launch_centroids(const RigidView& Z, double* cen, cudaStream_t s) {
  k_centroids<<<Z.ngroups, kThreads, 0, s>>>(Z, cen); note_launch();
}

template <typename T>
void launch_rigid_apply(const RigidView& Z, const T* r, T* z, double* part, double* zr, double* coef,
                        const double* Einv, const int* skip, cudaStream_t s) {
  int nb = rigid_blocks(Z);
  dim3 g(nb, Z.ngroups);
  k_ztr_partial<T><<<g, kThreads, 0, s>>>(Z, r, part, skip); note_launch();
  k_ztr_finish<<<1, kThreads, 0, s>>>(Z, nb, part, Einv, zr, coef, skip); note_launch();
  if (Einv) k_z_scatter<T><<<g, kThreads, 0, s>>>(Z, coef, z, skip); note_launch();
}

void launch_ztr(const RigidView& Z, const double* r, double* part, double* zr, cudaStream_t s) {
  int nb = rigid_blocks(Z);
  dim3 g(nb, Z.ngroups);
  k_ztr_partial<double><<<g, kThreads, 0, s>>>(Z, r, part, nullptr); note_launch();
  k_ztr_finish<<<1, kThreads, 0, s>>>(Z, nb, part, nullptr, zr, nullptr, nullptr); note_launch();
}

void launch_z_column(const RigidView& Z, int col, double* v, cudaStream_t s) {
  dim3 g(rigid_blocks(Z));
  k_z_column<<<g, kThreads, 0, s>>>(Z, col, v); note_launch();
}

template void launch_rigid_apply<float>(const RigidView&, const float*, float*, double*, double*, double*,
                                        const double*, const int*, cudaStream_t);
template void launch_rigid_apply<double>(const RigidView&, const double*, double*, double*, double*, double*,
                                         const double*, const int*, cudaStream_t);

}  // namespace feb
