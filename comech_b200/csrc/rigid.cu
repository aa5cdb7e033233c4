// Additive rigid-body-mode correction z += Z pinv(Z^T K Z) Z^T r (fe/gmg.py:127-135, rb/gpusolve.py:216-228).
// Z has 6 columns per node group (3 translations, rotations about x, y, z with r = (X - mean X) / 20,
// rb/splitfe.py:105-120); its entries are recomputed from the grid coordinates, never stored.
#include <algorithm>

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

// partial coordinate sums per group: grid (blocks per group, groups); part[g][blk][3]
__global__ void __launch_bounds__(kThreads) k_centroid_partial(RigidView Z, double* __restrict__ part) {
  const int g = blockIdx.y;
  double sx = 0, sy = 0, sz = 0;
  for (int e = Z.off[g] + blockIdx.x * kThreads + threadIdx.x; e < Z.off[g + 1]; e += gridDim.x * kThreads) {
    double x, y, z;
    node_xyz(Z, Z.nodes[e], x, y, z);
    sx += x; sy += y; sz += z;
  }
  double v[3] = {sx, sy, sz};
  for (int c = 0; c < 3; ++c) {
    double t = block_sum(v[c]);
    if (threadIdx.x == 0) part[((size_t)g * gridDim.x + blockIdx.x) * 3 + c] = t;
    __syncthreads();
  }
}

__global__ void k_centroid_finish(RigidView Z, int nblk, const double* __restrict__ part, double* __restrict__ cen) {
  int t = threadIdx.x;
  if (t >= 3 * Z.ngroups) return;
  int g = t / 3, c = t % 3;
  double s = 0.0;
  for (int b = 0; b < nblk; ++b) s += part[((size_t)g * nblk + b) * 3 + c];
  cen[t] = s / double(Z.off[g + 1] - Z.off[g]);
}

__global__ void k_rigid_rho(RigidView Z, double* __restrict__ rho) {
  const int g = blockIdx.y;
  const double cx = Z.cen[3 * g], cy = Z.cen[3 * g + 1], cz = Z.cen[3 * g + 2];
  for (int e = Z.off[g] + blockIdx.x * blockDim.x + threadIdx.x; e < Z.off[g + 1]; e += gridDim.x * blockDim.x) {
    double x, y, z;
    node_xyz(Z, Z.nodes[e], x, y, z);
    rho[3 * e] = (x - cx) / 20.0; rho[3 * e + 1] = (y - cy) / 20.0; rho[3 * e + 2] = (z - cz) / 20.0;
  }
}

// partial Z^T r: grid (blocks per group, groups); out[g][blk][6]
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_ztr_partial(RigidView Z, const T* __restrict__ r, double* __restrict__ part, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int g = blockIdx.y;
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (int e = Z.off[g] + blockIdx.x * kThreads + threadIdx.x; e < Z.off[g + 1]; e += gridDim.x * kThreads) {
    const int64_t n = Z.nodes[e];
    const double rx = Z.rho[3 * e], ry = Z.rho[3 * e + 1], rz = Z.rho[3 * e + 2];
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

// zr = Z^T r from the partials, coef = Einv zr (when Einv is given); run by one block
__device__ void ztr_finish(const RigidView& Z, int nblk, const double* part, const double* __restrict__ Einv,
                           double* __restrict__ zr, double* __restrict__ coef) {
  const int nc = 6 * Z.ngroups;
  for (int t = threadIdx.x; t < nc; t += blockDim.x) {
    int g = t / 6, m = t % 6;
    double s = 0.0;
    for (int b = 0; b < nblk; ++b) s += ((const volatile double*)part)[((size_t)g * nblk + b) * 6 + m];
    zr[t] = s;
  }
  __syncthreads();
  if (Einv == nullptr) return;
  for (int t = threadIdx.x; t < nc; t += blockDim.x) {
    double s = 0.0;
    for (int q = 0; q < nc; ++q) s += Einv[(size_t)t * nc + q] * ((const volatile double*)zr)[q];
    coef[t] = s;
  }
}

// k_ztr_partial with ztr_finish in the block that arrives last (counted on ctr after a fence that publishes
// the block's partials; the counter is re-armed for the next use)
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_ztr_fused(RigidView Z, const T* __restrict__ r, double* part, const double* __restrict__ Einv, double* zr,
            double* coef, unsigned int* ctr, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int g = blockIdx.y;
  double s[6] = {0, 0, 0, 0, 0, 0};
  for (int e = Z.off[g] + blockIdx.x * kThreads + threadIdx.x; e < Z.off[g + 1]; e += gridDim.x * kThreads) {
    const int64_t n = Z.nodes[e];
    const double rx = Z.rho[3 * e], ry = Z.rho[3 * e + 1], rz = Z.rho[3 * e + 2];
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
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ctr, 1u) == gridDim.x * gridDim.y - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  ztr_finish(Z, gridDim.x, part, Einv, zr, coef);
  if (threadIdx.x == 0) *ctr = 0u;
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
  const double* c = coef + 6 * g;
  for (int e = Z.off[g] + blockIdx.x * blockDim.x + threadIdx.x; e < Z.off[g + 1]; e += gridDim.x * blockDim.x) {
    const int64_t n = Z.nodes[e];
    const double rx = Z.rho[3 * e], ry = Z.rho[3 * e + 1], rz = Z.rho[3 * e + 2];
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
  for (int e = Z.off[g] + blockIdx.x * blockDim.x + threadIdx.x; e < Z.off[g + 1]; e += gridDim.x * blockDim.x) {
    const int64_t n = Z.nodes[e];
    double w[3];
    mode_vec(m, Z.rho[3 * e], Z.rho[3 * e + 1], Z.rho[3 * e + 2], w);
    v[3 * n] += w[0]; v[3 * n + 1] += w[1]; v[3 * n + 2] += w[2];
  }
}

}  // namespace

int rigid_blocks(const RigidView& Z) { (void)Z; return 2 * kSmCount / 4; }

void launch_centroids(const RigidView& Z, double* cen, double* part, cudaStream_t s) {
  int nb = rigid_blocks(Z);
  dim3 g(nb, Z.ngroups);
  k_centroid_partial<<<g, kThreads, 0, s>>>(Z, part); note_launch();
  k_centroid_finish<<<1, std::max(32, ((3 * Z.ngroups + 31) / 32) * 32), 0, s>>>(Z, nb, part, cen); note_launch();
}

template <typename T>
void launch_rigid_apply(const RigidView& Z, const T* r, T* z, double* part, double* zr, double* coef,
                        const double* Einv, const int* skip, cudaStream_t s, unsigned int* ctr) {
  int nb = rigid_blocks(Z);
  dim3 g(nb, Z.ngroups);
  if (ctr) {
    k_ztr_fused<T><<<g, kThreads, 0, s>>>(Z, r, part, Einv, zr, coef, ctr, skip); note_launch();
  } else {
    k_ztr_partial<T><<<g, kThreads, 0, s>>>(Z, r, part, skip); note_launch();
    k_ztr_finish<<<1, kThreads, 0, s>>>(Z, nb, part, Einv, zr, coef, skip); note_launch();
  }
  if (Einv) k_z_scatter<T><<<g, kThreads, 0, s>>>(Z, coef, z, skip); note_launch();
}

template <typename T>
void launch_rigid_coef(const RigidView& Z, const T* r, double* part, double* zr, double* coef, const double* Einv,
                       const int* skip, cudaStream_t s, unsigned int* ctr) {
  dim3 g(rigid_blocks(Z), Z.ngroups);
  k_ztr_fused<T><<<g, kThreads, 0, s>>>(Z, r, part, Einv, zr, coef, ctr, skip); note_launch();
}

template <typename T>
void launch_rigid_scatter(const RigidView& Z, const double* coef, T* z, const int* skip, cudaStream_t s) {
  dim3 g(rigid_blocks(Z), Z.ngroups);
  k_z_scatter<T><<<g, kThreads, 0, s>>>(Z, coef, z, skip); note_launch();
}

void launch_rigid_rho(const RigidView& Z, double* rho, cudaStream_t s) {
  dim3 g(rigid_blocks(Z), Z.ngroups);
  k_rigid_rho<<<g, kThreads, 0, s>>>(Z, rho); note_launch();
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
                                        const double*, const int*, cudaStream_t, unsigned int*);
template void launch_rigid_apply<double>(const RigidView&, const double*, double*, double*, double*, double*,
                                         const double*, const int*, cudaStream_t, unsigned int*);
template void launch_rigid_coef<float>(const RigidView&, const float*, double*, double*, double*, const double*,
                                       const int*, cudaStream_t, unsigned int*);
template void launch_rigid_coef<double>(const RigidView&, const double*, double*, double*, double*, const double*,
                                        const int*, cudaStream_t, unsigned int*);
template void launch_rigid_scatter<float>(const RigidView&, const double*, float*, const int*, cudaStream_t);
template void launch_rigid_scatter<double>(const RigidView&, const double*, double*, const int*, cudaStream_t);

}  // namespace feb
