// Stress / von Mises recovery and element forces (fe/solver.py:257-272, rb/splitfe.py:161-193),
// nodal accumulation of loads (rb/splitfe.py:144-147).
#include <mutex>

#include "element.cuh"

namespace feb {

namespace {

struct GridGeom {
  int nx, ny, nz;
  const double* dx; const double* dy; const double* dz;
};

// cell id (reference order, z fastest) -> 8 node ids
__device__ __forceinline__ void cell_nodes(const GridGeom& G, int64_t cell, const int64_t* cn, int64_t (&nd)[8],
                                           int& i, int& j, int& k) {
  k = int(cell % G.nz);
  j = int((cell / G.nz) % G.ny);
  i = int(cell / ((int64_t)G.nz * G.ny));
  const int64_t nx1 = G.nx + 1, ny1 = G.ny + 1;
#pragma unroll
  for (int l = 0; l < 8; ++l)
    nd[l] = cn ? cn[8 * cell + l] : (i + (l & 1)) + nx1 * ((j + ((l >> 1) & 1)) + ny1 * (k + ((l >> 2) & 1)));
}

__global__ void k_cell_stress(GridGeom G, int mode, const double* __restrict__ mat, int64_t ncell_total,
                              const double* __restrict__ U, int64_t ncells, const int64_t* __restrict__ cells,
                              const int64_t* __restrict__ cn, int nan_to_zero, double* __restrict__ sig,
                              double* __restrict__ vm, double* __restrict__ eps_out) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ncells) return;
  int64_t cell = cells[e];
  int64_t nd[8];
  int i, j, k;
  cell_nodes(G, cell, cn, nd, i, j, k);
  double u[3][8];
#pragma unroll
  for (int l = 0; l < 8; ++l)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double v = U[3 * nd[l] + c];
      u[c][l] = (nan_to_zero && isnan(v)) ? 0.0 : v;
    }
  double ep[6];
  hex8_centre_strain(u, 1.0 / G.dx[i], 1.0 / G.dy[j], 1.0 / G.dz[k], ep);
  double s[6];
  if (mode == MAT_ORTHO) {
    const double* c = mat + 6 * cell;
    s[0] = c[0] * ep[0] + c[1] * ep[1] + c[2] * ep[2];
    s[1] = c[1] * ep[0] + c[0] * ep[1] + c[2] * ep[2];
    s[2] = c[2] * ep[0] + c[2] * ep[1] + c[3] * ep[2];
    s[3] = c[4] * ep[3];
    s[4] = c[5] * ep[4];
    s[5] = c[5] * ep[5];
  } else {
    double lam = mat[cell], mu = mat[ncell_total + cell];
    double tr = ep[0] + ep[1] + ep[2];
    for (int q = 0; q < 3; ++q) s[q] = lam * tr + 2.0 * mu * ep[q];
    for (int q = 3; q < 6; ++q) s[q] = mu * ep[q];
  }
  double a = s[0] - s[1], b = s[1] - s[2], c = s[2] - s[0];
  vm[e] = sqrt(0.5 * (a * a + b * b + c * c) + 3.0 * (s[3] * s[3] + s[4] * s[4] + s[5] * s[5]));
  for (int q = 0; q < 6; ++q) sig[6 * e + q] = s[q];
  if (eps_out)
    for (int q = 0; q < 6; ++q) eps_out[6 * e + q] = ep[q];
}

__global__ void k_element_forces(GridGeom G, const double* __restrict__ mat, int64_t ncell_total,
                                 const double* __restrict__ U, int64_t ncells, const int64_t* __restrict__ cells,
                                 const int64_t* __restrict__ cn, double* __restrict__ out) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= ncells) return;
  int64_t cell = cells[e];
  int64_t nd[8];
  int i, j, k;
  cell_nodes(G, cell, cn, nd, i, j, k);
  double u[3][8], f[3][8];
#pragma unroll
  for (int l = 0; l < 8; ++l)
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double v = U[3 * nd[l] + c];
      u[c][l] = isnan(v) ? 0.0 : v;
    }
  double p[2] = {mat[cell], mat[ncell_total + cell]};
  Material<double> m = make_material<double, MAT_ISO_SRI>(p);
  double a = G.dx[i], b = G.dy[j], c = G.dz[k];
  hex8_apply(u, a, b, c, 1.0 / a, 1.0 / b, 1.0 / c, m, f);
#pragma unroll
  for (int l = 0; l < 8; ++l)
#pragma unroll
    for (int q = 0; q < 3; ++q) out[24 * e + 3 * l + q] = f[q][l];
}

__global__ void k_accumulate_nodal(int64_t n, const int64_t* __restrict__ nodes, const double* __restrict__ vals,
                                   double* __restrict__ dst) {
  int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n) return;
  int64_t node = nodes[e];
  for (int c = 0; c < 3; ++c) atomicAdd(dst + 3 * node + c, vals[3 * e + c]);
}

int make_geom(const FebGrid* grid, GridGeom& G, double** buf, cudaStream_t s) {
  G.nx = grid->nx; G.ny = grid->ny; G.nz = grid->nz;
  size_t n = (size_t)G.nx + G.ny + G.nz;
  double* h = (double*)malloc(n * sizeof(double));
  if (!h) return FEB_ERR_NOMEM;
  for (int i = 0; i < G.nx; ++i) h[i] = grid->xe[i + 1] - grid->xe[i];
  for (int j = 0; j < G.ny; ++j) h[G.nx + j] = grid->ye[j + 1] - grid->ye[j];
  for (int k = 0; k < G.nz; ++k) h[G.nx + G.ny + k] = grid->ze[k + 1] - grid->ze[k];
  cudaError_t e = cudaMallocAsync((void**)buf, n * sizeof(double), s);
  if (e == cudaSuccess) e = cudaMemcpyAsync(*buf, h, n * sizeof(double), cudaMemcpyHostToDevice, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  free(h);
  if (e != cudaSuccess) {
    set_last_error("grid upload: %s", cudaGetErrorString(e));
    return FEB_ERR_CUDA;
  }
  G.dx = *buf; G.dy = *buf + G.nx; G.dz = *buf + G.nx + G.ny;
  return FEB_OK;
}

}  // namespace

}  // namespace feb

using namespace feb;

extern "C" int feb_cell_stress(const FebGrid* grid, int32_t mat_mode, const double* mat, const double* U,
                               int64_t ncells, const int64_t* cells, const int64_t* cn, int32_t nan_to_zero,
                               double* sig, double* vm, double* eps, void* stream) {
  if (!grid || !mat || !U || !cells || !sig || !vm || ncells < 0) {
    set_last_error("feb_cell_stress: null argument");
    return FEB_ERR_ARG;
  }
  if (ncells == 0) return FEB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  GridGeom G;
  double* buf = nullptr;
  FEB_TRY(make_geom(grid, G, &buf, s));
  int64_t nct = (int64_t)grid->nx * grid->ny * grid->nz;
  k_cell_stress<<<div_up(ncells, kThreads), kThreads, 0, s>>>(G, mat_mode, mat, nct, U, ncells, cells, cn,
                                                              nan_to_zero, sig, vm, eps); note_launch();
  FEB_CUDA(cudaGetLastError());
  FEB_CUDA(cudaFreeAsync(buf, s));
  return FEB_OK;
}

extern "C" int feb_element_forces(const FebGrid* grid, const double* mat, const double* U, int64_t ncells,
                                  const int64_t* cells, const int64_t* cn, double* out, void* stream) {
  if (!grid || !mat || !U || !cells || !out || ncells < 0) {
    set_last_error("feb_element_forces: null argument");
    return FEB_ERR_ARG;
  }
  if (ncells == 0) return FEB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  GridGeom G;
  double* buf = nullptr;
  FEB_TRY(make_geom(grid, G, &buf, s));
  int64_t nct = (int64_t)grid->nx * grid->ny * grid->nz;
  k_element_forces<<<div_up(ncells, kThreads), kThreads, 0, s>>>(G, mat, nct, U, ncells, cells, cn, out); note_launch();
  FEB_CUDA(cudaGetLastError());
  FEB_CUDA(cudaFreeAsync(buf, s));
  return FEB_OK;
}

extern "C" int feb_accumulate_nodal(int64_t n, const int64_t* nodes, const double* vals, double* dst, void* stream) {
  if (n < 0 || (n > 0 && (!nodes || !vals || !dst))) {
    set_last_error("feb_accumulate_nodal: bad argument");
    return FEB_ERR_ARG;
  }
  if (n == 0) return FEB_OK;
  k_accumulate_nodal<<<div_up(n, kThreads), kThreads, 0, (cudaStream_t)stream>>>(n, nodes, vals, dst); note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

// ------------------------------------------------------------------------------------------------
// Allocation-free variant of feb_cell_stress.
//
// feb_cell_stress keeps the per-axis cell widths in a scratch buffer that it allocates on every call.
// Some callers cannot allocate device memory at the point where they need stresses: a host framework
// that hands the library a fixed memory arena and forbids allocations inside its step, an enqueue
// callback of a plugin interface, or a latency-critical loop in which cudaMalloc's implicit device
// synchronisation is unacceptable.  For them this variant keeps the scratch (grid edges and cell
// widths) in one file-scope device array of fixed size, so the call allocates nothing.
//
// Limits and contract:
//   * at most kNoAllocMaxCells cells along each axis (192 KB of device memory, held by every GPU that
//     loads the library until the process exits); larger grids are rejected with FEB_ERR_ARG;
//   * the first call on a device looks up the array's device address (cudaGetSymbolAddress) with that
//     device current, and caches it per device: make that first call before any stream capture;
//   * all calls share the one array and it keeps the last call's contents (every call overwrites all
//     of it that it reads), so calls whose work overlaps on the GPU race: order them on one stream.
namespace feb {
namespace {

constexpr int kNoAllocMaxCells = 4096;
constexpr int kNoAllocEdges = kNoAllocMaxCells + 1;
static __device__ __align__(256) double g_noalloc_scratch[3 * kNoAllocEdges + 3 * kNoAllocMaxCells];

constexpr int kMaxDevices = 64;
static std::mutex g_noalloc_mu;
static double* g_noalloc_ptr[kMaxDevices] = {};

// device address of g_noalloc_scratch on the current device (looked up once per device)
int noalloc_scratch(double** out) {
  int dev = -1;
  FEB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) {
    set_last_error("feb_cell_stress_noalloc: device %d out of range", dev);
    return FEB_ERR_ARG;
  }
  std::lock_guard<std::mutex> lock(g_noalloc_mu);
  if (g_noalloc_ptr[dev] == nullptr) {
    void* p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || p == nullptr) {
      set_last_error("feb_cell_stress_noalloc: cudaGetSymbolAddress: %s", cudaGetErrorString(e));
      return FEB_ERR_CUDA;
    }
    g_noalloc_ptr[dev] = (double*)p;
  }
  *out = g_noalloc_ptr[dev];
  return FEB_OK;
}

// widths[a][i] = edges[a][i+1] - edges[a][i] inside the scratch array
__global__ void k_noalloc_widths(const double* __restrict__ edges, double* __restrict__ widths, int nx, int ny,
                                 int nz) {
  int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int n[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) {
    if (t < n[a]) {
      const double* e = edges + a * kNoAllocEdges;
      widths[a * kNoAllocMaxCells + t] = e[t + 1] - e[t];
    }
  }
}

}  // namespace
}  // namespace feb

extern "C" int feb_cell_stress_noalloc(const FebGrid* grid, int32_t mat_mode, const double* mat, const double* U,
                                       int64_t ncells, const int64_t* cells, const int64_t* cn, int32_t nan_to_zero,
                                       double* sig, double* vm, double* eps, void* stream) {
  if (!grid || !grid->xe || !grid->ye || !grid->ze || !mat || !U || !cells || !sig || !vm || ncells < 0) {
    set_last_error("feb_cell_stress_noalloc: null argument");
    return FEB_ERR_ARG;
  }
  if (grid->nx < 1 || grid->ny < 1 || grid->nz < 1 || grid->nx > kNoAllocMaxCells || grid->ny > kNoAllocMaxCells ||
      grid->nz > kNoAllocMaxCells) {
    set_last_error("feb_cell_stress_noalloc: grid %d x %d x %d cells; this entry point supports 1..%d cells per axis",
                   grid->nx, grid->ny, grid->nz, kNoAllocMaxCells);
    return FEB_ERR_ARG;
  }
  double* scratch = nullptr;
  FEB_TRY(noalloc_scratch(&scratch));
  if (ncells == 0) return FEB_OK;
  cudaStream_t s = (cudaStream_t)stream;
  double* edges = scratch;
  double* widths = scratch + 3 * kNoAllocEdges;
  const double* src[3] = {grid->xe, grid->ye, grid->ze};
  const int n[3] = {grid->nx, grid->ny, grid->nz};
  for (int a = 0; a < 3; ++a)
    FEB_CUDA(cudaMemcpyAsync(edges + a * kNoAllocEdges, src[a], (n[a] + 1) * sizeof(double), cudaMemcpyHostToDevice, s));
  int mx = std::max(n[0], std::max(n[1], n[2]));
  k_noalloc_widths<<<div_up(mx, kThreads), kThreads, 0, s>>>(edges, widths, n[0], n[1], n[2]); note_launch();
  GridGeom G;
  G.nx = n[0]; G.ny = n[1]; G.nz = n[2];
  G.dx = widths; G.dy = widths + kNoAllocMaxCells; G.dz = widths + 2 * kNoAllocMaxCells;
  int64_t nct = (int64_t)n[0] * n[1] * n[2];
  k_cell_stress<<<div_up(ncells, kThreads), kThreads, 0, s>>>(G, mat_mode, mat, nct, U, ncells, cells, cn,
                                                              nan_to_zero, sig, vm, eps); note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}
