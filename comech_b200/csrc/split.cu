// Split-node connectivity between bones on the device (rb/splitfe.py:261-305, equal to :17-55), bit for bit:
//   * a grid node touched by active bone cells of two or more bones is split, one id per (node, bone);
//   * the lowest bone keeps the grid id; the other (node, bone) pairs get ids nnode, nnode+1, ... in ascending
//     (node, bone) order; orig maps every id to its grid node;
//   * a bone cell uses its own bone's id; an active joint / soft cell (part 0) at a split node uses the bone
//     with the largest share in the cell (first maximum in ascending bone order) when that share is positive,
//     else the bone with the most bone cells at the node (first maximum); inactive cells keep grid ids.
// Counts per (node, bone) live in a dense nnode x nb array (nb = bone ids + 1, a few).
#include <cub/cub.cuh>

#include "common.cuh"

namespace feb {

namespace {

__device__ __forceinline__ int64_t grid_corner(int nx, int ny, int nz, int64_t c, int l) {
  const int k = int(c % nz), j = int((c / nz) % ny), i = int(c / ((int64_t)nz * ny));
  return (i + (l & 1)) + (int64_t)(nx + 1) * ((j + ((l >> 1) & 1)) + (int64_t)(ny + 1) * (k + ((l >> 2) & 1)));
}

// multiplicity of every (node, bone) incidence of active bone cells
__global__ void k_split_count(int nx, int ny, int nz, const uint8_t* __restrict__ active,
                              const int32_t* __restrict__ part, int nb, int32_t* __restrict__ cnt) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= (int64_t)nx * ny * nz || !active[c]) return;
  const int p = part[c];
  if (p <= 0 || p >= nb) return;
#pragma unroll
  for (int l = 0; l < 8; ++l) atomicAdd(cnt + grid_corner(nx, ny, nz, c, l) * nb + p, 1);
}

// extra ids of a node: its bones with incidences, minus the lead one, when there are two or more
__global__ void k_split_extra(int64_t nnode, int nb, const int32_t* __restrict__ cnt, int32_t* __restrict__ extra) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  int k = 0;
  for (int b = 1; b < nb; ++b) k += cnt[n * nb + b] > 0;
  extra[n] = k >= 2 ? k - 1 : 0;
}

// orig of the copies: for node n with extra ids, ids nnode + first[n] ... in ascending bone order
__global__ void k_split_orig(int64_t nnode, int nb, const int32_t* __restrict__ cnt, const int32_t* __restrict__ extra,
                             const int64_t* __restrict__ first, int64_t* __restrict__ orig) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= nnode) return;
  orig[n] = n;
  if (extra[n] == 0) return;
  for (int q = 0; q < extra[n]; ++q) orig[nnode + first[n] + q] = n;
}

// id of (node, bone): the grid id for the lead bone of a split node, else nnode + first + rank - 1
__device__ __forceinline__ int64_t split_id(int64_t node, int bone, int nb, int64_t nnode, const int32_t* cnt,
                                            const int64_t* first) {
  int rank = -1;
  for (int b = 1; b <= bone; ++b) rank += cnt[node * nb + b] > 0;
  return rank <= 0 ? node : nnode + first[node] + rank - 1;
}

__global__ void k_split_cn(int nx, int ny, int nz, const uint8_t* __restrict__ active, const int32_t* __restrict__ part,
                           const double* __restrict__ share, int nb, const int32_t* __restrict__ cnt,
                           const int32_t* __restrict__ extra, const int64_t* __restrict__ first,
                           int64_t* __restrict__ cn) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= (int64_t)nx * ny * nz) return;
  const int64_t nnode = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
  for (int l = 0; l < 8; ++l) {
    const int64_t node = grid_corner(nx, ny, nz, c, l);
    int64_t id = node;
    if (active[c] && extra[node] > 0) {
      int bone = part[c];
      if (bone <= 0) {
        // among the node's bones (ascending): largest share in the cell if positive, else most bone cells
        int by_share = -1, by_count = -1;
        double best_share = 0.0;
        int best_count = -1;
        bool any = false;
        for (int b = 1; b < nb; ++b) {
          const int m = cnt[node * nb + b];
          if (m <= 0) continue;
          const double sh = share[c * nb + b];
          if (!any || sh > best_share) { best_share = sh; by_share = b; }
          if (m > best_count) { best_count = m; by_count = b; }
          any = true;
        }
        bone = best_share > 0.0 ? by_share : by_count;
      }
      id = split_id(node, bone, nb, nnode, cnt, first);
    }
    cn[8 * c + l] = id;
  }
}

__global__ void k_count_positive(int64_t n, const int32_t* __restrict__ v, unsigned long long* __restrict__ out) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int one = (e < n && v[e] > 0) ? 1 : 0;
  const unsigned ballot = __ballot_sync(0xffffffffu, one);
  if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(out, (unsigned long long)__popc(ballot));
}

}  // namespace
}  // namespace feb

using namespace feb;

extern "C" int feb_split_connectivity(const FebGrid* grid, const uint8_t* active, const int32_t* part,
                                      const double* share, int32_t nb, int64_t* cn, int64_t* orig, int64_t orig_cap,
                                      int64_t* nnode_total, int64_t* nsplit, void* stream) {
  if (!grid || !active || !part || !share || !nnode_total || !nsplit || nb < 1 || (orig && !cn)) {
    set_last_error("feb_split_connectivity: bad argument");
    return FEB_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int nx = grid->nx, ny = grid->ny, nz = grid->nz;
  const int64_t ncell = (int64_t)nx * ny * nz, nnode = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
  int32_t *cnt = nullptr, *extra = nullptr;
  int64_t* first = nullptr;
  unsigned long long* nspl_d = nullptr;
  FEB_CUDA(cudaMallocAsync((void**)&cnt, (size_t)nnode * nb * sizeof(int32_t), s));
  FEB_CUDA(cudaMemsetAsync(cnt, 0, (size_t)nnode * nb * sizeof(int32_t), s));
  FEB_CUDA(cudaMallocAsync((void**)&extra, (size_t)(nnode + 1) * sizeof(int32_t), s));
  FEB_CUDA(cudaMemsetAsync(extra + nnode, 0, sizeof(int32_t), s));
  FEB_CUDA(cudaMallocAsync((void**)&first, (size_t)(nnode + 1) * sizeof(int64_t), s));
  FEB_CUDA(cudaMallocAsync((void**)&nspl_d, sizeof(unsigned long long), s));
  FEB_CUDA(cudaMemsetAsync(nspl_d, 0, sizeof(unsigned long long), s));
  k_split_count<<<div_up(ncell, kThreads), kThreads, 0, s>>>(nx, ny, nz, active, part, nb, cnt); note_launch();
  k_split_extra<<<div_up(nnode, kThreads), kThreads, 0, s>>>(nnode, nb, cnt, extra); note_launch();
  k_count_positive<<<div_up(nnode, kThreads), kThreads, 0, s>>>(nnode, extra, nspl_d); note_launch();
  // first[n]: extra ids of the nodes before n (first[nnode]: all of them)
  size_t tb = 0;
  FEB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, extra, first, nnode + 1, s));
  void* tmp = nullptr;
  FEB_CUDA(cudaMallocAsync(&tmp, tb, s));
  FEB_CUDA(cub::DeviceScan::ExclusiveSum(tmp, tb, extra, first, nnode + 1, s));
  int64_t ncopies = 0;
  unsigned long long nspl = 0;
  FEB_CUDA(cudaMemcpyAsync(&ncopies, first + nnode, sizeof(int64_t), cudaMemcpyDeviceToHost, s));
  FEB_CUDA(cudaMemcpyAsync(&nspl, nspl_d, sizeof(unsigned long long), cudaMemcpyDeviceToHost, s));
  FEB_CUDA(cudaStreamSynchronize(s));
  *nnode_total = nnode + ncopies;
  *nsplit = (int64_t)nspl;
  int st = FEB_OK;
  if (orig && orig_cap < nnode + ncopies) {
    set_last_error("feb_split_connectivity: orig holds %lld entries, %lld needed", (long long)orig_cap,
                   (long long)(nnode + ncopies));
    st = FEB_ERR_ARG;
  } else if (orig) {
    k_split_orig<<<div_up(nnode, kThreads), kThreads, 0, s>>>(nnode, nb, cnt, extra, first, orig); note_launch();
  }
  if (cn && st == FEB_OK) {
    k_split_cn<<<div_up(ncell, kThreads), kThreads, 0, s>>>(nx, ny, nz, active, part, share, nb, cnt, extra, first, cn);
    note_launch();
  }
  FEB_CUDA(cudaGetLastError());
  for (void* p : {(void*)tmp, (void*)cnt, (void*)extra, (void*)first, (void*)nspl_d}) FEB_CUDA(cudaFreeAsync(p, s));
  return st;
}
