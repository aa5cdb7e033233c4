// Level-0 K.u of the regular cells on the 5th-generation tensor cores (tcgen05), FP32 operator.
//
// For equal cubic cells of edge h the element matrices of the isotropic models are h times fixed matrices
// whose entries are integers over 72 (2x2x2 mu part and full lambda part) or the outer product s s^T / 16 of
// the centre divergence row s in {-1, +1}^24 (one-point lambda part, rb/splitfe.py:58-69).  Those integers
// (|.| <= 32) are exact in BF16, so the element contraction is an exact BF16 tensor-core product once u is
// split into three BF16 slices u = u0 + u1 + u2 (u1, u2 the rounding remainders; together ~24 significant
// bits): D[cell][n] = sum_k (u0 + u1 + u2)[cell][k] B[n][k], accumulated in FP32 in the tensor memory.  The
// per-cell material and the factor h enter in the epilogue: f = (h mu / 72) D_mu + lambda term.
//
// Tiling.  A CTA owns 31 x 15 grid nodes of a node-plane chunk [z0, z1) and computes the 32 x 16 cells
// touching them, layer by layer in z.  One MMA (M = 128) covers 4 cell rows x 32 cells; row m = 32 w + i is
// cell i of row w.  Its A operand is read straight from the staged node planes: a K-major, unswizzled
// layout of 16-byte "pair-words" (nodes i and i+1 of one node row, components c0 c1 c2 and a zero pad, one
// BF16 slice); K-chunk 0 of row m is the pair-word of node row w, K-chunk 1 the pair-word of node row w + 1
// (leading-dimension offset = one node row), so K = 16 covers the 4 nodes of one cell face.  Per cell row
// group and layer: 2 faces (planes k, k+1) x 3 slices = 6 MMAs of M128 x N x K16 into one TMEM accumulator.
//
// Pipeline (256 threads, all warps do everything but issue): node planes live in a ring of 3 shared-memory
// slots; iteration `it` issues the MMAs of layer z0-1+it (thread 0, completion on an mbarrier), then every
// warp waits for the previous layer's MMAs, stages plane z0+1+it into the slot they freed, and runs the
// epilogue of the previous layer from the other TMEM buffer: TMEM -> registers, material scaling, x-sums by
// warp shuffles, y-sums through shared memory, z-sums in registers carried to the next layer, and one
// store per owned node.  The tensor cores work on layer k while the SIMT pipes do layer k-1.
#include <cuda_bf16.h>

#include "fine.cuh"
#include "tcgen05.cuh"

namespace feb {

namespace {

using namespace tc;

constexpr int kRows = 8;                        // cell rows per CTA: 2 MMA groups of 4 rows x 32 cells
constexpr int kGroups = kRows / 4;
constexpr int kNodeRows = kRows + 1;
constexpr int kSlices = 3;
constexpr int kThreadsTc = 128;                 // 4 warps; warp q reads TMEM lane quarter q
constexpr int kWarpsTc = kThreadsTc / 32;
constexpr int kStageRows = (kNodeRows + kWarpsTc - 1) / kWarpsTc;   // node rows a warp stages per plane
constexpr int kRowBytes = 32 * 16;              // one node row of pair-words
constexpr int kSliceBytes = kNodeRows * kRowBytes;
constexpr int kPlaneBytes = kSlices * kSliceBytes;
constexpr int kXchBytes = 2 * kRows * 6 * 32 * 4;   // y exchange, double-buffered by layer

template <int MODE> struct TcCols { static constexpr int value = (MODE == MAT_ISO_SRI) ? 32 : 48; };

constexpr size_t tc_smem_bytes(int ncol) { return (size_t)3 * kPlaneBytes + 64 * (size_t)ncol + kXchBytes + 32; }

// three BF16 slices of a node's (c0, c1, c2): per slice two 32-bit words (c0 c1) and (c2, 0)
__device__ __forceinline__ void split3(float a, float b, float c, uint32_t (&lo)[kSlices], uint32_t (&hi)[kSlices]) {
#pragma unroll
  for (int s = 0; s < kSlices; ++s) {
    const __nv_bfloat162 p = __floats2bfloat162_rn(a, b);
    const __nv_bfloat16 q = __float2bfloat16_rn(c);
    lo[s] = *reinterpret_cast<const uint32_t*>(&p);
    hi[s] = (uint32_t)(*reinterpret_cast<const unsigned short*>(&q));
    a -= __low2float(p);
    b -= __high2float(p);
    c -= __bfloat162float(q);
  }
}

// One node plane of this warp's node rows, held in registers between its load and its staging.
struct PlaneRegs {
  float v[kStageRows][3];
  float nb[kStageRows][3];     // lane 31: the node after the last one of the row (x0 + 32)
};

// node plane p (any index; outside the grid: zeros) -> registers
__device__ __forceinline__ void load_plane(PlaneRegs& R, int p, const FineView<float>& F,
                                           const float* __restrict__ u, int x0, int j0, int warp, int lane) {
  const bool pin = p >= 0 && p < F.nzn;
  const int x = x0 + lane;
#pragma unroll
  for (int t = 0; t < kStageRows; ++t) {
    const int r = warp + kWarpsTc * t, j = j0 + r;
    const bool rin = pin && r < kNodeRows && j >= 0 && j < F.nyn;
    const int64_t row = (int64_t)F.nxn * (j + (int64_t)F.nyn * p);
    R.v[t][0] = R.v[t][1] = R.v[t][2] = 0.f;
    R.nb[t][0] = R.nb[t][1] = R.nb[t][2] = 0.f;
    if (rin && x >= 0 && x < F.nxn) {
      const float* q = u + 3 * (row + x);
      R.v[t][0] = q[0]; R.v[t][1] = q[1]; R.v[t][2] = q[2];
    }
    if (lane == 31 && rin && x + 1 < F.nxn) {
      const float* q = u + 3 * (row + x + 1);
      R.nb[t][0] = q[0]; R.nb[t][1] = q[1]; R.nb[t][2] = q[2];
    }
  }
}

// registers of plane p -> its ring slot: three BF16 slices of pair-words (node i, node i+1)
__device__ __forceinline__ void store_plane(const PlaneRegs& R, unsigned char* planes, int p, int warp, int lane) {
  unsigned char* slot = planes + ((p % 3 + 3) % 3) * kPlaneBytes;
#pragma unroll
  for (int t = 0; t < kStageRows; ++t) {
    const int r = warp + kWarpsTc * t;
    if (r >= kNodeRows) break;                 // warp-uniform
    uint32_t lo[kSlices], hi[kSlices], lon[kSlices], hin[kSlices];
    split3(R.v[t][0], R.v[t][1], R.v[t][2], lo, hi);
    split3(R.nb[t][0], R.nb[t][1], R.nb[t][2], lon, hin);
#pragma unroll
    for (int s = 0; s < kSlices; ++s) {
      uint32_t nlo = __shfl_down_sync(0xffffffffu, lo[s], 1), nhi = __shfl_down_sync(0xffffffffu, hi[s], 1);
      if (lane == 31) { nlo = lon[s]; nhi = hin[s]; }
      *reinterpret_cast<uint4*>(slot + s * kSliceBytes + r * kRowBytes + lane * 16) = make_uint4(lo[s], hi[s], nlo, nhi);
    }
  }
}

// (lambda, mu) of this lane's cell in cell row r of the tile, layer kl (zero outside the grid)
__device__ __forceinline__ float2 load_cell(const FineView<float>& F, int x, int j, int kl) {
  if (x >= 0 && x < F.nx && j >= 0 && j < F.ny && kl >= 0 && kl < F.nz)
    return *reinterpret_cast<const float2*>(F.mat + 2 * (x + (int64_t)F.nx * (j + (int64_t)F.ny * kl)));
  return make_float2(0.f, 0.f);
}

template <int MODE>
__global__ void __launch_bounds__(kThreadsTc, 4)
k_fine_tc(FineView<float> F, const uint4* __restrict__ btab, const float* __restrict__ u, float* __restrict__ y,
          const int* __restrict__ skip, int zchunk) {
  if (skip && *skip) return;
  constexpr int N = TcCols<MODE>::value;
  constexpr uint32_t kCols = (2 * kGroups * N <= 128) ? 128 : 256;
  extern __shared__ __align__(128) unsigned char smem[];
  unsigned char* planes = smem;
  uint4* bsm = reinterpret_cast<uint4*>(smem + 3 * kPlaneBytes);
  float* xch = reinterpret_cast<float*>(smem + 3 * kPlaneBytes + 64 * N);
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + 3 * kPlaneBytes + 64 * N + kXchBytes);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + 2);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int x0 = blockIdx.x * 31 - 1, j0 = blockIdx.y * (kRows - 1) - 1;
  const int z0 = blockIdx.z * zchunk, z1 = min(z0 + zchunk, F.nzn);
  const int L = z1 - z0 + 1;                   // layers z0-1 .. z1-1

  for (int e = tid; e < 4 * N; e += kThreadsTc) bsm[e] = btab[e];
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar + 1)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(tslot)), "r"(kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  PlaneRegs pf;
  load_plane(pf, z0 - 1, F, u, x0, j0, warp, lane);
  store_plane(pf, planes, z0 - 1, warp, lane);
  load_plane(pf, z0, F, u, x0, j0, warp, lane);
  store_plane(pf, planes, z0, warp, lane);
  load_plane(pf, z0 + 1, F, u, x0, j0, warp, lane);      // staged in iteration 0
  const int xc = x0 + lane;                                // this lane's cell / node column
  float2 mat[kGroups];
#pragma unroll
  for (int g = 0; g < kGroups; ++g) mat[g] = load_cell(F, xc, j0 + 4 * g + warp, z0 - 1);
  sync_for_tensor_core();
  const uint32_t tmem = *tslot;

  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((128u >> 4) << 24);
  const uint32_t pbase = smem_addr(planes), bbase = smem_addr(bsm);
  const float hmu = F.tc_hmu, hlam = F.tc_hlam;
  float carry[kGroups][3];
  float g0[kGroups][6];
#pragma unroll
  for (int g = 0; g < kGroups; ++g) {
    carry[g][0] = carry[g][1] = carry[g][2] = 0.f;
#pragma unroll
    for (int e = 0; e < 6; ++e) g0[g][e] = 0.f;
  }
  bool ok = true;

  for (int it = 0; it <= L + 1; ++it) {
    const int k = z0 - 1 + it;                 // layer whose MMAs this iteration issues
    if (it < L && tid == 0 && ok) {
#pragma unroll
      for (int g = 0; g < kGroups; ++g) {
        const uint32_t dcol = tmem + (uint32_t)(((it & 1) * kGroups + g) * N);
        int acc = 0;
#pragma unroll
        for (int cz = 0; cz < 2; ++cz) {
          const int slot = ((k + cz) % 3 + 3) % 3;
          const uint64_t bd = smem_desc(bbase + cz * 2 * N * 16, N * 16, 128);
#pragma unroll
          for (int s = 0; s < kSlices; ++s) {
            const uint64_t ad = smem_desc(pbase + slot * kPlaneBytes + s * kSliceBytes + 4 * g * kRowBytes, kRowBytes, 128);
            mma_bf16(dcol, ad, bd, idesc, acc);
            acc = 1;
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_addr(mbar + (it & 1)))
                   : "memory");
    }
    if (it >= 1 && it <= L && ok) {
      ok = __all_sync(0xffffffffu, mbar_wait(smem_addr(mbar + ((it - 1) & 1)), (uint32_t)(((it - 1) >> 1) & 1)));
      if (!ok && lane == 0 && F.tc_status) atomicExch(F.tc_status, 1);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    }
    // plane k+2 into the slot the MMAs of layer k-1 have released; the loads of plane k+3 then overlap the rest
    if (it <= L - 2 && ok) store_plane(pf, planes, k + 2, warp, lane);
    if (it + 1 <= L - 2) load_plane(pf, k + 3, F, u, x0, j0, warp, lane);
    // finalize layer k-2: y-sums from the exchange written last iteration, z-sum with the carried part
    if (it >= 2) {
      const int kl = k - 2;
      const float* xin = xch + ((it - 1) & 1) * (kRows * 6 * 32);
#pragma unroll
      for (int g = 0; g < kGroups; ++g) {
        const int r = 4 * g + warp, jn = j0 + r;
        float v[6];
#pragma unroll
        for (int e = 0; e < 6; ++e) v[e] = g0[g][e] + (r >= 1 ? xin[((r - 1) * 6 + e) * 32 + lane] : 0.f);
        if (lane >= 1 && xc < F.nxn && r >= 1 && jn < F.nyn && kl >= z0 && kl < z1) {
          float* dst = y + 3 * (xc + (int64_t)F.nxn * (jn + (int64_t)F.nyn * kl));
          dst[0] = v[0] + carry[g][0];
          dst[1] = v[1] + carry[g][1];
          dst[2] = v[2] + carry[g][2];
        }
        carry[g][0] = v[3]; carry[g][1] = v[4]; carry[g][2] = v[5];
      }
    }
    // epilogue of layer k-1: TMEM -> element forces -> x-sums; the next-row halves go to the exchange
    if (it >= 1 && it <= L) {
      float* xout = xch + (it & 1) * (kRows * 6 * 32);
#pragma unroll
      for (int g = 0; g < kGroups; ++g) {
        const int r = 4 * g + warp;
        float D[32], f[24];
        const uint32_t taddr = tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)((((it - 1) & 1) * kGroups + g) * N);
        if (ok) {
          tmem_ld32(taddr, D);
        } else {
#pragma unroll
          for (int n = 0; n < 32; ++n) D[n] = 0.f;
        }
        const float al = mat[g].y * hmu;
        if constexpr (MODE == MAT_ISO_SRI) {
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          const float bd = mat[g].x * hlam * D[24];
#pragma unroll
          for (int n = 0; n < 24; ++n) f[n] = fmaf(al, D[n], (((n / 3) >> (n % 3)) & 1) ? bd : -bd);
        } else {
          float E[16];
          if (ok) {
            tmem_ld16(taddr + 32, E);
          } else {
#pragma unroll
            for (int n = 0; n < 16; ++n) E[n] = 0.f;
          }
          asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
          const float bl = mat[g].x * hlam;
#pragma unroll
          for (int n = 0; n < 24; ++n) f[n] = fmaf(al, D[n], bl * (n + 24 < 32 ? D[n + 24] : E[n - 8]));
        }
#pragma unroll
        for (int b = 0; b < 2; ++b)
#pragma unroll
          for (int cz = 0; cz < 2; ++cz)
#pragma unroll
            for (int c = 0; c < 3; ++c) {
              const float from_left = __shfl_up_sync(0xffffffffu, f[3 * (1 + 2 * b + 4 * cz) + c], 1);
              const float v = f[3 * (2 * b + 4 * cz) + c] + from_left;
              if (b == 0) g0[g][3 * cz + c] = v;
              else xout[(r * 6 + 3 * cz + c) * 32 + lane] = v;
            }
        mat[g] = load_cell(F, xc, j0 + r, k);   // the next epilogue's layer
      }
    }
    sync_for_tensor_core();
  }
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kCols));
}

// K_lambda and K_mu (24 x 24, dof 3 l + c) of the unit cube with the material model's integration rule
template <int MODE>
__global__ void k_unit_element(double* __restrict__ out) {
  const int col = threadIdx.x;
  if (col >= 48) return;
  const int part = col / 24, dof = col % 24;
  double uc[3][8], f[3][8];
  for (int l = 0; l < 8; ++l)
    for (int c = 0; c < 3; ++c) uc[c][l] = (3 * l + c == dof) ? 1.0 : 0.0;
  double m[2] = {part == 0 ? 1.0 : 0.0, part == 1 ? 1.0 : 0.0};
  Material<double> mat = make_material<double, MODE>(m);
  hex8_apply(uc, 1.0, 1.0, 1.0, 1.0, 1.0, 1.0, mat, f);
  for (int l = 0; l < 8; ++l)
    for (int c = 0; c < 3; ++c) out[part * 576 + (3 * l + c) * 24 + dof] = f[c][l];
}

}  // namespace

template <int MODE>
int tc_columns() { return TcCols<MODE>::value; }

template <int MODE>
void launch_unit_element(double* out, cudaStream_t s) {
  k_unit_element<MODE><<<1, 64, 0, s>>>(out); note_launch();
}

template <int MODE>
cudaError_t prepare_fine_tc() {
  return cudaFuncSetAttribute(k_fine_tc<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)tc_smem_bytes(TcCols<MODE>::value));
}

template <int MODE>
void launch_fine_struct_tc(const FineView<float>& F, const float* u, float* y, const int* skip, int zchunk,
                           cudaStream_t s) {
  const int zc = zchunk > 0 ? zchunk : 16;
  dim3 grid(div_up(F.nxn, 31), div_up(F.nyn, kRows - 1), div_up(F.nzn, zc));
  k_fine_tc<MODE><<<grid, kThreadsTc, tc_smem_bytes(TcCols<MODE>::value), s>>>(
      F, reinterpret_cast<const uint4*>(F.tc_b), u, y, skip, zc);
  note_launch();
}

template int tc_columns<MAT_ISO_SRI>();
template int tc_columns<MAT_ISO_FULL>();
template void launch_unit_element<MAT_ISO_SRI>(double*, cudaStream_t);
template void launch_unit_element<MAT_ISO_FULL>(double*, cudaStream_t);
template cudaError_t prepare_fine_tc<MAT_ISO_SRI>();
template cudaError_t prepare_fine_tc<MAT_ISO_FULL>();
template void launch_fine_struct_tc<MAT_ISO_SRI>(const FineView<float>&, const float*, float*, const int*, int,
                                                  cudaStream_t);
template void launch_fine_struct_tc<MAT_ISO_FULL>(const FineView<float>&, const float*, float*, const int*, int,
                                                   cudaStream_t);

}  // namespace feb
