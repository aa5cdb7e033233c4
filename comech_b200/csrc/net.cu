// Learned warm start: the layers of a 3D convolutional encoder-decoder, its training steps, and its coupling to
// the solve (network input from the solve's inputs, targets from solutions, the initial guess from a prediction).
//
// Convolutions are implicit GEMMs on the 5th-generation tensor cores.  A CTA of 128 threads owns 128 output rows
// (256 for 3x3x3 convolutions, in two accumulators; rows are voxels of the padded grid) x NT output channels, its
// FP32 accumulators in tensor memory.  The K loop runs over (tap group, 32-channel slice): each step stages the
// gathered input rows x 32 channels (cp.async, zero fill for rows outside the grid) and the weight rows in a 3- or
// 4-slot shared-memory ring, in the K-major unswizzled core-matrix layout, and one thread issues the step's
// M128 x NT x K16 BF16 MMAs (2 per tap and accumulator) and commits them to the slot's mbarrier; the slot is
// refilled once those MMAs have completed, so loads run ahead of the tensor core.  The epilogue reads the
// accumulators back (tcgen05.ld), adds the bias, applies ReLU / the ReLU-gradient mask / accumulation, and stores
// BF16 rows (direct, or scattered to the 8 fine cells of a transposed stride-2 conv).
//
// Weight gradients (a reduction over voxels) use warp-level mma.sync with transposing ldmatrix loads of the
// row-major activation tiles, split over row chunks with FP32 atomics into the gradient.
#include <cuda_bf16.h>

#include <cfloat>

#include "common.cuh"
#include "element.cuh"
#include "tcgen05.cuh"

namespace feb {

namespace {

using bf16 = __nv_bfloat16;

constexpr int kConvThreads = 128;
constexpr int kKS = 32;                          // channels per K step slice (two K16 MMAs per tap)

// Shared-memory ring of the convolution.  A 3x3x3 (SHIFT) CTA owns 256 output rows (two M128 accumulators) and a
// step covers the three z taps of one (x, y) offset: the rows they read are one window of 258 rows (stored as 264)
// shifted by one row per tap, so one A tile serves the three taps and both halves through descriptors 16 bytes
// apart (12 MMAs per step), and B holds the three taps' weights.  Other gathers: 128 rows, one tap per step.
template <int NT, int GATHER> struct ConvSmem {
  static constexpr bool kZ3 = GATHER == FEB_GATHER_SHIFT;
  static constexpr int kM = kZ3 ? 256 : 128;     // output rows per CTA (kM / 128 accumulators of NT columns)
  static constexpr int kHalves = kM / 128;
  static constexpr int kARows = kZ3 ? kM + 8 : 128;
  static constexpr int kAHalf = kARows * 16;     // bytes between 8-channel core-matrix columns of A
  static constexpr int kA = kARows * kKS * 2;
  static constexpr int kTaps = kZ3 ? 3 : 1;      // taps per step
  static constexpr int kBTap = NT * kKS * 2;
  static constexpr int kB = kTaps * kBTap;
  static constexpr int kStage = kA + kB;
  static constexpr int kStages = kZ3 ? 3 : 4;    // 3x3x3: 3 slots keep 3 CTAs per SM at N = 32
  static constexpr size_t kTotal = (size_t)kStages * kStage + 8 * kStages + 16;
};

__device__ __forceinline__ void cp16(uint32_t dst, const void* src, int nbytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(dst), "l"(src), "r"(nbytes) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

__host__ __device__ __forceinline__ int64_t grid_rows(const FebNetGrid& g) {
  return (int64_t)(g.nx + 2) * (g.ny + 2) * (g.nz + 2);
}

__device__ __forceinline__ int64_t prow(const FebNetGrid& g, int x, int y, int z) {
  return ((int64_t)(x + 1) * (g.ny + 2) + (y + 1)) * (g.nz + 2) + (z + 1);
}

// cell of a row; false for shell rows and rows past the end
__device__ __forceinline__ bool row_cell(const FebNetGrid& g, int64_t r, int& x, int& y, int& z) {
  const int Pz = g.nz + 2, Py = g.ny + 2;
  z = int(r % Pz) - 1;
  const int64_t q = r / Pz;
  y = int(q % Py) - 1;
  x = int(q / Py) - 1;
  return x >= 0 && x < g.nx && y >= 0 && y < g.ny && z >= 0 && z < g.nz;
}

__device__ __forceinline__ int64_t shift_off(const FebNetGrid& g, int tap) {
  const int dx = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dz = tap % 3 - 1;
  return ((int64_t)dx * (g.ny + 2) + dy) * (g.nz + 2) + dz;
}

__device__ __forceinline__ int64_t fine_off(const FebNetGrid& f, int tap) {
  return ((int64_t)(tap >> 2) * (f.ny + 2) + ((tap >> 1) & 1)) * (f.nz + 2) + (tap & 1);
}

// one K step of A (gathered rows) and B (weights) into a ring slot.  SHIFT: step = ((x, y) offset p, channel slice),
// A row i = input row m0 - 1 + i + offset(p), B = the weights of taps 3p, 3p+1, 3p+2 (dz = -1, 0, +1).  DOWN / ONE:
// step = (tap, channel slice), A row i = the tap's source row of output row m0 + i.
template <int NT, int GATHER>
__device__ __forceinline__ void conv_load(const FebConv& P, int step, int kcs, uint32_t sA, int64_t m0, int64_t M,
                                          int64_t Pin, const int64_t (&fbase)[4], int n0, int tid) {
  using S = ConvSmem<NT, GATHER>;
  const int grp = step / kcs, c0 = (step - grp * kcs) * kKS;
  const bf16* in = reinterpret_cast<const bf16*>(P.in);
  if (GATHER == FEB_GATHER_SHIFT) {
    const int dx = grp / 3 - 1, dy = grp % 3 - 1;
    const int64_t off = ((int64_t)dx * (P.grid.ny + 2) + dy) * (P.grid.nz + 2);
    for (int e = tid; e < S::kARows * 4; e += kConvThreads) {
      const int row = e >> 2, ch = e & 3;
      int64_t src = m0 - 1 + row + off;
      if (row >= S::kM + 2 || src < 0 || src >= Pin) src = -1;
      const bf16* g = src >= 0 ? in + src * P.in_ld + P.in_c0 + c0 + ch * 8 : in;
      cp16(sA + ch * S::kAHalf + row * 16, g, src >= 0 ? 16 : 0);
    }
  } else {
    const int ch = tid & 3;
    const int64_t off = GATHER == FEB_GATHER_DOWN ? fine_off(P.fine, grp) : 0;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int row = (tid >> 2) + 32 * i;
      const int64_t m = m0 + row;
      int64_t src;
      if (GATHER == FEB_GATHER_DOWN) src = fbase[i] >= 0 ? fbase[i] + off : -1;
      else src = m < M ? m : -1;
      const bf16* g = src >= 0 ? in + src * P.in_ld + P.in_c0 + c0 + ch * 8 : in;
      cp16(sA + ch * S::kAHalf + row * 16, g, src >= 0 ? 16 : 0);
    }
  }
  const bf16* wt = reinterpret_cast<const bf16*>(P.wt);
  const uint32_t sB = sA + S::kA;
  const int tap0 = GATHER == FEB_GATHER_SHIFT ? 3 * grp : grp;
#pragma unroll
  for (int i = 0; i < S::kTaps * NT / 32; ++i) {
    const int e = tid + kConvThreads * i, t = e / (4 * NT), rem = e - t * 4 * NT, n = rem >> 2, c = rem & 3;
    cp16(sB + t * S::kBTap + c * (NT * 16) + n * 16, wt + ((int64_t)(tap0 + t) * P.n + n0 + n) * P.kc + c0 + c * 8, 16);
  }
}

__device__ __forceinline__ void unpack8(const uint4& q, float* v) {
  const __nv_bfloat162* h = reinterpret_cast<const __nv_bfloat162*>(&q);
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const float2 f = __bfloat1622float2(h[e]);
    v[2 * e] = f.x;
    v[2 * e + 1] = f.y;
  }
}

__device__ __forceinline__ uint4 pack8(const float* v) {
  uint4 q;
  uint32_t* w = reinterpret_cast<uint32_t*>(&q);
#pragma unroll
  for (int e = 0; e < 4; ++e) {
    const __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * e], v[2 * e + 1]);
    w[e] = *reinterpret_cast<const uint32_t*>(&h);
  }
  return q;
}

template <int NT, int GATHER, int SCATTER>
__global__ void __launch_bounds__(kConvThreads) k_conv(const FebConv P, int64_t M, int64_t Pin) {
  extern __shared__ __align__(1024) unsigned char smem[];
  using S = ConvSmem<NT, GATHER>;
  constexpr int kStages = S::kStages;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + kStages * S::kStage);
  uint32_t* tslot = reinterpret_cast<uint32_t*>(mbar + kStages);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int64_t m0 = (int64_t)blockIdx.x * S::kM;
  const int n0 = blockIdx.y * NT;
  constexpr uint32_t kCols = NT * S::kHalves;

  if (tid == 0) {
#pragma unroll
    for (int s = 0; s < kStages; ++s) tc::mbar_init(mbar + s, 1);
    tc::mbar_fence_init();
  }
  if (warp == 0) tc::tmem_alloc(tslot, kCols);

  // DOWN gather: the fine row of cell 2V of this thread's four A rows (-1 for shell / out-of-range rows)
  int64_t fbase[4] = {-1, -1, -1, -1};
  if (GATHER == FEB_GATHER_DOWN) {
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int64_t m = m0 + (tid >> 2) + 32 * i;
      int x, y, z;
      if (m < M && row_cell(P.grid, m, x, y, z)) fbase[i] = prow(P.fine, 2 * x, 2 * y, 2 * z);
    }
  }
  const int kcs = P.kc / kKS;
  const int ngroups = GATHER == FEB_GATHER_SHIFT ? 9 : (GATHER == FEB_GATHER_DOWN ? 8 : 1);
  const int nk = ngroups * kcs;
  const uint32_t base = tc::smem_addr(smem);
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nk) conv_load<NT, GATHER>(P, s, kcs, base + s * S::kStage, m0, M, Pin, fbase, n0, tid);
    cp_commit();
  }
  tc::sync_for_tensor_core();
  const uint32_t tmem = *tslot;
  constexpr uint32_t idesc = tc::idesc_bf16(128, NT);

  bool ok = true;
  for (int it = 0; it < nk; ++it) {
    cp_wait<kStages - 2>();
    ok = tc::sync_for_tensor_core_and(ok);
    if (!ok) break;
    const int slot = it % kStages;
    if (tid == 0) {
      const uint32_t a = base + slot * S::kStage, b = a + S::kA;
#pragma unroll
      for (int h = 0; h < S::kHalves; ++h)
#pragma unroll
        for (int t = 0; t < S::kTaps; ++t)
#pragma unroll
          for (int s = 0; s < 2; ++s)
            tc::mma_bf16(tmem + (uint32_t)(h * NT), tc::smem_desc(a + (h * 128 + t) * 16 + 2 * s * S::kAHalf, S::kAHalf, 128),
                         tc::smem_desc(b + t * S::kBTap + 2 * s * NT * 16, NT * 16, 128), idesc, (it | t | s) != 0);
      tc::commit(mbar + slot);
    }
    const int nxt = it + kStages - 1;
    if (nxt < nk) {
      // the slot of step nxt was last read by the MMAs of step it - 1
      if (it >= 1) ok = tc::mbar_wait(tc::smem_addr(mbar + (it - 1) % kStages), (uint32_t)(((it - 1) / kStages) & 1));
      if (ok) conv_load<NT, GATHER>(P, nxt, kcs, base + (nxt % kStages) * S::kStage, m0, M, Pin, fbase, n0, tid);
    }
    cp_commit();
  }
  if (ok) ok = tc::mbar_wait(tc::smem_addr(mbar + (nk - 1) % kStages), (uint32_t)(((nk - 1) / kStages) & 1));
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  ok = __syncthreads_and(ok ? 1 : 0) != 0;

  if (ok) {
   bf16* out = reinterpret_cast<bf16*>(P.out);
   const bf16* mask = reinterpret_cast<const bf16*>(P.mask);
#pragma unroll 1
   for (int h = 0; h < S::kHalves; ++h) {
    const int64_t m = m0 + h * 128 + 32 * warp + lane;
    int x = 0, y = 0, z = 0;
    const bool inside = m < M && row_cell(P.grid, m, x, y, z);
#pragma unroll 1
    for (int cc = 0; cc < NT; cc += 32) {
      float v[32];
      tc::tmem_ld32(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)(h * NT + cc), v);
      tc::wait_ld();
      const int n = n0 + cc;
      int64_t orow;
      int ocol;
      if (SCATTER) {
        if (!inside) continue;
        const int t = n / P.scatter_c;
        ocol = n - t * P.scatter_c;
        orow = prow(P.fine, 2 * x + (t >> 2), 2 * y + ((t >> 1) & 1), 2 * z + (t & 1));
      } else {
        if (m >= M) continue;
        orow = m;
        ocol = n;
        if (!inside) {
          uint4* dst = reinterpret_cast<uint4*>(out + orow * P.out_ld + P.out_c0 + ocol);
#pragma unroll
          for (int q = 0; q < 4; ++q) dst[q] = make_uint4(0u, 0u, 0u, 0u);
          continue;
        }
      }
      if (P.bias) {
#pragma unroll
        for (int q = 0; q < 32; ++q) v[q] += P.bias[ocol + q];
      }
      if (P.relu) {
#pragma unroll
        for (int q = 0; q < 32; ++q) v[q] = fmaxf(v[q], 0.f);
      }
      uint4* dst = reinterpret_cast<uint4*>(out + orow * P.out_ld + P.out_c0 + ocol);
      if (P.accumulate) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float o[8];
          unpack8(dst[q], o);
#pragma unroll
          for (int e = 0; e < 8; ++e) v[8 * q + e] += o[e];
        }
      }
      if (mask) {
        const uint4* mk = reinterpret_cast<const uint4*>(mask + orow * P.mask_ld + P.mask_c0 + ocol);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          float o[8];
          unpack8(mk[q], o);
#pragma unroll
          for (int e = 0; e < 8; ++e) v[8 * q + e] = o[e] > 0.f ? v[8 * q + e] : 0.f;
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) dst[q] = pack8(v + 8 * q);
    }
   }
  } else if (tid == 0 && P.status) {
    atomicExch(P.status, 1);
  }
  cp_wait<0>();
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) tc::tmem_free(tmem, kCols);
}

// ------------------------------------------------------------------------------------------ weight gradient
constexpr int kWR = 32;                          // rows per stage

__device__ __forceinline__ void ldsm_x4_trans(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}

__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// rows of P and Q for row r of the row grid and tap t (-1: zero)
template <int MODE>
__device__ __forceinline__ void wg_rows(const FebWgrad& W, int64_t r, int64_t R, int tap, int64_t& rp, int64_t& rq) {
  rp = rq = -1;
  if (r >= R) return;
  if (MODE == FEB_GATHER_SHIFT) {
    const int64_t s = r + shift_off(W.grid, tap);
    if (s >= 0 && s < R) { rp = r; rq = s; }
  } else {
    int x, y, z;
    if (!row_cell(W.grid, r, x, y, z)) return;
    const int64_t f = prow(W.fine, 2 * x, 2 * y, 2 * z) + fine_off(W.fine, tap);
    if (MODE == FEB_GATHER_DOWN) { rp = r; rq = f; }
    else { rp = f; rq = r; }
  }
}

template <int TA, int TB, int MODE>
__global__ void __launch_bounds__(128) k_wgrad(const FebWgrad W, int64_t R, int rows_per_cta) {
  constexpr int LDA = TA + 8, LDB = TB + 8;
  __shared__ __align__(16) bf16 sP[3][kWR][LDA];
  __shared__ __align__(16) bf16 sQ[3][kWR][LDB];
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int tap = blockIdx.y;
  const int ta = W.na / TA;
  const int a0 = (blockIdx.z % ta) * TA, b0 = (blockIdx.z / ta) * TB;
  const int64_t r0 = (int64_t)blockIdx.x * rows_per_cta;
  const int nst = (rows_per_cta + kWR - 1) / kWR;
  const bf16* Pp = reinterpret_cast<const bf16*>(W.p);
  const bf16* Qp = reinterpret_cast<const bf16*>(W.q);

  auto load = [&](int st, int slot) {
    constexpr int CA = TA / 8, CB = TB / 8;
    for (int e = tid; e < kWR * (CA + CB); e += 128) {
      const bool isp = e < kWR * CA;
      const int ee = isp ? e : e - kWR * CA;
      const int C = isp ? CA : CB;
      const int rr = ee / C, cc = ee - rr * C;
      const int64_t r = r0 + (int64_t)st * kWR + rr;
      int64_t rp, rq;
      wg_rows<MODE>(W, (r < r0 + rows_per_cta) ? r : R, R, tap, rp, rq);
      if (isp) {
        const bf16* g = rp >= 0 ? Pp + rp * W.p_ld + W.p_c0 + a0 + cc * 8 : Pp;
        cp16(tc::smem_addr(&sP[slot][rr][cc * 8]), g, (rp >= 0 && rq >= 0) ? 16 : 0);
      } else {
        const bf16* g = rq >= 0 ? Qp + rq * W.q_ld + W.q_c0 + b0 + cc * 8 : Qp;
        cp16(tc::smem_addr(&sQ[slot][rr][cc * 8]), g, (rp >= 0 && rq >= 0) ? 16 : 0);
      }
    }
  };

  constexpr int WA = TA / 2, WB = TB / 2, MT = WA / 16, NT8 = WB / 8;
  const int wa = warp >> 1, wb = warp & 1;
  float acc[MT][NT8][4];
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT8; ++j)
#pragma unroll
      for (int e = 0; e < 4; ++e) acc[i][j][e] = 0.f;

  load(0, 0);
  cp_commit();
  if (nst > 1) load(1, 1);
  cp_commit();
  const int q = lane >> 3, rr8 = lane & 7;
  for (int st = 0; st < nst; ++st) {
    cp_wait<1>();
    __syncthreads();
    const int slot = st % 3;
#pragma unroll
    for (int kk = 0; kk < kWR; kk += 16) {
      uint32_t af[MT][4];
#pragma unroll
      for (int i = 0; i < MT; ++i) {
        const int k = kk + rr8 + 8 * (q >> 1), a = wa * WA + i * 16 + 8 * (q & 1);
        ldsm_x4_trans(tc::smem_addr(&sP[slot][k][a]), af[i][0], af[i][1], af[i][2], af[i][3]);
      }
#pragma unroll
      for (int j = 0; j < NT8; j += 2) {
        const int k = kk + rr8 + 8 * (q & 1), b = wb * WB + j * 8 + 8 * (q >> 1);
        uint32_t b00, b01, b10, b11;
        ldsm_x4_trans(tc::smem_addr(&sQ[slot][k][b]), b00, b01, b10, b11);
#pragma unroll
        for (int i = 0; i < MT; ++i) {
          mma16816(acc[i][j], af[i], b00, b01);
          mma16816(acc[i][j + 1], af[i], b10, b11);
        }
      }
    }
    if (st + 2 < nst) load(st + 2, (st + 2) % 3);
    cp_commit();
  }
  cp_wait<0>();
  const int g = lane >> 2, c2 = (lane & 3) * 2;
  float* dw = W.dw + (int64_t)tap * W.na * W.nb;
#pragma unroll
  for (int i = 0; i < MT; ++i)
#pragma unroll
    for (int j = 0; j < NT8; ++j) {
      const int a = a0 + wa * WA + i * 16 + g, b = b0 + wb * WB + j * 8 + c2;
      atomicAdd(dw + (int64_t)a * W.nb + b, acc[i][j][0]);
      atomicAdd(dw + (int64_t)a * W.nb + b + 1, acc[i][j][1]);
      atomicAdd(dw + (int64_t)(a + 8) * W.nb + b, acc[i][j][2]);
      atomicAdd(dw + (int64_t)(a + 8) * W.nb + b + 1, acc[i][j][3]);
    }
}

// ------------------------------------------------------------------------------------------ small kernels
__global__ void k_colsum(const bf16* __restrict__ g, int64_t rows, int ld, int c0, int nc, int rows_per_block,
                         float* __restrict__ out) {
  __shared__ float part[256];
  const int c = threadIdx.x % nc, lane_rows = blockDim.x / nc, sub = threadIdx.x / nc;
  float s = 0.f;
  if (sub < lane_rows) {
    const int64_t rb = (int64_t)blockIdx.x * rows_per_block, re = min(rows, rb + rows_per_block);
    for (int64_t r = rb + sub; r < re; r += lane_rows) s += __bfloat162float(g[r * ld + c0 + c]);
  }
  part[threadIdx.x] = s;
  __syncthreads();
  if (threadIdx.x < nc) {
    float t = 0.f;
    for (int k = 0; k < lane_rows; ++k) t += part[threadIdx.x + k * nc];
    atomicAdd(out + threadIdx.x, t);
  }
}

__global__ void k_weights(const float* __restrict__ W, int taps, int co, int ci, bf16* __restrict__ fwd,
                          bf16* __restrict__ bwd, int flip) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const int64_t n = (int64_t)taps * co * ci;
  if (e >= n) return;
  const int t = int(e / ((int64_t)co * ci)), o = int((e / ci) % co), i = int(e % ci);
  const bf16 v = __float2bfloat16_rn(W[e]);
  fwd[e] = v;
  if (bwd) {
    const int tb = flip ? taps - 1 - t : t;
    bwd[((int64_t)tb * ci + i) * co + o] = v;
  }
}

constexpr int kHeadC = 32;

__global__ void __launch_bounds__(128) k_head(const bf16* __restrict__ X, int x_ld, int64_t rows,
                                              const float* __restrict__ W, const float* __restrict__ b,
                                              float* __restrict__ pred, const float* __restrict__ target,
                                              const float* __restrict__ wgt, float inv_n, double* __restrict__ loss,
                                              bf16* __restrict__ dX, int dx_ld, float* __restrict__ dW,
                                              float* __restrict__ db, const float* __restrict__ dpred_in) {
  __shared__ float sW[3 * kHeadC + 3];
  __shared__ float sdW[3 * kHeadC + 3];
  for (int e = threadIdx.x; e < 3 * kHeadC + 3; e += blockDim.x) {
    sW[e] = e < 3 * kHeadC ? W[e] : b[e - 3 * kHeadC];
    sdW[e] = 0.f;
  }
  __syncthreads();
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  const bool live = r < rows;
  float x[kHeadC];
  if (live) {
    const uint4* src = reinterpret_cast<const uint4*>(X + r * x_ld);
#pragma unroll
    for (int q = 0; q < kHeadC / 8; ++q) unpack8(src[q], x + 8 * q);
  } else {
#pragma unroll
    for (int k = 0; k < kHeadC; ++k) x[k] = 0.f;
  }
  float o[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    float s = sW[3 * kHeadC + c];
#pragma unroll
    for (int k = 0; k < kHeadC; ++k) s = fmaf(x[k], sW[c * kHeadC + k], s);
    o[c] = s;
  }
  if (live && pred) {
#pragma unroll
    for (int c = 0; c < 3; ++c) pred[3 * r + c] = o[c];
  }
  if (!target && !dpred_in) return;
  float d[3] = {0.f, 0.f, 0.f};
  double l = 0.0;
  if (live) {
    if (dpred_in) {                       // a given gradient of the output (the caller's loss)
#pragma unroll
      for (int c = 0; c < 3; ++c) d[c] = dpred_in[3 * r + c];
    } else {
      const float w = wgt[r];
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const float e = w > 0.f ? o[c] - target[3 * r + c] : 0.f;
        l += (double)(w * e * e) * inv_n;
        d[c] = 2.f * inv_n * w * e;
      }
    }
    float dx[kHeadC];
#pragma unroll
    for (int k = 0; k < kHeadC; ++k) {
      const float s = d[0] * sW[k] + d[1] * sW[kHeadC + k] + d[2] * sW[2 * kHeadC + k];
      dx[k] = x[k] > 0.f ? s : 0.f;
    }
    uint4* dst = reinterpret_cast<uint4*>(dX + r * dx_ld);
#pragma unroll
    for (int q = 0; q < kHeadC / 8; ++q) dst[q] = pack8(dx + 8 * q);
  }
  // dW[c][k] = sum d[c] x[k], db[c] = sum d[c]: warp sums, then shared, then global
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll 4
    for (int k = 0; k < kHeadC; ++k) {
      const float s = warp_sum(d[c] * x[k]);
      if (lane == 0) atomicAdd(&sdW[c * kHeadC + k], s);
    }
    const float s = warp_sum(d[c]);
    if (lane == 0) atomicAdd(&sdW[3 * kHeadC + c], s);
  }
  l = warp_sum(l);
  if (lane == 0 && l != 0.0 && loss) atomicAdd(loss, l);
  __syncthreads();
  for (int e = threadIdx.x; e < 3 * kHeadC + 3; e += blockDim.x) {
    if (e < 3 * kHeadC) atomicAdd(dW + e, sdW[e]);
    else atomicAdd(db + e - 3 * kHeadC, sdW[e]);
  }
}

// Loss of a prediction on a network grid: weighted squared error (mse_scale) plus the stiffness-weighted squared
// error of its differences along the grid edges (h1_scale): the edge from node (x,y,z) to its +1 neighbour along
// an axis carries the weight E / e_ref of the cell at (x,y,z) (E from the input channel 0 = log10 E / 4; zero for
// inactive cells), so the second term follows the strain energy of the error the way the solve weighs it.  pred
// NULL: the target's own norms (loss only).  Adds the gradient to dpred (if not NULL) and the loss to *loss.
__global__ void k_loss(FebNetGrid net, const bf16* __restrict__ xin, const float* __restrict__ pred,
                       const float* __restrict__ T, const float* __restrict__ wgt, float e_ref_inv, float mse_scale,
                       float h1_scale, double* __restrict__ loss, float* __restrict__ dpred) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double l = 0.0;
  int x, y, z;
  if (r < grid_rows(net) && row_cell(net, r, x, y, z) && wgt[r] > 0.f) {
    float e0[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) e0[c] = (pred ? pred[3 * r + c] : 0.f) - T[3 * r + c];
    if (mse_scale != 0.f) {
      l += (double)mse_scale * (e0[0] * e0[0] + e0[1] * e0[1] + e0[2] * e0[2]);
      if (dpred) {
#pragma unroll
        for (int c = 0; c < 3; ++c) atomicAdd(dpred + 3 * r + c, 2.f * mse_scale * e0[c]);
      }
    }
    const bf16* xr = xin + r * 32;
    const float w = __bfloat162float(xr[2]) > 0.f ? exp10f(4.f * __bfloat162float(xr[0])) * e_ref_inv : 0.f;
    if (h1_scale != 0.f && w > 0.f) {
      const int n3[3] = {net.nx, net.ny, net.nz};
      const int c3[3] = {x, y, z};
      const int64_t off[3] = {(int64_t)(net.ny + 2) * (net.nz + 2), net.nz + 2, 1};
#pragma unroll
      for (int a = 0; a < 3; ++a) {
        if (c3[a] + 1 >= n3[a]) continue;
        const int64_t r2 = r + off[a];
        if (!(wgt[r2] > 0.f)) continue;
        float dd[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) dd[c] = ((pred ? pred[3 * r2 + c] : 0.f) - T[3 * r2 + c]) - e0[c];
        l += (double)(h1_scale * w) * (dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
        if (dpred) {
#pragma unroll
          for (int c = 0; c < 3; ++c) {
            const float g = 2.f * h1_scale * w * dd[c];
            atomicAdd(dpred + 3 * r2 + c, g);
            atomicAdd(dpred + 3 * r + c, -g);
          }
        }
      }
    }
  }
  l = block_sum(l);
  if (threadIdx.x == 0 && l != 0.0) atomicAdd(loss, l);
}

// Strain energy of a prediction's error on a network grid equal to the FE grid: for every cell whose 8 corner nodes
// are network nodes (x < nx-1, y < ny-1, z < nz-1) and have targets, with the cell active, e^T K_e e with e = pred -
// target at the corners and K_e the solve's hex8 element (lambda at the centre, mu 2x2x2) of the cell's Lame
// constants, read from the network input (channel 0 = log10 E / 4, channel 1 = (nu - 0.3) * 4, channel 2 = active).
// loss += scale * sum; dpred[corner] += 2 scale K_e e.  pred NULL: the target's own energy.
__global__ void k_energy_loss(FebNetGrid net, float hx, float hy, float hz, const bf16* __restrict__ xin,
                              const float* __restrict__ pred, const float* __restrict__ T, const float* __restrict__ wgt,
                              float scale, double* __restrict__ loss, float* __restrict__ dpred) {
  const int64_t ncell = (int64_t)(net.nx - 1) * (net.ny - 1) * (net.nz - 1);
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  double l = 0.0;
  if (c < ncell) {
    const int z = int(c % (net.nz - 1)), y = int((c / (net.nz - 1)) % (net.ny - 1)),
              x = int(c / ((int64_t)(net.nz - 1) * (net.ny - 1)));
    const bf16* xr = xin + prow(net, x, y, z) * 32;
    bool ok = __bfloat162float(xr[2]) > 0.f;
    int64_t rows[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) {
      rows[k] = prow(net, x + (k & 1), y + ((k >> 1) & 1), z + (k >> 2));
      ok = ok && wgt[rows[k]] > 0.f;
    }
    if (ok) {
      float u[3][8], f[3][8];
#pragma unroll
      for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int q = 0; q < 3; ++q) u[q][k] = (pred ? pred[3 * rows[k] + q] : 0.f) - T[3 * rows[k] + q];
      const float E = exp10f(4.f * __bfloat162float(xr[0])), nu = 0.25f * __bfloat162float(xr[1]) + 0.3f;
      const float m[2] = {E * nu / ((1.f + nu) * (1.f - 2.f * nu)), E / (2.f * (1.f + nu))};
      const Material<float> mat = make_material<float, MAT_ISO_SRI>(m);
      hex8_apply<float>(u, hx, hy, hz, 1.f / hx, 1.f / hy, 1.f / hz, mat, f);
      float s = 0.f;
#pragma unroll
      for (int k = 0; k < 8; ++k)
#pragma unroll
        for (int q = 0; q < 3; ++q) {
          s += u[q][k] * f[q][k];
          if (dpred) atomicAdd(dpred + 3 * rows[k] + q, 2.f * scale * f[q][k]);
        }
      l = (double)scale * s;
    }
  }
  l = block_sum(l);
  if (threadIdx.x == 0 && l != 0.0) atomicAdd(loss, l);
}

__global__ void k_adam(float* __restrict__ w, float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       int64_t n, float lr_t, float b1, float b2, float eps, float gscale) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i] * gscale;
  const float mi = b1 * m[i] + (1.f - b1) * gi;
  const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  w[i] -= lr_t * mi / (sqrtf(vi) + eps);
  g[i] = 0.f;
}

__global__ void k_sumsq(const float* __restrict__ g, int64_t n, double* __restrict__ out) {
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    s += (double)g[i] * g[i];
  s = block_sum(s);
  if (threadIdx.x == 0) atomicAdd(out, s);
}

// ------------------------------------------------------------------------------------------ coupling to the solve
struct Axes {
  double h[3], hn[3];
  int n[3], nn[3];
};

__global__ void k_net_cells(FebNetGrid net, Axes A, const double* __restrict__ mat, const uint8_t* __restrict__ active,
                            int64_t fe_cells, bf16* __restrict__ out) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= grid_rows(net)) return;
  float v[32];
#pragma unroll
  for (int c = 0; c < 32; ++c) v[c] = 0.f;
  int x, y, z;
  if (row_cell(net, r, x, y, z)) {
    const int c3[3] = {x, y, z};
    int fi[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      const int f = int(floor((c3[d] + 0.5) * A.hn[d] / A.h[d]));
      fi[d] = min(max(f, 0), A.n[d] - 1);
    }
    const int64_t cell = ((int64_t)fi[0] * A.n[1] + fi[1]) * A.n[2] + fi[2];
    if (active[cell]) {
      const double lam = mat[cell], mu = mat[fe_cells + cell];
      const double E = mu * (3.0 * lam + 2.0 * mu) / (lam + mu), nu = lam / (2.0 * (lam + mu));
      v[0] = float(log10(fmax(E, 1e-30)) * 0.25);
      v[1] = float((nu - 0.3) * 4.0);
      v[2] = 1.f;
    }
  }
  uint4* dst = reinterpret_cast<uint4*>(out + r * 32);
#pragma unroll
  for (int q = 0; q < 4; ++q) dst[q] = pack8(v + 8 * q);
}

__device__ __forceinline__ int64_t node_net_cell(Axes A, int64_t node) {
  const int n1x = A.n[0] + 1, n1y = A.n[1] + 1;
  const int i = int(node % n1x), j = int((node / n1x) % n1y), k = int(node / ((int64_t)n1x * n1y));
  const int c3[3] = {i, j, k};
  int ci[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const int f = int(floor(c3[d] * A.h[d] / A.hn[d] + 1e-9));
    ci[d] = min(max(f, 0), A.nn[d] - 1);
  }
  return ((int64_t)ci[0] * A.nn[1] + ci[1]) * A.nn[2] + ci[2];
}

__global__ void k_net_marks(Axes A, int64_t n, const int64_t* __restrict__ nodes, const double* __restrict__ vals,
                            double vscale, int ch, float* __restrict__ scratch) {
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= n) return;
  const int64_t c = node_net_cell(A, nodes[e]);
  atomicAdd(scratch + 3 * c + ch, vals ? float(vals[e] * vscale) : 1.f);
}

__global__ void k_net_finish(FebNetGrid net, const float* __restrict__ scratch, bf16* __restrict__ out) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  int x, y, z;
  if (r >= grid_rows(net) || !row_cell(net, r, x, y, z)) return;
  const float* s = scratch + 3 * (((int64_t)x * net.ny + y) * net.nz + z);
  bf16* o = out + r * 32;
  o[3] = __float2bfloat16_rn(fminf(s[0], 1.f));
  o[4] = __float2bfloat16_rn(fminf(s[1], 1.f));
  o[5] = __float2bfloat16_rn(s[2]);
}

__global__ void k_net_targets(FebNetGrid net, const double* __restrict__ U, double inv_scale, float* __restrict__ T,
                              float* __restrict__ wgt) {
  const int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (r >= grid_rows(net)) return;
  int x, y, z;
  float t[3] = {0.f, 0.f, 0.f}, w = 0.f;
  if (row_cell(net, r, x, y, z)) {
    const int64_t node = x + (int64_t)(net.nx + 1) * (y + (int64_t)(net.ny + 1) * z);
    const double u0 = U[3 * node], u1 = U[3 * node + 1], u2 = U[3 * node + 2];
    if (isfinite(u0) && isfinite(u1) && isfinite(u2)) {
      t[0] = float(u0 * inv_scale); t[1] = float(u1 * inv_scale); t[2] = float(u2 * inv_scale);
      w = 1.f;
    }
  }
  T[3 * r] = t[0]; T[3 * r + 1] = t[1]; T[3 * r + 2] = t[2];
  wgt[r] = w;
}

__global__ void k_net_to_nodes(FebNetGrid net, Axes A, const float* __restrict__ pred, double scale,
                               const int64_t* __restrict__ orig, int64_t ntotal, double* __restrict__ x0) {
  const int64_t n = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (n >= ntotal) return;
  const int64_t g = orig ? orig[n] : n;
  const int n1x = A.n[0] + 1, n1y = A.n[1] + 1;
  const int c3[3] = {int(g % n1x), int((g / n1x) % n1y), int(g / ((int64_t)n1x * n1y))};
  int i0[3];
  double f[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    const double s = c3[d] * A.h[d] / A.hn[d];
    int i = int(floor(s));
    double t = s - i;
    if (i < 0) { i = 0; t = 0.0; }
    if (i >= A.nn[d] - 1) { i = A.nn[d] - 1; t = 0.0; }
    i0[d] = i;
    f[d] = t;
  }
  double acc[3] = {0.0, 0.0, 0.0};
#pragma unroll
  for (int corner = 0; corner < 8; ++corner) {
    const int dx = corner & 1, dy = (corner >> 1) & 1, dz = corner >> 2;
    const double w = (dx ? f[0] : 1.0 - f[0]) * (dy ? f[1] : 1.0 - f[1]) * (dz ? f[2] : 1.0 - f[2]);
    if (w == 0.0) continue;
    const int x = min(i0[0] + dx, A.nn[0] - 1), y = min(i0[1] + dy, A.nn[1] - 1), z = min(i0[2] + dz, A.nn[2] - 1);
    const float* p = pred + 3 * prow(net, x, y, z);
    acc[0] += w * p[0];
    acc[1] += w * p[1];
    acc[2] += w * p[2];
  }
  x0[3 * n] = scale * acc[0];
  x0[3 * n + 1] = scale * acc[1];
  x0[3 * n + 2] = scale * acc[2];
}

template <int NT, int GATHER, int SCATTER>
int launch_conv(const FebConv& c, int64_t M, int64_t Pin, cudaStream_t s) {
  // set on every launch (microseconds): the attribute belongs to the current device, and a process may use several
  FEB_CUDA(cudaFuncSetAttribute(k_conv<NT, GATHER, SCATTER>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)ConvSmem<NT, GATHER>::kTotal));
  const dim3 grid(div_up(M, ConvSmem<NT, GATHER>::kM), c.n / NT);
  k_conv<NT, GATHER, SCATTER><<<grid, kConvThreads, ConvSmem<NT, GATHER>::kTotal, s>>>(c, M, Pin);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

template <int GATHER, int SCATTER>
int dispatch_nt(const FebConv& c, int64_t M, int64_t Pin, cudaStream_t s) {
  if (c.n % 128 == 0) return launch_conv<128, GATHER, SCATTER>(c, M, Pin, s);
  if (c.n % 64 == 0) return launch_conv<64, GATHER, SCATTER>(c, M, Pin, s);
  return launch_conv<32, GATHER, SCATTER>(c, M, Pin, s);
}

template <int TA, int TB, int MODE>
int launch_wgrad(const FebWgrad& w, int64_t R, int taps, cudaStream_t s) {
  const int rows_per_cta = R > 200000 ? 2048 : (R > 20000 ? 512 : 128);
  const dim3 grid(div_up(R, rows_per_cta), taps, (w.na / TA) * (w.nb / TB));
  k_wgrad<TA, TB, MODE><<<grid, 128, 0, s>>>(w, R, rows_per_cta);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

template <int MODE>
int dispatch_wgrad(const FebWgrad& w, int64_t R, int taps, cudaStream_t s) {
  const bool a64 = w.na % 64 == 0, b64 = w.nb % 64 == 0;
  if (a64 && b64) return launch_wgrad<64, 64, MODE>(w, R, taps, s);
  if (a64) return launch_wgrad<64, 32, MODE>(w, R, taps, s);
  if (b64) return launch_wgrad<32, 64, MODE>(w, R, taps, s);
  return launch_wgrad<32, 32, MODE>(w, R, taps, s);
}

bool grid_ok(const FebNetGrid& g) { return g.nx >= 1 && g.ny >= 1 && g.nz >= 1; }

bool axes_from(const FebNetGrid& net, const double* hn, const FebGrid* fe, const double* h, Axes& A) {
  if (!fe || !hn || !h) return false;
  A.n[0] = fe->nx; A.n[1] = fe->ny; A.n[2] = fe->nz;
  A.nn[0] = net.nx; A.nn[1] = net.ny; A.nn[2] = net.nz;
  for (int d = 0; d < 3; ++d) {
    A.h[d] = h[d];
    A.hn[d] = hn[d];
    if (!(h[d] > 0.0) || !(hn[d] > 0.0) || A.n[d] < 1 || A.nn[d] < 1) return false;
  }
  return true;
}

}  // namespace
}  // namespace feb

using namespace feb;

extern "C" int feb_net_conv(const FebConv* c, void* stream) {
  if (!c || !c->in || !c->wt || !c->out || !grid_ok(c->grid) || c->kc < 32 || c->kc % 32 || c->n < 32 || c->n % 32 ||
      c->in_ld % 8 || c->in_c0 % 8 || c->out_ld % 8 || c->out_c0 % 8 || (c->mask && (c->mask_ld % 8 || c->mask_c0 % 8)) ||
      c->gather < FEB_GATHER_SHIFT || c->gather > FEB_GATHER_ONE) {
    set_last_error("feb_net_conv: bad argument");
    return FEB_ERR_ARG;
  }
  if ((c->gather == FEB_GATHER_DOWN || c->scatter) &&
      (!grid_ok(c->fine) || c->fine.nx != 2 * c->grid.nx || c->fine.ny != 2 * c->grid.ny || c->fine.nz != 2 * c->grid.nz)) {
    set_last_error("feb_net_conv: the fine grid must be twice the row grid");
    return FEB_ERR_ARG;
  }
  if (c->scatter && (c->gather != FEB_GATHER_ONE || c->scatter_c < 32 || c->scatter_c % 32 || c->n != 8 * c->scatter_c)) {
    set_last_error("feb_net_conv: a scatter needs gather ONE and n = 8 scatter_c");
    return FEB_ERR_ARG;
  }
  const int ncols = c->scatter ? c->scatter_c : c->n;
  if (c->in_c0 + c->kc > c->in_ld || c->out_c0 + ncols > c->out_ld || (c->mask && c->mask_c0 + ncols > c->mask_ld)) {
    set_last_error("feb_net_conv: a channel range runs past its row");
    return FEB_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t M = grid_rows(c->grid);
  const int64_t Pin = c->gather == FEB_GATHER_DOWN ? grid_rows(c->fine) : M;
  if (c->scatter) return dispatch_nt<FEB_GATHER_ONE, 1>(*c, M, Pin, s);
  if (c->gather == FEB_GATHER_SHIFT) return dispatch_nt<FEB_GATHER_SHIFT, 0>(*c, M, Pin, s);
  if (c->gather == FEB_GATHER_DOWN) return dispatch_nt<FEB_GATHER_DOWN, 0>(*c, M, Pin, s);
  return dispatch_nt<FEB_GATHER_ONE, 0>(*c, M, Pin, s);
}

extern "C" int feb_net_wgrad(const FebWgrad* w, void* stream) {
  if (!w || !w->p || !w->q || !w->dw || !grid_ok(w->grid) || w->na < 32 || w->na % 32 || w->nb < 32 || w->nb % 32 ||
      w->p_ld % 8 || w->p_c0 % 8 || w->q_ld % 8 || w->q_c0 % 8 || w->mode < FEB_GATHER_SHIFT || w->mode > FEB_GATHER_UP ||
      w->mode == FEB_GATHER_ONE) {
    set_last_error("feb_net_wgrad: bad argument");
    return FEB_ERR_ARG;
  }
  if (w->mode != FEB_GATHER_SHIFT &&
      (!grid_ok(w->fine) || w->fine.nx != 2 * w->grid.nx || w->fine.ny != 2 * w->grid.ny || w->fine.nz != 2 * w->grid.nz)) {
    set_last_error("feb_net_wgrad: the fine grid must be twice the row grid");
    return FEB_ERR_ARG;
  }
  if (w->p_c0 + w->na > w->p_ld || w->q_c0 + w->nb > w->q_ld) {
    set_last_error("feb_net_wgrad: a channel range runs past its row");
    return FEB_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t R = grid_rows(w->grid);
  if (w->mode == FEB_GATHER_SHIFT) return dispatch_wgrad<FEB_GATHER_SHIFT>(*w, R, 27, s);
  if (w->mode == FEB_GATHER_DOWN) return dispatch_wgrad<FEB_GATHER_DOWN>(*w, R, 8, s);
  return dispatch_wgrad<FEB_GATHER_UP>(*w, R, 8, s);
}

extern "C" int feb_net_colsum(const void* g, int64_t rows, int32_t ld, int32_t c0, int32_t nc, float* out,
                              void* stream) {
  if (!g || !out || rows < 1 || nc < 1 || nc > 256 || ld < c0 + nc) {
    set_last_error("feb_net_colsum: bad argument");
    return FEB_ERR_ARG;
  }
  const int rpb = 2048;
  k_colsum<<<div_up(rows, rpb), 256, 0, (cudaStream_t)stream>>>(reinterpret_cast<const bf16*>(g), rows, ld, c0, nc, rpb,
                                                                 out);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

extern "C" int feb_net_weights(const float* W, int32_t taps, int32_t co, int32_t ci, void* fwd, void* bwd, int32_t flip,
                               void* stream) {
  if (!W || !fwd || taps < 1 || co < 1 || ci < 1) {
    set_last_error("feb_net_weights: bad argument");
    return FEB_ERR_ARG;
  }
  const int64_t n = (int64_t)taps * co * ci;
  k_weights<<<div_up(n, kThreads), kThreads, 0, (cudaStream_t)stream>>>(W, taps, co, ci, reinterpret_cast<bf16*>(fwd),
                                                                         reinterpret_cast<bf16*>(bwd), flip);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

extern "C" int feb_net_head(const void* X, int32_t x_ld, int64_t rows, const float* W, const float* b, float* pred,
                            const float* target, const float* wgt, float inv_n, double* loss, void* dX, int32_t dx_ld,
                            float* dW, float* db, void* stream) {
  if (!X || !W || !b || rows < 1 || x_ld < kHeadC || x_ld % 8 ||
      (target && (!wgt || !loss || !dX || !dW || !db || dx_ld < kHeadC || dx_ld % 8))) {
    set_last_error("feb_net_head: bad argument");
    return FEB_ERR_ARG;
  }
  k_head<<<div_up(rows, 128), 128, 0, (cudaStream_t)stream>>>(reinterpret_cast<const bf16*>(X), x_ld, rows, W, b, pred,
                                                              target, wgt, inv_n, loss, reinterpret_cast<bf16*>(dX),
                                                              dx_ld, dW, db, nullptr);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

extern "C" int feb_net_adam(float* w, float* g, float* m, float* v, int64_t n, float lr, float beta1, float beta2,
                            float eps, int32_t step, float gscale, void* stream) {
  if (!w || !g || !m || !v || n < 1 || step < 1) {
    set_last_error("feb_net_adam: bad argument");
    return FEB_ERR_ARG;
  }
  const double c1 = 1.0 - pow((double)beta1, step), c2 = 1.0 - pow((double)beta2, step);
  const float lr_t = float(lr * sqrt(c2) / c1);
  k_adam<<<div_up(n, kThreads), kThreads, 0, (cudaStream_t)stream>>>(w, g, m, v, n, lr_t, beta1, beta2, eps, gscale);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

extern "C" int feb_net_sumsq(const float* g, int64_t n, double* out, void* stream) {
  if (!g || !out || n < 1) {
    set_last_error("feb_net_sumsq: bad argument");
    return FEB_ERR_ARG;
  }
  k_sumsq<<<min(div_up(n, kThreads), 4 * kSmCount), kThreads, 0, (cudaStream_t)stream>>>(g, n, out);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

extern "C" int feb_net_inputs(FebNetGrid net, const double* hn, const FebGrid* fe, const double* h, const double* mat,
                              const uint8_t* active, int64_t nsplit, const int64_t* split_nodes, int64_t ncontact,
                              const int64_t* contact_nodes, int64_t nload, const int64_t* load_nodes,
                              const double* load_z, double load_scale, float* scratch, void* out, void* stream) {
  Axes A;
  if (!grid_ok(net) || !axes_from(net, hn, fe, h, A) || !mat || !active || !scratch || !out ||
      (nsplit > 0 && !split_nodes) || (ncontact > 0 && !contact_nodes) || (nload > 0 && (!load_nodes || !load_z))) {
    set_last_error("feb_net_inputs: bad argument");
    return FEB_ERR_ARG;
  }
  cudaStream_t s = (cudaStream_t)stream;
  const int64_t rows = grid_rows(net), ncell = (int64_t)net.nx * net.ny * net.nz;
  const int64_t fe_cells = (int64_t)fe->nx * fe->ny * fe->nz;
  bf16* o = reinterpret_cast<bf16*>(out);
  k_net_cells<<<div_up(rows, kThreads), kThreads, 0, s>>>(net, A, mat, active, fe_cells, o); note_launch();
  FEB_CUDA(cudaMemsetAsync(scratch, 0, (size_t)ncell * 3 * sizeof(float), s));
  if (nsplit > 0) { k_net_marks<<<div_up(nsplit, kThreads), kThreads, 0, s>>>(A, nsplit, split_nodes, nullptr, 0.0, 0, scratch); note_launch(); }
  if (ncontact > 0) { k_net_marks<<<div_up(ncontact, kThreads), kThreads, 0, s>>>(A, ncontact, contact_nodes, nullptr, 0.0, 1, scratch); note_launch(); }
  if (nload > 0) { k_net_marks<<<div_up(nload, kThreads), kThreads, 0, s>>>(A, nload, load_nodes, load_z, load_scale, 2, scratch); note_launch(); }
  k_net_finish<<<div_up(rows, kThreads), kThreads, 0, s>>>(net, scratch, o); note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

extern "C" int feb_net_targets(FebNetGrid net, const double* U, double scale, float* target, float* wgt, void* stream) {
  if (!grid_ok(net) || !U || !target || !wgt || !(scale > 0.0)) {
    set_last_error("feb_net_targets: bad argument");
    return FEB_ERR_ARG;
  }
  const int64_t rows = grid_rows(net);
  k_net_targets<<<div_up(rows, kThreads), kThreads, 0, (cudaStream_t)stream>>>(net, U, 1.0 / scale, target, wgt);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

extern "C" int feb_net_to_nodes(FebNetGrid net, const double* hn, const float* pred, double scale, const FebGrid* fe,
                                const double* h, const int64_t* orig, int64_t nnode_total, double* x0, void* stream) {
  Axes A;
  if (!grid_ok(net) || !axes_from(net, hn, fe, h, A) || !pred || !x0 || nnode_total < 1) {
    set_last_error("feb_net_to_nodes: bad argument");
    return FEB_ERR_ARG;
  }
  k_net_to_nodes<<<div_up(nnode_total, kThreads), kThreads, 0, (cudaStream_t)stream>>>(net, A, pred, scale, orig,
                                                                                       nnode_total, x0);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

extern "C" int feb_net_head_grad(const void* X, int32_t x_ld, int64_t rows, const float* W, const float* dpred,
                                 void* dX, int32_t dx_ld, float* dW, float* db, void* stream) {
  if (!X || !W || !dpred || !dX || !dW || !db || rows < 1 || x_ld < kHeadC || x_ld % 8 || dx_ld < kHeadC || dx_ld % 8) {
    set_last_error("feb_net_head_grad: bad argument");
    return FEB_ERR_ARG;
  }
  // the bias only enters the recomputed output, which this pass does not use
  k_head<<<div_up(rows, 128), 128, 0, (cudaStream_t)stream>>>(reinterpret_cast<const bf16*>(X), x_ld, rows, W, W,
                                                              nullptr, nullptr, nullptr, 0.f, nullptr,
                                                              reinterpret_cast<bf16*>(dX), dx_ld, dW, db, dpred);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

extern "C" int feb_net_loss(FebNetGrid net, const void* xin, const float* pred, const float* target, const float* wgt,
                            float e_ref_inv, float mse_scale, float h1_scale, double* loss, float* dpred, void* stream) {
  if (!grid_ok(net) || !xin || !target || !wgt || !loss || !(e_ref_inv > 0.f)) {
    set_last_error("feb_net_loss: bad argument");
    return FEB_ERR_ARG;
  }
  const int64_t rows = grid_rows(net);
  k_loss<<<div_up(rows, kThreads), kThreads, 0, (cudaStream_t)stream>>>(net, reinterpret_cast<const bf16*>(xin), pred,
                                                                        target, wgt, e_ref_inv, mse_scale, h1_scale,
                                                                        loss, dpred);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}

extern "C" int feb_net_energy_loss(FebNetGrid net, const double* h, const void* xin, const float* pred, const float* target,
                                   const float* wgt, float scale, double* loss, float* dpred, void* stream) {
  if (!grid_ok(net) || net.nx < 2 || net.ny < 2 || net.nz < 2 || !h || !(h[0] > 0) || !(h[1] > 0) || !(h[2] > 0) ||
      !xin || !target || !wgt || !loss) {
    set_last_error("feb_net_energy_loss: bad argument");
    return FEB_ERR_ARG;
  }
  const int64_t ncell = (int64_t)(net.nx - 1) * (net.ny - 1) * (net.nz - 1);
  k_energy_loss<<<div_up(ncell, kThreads), kThreads, 0, (cudaStream_t)stream>>>(
      net, (float)h[0], (float)h[1], (float)h[2], reinterpret_cast<const bf16*>(xin), pred, target, wgt, scale, loss,
      dpred);
  note_launch();
  FEB_CUDA(cudaGetLastError());
  return FEB_OK;
}
