// Level-0 K.u on the voxel grid with paired node rows, and the smoother steps fused into its epilogue.
//
// Work split (one product y = K u, or one Chebyshev / residual step of the smoother):
//   * the sparse remainder of the level-0 operator (cells touching split copies, penalty springs, extra
//     entries) is accumulated first, with atomics, into the scratch vector `tsp` (k_fine_sparse);
//   * k_fine_pair then computes the regular cells matrix-free.  A grid node whose 8 cells are all handled
//     here (the bulk) is finished in registers: its product is stored, or the smoother update of that node
//     runs on the spot (r -= K d, z = Dinv r, d' = a1 d + a2 z, x += d').  A node flagged "special" adds
//     and clears its `tsp` entry first; split copies (ids >= nnode) are finished by tail blocks of the
//     same launch from `tsp` alone.  `tsp` is zero again when the launch ends.
//
// Tiling: a warp holds 32 node columns (30 owned, one halo column on each side) of two neighbouring node
// rows; a CTA of WY warps holds 2 WY rows (2 WY - 2 owned) and marches in z over `zchunk` node planes.
// The two rows are processed as packed pairs (fma/add/sub/mul.rn.f32x2 on sm_100), so every arithmetic
// instruction serves two cells.  The element operator is the modal form of element.cuh, sum-factorised
// over the grid: x-edge butterflies by warp shuffle, y by one shared-memory exchange with the warp above
// (forward) and below (backward), z in registers along the march.  On cubic cells with the SRI isotropic
// model (the engine's voxel model, rb/splitfe.py:58-69) the modal core collapses to 27 pair operations
// with 5 per-cell constants (see cube_sri_core); other materials and rectilinear grids run the general
// modal core.  Cell materials are 7-bit ids into a table held in shared memory: one 16-bit load gives
// the two cells of a thread's rows plus the "special" flags of its two nodes.
#include <algorithm>

#include "fine.cuh"
#include "pair.cuh"
#include "vec.cuh"

namespace feb {

namespace {

constexpr int kXOwn = 30;
#ifndef FEB_PAIR_MINB
#define FEB_PAIR_MINB 1
#endif
#ifndef FEB_PAIR_UNROLL
#define FEB_PAIR_UNROLL 1
#endif
// FP32 marches two planes per trip (no register copies between planes)
constexpr bool kPairUnroll = FEB_PAIR_UNROLL != 0;

template <typename T>
using V2 = typename Vec2<T>::type;

template <typename T>
__device__ __forceinline__ V2<T> mk2(T a, T b) {
  V2<T> r;
  r.x = a;
  r.y = b;
  return r;
}

// Modal core of the SRI isotropic element on a cube of edge h (rb/splitfe.py:58-69 with equal edges).
// With unscaled modal inputs (butterfly_fwd) the general core (hex8_modal) reduces to, per cell:
//   modes with one difference index:  FX1 = (mu h/8) X1 + T,  FY2 = (mu h/8) Y2 + T,  FZ4 = (mu h/8) Z4 + T,
//                                      T = (lam h/16)(X1 + Y2 + Z4);
//                                      FY1 = FX2 = (mu h/16)(X2 + Y1), FZ1 = FX4 = (mu h/16)(X4 + Z1),
//                                      FZ2 = FY4 = (mu h/16)(Y4 + Z2);
//   two difference indices:            FX3 = (mu h/16) X3, FY3, FX5, FZ5, FY6, FZ6 likewise,
//                                      FZ3 = (mu h/48)(Z3 + A), FY5 = (mu h/48)(Y5 + A), FX6 = (mu h/48)(X6 + A),
//                                      A = X6 + Y5 + Z3;
//   three:                             F.7 = (mu h/36) .7
// (the q = 1/16, 1/48, 1/144 mode weights folded into the constants; mode 0 carries no force).
template <typename T>
__device__ __forceinline__ void cube_sri_core(const P2<T> (&X)[8], const P2<T> (&Y)[8], const P2<T> (&Z)[8],
                                              P2<T> L16, P2<T> M48, P2<T> (&FX)[8], P2<T> (&FY)[8],
                                              P2<T> (&FZ)[8]) {
  const P2<T> M16 = M48 * P2<T>(T(3)), M8 = M48 * P2<T>(T(6)), M36 = M48 * P2<T>(T(4.0 / 3.0));
  const P2<T> sxy = M16 * (X[2] + Y[1]), sxz = M16 * (X[4] + Z[1]), syz = M16 * (Y[4] + Z[2]);
  const P2<T> tc = L16 * (X[1] + Y[2] + Z[4]);
  FX[1] = fma2(M8, X[1], tc); FY[2] = fma2(M8, Y[2], tc); FZ[4] = fma2(M8, Z[4], tc);
  FY[1] = sxy; FX[2] = sxy; FZ[1] = sxz; FX[4] = sxz; FZ[2] = syz; FY[4] = syz;
  const P2<T> ma = M48 * (X[6] + Y[5] + Z[3]);
  FZ[3] = fma2(M48, Z[3], ma); FY[5] = fma2(M48, Y[5], ma); FX[6] = fma2(M48, X[6], ma);
  FX[3] = M16 * X[3]; FY[3] = M16 * Y[3]; FX[5] = M16 * X[5];
  FZ[5] = M16 * Z[5]; FY[6] = M16 * Y[6]; FZ[6] = M16 * Z[6];
  FX[7] = M36 * X[7]; FY[7] = M36 * Y[7]; FZ[7] = M36 * Z[7];
}

// General modal core on pairs (any material model, rectilinear cells): hex8_modal with fused
// multiply-adds.
template <typename T, bool HAS12>
__device__ __forceinline__ void pair_modal(P2<T> (&X)[8], P2<T> (&Y)[8], P2<T> (&Z)[8], const ElemCoef<P2<T>>& k,
                                           P2<T> (&FX)[8], P2<T> (&FY)[8], P2<T> (&FZ)[8]) {
  using V = P2<T>;
#pragma unroll
  for (int l = 1; l < 8; ++l) {
    const int nd = (l & 1) + ((l >> 1) & 1) + ((l >> 2) & 1);
    const V q(T(nd == 1 ? 1.0 / 16.0 : (nd == 2 ? 1.0 / 48.0 : 1.0 / 144.0)));
    X[l] = X[l] * q; Y[l] = Y[l] * q; Z[l] = Z[l] * q;
  }
#pragma unroll
  for (int be = 0; be < 2; ++be)
#pragma unroll
    for (int ga = 0; ga < 2; ++ga) {
      const int l = 1 + 2 * be + 4 * ga;
      const bool ce = (be == 0) && (ga == 0);
      V fx = (ce ? k.ex0 : k.dx0) * X[l];
      if (be == 0 && (HAS12 || ce)) fx = fma2(ce ? k.ec1c : k.c1c, Y[2 + 4 * ga], fx);
      if (ga == 0 && (HAS12 || ce)) fx = fma2(ce ? k.ec2b : k.c2b, Z[4 + 2 * be], fx);
      V fy = k.x4 * Y[l];
      if (be == 0) fy = fma2(k.c4c, X[2 + 4 * ga], fy);
      V fz = k.x5 * Z[l];
      if (ga == 0) fz = fma2(k.c5b, X[4 + 2 * be], fz);
      FX[l] = fx; FY[l] = fy; FZ[l] = fz;
    }
#pragma unroll
  for (int al = 0; al < 2; ++al)
#pragma unroll
    for (int ga = 0; ga < 2; ++ga) {
      const int l = al + 2 + 4 * ga;
      const bool ce = (al == 0) && (ga == 0);
      const V z0(T(0));
      V fy = fma2(ce ? k.ey0 : k.dy0, Y[l], al ? FY[l] : z0);
      if (al == 0 && (HAS12 || ce)) fy = fma2(ce ? k.ec1c : k.c1c, X[1 + 4 * ga], fy);
      if (ga == 0 && (HAS12 || ce)) fy = fma2(ce ? k.ec2a : k.c2a, Z[al + 4], fy);
      V fx = fma2(k.y4, X[l], al ? FX[l] : z0);
      if (al == 0) fx = fma2(k.c4c, Y[1 + 4 * ga], fx);
      V fz = fma2(k.y5, Z[l], al ? FZ[l] : z0);
      if (ga == 0) fz = fma2(k.c5a, Y[al + 4], fz);
      FX[l] = fx; FY[l] = fy; FZ[l] = fz;
    }
#pragma unroll
  for (int al = 0; al < 2; ++al)
#pragma unroll
    for (int be = 0; be < 2; ++be) {
      const int l = al + 2 * be + 4;
      const bool ce = (al == 0) && (be == 0);
      const bool acc = al || be;
      const V z0(T(0));
      V fz = fma2(ce ? k.ez3 : k.dz3, Z[l], acc ? FZ[l] : z0);
      if (al == 0 && (HAS12 || ce)) fz = fma2(ce ? k.ec2b : k.c2b, X[1 + 2 * be], fz);
      if (be == 0 && (HAS12 || ce)) fz = fma2(ce ? k.ec2a : k.c2a, Y[al + 2], fz);
      V fy = fma2(k.z5, Y[l], acc ? FY[l] : z0);
      if (be == 0) fy = fma2(k.c5a, Z[al + 2], fy);
      V fx = fma2(k.z5, X[l], acc ? FX[l] : z0);
      if (al == 0) fx = fma2(k.c5b, Z[1 + 2 * be], fx);
      FX[l] = fx; FY[l] = fy; FZ[l] = fz;
    }
}

// Operands of the smoother update at one node, loaded a step before they are used: residual before the
// product, iterate, direction (the product's input) and the symmetric block-Jacobi inverse.
template <typename T>
struct NodeOps {
  T r[3], x[3], d[3], D[6];
};

template <typename T>
__device__ __forceinline__ void load_node_ops(const PairView<T>& F, const SmoothArgs<T>& S, const T* __restrict__ u,
                                              bool need_dir, int n, NodeOps<T>& o) {
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    o.r[c] = S.r_in[3 * n + c];
    o.x[c] = S.x_in ? S.x_in[3 * n + c] : T(0);
    o.d[c] = need_dir ? u[3 * n + c] : T(0);
  }
  if (S.updates()) {
    const T* D = F.dinv6 + n;
#pragma unroll
    for (int q = 0; q < 6; ++q) o.D[q] = D[(size_t)q * F.ntotal];
  }
}

// smoother update of one node from t = K u at the node and its operands
template <typename T>
__device__ __forceinline__ void node_update(const SmoothArgs<T>& S, T a1, T a2, int n, const T (&t)[3],
                                            const NodeOps<T>& o) {
  T r[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) r[c] = o.r[c] - t[c];
  if (S.r_out) {
#pragma unroll
    for (int c = 0; c < 3; ++c) S.r_out[3 * n + c] = r[c];
  }
  if (!S.updates()) return;
  T z[3];
  z[0] = o.D[0] * r[0] + o.D[3] * r[1] + o.D[4] * r[2];
  z[1] = o.D[3] * r[0] + o.D[1] * r[1] + o.D[5] * r[2];
  z[2] = o.D[4] * r[0] + o.D[5] * r[1] + o.D[2] * r[2];
  T dn[3];
#pragma unroll
  for (int c = 0; c < 3; ++c) dn[c] = a2 * z[c] + a1 * o.d[c];
  if (S.d_out) {
#pragma unroll
    for (int c = 0; c < 3; ++c) S.d_out[3 * n + c] = dn[c];
  }
  if (S.x_out) {
#pragma unroll
    for (int c = 0; c < 3; ++c) S.x_out[3 * n + c] = o.x[c] + dn[c];
  }
  if (S.x_out64) {
#pragma unroll
    for (int c = 0; c < 3; ++c) S.x_out64[3 * n + c] = double(o.x[c] + dn[c]);
  }
}

template <typename T, int MODE, bool CUBE, int WY>
constexpr size_t pair_smem_bytes() {
  return 4 * sizeof(V2<T>) * 3 * WY * 32 + sizeof(T) * kMaxMatIds * (CUBE ? 2 : MatWidth<MODE>::value);
}

template <typename T, int MODE, bool CUBE, int WY, bool SMOOTH>
__global__ void __launch_bounds__(32 * WY, FEB_PAIR_MINB)
k_fine_pair(PairView<T> F, const T* __restrict__ u, T* __restrict__ y, SmoothArgs<T> S, const int* __restrict__ skip,
            int zchunk, int nbx, int nby, int nbz) {
  if (skip && *skip) return;
  constexpr int W = MatWidth<MODE>::value;
  constexpr bool HAS12 = (MODE != MAT_ISO_SRI);
  constexpr int OY = 2 * WY - 2;
  constexpr int MW = CUBE ? 2 : W;
  // FP32 smoothing loads the epilogue operands one step ahead; FP64 (no register room) loads them in finish()
  constexpr bool PREF = SMOOTH && std::is_same<T, float>::value;
  using V = P2<T>;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  // forward: (sum, diff) x-edge of the lower row per component; backward: (mean, diff) x-edge force of the
  // row above the pair; both double-buffered by plane parity
  V2<T> (*sE)[3][WY][32] = reinterpret_cast<V2<T> (*)[3][WY][32]>(smem_raw);
  V2<T> (*sB)[3][WY][32] = reinterpret_cast<V2<T> (*)[3][WY][32]>(smem_raw + 2 * sizeof(V2<T>) * 3 * WY * 32);
  T (*sMat)[MW] = reinterpret_cast<T (*)[MW]>(smem_raw + 4 * sizeof(V2<T>) * 3 * WY * 32);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  T a1 = T(0), a2 = T(0);
  if constexpr (SMOOTH) {   // the Chebyshev coefficients (a residual-only step carries no parameters)
    if (S.lp && S.updates()) {
      a1 = S.k < 0 ? T(0) : T(S.lp->a1[S.k]);
      a2 = S.k < 0 ? T(S.lp->c_init) : T(S.lp->a2[S.k]);
    }
  }
  const int64_t ntiles = (int64_t)nbx * nby * nbz;
  if (blockIdx.x >= ntiles) {   // split copies: finished from the sparse accumulator alone
    const int64_t n = F.nnode + (int64_t)(blockIdx.x - ntiles) * (32 * WY) + threadIdx.x;
    if (n >= F.ntotal) return;
    T t[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) { t[c] = F.tsp[3 * n + c]; F.tsp[3 * n + c] = T(0); }
    if constexpr (SMOOTH) {
      NodeOps<T> o;
      load_node_ops(F, S, u, a1 != T(0), (int)n, o);
      node_update(S, a1, a2, (int)n, t, o);
    } else {
#pragma unroll
      for (int c = 0; c < 3; ++c) y[3 * n + c] = t[c];
    }
    return;
  }
  for (int q = threadIdx.x; q < kMaxMatIds; q += blockDim.x) {
    if constexpr (CUBE) {
      sMat[q][0] = q < F.nmat ? T(F.mtab[W * q] * F.h / 16.0) : T(0);
      sMat[q][1] = q < F.nmat ? T(F.mtab[W * q + 1] * F.h / 48.0) : T(0);
    } else {
#pragma unroll
      for (int p = 0; p < W; ++p) sMat[q][p] = q < F.nmat ? T(F.mtab[W * q + p]) : T(0);
    }
  }
  const int bx = int(blockIdx.x % nbx), by = int((blockIdx.x / nbx) % nby), bz = int(blockIdx.x / ((int64_t)nbx * nby));
  const int i = bx * kXOwn - 1 + lane;
  const int r0 = by * OY - 1 + 2 * w, r1 = r0 + 1;
  const int m = by * (OY / 2) + w;    // row pair (2m-1, 2m) of the cell-pair words
  const int K0 = bz * zchunk;
  const int K1 = min(K0 + zchunk, F.nzn);
  const bool xin = i >= 0 && i < F.nxn;
  const bool in0 = xin && r0 >= 0 && r0 < F.nyn, in1 = xin && r1 < F.nyn;
  const bool own_x = lane >= 1 && lane <= kXOwn && i < F.nxn;
  const bool own0 = own_x && w >= 1 && r0 < F.nyn, own1 = own_x && w <= WY - 2 && r1 < F.nyn;
  // 32-bit node offsets (feb_create keeps 3 x nodes below 2^31)
  const int plane = F.nxn * F.nyn;
  const int n0base = in0 ? i + F.nxn * r0 : 0, n1base = in1 ? i + F.nxn * r1 : 0;
  const int cpl = F.nxn * F.mp;
  const int cbase = (xin && m < F.mp) ? i + F.nxn * m : -1;
  const bool need_dir = SMOOTH && a1 != T(0);
  // geometry of the general path: this thread's x width and its two rows' y widths
  V ga(T(1)), gb(T(1)), gia(T(1)), gib(T(1));
  if constexpr (!CUBE) {
    const int ic = min(max(i, 0), F.nx - 1);
    const int j0 = min(max(r0, 0), F.ny - 1), j1 = min(max(r1, 0), F.ny - 1);
    ga = V(F.dx[ic]); gia = V(F.idx[ic]);
    gb = V(F.dy[j0], F.dy[j1]); gib = V(F.idy[j0], F.idy[j1]);
  }

  auto load_plane = [&](int k, V (&v)[3]) {
    const bool kin = k >= 0 && k < F.nzn;
    const int pk = plane * k;
    const T* p0 = u + 3 * (n0base + pk);
    const T* p1 = u + 3 * (n1base + pk);
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = V((kin && in0) ? p0[c] : T(0), (kin && in1) ? p1[c] : T(0));
  };
  auto load_cells = [&](int k) -> uint32_t {
    return (cbase >= 0 && k >= 0 && k < F.nzn) ? (uint32_t)F.cellpair[cbase + cpl * k] : 0u;
  };
  auto slot = [](int p) { return (p + 2) & 1; };
  // x-edge of a plane: E[c][0] = v + v(+x), E[c][1] = v(+x) - v
  auto edge = [&](const V (&v)[3], V (&E)[3][2]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const V nb = shfl_down2(v[c], 1);
      E[c][0] = v[c] + nb;
      E[c][1] = nb - v[c];
    }
  };
  auto put_edge = [&](int sl, const V (&E)[3][2]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) sE[sl][c][w][lane] = mk2<T>(E[c][0].lo(), E[c][1].lo());
  };
  // xy-face modes of the pair's two faces from this pair's edges and the row above: F[c][q] y-sum, F[c][q+2] y-diff
  auto face = [&](int sl, const V (&E)[3][2], V (&Fc)[3][4]) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      V2<T> a = mk2<T>(T(0), T(0));
      if (w + 1 < WY) a = sE[sl][c][w + 1][lane];
      const V up0 = shift_up(E[c][0], a.x), up1 = shift_up(E[c][1], a.y);
      Fc[c][0] = E[c][0] + up0; Fc[c][2] = up0 - E[c][0];
      Fc[c][1] = E[c][1] + up1; Fc[c][3] = up1 - E[c][1];
    }
  };
  // finishes node plane kk: y-edge totals (lower share + the share from the pair below), x back-transform,
  // epilogue of the owned nodes
  auto finish = [&](int kk, int sl, const V (&Lw)[3][2], const T (&Uhi)[3][2], uint32_t flags, const NodeOps<T>& o0,
                    const NodeOps<T>& o1) {
    V tot[3][2];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      V2<T> b = mk2<T>(T(0), T(0));
      if (w >= 1) b = sB[sl][c][w - 1][lane];
      tot[c][0] = Lw[c][0] + V(b.x, Uhi[c][0]);
      tot[c][1] = Lw[c][1] + V(b.y, Uhi[c][1]);
    }
    V out[3];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const V lo = tot[c][0] - tot[c][1], hi = tot[c][0] + tot[c][1];
      V left = shfl_up2(hi, 1);
      if (lane == 0) left = V(T(0));
      out[c] = lo + left;
    }
    if (kk < K0 || kk >= K1) return;
    const int n0 = n0base + plane * kk, n1 = n1base + plane * kk;
    T t0[3] = {out[0].lo(), out[1].lo(), out[2].lo()}, t1[3] = {out[0].hi(), out[1].hi(), out[2].hi()};
    if (own0 && (flags & 0x80u)) {
#pragma unroll
      for (int c = 0; c < 3; ++c) { t0[c] += F.tsp[3 * n0 + c]; F.tsp[3 * n0 + c] = T(0); }
    }
    if (own1 && (flags & 0x8000u)) {
#pragma unroll
      for (int c = 0; c < 3; ++c) { t1[c] += F.tsp[3 * n1 + c]; F.tsp[3 * n1 + c] = T(0); }
    }
    if constexpr (PREF) {
      if (own0) node_update(S, a1, a2, n0, t0, o0);
      if (own1) node_update(S, a1, a2, n1, t1, o1);
    } else if constexpr (SMOOTH) {
      NodeOps<T> o;
      if (own0) { load_node_ops(F, S, u, need_dir, n0, o); node_update(S, a1, a2, n0, t0, o); }
      if (own1) { load_node_ops(F, S, u, need_dir, n1, o); node_update(S, a1, a2, n1, t1, o); }
    } else {
      if (own0) {
#pragma unroll
        for (int c = 0; c < 3; ++c) y[3 * n0 + c] = t0[c];
      }
      if (own1) {
#pragma unroll
        for (int c = 0; c < 3; ++c) y[3 * n1 + c] = t1[c];
      }
    }
  };

  // Planes alternate between two register sets (input planes, faces, cell words, epilogue operands), and the
  // march takes two planes per trip, so no set is ever copied into the other.
  V va[3], vb[3];
  V Fa[3][4], Fb[3][4], topc[3][4], Lw[3][2];
  T Uhi[3][2];
  uint32_t ca, cb = 0u, flags_prev = 0u;
  NodeOps<T> oa0, oa1, ob0, ob1;
  auto prefetch = [&](int kk, NodeOps<T>& o0, NodeOps<T>& o1) {
    if constexpr (PREF) {
      if (kk >= K0 && kk < K1) {
        if (own0) load_node_ops(F, S, u, need_dir, n0base + plane * kk, o0);
        if (own1) load_node_ops(F, S, u, need_dir, n1base + plane * kk, o1);
      }
    }
  };
  {   // prologue: face of plane K0-1
    V v0[3], E[3][2];
    load_plane(K0 - 1, v0);
    load_plane(K0, va);
    load_plane(K0 + 1, vb);
    ca = load_cells(K0 - 1);
    edge(v0, E);
    put_edge(slot(K0 - 1), E);
    __syncthreads();
    face(slot(K0 - 1), E, Fa);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
#pragma unroll
      for (int l = 0; l < 4; ++l) topc[c][l] = V(T(0));
      Lw[c][0] = Lw[c][1] = V(T(0));
      Uhi[c][0] = Uhi[c][1] = T(0);
    }
  }
  prefetch(K0 - 1, oa0, oa1);
  // one step of the march at plane k: vin holds plane k+1 (and receives plane k+3), Fin the face of plane k,
  // Fout receives the face of plane k+1; cin holds the cell word of layer k, cout receives layer k+1; oin
  // holds the epilogue operands of plane k-1, oout receives those of plane k
  auto step = [&](int k, V (&vin)[3], V (&Fin)[3][4], V (&Fout)[3][4], uint32_t cin, uint32_t& cout,
                  NodeOps<T>& oin0, NodeOps<T>& oin1, NodeOps<T>& oout0, NodeOps<T>& oout1) {
    // (a) x-edge of plane k+1; prefetch plane k+3, the cells of layer k+1 and the epilogue operands of plane k
    V E[3][2];
    edge(vin, E);
    put_edge(slot(k + 1), E);
    load_plane(k + 3, vin);
    cout = load_cells(k + 1);
    prefetch(k, oout0, oout1);
    __syncthreads();
    // (b) finish plane k-1
    if (k > K0 - 1) finish(k - 1, slot(k - 1), Lw, Uhi, flags_prev, oin0, oin1);
    flags_prev = cin;
    // (c) faces of plane k+1, z butterfly -> modal coefficients of cell layer k
    face(slot(k + 1), E, Fout);
    V X[8], Y[8], Z[8];
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      X[l] = Fin[0][l] + Fout[0][l]; X[l + 4] = Fout[0][l] - Fin[0][l];
      Y[l] = Fin[1][l] + Fout[1][l]; Y[l + 4] = Fout[1][l] - Fin[1][l];
      Z[l] = Fin[2][l] + Fout[2][l]; Z[l + 4] = Fout[2][l] - Fin[2][l];
    }
    // (d) element core of the two cells (i, r0, k), (i, r1, k)
    V FX[8], FY[8], FZ[8];
    const int id0 = (lane < 31) ? int(cin & 0x7fu) : 0, id1 = (lane < 31) ? int((cin >> 8) & 0x7fu) : 0;
    if constexpr (CUBE) {
      const V L16(sMat[id0][0], sMat[id1][0]), M48(sMat[id0][1], sMat[id1][1]);
      cube_sri_core<T>(X, Y, Z, L16, M48, FX, FY, FZ);
    } else {
      Material<V> mt;
      {
        V mv[W];
#pragma unroll
        for (int p = 0; p < W; ++p) mv[p] = V(sMat[id0][p], sMat[id1][p]);
        mt = make_material<V, MODE>(mv);
      }
      const int kc = min(max(k, 0), F.nz - 1);
      const V gc(F.dz[kc]), gic(F.idz[kc]);
      pair_modal<T, HAS12>(X, Y, Z, make_coef(ga, gb, gc, gia, gib, gic, mt), FX, FY, FZ);
    }
    FX[0] = FY[0] = FZ[0] = V(T(0));
    // (e) z back-transform: the bottom share completes the faces of plane k, the top share carries to k+1
    V G[3][4];
#pragma unroll
    for (int l = 0; l < 4; ++l) {
      G[0][l] = topc[0][l] + (FX[l] - FX[l + 4]); topc[0][l] = FX[l] + FX[l + 4];
      G[1][l] = topc[1][l] + (FY[l] - FY[l + 4]); topc[1][l] = FY[l] + FY[l + 4];
      G[2][l] = topc[2][l] + (FZ[l] - FZ[l + 4]); topc[2][l] = FZ[l] + FZ[l + 4];
    }
    // (f) y back-transform of plane k: lower edges stay (rows r0, r1), upper edges go one row up; the
    //     upper edge of face r1 (row r1 + 1) goes to the warp above through shared memory
    const int sl = slot(k);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      V U[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) {
        Lw[c][q] = G[c][q] - G[c][q + 2];
        U[q] = G[c][q] + G[c][q + 2];
        Uhi[c][q] = U[q].lo();
      }
      sB[sl][c][w][lane] = mk2<T>(U[0].hi(), U[1].hi());
    }
  };
  if constexpr (kPairUnroll && std::is_same<T, float>::value) {
    int k = K0 - 1;
    for (; k + 1 < K1; k += 2) {
      step(k, va, Fa, Fb, ca, cb, oa0, oa1, ob0, ob1);
      step(k + 1, vb, Fb, Fa, cb, ca, ob0, ob1, oa0, oa1);
    }
    if (k < K1) {   // odd number of steps: the last one runs on the first set
      step(k, va, Fa, Fb, ca, cb, oa0, oa1, ob0, ob1);
      __syncthreads();
      finish(K1 - 1, slot(K1 - 1), Lw, Uhi, flags_prev, ob0, ob1);
    } else {
      __syncthreads();
      finish(K1 - 1, slot(K1 - 1), Lw, Uhi, flags_prev, oa0, oa1);
    }
  } else {   // FP64: one plane per trip, the second set copied into the first (no register room for both)
    for (int k = K0 - 1; k < K1; ++k) {
      step(k, va, Fa, Fb, ca, cb, oa0, oa1, ob0, ob1);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const V t = va[c]; va[c] = vb[c]; vb[c] = t;
#pragma unroll
        for (int l = 0; l < 4; ++l) Fa[c][l] = Fb[c][l];
      }
      ca = cb;
      if constexpr (PREF) { oa0 = ob0; oa1 = ob1; }
    }
    __syncthreads();
    finish(K1 - 1, slot(K1 - 1), Lw, Uhi, flags_prev, oa0, oa1);
  }
}

template <typename T, int MODE, bool CUBE, int WY, bool SMOOTH>
int launch_pair_kernel(const PairView<T>& F, const T* u, T* y, const SmoothArgs<T>& A, const int* skip, int zc,
                       cudaStream_t s) {
  constexpr int OY = 2 * WY - 2;
  const int nbx = div_up(F.nxn, kXOwn), nby = div_up(F.nyn, OY), nbz = div_up(F.nzn, zc);
  const int64_t blocks = (int64_t)nbx * nby * nbz + div_up(F.ntotal - F.nnode, 32 * WY);
  constexpr size_t smem = pair_smem_bytes<T, MODE, CUBE, WY>();
  auto kern = k_fine_pair<T, MODE, CUBE, WY, SMOOTH>;
  FEB_TRY(set_dyn_smem((const void*)kern, (int)smem));
  kern<<<(unsigned)blocks, 32 * WY, smem, s>>>(F, u, y, A, skip, zc, nbx, nby, nbz);
  note_launch();
  return FEB_OK;
}

template <typename T, int MODE, bool CUBE, int WY, bool SMOOTH>
int prepare_pair_kernel() {
  constexpr size_t smem = pair_smem_bytes<T, MODE, CUBE, WY>();
  return set_dyn_smem((const void*)k_fine_pair<T, MODE, CUBE, WY, SMOOTH>, (int)smem);
}

template <typename T, int MODE>
int prepare_pair_precision(bool cube) {
  if constexpr (MODE == MAT_ISO_SRI && std::is_same<T, float>::value) {
    if (cube) FEB_TRY((prepare_pair_kernel<T, MODE, true, 16, false>()));
  }
  if constexpr (MODE == MAT_ISO_SRI) {
    if (cube) {
      FEB_TRY((prepare_pair_kernel<T, MODE, true, 8, false>()));
      FEB_TRY((prepare_pair_kernel<T, MODE, true, 8, true>()));
    }
  }
  FEB_TRY((prepare_pair_kernel<T, MODE, false, 8, false>()));
  FEB_TRY((prepare_pair_kernel<T, MODE, false, 8, true>()));
  return FEB_OK;
}

template <typename T, int MODE, bool SMOOTH>
int launch_pair_wy(const PairView<T>& F, const T* u, T* y, const SmoothArgs<T>& A, const int* skip, PairConfig cfg,
                   cudaStream_t s) {
  if (SMOOTH) cfg.wy = 8;   // the smoothing variants need the register room of 8-warp CTAs
  const int zc = std::max(1, SMOOTH ? cfg.zchunk_smooth : cfg.zchunk);
  if constexpr (MODE == MAT_ISO_SRI) {
    if (F.cube) {
      if constexpr (std::is_same<T, float>::value && !SMOOTH) {
        if (cfg.wy == 16) return launch_pair_kernel<T, MODE, true, 16, SMOOTH>(F, u, y, A, skip, zc, s);
      }
      return launch_pair_kernel<T, MODE, true, 8, SMOOTH>(F, u, y, A, skip, zc, s);
    }
  }
  return launch_pair_kernel<T, MODE, false, 8, SMOOTH>(F, u, y, A, skip, zc, s);
}

// ------------------------------------------------------------------------------------------------ set-up
__device__ __forceinline__ uint64_t mix64(uint64_t z) {   // splitmix64 finaliser
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  return z ^ (z >> 31);
}

// Material id of every regular cell: open addressing over ids 1..kMaxMatIds-1 keyed by a 64-bit hash of the
// cell's W FP64 values.  The first thread to claim a slot writes its values; k_pack_pairs then checks every
// cell against the table (a hash collision or a full table sets the status word and the operator keeps the
// per-cell kernel).
template <int W>
__global__ void k_mat_ids(const double* __restrict__ mat_s, int64_t ncell, unsigned long long* __restrict__ keys,
                          double* __restrict__ vals, uint8_t* __restrict__ ids, int* __restrict__ status) {
  const int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (c >= ncell) return;
  double v[W];
  bool nz = false;
  uint64_t h = 0x9e3779b97f4a7c15ull;
#pragma unroll
  for (int q = 0; q < W; ++q) {
    v[q] = mat_s[W * c + q];
    nz |= (v[q] != 0.0);
    h = mix64(h ^ (uint64_t)__double_as_longlong(v[q]));
  }
  if (!nz) { ids[c] = 0; return; }
  h |= 1ull;
  const int nslot = kMaxMatIds - 1;
  const int s0 = int(h % (uint64_t)nslot);
  for (int p = 0; p < nslot; ++p) {
    const int sl = 1 + (s0 + p) % nslot;
    unsigned long long old = keys[sl];
    if (old == 0ull) old = atomicCAS(&keys[sl], 0ull, (unsigned long long)h);
    if (old == 0ull) {
#pragma unroll
      for (int q = 0; q < W; ++q) vals[W * sl + q] = v[q];
      ids[c] = (uint8_t)sl;
      return;
    }
    if (old == (unsigned long long)h) { ids[c] = (uint8_t)sl; return; }
  }
  ids[c] = 0;
  atomicOr(status, 1);
}

// node flags: grid nodes that receive a sparse contribution (penalty, extra entry, irregular cell corner)
__global__ void k_flag_nodes(const int* __restrict__ pen_node, int npen, const int* __restrict__ irr_nodes, int nirr,
                             const int* __restrict__ row_dof, int nrow, int64_t nnode, uint8_t* __restrict__ flag) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e < npen && pen_node[e] < nnode) flag[pen_node[e]] = 1;
  if (e < 8 * nirr && irr_nodes[e] < nnode) flag[irr_nodes[e]] = 1;
  if (e < nrow && row_dof[e] / 3 < nnode) flag[row_dof[e] / 3] = 1;
}

// cell-pair words [nzn][mp][nxn]: byte h (h = 0, 1) describes row j = 2m - 1 + h: bits 0-6 the material id
// of cell (i, j, k) (0 when the cell does not exist or is not regular), bit 7 the flag of node (i, j, k)
template <int W>
__global__ void k_pack_pairs(int nx, int ny, int nz, int mp, const uint8_t* __restrict__ ids,
                             const uint8_t* __restrict__ flag, const double* __restrict__ mat_s,
                             const double* __restrict__ vals, uint16_t* __restrict__ cellpair, int* __restrict__ status) {
  const int nxn = nx + 1, nyn = ny + 1, nzn = nz + 1;
  const int64_t total = (int64_t)nxn * mp * nzn;
  const int64_t e = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (e >= total) return;
  const int i = int(e % nxn), m = int((e / nxn) % mp), k = int(e / ((int64_t)nxn * mp));
  uint32_t word = 0;
  for (int hh = 0; hh < 2; ++hh) {
    const int j = 2 * m - 1 + hh;
    if (j < 0 || j >= nyn) continue;
    uint32_t byte = 0;
    if (i < nx && j < ny && k < nz) {
      const int64_t c = i + (int64_t)nx * (j + (int64_t)ny * k);
      const int id = ids[c];
      byte = (uint32_t)id;
      bool same = true;
#pragma unroll
      for (int q = 0; q < W; ++q) same &= (vals[W * id + q] == mat_s[W * c + q]);
      if (!same) atomicOr(status, 2);
    }
    if (flag[i + (int64_t)nxn * (j + (int64_t)nyn * k)]) byte |= 0x80u;
    word |= byte << (8 * hh);
  }
  cellpair[e] = (uint16_t)word;
}

// symmetric block-Jacobi inverse [6][n] (00 11 22 01 02 12) from the SoA [9][n] inverse
template <typename T>
__global__ void k_dinv6(const double* __restrict__ D, int64_t n, T* __restrict__ out) {
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  out[i] = T(D[i]);
  out[n + i] = T(D[4 * n + i]);
  out[2 * n + i] = T(D[8 * n + i]);
  out[3 * n + i] = T(0.5 * (D[n + i] + D[3 * n + i]));
  out[4 * n + i] = T(0.5 * (D[2 * n + i] + D[6 * n + i]));
  out[5 * n + i] = T(0.5 * (D[5 * n + i] + D[7 * n + i]));
}

// first Chebyshev step from a zero start: d = (1/theta) Dinv b (and x = d when x is given)
template <typename T>
__global__ void k_cheb_first6(const T* __restrict__ b, const T* __restrict__ D, const LevelParams* __restrict__ lp,
                              T* __restrict__ d, T* __restrict__ x, int64_t n, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T c = T(lp->c_init);
  const T r0 = b[3 * i], r1 = b[3 * i + 1], r2 = b[3 * i + 2];
  const T d00 = D[i], d11 = D[n + i], d22 = D[2 * n + i], d01 = D[3 * n + i], d02 = D[4 * n + i], d12 = D[5 * n + i];
  const T z0 = c * (d00 * r0 + d01 * r1 + d02 * r2);
  const T z1 = c * (d01 * r0 + d11 * r1 + d12 * r2);
  const T z2 = c * (d02 * r0 + d12 * r1 + d22 * r2);
  d[3 * i] = z0; d[3 * i + 1] = z1; d[3 * i + 2] = z2;
  if (x) { x[3 * i] = z0; x[3 * i + 1] = z1; x[3 * i + 2] = z2; }
}

}  // namespace

template <typename T, int MODE>
int launch_fine_pair(const PairView<T>& F, const FineView<T>& G, const T* u, T* y, const SmoothArgs<T>* S,
                     const int* skip, PairConfig cfg, cudaStream_t s) {
  if (G.nirr + G.npen + G.nrow > 0) launch_fine_sparse_into<T, MODE>(G, u, F.tsp, skip, s);
  if (S) return launch_pair_wy<T, MODE, true>(F, u, y, *S, skip, cfg, s);
  return launch_pair_wy<T, MODE, false>(F, u, y, SmoothArgs<T>{}, skip, cfg, s);
}

template <typename T, int MODE, bool CUBE, int WY, bool SMOOTH>
int pair_occupancy() {
  int nb = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, k_fine_pair<T, MODE, CUBE, WY, SMOOTH>, 32 * WY,
                                                    pair_smem_bytes<T, MODE, CUBE, WY>()) != cudaSuccess)
    return 1;
  return std::max(nb, 1);
}

template <typename T, bool SMOOTH>
int pair_occupancy_mode(int mode, bool cube) {
  if (mode == MAT_ISO_SRI && cube) return pair_occupancy<T, MAT_ISO_SRI, true, 8, SMOOTH>();
  switch (mode) {
    case MAT_ISO_SRI: return pair_occupancy<T, MAT_ISO_SRI, false, 8, SMOOTH>();
    case MAT_ISO_FULL: return pair_occupancy<T, MAT_ISO_FULL, false, 8, SMOOTH>();
    default: return pair_occupancy<T, MAT_ORTHO, false, 8, SMOOTH>();
  }
}

template <typename T>
int fine_pair_blocks_per_sm(int mode, bool cube, int wy, bool smooth) {
  if (smooth) return pair_occupancy_mode<T, true>(mode, cube);
  if constexpr (std::is_same<T, float>::value) {
    if (wy == 16 && mode == MAT_ISO_SRI && cube) return pair_occupancy<T, MAT_ISO_SRI, true, 16, false>();
  }
  return pair_occupancy_mode<T, false>(mode, cube);
}
template int fine_pair_blocks_per_sm<float>(int, bool, int, bool);
template int fine_pair_blocks_per_sm<double>(int, bool, int, bool);

int fine_pair_tiles_xy(int nxn, int nyn, int wy) { return div_up(nxn, kXOwn) * div_up(nyn, 2 * wy - 2); }

int prepare_fine_pair(int mode, bool cube) {
  switch (mode) {
    case MAT_ISO_SRI:
      FEB_TRY((prepare_pair_precision<float, MAT_ISO_SRI>(cube)));
      return prepare_pair_precision<double, MAT_ISO_SRI>(cube);
    case MAT_ISO_FULL:
      FEB_TRY((prepare_pair_precision<float, MAT_ISO_FULL>(cube)));
      return prepare_pair_precision<double, MAT_ISO_FULL>(cube);
    default:
      FEB_TRY((prepare_pair_precision<float, MAT_ORTHO>(cube)));
      return prepare_pair_precision<double, MAT_ORTHO>(cube);
  }
}

template <int W>
void launch_mat_ids(const double* mat_s, int64_t ncell, unsigned long long* keys, double* vals, uint8_t* ids,
                    int* status, cudaStream_t s) {
  k_mat_ids<W><<<div_up(ncell, kThreads), kThreads, 0, s>>>(mat_s, ncell, keys, vals, ids, status); note_launch();
}
void launch_flag_nodes(const int* pen_node, int npen, const int* irr_nodes, int nirr, const int* row_dof, int nrow,
                       int64_t nnode, uint8_t* flag, cudaStream_t s) {
  const int n = std::max(npen, std::max(8 * nirr, nrow));
  if (n > 0) {
    k_flag_nodes<<<div_up(n, kThreads), kThreads, 0, s>>>(pen_node, npen, irr_nodes, nirr, row_dof, nrow, nnode, flag);
    note_launch();
  }
}
template <int W>
void launch_pack_pairs(int nx, int ny, int nz, int mp, const uint8_t* ids, const uint8_t* flag, const double* mat_s,
                       const double* vals, uint16_t* cellpair, int* status, cudaStream_t s) {
  const int64_t total = (int64_t)(nx + 1) * mp * (nz + 1);
  k_pack_pairs<W><<<div_up(total, kThreads), kThreads, 0, s>>>(nx, ny, nz, mp, ids, flag, mat_s, vals, cellpair, status);
  note_launch();
}
template <typename T>
void launch_dinv6(const double* D9, int64_t n, T* out, cudaStream_t s) {
  k_dinv6<T><<<div_up(n, kThreads), kThreads, 0, s>>>(D9, n, out); note_launch();
}
template <typename T>
void launch_cheb_first6(const T* b, const T* D6, const LevelParams* lp, T* d, T* x, int64_t n, const int* skip,
                        cudaStream_t s) {
  k_cheb_first6<T><<<div_up(n, kThreads), kThreads, 0, s>>>(b, D6, lp, d, x, n, skip); note_launch();
}

#define INST(T, M)                                                                                          \
  template int launch_fine_pair<T, M>(const PairView<T>&, const FineView<T>&, const T*, T*, const SmoothArgs<T>*, \
                                      const int*, PairConfig, cudaStream_t);
INST(float, MAT_ISO_SRI) INST(float, MAT_ISO_FULL) INST(float, MAT_ORTHO)
INST(double, MAT_ISO_SRI) INST(double, MAT_ISO_FULL) INST(double, MAT_ORTHO)
#undef INST
template void launch_mat_ids<2>(const double*, int64_t, unsigned long long*, double*, uint8_t*, int*, cudaStream_t);
template void launch_mat_ids<6>(const double*, int64_t, unsigned long long*, double*, uint8_t*, int*, cudaStream_t);
template void launch_pack_pairs<2>(int, int, int, int, const uint8_t*, const uint8_t*, const double*, const double*,
                                   uint16_t*, int*, cudaStream_t);
template void launch_pack_pairs<6>(int, int, int, int, const uint8_t*, const uint8_t*, const double*, const double*,
                                   uint16_t*, int*, cudaStream_t);
template void launch_dinv6<float>(const double*, int64_t, float*, cudaStream_t);
template void launch_dinv6<double>(const double*, int64_t, double*, cudaStream_t);
template void launch_cheb_first6<float>(const float*, const float*, const LevelParams*, float*, float*, int64_t,
                                        const int*, cudaStream_t);
template void launch_cheb_first6<double>(const double*, const double*, const LevelParams*, double*, double*, int64_t,
                                         const int*, cudaStream_t);

}  // namespace feb
