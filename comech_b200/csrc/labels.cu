// Voxel labelling of a foot lattice (rb/rbgeom.py:493-524 label_lattice, :358-464 label_points).
//
// One thread per lattice point; the point's label is independent of every other point's, so the reference's
// array-wide masks become per-point branches.  Points that no edit can reach (outside the joint box and the
// regions of the active warps, rb/rbgeom.py:507-520) take the raster label at their template position; every
// other point runs the whole label_points rule.  All arithmetic is FP64 in the reference's operation order, and
// the file is compiled without multiply-add contraction (-fmad=false) so each product and sum rounds on its own
// as NumPy's elementwise operations do.  The joint-distance maps are FP32 and are summed and compared in FP32, as
// NumPy compares a float32 array with a Python float (the float is cast to float32 first).
#include <cmath>

#include "common.cuh"
#include "../../include/feb200.h"

namespace feb {

namespace {

constexpr int kSoft = 63, kCoal = 101, kFib = 102, kInterp = 103, kFuse = 104, kGap = 105;
constexpr int kPost = 12, kMid = 8, kAnt = 10;   // facet cartilage labels; facet index 0 post, 1 mid, 2 ant
__device__ __forceinline__ int facet_label(int f) { return f == 0 ? kPost : (f == 1 ? kMid : kAnt); }

struct V3 {
  double x, y, z;
};

__device__ __forceinline__ double dot3(V3 q, const double (&e)[3]) { return (q.x * e[0] + q.y * e[1]) + q.z * e[2]; }

__device__ __forceinline__ bool is_static(const FebLabelParams& p, int L) {
  return L >= 0 && L < 128 && ((p.static_mask[L >> 5] >> (L & 31)) & 1u);
}

__device__ __forceinline__ int lookup(const FebLabelParams& p, V3 q) {
  const double fx = floor((q.x - p.o[0]) / p.h), fy = floor((q.y - p.o[1]) / p.h), fz = floor((q.z - p.o[2]) / p.h);
  if (!(fx >= 0.0 && fx < p.lnx && fy >= 0.0 && fy < p.lny && fz >= 0.0 && fz < p.lnz)) return 0;
  return p.lab[((int64_t)fx * p.lny + (int64_t)fy) * p.lnz + (int64_t)fz];
}

__device__ __forceinline__ float sub_lookup(const FebLabelParams& p, const float* arr, V3 q) {
  const double fx = floor((q.x - p.so[0]) / p.h), fy = floor((q.y - p.so[1]) / p.h), fz = floor((q.z - p.so[2]) / p.h);
  if (!(fx >= 0.0 && fx < p.snx && fy >= 0.0 && fy < p.sny && fz >= 0.0 && fz < p.snz)) return 99.0f;
  return arr[((int64_t)fx * p.sny + (int64_t)fy) * p.snz + (int64_t)fz];
}

// smooth local displacement template -> foot (rb/rbgeom.py:243-256)
__device__ V3 warp(const FebLabelParams& p, V3 P) {
  V3 d = {0.0, 0.0, 0.0};
  const FebLabelFacet& fm = p.facet[1];
  const FebLabelFacet& fp = p.facet[0];
  if (p.sust_y != 11.0) {
    const double ax = P.x - fm.c[0], ay = P.y - fm.c[1], az = P.z - fm.c[2];
    const double r2 = (ax * ax + ay * ay) + az * az;
    d.y = d.y + (p.sust_y - 11.0) * exp(-r2 / 128.0);
  }
  if (p.post_dome != 1.5) {
    const V3 q = {P.x - fp.c[0], P.y - fp.c[1], P.z - fp.c[2]};
    const double u = (dot3(q, fp.e1) - fp.uc) / (fp.a0 + 2.0);
    const double v = (dot3(q, fp.e2) - fp.vc) / (fp.b0 + 2.0);
    const double w = dot3(q, fp.n);
    const double amp = ((p.post_dome - 1.5) * fmax((1.0 - u * u) - v * v, 0.0)) * exp(-(w * w) / 72.0);
    d.x = d.x + amp * fp.n[0];
    d.y = d.y + amp * fp.n[1];
    d.z = d.z + amp * fp.n[2];
  }
  return d;
}

// template point of world content p2 (after the scale and the fragment shift): shear, then the warps undone
// by three fixed-point steps (rb/rbgeom.py:298-305)
__device__ V3 unwarp(const FebLabelParams& p, V3 p2) {
  V3 p1 = p2;
  if (p.align_on) {
    const double w = fmin(fmax((p.x_w1 - p2.x) / (p.x_w1 - p.x_w0), 0.0), 1.0);
    p1.y = p2.y - ((-p.tan_align) * fmax(p.z_ref - p2.z, 0.0)) * w;
  }
  if (p.sust_y != 11.0 || p.post_dome != 1.5) {
    V3 d = warp(p, p1);
    V3 q = {p1.x - d.x, p1.y - d.y, p1.z - d.z};
    for (int it = 0; it < 3; ++it) {
      d = warp(p, q);
      q = {p1.x - d.x, p1.y - d.y, p1.z - d.z};
    }
    return q;
  }
  return p1;
}

__device__ __forceinline__ bool footprint(const FebLabelFacet& F, double u, double v) {
  const double fu = floor((u - F.ua) / F.res), fv = floor((v - F.va) / F.res);
  if (!(fu >= 0.0 && fu < F.nu && fv >= 0.0 && fv < F.nv)) return false;
  return F.F0[(int64_t)fu * F.nv + (int64_t)fv] != 0;
}

__device__ __forceinline__ bool front(const FebLabelFacet& F, const FebLabelGrown& g, double u, double v) {
  return g.on && ((u - F.uc) * g.d[0] + (v - F.vc) * g.d[1] <= g.thr);
}

// label_points at one world point (rb/rbgeom.py:358-464)
__device__ int label_point(const FebLabelParams& p, V3 P) {
  const V3 p3 = {p.c0[0] + (P.x - p.c0[0]) / p.scale, p.c0[1] + (P.y - p.c0[1]) / p.scale,
                 p.c0[2] + (P.z - p.c0[2]) / p.scale};
  bool frag = false;
  if (p.osteo != 0.0) frag = (p3.x < p.x_cut0 + p.cut_slope * (p3.z - p.z_cut0)) && (p3.z < p.z_frag_top);
  const V3 ps = unwarp(p, p3);
  int L = lookup(p, ps);
  if (frag) {
    const V3 pm = unwarp(p, {p3.x, p3.y - p.osteo, p3.z});
    const int Lm = lookup(p, pm);
    if (!is_static(p, L)) L = is_static(p, Lm) ? kSoft : Lm;
    return L;   // fragment points take no subtalar edit
  }
  // subtalar edits near the joint
  const bool near = ps.x >= p.so[0] && ps.x < p.so[0] + p.snx * p.h && ps.y >= p.so[1] && ps.y < p.so[1] + p.sny * p.h &&
                    ps.z >= p.so[2] && ps.z < p.so[2] + p.snz * p.h;
  if (!near) return L;
  const float dt = sub_lookup(p, p.dt, ps), dc = sub_lookup(p, p.dc, ps);
  const float gapw = dt + dc;
  double fu[3], fv[3], fw[3];
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    const FebLabelFacet& F = p.facet[f];
    const V3 q = {ps.x - F.c[0], ps.y - F.c[1], ps.z - F.c[2]};
    fu[f] = dot3(q, F.e1); fv[f] = dot3(q, F.e2); fw[f] = dot3(q, F.n);
  }
  auto soft_or_empty = [&](int l) { return l == kSoft || l == 0; };
  // facet sizes: cartilage outside the scaled footprint removed, added in the thin gap inside it
#pragma unroll
  for (int f = 0; f < 3; ++f) {
    const FebLabelFacet& F = p.facet[f];
    const double fa = p.fa[f], fb = p.fb[f];
    const double u = fu[f], v = fv[f], w = fw[f];
    bool ins = fabs(w) <= F.wmax + 1.0 && fabs(u - F.uc) <= (1.7 * F.a0) * fmax(fa, 1.0) &&
               fabs(v - F.vc) <= (1.7 * F.b0) * fmax(fb, 1.0);
    ins = ins && footprint(F, F.uc + (u - F.uc) / fa, F.vc + (v - F.vc) / fb);
    if (fa != 1.0 || fb != 1.0) {
      if (ins && gapw <= (float)(1.6 * F.gap) && soft_or_empty(L)) L = facet_label(f);
      if (L == facet_label(f) && !ins) L = kSoft;
    }
  }
  const FebLabelFacet& Fp = p.facet[0];
  const FebLabelFacet& Fm = p.facet[1];
  const FebLabelFacet& Fa = p.facet[2];
  if (p.ant_mode == 1) {   // anterior facet confluent with the middle one
    const double s0 = Fa.c[0] - Fm.c[0], s1 = Fa.c[1] - Fm.c[1], s2 = Fa.c[2] - Fm.c[2];
    const double q0 = ps.x - Fm.c[0], q1 = ps.y - Fm.c[1], q2 = ps.z - Fm.c[2];
    const double t = ((q0 * s0 + q1 * s1) + q2 * s2) / ((s0 * s0 + s1 * s1) + s2 * s2);
    const double r0 = q0 - t * s0, r1 = q1 - t * s1, r2 = q2 - t * s2;
    const double dist = sqrt((r0 * r0 + r1 * r1) + r2 * r2);
    if (t > 0.0 && t < 1.0 && dist < 0.75 * fmin(Fm.b0 * p.fb[1], Fa.b0 * p.fb[2]) &&
        gapw <= (float)(1.6 * fmax(Fm.gap, Fa.gap)) && soft_or_empty(L))
      L = kAnt;
  } else if (p.ant_mode == 2) {
    if (L == kAnt) L = kSoft;
  }
  // coalitions and defects
  const bool mid_c = L == kMid, post_c = L == kPost;
  const double um = fu[1], vm = fv[1], wm = fw[1], up = fu[0], vp = fv[0];
  const double kk = 2.0 / sqrt(M_PI);
  bool br = false, fib = false;
  if (p.ctype != 0) {
    const bool gap_bar = dt <= 4.0f && dc <= 4.0f && soft_or_empty(L);
    if (p.ctype == 1 || p.ctype == 4) {
      if (p.rtype >= 1 && p.rtype <= 3) {
        const double bb = Fm.b0 * p.fb[1];
        const bool band = mid_c && vm >= Fm.vc + bb * (1.0 - 2.0 * p.cov_mid);
        br = br || band;
        if (p.rtype == 2) {
          const double xe = Fm.c[0] - (Fm.c[0] - Fm.xyz_lo[0]) * p.fa[1];
          const double a = (ps.x - (xe - 2.5)) / (3.5 * kk), b = (ps.y - (Fm.c[1] + 1.5)) / (2.0 * kk);
          br = br || (gap_bar && a * a + b * b <= 1.0 && fabs(wm) < 6.0);
        }
        if (p.rtype == 3) {
          const double aa = Fm.a0 * p.fa[1];
          fib = band && um < (Fm.uc - aa) + (2.0 * aa) * p.fib_frac;
          br = br && !fib;
        }
      } else {
        br = br || (mid_c && front(Fm, p.g_cov_mid, um, vm));
      }
    }
    if (p.ctype == 2 || p.ctype == 4) br = br || (post_c && front(Fp, p.g_cov_post, up, vp));
    if (p.ctype == 3 || p.ctype == 4) {
      const double x_lo = Fp.c[0] + 2.0;
      const double x_hi = (Fm.c[0] - (Fm.c[0] - Fm.xyz_lo[0]) * p.fa[1]) + 1.0;
      const double y_lo = (Fp.c[1] + (Fp.xyz_hi[1] - Fp.c[1]) * p.fb[0]) - 3.0;
      const double y_hi = Fm.c[1] + 3.0;
      const double ex = (0.5 * (x_hi - x_lo)) * kk, ey = (0.5 * (y_hi - y_lo)) * kk;
      const double a = (ps.x - 0.5 * (x_lo + x_hi)) / ex, b = (ps.y - 0.5 * (y_lo + y_hi)) / ey;
      br = br || (gap_bar && a * a + b * b <= 1.0);
    }
  }
  const bool dm = mid_c && front(Fm, p.g_d_mid, um, vm);
  const bool dp = post_c && front(Fp, p.g_d_post, up, vp);
  if (p.fusion) {
    const bool facet = L == kPost || L == kMid || L == kAnt;
    if (facet || br || fib || (gapw <= 4.0f && dt <= 4.0f && dc <= 4.0f && soft_or_empty(L))) L = kFuse;
  } else if (p.resect) {
    const bool hole = br || fib || dm || dp;
    if (hole) {
      if (p.interp) L = kInterp;
      else if (p.void_fill) L = kGap;
      else L = (mid_c || post_c) ? kSoft : kGap;
    }
  } else {
    if (br) L = kCoal;
    if (fib) L = kFib;
    if ((dm || dp) && !br && !fib) L = p.void_fill ? kGap : kSoft;
  }
  return L;
}

__global__ void k_label_lattice(FebLabelParams p, const double* __restrict__ sx, int nx, const double* __restrict__ sy,
                                int ny, const double* __restrict__ sz, int nz, int16_t* __restrict__ out) {
  const int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (t >= (int64_t)nx * ny * nz) return;
  const int k = int(t % nz), j = int((t / nz) % ny), i = int(t / ((int64_t)nz * ny));
  const V3 P = {sx[i], sy[j], sz[k]};
  const double tx = p.c0[0] + (P.x - p.c0[0]) / p.scale, ty = p.c0[1] + (P.y - p.c0[1]) / p.scale,
               tz = p.c0[2] + (P.z - p.c0[2]) / p.scale;
  // the points an edit can reach (rb/rbgeom.py:507-520)
  bool need = tx >= -82.0 && tx <= -12.0 && ty >= -32.0 && ty <= 32.0 && tz >= 36.0 && tz <= 92.0;
  if (p.align_on) need = need || (tx < p.x_w1 + 1.0 && tz < p.z_ref + 1.0);
  if (p.osteo != 0.0) need = need || (tx < (p.x_cut0 + p.cut_slope * (tz - p.z_cut0)) + 1.0 && tz < p.z_frag_top + 1.0);
  if (p.sust_y != 11.0) {
    const double* c = p.facet[1].c;
    const double r = ((4 * 8.0) + fabs(p.sust_y - 11.0)) + 1.0;
    need = need || (fabs(tx - c[0]) < r && fabs(ty - c[1]) < r && fabs(tz - c[2]) < r);
  }
  if (p.post_dome != 1.5) {
    const double* c = p.facet[0].c;
    need = need || (fabs(tx - c[0]) < 40.0 && fabs(ty - c[1]) < 40.0 && fabs(tz - c[2]) < 40.0);
  }
  out[t] = (int16_t)(need ? label_point(p, P) : lookup(p, {tx, ty, tz}));
}

}  // namespace

}  // namespace feb

extern "C" FEB_API int feb_label_lattice(const FebLabelParams* p, const double* sx, int32_t nx, const double* sy,
                                         int32_t ny, const double* sz, int32_t nz, int16_t* L, void* stream) {
  if (!p || !sx || !sy || !sz || !L || nx < 0 || ny < 0 || nz < 0 || !p->lab || p->scale == 0.0) {
    feb::set_last_error("feb_label_lattice: bad argument");
    return FEB_ERR_ARG;
  }
  for (int f = 0; f < 3; ++f)
    if (!p->facet[f].F0 && (p->facet[f].nu > 0 && p->facet[f].nv > 0)) {
      feb::set_last_error("feb_label_lattice: facet %d has no footprint raster", f);
      return FEB_ERR_ARG;
    }
  if (!p->dt || !p->dc) { feb::set_last_error("feb_label_lattice: distance maps missing"); return FEB_ERR_ARG; }
  const int64_t n = (int64_t)nx * ny * nz;
  if (n == 0) return FEB_OK;
  feb::k_label_lattice<<<(unsigned)feb::div_up(n, 256), 256, 0, (cudaStream_t)stream>>>(*p, sx, nx, sy, ny, sz, nz, L);
  feb::note_launch();
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) { feb::set_last_error("feb_label_lattice: %s", cudaGetErrorString(e)); return FEB_ERR_CUDA; }
  return FEB_OK;
}
