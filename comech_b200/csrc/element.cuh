// Matrix-free hex8 element operator in a modal (mean / difference per axis) basis.
//
// The reference forms K_e = lam K_lambda + mu K_mu (24x24, 2x2x2 Gauss, fe/solver.py:77-90; the split
// engine uses the one-point lambda matrix, rb/splitfe.py:58-69) and multiplies it with u_e.  Here the
// same product is evaluated exactly with ~200 operations instead of 2 x 576 FMAs:
//
//  * per axis the two nodal values (v0, v1) become (m, d) = ((v0+v1)/2, v1-v0), the coefficients of the
//    orthogonal basis {1, s-1/2} on [0,1] (norms 1 and 1/12);
//  * a trilinear field's derivative along x only has modes that are constant in x, so every strain
//    component is a short list of modal coefficients; products of modes integrate to a diagonal
//    weight vol * prod(N), which is what the 2x2x2 Gauss rule integrates exactly;
//  * stresses are D times strains mode by mode; the nodal forces are the transpose of the strain map,
//    then the transpose of the modal transform;
//  * the factors 1/2 and N, the material and the geometry fold into 20 per-cell constants, so the
//    transforms are pure additions and the core is ~50 FMAs.
//
// The result equals K_e u_e of the reference to rounding (checked against the reference's element
// matrices for SRI, full and orthotropic materials).
#pragma once
#include "common.cuh"

namespace feb {

template <typename T>
struct Material {
  T c0, c1, c2, c3, c4, c5;   // D pattern coefficients (fe/solver.py:43-52), integrated 2x2x2
  T lamc;                      // lambda at the cell centre (one-point, SRI)
};

template <typename T, int MODE>
__device__ __forceinline__ Material<T> make_material(const T* p) {
  Material<T> m;
  if constexpr (MODE == MAT_ORTHO) {
    m.c0 = p[0]; m.c1 = p[1]; m.c2 = p[2]; m.c3 = p[3]; m.c4 = p[4]; m.c5 = p[5]; m.lamc = T(0);
  } else {
    T lam = p[0], mu = p[1];
    T lf = (MODE == MAT_ISO_FULL) ? lam : T(0);
    m.c0 = lf + T(2) * mu; m.c1 = lf; m.c2 = lf; m.c3 = lf + T(2) * mu; m.c4 = mu; m.c5 = mu;
    m.lamc = (MODE == MAT_ISO_SRI) ? lam : T(0);
  }
  return m;
}

// Per-cell constants of the element operator: products of the material pattern coefficients with the
// cell geometry (gx = bc/a, gy = ac/b, gz = ab/c and the edge lengths), the centre-mode versions carrying
// the one-point lambda term.
template <typename T>
struct ElemCoef {
  T dx0, dy0, dz3;              // c0 gx, c0 gy, c3 gz
  T x4, x5, y4, y5, z5;         // c4 gx, c5 gx, c4 gy, c5 gy, c5 gz
  T c1c, c2b, c2a;              // c1 c, c2 b, c2 a
  T c4c, c5b, c5a;              // c4 c, c5 b, c5 a
  T ex0, ey0, ez3, ec1c, ec2b, ec2a;   // centre mode: c -> c + lambda_c
};

template <typename T>
__device__ __forceinline__ ElemCoef<T> make_coef(T a, T b, T cc, T ia, T ib, T ic, const Material<T>& m) {
  ElemCoef<T> k;
  const T gx = b * cc * ia, gy = a * cc * ib, gz = a * b * ic;
  k.dx0 = m.c0 * gx; k.dy0 = m.c0 * gy; k.dz3 = m.c3 * gz;
  k.x4 = m.c4 * gx; k.x5 = m.c5 * gx; k.y4 = m.c4 * gy; k.y5 = m.c5 * gy; k.z5 = m.c5 * gz;
  k.c1c = m.c1 * cc; k.c2b = m.c2 * b; k.c2a = m.c2 * a;
  k.c4c = m.c4 * cc; k.c5b = m.c5 * b; k.c5a = m.c5 * a;
  k.ex0 = (m.c0 + m.lamc) * gx; k.ey0 = (m.c0 + m.lamc) * gy; k.ez3 = (m.c3 + m.lamc) * gz;
  k.ec1c = (m.c1 + m.lamc) * cc; k.ec2b = (m.c2 + m.lamc) * b; k.ec2a = (m.c2 + m.lamc) * a;
  return k;
}

// Unscaled butterflies: (v0, v1) -> (v0 + v1, v1 - v0) per axis, and the transpose (f0, f1) -> (f0 - f1, f0 + f1).
// With them the true modal coefficients carry a factor 2^-(#mean indices) on both sides; together with the
// basis norms N = 12^-(#difference indices) every output mode l is scaled by Q(#difference indices of l):
// Q = 12 4^-#m 12^-#d = 1/16, 1/48, 1/144 for 1, 2, 3 difference indices (applied once, to the inputs).
template <typename T>
__device__ __forceinline__ void butterfly_fwd(T (&v)[8]) {
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1)
#pragma unroll
    for (int l = 0; l < 8; ++l)
      if (!(l & bit)) {
        T v0 = v[l], v1 = v[l | bit];
        v[l] = v0 + v1;
        v[l | bit] = v1 - v0;
      }
}

template <typename T>
__device__ __forceinline__ void butterfly_bwd(T (&f)[8]) {
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1)
#pragma unroll
    for (int l = 0; l < 8; ++l)
      if (!(l & bit)) {
        T m = f[l], d = f[l | bit];
        f[l] = m - d;
        f[l | bit] = m + d;
      }
}

// Modal core: X, Y, Z hold the unscaled modal coefficients (butterfly_fwd of the corner values) of the
// three displacement components; on return FX, FY, FZ hold the modal forces to feed butterfly_bwd.
// HAS12: the material has nonzero c1 / c2 (false for the SRI isotropic model, whose cross normal terms
// vanish outside the centre mode).
template <typename T, bool HAS12>
__device__ __forceinline__ void hex8_modal(T (&X)[8], T (&Y)[8], T (&Z)[8], const ElemCoef<T>& k, T (&FX)[8],
                                           T (&FY)[8], T (&FZ)[8]) {
#pragma unroll
  for (int l = 1; l < 8; ++l) {
    const int nd = (l & 1) + ((l >> 1) & 1) + ((l >> 2) & 1);
    const T q = nd == 1 ? T(1.0 / 16.0) : (nd == 2 ? T(1.0 / 48.0) : T(1.0 / 144.0));
    X[l] *= q; Y[l] *= q; Z[l] *= q;
  }
  FX[0] = FY[0] = FZ[0] = T(0);
  // x-derivative slots: modes (d, be, ga)
#pragma unroll
  for (int be = 0; be < 2; ++be)
#pragma unroll
    for (int ga = 0; ga < 2; ++ga) {
      const int l = 1 + 2 * be + 4 * ga;
      const bool ce = (be == 0) && (ga == 0);
      T fx = (ce ? k.ex0 : k.dx0) * X[l];
      if (be == 0 && (HAS12 || ce)) fx += (ce ? k.ec1c : k.c1c) * Y[2 + 4 * ga];
      if (ga == 0 && (HAS12 || ce)) fx += (ce ? k.ec2b : k.c2b) * Z[4 + 2 * be];
      T fy = k.x4 * Y[l];
      if (be == 0) fy += k.c4c * X[2 + 4 * ga];
      T fz = k.x5 * Z[l];
      if (ga == 0) fz += k.c5b * X[4 + 2 * be];
      FX[l] = fx; FY[l] = fy; FZ[l] = fz;
    }
  // y-derivative slots: modes (al, d, ga); (1,1,ga) was written by the x slots
#pragma unroll
  for (int al = 0; al < 2; ++al)
#pragma unroll
    for (int ga = 0; ga < 2; ++ga) {
      const int l = al + 2 + 4 * ga;
      const bool ce = (al == 0) && (ga == 0);
      T fy = (ce ? k.ey0 : k.dy0) * Y[l];
      if (al == 0 && (HAS12 || ce)) fy += (ce ? k.ec1c : k.c1c) * X[1 + 4 * ga];
      if (ga == 0 && (HAS12 || ce)) fy += (ce ? k.ec2a : k.c2a) * Z[al + 4];
      T fx = k.y4 * X[l];
      if (al == 0) fx += k.c4c * Y[1 + 4 * ga];
      T fz = k.y5 * Z[l];
      if (ga == 0) fz += k.c5a * Y[al + 4];
      if (al) { FX[l] += fx; FY[l] += fy; FZ[l] += fz; }
      else { FX[l] = fx; FY[l] = fy; FZ[l] = fz; }
    }
  // z-derivative slots: modes (al, be, d)
#pragma unroll
  for (int al = 0; al < 2; ++al)
#pragma unroll
    for (int be = 0; be < 2; ++be) {
      const int l = al + 2 * be + 4;
      const bool ce = (al == 0) && (be == 0);
      T fz = (ce ? k.ez3 : k.dz3) * Z[l];
      if (al == 0 && (HAS12 || ce)) fz += (ce ? k.ec2b : k.c2b) * X[1 + 2 * be];
      if (be == 0 && (HAS12 || ce)) fz += (ce ? k.ec2a : k.c2a) * Y[al + 2];
      T fy = k.z5 * Y[l];
      if (be == 0) fy += k.c5a * Z[al + 2];
      T fx = k.z5 * X[l];
      if (al == 0) fx += k.c5b * Z[1 + 2 * be];
      if (al || be) { FX[l] += fx; FY[l] += fy; FZ[l] += fz; }
      else { FX[l] = fx; FY[l] = fy; FZ[l] = fz; }
    }
}

// f = K_e u with the constants k (u, f: [component][corner], corner l = a + 2b + 4c)
template <typename T, bool HAS12>
__device__ __forceinline__ void hex8_core(const T (&u)[3][8], const ElemCoef<T>& k, T (&f)[3][8]) {
  T X[8], Y[8], Z[8];
#pragma unroll
  for (int l = 0; l < 8; ++l) { X[l] = u[0][l]; Y[l] = u[1][l]; Z[l] = u[2][l]; }
  butterfly_fwd(X);
  butterfly_fwd(Y);
  butterfly_fwd(Z);
  T FX[8], FY[8], FZ[8];
  hex8_modal<T, HAS12>(X, Y, Z, k, FX, FY, FZ);
  butterfly_bwd(FX);
  butterfly_bwd(FY);
  butterfly_bwd(FZ);
#pragma unroll
  for (int l = 0; l < 8; ++l) { f[0][l] = FX[l]; f[1][l] = FY[l]; f[2][l] = FZ[l]; }
}

// f = K_e u (the reference's lam K_lambda + mu K_mu product, or sum_k c_k K_k for orthotropic cells)
template <typename T>
__device__ __forceinline__ void hex8_apply(const T (&u)[3][8], T a, T b, T cc, T ia, T ib, T ic,
                                           const Material<T>& m, T (&f)[3][8]) {
  hex8_core<T, true>(u, make_coef(a, b, cc, ia, ib, ic, m), f);
}

// Centre-point strain (Voigt xx yy zz xy yz xz, engineering shear): eps = B_c u (fe/solver.py:257-261).
template <typename T>
__device__ __forceinline__ void hex8_centre_strain(const T (&u)[3][8], T ia, T ib, T ic, T (&eps)[6]) {
  // at the centre every derivative is the mean over the four edges of the difference along that axis
  T d[3][3];   // d[c][axis]
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    T sx = 0, sy = 0, sz = 0;
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      T s = u[c][l];
      sx += (l & 1) ? s : -s;
      sy += (l & 2) ? s : -s;
      sz += (l & 4) ? s : -s;
    }
    d[c][0] = T(0.25) * sx * ia;
    d[c][1] = T(0.25) * sy * ib;
    d[c][2] = T(0.25) * sz * ic;
  }
  eps[0] = d[0][0];
  eps[1] = d[1][1];
  eps[2] = d[2][2];
  eps[3] = d[0][1] + d[1][0];
  eps[4] = d[1][2] + d[2][1];
  eps[5] = d[0][2] + d[2][0];
}

}  // namespace feb
