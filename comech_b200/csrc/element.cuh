// Matrix-free hex8 element operator in a modal (mean / difference per axis) basis.
//
// The reference forms K_e = lam K_lambda + mu K_mu (24x24, 2x2x2 Gauss, fe/solver.py:77-90; the split
// engine uses the one-point lambda matrix, rb/splitfe.py:58-69) and multiplies it with u_e.  Here the
// same product is evaluated exactly, with ~300 flops instead of 2x576 FMAs:
//
//  * per axis the two nodal values (v0, v1) become (m, d) = ((v0+v1)/2, v1-v0), i.e. the coefficients
//    of the orthogonal basis {1, s-1/2} on [0,1] (norms 1 and 1/12);
//  * a trilinear field's derivative along x only has modes that are constant in x, so every strain
//    component is a short list of modal coefficients; products of modes integrate to a diagonal
//    weight vol * prod(N), which is what the 2x2x2 Gauss rule integrates exactly;
//  * stresses are D times strains mode by mode; the nodal forces are the transpose of the strain map,
//    then the transpose of the modal transform.
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

// (v0, v1) -> (mean, difference) along the axis of bit `bit` of the corner index
template <typename T>
__device__ __forceinline__ void modal_forward(T (&v)[8]) {
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1) {
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      if (!(l & bit)) {
        T v0 = v[l], v1 = v[l | bit];
        v[l] = T(0.5) * (v0 + v1);
        v[l | bit] = v1 - v0;
      }
    }
  }
}

// transpose of modal_forward (forces in the modal basis -> nodal forces)
template <typename T>
__device__ __forceinline__ void modal_backward(T (&f)[8]) {
#pragma unroll
  for (int bit = 1; bit < 8; bit <<= 1) {
#pragma unroll
    for (int l = 0; l < 8; ++l) {
      if (!(l & bit)) {
        T fm = f[l], fd = f[l | bit];
        f[l] = T(0.5) * fm - fd;
        f[l | bit] = T(0.5) * fm + fd;
      }
    }
  }
}

// f = K_e u.  u[c][l], f[c][l]: component c, corner l = a + 2b + 4c.  a, b, c: cell edge lengths,
// ia, ib, ic their inverses.
template <typename T>
__device__ __forceinline__ void hex8_apply(const T (&u)[3][8], T a, T b, T cc, T ia, T ib, T ic,
                                           const Material<T>& m, T (&f)[3][8]) {
  constexpr T N1 = T(1) / T(12);
  T U[3][8];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int l = 0; l < 8; ++l) U[c][l] = u[c][l];
    modal_forward(U[c]);
  }
  // derivative modes: X[c][be + 2 ga] = d u_c / dx at mode (m, be, ga), etc.
  T X[3][4], Y[3][4], Z[3][4];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
#pragma unroll
    for (int i = 0; i < 2; ++i) {
#pragma unroll
      for (int j = 0; j < 2; ++j) {
        X[c][i + 2 * j] = U[c][1 + 2 * i + 4 * j] * ia;
        Y[c][i + 2 * j] = U[c][i + 2 + 4 * j] * ib;
        Z[c][i + 2 * j] = U[c][i + 2 * j + 4] * ic;
      }
    }
  }
  T F[3][8];
#pragma unroll
  for (int c = 0; c < 3; ++c)
#pragma unroll
    for (int l = 0; l < 8; ++l) F[c][l] = T(0);
  const T bc = b * cc, ac = a * cc, ab = a * b;
  // x-derivative slots: modes (m, be, ga)
#pragma unroll
  for (int be = 0; be < 2; ++be) {
#pragma unroll
    for (int ga = 0; ga < 2; ++ga) {
      T w = bc * (be ? N1 : T(1)) * (ga ? N1 : T(1));
      T s1 = m.c0 * X[0][be + 2 * ga];
      if (be == 0) s1 += m.c1 * Y[1][0 + 2 * ga];
      if (ga == 0) s1 += m.c2 * Z[2][0 + 2 * be];
      T g4 = X[1][be + 2 * ga];
      if (be == 0) g4 += Y[0][0 + 2 * ga];
      T g6 = X[2][be + 2 * ga];
      if (ga == 0) g6 += Z[0][0 + 2 * be];
      const int l = 1 + 2 * be + 4 * ga;
      F[0][l] += w * s1;
      F[1][l] += w * (m.c4 * g4);
      F[2][l] += w * (m.c5 * g6);
    }
  }
  // y-derivative slots: modes (al, m, ga)
#pragma unroll
  for (int al = 0; al < 2; ++al) {
#pragma unroll
    for (int ga = 0; ga < 2; ++ga) {
      T w = ac * (al ? N1 : T(1)) * (ga ? N1 : T(1));
      T s2 = m.c0 * Y[1][al + 2 * ga];
      if (al == 0) s2 += m.c1 * X[0][0 + 2 * ga];
      if (ga == 0) s2 += m.c2 * Z[2][al + 0];
      T g4 = Y[0][al + 2 * ga];
      if (al == 0) g4 += X[1][0 + 2 * ga];
      T g5 = Y[2][al + 2 * ga];
      if (ga == 0) g5 += Z[1][al + 0];
      const int l = al + 2 + 4 * ga;
      F[0][l] += w * (m.c4 * g4);
      F[1][l] += w * s2;
      F[2][l] += w * (m.c5 * g5);
    }
  }
  // z-derivative slots: modes (al, be, m)
#pragma unroll
  for (int al = 0; al < 2; ++al) {
#pragma unroll
    for (int be = 0; be < 2; ++be) {
      T w = ab * (al ? N1 : T(1)) * (be ? N1 : T(1));
      T s3 = m.c3 * Z[2][al + 2 * be];
      if (al == 0) s3 += m.c2 * X[0][be + 0];
      if (be == 0) s3 += m.c2 * Y[1][al + 0];
      T g5 = Z[1][al + 2 * be];
      if (be == 0) g5 += Y[2][al + 0];
      T g6 = Z[0][al + 2 * be];
      if (al == 0) g6 += X[2][be + 0];
      const int l = al + 2 * be + 4;
      F[0][l] += w * (m.c5 * g6);
      F[1][l] += w * (m.c5 * g5);
      F[2][l] += w * s3;
    }
  }
  // one-point volumetric term at the centre (SRI)
  {
    T t = m.lamc * (X[0][0] + Y[1][0] + Z[2][0]);
    F[0][1] += bc * t;
    F[1][2] += ac * t;
    F[2][4] += ab * t;
  }
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    modal_backward(F[c]);
#pragma unroll
    for (int l = 0; l < 8; ++l) f[c][l] = F[c][l];
  }
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
