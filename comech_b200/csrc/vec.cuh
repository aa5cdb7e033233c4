// Vector kernels of the CG iteration and the Chebyshev smoother; all scalars live in device memory so
// a whole iteration can be captured in a CUDA graph with no host round trip.
#pragma once
#include "common.cuh"

namespace feb {

constexpr int kRedBlocks = 4 * kSmCount;   // partial sums per reduction

// CG state (one per solve); SciPy cg semantics (stop when ||r|| < tol ||b|| before an iteration).
struct CgState {
  double rz, rz_old, pq, alpha, beta, rr, thr2;
  int it, done, flag, status, maxiter, pad;
  double tol2;   // batched solves: thr2 = tol2 ||f||^2 is formed on the device (FIN_THR)
  double fn2;    // ||f||^2 (FIN_THR)
  double rtrue;  // ||f - K x||^2 of the result (FIN_TRUE)
};

// Rank-1 term dots formed by the kernel that writes a coarse-level vector, instead of a dot pass before every
// stencil product that reads it: for each node the kernel writes that some term touches (tn_ptr), the term's
// lam_t v_t(node) . delta(node) is added atomically to dot_a[t] and dot_b[t] (either may be null; both zeroed
// beforehand), delta being the written direction or the change of the iterate.  tn_ptr null: nothing to do.
template <typename T>
struct TermAcc {
  const int* tn_ptr = nullptr;
  const int* tn_term = nullptr;
  const T* tn_coef = nullptr;    // v_t at the node, 3 components per (node, term) pair
  const T* t_lam = nullptr;
  T* dot_a = nullptr;
  T* dot_b = nullptr;
};

template <typename T>
__device__ __forceinline__ void term_acc(const TermAcc<T>& A, int64_t n, T v0, T v1, T v2) {
  if (!A.tn_ptr) return;
  const int pe = A.tn_ptr[n + 1];
  for (int p = A.tn_ptr[n]; p < pe; ++p) {
    const int t = A.tn_term[p];
    const T c = A.t_lam[t] * (A.tn_coef[3 * p] * v0 + A.tn_coef[3 * p + 1] * v1 + A.tn_coef[3 * p + 2] * v2);
    if (A.dot_a) atomicAdd(A.dot_a + t, c);
    if (A.dot_b) atomicAdd(A.dot_b + t, c);
  }
}
// one component `comp` of the node's delta (a kernel whose threads own single components)
template <typename T>
__device__ __forceinline__ void term_acc1(const TermAcc<T>& A, int64_t n, int comp, T v) {
  if (!A.tn_ptr) return;
  const int pe = A.tn_ptr[n + 1];
  for (int p = A.tn_ptr[n]; p < pe; ++p) {
    const int t = A.tn_term[p];
    const T c = A.t_lam[t] * A.tn_coef[3 * p + comp] * v;
    if (A.dot_a) atomicAdd(A.dot_a + t, c);
    if (A.dot_b) atomicAdd(A.dot_b + t, c);
  }
}

// Per-level smoother parameters written by the power iteration.
struct LevelParams {
  double lam, lmax, lmin;
  double xnorm;              // power iteration: ||x|| of the current iterate
  double inv;                // power iteration: 1 / ||y||
  double c_init;             // Chebyshev: 1 / theta
  double a1[8], a2[8];       // Chebyshev step k: d = a1[k] d + a2[k] M r
};

// sets the while-loop condition of a conditional graph node: continue while the CG is not done
void launch_set_condition(cudaGraphConditionalHandle h, const CgState* st, cudaStream_t s);

template <typename Ta, typename Tb>
void launch_dot_partial(const Ta* a, const Tb* b, int64_t n, double* partials, const int* skip, cudaStream_t s);

// kinds of the single-block finalisation kernel
enum FinKind : int { FIN_RZ = 0, FIN_ALPHA = 1, FIN_CONV = 2, FIN_INIT = 3, FIN_POWER0 = 4, FIN_POWER = 5,
                     FIN_THR = 6, FIN_TRUE = 7 };
void launch_finalize(int kind, const double* partials, CgState* st, LevelParams* lp, int deg, const int* skip,
                     cudaStream_t s);

template <typename T>
void launch_update_p(const T* z, T* p, const CgState* st, int64_t n, const int* skip, cudaStream_t s);
template <typename T>
void launch_update_xr(const T* p, const T* q, T* x, T* r, const CgState* st, int64_t n, double* partials,
                      const int* skip, cudaStream_t s);
// the CG's x/r update with the convergence step (FIN_CONV) in its last block; rf (optional) receives r in
// FP32.  ctr: a zeroed counter, re-armed by the kernel, used by one reduction at a time on the stream.
template <typename T>
void launch_update_xr_conv(const T* p, const T* q, T* x, T* r, float* rf, CgState* st, int64_t n, double* partials,
                           unsigned int* ctr, const int* skip, cudaStream_t s);
// a.b with the step `kind` (FIN_RZ, FIN_ALPHA) in the last block
template <typename Ta, typename Tb>
void launch_dot_finalize(int kind, const Ta* a, const Tb* b, int64_t n, double* partials, unsigned int* ctr,
                         CgState* st, const int* skip, cudaStream_t s);

// Chebyshev smoother pieces (Dinv SoA [9][nn], vectors AoS [3 nn])
template <typename T>
void launch_cheb_first(const T* b, T* r, T* d, T* x, const T* Dinv, const LevelParams* lp, int64_t nn,
                       const int* skip, cudaStream_t s, const TermAcc<T>& acc = TermAcc<T>());
template <typename T>
void launch_cheb_init(const T* b, const T* Ax, T* r, T* d, T* x, const T* Dinv, const LevelParams* lp, int64_t nn,
                      const int* skip, cudaStream_t s);
template <typename T>
void launch_cheb_step(const T* Ad, T* r, T* d, T* x, const T* Dinv, const LevelParams* lp, int k, int64_t nn,
                      const int* skip, cudaStream_t s);
// d = (1/theta) Dinv r, x += d  (Chebyshev start from a given residual)
template <typename T>
void launch_cheb_from_r(const T* r, T* d, T* x, const T* Dinv, const LevelParams* lp, int64_t nn, const int* skip,
                        cudaStream_t s, const TermAcc<T>& acc = TermAcc<T>());
template <typename T>
void launch_residual(const T* b, const T* Ax, T* r, int64_t n, const int* skip, cudaStream_t s);

// power iteration
template <typename T>
void launch_random_start(T* x, const uint8_t* mask, int64_t nn, uint64_t seed, cudaStream_t s);
// y = f Dinv v (f = scale->inv, or 1 without scale) and partial squared norms; with ctr (a zeroed counter) the last
// block also runs the power step FIN_POWER on fin
template <typename T>
void launch_bj_apply_norm(const T* Dinv, const T* v, T* y, int64_t nn, double* partials, cudaStream_t s,
                          const LevelParams* scale = nullptr, LevelParams* fin = nullptr, unsigned int* ctr = nullptr,
                          int deg = 0);

// conversions and small helpers
template <typename Ts, typename Td>
void launch_convert(const Ts* src, Td* dst, int64_t n, const int* skip, cudaStream_t s);
template <typename T>
void launch_axpy_dev(const T* x, T* y, int64_t n, const int* skip, cudaStream_t s);   // y += x
void launch_add_scaled(const float* e, double* x, const double* scale, int64_t n, const int* skip, cudaStream_t s);
void launch_scale_to_float(const double* r, float* rf, const double* scale_inv, int64_t n, const int* skip,
                           cudaStream_t s);
void launch_mask_vector(double* v, const uint8_t* used, int64_t nn, double fill, cudaStream_t s);

}  // namespace feb
