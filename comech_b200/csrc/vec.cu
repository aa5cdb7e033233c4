// Vector kernels: deterministic two-stage reductions, CG updates, Chebyshev smoother steps.
#include "vec.cuh"

namespace feb {

namespace {

template <typename Ta, typename Tb>
__global__ void __launch_bounds__(kThreads)
k_dot_partial(const Ta* __restrict__ a, const Tb* __restrict__ b, int64_t n, double* __restrict__ partials,
              const int* __restrict__ skip) {
  if (skip && *skip) return;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  for (; i + 3 * stride < n; i += 4 * stride) {     // four independent loads in flight per thread
    s0 += double(a[i]) * double(b[i]);
    s1 += double(a[i + stride]) * double(b[i + stride]);
    s2 += double(a[i + 2 * stride]) * double(b[i + 2 * stride]);
    s3 += double(a[i + 3 * stride]) * double(b[i + 3 * stride]);
  }
  for (; i < n; i += stride) s0 += double(a[i]) * double(b[i]);
  double s = block_sum((s0 + s1) + (s2 + s3));
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// The scalar step of a reduction's caller, given the reduction's value s (thread 0 only).
__device__ void finalize_step(int kind, double s, CgState* st, LevelParams* lp, int deg) {
  switch (kind) {
    case FIN_RZ:
      st->rz = s;
      st->beta = (st->it == 0) ? 0.0 : s / st->rz_old;
      break;
    case FIN_ALPHA:
      st->pq = s;
      if (!(s > 0.0) || !isfinite(s)) {
        st->status = isfinite(s) ? FEB_ERR_BREAKDOWN : FEB_ERR_NAN;
        st->done = 1;
        st->flag = st->maxiter;
      } else {
        st->alpha = st->rz / s;
      }
      break;
    case FIN_CONV:
      st->rr = s;
      st->rz_old = st->rz;
      st->it += 1;
      if (!isfinite(s)) {
        st->status = FEB_ERR_NAN; st->done = 1; st->flag = st->maxiter;
      } else if (s < st->thr2) {
        st->done = 1; st->flag = 0;
      } else if (st->it >= st->maxiter) {
        st->done = 1; st->flag = st->maxiter;
      }
      break;
    case FIN_INIT:
      st->rr = s;
      if (!isfinite(s)) { st->status = FEB_ERR_NAN; st->done = 1; st->flag = st->maxiter; }
      else if (s < st->thr2) { st->done = 1; st->flag = 0; }
      else if (st->maxiter <= 0) { st->done = 1; st->flag = st->maxiter; }
      break;
    case FIN_THR:   // stop threshold from ||f||^2; a zero right-hand side stops before the first iteration
      st->fn2 = s;
      st->thr2 = s > 0.0 ? st->tol2 * s : INFINITY;
      break;
    case FIN_TRUE:
      st->rtrue = s;
      break;
    case FIN_POWER0:
      lp->xnorm = sqrt(s);
      break;
    case FIN_POWER: {
      double ny = sqrt(s);
      lp->lam = ny / lp->xnorm;
      lp->inv = 1.0 / ny;
      lp->xnorm = 1.0;
      double lmax = 1.1 * lp->lam, lmin = lmax / 30.0;
      double theta = 0.5 * (lmax + lmin), delta = 0.5 * (lmax - lmin), sigma = theta / delta;
      double rho = 1.0 / sigma;
      lp->lmax = lmax; lp->lmin = lmin;
      lp->c_init = 1.0 / theta;
      for (int k = 0; k < deg - 1 && k < 8; ++k) {
        double rn = 1.0 / (2.0 * sigma - rho);
        lp->a1[k] = rn * rho;
        lp->a2[k] = 2.0 * rn / delta;
        rho = rn;
      }
      break;
    }
  }
}

// Sums the partials in a fixed order (deterministic) and runs the scalar step of the caller.
__global__ void __launch_bounds__(kThreads)
k_finalize(int kind, const double* __restrict__ partials, int np, CgState* st, LevelParams* lp, int deg,
           const int* __restrict__ skip) {
  if (skip && *skip) return;
  double s = 0.0;
  for (int i = threadIdx.x; i < np; i += kThreads) s += partials[i];
  s = block_sum(s);
  if (threadIdx.x == 0) finalize_step(kind, s, st, lp, deg);
}

// Last-block finalisation of a grid reduction: every block has stored its partial; the block that arrives
// last (counted on `ctr`, after a fence that publishes the partial) sums all partials in the same fixed order
// as k_finalize, runs the scalar step and re-arms the counter.  Block-uniform; no block waits for another.
__device__ __forceinline__ void last_block_finalize(int kind, double* partials, unsigned int* ctr, CgState* st) {
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ctr, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  double s = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += kThreads) s += ((volatile double*)partials)[i];
  s = block_sum(s);
  if (threadIdx.x == 0) {
    finalize_step(kind, s, st, nullptr, 0);
    *ctr = 0u;
  }
}

// dot product with the caller's scalar step in the last block (FIN_RZ, FIN_ALPHA)
template <typename Ta, typename Tb>
__global__ void __launch_bounds__(kThreads)
k_dot_finalize(int kind, const Ta* __restrict__ a, const Tb* __restrict__ b, int64_t n, double* partials,
               unsigned int* ctr, CgState* st, const int* __restrict__ skip) {
  if (skip && *skip) return;
  double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  for (; i + 3 * stride < n; i += 4 * stride) {
    s0 += double(a[i]) * double(b[i]);
    s1 += double(a[i + stride]) * double(b[i + stride]);
    s2 += double(a[i + 2 * stride]) * double(b[i + 2 * stride]);
    s3 += double(a[i + 3 * stride]) * double(b[i + 3 * stride]);
  }
  for (; i < n; i += stride) s0 += double(a[i]) * double(b[i]);
  double s = block_sum((s0 + s1) + (s2 + s3));
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
  last_block_finalize(kind, partials, ctr, st);
}

template <typename T>
__global__ void k_update_p(const T* __restrict__ z, T* __restrict__ p, const CgState* __restrict__ st, int64_t n,
                           const int* __restrict__ skip) {
  if (skip && *skip) return;
  const T beta = T(st->beta);
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    p[i] = z[i] + beta * p[i];
}

// x += alpha p, r -= alpha q, partial ||r||^2; rf (optional) receives r in FP32 for the next FP32 V-cycle;
// with ctr the last block runs the convergence step (FIN_CONV) itself
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_update_xr(const T* __restrict__ p, const T* __restrict__ q, T* __restrict__ x, T* __restrict__ r,
            float* __restrict__ rf, CgState* st, int64_t n, double* partials, unsigned int* ctr,
            const int* __restrict__ skip) {
  if (skip && *skip) return;
  const T alpha = T(st->alpha);
  double s0 = 0.0, s1 = 0.0;
  const int64_t stride = (int64_t)gridDim.x * kThreads;
  int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x;
  for (; i + stride < n; i += 2 * stride) {
    const T p0 = p[i], p1 = p[i + stride], q0 = q[i], q1 = q[i + stride];
    const T x0 = x[i], x1 = x[i + stride], ra = r[i], rb = r[i + stride];
    x[i] = x0 + alpha * p0; x[i + stride] = x1 + alpha * p1;
    const T r0 = ra - alpha * q0, r1 = rb - alpha * q1;
    r[i] = r0; r[i + stride] = r1;
    if (rf) { rf[i] = float(r0); rf[i + stride] = float(r1); }
    s0 += double(r0) * double(r0);
    s1 += double(r1) * double(r1);
  }
  for (; i < n; i += stride) {
    x[i] += alpha * p[i];
    T ri = r[i] - alpha * q[i];
    r[i] = ri;
    if (rf) rf[i] = float(ri);
    s0 += double(ri) * double(ri);
  }
  double s = block_sum(s0 + s1);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
  if (ctr) last_block_finalize(FIN_CONV, partials, ctr, st);
}

template <typename T>
__device__ __forceinline__ void bj(const T* __restrict__ D, int64_t nn, int64_t i, T r0, T r1, T r2, T& z0, T& z1,
                                   T& z2) {
  z0 = D[i] * r0 + D[nn + i] * r1 + D[2 * nn + i] * r2;
  z1 = D[3 * nn + i] * r0 + D[4 * nn + i] * r1 + D[5 * nn + i] * r2;
  z2 = D[6 * nn + i] * r0 + D[7 * nn + i] * r1 + D[8 * nn + i] * r2;
}

template <typename T>
__global__ void k_cheb_first(const T* __restrict__ b, T* __restrict__ r, T* __restrict__ d, T* __restrict__ x,
                             const T* __restrict__ D, const LevelParams* __restrict__ lp, int64_t nn,
                             const int* __restrict__ skip, TermAcc<T> acc) {
  if (skip && *skip) return;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const T c = T(lp->c_init);
  T r0 = b[3 * i], r1 = b[3 * i + 1], r2 = b[3 * i + 2], z0, z1, z2;
  bj(D, nn, i, r0, r1, r2, z0, z1, z2);
  r[3 * i] = r0; r[3 * i + 1] = r1; r[3 * i + 2] = r2;
  z0 *= c; z1 *= c; z2 *= c;
  d[3 * i] = z0; d[3 * i + 1] = z1; d[3 * i + 2] = z2;
  x[3 * i] = z0; x[3 * i + 1] = z1; x[3 * i + 2] = z2;
  term_acc(acc, i, z0, z1, z2);
}

template <typename T>
__global__ void k_cheb_init(const T* __restrict__ b, const T* __restrict__ Ax, T* __restrict__ r, T* __restrict__ d,
                            T* __restrict__ x, const T* __restrict__ D, const LevelParams* __restrict__ lp, int64_t nn,
                            const int* __restrict__ skip) {
  if (skip && *skip) return;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const T c = T(lp->c_init);
  T r0 = b[3 * i] - Ax[3 * i], r1 = b[3 * i + 1] - Ax[3 * i + 1], r2 = b[3 * i + 2] - Ax[3 * i + 2], z0, z1, z2;
  bj(D, nn, i, r0, r1, r2, z0, z1, z2);
  r[3 * i] = r0; r[3 * i + 1] = r1; r[3 * i + 2] = r2;
  z0 *= c; z1 *= c; z2 *= c;
  d[3 * i] = z0; d[3 * i + 1] = z1; d[3 * i + 2] = z2;
  x[3 * i] += z0; x[3 * i + 1] += z1; x[3 * i + 2] += z2;
}

template <typename T>
__global__ void k_cheb_step(const T* __restrict__ Ad, T* __restrict__ r, T* __restrict__ d, T* __restrict__ x,
                            const T* __restrict__ D, const LevelParams* __restrict__ lp, int k, int64_t nn,
                            const int* __restrict__ skip) {
  if (skip && *skip) return;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const T a1 = T(lp->a1[k]), a2 = T(lp->a2[k]);
  T r0 = r[3 * i] - Ad[3 * i], r1 = r[3 * i + 1] - Ad[3 * i + 1], r2 = r[3 * i + 2] - Ad[3 * i + 2], z0, z1, z2;
  bj(D, nn, i, r0, r1, r2, z0, z1, z2);
  r[3 * i] = r0; r[3 * i + 1] = r1; r[3 * i + 2] = r2;
  T d0 = a1 * d[3 * i] + a2 * z0, d1 = a1 * d[3 * i + 1] + a2 * z1, d2 = a1 * d[3 * i + 2] + a2 * z2;
  d[3 * i] = d0; d[3 * i + 1] = d1; d[3 * i + 2] = d2;
  x[3 * i] += d0; x[3 * i + 1] += d1; x[3 * i + 2] += d2;
}

template <typename T>
__global__ void k_cheb_from_r(const T* __restrict__ r, T* __restrict__ d, T* __restrict__ x, const T* __restrict__ D,
                              const LevelParams* __restrict__ lp, int64_t nn, const int* __restrict__ skip,
                              TermAcc<T> acc) {
  if (skip && *skip) return;
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= nn) return;
  const T c = T(lp->c_init);
  T z0, z1, z2;
  bj(D, nn, i, r[3 * i], r[3 * i + 1], r[3 * i + 2], z0, z1, z2);
  z0 *= c; z1 *= c; z2 *= c;
  d[3 * i] = z0; d[3 * i + 1] = z1; d[3 * i + 2] = z2;
  x[3 * i] += z0; x[3 * i + 1] += z1; x[3 * i + 2] += z2;
  term_acc(acc, i, z0, z1, z2);
}

template <typename T>
__global__ void k_residual(const T* __restrict__ b, const T* __restrict__ Ax, T* __restrict__ r, int64_t n,
                           const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    r[i] = b[i] - Ax[i];
}

__device__ __forceinline__ uint64_t splitmix(uint64_t z) {
  z += 0x9E3779B97F4A7C15ull;
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

// standard normal start vector of the power iteration (Box-Muller on a counter-based hash), 0 where masked out
template <typename T>
__global__ void k_random_start(T* __restrict__ x, const uint8_t* __restrict__ mask, int64_t nn, uint64_t seed) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= 3 * nn) return;
  uint64_t h = splitmix(seed ^ splitmix((uint64_t)i));
  double u1 = ((h >> 11) + 1.0) * (1.0 / 9007199254740993.0);
  double u2 = (splitmix(h) >> 11) * (1.0 / 9007199254740992.0);
  double g = sqrt(-2.0 * log(u1)) * cospi(2.0 * u2);
  x[i] = (mask == nullptr || mask[i / 3]) ? T(g) : T(0);
}

// y = f Dinv v and its squared norm; f = scale->inv (the previous power step's 1 / ||y||, so that the product
// that formed v could take the unscaled vector) or 1.  With ctr the last block runs the power step FIN_POWER on
// fin (no separate finalize launch); each block reads scale->inv before it arrives, the last block writes it after.
template <typename T>
__global__ void __launch_bounds__(kThreads)
k_bj_apply_norm(const T* __restrict__ D, const T* __restrict__ v, T* __restrict__ y, int64_t nn,
                double* __restrict__ partials, const LevelParams* scale, LevelParams* fin, unsigned int* ctr,
                int deg) {
  const T f = scale ? T(scale->inv) : T(1);
  double s = 0.0;
  for (int64_t i = blockIdx.x * (int64_t)kThreads + threadIdx.x; i < nn; i += (int64_t)gridDim.x * kThreads) {
    T z0, z1, z2;
    bj(D, nn, i, v[3 * i], v[3 * i + 1], v[3 * i + 2], z0, z1, z2);
    z0 *= f; z1 *= f; z2 *= f;
    y[3 * i] = z0; y[3 * i + 1] = z1; y[3 * i + 2] = z2;
    s += double(z0) * double(z0) + double(z1) * double(z1) + double(z2) * double(z2);
  }
  s = block_sum(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
  if (!ctr) return;
  __shared__ bool last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) last = atomicAdd(ctr, 1u) == gridDim.x - 1;
  __syncthreads();
  if (!last) return;
  __threadfence();
  double t = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += kThreads) t += ((volatile double*)partials)[i];
  t = block_sum(t);
  if (threadIdx.x == 0) {
    finalize_step(FIN_POWER, t, nullptr, fin, deg);
    *ctr = 0u;
  }
}


template <typename Ts, typename Td>
__global__ void k_convert(const Ts* __restrict__ a, Td* __restrict__ b, int64_t n, const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    b[i] = Td(a[i]);
}

template <typename T>
__global__ void k_axpy_dev(const T* __restrict__ x, T* __restrict__ y, int64_t n, const int* __restrict__ skip) {
  if (skip && *skip) return;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    y[i] += x[i];
}

__global__ void k_add_scaled(const float* __restrict__ e, double* __restrict__ x, const double* __restrict__ scale,
                             int64_t n, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const double s = *scale;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    x[i] += s * double(e[i]);
}

__global__ void k_scale_to_float(const double* __restrict__ r, float* __restrict__ rf,
                                 const double* __restrict__ scale_inv, int64_t n, const int* __restrict__ skip) {
  if (skip && *skip) return;
  const double s = *scale_inv;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x)
    rf[i] = float(r[i] * s);
}

__global__ void k_mask_vector(double* __restrict__ v, const uint8_t* __restrict__ used, int64_t nn, double fill) {
  int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
  if (i >= 3 * nn) return;
  if (!used[i / 3]) v[i] = fill;
}

__global__ void k_set_condition(cudaGraphConditionalHandle h, const CgState* __restrict__ st) {
  cudaGraphSetConditional(h, st->done ? 0u : 1u);
}

inline int grid_for(int64_t n) { return int(std::min<int64_t>((n + kThreads - 1) / kThreads, 8 * kSmCount)); }

}  // namespace

void launch_set_condition(cudaGraphConditionalHandle h, const CgState* st, cudaStream_t s) {
  k_set_condition<<<1, 1, 0, s>>>(h, st); note_launch();
}

template <typename Ta, typename Tb>
void launch_dot_partial(const Ta* a, const Tb* b, int64_t n, double* partials, const int* skip, cudaStream_t s) {
  k_dot_partial<Ta, Tb><<<kRedBlocks, kThreads, 0, s>>>(a, b, n, partials, skip); note_launch();
}

void launch_finalize(int kind, const double* partials, CgState* st, LevelParams* lp, int deg, const int* skip,
                     cudaStream_t s) {
  k_finalize<<<1, kThreads, 0, s>>>(kind, partials, kRedBlocks, st, lp, deg, skip); note_launch();
}

template <typename T>
void launch_update_p(const T* z, T* p, const CgState* st, int64_t n, const int* skip, cudaStream_t s) {
  k_update_p<T><<<grid_for(n), kThreads, 0, s>>>(z, p, st, n, skip); note_launch();
}

template <typename T>
void launch_update_xr(const T* p, const T* q, T* x, T* r, const CgState* st, int64_t n, double* partials,
                      const int* skip, cudaStream_t s) {
  k_update_xr<T><<<kRedBlocks, kThreads, 0, s>>>(p, q, x, r, nullptr, const_cast<CgState*>(st), n, partials, nullptr,
                                                 skip); note_launch();
}

template <typename T>
void launch_update_xr_conv(const T* p, const T* q, T* x, T* r, float* rf, CgState* st, int64_t n, double* partials,
                           unsigned int* ctr, const int* skip, cudaStream_t s) {
  k_update_xr<T><<<kRedBlocks, kThreads, 0, s>>>(p, q, x, r, rf, st, n, partials, ctr, skip); note_launch();
}

template <typename Ta, typename Tb>
void launch_dot_finalize(int kind, const Ta* a, const Tb* b, int64_t n, double* partials, unsigned int* ctr,
                         CgState* st, const int* skip, cudaStream_t s) {
  k_dot_finalize<Ta, Tb><<<kRedBlocks, kThreads, 0, s>>>(kind, a, b, n, partials, ctr, st, skip); note_launch();
}

template <typename T>
void launch_cheb_first(const T* b, T* r, T* d, T* x, const T* Dinv, const LevelParams* lp, int64_t nn,
                       const int* skip, cudaStream_t s, const TermAcc<T>& acc) {
  k_cheb_first<T><<<div_up(nn, kThreads), kThreads, 0, s>>>(b, r, d, x, Dinv, lp, nn, skip, acc); note_launch();
}

template <typename T>
void launch_cheb_init(const T* b, const T* Ax, T* r, T* d, T* x, const T* Dinv, const LevelParams* lp, int64_t nn,
                      const int* skip, cudaStream_t s) {
  k_cheb_init<T><<<div_up(nn, kThreads), kThreads, 0, s>>>(b, Ax, r, d, x, Dinv, lp, nn, skip); note_launch();
}

template <typename T>
void launch_cheb_step(const T* Ad, T* r, T* d, T* x, const T* Dinv, const LevelParams* lp, int k, int64_t nn,
                      const int* skip, cudaStream_t s) {
  k_cheb_step<T><<<div_up(nn, kThreads), kThreads, 0, s>>>(Ad, r, d, x, Dinv, lp, k, nn, skip); note_launch();
}

template <typename T>
void launch_cheb_from_r(const T* r, T* d, T* x, const T* Dinv, const LevelParams* lp, int64_t nn, const int* skip,
                        cudaStream_t s, const TermAcc<T>& acc) {
  k_cheb_from_r<T><<<div_up(nn, kThreads), kThreads, 0, s>>>(r, d, x, Dinv, lp, nn, skip, acc); note_launch();
}

template <typename T>
void launch_residual(const T* b, const T* Ax, T* r, int64_t n, const int* skip, cudaStream_t s) {
  k_residual<T><<<grid_for(n), kThreads, 0, s>>>(b, Ax, r, n, skip); note_launch();
}

template <typename T>
void launch_random_start(T* x, const uint8_t* mask, int64_t nn, uint64_t seed, cudaStream_t s) {
  k_random_start<T><<<div_up(3 * nn, kThreads), kThreads, 0, s>>>(x, mask, nn, seed); note_launch();
}

template <typename T>
void launch_bj_apply_norm(const T* Dinv, const T* v, T* y, int64_t nn, double* partials, cudaStream_t s,
                          const LevelParams* scale, LevelParams* fin, unsigned int* ctr, int deg) {
  k_bj_apply_norm<T><<<kRedBlocks, kThreads, 0, s>>>(Dinv, v, y, nn, partials, scale, fin, ctr, deg); note_launch();
}

template void launch_random_start<float>(float*, const uint8_t*, int64_t, uint64_t, cudaStream_t);
template void launch_random_start<double>(double*, const uint8_t*, int64_t, uint64_t, cudaStream_t);
template void launch_bj_apply_norm<float>(const float*, const float*, float*, int64_t, double*, cudaStream_t,
                                          const LevelParams*, LevelParams*, unsigned int*, int);
template void launch_bj_apply_norm<double>(const double*, const double*, double*, int64_t, double*, cudaStream_t,
                                           const LevelParams*, LevelParams*, unsigned int*, int);

template <typename Ts, typename Td>
void launch_convert(const Ts* src, Td* dst, int64_t n, const int* skip, cudaStream_t s) {
  k_convert<Ts, Td><<<grid_for(n), kThreads, 0, s>>>(src, dst, n, skip); note_launch();
}

template <typename T>
void launch_axpy_dev(const T* x, T* y, int64_t n, const int* skip, cudaStream_t s) {
  k_axpy_dev<T><<<grid_for(n), kThreads, 0, s>>>(x, y, n, skip); note_launch();
}

void launch_add_scaled(const float* e, double* x, const double* scale, int64_t n, const int* skip, cudaStream_t s) {
  k_add_scaled<<<grid_for(n), kThreads, 0, s>>>(e, x, scale, n, skip); note_launch();
}

void launch_scale_to_float(const double* r, float* rf, const double* scale_inv, int64_t n, const int* skip,
                           cudaStream_t s) {
  k_scale_to_float<<<grid_for(n), kThreads, 0, s>>>(r, rf, scale_inv, n, skip); note_launch();
}

void launch_mask_vector(double* v, const uint8_t* used, int64_t nn, double fill, cudaStream_t s) {
  k_mask_vector<<<div_up(3 * nn, kThreads), kThreads, 0, s>>>(v, used, nn, fill); note_launch();
}

#define INST_T(T)                                                                                              \
  template void launch_update_p<T>(const T*, T*, const CgState*, int64_t, const int*, cudaStream_t);          \
  template void launch_update_xr<T>(const T*, const T*, T*, T*, const CgState*, int64_t, double*, const int*,   \
                                    cudaStream_t);                                                             \
  template void launch_cheb_first<T>(const T*, T*, T*, T*, const T*, const LevelParams*, int64_t, const int*,   \
                                     cudaStream_t, const TermAcc<T>&);                                         \
  template void launch_cheb_init<T>(const T*, const T*, T*, T*, T*, const T*, const LevelParams*, int64_t,      \
                                    const int*, cudaStream_t);                                                 \
  template void launch_cheb_step<T>(const T*, T*, T*, T*, const T*, const LevelParams*, int, int64_t,           \
                                    const int*, cudaStream_t);                                                 \
  template void launch_residual<T>(const T*, const T*, T*, int64_t, const int*, cudaStream_t);                 \
  template void launch_cheb_from_r<T>(const T*, T*, T*, const T*, const LevelParams*, int64_t, const int*,      \
                                      cudaStream_t, const TermAcc<T>&);                                        \
  template void launch_axpy_dev<T>(const T*, T*, int64_t, const int*, cudaStream_t);
INST_T(float)
INST_T(double)
#undef INST_T
template void launch_dot_partial<double, double>(const double*, const double*, int64_t, double*, const int*,
                                                 cudaStream_t);
template void launch_dot_partial<float, float>(const float*, const float*, int64_t, double*, const int*,
                                               cudaStream_t);
template void launch_convert<double, float>(const double*, float*, int64_t, const int*, cudaStream_t);
template void launch_update_xr_conv<double>(const double*, const double*, double*, double*, float*, CgState*, int64_t,
                                            double*, unsigned int*, const int*, cudaStream_t);
template void launch_update_xr_conv<float>(const float*, const float*, float*, float*, float*, CgState*, int64_t,
                                           double*, unsigned int*, const int*, cudaStream_t);
template void launch_dot_finalize<double, double>(int, const double*, const double*, int64_t, double*, unsigned int*,
                                                  CgState*, const int*, cudaStream_t);
template void launch_dot_finalize<float, float>(int, const float*, const float*, int64_t, double*, unsigned int*,
                                                CgState*, const int*, cudaStream_t);
template void launch_convert<float, double>(const float*, double*, int64_t, const int*, cudaStream_t);

}  // namespace feb
