// Packed pairs: two values of the same quantity at two neighbouring node rows, processed by one thread.
//
// FP32 pairs use sm_100's packed arithmetic (add/sub/mul/fma.rn.f32x2 on a 64-bit register pair): one
// instruction issues both lanes, so a kernel whose every operation is duplicated over two rows needs half
// the issue slots.  FP64 pairs are two scalar operations (there is no packed FP64 form).
#pragma once
#include "common.cuh"

namespace feb {

template <typename T> struct P2;

template <>
struct P2<float> {
  float2 v;
  __device__ __forceinline__ P2() {}
  __device__ __forceinline__ P2(float a, float b) : v(make_float2(a, b)) {}
  __device__ __forceinline__ explicit P2(float s) : v(make_float2(s, s)) {}
  __device__ __forceinline__ float lo() const { return v.x; }
  __device__ __forceinline__ float hi() const { return v.y; }
  __device__ __forceinline__ uint64_t bits() const { return *reinterpret_cast<const uint64_t*>(&v); }
  static __device__ __forceinline__ P2 from_bits(uint64_t b) {
    P2 r;
    r.v = *reinterpret_cast<const float2*>(&b);
    return r;
  }
};

template <>
struct P2<double> {
  double x, y;
  __device__ __forceinline__ P2() {}
  __device__ __forceinline__ P2(double a, double b) : x(a), y(b) {}
  __device__ __forceinline__ explicit P2(double s) : x(s), y(s) {}
  __device__ __forceinline__ double lo() const { return x; }
  __device__ __forceinline__ double hi() const { return y; }
};

__device__ __forceinline__ P2<float> operator+(P2<float> a, P2<float> b) {
  uint64_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a.bits()), "l"(b.bits()));
  return P2<float>::from_bits(d);
}
__device__ __forceinline__ P2<float> operator-(P2<float> a, P2<float> b) {
  uint64_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a.bits()), "l"(b.bits()));
  return P2<float>::from_bits(d);
}
__device__ __forceinline__ P2<float> operator*(P2<float> a, P2<float> b) {
  uint64_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a.bits()), "l"(b.bits()));
  return P2<float>::from_bits(d);
}
// a * b + c, one rounding per lane
__device__ __forceinline__ P2<float> fma2(P2<float> a, P2<float> b, P2<float> c) {
  uint64_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a.bits()), "l"(b.bits()), "l"(c.bits()));
  return P2<float>::from_bits(d);
}

__device__ __forceinline__ P2<double> operator+(P2<double> a, P2<double> b) { return P2<double>(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ P2<double> operator-(P2<double> a, P2<double> b) { return P2<double>(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ P2<double> operator*(P2<double> a, P2<double> b) { return P2<double>(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ P2<double> fma2(P2<double> a, P2<double> b, P2<double> c) {
  return P2<double>(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}

template <typename T>
__device__ __forceinline__ P2<T>& operator+=(P2<T>& a, P2<T> b) { a = a + b; return a; }
template <typename T>
__device__ __forceinline__ P2<T>& operator*=(P2<T>& a, P2<T> b) { a = a * b; return a; }

// (hi of a, b): the pair one row up, built from this thread's upper row and the neighbour's lower row
template <typename T>
__device__ __forceinline__ P2<T> shift_up(P2<T> a, T b) { return P2<T>(a.hi(), b); }

template <typename T>
__device__ __forceinline__ P2<T> shfl_down2(P2<T> v, int d) {
  return P2<T>(__shfl_down_sync(0xffffffffu, v.lo(), d), __shfl_down_sync(0xffffffffu, v.hi(), d));
}
template <typename T>
__device__ __forceinline__ P2<T> shfl_up2(P2<T> v, int d) {
  return P2<T>(__shfl_up_sync(0xffffffffu, v.lo(), d), __shfl_up_sync(0xffffffffu, v.hi(), d));
}

}  // namespace feb
