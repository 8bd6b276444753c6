// pair.cuh -- two y-adjacent lattice sites processed together.
//
// For FP32 the pair maps onto Blackwell's packed FP32x2 datapath (__fadd2_rn,
// __fmul2_rn, __ffma2_rn on sm_100): one instruction advances both sites.  For
// FP64 the pair is two scalars.  The physics code is written once against this
// interface (+, -, *, unary -, fma(), broadcast construction from a constant).
#pragma once

#include <cuda_runtime.h>

namespace ssb {

struct PF {  // packed pair of floats
  float2 v;
  __device__ PF() {}
  __device__ explicit PF(double c) : v(make_float2((float)c, (float)c)) {}
  __device__ explicit PF(float c) : v(make_float2(c, c)) {}
  __device__ explicit PF(int c) : v(make_float2((float)c, (float)c)) {}
  __device__ PF(float2 a) : v(a) {}
  __device__ PF(float a, float b) : v(make_float2(a, b)) {}
  __device__ float lane(int i) const { return i ? v.y : v.x; }
};
__device__ __forceinline__ PF operator+(PF a, PF b) { return PF(__fadd2_rn(a.v, b.v)); }
__device__ __forceinline__ PF operator-(PF a) { return PF(make_float2(-a.v.x, -a.v.y)); }
__device__ __forceinline__ PF operator-(PF a, PF b) { return PF(__fadd2_rn(a.v, make_float2(-b.v.x, -b.v.y))); }
__device__ __forceinline__ PF operator*(PF a, PF b) { return PF(__fmul2_rn(a.v, b.v)); }
__device__ __forceinline__ PF& operator+=(PF& a, PF b) { return a = a + b; }
__device__ __forceinline__ PF& operator-=(PF& a, PF b) { return a = a - b; }
__device__ __forceinline__ PF& operator*=(PF& a, PF b) { return a = a * b; }
__device__ __forceinline__ PF vfma(PF a, PF b, PF c) { return PF(__ffma2_rn(a.v, b.v, c.v)); }

struct PD {  // pair of doubles
  double x, y;
  __device__ PD() {}
  __device__ explicit PD(double c) : x(c), y(c) {}
  __device__ PD(double a, double b) : x(a), y(b) {}
  __device__ double lane(int i) const { return i ? y : x; }
};
__device__ __forceinline__ PD operator+(PD a, PD b) { return PD(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ PD operator-(PD a) { return PD(-a.x, -a.y); }
__device__ __forceinline__ PD operator-(PD a, PD b) { return PD(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ PD operator*(PD a, PD b) { return PD(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ PD& operator+=(PD& a, PD b) { return a = a + b; }
__device__ __forceinline__ PD& operator-=(PD& a, PD b) { return a = a - b; }
__device__ __forceinline__ PD& operator*=(PD& a, PD b) { return a = a * b; }
__device__ __forceinline__ PD vfma(PD a, PD b, PD c) { return PD(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y)); }

// scalar overloads so that theory code can use vfma for any R
__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ double vfma(double a, double b, double c) { return fma(a, b, c); }

template <typename R>
struct PairOf;
template <>
struct PairOf<float> {
  using type = PF;
  using vec2 = float2;
};
template <>
struct PairOf<double> {
  using type = PD;
  using vec2 = double2;
};

// number of lanes and lane access, for code that must go scalar (transcendentals,
// per-site branches)
template <typename V>
struct Lanes {
  static constexpr int N = 1;
  __device__ static V get(V v, int) { return v; }
  __device__ static void set(V& v, int, V x) { v = x; }
};
template <>
struct Lanes<PF> {
  static constexpr int N = 2;
  __device__ static float get(PF v, int i) { return i ? v.v.y : v.v.x; }
  __device__ static void set(PF& v, int i, float x) {
    if (i) v.v.y = x; else v.v.x = x;
  }
};
template <>
struct Lanes<PD> {
  static constexpr int N = 2;
  __device__ static double get(PD v, int i) { return i ? v.y : v.x; }
  __device__ static void set(PD& v, int i, double x) {
    if (i) v.y = x; else v.x = x;
  }
};
template <typename V>
struct ScalarOf {
  using type = V;
};
template <>
struct ScalarOf<PF> {
  using type = float;
};
template <>
struct ScalarOf<PD> {
  using type = double;
};

// 8- / 16-byte shared memory pair loads and global pair stores
__device__ __forceinline__ PF ld_pair(const float* p) { return PF(*reinterpret_cast<const float2*>(p)); }
__device__ __forceinline__ PD ld_pair(const double* p) {
  const double2 t = *reinterpret_cast<const double2*>(p);
  return PD(t.x, t.y);
}
__device__ __forceinline__ void st_pair(float* p, PF v) { *reinterpret_cast<float2*>(p) = v.v; }
__device__ __forceinline__ void st_pair(double* p, PD v) { *reinterpret_cast<double2*>(p) = make_double2(v.x, v.y); }
// two consecutive pairs as one 16-byte shared-memory access
__device__ __forceinline__ void ld_quad(const float* p, PF& a, PF& b) {
  const float4 t = *reinterpret_cast<const float4*>(p);
  a = PF(t.x, t.y);
  b = PF(t.z, t.w);
}
__device__ __forceinline__ void st_quad(float* p, PF a, PF b) {
  *reinterpret_cast<float4*>(p) = make_float4(a.v.x, a.v.y, b.v.x, b.v.y);
}
__device__ __forceinline__ void ld_quad(const double* p, PD& a, PD& b) {
  a = ld_pair(p);
  b = ld_pair(p + 2);
}
__device__ __forceinline__ void st_quad(double* p, PD a, PD b) {
  st_pair(p, a);
  st_pair(p + 2, b);
}
// pair made of the second lane of a and the first lane of b (one-site shift along y)
__device__ __forceinline__ PF shift1(PF a, PF b) { return PF(a.v.y, b.v.x); }
__device__ __forceinline__ PD shift1(PD a, PD b) { return PD(a.y, b.x); }

}  // namespace ssb
