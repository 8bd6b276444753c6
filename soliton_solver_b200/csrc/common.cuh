// common.cuh -- shared types and device helpers of the soliton_b200 kernels.
//
// Lattice layout (identical to the reference, soliton_solver/core/utils.py:17-42):
// component planes, y fastest:  idx(a, x, y) = y + x*ylen + a*xlen*ylen.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>
#include <math.h>

namespace ssb {

// ---------------------------------------------------------------------------
// parameters (decoded on the host from the reference's packed p_i / p_f)
// ---------------------------------------------------------------------------
struct Grid {
  int X, Y, halo;       // xlen, ylen, halo           (p_i[0], p_i[1], p_i[2])
  long long N;          // xlen*ylen                  (p_i[5])
  double lsx, lsy;      // lattice spacings           (p_f[2], p_f[3])
  double dA, dt;        // grid_volume, time_step     (p_f[4], p_f[5])
  int killkinen;        // arrest on energy increase  (p_i[7])
  int unit_mag;         // unit_magnetization         (p_i[9])
  double ihx, ihy;      // 1/lsx, 1/lsy
  double ihx2, ihy2;    // 1/lsx^2, 1/lsy^2
  double ih2dA;         // 1/(2 dA)
  // host-precomputed stencil / time-step constants in both precisions (GK_* slots)
  double kd[16];
  float kf[16];
};

// slots of Grid::kd / Grid::kf
enum {
  GK_C23HX = 0, GK_MC12HX, GK_C43HX2, GK_MC12HX2, GK_C23HY, GK_MC12HY, GK_C43HY2, GK_MC12HY2, GK_C43HD,
  GK_MC12HD, GK_DT, GK_MDT, GK_HDT, GK_DT6, GK_SIXTH, GK_COUNT
};

// Theory constants.  Meaning of the slots per theory is documented in theories.cuh;
// cf holds the same values rounded to FP32 (filled on the host) so that FP32 kernels
// use them without conversions.
struct Phys {
  double c[24];
  float cf[24];
  int k[12];
};

template <typename S>
__device__ __forceinline__ S grid_k(const Grid& G, int i) {
  if constexpr (sizeof(S) == 4) return G.kf[i]; else return G.kd[i];
}
template <typename S>
__device__ __forceinline__ S phys_k(const Phys& P, int i) {
  if constexpr (sizeof(S) == 4) return P.cf[i]; else return P.c[i];
}

// Device-side state of one lattice's flow (lives in the caller's workspace).
struct StepState {
  double E_last;                 // energy the next arrest test compares against
  unsigned long long err_enc;    // running signed max of the stage-4 gradient (ordered encoding)
  unsigned int ticket;           // last-block-done counter, reset by the last block
  int arrest;                    // 1: treat the velocity as zero in this step's stages 2-4
  int status;                    // 0 ok, SS_ERR_NONFINITE on a non-finite reduction
  int pad;
  double scalar;                 // result slot of single reductions (energy / charge / coupling)
};

// ---------------------------------------------------------------------------
// ordered encoding of doubles for atomicMax (0 encodes below every value)
// ---------------------------------------------------------------------------
__host__ __device__ inline unsigned long long enc_max(double v) {
  long long b;
#ifdef __CUDA_ARCH__
  b = __double_as_longlong(v);
#else
  memcpy(&b, &v, 8);
#endif
  return b >= 0 ? ((unsigned long long)b | 0x8000000000000000ULL) : ~(unsigned long long)b;
}
__host__ __device__ inline double dec_max(unsigned long long u) {
  long long b = (u & 0x8000000000000000ULL) ? (long long)(u & 0x7fffffffffffffffULL) : (long long)~u;
#ifdef __CUDA_ARCH__
  return __longlong_as_double(b);
#else
  double v;
  memcpy(&v, &b, 8);
  return v;
#endif
}

// ---------------------------------------------------------------------------
// jets of derivatives at one site
// ---------------------------------------------------------------------------
template <typename R, int NF>
struct Jet {
  R f[NF];
  R dx[NF], dy[NF];
  R dxx[NF], dyy[NF], dxy[NF];
};

template <typename R, int NF>
struct Jet1 {
  R f[NF];
  R dx[NF], dy[NF];
};

// Derivative masks of the reference (soliton_solver/core/derivatives.py:50-57, 97-115):
// first and pure second derivatives are zero unless halo <= coordinate <= len-halo-1;
// the mixed derivative is zero unless halo < x < xlen-halo and halo < y < ylen-halo.
struct Masks {
  bool x, y, xy;
};
__device__ inline Masks site_masks(const Grid& G, int gx, int gy) {
  Masks m;
  m.x = gx >= G.halo && gx <= G.X - G.halo - 1;
  m.y = gy >= G.halo && gy <= G.Y - G.halo - 1;
  m.xy = gx > G.halo && gx < G.X - G.halo && gy > G.halo && gy < G.Y - G.halo;
  return m;
}

// Finite-difference weights of the reference's 4th-order central stencils.
struct FD {
  static constexpr double c12 = 1.0 / 12.0;
  static constexpr double c23 = 2.0 / 3.0;
  static constexpr double c43 = 4.0 / 3.0;
  static constexpr double c52 = 5.0 / 2.0;
};

// First and second derivatives from the 5-point stencil values, in difference
// form: for a smooth field f(+k) - f(-k) and f(+k) - f(0) are exact (Sterbenz), so
// the rounding error scales with the derivative rather than with |f|, and a
// constant field has exactly zero derivatives.  (The reference's association,
// derivatives.py:51-110, leaves O(eps |f| / h) residues; the two agree to that level.)
template <typename R>
__device__ inline R d1_stencil(R m2, R m1, R p1, R p2, R inv_h) {
  return ((R)FD::c23 * (p1 - m1) - (R)FD::c12 * (p2 - m2)) * inv_h;
}
template <typename R>
__device__ inline R d2_stencil(R m2, R m1, R c, R p1, R p2, R inv_h2) {
  return ((R)FD::c43 * ((p1 - c) + (m1 - c)) - (R)FD::c12 * ((p2 - c) + (m2 - c))) * inv_h2;
}

// Inverse spacings in the working precision.
template <typename R>
struct Inv {
  R hx, hy, hx2, hy2, h2dA;
  __device__ explicit Inv(const Grid& G) {
    hx = (R)G.ihx;
    hy = (R)G.ihy;
    hx2 = (R)G.ihx2;
    hy2 = (R)G.ihy2;
    h2dA = (R)G.ih2dA;
  }
};

// Fill a full jet (value, first, second and mixed derivatives) from an accessor
// S(dx, dy) returning the value of one component at offset (dx, dy).
template <typename R, class S>
__device__ inline void fill_jet_comp(const S& s, const Masks& m, const Inv<R>& iv, R& f, R& dx, R& dy,
                                     R& dxx, R& dyy, R& dxy, bool need_xy) {
  const R c = s(0, 0);
  f = c;
  const R xm2 = s(-2, 0), xm1 = s(-1, 0), xp1 = s(1, 0), xp2 = s(2, 0);
  const R ym2 = s(0, -2), ym1 = s(0, -1), yp1 = s(0, 1), yp2 = s(0, 2);
  const R ddx = d1_stencil<R>(xm2, xm1, xp1, xp2, iv.hx);
  const R ddy = d1_stencil<R>(ym2, ym1, yp1, yp2, iv.hy);
  const R dxx_raw = d2_stencil<R>(xm2, xm1, c, xp1, xp2, iv.hx2);
  const R dyy_raw = d2_stencil<R>(ym2, ym1, c, yp1, yp2, iv.hy2);
  dx = m.x ? ddx : (R)0;
  dy = m.y ? ddy : (R)0;
  dxx = m.x ? dxx_raw : (R)0;
  dyy = m.y ? dyy_raw : (R)0;
  R mixed = (R)0;
  if (need_xy) {
    const R diag = d2_stencil<R>(s(-2, -2), s(-1, -1), c, s(1, 1), s(2, 2), iv.h2dA);
    mixed = diag - (R)0.5 * dxx_raw - (R)0.5 * dyy_raw;
  }
  dxy = m.xy ? mixed : (R)0;
}

template <typename R, class S>
__device__ inline void fill_jet1_comp(const S& s, const Masks& m, const Inv<R>& iv, R& f, R& dx, R& dy) {
  f = s(0, 0);
  const R ddx = d1_stencil<R>(s(-2, 0), s(-1, 0), s(1, 0), s(2, 0), iv.hx);
  const R ddy = d1_stencil<R>(s(0, -2), s(0, -1), s(0, 1), s(0, 2), iv.hy);
  dx = m.x ? ddx : (R)0;
  dy = m.y ? ddy : (R)0;
}

// ---------------------------------------------------------------------------
// deterministic block reductions
// ---------------------------------------------------------------------------
template <int NT>
__device__ inline double block_sum_fixed(double v, double* sh) {
  // fixed xor-butterfly inside warps, then warp results summed in warp order
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) sh[w] = v;
  __syncthreads();
  double t = 0.0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NT / 32; ++i) t += sh[i];
  }
  __syncthreads();
  return t;  // valid in thread 0
}

template <int NT>
__device__ inline double block_max(double v, double* sh) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  const int w = threadIdx.x >> 5;
  if ((threadIdx.x & 31) == 0) sh[w] = v;
  __syncthreads();
  double t = -INFINITY;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < NT / 32; ++i) t = fmax(t, sh[i]);
  }
  __syncthreads();
  return t;
}

// Compensated (Kahan-Babuska/Neumaier) accumulation.
struct KSum {
  double s = 0.0, c = 0.0;
  __device__ inline void add(double v) {
    const double t = s + v;
    if (fabs(s) >= fabs(v))
      c += (s - t) + v;
    else
      c += (v - t) + s;
    s = t;
  }
  __device__ inline double value() const { return s + c; }
};

// Sum nb block partials in a fixed order with compensation.  Called by every thread
// of the last block; result valid in thread 0.
template <int NT>
__device__ inline double fixed_order_sum(const double* partial, int nb, double* sh_s, double* sh_c) {
  KSum k;
  for (int i = threadIdx.x; i < nb; i += NT) k.add(__ldcg(partial + i));
  sh_s[threadIdx.x] = k.s;
  sh_c[threadIdx.x] = k.c;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x == 0) {
    KSum t;
    for (int i = 0; i < NT; ++i) t.add(sh_s[i]);
    double c = 0.0;
    for (int i = 0; i < NT; ++i) c += sh_c[i];
    r = t.value() + c;
  }
  __syncthreads();
  return r;
}

}  // namespace ssb
