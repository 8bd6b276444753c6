// adjoint.cuh -- the exact derivative of the discrete energy sum.
//
// The reference's energy is E_h = dA sum_s e(phi(s), Dx phi(s), Dy phi(s)) with the
// 4th-order first-derivative stencils Dx, Dy masked to zero within `halo` of the edge
// (core/derivatives.py:13-57).  Its flow follows the 4th-order functional derivative
// (the gradient stencil), which equals dE_h/dphi / dA only up to O(h^4) in the
// interior.  The exact derivative is
//   dE_h/dphi_a(t) / dA = de/df_a(t) - D1x[Qx_a](t) - D1y[Qy_a](t),
//   Qx_a(s) = mask_x(s) de/d(dx_a)(s),  Qy_a(s) = mask_y(s) de/d(dy_a)(s),
// where D1 is the same 5-point first-derivative stencil without masks and Q is zero
// outside the lattice (the transpose of a masked antisymmetric stencil).  The partial
// derivatives of the energy point come from forward-mode dual numbers carried through
// the theory's own energy() (exact to FP64 rounding, every theory's e is polynomial in
// its jet).  Two passes: exact_partials_kernel writes de/df into the output and Qx, Qy
// into scratch; exact_transpose_kernel adds the transposed stencil.
#pragma once

#include "common.cuh"

namespace ssb {

// Forward-mode dual number with K tangent directions.
template <int K>
struct Dual {
  double v;
  double d[K];
  __device__ Dual() {}
  __device__ Dual(double x) : v(x) {
#pragma unroll
    for (int k = 0; k < K; ++k) d[k] = 0.0;
  }
};
template <int K>
__device__ inline Dual<K> operator+(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
  return r;
}
template <int K>
__device__ inline Dual<K> operator-(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
  return r;
}
template <int K>
__device__ inline Dual<K> operator-(const Dual<K>& a) {
  Dual<K> r;
  r.v = -a.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
  return r;
}
template <int K>
__device__ inline Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) {
  Dual<K> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
  return r;
}
template <int K>
__device__ inline Dual<K> operator*(double s, const Dual<K>& a) {
  Dual<K> r;
  r.v = s * a.v;
#pragma unroll
  for (int k = 0; k < K; ++k) r.d[k] = s * a.d[k];
  return r;
}
template <int K>
__device__ inline Dual<K> operator*(const Dual<K>& a, double s) { return s * a; }
template <int K>
__device__ inline Dual<K> operator/(const Dual<K>& a, double s) { return (1.0 / s) * a; }
template <int K>
__device__ inline Dual<K> operator+(double s, const Dual<K>& a) { Dual<K> r = a; r.v = s + a.v; return r; }
template <int K>
__device__ inline Dual<K> operator+(const Dual<K>& a, double s) { return s + a; }
template <int K>
__device__ inline Dual<K> operator-(double s, const Dual<K>& a) { Dual<K> r = -a; r.v = s - a.v; return r; }
template <int K>
__device__ inline Dual<K> operator-(const Dual<K>& a, double s) { Dual<K> r = a; r.v = a.v - s; return r; }
template <int K>
__device__ inline Dual<K>& operator+=(Dual<K>& a, const Dual<K>& b) { a = a + b; return a; }
template <int K>
__device__ inline Dual<K>& operator-=(Dual<K>& a, const Dual<K>& b) { a = a - b; return a; }
template <int K>
__device__ inline Dual<K>& operator-=(Dual<K>& a, double s) { a.v -= s; return a; }

// Pass 1: de/df_a into grad (nf planes of N) and mask x de/d(dx_a), mask x de/d(dy_a)
// into q (2 nf planes of N: x planes, then y planes).  Jets: FP64 difference-form
// stencils of the stored values (as the energy observable), masked like the reference.
template <class TH, typename R>
__global__ void exact_partials_kernel(const R* __restrict__ phi, double* __restrict__ grad, double* __restrict__ q,
                                      Grid G, Phys P) {
  constexpr int NF = TH::NF, K = 3 * NF;
  const long long N = G.N;
  const Inv<double> iv(G);
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x) {
    const int gx = (int)(s / G.Y), gy = (int)(s - (long long)gx * G.Y);
    const Masks m = site_masks(G, gx, gy);
    Jet1<Dual<K>, NF> J;
#pragma unroll
    for (int a = 0; a < NF; ++a) {
      const R* pa = phi + a * N;
      auto acc = [&](int ox, int oy) -> double {
        const int x = gx + ox, y = gy + oy;
        if (x < 0 || x >= G.X || y < 0 || y >= G.Y) return 0.0;
        return (double)pa[(long long)x * G.Y + y];
      };
      double f, dx, dy;
      fill_jet1_comp<double>(acc, m, iv, f, dx, dy);
      J.f[a] = Dual<K>(f);
      J.dx[a] = Dual<K>(dx);
      J.dy[a] = Dual<K>(dy);
      J.f[a].d[a] = 1.0;
      J.dx[a].d[NF + a] = 1.0;
      J.dy[a].d[2 * NF + a] = 1.0;
    }
    const Dual<K> e = TH::template energy<Dual<K>>(J, P, 1.0);
#pragma unroll
    for (int a = 0; a < NF; ++a) {
      grad[a * N + s] = e.d[a];
      q[a * N + s] = m.x ? e.d[NF + a] : 0.0;
      q[(NF + a) * N + s] = m.y ? e.d[2 * NF + a] : 0.0;
    }
  }
}

// Pass 2: grad_a(t) -= D1x[Qx_a](t) + D1y[Qy_a](t) (unmasked stencil, Q zero outside
// the lattice); with `sub` (nullable, element type R) the flow's functional derivative
// in the same rows is subtracted afterwards: grad = dE_h/dphi / dA - sub.
template <typename R>
__global__ void exact_transpose_kernel(double* __restrict__ grad, const double* __restrict__ q,
                                       const R* __restrict__ sub, int nf, Grid G) {
  const long long N = G.N;
  const double c23x = FD::c23 * G.ihx, c12x = FD::c12 * G.ihx, c23y = FD::c23 * G.ihy, c12y = FD::c12 * G.ihy;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nf * N;
       i += (long long)gridDim.x * blockDim.x) {
    const int a = (int)(i / N);
    const long long s = i - (long long)a * N;
    const int gx = (int)(s / G.Y), gy = (int)(s - (long long)gx * G.Y);
    const double* qx = q + (long long)a * N;
    const double* qy = q + (long long)(nf + a) * N;
    auto QX = [&](int ox) -> double {
      const int x = gx + ox;
      return (x < 0 || x >= G.X) ? 0.0 : qx[(long long)x * G.Y + gy];
    };
    auto QY = [&](int oy) -> double {
      const int y = gy + oy;
      return (y < 0 || y >= G.Y) ? 0.0 : qy[(long long)gx * G.Y + y];
    };
    const double dqx = c23x * (QX(1) - QX(-1)) - c12x * (QX(2) - QX(-2));
    const double dqy = c23y * (QY(1) - QY(-1)) - c12y * (QY(2) - QY(-2));
    double g = grad[i] - (dqx + dqy);
    if (sub) g -= (double)sub[i];
    grad[i] = g;
  }
}

}  // namespace ssb
