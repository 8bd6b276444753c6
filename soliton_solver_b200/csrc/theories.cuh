// theories.cuh -- per-site physics of the four theories on the hot path.
//
// Each theory is a struct with
//   NF, NMAG         number of field components / of unit-vector components
//   CONSTRAINED      unit-vector theory: gradient projected orthogonal to m and
//                    RK4 finalize normalises m (when unit_magnetization is set)
//   HALO_ZERO        gradient zeroed within `halo` of the edge (chiral magnet only)
//   NEED_XY          mixed derivatives used
//   gradient<R>()    dE/dphi at one site in working precision R (before projection)
//   energy()         energy density (FP64), already multiplied by dA
//   PAIR_ENERGY      energy_pair<V>() exists: the energy point (without dA) of a packed
//                    FP32 site pair, used for the flow's per-step energy in stage 1
//   S1_CTAS          resident CTAs per SM of the pipelined stage 1 and energy pass: 4
//                    (256 threads, 64 registers) for the light chiral stencil, else 1
//                    (512 threads)
// plus the charge densities / coupling partials it supports.  Every function
// states the reference lines it restates.
#pragma once

#include "common.cuh"
#include "pair.cuh"

namespace ssb {

enum { CH_SKYRMION = 0, CH_MAGNETIC = 1, CH_VORTEX = 2 };

// constant slot i of P as R (scalar or broadcast pair) in R's precision
template <typename R>
__device__ __forceinline__ R pk(const Phys& P, int i) {
  return R(phys_k<typename ScalarOf<R>::type>(P, i));
}
enum { CP_KAPPA = 0, CP_MPI = 1, CP_LAMBDA = 2, CP_COUP_K = 3, CP_COUP_H = 4, CP_COUP_MU = 5 };

// m.(dx m x dy m) dA / 4pi  (chiral_magnet/kernels.py:254-291, baby_skyrme/kernels.py:237-270)
template <int NF>
__device__ inline double skyrmion_density(const Jet1<double, NF>& J, double dA) {
  const double cx0 = J.dx[1] * J.dy[2] - J.dx[2] * J.dy[1];
  const double cx1 = J.dx[2] * J.dy[0] - J.dx[0] * J.dy[2];
  const double cx2 = J.dx[0] * J.dy[1] - J.dx[1] * J.dy[0];
  const double charge = J.f[0] * cx0 + J.f[1] * cx1 + J.f[2] * cx2;
  return charge * (dA / (4.0 * 3.14159265358979323846));
}

// ===========================================================================
// Chiral magnet  (theories/chiral_magnet/kernels.py)
//   c[0] coup_K  c[1] coup_h  c[2] coup_mu  c[3..6] D00 D01 D10 D11   k[0] demag
// ===========================================================================
struct ChiralMagnet {
  static constexpr int NF = 4, NMAG = 3;
  static constexpr bool CONSTRAINED = true, HALO_ZERO = true, NEED_XY = false, PAIR_ENERGY = true;
  static constexpr int S1_CTAS = 4;

  // do_gradient_step_point, kernels.py:398-503 (halo zeroing and projection are
  // applied by the caller, kernels.py:505-511).  Constants are pre-scaled so every
  // term is one fused multiply-add; R is a scalar or a packed pair of sites.
  // derived slots filled on the host (ChiralMagnet::derive):
  //   c[12] -2 D10  c[13] -2 D11  c[14] 2 D00  c[15] 2 D01  c[16] 2 D10  c[17] 2 D11
  //   c[18] -2 D00  c[19] -2 D01  c[20] -2 coup_K  c[21] 1/(2 coup_mu)  c[22] -1/coup_mu
  //   c[23] -coup_mu
  static void derive(Phys& P) {
    P.c[12] = -2.0 * P.c[5]; P.c[13] = -2.0 * P.c[6]; P.c[14] = 2.0 * P.c[3]; P.c[15] = 2.0 * P.c[4];
    P.c[16] = 2.0 * P.c[5]; P.c[17] = 2.0 * P.c[6]; P.c[18] = -2.0 * P.c[3]; P.c[19] = -2.0 * P.c[4];
    P.c[20] = -2.0 * P.c[0];
    P.c[21] = P.c[2] != 0.0 ? 1.0 / (2.0 * P.c[2]) : 0.0;
    P.c[22] = P.c[2] != 0.0 ? -1.0 / P.c[2] : 0.0;
    P.c[23] = -P.c[2];
  }
  template <typename R>
  __device__ static inline void gradient(const Jet<R, NF>& J, const Phys& P, R g[NF]) {
    const double D00 = P.c[3], D01 = P.c[4], D10 = P.c[5], D11 = P.c[6];
#pragma unroll
    for (int a = 0; a < 3; ++a) g[a] = -(J.dxx[a] + J.dyy[a]);
    g[3] = R(0.0);
    if (D00 != 0.0 || D01 != 0.0 || D10 != 0.0 || D11 != 0.0) {
      // 2 sum_{ij} D_ij eps(j,k,l) d_i m_l  in the reference's (i, j) loop order
      if (D10 != 0.0) g[0] = vfma(pk<R>(P, 12), J.dx[2], g[0]);
      if (D11 != 0.0) g[0] = vfma(pk<R>(P, 13), J.dy[2], g[0]);
      g[1] = vfma(pk<R>(P, 14), J.dx[2], g[1]);
      if (D01 != 0.0) g[1] = vfma(pk<R>(P, 15), J.dy[2], g[1]);
      if (D10 != 0.0) g[2] = vfma(pk<R>(P, 16), J.dx[0], g[2]);
      if (D11 != 0.0) g[2] = vfma(pk<R>(P, 17), J.dy[0], g[2]);
      g[2] = vfma(pk<R>(P, 18), J.dx[1], g[2]);
      if (D01 != 0.0) g[2] = vfma(pk<R>(P, 19), J.dy[1], g[2]);
    }
    // Zeeman and anisotropy: g_z -= coup_h + 2 coup_K m_z
    g[2] = vfma(pk<R>(P, 20), J.f[2], g[2] - pk<R>(P, 1));
    if (P.k[0]) {
      const R cmu = pk<R>(P, 2);
      g[0] += J.dx[3];
      g[3] = vfma(cmu, J.dx[0], g[3]) - J.dxx[3];
      g[1] += J.dy[3];
      g[3] = vfma(cmu, J.dy[1], g[3]) - J.dyy[3];
    }
  }

  // The flow's psi row is -coup_mu * dE/dpsi (psi is maximised, kernels.py:498-503):
  // dE/dpsi = -div m + lap(psi)/coup_mu = -row / coup_mu.
  template <typename R>
  __device__ static inline void true_rows(R g[NF], const Phys& P) {
    if (P.k[0]) g[3] = g[3] * pk<R>(P, 22);
  }
  // the inverse: rows of dE/dphi as the flow stores them
  template <typename R>
  __device__ static inline void flow_rows(R g[NF], const Phys& P) {
    if (P.k[0]) g[3] = g[3] * pk<R>(P, 23);
  }

  // compute_energy_point, kernels.py:125-216.  T is double, or a dual number for the
  // derivatives of the energy point with respect to its jet (adjoint.cuh).
  template <typename T>
  __device__ static inline T energy(const Jet1<T, NF>& J, const Phys& P, double dA) {
    const double cK = P.c[0], ch = P.c[1];
    const double D00 = P.c[3], D01 = P.c[4], D10 = P.c[5], D11 = P.c[6];
    T e = T(0.0);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      e += 0.5 * J.dx[a] * J.dx[a];
      e += 0.5 * J.dy[a] * J.dy[a];
    }
    const T* m = J.f;
    // i = x
    if (D00 != 0.0) { e += D00 * m[1] * J.dx[2]; e -= D00 * m[2] * J.dx[1]; }
    if (D10 != 0.0) { e -= D10 * m[0] * J.dx[2]; e += D10 * m[2] * J.dx[0]; }
    const double i2mu = P.c[21];  // 1 / (2 coup_mu), precomputed on the host
    if (P.k[0]) e -= m[3] * J.dx[0] + J.dx[3] * J.dx[3] * i2mu;
    // i = y
    if (D01 != 0.0) { e += D01 * m[1] * J.dy[2]; e -= D01 * m[2] * J.dy[1]; }
    if (D11 != 0.0) { e -= D11 * m[0] * J.dy[2]; e += D11 * m[2] * J.dy[0]; }
    if (P.k[0]) e -= m[3] * J.dy[1] + J.dy[3] * J.dy[3] * i2mu;
    const T mz = m[2];
    e += ch * (1.0 - mz);
    e += cK * (1.0 - mz * mz);
    return e * dA;
  }

  // The same energy point (without dA) in the stage's own arithmetic, for a packed
  // FP32 site pair of jets: the flow's per-step energy in stage 1.
  template <typename V>
  __device__ static inline V energy_pair(const Jet<V, NF>& J, const Phys& P) {
    const double D00 = P.c[3], D01 = P.c[4], D10 = P.c[5], D11 = P.c[6];
    V q = J.dx[0] * J.dx[0];
    q = vfma(J.dx[1], J.dx[1], q);
    q = vfma(J.dx[2], J.dx[2], q);
    q = vfma(J.dy[0], J.dy[0], q);
    q = vfma(J.dy[1], J.dy[1], q);
    q = vfma(J.dy[2], J.dy[2], q);
    V e = q * V(0.5f);
    const V* m = J.f;
    if (D00 != 0.0) e = vfma(pk<V>(P, 3), vfma(m[1], J.dx[2], -(m[2] * J.dx[1])), e);
    if (D10 != 0.0) e = vfma(pk<V>(P, 5), vfma(m[2], J.dx[0], -(m[0] * J.dx[2])), e);
    if (D01 != 0.0) e = vfma(pk<V>(P, 4), vfma(m[1], J.dy[2], -(m[2] * J.dy[1])), e);
    if (D11 != 0.0) e = vfma(pk<V>(P, 6), vfma(m[2], J.dy[0], -(m[0] * J.dy[2])), e);
    if (P.k[0]) {
      const V g2 = vfma(J.dx[3], J.dx[3], J.dy[3] * J.dy[3]);
      e = e - vfma(m[3], J.dx[0] + J.dy[1], g2 * pk<V>(P, 21));
    }
    const V one(1.0f);
    e = vfma(pk<V>(P, 1), one - m[2], e);
    e = vfma(pk<V>(P, 0), vfma(-m[2], m[2], one), e);
    return e;
  }

  __device__ static inline double charge(const Jet1<double, NF>& J, const Phys&, int which, double dA) {
    if (which == CH_SKYRMION) return skyrmion_density<NF>(J, dA);
    // compute_magnetic_charge_point, kernels.py:329-360
    double c = 0.0;
    c -= J.dx[0];
    c -= J.dy[1];
    return c * dA;
  }
  static constexpr bool has_charge(int which) { return which == CH_SKYRMION || which == CH_MAGNETIC; }

  // partial derivative of e*dA with respect to a reduced coupling at fixed field
  __device__ static inline double coupling(const Jet1<double, NF>& J, const Phys& P, int which, double dA) {
    const double mz = J.f[2];
    if (which == CP_COUP_K) return (1.0 - mz * mz) * dA;
    if (which == CP_COUP_H) return (1.0 - mz) * dA;
    if (which == CP_COUP_MU && P.k[0]) {
      const double mu = P.c[2];
      return (J.dx[3] * J.dx[3] + J.dy[3] * J.dy[3]) / (2.0 * mu * mu) * dA;
    }
    return 0.0;
  }
  static constexpr bool has_coupling(int w) { return w == CP_COUP_K || w == CP_COUP_H || w == CP_COUP_MU; }
};

// ===========================================================================
// Baby Skyrme model  (theories/baby_skyrme/kernels.py)
//   c[0] mpi  c[1] kappa   k[0..7] potential flags (Standard, Holomorphic, EasyPlane,
//   Dihedral2, Aloof, Dihedral3, Broken, DoubleVacua)  k[8] N
// ===========================================================================
struct BabySkyrme {
  static constexpr int NF = 3, NMAG = 3;
  static constexpr bool CONSTRAINED = true, HALO_ZERO = false, NEED_XY = true, PAIR_ENERGY = true;
  static constexpr int S1_CTAS = 1;
  template <typename R>
  __device__ static inline void true_rows(R*, const Phys&) {}
  template <typename R>
  __device__ static inline void flow_rows(R*, const Phys&) {}

  template <typename S>
  __device__ static inline S spow(S a, S b) {
    if constexpr (sizeof(S) == 8) return pow(a, b); else return powf(a, b);
  }

  // Broken-potential gradient terms at one site (baby_skyrme/kernels.py:427-446)
  template <typename S>
  __device__ static inline void broken(S m1, S m2, S m3, S mpi2, int N, S& g0, S& g1, S& g2) {
    const S r2 = m1 * m1 + m2 * m2;
    const S theta = atan2(m2, m1);
    const S rN2 = spow<S>(r2, (S)(0.5 * N));
    const S rN = spow<S>(r2, (S)(1.0 * N));
    const S c = cos((S)N * theta), s = sin((S)N * theta);
    const S norm1mzN = (S)1 - (S)2 * c * rN2 + rN;
    const S denom = sqrt(norm1mzN);
    if (denom != (S)0 && r2 != (S)0) {
      const S pref = (S)2 * mpi2 * (S)N * sqrt(norm1mzN) * spow<S>(r2, (S)(-1.0 + 0.5 * N)) * ((S)-1 + m3) / denom;
      g0 += pref * (s * m2 + m1 * (c - rN2));
      g1 += -pref * (s * m1 + m2 * (-c + rN2));
    }
    g2 -= mpi2 * norm1mzN;
  }

  // derived slots: c[2] mpi^2, c[3] kappa^2
  static void derive(Phys& P) {
    P.c[2] = P.c[0] * P.c[0];
    P.c[3] = P.c[1] * P.c[1];
  }

  // do_gradient_step_point, kernels.py:308-458 (projection applied by the caller)
  template <typename R>
  __device__ static inline void gradient(const Jet<R, NF>& J, const Phys& P, R g[NF]) {
    const R mpi2 = pk<R>(P, 2), kappa2 = pk<R>(P, 3);
    const R m1 = J.f[0], m2 = J.f[1], m3 = J.f[2];
    const R F00 = J.dx[0], F01 = J.dx[1], F02 = J.dx[2];
    const R F10 = J.dy[0], F11 = J.dy[1], F12 = J.dy[2];
    const R S000 = J.dxx[0], S001 = J.dxx[1], S002 = J.dxx[2];
    const R S110 = J.dyy[0], S111 = J.dyy[1], S112 = J.dyy[2];
    const R S010 = J.dxy[0], S011 = J.dxy[1], S012 = J.dxy[2];
    const R S100 = S010, S101 = S011, S102 = S012;
    const R sum_F0_sq = F00 * F00 + F01 * F01 + F02 * F02;
    const R sum_F1_sq = F10 * F10 + F11 * F11 + F12 * F12;
    R g0 = -(S000 + S110), g1 = -(S001 + S111), g2 = -(S002 + S112);
    const R sum_all_sq = sum_F0_sq + sum_F1_sq;
    g0 -= kappa2 * S000 * sum_all_sq;
    g1 -= kappa2 * S001 * sum_all_sq;
    g2 -= kappa2 * S002 * sum_all_sq;
    g0 += kappa2 * S000 * sum_F0_sq;
    g1 += kappa2 * S001 * sum_F0_sq;
    g2 += kappa2 * S002 * sum_F0_sq;
    const R sumA = (S010 * F10 - S110 * F00) + (S011 * F11 - S111 * F01) + (S012 * F12 - S112 * F02);
    const R dot01 = F00 * F10 + F01 * F11 + F02 * F12;
    g0 -= kappa2 * (F00 * sumA - S010 * dot01);
    g1 -= kappa2 * (F01 * sumA - S011 * dot01);
    g2 -= kappa2 * (F02 * sumA - S012 * dot01);
    g0 -= kappa2 * S110 * sum_all_sq;
    g1 -= kappa2 * S111 * sum_all_sq;
    g2 -= kappa2 * S112 * sum_all_sq;
    g0 += kappa2 * S110 * sum_F1_sq;
    g1 += kappa2 * S111 * sum_F1_sq;
    g2 += kappa2 * S112 * sum_F1_sq;
    const R sumB = (S100 * F00 - S000 * F10) + (S101 * F01 - S001 * F11) + (S102 * F02 - S002 * F12);
    g0 -= kappa2 * (F10 * sumB - S100 * dot01);
    g1 -= kappa2 * (F11 * sumB - S101 * dot01);
    g2 -= kappa2 * (F12 * sumB - S102 * dot01);
    if (P.k[0]) g2 -= mpi2;
    if (P.k[1]) { const R t = (R)1 - m3; g2 -= (R)4 * mpi2 * t * t * t; }
    if (P.k[2]) g0 += mpi2 * m1;
    if (P.k[3]) {
      g0 -= mpi2 * ((R)1 - m3 * m3) * m1;
      g2 -= mpi2 * ((R)1 - m1 * m1) * m3;
    }
    if (P.k[4]) {
      const R t = (R)1 - m3, t3 = t * t * t;
      g2 -= mpi2 * ((R)0.5 * ((R)1 + t3) + (R)1.5 * t3);
    }
    if (P.k[5]) {
      g0 += (R)48 * mpi2 * (m2 * m2 - m1 * m1) * ((R)1 - m3);
      g1 += (R)96 * mpi2 * m1 * m2 * ((R)1 - m3);
      g2 -= (R)16 * mpi2 * (-(m1 * m1 * m1) + (R)3 * m1 * (m2 * m2) + ((R)1 - (R)3 * m3) * ((R)1 - (R)3 * m3));
    }
    if (P.k[6]) {
      // broken potential: transcendental, evaluated site by site
      using S = typename ScalarOf<R>::type;
#pragma unroll
      for (int l = 0; l < Lanes<R>::N; ++l) {
        S a0 = Lanes<R>::get(g0, l), a1 = Lanes<R>::get(g1, l), a2 = Lanes<R>::get(g2, l);
        broken<S>(Lanes<R>::get(m1, l), Lanes<R>::get(m2, l), Lanes<R>::get(m3, l), phys_k<S>(P, 2), P.k[8],
                  a0, a1, a2);
        Lanes<R>::set(g0, l, a0);
        Lanes<R>::set(g1, l, a1);
        Lanes<R>::set(g2, l, a2);
      }
    }
    if (P.k[7]) g2 -= (R)2 * mpi2 * m3;
    g[0] = g0; g[1] = g1; g[2] = g2;
  }

  // potential terms of compute_energy_point without the mpi^2 factor, kernels.py:176-199
  __device__ static inline double potential_unit(const double* m, const Phys& P) {
    const double m1 = m[0], m2 = m[1], m3 = m[2];
    double u = 0.0;
    if (P.k[0]) u += (1.0 - m3);
    if (P.k[1]) { const double t = 1.0 - m3; u += t * t * t * t; }
    if (P.k[2]) u += 0.5 * m1 * m1;
    if (P.k[3]) u += 0.5 * (1.0 - m1 * m1) * (1.0 - m3 * m3);
    if (P.k[4]) { const double t = 1.0 - m3; u += 0.5 * t * (1.0 + t * t * t); }
    if (P.k[5]) u += 16.0 * (1.0 - m3) * (1.0 + 3.0 * m3 * m3 + 3.0 * m1 * m2 * m2 - m1 * m1 * m1);
    if (P.k[6]) {
      double zr = m1, zi = m2;
      for (int i = 0; i < P.k[8] - 1; ++i) {
        const double tr = zr * m1 - zi * m2;
        zi = zr * m2 + zi * m1;
        zr = tr;
      }
      const double wr = 1.0 - zr, wi = -zi;
      u += (1.0 - m3) * (wr * wr + wi * wi);
    }
    if (P.k[7]) u += (1.0 - m3 * m3);
    return u;
  }

  // compute_energy_point, kernels.py:127-199 (T: double, or a dual number, adjoint.cuh)
  template <typename T>
  __device__ static inline T energy(const Jet1<T, NF>& J, const Phys& P, double dA) {
    const double mpi = P.c[0], mpi2 = mpi * mpi, kappa = P.c[1], kappa2 = kappa * kappa;
    const T gx = J.dx[0] * J.dx[0] + J.dx[1] * J.dx[1] + J.dx[2] * J.dx[2];
    const T gy = J.dy[0] * J.dy[0] + J.dy[1] * J.dy[1] + J.dy[2] * J.dy[2];
    T e = 0.5 * (gx + gy);
    const T cx = J.dx[1] * J.dy[2] - J.dx[2] * J.dy[1];
    const T cy = J.dx[2] * J.dy[0] - J.dx[0] * J.dy[2];
    const T cz = J.dx[0] * J.dy[1] - J.dx[1] * J.dy[0];
    e += 0.5 * kappa2 * (cx * cx + cy * cy + cz * cz);
    const T m1 = J.f[0], m2 = J.f[1], m3 = J.f[2];
    if (P.k[0]) e += mpi2 * (1.0 - m3);
    if (P.k[1]) { const T t = 1.0 - m3; e += mpi2 * t * t * t * t; }
    if (P.k[2]) e += 0.5 * mpi2 * m1 * m1;
    if (P.k[3]) e += 0.5 * mpi2 * (1.0 - m1 * m1) * (1.0 - m3 * m3);
    if (P.k[4]) { const T t = 1.0 - m3; e += 0.5 * mpi2 * t * (1.0 + t * t * t); }
    if (P.k[5]) e += 16.0 * mpi2 * (1.0 - m3) * (1.0 + 3.0 * m3 * m3 + 3.0 * m1 * m2 * m2 - m1 * m1 * m1);
    if (P.k[6]) {
      T zr = m1, zi = m2;
      for (int i = 0; i < P.k[8] - 1; ++i) {
        const T tr = zr * m1 - zi * m2;
        zi = zr * m2 + zi * m1;
        zr = tr;
      }
      const T wr = 1.0 - zr, wi = -zi;
      e += mpi2 * (1.0 - m3) * (wr * wr + wi * wi);
    }
    if (P.k[7]) e += mpi2 * (1.0 - m3 * m3);
    return e * dA;
  }

  // the same energy point for a packed FP32 site pair, without dA (the flow's per-step
  // energy from the gradient's jets; FP32 rounding per site, FP64 sums)
  template <typename V>
  __device__ static inline V energy_pair(const Jet<V, NF>& J, const Phys& P) {
    const V mpi2(P.cf[0] * P.cf[0]), hk2(0.5f * (P.cf[1] * P.cf[1])), half(0.5f), one(1.0f);
    V g = J.dx[0] * J.dx[0];
    g = vfma(J.dx[1], J.dx[1], g);
    g = vfma(J.dx[2], J.dx[2], g);
    g = vfma(J.dy[0], J.dy[0], g);
    g = vfma(J.dy[1], J.dy[1], g);
    g = vfma(J.dy[2], J.dy[2], g);
    V e = half * g;
    const V cx = vfma(J.dx[1], J.dy[2], -(J.dx[2] * J.dy[1]));
    const V cy = vfma(J.dx[2], J.dy[0], -(J.dx[0] * J.dy[2]));
    const V cz = vfma(J.dx[0], J.dy[1], -(J.dx[1] * J.dy[0]));
    e = vfma(hk2, vfma(cx, cx, vfma(cy, cy, cz * cz)), e);
    const V m1 = J.f[0], m2 = J.f[1], m3 = J.f[2];
    const V t = one - m3;
    V u(0.0f);
    if (P.k[0]) u = u + t;
    if (P.k[1]) u = vfma(t * t, t * t, u);
    if (P.k[2]) u = vfma(half * m1, m1, u);
    if (P.k[3]) u = vfma(half * vfma(-m1, m1, one), vfma(-m3, m3, one), u);
    if (P.k[4]) u = vfma(half * t, vfma(t * t, t, one), u);
    if (P.k[5]) {
      const V q = vfma(V(3.0f) * m1, m2 * m2, vfma(V(3.0f) * m3, m3, one)) - m1 * m1 * m1;
      u = vfma(V(16.0f) * t, q, u);
    }
    if (P.k[6]) {
      V zr = m1, zi = m2;
      for (int i = 0; i < P.k[8] - 1; ++i) {
        const V tr = vfma(zr, m1, -(zi * m2));
        zi = vfma(zr, m2, zi * m1);
        zr = tr;
      }
      const V wr = one - zr;
      u = vfma(t, vfma(wr, wr, zi * zi), u);
    }
    if (P.k[7]) u = u + vfma(-m3, m3, one);
    return vfma(mpi2, u, e);
  }

  __device__ static inline double charge(const Jet1<double, NF>& J, const Phys&, int, double dA) {
    return skyrmion_density<NF>(J, dA);
  }
  static constexpr bool has_charge(int which) { return which == CH_SKYRMION; }

  __device__ static inline double coupling(const Jet1<double, NF>& J, const Phys& P, int which, double dA) {
    if (which == CP_KAPPA) {
      const double cx = J.dx[1] * J.dy[2] - J.dx[2] * J.dy[1];
      const double cy = J.dx[2] * J.dy[0] - J.dx[0] * J.dy[2];
      const double cz = J.dx[0] * J.dy[1] - J.dx[1] * J.dy[0];
      return P.c[1] * (cx * cx + cy * cy + cz * cz) * dA;
    }
    if (which == CP_MPI) return 2.0 * P.c[0] * potential_unit(J.f, P) * dA;
    return 0.0;
  }
  static constexpr bool has_coupling(int w) { return w == CP_KAPPA || w == CP_MPI; }
};

// ===========================================================================
// Ginzburg-Landau / Abelian Higgs  (theories/ginzburg_landau_superconductor/kernels.py)
//   c[0] q  c[1] Lambda  c[2] u1 (p_f[8], used by the gradient)
//   c[3] p_f[9] (vortex_number, which the reference's energy reads as u1)
// ===========================================================================
struct GinzburgLandau {
  static constexpr int NF = 4, NMAG = 0;
  static constexpr bool CONSTRAINED = false, HALO_ZERO = false, NEED_XY = true, PAIR_ENERGY = true;
  static constexpr int S1_CTAS = 1;
  template <typename R>
  __device__ static inline void true_rows(R*, const Phys&) {}
  template <typename R>
  __device__ static inline void flow_rows(R*, const Phys&) {}

  // derived slot: c[4] Lambda / 2
  static void derive(Phys& P) { P.c[4] = 0.5 * P.c[1]; }

  // do_gradient_step_point, kernels.py:343-419
  template <typename R>
  __device__ static inline void gradient(const Jet<R, NF>& J, const Phys& P, R g[NF]) {
    const R q = pk<R>(P, 0), u1 = pk<R>(P, 2);
    const R A1 = J.f[0], A2 = J.f[1], psi1 = J.f[2], psi2 = J.f[3];
    const R psi_sq = psi1 * psi1 + psi2 * psi2;
    const R dA1dx = J.dx[0], dA1dy = J.dy[0], dA2dx = J.dx[1], dA2dy = J.dy[1];
    const R dpsi1dx = J.dx[2], dpsi1dy = J.dy[2], dpsi2dx = J.dx[3], dpsi2dy = J.dy[3];
    const R pot = pk<R>(P, 4) * (u1 * u1 - psi_sq);
    const R Asq = A1 * A1 + A2 * A2;
    (void)dA2dx;
    (void)dA1dy;
    g[0] = -J.dyy[0] + J.dxy[1] + q * (psi1 * dpsi2dx - psi2 * dpsi1dx) + q * q * A1 * psi_sq;
    g[1] = -J.dxx[1] + J.dxy[0] + q * (psi1 * dpsi2dy - psi2 * dpsi1dy) + q * q * A2 * psi_sq;
    g[2] = -J.dxx[2] - J.dyy[2] + (R)2 * q * (A1 * dpsi2dx + A2 * dpsi2dy) + q * psi2 * (dA1dx + dA2dy) +
           q * q * Asq * psi1 - pot * psi1;
    g[3] = -J.dxx[3] - J.dyy[3] - (R)2 * q * (A1 * dpsi1dx + A2 * dpsi1dy) - q * psi1 * (dA1dx + dA2dy) +
           q * q * Asq * psi2 - pot * psi2;
  }

  // compute_energy_point, kernels.py:46-108 (u read from p_f[9] as the reference does;
  // T: double, or a dual number, adjoint.cuh)
  template <typename T>
  __device__ static inline T energy(const Jet1<T, NF>& J, const Phys& P, double dA) {
    const double q = P.c[0], lam = P.c[1], u1 = P.c[3];
    const T A1 = J.f[0], A2 = J.f[1], psi1 = J.f[2], psi2 = J.f[3];
    const T dpsi1dx = J.dx[2], dpsi1dy = J.dy[2], dpsi2dx = J.dx[3], dpsi2dy = J.dy[3];
    const T psi_sq = psi1 * psi1 + psi2 * psi2;
    const T A_sq = A1 * A1 + A2 * A2;
    T e = T(0.0);
    e += 0.5 * (dpsi1dx * dpsi1dx + dpsi1dy * dpsi1dy + dpsi2dx * dpsi2dx + dpsi2dy * dpsi2dy);
    e += q * A1 * (psi1 * dpsi2dx - psi2 * dpsi1dx);
    e += q * A2 * (psi1 * dpsi2dy - psi2 * dpsi1dy);
    e += 0.5 * q * q * A_sq * psi_sq;
    e += lam / 8.0 * (u1 * u1 - psi_sq) * (u1 * u1 - psi_sq);
    const T curlA = J.dx[1] - J.dy[0];
    e += 0.5 * curlA * curlA;
    return e * dA;
  }

  // the same energy point for a packed FP32 site pair, without dA (flow energies from
  // the gradient's jets, FP64 sums); u as above
  template <typename V>
  __device__ static inline V energy_pair(const Jet<V, NF>& J, const Phys& P) {
    const float qf = P.cf[0], uf = P.cf[3];
    const V q(qf), hq2(0.5f * (qf * qf)), lam8(0.125f * P.cf[1]), u2(uf * uf), half(0.5f);
    const V A1 = J.f[0], A2 = J.f[1], p1 = J.f[2], p2 = J.f[3];
    const V p1x = J.dx[2], p1y = J.dy[2], p2x = J.dx[3], p2y = J.dy[3];
    const V psq = vfma(p1, p1, p2 * p2);
    const V Asq = vfma(A1, A1, A2 * A2);
    V g = p1x * p1x;
    g = vfma(p1y, p1y, g);
    g = vfma(p2x, p2x, g);
    g = vfma(p2y, p2y, g);
    V e = half * g;
    e = vfma(q * A1, vfma(p1, p2x, -(p2 * p1x)), e);
    e = vfma(q * A2, vfma(p1, p2y, -(p2 * p1y)), e);
    e = vfma(hq2 * Asq, psq, e);
    const V d = u2 - psq;
    e = vfma(lam8 * d, d, e);
    const V curl = J.dx[1] - J.dy[0];
    return vfma(half * curl, curl, e);
  }

  // compute_vortex_density, kernels.py:146-178
  __device__ static inline double charge(const Jet1<double, NF>& J, const Phys& P, int, double dA) {
    const double b = J.dx[1] - J.dy[0];
    return b * (dA / (2.0 * 3.14159265358979323846 * P.c[0]));
  }
  static constexpr bool has_charge(int which) { return which == CH_VORTEX; }

  __device__ static inline double coupling(const Jet1<double, NF>& J, const Phys& P, int which, double dA) {
    if (which != CP_LAMBDA) return 0.0;
    const double u = P.c[3];
    const double psi_sq = J.f[2] * J.f[2] + J.f[3] * J.f[3];
    return (u * u - psi_sq) * (u * u - psi_sq) / 8.0 * dA;
  }
  static constexpr bool has_coupling(int w) { return w == CP_LAMBDA; }
};

// ===========================================================================
// Anisotropic s+id superconductor  (theories/anisotropic_superconductor/kernels.py)
//   c[0] kappa c[1] Q c[2] alpha1 c[3] alpha2 c[4..7] beta1..beta4
//   c[8] gamma1 c[9] gamma2 c[10] gamma12 c[11] vacuum energy density (kernels.py:169)
// The anisotropy tensor gamma_entry(i, j, a, b) (kernels.py:46-94) vanishes for i != j.
// ===========================================================================
struct Anisotropic {
  static constexpr int NF = 6, NMAG = 0;
  static constexpr bool CONSTRAINED = false, HALO_ZERO = false, NEED_XY = true, PAIR_ENERGY = false;
  static constexpr int S1_CTAS = 1;
  template <typename R>
  __device__ static inline void true_rows(R*, const Phys&) {}
  template <typename R>
  __device__ static inline void flow_rows(R*, const Phys&) {}

  template <typename R>
  __device__ static inline R gamR(int i, int a, int b, const Phys& P) {
    if (a == 0 && b == 0) return pk<R>(P, 13);
    if (a == 1 && b == 1) return pk<R>(P, 14);
    return i == 0 ? -pk<R>(P, 15) : pk<R>(P, 15);
  }
  __device__ static inline double gam(int i, int a, int b, const Phys& P) {
    if (a == 0 && b == 0) return 2.0 * P.c[8];
    if (a == 1 && b == 1) return 2.0 * P.c[9];
    return (i == 0 ? -2.0 : 2.0) * P.c[10];
  }

  // derived slots: c[12] kappa^2, c[13..15] 2 gamma1, 2 gamma2, 2 gamma12
  static void derive(Phys& P) {
    P.c[12] = P.c[0] * P.c[0];
    P.c[13] = 2.0 * P.c[8];
    P.c[14] = 2.0 * P.c[9];
    P.c[15] = 2.0 * P.c[10];
  }

  // do_gradient_step_point, kernels.py:556-658
  template <typename R>
  __device__ static inline void gradient(const Jet<R, NF>& J, const Phys& P, R g[NF]) {
    const R Q = pk<R>(P, 1);
    const R a1 = pk<R>(P, 2), a2 = pk<R>(P, 3);
    const R b1 = pk<R>(P, 4), b2 = pk<R>(P, 5), b3 = pk<R>(P, 6), b4 = pk<R>(P, 7);
    const R A[2] = {J.f[0], J.f[1]};
    const R p1r = J.f[2], p1i = J.f[3], p2r = J.f[4], p2i = J.f[5];
    const R k2 = pk<R>(P, 12);
    // second derivative d_i d_j of component a
    auto d2 = [&](int i, int j, int a) -> R { return i != j ? J.dxy[a] : (i == 0 ? J.dxx[a] : J.dyy[a]); };
    auto d1 = [&](int i, int a) -> R { return i == 0 ? J.dx[a] : J.dy[a]; };
    R EG[6] = {(R)0, (R)0, (R)0, (R)0, (R)0, (R)0};
#pragma unroll
    for (int j = 0; j < 2; ++j) {
#pragma unroll
      for (int k = 0; k < 2; ++k) {
        R val = k2 * (d2(j, k, k) - d2(k, k, j));
        if (k == j) {
          const R Ak = A[k];
          const R g00 = gamR<R>(k, 0, 0, P), g01 = gamR<R>(k, 0, 1, P), g10 = gamR<R>(k, 1, 0, P),
                  g11 = gamR<R>(k, 1, 1, P);
          val -= Q * g00 * (p1i * d1(k, 2) - p1r * d1(k, 3) - Q * Ak * (p1r * p1r + p1i * p1i));
          val -= Q * g01 * (p2i * d1(k, 2) - p2r * d1(k, 3) - Q * Ak * (p1r * p2r + p1i * p2i));
          val -= Q * g10 * (p1i * d1(k, 4) - p1r * d1(k, 5) - Q * Ak * (p2r * p1r + p2i * p1i));
          val -= Q * g11 * (p2i * d1(k, 4) - p2r * d1(k, 5) - Q * Ak * (p2r * p2r + p2i * p2i));
        }
        EG[j] += val;
      }
    }
    const R p1sq = p1r * p1r + p1i * p1i, p2sq = p2r * p2r + p2i * p2i;
    EG[2] += (R)2 * ((R)2 * a1 * p1r + (R)4 * b1 * p1r * p1sq + (R)2 * b3 * p1r * p2sq +
                     (R)2 * b4 * ((R)2 * p1r * (p2r * p2r - p2i * p2i) + (R)4 * p1i * p2r * p2i));
    EG[3] += (R)2 * ((R)2 * a1 * p1i + (R)4 * b1 * p1i * p1sq + (R)2 * b3 * p1i * p2sq +
                     (R)2 * b4 * ((R)-2 * p1i * (p2r * p2r - p2i * p2i) + (R)4 * p1r * p2r * p2i));
    EG[4] += (R)2 * ((R)2 * a2 * p2r + (R)4 * b2 * p2r * p2sq + (R)2 * b3 * p2r * p1sq +
                     (R)2 * b4 * ((R)2 * p2r * (p1r * p1r - p1i * p1i) + (R)4 * p1r * p1i * p2i));
    EG[5] += (R)2 * ((R)2 * a2 * p2i + (R)4 * b2 * p2i * p2sq + (R)2 * b3 * p2i * p1sq +
                     (R)2 * b4 * ((R)-2 * p2i * (p1r * p1r - p1i * p1i) + (R)4 * p1r * p1i * p2r));
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const R Ai = A[i];
      const R g00 = gamR<R>(i, 0, 0, P), g01 = gamR<R>(i, 0, 1, P), g10 = gamR<R>(i, 1, 0, P),
              g11 = gamR<R>(i, 1, 1, P);
      const R dAii = d1(i, i);
      const R QQAA = Q * Q * Ai * Ai;
      EG[2] -= g00 * (d2(i, i, 2) - QQAA * p1r - Q * (p1i * dAii + Ai * d1(i, 3) + Ai * d1(i, 3)));
      EG[2] -= g01 * (d2(i, i, 4) - QQAA * p2r - Q * (p2i * dAii + Ai * d1(i, 5) + Ai * d1(i, 5)));
      EG[3] -= g00 * (d2(i, i, 3) - QQAA * p1i + Q * (p1r * dAii + Ai * d1(i, 2) + Ai * d1(i, 2)));
      EG[3] -= g01 * (d2(i, i, 5) - QQAA * p2i + Q * (p2r * dAii + Ai * d1(i, 4) + Ai * d1(i, 4)));
      EG[4] -= g10 * (d2(i, i, 2) - QQAA * p1r - Q * (p1i * dAii + Ai * d1(i, 3) + Ai * d1(i, 3)));
      EG[4] -= g11 * (d2(i, i, 4) - QQAA * p2r - Q * (p2i * dAii + Ai * d1(i, 5) + Ai * d1(i, 5)));
      EG[5] -= g10 * (d2(i, i, 3) - QQAA * p1i + Q * (p1r * dAii + Ai * d1(i, 2) + Ai * d1(i, 2)));
      EG[5] -= g11 * (d2(i, i, 5) - QQAA * p2i + Q * (p2r * dAii + Ai * d1(i, 4) + Ai * d1(i, 4)));
    }
#pragma unroll
    for (int a = 0; a < 6; ++a) g[a] = EG[a];
  }

  // compute_energy_point, kernels.py:97-170 (T: double, or a dual number, adjoint.cuh)
  template <typename T>
  __device__ static inline T energy(const Jet1<T, NF>& J, const Phys& P, double dA) {
    const double kappa = P.c[0], Q = P.c[1], a1 = P.c[2], a2 = P.c[3];
    const double b1 = P.c[4], b2 = P.c[5], b3 = P.c[6], b4 = P.c[7];
    const T A[2] = {J.f[0], J.f[1]};
    const T p1r = J.f[2], p1i = J.f[3], p2r = J.f[4], p2i = J.f[5];
    const T p1sq = p1r * p1r + p1i * p1i, p2sq = p2r * p2r + p2i * p2i;
    const T curl = J.dx[1] - J.dy[0];
    const T F_mag = 0.5 * kappa * kappa * (curl * curl);
    T F_pot = T(0.0);
    F_pot += a1 * p1sq + a2 * p2sq;
    F_pot += b1 * p1sq * p1sq + b2 * p2sq * p2sq + b3 * p1sq * p2sq;
    F_pot += 2.0 * b4 * (p1r * p1r * p2r * p2r + p1i * p1i * p2i * p2i - p1i * p1i * p2r * p2r -
                         p1r * p1r * p2i * p2i + 4.0 * p1r * p1i * p2r * p2i);
    T F_kin = T(0.0);
#pragma unroll
    for (int i = 0; i < 2; ++i) {
      const T Ai = A[i];
      const T* d = (i == 0) ? J.dx : J.dy;
      const double g00 = gam(i, 0, 0, P), g01 = gam(i, 0, 1, P), g10 = gam(i, 1, 0, P), g11 = gam(i, 1, 1, P);
      const T r1 = d[2], i1 = d[3], r2 = d[4], i2 = d[5];
      F_kin += 0.5 * g00 * (r1 * r1 + i1 * i1 + Q * Ai * (p1r * i1 - p1i * r1) + Q * Ai * (p1r * i1 - p1i * r1) +
                            Q * Q * Ai * Ai * p1sq);
      F_kin += 0.5 * g01 * (r1 * r2 + i1 * i2 + Q * Ai * (p1r * i2 - p1i * r2) + Q * Ai * (p2r * i1 - p2i * r1) +
                            Q * Q * Ai * Ai * (p1r * p2r + p1i * p2i));
      F_kin += 0.5 * g10 * (r2 * r1 + i2 * i1 + Q * Ai * (p2r * i1 - p2i * r1) + Q * Ai * (p1r * i2 - p1i * r2) +
                            Q * Q * Ai * Ai * (p2r * p1r + p2i * p1i));
      F_kin += 0.5 * g11 * (r2 * r2 + i2 * i2 + Q * Ai * (p2r * i2 - p2i * r2) + Q * Ai * (p2r * i2 - p2i * r2) +
                            Q * Q * Ai * Ai * p2sq);
    }
    T e = F_kin + F_mag + F_pot;
    e -= P.c[11];
    return e * dA;
  }

  // compute_vortex_density, kernels.py:208-240 (q = p_f[7])
  __device__ static inline double charge(const Jet1<double, NF>& J, const Phys& P, int, double dA) {
    const double b = J.dx[1] - J.dy[0];
    return b * (dA / (2.0 * 3.14159265358979323846 * P.c[1]));
  }
  static constexpr bool has_charge(int which) { return which == CH_VORTEX; }
  __device__ static inline double coupling(const Jet1<double, NF>&, const Phys&, int, double) { return 0.0; }
  static constexpr bool has_coupling(int) { return false; }
};

}  // namespace ssb
