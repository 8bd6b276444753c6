// flow.cuh -- fused single-pass-per-stage kernels of the arrested-Newton-flow step.
//
// One RK4 step of the reference (core/integrator.py:217-348) is
//   k1 = dt V,            T1 = phi,           l1 = -dt G(T1)
//   k2 = dt (V + l1/2),   T2 = phi + k1/2,    l2 = -dt G(T2)
//   k3 = dt (V + l2/2),   T3 = phi + k2/2,    l3 = -dt G(T3)
//   k4 = dt (V + l3),     T4 = phi + k3,      l4 = -dt G(T4)
//   V' = V + (l1 + 2 l2 + 2 l3 + l4)/6,  phi' = phi + (k1 + 2 k2 + 2 k3 + k4)/6
// followed by the unit-norm re-projection, the energy of phi', the arrest test
// (E' > E -> V' = 0) and err = max G(T4).  The update is linear in V and the l_s, so
// everything stage 4 needs besides l4 is known once l2 and l3 are:
//   T4 = phi + dt (V + l2/2),  cV = V + (l1 + 2 l2 + 2 l3)/6,  cP = phi + dt V + dt (l1 + l2 + l3)/6
//   V' = cV + l4/6,            phi' = cP (re-projected)
// Stage s recomputes its T_s from (phi, V, l_s) while a tile is staged:
//   S1  reads phi                        writes l1  (+ energy of phi, see below)
//   S2  reads phi, V                     writes l2
//   S3  reads phi, V, l1 (+ l2 centres)  writes T4, cV, cP
//   S4  reads T4 (halo tile), cP, cV     writes phi', V', err
// Stage 4 reads neither phi nor V, so it writes the caller's buffers in place (no
// ping-pong copies).  The energy of a step's result is computed by the NEXT step's S1,
// which stages exactly that field anyway, and the arrest decision is kept on the
// device (StepState.arrest) and applied by S2/S3 as "V = 0".  A trailing energy pass
// closes a call.  Compulsory traffic: 13 words per site and step when stages 2 and 3
// run as one kernel (M_S23: S1 2, S2+S3 6, S4 5), 17 as four kernels (S2 3, S3 7 with
// the l2 centres).
#pragma once

#include <cuda.h>

#include "common.cuh"
#include "pair.cuh"
#include "theories.cuh"

namespace ssb {

// M_S23: stages 2 and 3 fused (one staging of phi, V, l1; writes l2 and l3)
enum FlowMode { M_GRAD = 0, M_S1 = 1, M_S2 = 2, M_S3 = 3, M_S4 = 4, M_ENERGY = 5, M_S23 = 6 };
constexpr int N_FLOW_MODES = 7;
enum { ST_TIMEOUT = 6 };

// Default bound of a device-side wait on an mbarrier (~1 s at 1.9 GHz).  On expiry
// the kernel records ST_TIMEOUT, waits the same bound again for its copies in
// flight and returns without computing.
constexpr long long WAIT_CYCLES = 2000000000LL;

template <typename R>
struct FlowArgs {
  CUtensorMap tm_phi;  // TMA maps (used when the kernel is instantiated with TMA):
  CUtensorMap tm_vel;  //   halo boxes of the staged field (phi; T4 in S4), of V,
  CUtensorMap tm_l;    //   of l1 (S3, M_S23),
  CUtensorMap tm_cp;   //   and centre boxes of cP and cV (pipelined S4)
  CUtensorMap tm_cv;
  const R* phi;  // the staged field: phi, or T4 in S4
  const R* vel;  // V (S2, S3, M_S23)
  const R* la;   // l1 (S3, M_S23)
  const R* lb;   // l2 (S3)
  const R* cp;   // S4: cP = phi + dt V + dt (l1 + l2 + l3)/6
  const R* cv;   // S4: cV = V + (l1 + 2 l2 + 2 l3)/6
  R* out_l;      // S1, S2: l_s;  M_GRAD: l_out (nullable)
  R* out_t4;     // S3 / M_S23: T4 = phi + dt (V + l2/2)
  R* out_cp;     // S3 / M_S23: cP
  R* out_cv;     // S3 / M_S23: cV
  R* out_eg;     // M_GRAD: energy gradient (nullable)
  R* phi_out;    // S4: phi' (may be the caller's phi: stage 4 reads neither phi nor V)
  R* vel_out;    // S4: V'
  const double* force;  // FP64 fields (nullable): added to the flow's gradient rows in every stage
  double* partial;  // per-block energy partials
  StepState* st;
  double* E_traj;   // nullable
  double* err_traj; // nullable
  int E_idx;        // slot of E_traj the energy goes to (< 0: none)
  int err_idx;      // slot of err_traj the S4 error goes to (< 0: none)
  int mode;
  int with_energy;    // S1 / M_ENERGY: reduce the energy of the staged field
  int arrest_update;  // after the energy: arrest = killkinen && E > E_last; E_last = E
  int init_state;     // first S1 of a call: arrest = 0 and (unless NaN) E_last = prev_energy
  double prev_energy;
  int grad_raw;           // M_GRAD: unprojected, not halo-zeroed dE/dphi with true saddle rows
  int exact_energy;       // M_ENERGY on FP32 fields: 1 = FP64 stencil of the stored values
                          // (observables), 0 = from the FP32 jets like stage 1 (flow energies)
  long long wait_cycles;  // bound of every mbarrier wait (clock64 cycles)
  unsigned tx_extra;      // test hook: bytes the barrier expects beyond what is loaded (normally 0)
  Grid G;
  Phys P;
};

// Tile of TX x TY sites.  Staged planes hold rows x0-2 .. x0+TX+1 and columns
// y0-4 .. y0+TY+3: the y start is rounded down to a 16-byte boundary so the same
// geometry serves TMA boxes and plain loads; the stencil uses columns 2 .. TY+5.
template <int TX, int TY, int NT>
struct TileShape {
  static constexpr int HX = TX + 4, HY = TY + 8, YOFF = 4;
  static constexpr int PLANE = HX * HY;
  static constexpr int ROWS_PER_PASS = NT / TY;
  static constexpr int SITES_PER_THREAD = TX / ROWS_PER_PASS;
  static_assert(NT % TY == 0 && TX % (NT / TY) == 0, "tile/thread mismatch");
  static_assert(TY % 4 == 0, "TY must keep the y start 16-byte aligned");
};

template <typename R, int NF, int TX, int TY>
__host__ __device__ constexpr size_t tile_buf_bytes() {
  return sizeof(R) * NF * (TX + 4) * (TY + 8);
}

// number of staged halo buffers a mode needs (phi, then V, then l1; T4 alone in S4)
__host__ __device__ constexpr int flow_buffers(int mode) {
  return mode == M_S2 ? 2 : (mode == M_S3 || mode == M_S23) ? 3 : 1;
}

// ---------------------------------------------------------------------------
// TMA / mbarrier helpers (inline PTX, sm_90+ instructions, used on sm_100a)
// ---------------------------------------------------------------------------
__device__ inline uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ inline void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ inline void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// try_wait with a suspend-time hint: the thread sleeps until the phase completes or
// ~1 ms passes instead of spinning, so waiting warps take no issue slots from the
// warps that compute.
__device__ inline bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity), "r"(1000000u)
      : "memory");
  return ok != 0;
}
// 3-D tiled bulk tensor load global -> shared (no multicast), completion on `bar`.
__device__ inline void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
      ::"r"(smem_u32(dst)), "l"((uint64_t)map), "r"(c0), "r"(c1), "r"(c2), "r"(smem_u32(bar))
      : "memory");
}
// Bounded wait; returns false when `limit` clock64 cycles elapsed first.
__device__ inline bool mbar_wait_bounded(uint64_t* bar, uint32_t parity, long long limit) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > limit) return false;
  }
  return true;
}

// T_s for one element from the staged inputs (the reference's k / Temp algebra,
// core/integrator.py:51-96 and :323-334); stage 4's T4 is stored by stage 3
template <typename R>
__device__ inline R stage_value(int mode, R p, R v, R w, R dt) {
  const R half = (R)0.5;
  if (mode == M_S2) return p + half * (dt * v);
  if (mode == M_S3) return p + half * (dt * (v + half * w));
  return p;
}

// Plain-load staging of one halo buffer T = T_s(psrc, vsrc, wsrc) (all components;
// vsrc / wsrc nullable), used when a TMA map cannot describe the buffers (row pitch
// not a multiple of 16 bytes).  Every thread first issues all loads of one component
// plane, then combines and stores, so each plane costs one memory round trip.
template <int NF, typename R, int TX, int TY, int NT>
__device__ inline void stage_plain_buf(R* T, const Grid& G, const R* psrc, const R* vsrc, const R* wsrc, int x0,
                                       int y0, int mode) {
  using TS = TileShape<TX, TY, NT>;
  constexpr int KM = (TS::PLANE + NT - 1) / NT;
  const long long N = G.N;
  const R dt = (R)G.dt;
  long long off[KM];
  bool ok[KM];
#pragma unroll
  for (int k = 0; k < KM; ++k) {
    const int i = threadIdx.x + k * NT;
    const int r = i / TS::HY, c = i - r * TS::HY;
    const int gx = x0 - 2 + r, gy = y0 - TS::YOFF + c;
    ok[k] = i < TS::PLANE && gx >= 0 && gx < G.X && gy >= 0 && gy < G.Y;
    off[k] = (long long)gx * G.Y + gy;
  }
#pragma unroll
  for (int a = 0; a < NF; ++a) {
    R p[KM], v[KM], w[KM];
    const long long base = (long long)a * N;
#pragma unroll
    for (int k = 0; k < KM; ++k) {
      p[k] = ok[k] ? psrc[base + off[k]] : (R)0;
      v[k] = (ok[k] && vsrc) ? vsrc[base + off[k]] : (R)0;
      w[k] = (ok[k] && wsrc) ? wsrc[base + off[k]] : (R)0;
    }
#pragma unroll
    for (int k = 0; k < KM; ++k) {
      const int i = threadIdx.x + k * NT;
      if (i < TS::PLANE) T[a * TS::PLANE + i] = stage_value<R>(mode, p[k], v[k], w[k], dt);
    }
  }
}

// Plain-load staging of T_s into T (T4, stored by stage 3, in S4)
template <int NF, typename R, int TX, int TY, int NT>
__device__ inline void stage_plain(R* T, const FlowArgs<R>& A, int x0, int y0, int mode, bool arrest) {
  const bool need_v = (mode == M_S2 || mode == M_S3) && !arrest;
  stage_plain_buf<NF, R, TX, TY, NT>(T, A.G, A.phi, need_v ? A.vel : nullptr, mode == M_S3 ? A.la : nullptr, x0, y0,
                                     mode);
}

// The unit-norm re-projection of a site pair's magnetisation components
// (compute_norm_magnetization, chiral_magnet/kernels.py:48-84): m / |m| where |m| > 0.
template <int NMAG, typename V>
__device__ __forceinline__ void unit_project(V* m) {
  using S = typename ScalarOf<V>::type;
  V s2 = m[0] * m[0];
#pragma unroll
  for (int a = 1; a < NMAG; ++a) s2 = vfma(m[a], m[a], s2);
  V inv(1.0);
#pragma unroll
  for (int l = 0; l < 2; ++l) {
    const S s = sqrt(Lanes<V>::get(s2, l));
    if (s != (S)0) Lanes<V>::set(inv, l, (S)1 / s);
  }
#pragma unroll
  for (int a = 0; a < NMAG; ++a) m[a] = m[a] * inv;
}

// Stencil weights pre-scaled by the lattice spacings, as broadcast pairs.
template <typename V>
struct PairCoef {
  using S = typename ScalarOf<V>::type;
  V c23hx, mc12hx, c43hx2, mc12hx2, c23hy, mc12hy, c43hy2, mc12hy2, c43hd, mc12hd;
  __device__ explicit PairCoef(const Grid& G)
      : c23hx(grid_k<S>(G, GK_C23HX)), mc12hx(grid_k<S>(G, GK_MC12HX)), c43hx2(grid_k<S>(G, GK_C43HX2)),
        mc12hx2(grid_k<S>(G, GK_MC12HX2)), c23hy(grid_k<S>(G, GK_C23HY)), mc12hy(grid_k<S>(G, GK_MC12HY)),
        c43hy2(grid_k<S>(G, GK_C43HY2)), mc12hy2(grid_k<S>(G, GK_MC12HY2)), c43hd(grid_k<S>(G, GK_C43HD)),
        mc12hd(grid_k<S>(G, GK_MC12HD)) {}
};

// Unmasked jet of one component for the site pair (x, y), (x, y+1) whose centre
// pair starts at `row` in the staged tile (rows HY apart).  Difference form as in
// d1_stencil / d2_stencil; Dx1 = f(x+1)-f(x-1), Dx2 = f(x+2)-f(x-2) and the y
// analogues are returned for the FP64 energy.
template <typename V, typename R, int HY, bool XY>
__device__ __forceinline__ void pair_jet(const R* row, const PairCoef<V>& k, V& f, V& dx, V& dy, V& dxx, V& dyy,
                                         V& dxy, V& Dx1, V& Dx2, V& Dy1, V& Dy2) {
  const V A = ld_pair(row - 2), B = ld_pair(row), C = ld_pair(row + 2);
  const V xm1 = ld_pair(row - HY), xp1 = ld_pair(row + HY);
  const V xm2 = ld_pair(row - 2 * HY), xp2 = ld_pair(row + 2 * HY);
  const V ym1 = shift1(A, B), yp1 = shift1(B, C);
  f = B;
  Dx1 = xp1 - xm1;
  Dx2 = xp2 - xm2;
  Dy1 = yp1 - ym1;
  Dy2 = C - A;
  dx = vfma(Dx1, k.c23hx, Dx2 * k.mc12hx);
  dy = vfma(Dy1, k.c23hy, Dy2 * k.mc12hy);
  dxx = vfma((xp1 - B) + (xm1 - B), k.c43hx2, ((xp2 - B) + (xm2 - B)) * k.mc12hx2);
  dyy = vfma((yp1 - B) + (ym1 - B), k.c43hy2, ((C - B) + (A - B)) * k.mc12hy2);
  if constexpr (XY) {
    // main diagonal (x+k, y+k), soliton_solver/core/derivatives.py:105-112
    const V dp1 = shift1(xp1, ld_pair(row + HY + 2));
    const V dp2 = ld_pair(row + 2 * HY + 2);
    const V dm1 = shift1(ld_pair(row - HY - 2), xm1);
    const V dm2 = ld_pair(row - 2 * HY - 2);
    const V diag = vfma((dp1 - B) + (dm1 - B), k.c43hd, ((dp2 - B) + (dm2 - B)) * k.mc12hd);
    dxy = vfma(dxx, V(-0.5), vfma(dyy, V(-0.5), diag));
  } else {
    dxy = V(0.0);
  }
}

template <typename V>
__device__ __forceinline__ V mask_lanes(V v, bool m0, bool m1) {
  using S = typename ScalarOf<V>::type;
  if (!m0) Lanes<V>::set(v, 0, (S)0);
  if (!m1) Lanes<V>::set(v, 1, (S)0);
  return v;
}

// global pair load / store; `fast` pairs are aligned and both in range
template <typename V, typename R>
__device__ __forceinline__ V gload(const R* p, bool fast, bool v1) {
  using S = typename ScalarOf<V>::type;
  if (fast) return ld_pair(p);
  V r(0.0);
  Lanes<V>::set(r, 0, (S)p[0]);
  if (v1) Lanes<V>::set(r, 1, (S)p[1]);
  return r;
}
template <typename V, typename R>
__device__ __forceinline__ void gstore(R* p, V v, bool fast, bool v1) {
  if (fast) {
    st_pair(p, v);
    return;
  }
  p[0] = Lanes<V>::get(v, 0);
  if (v1) p[1] = Lanes<V>::get(v, 1);
}

// Stored value -> FP64 for the energy stencil.  For FP32 the float's bits are placed
// in a double without re-biasing the exponent (two ALU ops and a shift instead of an
// F2F conversion, which issues on the narrow XU pipe): the result is x * 2^-896
// exactly for zero, normal and subnormal x (2^-126 * 2^-896 = 2^-1022, the smallest
// normal double).  Derivative coefficients carry the factor 2^896 back and centre
// values are multiplied by it, both exact, so every derivative and density is
// bitwise what an F2F conversion gives.  Inf/NaN map to finite values here; the
// caller folds v * 0 of every centre value into a sentinel instead.
template <typename E>
struct ScaledValue {
  static constexpr double SCALE = 1.0;
  __device__ static __forceinline__ double get(E x) { return (double)x; }
};
template <>
struct ScaledValue<float> {
  static constexpr double SCALE = 0x1p896;
  __device__ static __forceinline__ double get(float x) {
    const int u = __float_as_int(x);
    return __hiloint2double((u >> 3) & (int)0x8fffffff, u << 29);
  }
};

// FP64 energy of an FP32 site pair from the jets the gradient stencil already built
// (f, dx, dy after masking): the theory's energy point evaluated in FP64 on the
// converted jets, so a flow stage pays no second stencil for its energy.  The jets
// carry FP32 rounding (~1e-7 relative per site), the precision the flow's gradient
// has.  `chk` folds v * 0 of every jet value (Inf/NaN -> NaN, see ScaledValue).
template <class TH, typename V, int NF>
__device__ __forceinline__ double jet_energy(const Jet<V, NF>& J, const Phys& P, double dA, bool v1, V& chk) {
  using SV = ScaledValue<float>;
  Jet1<double, NF> J0, J1;
#pragma unroll
  for (int a = 0; a < NF; ++a) {
    chk = vfma(J.f[a], V(0.0f), chk);
    chk = vfma(J.dx[a], V(0.0f), chk);
    chk = vfma(J.dy[a], V(0.0f), chk);
    J0.f[a] = SV::get(Lanes<V>::get(J.f[a], 0)) * SV::SCALE;
    J1.f[a] = SV::get(Lanes<V>::get(J.f[a], 1)) * SV::SCALE;
    J0.dx[a] = SV::get(Lanes<V>::get(J.dx[a], 0)) * SV::SCALE;
    J1.dx[a] = SV::get(Lanes<V>::get(J.dx[a], 1)) * SV::SCALE;
    J0.dy[a] = SV::get(Lanes<V>::get(J.dy[a], 0)) * SV::SCALE;
    J1.dy[a] = SV::get(Lanes<V>::get(J.dy[a], 1)) * SV::SCALE;
  }
  double e = TH::energy(J0, P, dA);
  if (v1) e += TH::energy(J1, P, dA);
  return e;
}

// Jet of every component of the site pair whose centre starts at `toff` in the staged
// halo buffer T (NF planes of PLANE values), with the derivative masks applied.
template <class TH, typename V, typename R, int HY, int PLANE, bool FAST>
__device__ __forceinline__ void tile_jet(const R* T, int toff, const PairCoef<V>& kc, const Masks& m0, const Masks& m1,
                                         Jet<V, TH::NF>& J) {
#pragma unroll
  for (int a = 0; a < TH::NF; ++a) {
    V Dx1, Dx2, Dy1, Dy2;
    pair_jet<V, R, HY, TH::NEED_XY>(T + a * PLANE + toff, kc, J.f[a], J.dx[a], J.dy[a], J.dxx[a], J.dyy[a], J.dxy[a],
                                    Dx1, Dx2, Dy1, Dy2);
    if (!FAST) {
      J.dx[a] = mask_lanes(J.dx[a], m0.x, m1.x);
      J.dy[a] = mask_lanes(J.dy[a], m0.y, m1.y);
      J.dxx[a] = mask_lanes(J.dxx[a], m0.x, m1.x);
      J.dyy[a] = mask_lanes(J.dyy[a], m0.y, m1.y);
      J.dxy[a] = mask_lanes(J.dxy[a], m0.xy, m1.xy);
    }
  }
}

// The flow's constraints on a site pair's gradient rows: zero on the frozen ring
// (theories with HALO_ZERO) and the tangent projection g - (g . m) m
// (project_orthogonal_magnetization, chiral_magnet/kernels.py:86-122).
template <class TH, typename V, bool FAST>
__device__ __forceinline__ void flow_constraints(const Grid& G, const Jet<V, TH::NF>& J, V* g, int gx, int gy) {
  if (TH::HALO_ZERO && !FAST) {
    const bool e0 = gx < G.halo || gx > G.X - G.halo - 1 || gy < G.halo || gy > G.Y - G.halo - 1;
    const bool e1 = gx < G.halo || gx > G.X - G.halo - 1 || gy + 1 < G.halo || gy + 1 > G.Y - G.halo - 1;
#pragma unroll
    for (int a = 0; a < TH::NF; ++a) g[a] = mask_lanes(g[a], !e0, !e1);
  }
  if (TH::CONSTRAINED) {
    V lm = g[0] * J.f[0];
#pragma unroll
    for (int a = 1; a < TH::NMAG; ++a) lm = vfma(g[a], J.f[a], lm);
    const V mlm = -lm;
#pragma unroll
    for (int a = 0; a < TH::NMAG; ++a) g[a] = vfma(mlm, J.f[a], g[a]);
  }
}

// The per-site work of one staged tile.  Each thread owns y-adjacent site pairs;
// FAST: the tile is interior (every derivative mask true, no halo site) and the
// lattice row length is even, so pairs are aligned and need no lane masks.
//   T      the staged stencil field: T1 (S1, M_GRAD, M_ENERGY), T2 (S2), T3 (S3, M_S23), T4 (S4)
//   T2     M_S23: the staged T2 (l2 and l3 of a pair are computed in one pass)
//   Praw   S3 / M_S23: the staged phi (else phi is read from A.phi)
//   Vraw   S3: the staged V (else V is read from A.vel); unused when arrested
//   Cp, Cv S4: the staged cP and cV centre tiles (else read from A.cp, A.cv)
// JE (FP32 stage 1 and the energy pass): add the energy of the jets to *e_acc (when
// non-null); in M_ENERGY the gradient itself is skipped.
template <class TH, typename R, int TX, int TY, int NT, bool FAST, int MODE, bool JE = false>
__device__ __forceinline__ void grad_tile(const FlowArgs<R>& A, const R* T, int x0, int y0, bool arrest,
                                          double& err_max, double* e_acc = nullptr, const R* Praw = nullptr,
                                          const R* Vraw = nullptr, const R* T2 = nullptr, const R* Cp = nullptr,
                                          const R* Cv = nullptr, R* out_l = nullptr) {
  using TS = TileShape<TX, TY, NT>;
  using V = typename PairOf<R>::type;
  constexpr int NF = TH::NF;
  constexpr int PAIRS = TY / 2;
  constexpr int RPP = NT / PAIRS;
  static_assert(NT % PAIRS == 0 && TX % RPP == 0, "pair mapping");
  using S = typename ScalarOf<V>::type;
  const Grid& G = A.G;
  const long long N = G.N;
  const PairCoef<V> kc(G);
  const V mdt(grid_k<S>(G, GK_MDT));
  S emax = -INFINITY;
  V chk(0.0);
  double e_pair = 0.0;
  const int j = threadIdx.x % PAIRS;
  const int lxg = threadIdx.x / PAIRS;
  // stage 1 and the FP32 energy pass give each thread adjacent rows; the energy pass
  // unrolls them so that the rows share their x-neighbour loads
  constexpr bool ADJ = sizeof(R) == 4 && (MODE == M_S1 || MODE == M_ENERGY);
#pragma unroll((JE && MODE == M_ENERGY) ? 2 : 1)
  for (int pass = 0; pass < TX / RPP; ++pass) {
    const int lx = ADJ ? lxg * (TX / RPP) + pass : lxg + pass * RPP;
    const int gx = x0 + lx, gy = y0 + 2 * j;
    bool v1 = true;
    Masks m0{true, true, true}, m1{true, true, true};
    if (!FAST) {
      if (gx >= G.X || gy >= G.Y) continue;
      v1 = gy + 1 < G.Y;
      m0 = site_masks(G, gx, gy);
      m1 = site_masks(G, gx, gy + 1);
      if (!v1) m1 = Masks{false, false, false};
    }
    const int toff = (lx + 2) * TS::HY + TS::YOFF + 2 * j;
    const long long sidx = (long long)gx * G.Y + gy;
    // M_S23: the pair's V and l1 (overwritten by T2 and T3 in shared memory) come back
    // from L2; issued before the two stencils so that their latency hides behind them
    // (FP32, up to four components: the six of the s+id model, and FP64 pairs, would spill)
    constexpr bool PRE = MODE == M_S23 && NF <= 4 && sizeof(R) == 4;
    constexpr int NPRE = PRE ? NF : 1;
    V pre_v[NPRE], pre_l1[NPRE];
    if constexpr (PRE) {
#pragma unroll
      for (int a = 0; a < NF; ++a) {
        pre_v[a] = arrest ? V(0.0) : gload<V, R>(A.vel + a * N + sidx, FAST, v1);
        pre_l1[a] = gload<V, R>(A.la + a * N + sidx, FAST, v1);
      }
    }
    // S4 one tile per CTA (FP32, up to four components): cP and cV likewise, where they are
    // not staged
    constexpr bool PRE4 = MODE == M_S4 && sizeof(R) == 4 && NF <= 4;
    V pre_cp[PRE4 ? NF : 1], pre_cv[PRE4 ? NF : 1];
    if constexpr (PRE4) {
#pragma unroll
      for (int a = 0; a < NF; ++a) {
        if (!Cp) pre_cp[a] = gload<V, R>(A.cp + a * N + sidx, FAST, v1);
        if (!Cv) pre_cv[a] = gload<V, R>(A.cv + a * N + sidx, FAST, v1);
      }
    }

    Jet<V, NF> J;
    tile_jet<TH, V, R, TS::HY, TS::PLANE, FAST>(T, toff, kc, m0, m1, J);
    if constexpr (JE) {
      if (e_acc) {
        if constexpr (TH::PAIR_ENERGY) {
          // energy point in packed FP32; F2F keeps Inf/NaN
          const V ep = TH::energy_pair(J, A.P);
          e_pair += (double)Lanes<V>::get(ep, 0);
          if (v1) e_pair += (double)Lanes<V>::get(ep, 1);
        } else {
          *e_acc += jet_energy<TH, V, NF>(J, A.P, G.dA, v1, chk);
        }
      }
    }
    if constexpr (MODE == M_ENERGY) continue;

    // FP64 fields: a fixed field added to the flow's gradient rows (ss_set_forcing); uniform
    auto add_force = [&](V* g) {
      if constexpr (sizeof(R) == 8 && MODE != M_GRAD) {
        if (A.force) {
          V fo[NF];
#pragma unroll
          for (int a = 0; a < NF; ++a) fo[a] = gload<V, double>(A.force + a * N + sidx, FAST, v1);
          TH::flow_rows(fo, A.P);
#pragma unroll
          for (int a = 0; a < NF; ++a) g[a] = g[a] + fo[a];
        }
      }
    };
    V g[NF];
    TH::gradient(J, A.P, g);
    add_force(g);
    if constexpr (MODE == M_GRAD) {
      if (A.grad_raw) {
        // functional derivative of the energy: no halo zeroing, no projection, and
        // rows the flow stores scaled (saddle fields) converted to dE/dphi
        TH::true_rows(g, A.P);
#pragma unroll
        for (int a = 0; a < NF; ++a) {
          if (A.out_eg) gstore<V, R>(A.out_eg + a * N + sidx, g[a], FAST, v1);
        }
        continue;
      }
    }
    flow_constraints<TH, V, FAST>(G, J, g, gx, gy);
    if constexpr (MODE == M_GRAD) {
#pragma unroll
      for (int a = 0; a < NF; ++a) {
        if (A.out_eg) gstore<V, R>(A.out_eg + a * N + sidx, g[a], FAST, v1);
        if (A.out_l) gstore<V, R>(A.out_l + a * N + sidx, mdt * g[a], FAST, v1);
      }
    } else if constexpr (MODE == M_S1 || MODE == M_S2) {
      R* const lo = out_l ? out_l : A.out_l;
#pragma unroll
      for (int a = 0; a < NF; ++a) gstore<V, R>(lo + a * N + sidx, mdt * g[a], FAST, v1);
    } else if constexpr (MODE == M_S3 || MODE == M_S23) {
      // l3 from T3; l2 from T2 (M_S23) or the stored l2 (S3); then the stage-4 inputs
      // T4 = phi + dt (V + l2/2), cV = V + (l1 + 2 l2 + 2 l3)/6, cP = phi + dt V + dt (l1 + l2 + l3)/6
      // (core/integrator.py:151-189 with k1 = dt V, k2 = dt (V + l1/2), k3 = dt (V + l2/2))
      V l2[NF];
      if constexpr (MODE == M_S23) {
        Jet<V, NF> J2;
        tile_jet<TH, V, R, TS::HY, TS::PLANE, FAST>(T2, toff, kc, m0, m1, J2);
        TH::gradient(J2, A.P, l2);
        add_force(l2);
        flow_constraints<TH, V, FAST>(G, J2, l2, gx, gy);
#pragma unroll
        for (int a = 0; a < NF; ++a) l2[a] = mdt * l2[a];
      } else {
#pragma unroll
        for (int a = 0; a < NF; ++a) l2[a] = gload<V, R>(A.lb + a * N + sidx, FAST, v1);
      }
      const V half(0.5), sixth(grid_k<S>(G, GK_SIXTH)), two(2.0), dtv(grid_k<S>(G, GK_DT)),
          dt6(grid_k<S>(G, GK_DT6));
#pragma unroll
      for (int a = 0; a < NF; ++a) {
        const long long idx = a * N + sidx;
        const V p = Praw ? ld_pair(Praw + a * TS::PLANE + toff) : gload<V, R>(A.phi + idx, FAST, v1);
        V v, l1;
        if constexpr (PRE) {
          v = pre_v[a];
          l1 = pre_l1[a];
        } else {
          v = arrest ? V(0.0) : (Vraw ? ld_pair(Vraw + a * TS::PLANE + toff) : gload<V, R>(A.vel + idx, FAST, v1));
          l1 = gload<V, R>(A.la + idx, FAST, v1);
        }
        const V l3 = mdt * g[a];
        gstore<V, R>(A.out_t4 + idx, vfma(dtv, vfma(half, l2[a], v), p), FAST, v1);
        gstore<V, R>(A.out_cv + idx, vfma(sixth, vfma(two, l3, vfma(two, l2[a], l1)), v), FAST, v1);
        gstore<V, R>(A.out_cp + idx, vfma(dt6, (l1 + l2[a]) + l3, vfma(dtv, v, p)), FAST, v1);
      }
    } else {
      // S4: V' = cV + l4/6 and phi' = cP, re-projected onto the sphere, then V' projected
      // onto the tangent space of phi' (compute_norm_magnetization and
      // project_orthogonal_magnetization, chiral_magnet/kernels.py:48-122)
      V Pn[NF], Vn[NF];
      const V sixth(grid_k<S>(G, GK_SIXTH));
#pragma unroll
      for (int a = 0; a < NF; ++a) {
        const int coff = a * TX * TY + lx * TY + 2 * j;
        V cv;
        if constexpr (PRE4) {
          cv = Cv ? ld_pair(Cv + coff) : pre_cv[a];
          Pn[a] = Cp ? ld_pair(Cp + coff) : pre_cp[a];
        } else {
          cv = Cv ? ld_pair(Cv + coff) : gload<V, R>(A.cv + a * N + sidx, FAST, v1);
          Pn[a] = Cp ? ld_pair(Cp + coff) : gload<V, R>(A.cp + a * N + sidx, FAST, v1);
        }
        Vn[a] = vfma(sixth, mdt * g[a], cv);
        emax = fmax(emax, Lanes<V>::get(g[a], 0));
        if (v1) emax = fmax(emax, Lanes<V>::get(g[a], 1));
      }
      if (TH::CONSTRAINED && G.unit_mag) {
        unit_project<TH::NMAG>(Pn);
        V lm = Vn[0] * Pn[0];
#pragma unroll
        for (int a = 1; a < TH::NMAG; ++a) lm = vfma(Vn[a], Pn[a], lm);
        const V mlm = -lm;
#pragma unroll
        for (int a = 0; a < TH::NMAG; ++a) Vn[a] = vfma(mlm, Pn[a], Vn[a]);
      }
#pragma unroll
      for (int a = 0; a < NF; ++a) {
        gstore<V, R>(A.phi_out + a * N + sidx, Pn[a], FAST, v1);
        gstore<V, R>(A.vel_out + a * N + sidx, Vn[a], FAST, v1);
      }
    }
  }
  if (MODE == M_S4) err_max = fmax(err_max, (double)emax);
  if constexpr (JE) {
    if (e_acc) *e_acc += e_pair * G.dA + (double)(Lanes<V>::get(chk, 0) + Lanes<V>::get(chk, 1));
  }
}

// FP64 energy of the staged field (T_1 = phi): first derivatives from the exact
// differences f(x+k) - f(x-k) of the stored values, evaluated in FP64.
template <class TH, typename R, int TX, int TY, int NT, bool FAST, typename E = R>
__device__ __forceinline__ double energy_tile(const FlowArgs<R>& A, const E* T, int x0, int y0) {
  using TS = TileShape<TX, TY, NT>;
  using V = typename PairOf<E>::type;
  using SV = ScaledValue<E>;
  constexpr int NF = TH::NF;
  constexpr int PAIRS = TY / 2;
  constexpr int RPP = NT / PAIRS;
  const Grid& G = A.G;
  const double c23x = FD::c23 * G.ihx * SV::SCALE, c12x = FD::c12 * G.ihx * SV::SCALE;
  const double c23y = FD::c23 * G.ihy * SV::SCALE, c12y = FD::c12 * G.ihy * SV::SCALE;
  const int j = threadIdx.x % PAIRS;
  const int lxg = threadIdx.x / PAIRS;
  double e_acc = 0.0;
  V chk(0.0f);  // stays zero unless a centre value is Inf or NaN
#pragma unroll 1
  for (int pass = 0; pass < TX / RPP; ++pass) {
    const int lx = lxg + pass * RPP;
    const int gx = x0 + lx, gy = y0 + 2 * j;
    bool v1 = true;
    Masks m0{true, true, true}, m1{true, true, true};
    if (!FAST) {
      if (gx >= G.X || gy >= G.Y) continue;
      v1 = gy + 1 < G.Y;
      m0 = site_masks(G, gx, gy);
      m1 = site_masks(G, gx, gy + 1);
    }
    const int toff = (lx + 2) * TS::HY + TS::YOFF + 2 * j;
    Jet1<double, NF> J0, J1;
#pragma unroll
    for (int a = 0; a < NF; ++a) {
      const E* row = T + a * TS::PLANE + toff;
      // six y values cover both sites' y stencils; converted once
      const V Ap = ld_pair(row - 2), B = ld_pair(row), C = ld_pair(row + 2);
      chk = vfma(B, V(0.0f), chk);
      const double y_2 = SV::get(Lanes<V>::get(Ap, 0)), y_1 = SV::get(Lanes<V>::get(Ap, 1));
      const double y0v = SV::get(Lanes<V>::get(B, 0)), y1v = SV::get(Lanes<V>::get(B, 1));
      const double y2 = SV::get(Lanes<V>::get(C, 0)), y3 = SV::get(Lanes<V>::get(C, 1));
      const V xp1 = ld_pair(row + TS::HY), xm1 = ld_pair(row - TS::HY);
      const V xp2 = ld_pair(row + 2 * TS::HY), xm2 = ld_pair(row - 2 * TS::HY);
#pragma unroll
      for (int l = 0; l < 2; ++l) {
        Jet1<double, NF>& J = l ? J1 : J0;
        const Masks& m = l ? m1 : m0;
        const double ddx = (c23x * (SV::get(Lanes<V>::get(xp1, l)) - SV::get(Lanes<V>::get(xm1, l))) -
                            c12x * (SV::get(Lanes<V>::get(xp2, l)) - SV::get(Lanes<V>::get(xm2, l))));
        const double ddy = l ? (c23y * (y2 - y0v) - c12y * (y3 - y_1)) : (c23y * (y1v - y_1) - c12y * (y2 - y_2));
        J.f[a] = (l ? y1v : y0v) * SV::SCALE;
        J.dx[a] = m.x ? ddx : 0.0;
        J.dy[a] = m.y ? ddy : 0.0;
      }
    }
    e_acc += TH::energy(J0, A.P, G.dA);
    if (v1) e_acc += TH::energy(J1, A.P, G.dA);
  }
  return e_acc + (double)(Lanes<V>::get(chk, 0) + Lanes<V>::get(chk, 1));
}

// Expect and issue the TMA loads of one tile's staged halo buffers (called by one
// thread, after the barrier is initialised): tm_phi into B0 (phi; T4 in S4), then V
// into B0 + BUF in S2, S3 and M_S23 and l1 into B0 + 2 BUF in S3 and M_S23.  V is
// staged whether or not an arrest is pending (an arrested step ignores it).
template <class TH, typename R, int TX, int TY, int NT, int MODE>
__device__ __forceinline__ void issue_tile(R* B0, const CUtensorMap* tm_phi, const CUtensorMap* tm_vel,
                                           const CUtensorMap* tm_l, int x0, int y0, uint64_t* bar,
                                           unsigned tx_extra) {
  using TS = TileShape<TX, TY, NT>;
  constexpr int BUF = TH::NF * TS::PLANE;
  constexpr int NB = flow_buffers(MODE);
  constexpr uint32_t bytes = (uint32_t)(sizeof(R) * BUF) * (uint32_t)NB;
  mbar_expect_tx(bar, bytes + tx_extra);
  tma_load_3d(B0, tm_phi, y0 - TS::YOFF, x0 - 2, 0, bar);
  if constexpr (NB >= 2) tma_load_3d(B0 + BUF, tm_vel, y0 - TS::YOFF, x0 - 2, 0, bar);
  if constexpr (NB >= 3) tma_load_3d(B0 + 2 * BUF, tm_l, y0 - TS::YOFF, x0 - 2, 0, bar);
}

// Shared scratch of the one-tile-per-CTA stage kernels besides the staged tile.
template <int NT>
struct StageShared {
  double red[NT / 32];
  double sh_s[NT], sh_c[NT];
  uint64_t bar;
  int am_last;
};

// Stage, compute and reduce tile `tile` of a lattice of `nblk` tiles (one CTA per
// tile).  tm_phi / tm_vel / tm_l are TMA maps in parameter or global memory.
// issued: thread 0 has already initialised S.bar and issued the tile's loads
// (issue_tile), so the caller's set-up overlapped them.
template <class TH, typename R, int TX, int TY, int NT, bool TMA, int MODE>
__device__ __forceinline__ void flow_tile(const FlowArgs<R>& A, const CUtensorMap* tm_phi, const CUtensorMap* tm_vel,
                                          const CUtensorMap* tm_l, int tile, int nblk, unsigned char* smem_raw,
                                          StageShared<NT>& S, bool issued = false) {
  using TS = TileShape<TX, TY, NT>;
  constexpr int NF = TH::NF;
  constexpr int BUF = NF * TS::PLANE;
  R* B0 = reinterpret_cast<R*>(smem_raw);
  R* B1 = B0 + BUF;
  R* B2 = B1 + BUF;
  double* red = S.red;
  double* sh_s = S.sh_s;
  double* sh_c = S.sh_c;
  uint64_t& bar = S.bar;
  int& am_last = S.am_last;

  const Grid& G = A.G;
  const int tiles_y = (G.Y + TY - 1) / TY;
  const int x0 = (tile / tiles_y) * TX;
  const int y0 = (tile % tiles_y) * TY;
  StepState* st = A.st;
  constexpr bool uses_v = MODE == M_S2 || MODE == M_S3 || MODE == M_S23;
  // The arrest flag (set by the last block of stage 1) is read only after the TMA
  // copies are issued, so its global-memory round trip overlaps them.
  bool arrest = false;
  const bool do_energy = (MODE == M_S1 || MODE == M_ENERGY) && A.with_energy != 0;

  if (A.init_state && tile == 0 && threadIdx.x == 0) {
    st->arrest = 0;
    if (!isnan(A.prev_energy)) st->E_last = A.prev_energy;
  }

  // ---- stage the halo tiles --------------------------------------------
  R* T = B0;
  if constexpr (TMA) {
    if (!issued) {
      if (threadIdx.x == 0) mbar_init(&bar, 1);
      __syncthreads();
      if (threadIdx.x == 0) issue_tile<TH, R, TX, TY, NT, MODE>(B0, tm_phi, tm_vel, tm_l, x0, y0, &bar, A.tx_extra);
    }
    if constexpr (uses_v) arrest = st->arrest != 0;
    const bool ok = __syncthreads_and(mbar_wait_bounded(&bar, 0, A.wait_cycles));
    if (!ok) {
      if (threadIdx.x == 0) atomicExch(&st->status, (int)ST_TIMEOUT);
      mbar_wait_bounded(&bar, 0, A.wait_cycles);
      return;
    }
    using V = typename PairOf<R>::type;
    const V half(0.5), hdt(grid_k<R>(G, GK_HDT));
    if constexpr (MODE == M_S23) {
      // T3 = phi + dt/2 (V + l1/2) in place of l1 and T2 = phi + dt/2 V in place of V, in
      // one pass (each element reads its own phi, V, l1 before writing)
      for (int i = 4 * threadIdx.x; i < BUF; i += 4 * NT) {
        V p0, p1, v0(0.0), v1(0.0), w0, w1;
        ld_quad(B0 + i, p0, p1);
        if (!arrest) ld_quad(B1 + i, v0, v1);
        ld_quad(B2 + i, w0, w1);
        st_quad(B2 + i, vfma(hdt, vfma(half, w0, v0), p0), vfma(hdt, vfma(half, w1, v1), p1));
        st_quad(B1 + i, vfma(hdt, v0, p0), vfma(hdt, v1, p1));
      }
      __syncthreads();
    } else if constexpr (MODE == M_S2 || MODE == M_S3) {
      // T2 in place of V, or T3 in place of l1 (OOB entries are zero in all)
      R* dst = MODE == M_S3 ? B2 : B1;
      for (int i = 4 * threadIdx.x; i < BUF; i += 4 * NT) {
        V p0, p1, v0(0.0), v1(0.0), w0(0.0), w1(0.0);
        ld_quad(B0 + i, p0, p1);
        if (!arrest) ld_quad(B1 + i, v0, v1);
        if (MODE == M_S3) ld_quad(B2 + i, w0, w1);
        if (MODE == M_S2)
          st_quad(dst + i, vfma(hdt, v0, p0), vfma(hdt, v1, p1));
        else
          st_quad(dst + i, vfma(hdt, vfma(half, w0, v0), p0), vfma(hdt, vfma(half, w1, v1), p1));
      }
      __syncthreads();
      T = dst;
    }
  } else {
    if constexpr (uses_v) arrest = st->arrest != 0;
    stage_plain<NF, R, TX, TY, NT>(B0, A, x0, y0, MODE, arrest);
    __syncthreads();
  }

  double e_acc = 0.0;
  double err_max = -INFINITY;
  const bool fast = (G.Y % 2 == 0) && x0 >= G.halo + 1 && x0 + TX - 1 <= G.X - G.halo - 2 && y0 >= G.halo + 1 &&
                    y0 + TY - 1 <= G.Y - G.halo - 2;
  if constexpr (MODE == M_S23) {
    // l3 from T3 (staged in B2) and l2 from T2 (staged in B1) per site pair, then the
    // stage-4 inputs: the stage-2 and stage-3 arithmetic, so the results equal the two
    // separate stages bitwise
    if (fast)
      grad_tile<TH, R, TX, TY, NT, true, M_S23>(A, B2, x0, y0, arrest, err_max, nullptr, B0, nullptr, B1);
    else
      grad_tile<TH, R, TX, TY, NT, false, M_S23>(A, B2, x0, y0, arrest, err_max, nullptr, B0, nullptr, B1);
    return;
  } else if constexpr (MODE == M_S1 || MODE == M_ENERGY) {
    // FP32 fields: the flow energy from the stencil's jets (stage 1 and the trailing
    // pass), or (observables) the exact FP64 differences of the stored values; FP64
    // fields: the exact differences
    constexpr bool JE = sizeof(R) == 4;
    const bool je = JE && !(MODE == M_ENERGY && A.exact_energy);
    double* ep = (je && do_energy) ? &e_acc : nullptr;
    if (MODE == M_S1 || je) {
      if (fast)
        grad_tile<TH, R, TX, TY, NT, true, MODE, JE>(A, T, x0, y0, false, err_max, ep);
      else
        grad_tile<TH, R, TX, TY, NT, false, MODE, JE>(A, T, x0, y0, false, err_max, ep);
    }
    if (do_energy && !je) {
      if (fast)
        e_acc = energy_tile<TH, R, TX, TY, NT, true>(A, T, x0, y0);
      else
        e_acc = energy_tile<TH, R, TX, TY, NT, false>(A, T, x0, y0);
    }
  } else {
    // S2, S3, S4, M_GRAD; stage 3 combines with the staged phi and V (TMA staging)
    const R* Praw = (TMA && MODE == M_S3) ? B0 : nullptr;
    const R* Vraw = (TMA && MODE == M_S3) ? B1 : nullptr;
    if (fast)
      grad_tile<TH, R, TX, TY, NT, true, MODE>(A, T, x0, y0, arrest, err_max, nullptr, Praw, Vraw);
    else
      grad_tile<TH, R, TX, TY, NT, false, MODE>(A, T, x0, y0, arrest, err_max, nullptr, Praw, Vraw);
  }

  // ---- reductions -------------------------------------------------------
  const bool need_ticket = do_energy || MODE == M_S4;
  if (!need_ticket) return;
  if (do_energy) {
    const double bs = block_sum_fixed<NT>(e_acc, red);
    if (threadIdx.x == 0) A.partial[tile] = bs;
  }
  if (MODE == M_S4) {
    const double bm = block_max<NT>(err_max, red);
    if (threadIdx.x == 0 && bm > -INFINITY) atomicMax(&st->err_enc, enc_max(bm));
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned t = atomicAdd(&st->ticket, 1u);
    am_last = (t == (unsigned)nblk - 1u);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  if (do_energy) {
    const double E = fixed_order_sum<NT>(A.partial, nblk, sh_s, sh_c);
    if (threadIdx.x == 0) {
      st->scalar = E;
      if (!isfinite(E)) st->status = 3;
      if (A.E_traj && A.E_idx >= 0) A.E_traj[A.E_idx] = E;
      if (A.arrest_update) {
        st->arrest = (G.killkinen && E > st->E_last) ? 1 : 0;
        st->E_last = E;
      }
    }
  }
  if (threadIdx.x == 0) {
    if (MODE == M_S4) {
      const double err = dec_max(atomicExch(&st->err_enc, 0ULL));
      if (A.err_traj && A.err_idx >= 0) A.err_traj[A.err_idx] = err;
    }
    st->ticket = 0u;
  }
}

// Resident CTAs per SM a one-tile-per-CTA stage kernel is built for (the staging latency
// of a tile is hidden only by other resident CTAs).  The fused FP32 stages 2+3 evaluate
// two stencils per site pair: capped at three 256-thread CTAs (80 registers) for the
// theories with up to four components and at two (128 registers; its 104 KB of staging
// fits two anyway) for the six-component s+id.  FP64 stages 1 and 4 and the energy pass
// (one staged buffer each) at two 256-thread CTAs, 128 registers, up to four components
// (the s+id would spill ~380 bytes).  No bound otherwise.
template <class TH, typename R, int MODE, int NT>
__host__ __device__ constexpr int flow_min_ctas() {
  if (NT != 256) return 1;
  if (sizeof(R) == 4 && MODE == M_S23) return TH::NF <= 4 ? 3 : 2;
  if (sizeof(R) == 8 && (MODE == M_S4 || MODE == M_S1 || MODE == M_ENERGY)) return TH::NF <= 4 ? 2 : 1;
  return 1;
}

template <class TH, typename R, int TX, int TY, int NT, bool TMA, int MODE>
__global__ void __launch_bounds__(NT, (flow_min_ctas<TH, R, MODE, NT>()))
    flow_kernel(const __grid_constant__ FlowArgs<R> A) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ StageShared<NT> S;
  flow_tile<TH, R, TX, TY, NT, TMA, MODE>(A, &A.tm_phi, &A.tm_vel, &A.tm_l, blockIdx.x, gridDim.x, smem_raw, S);
}

// ---------------------------------------------------------------------------
// Persistent, TMA-pipelined form of flow_kernel (FP32 fields): one CTA per SM
// walks the tiles blockIdx.x, blockIdx.x + gridDim.x, ... through a ring of STAGES
// shared-memory slots, so the bulk tensor loads of the next tiles are in flight
// while the current tile is computed.  Stage 4 also stages the centre tiles of cP and cV.
// Energy partials are per CTA in tile order (deterministic for a fixed grid).
// ---------------------------------------------------------------------------
template <int MODE>
__host__ __device__ constexpr int pipe_halo_buffers() {
  return flow_buffers(MODE);
}
template <int MODE>
__host__ __device__ constexpr int pipe_centre_buffers() {
  return MODE == M_S4 ? 2 : 0;
}
template <typename R, int NF, int TX, int TY, int MODE>
__host__ __device__ constexpr size_t pipe_slot_bytes() {
  return tile_buf_bytes<R, NF, TX, TY>() * pipe_halo_buffers<MODE>() +
         sizeof(R) * NF * TX * TY * pipe_centre_buffers<MODE>();
}

// Persistent CTAs per SM: for stage 1 and the energy pass the theory's S1_CTAS (four
// 256-thread CTAs for the light chiral stencil, issue-bound: two site pairs per thread
// per tile halve the per-tile overhead, and four CTAs keep 32 warps per SM), one
// 512-thread CTA otherwise.
template <class TH, int MODE>
__host__ __device__ constexpr int pipe_ctas() {
  return (MODE == M_S1 || MODE == M_ENERGY) ? TH::S1_CTAS : 1;
}
template <class TH, int MODE>
__host__ __device__ constexpr int pipe_threads() {
  return pipe_ctas<TH, MODE>() == 4 ? 256 : 512;
}

template <class TH, typename R, int TX, int TY, int NT, int MODE, int STAGES>
__global__ void __launch_bounds__(NT, (pipe_ctas<TH, MODE>())) flow_kernel_pipe(const __grid_constant__ FlowArgs<R> A) {
  using TS = TileShape<TX, TY, NT>;
  constexpr int NF = TH::NF;
  constexpr int BUF = NF * TS::PLANE;             // elements of one halo buffer
  constexpr int CBUF = NF * TX * TY;              // elements of one centre buffer
  constexpr int SLOT = BUF * pipe_halo_buffers<MODE>() + CBUF * pipe_centre_buffers<MODE>();
  static_assert(MODE != M_S23, "the fused stages 2+3 run one tile per CTA");
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* ring = reinterpret_cast<R*>(smem_raw);
  __shared__ double red[NT / 32];
  __shared__ double sh_s[NT], sh_c[NT];
  __shared__ int am_last;
  __shared__ int timed_out;
  __shared__ __align__(8) uint64_t full[STAGES];

  const Grid& G = A.G;
  const int tiles_y = (G.Y + TY - 1) / TY;
  const int ntiles = ((G.X + TX - 1) / TX) * tiles_y;
  StepState* st = A.st;
  const bool arrest = (MODE == M_S2 || MODE == M_S3) && (st->arrest != 0);
  const bool do_energy = (MODE == M_S1 || MODE == M_ENERGY) && A.with_energy != 0;
  // second halo buffer: V in S2 / S3 (not loaded when arrested)
  const bool load_b1 = (MODE == M_S2 || MODE == M_S3) && !arrest;
  constexpr bool load_b2 = MODE == M_S3;
  const uint32_t bytes = (uint32_t)(sizeof(R) * (BUF * (1 + (load_b1 ? 1 : 0) + (load_b2 ? 1 : 0)) +
                                                 CBUF * pipe_centre_buffers<MODE>()));

  if (A.init_state && blockIdx.x == 0 && threadIdx.x == 0) {
    st->arrest = 0;
    if (!isnan(A.prev_energy)) st->E_last = A.prev_energy;
  }
  auto issue = [&](int slot, int tile) {
    R* base = ring + slot * SLOT;
    const int x0 = (tile / tiles_y) * TX, y0 = (tile % tiles_y) * TY;
    mbar_expect_tx(&full[slot], bytes + A.tx_extra);
    tma_load_3d(base, &A.tm_phi, y0 - TS::YOFF, x0 - 2, 0, &full[slot]);
    if (load_b1) tma_load_3d(base + BUF, &A.tm_vel, y0 - TS::YOFF, x0 - 2, 0, &full[slot]);
    if (load_b2) tma_load_3d(base + 2 * BUF, &A.tm_l, y0 - TS::YOFF, x0 - 2, 0, &full[slot]);
    if (MODE == M_S4) {
      tma_load_3d(base + BUF, &A.tm_cp, y0, x0, 0, &full[slot]);
      tma_load_3d(base + BUF + CBUF, &A.tm_cv, y0, x0, 0, &full[slot]);
    }
  };
  if (threadIdx.x == 0) {
    timed_out = 0;
    for (int s = 0; s < STAGES; ++s) mbar_init(&full[s], 1);
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      const int t = blockIdx.x + s * gridDim.x;
      if (t < ntiles) issue(s, t);
    }
  }

  double e_acc = 0.0;
  double err_max = -INFINITY;
  int k = 0;
  // tile coordinates advanced without a division per tile
  const int dq = gridDim.x / tiles_y, dr = gridDim.x % tiles_y;
  int tx = blockIdx.x / tiles_y, ty = blockIdx.x % tiles_y;
  for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++k) {
    const int slot = k % STAGES;
    const uint32_t parity = (uint32_t)((k / STAGES) & 1);
    const bool ok = __syncthreads_and(mbar_wait_bounded(&full[slot], parity, A.wait_cycles));
    if (!ok) {
      // record, then wait (bounded) for every load still in flight before leaving
      if (threadIdx.x == 0) atomicExch(&st->status, (int)ST_TIMEOUT);
      for (int s = 0; s < STAGES; ++s) {
        const int kk = k + s;
        if (blockIdx.x + kk * gridDim.x < ntiles)
          mbar_wait_bounded(&full[kk % STAGES], (uint32_t)((kk / STAGES) & 1), A.wait_cycles);
      }
      return;
    }
    R* base = ring + slot * SLOT;
    R* B0 = base;
    R* B1 = base + BUF;
    R* B2 = base + 2 * BUF;
    const int x0 = tx * TX, y0 = ty * TY;
    tx += dq;
    ty += dr;
    if (ty >= tiles_y) {
      ty -= tiles_y;
      ++tx;
    }
    R* T = B0;
    if constexpr (MODE == M_S2 || MODE == M_S3) {
      // T2 in place of V, or T3 in place of l1
      R* dst = MODE == M_S3 ? B2 : B1;
      using V = typename PairOf<R>::type;
      const V half(0.5), hdt(grid_k<R>(G, GK_HDT));
      for (int i = 4 * threadIdx.x; i < BUF; i += 4 * NT) {
        V p0, p1, v0(0.0), v1(0.0), w0(0.0), w1(0.0);
        ld_quad(B0 + i, p0, p1);
        if (!arrest) ld_quad(B1 + i, v0, v1);
        if (MODE == M_S3) ld_quad(B2 + i, w0, w1);
        if (MODE == M_S2)
          st_quad(dst + i, vfma(hdt, v0, p0), vfma(hdt, v1, p1));
        else
          st_quad(dst + i, vfma(hdt, vfma(half, w0, v0), p0), vfma(hdt, vfma(half, w1, v1), p1));
      }
      __syncthreads();
      T = dst;
    }
    const bool fast = (G.Y % 2 == 0) && x0 >= G.halo + 1 && x0 + TX - 1 <= G.X - G.halo - 2 &&
                      y0 >= G.halo + 1 && y0 + TY - 1 <= G.Y - G.halo - 2;
    if constexpr (MODE == M_S4) {
      const R* Cp = base + BUF;
      const R* Cv = base + BUF + CBUF;
      if (fast)
        grad_tile<TH, R, TX, TY, NT, true, M_S4>(A, T, x0, y0, false, err_max, nullptr, nullptr, nullptr, nullptr, Cp,
                                                 Cv);
      else
        grad_tile<TH, R, TX, TY, NT, false, M_S4>(A, T, x0, y0, false, err_max, nullptr, nullptr, nullptr, nullptr, Cp,
                                                  Cv);
    } else if constexpr (MODE == M_S1 || MODE == M_ENERGY) {
      constexpr bool JE = sizeof(R) == 4;
      // the four-CTA energy pass is built for the flow energy only (the exact FP64 energy
      // would spill out of its 64 registers); the host sends exact energies to flow_kernel
      constexpr bool EXACT = !(MODE == M_ENERGY && pipe_ctas<TH, MODE>() == 4);
      const bool je = JE && !(MODE == M_ENERGY && EXACT && A.exact_energy);
      double* ep = (je && do_energy) ? &e_acc : nullptr;
      if (MODE == M_S1 || je) {
        if (fast)
          grad_tile<TH, R, TX, TY, NT, true, MODE, JE>(A, T, x0, y0, false, err_max, ep);
        else
          grad_tile<TH, R, TX, TY, NT, false, MODE, JE>(A, T, x0, y0, false, err_max, ep);
      }
      if constexpr (EXACT) {
        if (do_energy && !je) {
          if (fast)
            e_acc += energy_tile<TH, R, TX, TY, NT, true>(A, T, x0, y0);
          else
            e_acc += energy_tile<TH, R, TX, TY, NT, false>(A, T, x0, y0);
        }
      }
    } else {
      const R* Praw = MODE == M_S3 ? B0 : nullptr;
      const R* Vraw = MODE == M_S3 ? B1 : nullptr;
      if (fast)
        grad_tile<TH, R, TX, TY, NT, true, MODE>(A, T, x0, y0, arrest, err_max, nullptr, Praw, Vraw);
      else
        grad_tile<TH, R, TX, TY, NT, false, MODE>(A, T, x0, y0, arrest, err_max, nullptr, Praw, Vraw);
    }
    __syncthreads();  // every thread is done with this slot
    if (threadIdx.x == 0) {
      const int nt = t + STAGES * gridDim.x;
      if (nt < ntiles) issue(slot, nt);
    }
  }

  // ---- reductions (as flow_kernel) ----------------------------------------
  const bool need_ticket = do_energy || MODE == M_S4;
  if (!need_ticket) return;
  if (do_energy) {
    const double bs = block_sum_fixed<NT>(e_acc, red);
    if (threadIdx.x == 0) A.partial[blockIdx.x] = bs;
  }
  if (MODE == M_S4) {
    const double bm = block_max<NT>(err_max, red);
    if (threadIdx.x == 0 && bm > -INFINITY) atomicMax(&st->err_enc, enc_max(bm));
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned tk = atomicAdd(&st->ticket, 1u);
    am_last = (tk == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  if (do_energy) {
    const double E = fixed_order_sum<NT>(A.partial, gridDim.x, sh_s, sh_c);
    if (threadIdx.x == 0) {
      st->scalar = E;
      if (!isfinite(E)) st->status = 3;
      if (A.E_traj && A.E_idx >= 0) A.E_traj[A.E_idx] = E;
      if (A.arrest_update) {
        st->arrest = (G.killkinen && E > st->E_last) ? 1 : 0;
        st->E_last = E;
      }
    }
  }
  if (threadIdx.x == 0) {
    if (MODE == M_S4) {
      const double err = dec_max(atomicExch(&st->err_enc, 0ULL));
      if (A.err_traj && A.err_idx >= 0) A.err_traj[A.err_idx] = err;
    }
    st->ticket = 0u;
  }
}

// Apply a pending arrest (V = 0) left by the trailing energy pass at the end of a call,
// and copy the call's status to status_out (nullable; e.g. mapped host memory).
template <typename R>
__global__ void finish_kernel(R* vel, long long n, const StepState* st, int* status_out) {
  if (status_out && blockIdx.x == 0 && threadIdx.x == 0) *(volatile int*)status_out = st->status;
  if (st->arrest == 0) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    vel[i] = (R)0;
}

// ---------------------------------------------------------------------------
// densities (energy, charges, coupling partials) with optional reduction
// ---------------------------------------------------------------------------
enum DensityKind { D_ENERGY = 0, D_CHARGE = 1, D_COUPLING = 2 };

template <class TH, typename R, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT)
    density_kernel(const R* __restrict__ phi, double* density, double* partial, StepState* st, int kind,
                   int which, Grid G, Phys P) {
  using TS = TileShape<TX, TY, NT>;
  constexpr int NF = TH::NF;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* tile = reinterpret_cast<R*>(smem_raw);
  __shared__ double red[NT / 32];
  __shared__ double sh_s[NT], sh_c[NT];
  __shared__ int am_last;
  const int tiles_y = (G.Y + TY - 1) / TY;
  const int x0 = (blockIdx.x / tiles_y) * TX;
  const int y0 = (blockIdx.x % tiles_y) * TY;
  {
    FlowArgs<R> A;
    A.phi = phi;
    A.G = G;
    stage_plain<NF, R, TX, TY, NT>(tile, A, x0, y0, M_GRAD, false);
  }
  __syncthreads();
  const Inv<double> ivd(G);
  const int ly = threadIdx.x % TY;
  const int lxg = threadIdx.x / TY;
  double acc = 0.0;
#pragma unroll 1
  for (int s = 0; s < TS::SITES_PER_THREAD; ++s) {
    const int lx = lxg + s * TS::ROWS_PER_PASS;
    const int gx = x0 + lx, gy = y0 + ly;
    if (gx >= G.X || gy >= G.Y) continue;
    const Masks mk = site_masks(G, gx, gy);
    const R* base = tile + (lx + 2) * TS::HY + (ly + TS::YOFF);
    Jet1<double, NF> J1;
#pragma unroll
    for (int a = 0; a < NF; ++a) {
      const R* pa = base + a * TS::PLANE;
      auto accs = [pa](int dx, int dy) -> double { return (double)pa[dx * TS::HY + dy]; };
      fill_jet1_comp<double>(accs, mk, ivd, J1.f[a], J1.dx[a], J1.dy[a]);
    }
    double v;
    if (kind == D_ENERGY)
      v = TH::energy(J1, P, G.dA);
    else if (kind == D_CHARGE)
      v = TH::charge(J1, P, which, G.dA);
    else
      v = TH::coupling(J1, P, which, G.dA);
    if (density) density[(long long)gx * G.Y + gy] = v;
    acc += v;
  }
  if (!partial) return;
  const double bs = block_sum_fixed<NT>(acc, red);
  if (threadIdx.x == 0) {
    partial[blockIdx.x] = bs;
    __threadfence();
    const unsigned t = atomicAdd(&st->ticket, 1u);
    am_last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!am_last) return;
  __threadfence();
  const double E = fixed_order_sum<NT>(partial, gridDim.x, sh_s, sh_c);
  if (threadIdx.x == 0) {
    st->scalar = E;
    if (!isfinite(E)) st->status = 3;
    st->ticket = 0u;
  }
}

// do_rk4_step_kernel (core/integrator.py:51-96)
template <typename R>
__global__ void rk4_stage_kernel(R* k_out, const R* vel, const R* l_in, R* temp, const R* phi, const R* k_prev,
                                 R factor, R dt, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const R k = dt * (vel[i] + factor * l_in[i]);
    const R t = phi[i] + factor * k_prev[i];
    k_out[i] = k;
    temp[i] = t;
  }
}

// do_rk4_kernel / do_rk4_kernel_no_constraint (core/integrator.py:99-189)
template <typename R, int NF, int NMAG>
__global__ void rk4_finalize_kernel(R* vel, R* phi, const R* k1, const R* k2, const R* k3, const R* k4, const R* l1,
                                    const R* l2, const R* l3, const R* l4, long long N, int normalize) {
  const R sixth = (R)(1.0 / 6.0), two = (R)2;
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x) {
    R P[NF], V[NF];
#pragma unroll
    for (int a = 0; a < NF; ++a) {
      const long long i = a * N + s;
      V[a] = vel[i] + sixth * (l1[i] + two * l2[i] + two * l3[i] + l4[i]);
      P[a] = phi[i] + sixth * (k1[i] + two * k2[i] + two * k3[i] + k4[i]);
    }
    if (NMAG > 0 && normalize) {
      R s2 = (R)0;
#pragma unroll
      for (int a = 0; a < NMAG; ++a) s2 += P[a] * P[a];
      const R nrm = sqrt(s2);
      if (nrm != (R)0) {
#pragma unroll
        for (int a = 0; a < NMAG; ++a) P[a] /= nrm;
      }
      R lm = (R)0;
#pragma unroll
      for (int a = 0; a < NMAG; ++a) lm += V[a] * P[a];
#pragma unroll
      for (int a = 0; a < NMAG; ++a) V[a] -= lm * P[a];
    }
#pragma unroll
    for (int a = 0; a < NF; ++a) {
      vel[a * N + s] = V[a];
      phi[a * N + s] = P[a];
    }
  }
}

// Copy of a field in another element type (S -> D), optionally with each site's
// unit-vector components divided by their FP64 norm (the projection the flow applies
// after every step).  A stored FP32 unit vector cannot hold m3 = 1 - |m_perp|^2/2 once
// |m_perp| < 2.4e-4: it rounds to 1 and |m|^2 - 1 = |m_perp|^2 > 0 there; an FP64
// projected copy restores the constraint to FP64 rounding.  Each site's components are
// read and normalised in FP64, then rounded once to D.
template <typename S, typename D, int NF, int NMAG>
__global__ void convert_kernel(const S* src, D* dst, long long N, int normalize) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x) {
    double P[NF];
#pragma unroll
    for (int a = 0; a < NF; ++a) P[a] = (double)src[a * N + s];
    if (NMAG > 0 && normalize) {
      double s2 = 0.0;
#pragma unroll
      for (int a = 0; a < NMAG; ++a) s2 += P[a] * P[a];
      if (s2 > 0.0) {
        const double nrm = sqrt(s2);
#pragma unroll
        for (int a = 0; a < NMAG; ++a) P[a] /= nrm;
      }
    }
#pragma unroll
    for (int a = 0; a < NF; ++a) dst[a * N + s] = (D)P[a];
  }
}

}  // namespace ssb
