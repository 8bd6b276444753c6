// flow.cuh -- fused single-pass-per-stage kernels of the arrested-Newton-flow step.
//
// One RK4 step of the reference (core/integrator.py:217-348) is
//   k1 = dt V,            T1 = phi,           l1 = -dt G(T1)
//   k2 = dt (V + l1/2),   T2 = phi + k1/2,    l2 = -dt G(T2)
//   k3 = dt (V + l2/2),   T3 = phi + k2/2,    l3 = -dt G(T3)
//   k4 = dt (V + l3),     T4 = phi + k3,      l4 = -dt G(T4)
//   V' = V + (l1 + 2 l2 + 2 l3 + l4)/6,  phi' = phi + (k1 + 2 k2 + 2 k3 + k4)/6
// followed by the unit-norm re-projection, the energy of phi', the arrest test
// (E' > E -> V' = 0) and err = max G(T4).  Here every k_s and T_s is recomputed from
// (phi, V, l_s) while a tile is staged, so stage s reads only what it needs:
//   S1 reads phi                       writes l1  (+ energy of phi, see below)
//   S2 reads phi, V                    writes l2
//   S3 reads phi, V, l1                writes l3
//   S4 reads phi, V, l1, l2, l3        writes phi', V' (ping-pong buffers), err
// The energy of a step's result is computed by the NEXT step's S1, which stages
// exactly that field anyway, and the arrest decision is kept on the device
// (StepState.arrest) and applied by S2..S4 as "V = 0".  A trailing energy pass
// closes a call.  Compulsory traffic: 16 words per site and step.
#pragma once

#include <cuda.h>

#include "common.cuh"
#include "theories.cuh"

namespace ssb {

enum FlowMode { M_GRAD = 0, M_S1 = 1, M_S2 = 2, M_S3 = 3, M_S4 = 4, M_ENERGY = 5 };
enum { ST_TIMEOUT = 6 };

// Upper bound of a device-side wait on an mbarrier (~1 s at 1.9 GHz).  On expiry
// the kernel records ST_TIMEOUT, waits the same bound again for its copies in
// flight and returns without computing.
constexpr long long WAIT_CYCLES = 2000000000LL;

template <typename R>
struct FlowArgs {
  CUtensorMap tm_phi;  // TMA maps (used when the kernel is instantiated with TMA)
  CUtensorMap tm_vel;
  CUtensorMap tm_l;    // l1 (S3) or l2 (S4)
  const R* phi;
  const R* vel;
  const R* la;  // l1 (S3, S4)
  const R* lb;  // l2 (S4)
  const R* lc;  // l3 (S4)
  R* out_l;     // S1..S3: l_s;  M_GRAD: l_out (nullable)
  R* out_eg;    // M_GRAD: energy gradient (nullable)
  R* phi_out;   // S4
  R* vel_out;   // S4
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

// number of staged buffers a mode needs (phi, then velocity, then l)
__host__ __device__ inline int flow_buffers(int mode) {
  return mode == M_S2 ? 2 : (mode == M_S3 || mode == M_S4) ? 3 : 1;
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
__device__ inline bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
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
// Bounded wait; returns false when WAIT_CYCLES elapsed first.
__device__ inline bool mbar_wait_bounded(uint64_t* bar, uint32_t parity) {
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > WAIT_CYCLES) return false;
  }
  return true;
}

// T_s for one element from the staged inputs (the reference's k / Temp algebra,
// core/integrator.py:51-96 and :323-334)
template <typename R>
__device__ inline R stage_value(int mode, R p, R v, R w, R dt) {
  const R half = (R)0.5;
  if (mode == M_S2) return p + half * (dt * v);
  if (mode == M_S3) return p + half * (dt * (v + half * w));
  if (mode == M_S4) return p + dt * (v + half * w);
  return p;
}

// Plain-load staging of T_s into `T` (all components), used when a TMA map cannot
// describe the buffers (row pitch not a multiple of 16 bytes).  Every thread first
// issues all loads of one component plane, then combines and stores, so each
// plane costs one memory round trip.
template <int NF, typename R, int TX, int TY, int NT>
__device__ inline void stage_plain(R* T, const FlowArgs<R>& A, int x0, int y0, int mode, bool arrest) {
  using TS = TileShape<TX, TY, NT>;
  constexpr int KM = (TS::PLANE + NT - 1) / NT;
  const Grid& G = A.G;
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
  const bool need_v = (mode == M_S2 || mode == M_S3 || mode == M_S4) && !arrest;
  const R* lsrc = mode == M_S3 ? A.la : (mode == M_S4 ? A.lb : nullptr);
#pragma unroll
  for (int a = 0; a < NF; ++a) {
    R p[KM], v[KM], w[KM];
    const long long base = (long long)a * N;
#pragma unroll
    for (int k = 0; k < KM; ++k) {
      p[k] = ok[k] ? A.phi[base + off[k]] : (R)0;
      v[k] = (ok[k] && need_v) ? A.vel[base + off[k]] : (R)0;
      w[k] = (ok[k] && lsrc) ? lsrc[base + off[k]] : (R)0;
    }
#pragma unroll
    for (int k = 0; k < KM; ++k) {
      const int i = threadIdx.x + k * NT;
      if (i < TS::PLANE) T[a * TS::PLANE + i] = stage_value<R>(mode, p[k], v[k], w[k], dt);
    }
  }
}

template <class TH, typename R, int TX, int TY, int NT, bool TMA>
__global__ void __launch_bounds__(NT) flow_kernel(const __grid_constant__ FlowArgs<R> A) {
  using TS = TileShape<TX, TY, NT>;
  constexpr int NF = TH::NF;
  constexpr int BUF = NF * TS::PLANE;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  R* B0 = reinterpret_cast<R*>(smem_raw);
  R* B1 = B0 + BUF;
  R* B2 = B1 + BUF;
  __shared__ double red[NT / 32];
  __shared__ double sh_s[NT], sh_c[NT];
  __shared__ int am_last;
  __shared__ __align__(8) uint64_t bar;

  const Grid& G = A.G;
  const int mode = A.mode;
  const int tiles_y = (G.Y + TY - 1) / TY;
  const int x0 = (blockIdx.x / tiles_y) * TX;
  const int y0 = (blockIdx.x % tiles_y) * TY;
  const long long N = G.N;
  StepState* st = A.st;
  const bool arrest = (mode == M_S2 || mode == M_S3 || mode == M_S4) && (st->arrest != 0);
  const bool do_energy = A.with_energy != 0;
  const R dt = (R)G.dt;

  if (A.init_state && blockIdx.x == 0 && threadIdx.x == 0) {
    st->arrest = 0;
    if (!isnan(A.prev_energy)) st->E_last = A.prev_energy;
  }

  // ---- stage the halo tile of T_s --------------------------------------
  R* T = B0;
  if constexpr (TMA) {
    const bool need_v = (mode == M_S2 || mode == M_S3 || mode == M_S4) && !arrest;
    const bool need_l = mode == M_S3 || mode == M_S4;
    if (threadIdx.x == 0) mbar_init(&bar, 1);
    __syncthreads();
    if (threadIdx.x == 0) {
      const uint32_t bytes = (uint32_t)(sizeof(R) * BUF) * (1u + (need_v ? 1u : 0u) + (need_l ? 1u : 0u));
      mbar_expect_tx(&bar, bytes);
      tma_load_3d(B0, &A.tm_phi, y0 - TS::YOFF, x0 - 2, 0, &bar);
      if (need_v) tma_load_3d(B1, &A.tm_vel, y0 - TS::YOFF, x0 - 2, 0, &bar);
      if (need_l) tma_load_3d(B2, &A.tm_l, y0 - TS::YOFF, x0 - 2, 0, &bar);
    }
    const bool ok = __syncthreads_and(mbar_wait_bounded(&bar, 0));
    if (!ok) {
      if (threadIdx.x == 0) atomicExch(&st->status, (int)ST_TIMEOUT);
      mbar_wait_bounded(&bar, 0);
      return;
    }
    if (mode == M_S2 || mode == M_S3 || mode == M_S4) {
      // combine in place into the last staged buffer (OOB entries are zero in all)
      R* dst = need_l ? B2 : (need_v ? B1 : B0);
      if (dst != B0) {
        for (int i = threadIdx.x; i < BUF; i += NT) {
          const R v = need_v ? B1[i] : (R)0;
          const R w = need_l ? B2[i] : (R)0;
          dst[i] = stage_value<R>(mode, B0[i], v, w, dt);
        }
        __syncthreads();
      }
      T = dst;
    }
  } else {
    stage_plain<NF, R, TX, TY, NT>(B0, A, x0, y0, mode, arrest);
    __syncthreads();
  }

  const Inv<R> iv(G);
  const Inv<double> ivd(G);
  const int ly = threadIdx.x % TY;
  const int lxg = threadIdx.x / TY;
  double e_acc = 0.0;
  double err_max = -INFINITY;

#pragma unroll 1
  for (int s = 0; s < TS::SITES_PER_THREAD; ++s) {
    const int lx = lxg + s * TS::ROWS_PER_PASS;
    const int gx = x0 + lx, gy = y0 + ly;
    if (gx >= G.X || gy >= G.Y) continue;
    const Masks mk = site_masks(G, gx, gy);
    const R* base = T + (lx + 2) * TS::HY + (ly + TS::YOFF);

    if (do_energy) {
      Jet1<double, NF> J1;
#pragma unroll
      for (int a = 0; a < NF; ++a) {
        const R* pa = base + a * TS::PLANE;
        auto acc = [pa](int dx, int dy) -> double { return (double)pa[dx * TS::HY + dy]; };
        fill_jet1_comp<double>(acc, mk, ivd, J1.f[a], J1.dx[a], J1.dy[a]);
      }
      e_acc += TH::energy(J1, A.P, G.dA);
    }
    if (mode == M_ENERGY) continue;

    Jet<R, NF> J;
#pragma unroll
    for (int a = 0; a < NF; ++a) {
      const R* pa = base + a * TS::PLANE;
      auto acc = [pa](int dx, int dy) -> R { return pa[dx * TS::HY + dy]; };
      fill_jet_comp<R>(acc, mk, iv, J.f[a], J.dx[a], J.dy[a], J.dxx[a], J.dyy[a], J.dxy[a], TH::NEED_XY);
    }
    R g[NF];
    TH::gradient(J, A.P, g);
    if (TH::HALO_ZERO) {
      const bool edge = gx < G.halo || gx > G.X - G.halo - 1 || gy < G.halo || gy > G.Y - G.halo - 1;
      if (edge) {
#pragma unroll
        for (int a = 0; a < NF; ++a) g[a] = (R)0;
      }
    }
    if (TH::CONSTRAINED) {  // project_orthogonal_magnetization (chiral_magnet/kernels.py:86-122)
      R lm = (R)0;
#pragma unroll
      for (int a = 0; a < TH::NMAG; ++a) lm += g[a] * J.f[a];
#pragma unroll
      for (int a = 0; a < TH::NMAG; ++a) g[a] -= lm * J.f[a];
    }
    const long long sidx = (long long)gx * G.Y + gy;
    if (mode == M_GRAD) {
#pragma unroll
      for (int a = 0; a < NF; ++a) {
        if (A.out_eg) A.out_eg[a * N + sidx] = g[a];
        if (A.out_l) A.out_l[a * N + sidx] = -dt * g[a];
      }
    } else if (mode != M_S4) {
#pragma unroll
      for (int a = 0; a < NF; ++a) A.out_l[a * N + sidx] = -dt * g[a];
    } else {
      // RK4 finalize (core/integrator.py:151-189) fused with stage 4
      R Pn[NF], Vn[NF];
      const R sixth = (R)(1.0 / 6.0), half = (R)0.5, two = (R)2;
#pragma unroll
      for (int a = 0; a < NF; ++a) {
        const long long idx = a * N + sidx;
        const R v = arrest ? (R)0 : A.vel[idx];
        const R p = A.phi[idx];
        const R l1 = A.la[idx], l2 = A.lb[idx], l3 = A.lc[idx];
        const R l4 = -dt * g[a];
        const R k1 = dt * v, k2 = dt * (v + half * l1), k3 = dt * (v + half * l2), k4 = dt * (v + l3);
        Vn[a] = v + sixth * (l1 + two * l2 + two * l3 + l4);
        Pn[a] = p + sixth * (k1 + two * k2 + two * k3 + k4);
        err_max = fmax(err_max, (double)g[a]);
      }
      if (TH::CONSTRAINED && G.unit_mag) {
        // compute_norm_magnetization + project_orthogonal_magnetization (kernels.py:48-122)
        R s2 = (R)0;
#pragma unroll
        for (int a = 0; a < TH::NMAG; ++a) s2 += Pn[a] * Pn[a];
        const R s = sqrt(s2);
        if (s != (R)0) {
#pragma unroll
          for (int a = 0; a < TH::NMAG; ++a) Pn[a] /= s;
        }
        R lm = (R)0;
#pragma unroll
        for (int a = 0; a < TH::NMAG; ++a) lm += Vn[a] * Pn[a];
#pragma unroll
        for (int a = 0; a < TH::NMAG; ++a) Vn[a] -= lm * Pn[a];
      }
#pragma unroll
      for (int a = 0; a < NF; ++a) {
        A.phi_out[a * N + sidx] = Pn[a];
        A.vel_out[a * N + sidx] = Vn[a];
      }
    }
  }

  // ---- reductions -------------------------------------------------------
  const bool need_ticket = do_energy || mode == M_S4;
  if (!need_ticket) return;
  if (do_energy) {
    const double bs = block_sum_fixed<NT>(e_acc, red);
    if (threadIdx.x == 0) A.partial[blockIdx.x] = bs;
  }
  if (mode == M_S4) {
    const double bm = block_max<NT>(err_max, red);
    if (threadIdx.x == 0 && bm > -INFINITY) atomicMax(&st->err_enc, enc_max(bm));
  }
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned t = atomicAdd(&st->ticket, 1u);
    am_last = (t == gridDim.x - 1);
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
    if (mode == M_S4) {
      const double err = dec_max(atomicExch(&st->err_enc, 0ULL));
      if (A.err_traj && A.err_idx >= 0) A.err_traj[A.err_idx] = err;
    }
    st->ticket = 0u;
  }
}

// Copy the ping-pong result back into the caller's buffers (when the step count
// was odd) and apply a pending arrest (V = 0) left by the trailing energy pass.
template <typename R>
__global__ void finish_kernel(const R* __restrict__ phi_src, const R* __restrict__ vel_src, R* phi_dst,
                              R* vel_dst, long long n, int copy, const StepState* st) {
  const bool arrest = st->arrest != 0;
  if (!copy && !arrest) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (copy) phi_dst[i] = phi_src[i];
    if (copy || arrest) vel_dst[i] = arrest ? (R)0 : vel_src[i];
  }
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

}  // namespace ssb
