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

#include "common.cuh"
#include "theories.cuh"

namespace ssb {

enum FlowMode { M_GRAD = 0, M_S1 = 1, M_S2 = 2, M_S3 = 3, M_S4 = 4, M_ENERGY = 5 };

template <typename R>
struct FlowArgs {
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

template <int TX, int TY, int NT>
struct TileShape {
  static constexpr int HX = TX + 4, HY = TY + 4;
  static constexpr int ROWS_PER_PASS = NT / TY;
  static constexpr int SITES_PER_THREAD = TX / ROWS_PER_PASS;
  static_assert(NT % TY == 0 && TX % (NT / TY) == 0, "tile/thread mismatch");
};

template <typename R, int NF, int TX, int TY>
__host__ __device__ constexpr size_t tile_bytes() {
  return sizeof(R) * NF * (TX + 4) * (TY + 4);
}

// Stage the (TX+4) x (TY+4) halo tile of T_s (formed on the fly from phi, V, l) into
// shared memory.  Out-of-lattice entries are 0 and never enter a masked derivative.
template <int NF, typename R, int TX, int TY, int NT>
__device__ inline void stage_tile(R* tile, const FlowArgs<R>& A, int x0, int y0, int mode, bool arrest) {
  using TS = TileShape<TX, TY, NT>;
  const Grid& G = A.G;
  const long long N = G.N;
  const R dt = (R)G.dt;
  const R half = (R)0.5;
#pragma unroll
  for (int a = 0; a < NF; ++a) {
    for (int i = threadIdx.x; i < TS::HX * TS::HY; i += NT) {
      const int r = i / TS::HY, c = i - r * TS::HY;
      const int gx = x0 - 2 + r, gy = y0 - 2 + c;
      R t = (R)0;
      if (gx >= 0 && gx < G.X && gy >= 0 && gy < G.Y) {
        const long long idx = (long long)a * N + (long long)gx * G.Y + gy;
        const R p = A.phi[idx];
        if (mode == M_S2) {
          const R v = arrest ? (R)0 : A.vel[idx];
          t = p + half * (dt * v);
        } else if (mode == M_S3) {
          const R v = arrest ? (R)0 : A.vel[idx];
          const R w = A.la[idx];
          t = p + half * (dt * (v + half * w));
        } else if (mode == M_S4) {
          const R v = arrest ? (R)0 : A.vel[idx];
          const R w = A.lb[idx];
          t = p + dt * (v + half * w);
        } else {
          t = p;
        }
      }
      tile[(a * TS::HX + r) * TS::HY + c] = t;
    }
  }
}

template <class TH, typename R, int TX, int TY, int NT>
__global__ void __launch_bounds__(NT) flow_kernel(const FlowArgs<R> A) {
  using TS = TileShape<TX, TY, NT>;
  constexpr int NF = TH::NF;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* tile = reinterpret_cast<R*>(smem_raw);
  __shared__ double red[NT / 32];
  __shared__ double sh_s[NT], sh_c[NT];
  __shared__ int am_last;

  const Grid& G = A.G;
  const int mode = A.mode;
  const int tiles_y = (G.Y + TY - 1) / TY;
  const int x0 = (blockIdx.x / tiles_y) * TX;
  const int y0 = (blockIdx.x % tiles_y) * TY;
  const long long N = G.N;
  StepState* st = A.st;
  const bool arrest = (mode == M_S2 || mode == M_S3 || mode == M_S4) && (st->arrest != 0);
  const bool do_energy = A.with_energy != 0;

  if (A.init_state && blockIdx.x == 0 && threadIdx.x == 0) {
    st->arrest = 0;
    if (!isnan(A.prev_energy)) st->E_last = A.prev_energy;
  }

  stage_tile<NF, R, TX, TY, NT>(tile, A, x0, y0, mode, arrest);
  __syncthreads();

  const Inv<R> iv(G);
  const Inv<double> ivd(G);
  const R dt = (R)G.dt;
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
    const R* base = tile + (lx + 2) * TS::HY + (ly + 2);

    if (do_energy) {
      Jet1<double, NF> J1;
#pragma unroll
      for (int a = 0; a < NF; ++a) {
        const R* pa = base + a * TS::HX * TS::HY;
        auto acc = [pa](int dx, int dy) -> double { return (double)pa[dx * TS::HY + dy]; };
        fill_jet1_comp<double>(acc, mk, ivd, J1.f[a], J1.dx[a], J1.dy[a]);
      }
      e_acc += TH::energy(J1, A.P, G.dA);
    }
    if (mode == M_ENERGY) continue;

    Jet<R, NF> J;
#pragma unroll
    for (int a = 0; a < NF; ++a) {
      const R* pa = base + a * TS::HX * TS::HY;
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
  extern __shared__ __align__(16) unsigned char smem_raw[];
  R* tile = reinterpret_cast<R*>(smem_raw);
  __shared__ double red[NT / 32];
  __shared__ double sh_s[NT], sh_c[NT];
  __shared__ int am_last;
  const int tiles_y = (G.Y + TY - 1) / TY;
  const int x0 = (blockIdx.x / tiles_y) * TX;
  const int y0 = (blockIdx.x % tiles_y) * TY;
  const long long N = G.N;
#pragma unroll
  for (int a = 0; a < NF; ++a) {
    for (int i = threadIdx.x; i < TS::HX * TS::HY; i += NT) {
      const int r = i / TS::HY, c = i - r * TS::HY;
      const int gx = x0 - 2 + r, gy = y0 - 2 + c;
      R t = (R)0;
      if (gx >= 0 && gx < G.X && gy >= 0 && gy < G.Y) t = phi[(long long)a * N + (long long)gx * G.Y + gy];
      tile[(a * TS::HX + r) * TS::HY + c] = t;
    }
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
    const R* base = tile + (lx + 2) * TS::HY + (ly + 2);
    Jet1<double, NF> J1;
#pragma unroll
    for (int a = 0; a < NF; ++a) {
      const R* pa = base + a * TS::HX * TS::HY;
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
