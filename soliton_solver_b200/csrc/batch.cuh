// batch.cuh -- many independent lattices of one theory advanced together.
//
// One launch per RK stage covers the tiles of every lattice: block b works on tile
// b - tile0[i] of lattice i = tile_inst[b].  Each lattice keeps its own parameters,
// buffers, reduction partials and device step state (energy, arrest flag, err), so
// sizes, couplings and arrest histories are independent; the per-lattice last block
// (ticket counted per lattice) finalises that lattice's reductions.
#pragma once

#include "flow.cuh"

namespace ssb {

struct BatchInst {
  CUtensorMap tm[6];  // halo-box TMA maps: field, velocity, phi_alt, vel_alt, l1, l2
  Grid G;
  Phys P;
  void* buf[7];       // field, velocity, phi_alt, vel_alt, l1, l2, l3
  StepState* st;
  double* partial;    // one slot per tile of this lattice
  double* E_traj;     // per-lattice trajectory rows
  double* err_traj;
  int tile0, ntiles;
};

struct BatchStep {
  int parity;         // 0: the caller's buffers hold the current field; 1: the alternates do
  int copy_out;       // S2 / M_S23 at parity 0: also copy phi's and V's centres into the
                      // alternates (the last step of an odd count; its S4 runs at parity 1)
  int with_energy, arrest_update, init_state;
  int E_idx, err_idx;
  const double* prev_energy;  // device, one per lattice (NaN keeps E_last); read with init_state
  long long wait_cycles;
};

// Resident CTAs per SM the batched stage kernels are built for.  Each CTA stages,
// computes and stores one tile, so the staging latency is hidden only by other
// resident CTAs: FP32 fields cap the registers for three 256-thread CTAs (85 per
// thread) instead of the two that the heavier stencils (the Baby Skyrme term) would
// otherwise get, and for six 128-thread CTAs of the small 8 x 32 tiles.
template <typename R, int MODE, int NT>
__host__ __device__ constexpr int batch_ctas() {
  return sizeof(R) == 4 ? (NT <= 128 ? 6 : 3) : 1;
}

template <class TH, typename R, int TX, int TY, int NT, bool TMA, int MODE>
__global__ void __launch_bounds__(NT, (batch_ctas<R, MODE, NT>()))
    batch_flow_kernel(const BatchInst* __restrict__ insts, const int* __restrict__ tile_inst,
                      const __grid_constant__ BatchStep B) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ StageShared<NT> S;
  __shared__ FlowArgs<R> A;
  const int inst = tile_inst[blockIdx.x];
  const BatchInst& I = insts[inst];
  const int cur = B.parity;
  const CUtensorMap* tm_phi = &I.tm[cur ? 2 : 0];
  const CUtensorMap* tm_vel = &I.tm[cur ? 3 : 1];
  const CUtensorMap* tm_l = &I.tm[(MODE == M_S3 || MODE == M_S23) ? 4 : 5];
  if constexpr (TMA) {
    // the tile's loads first, so the set-up below overlaps them
    if (threadIdx.x == 0) {
      const int tile = blockIdx.x - I.tile0;
      const int tiles_y = (I.G.Y + TY - 1) / TY;
      mbar_init(&S.bar, 1);
      issue_tile<TH, R, TX, TY, NT, MODE>(reinterpret_cast<R*>(smem_raw), tm_phi, tm_vel, tm_l, (tile / tiles_y) * TX,
                                          (tile % tiles_y) * TY, &S.bar, 0u);
    }
  }
  {  // the lattice's parameters into shared memory (word copy)
    const int* src = reinterpret_cast<const int*>(&I.G);
    int* dst = reinterpret_cast<int*>(&A.G);
    for (int i = threadIdx.x; i < (int)(sizeof(Grid) / 4); i += NT) dst[i] = src[i];
    src = reinterpret_cast<const int*>(&I.P);
    dst = reinterpret_cast<int*>(&A.P);
    for (int i = threadIdx.x; i < (int)(sizeof(Phys) / 4); i += NT) dst[i] = src[i];
  }
  if (threadIdx.x == 0) {
    A.phi = (const R*)I.buf[cur ? 2 : 0];
    A.vel = (const R*)I.buf[cur ? 3 : 1];
    A.la = (const R*)I.buf[4];
    A.lb = (const R*)I.buf[5];
    A.lc = (const R*)I.buf[6];
    A.out_l = MODE == M_S1 ? (R*)I.buf[4] : MODE == M_S2 ? (R*)I.buf[5] : (MODE == M_S3 || MODE == M_S23)
                                                                            ? (R*)I.buf[6] : nullptr;
    A.out_l2 = MODE == M_S23 ? (R*)I.buf[5] : nullptr;
    A.out_eg = nullptr;
    A.phi_out = (R*)I.buf[cur ? 0 : 2];
    A.vel_out = (R*)I.buf[cur ? 1 : 3];
    const bool copy = (MODE == M_S2 || MODE == M_S23) && B.copy_out;
    A.copy_phi = copy ? (R*)I.buf[2] : nullptr;
    A.copy_vel = copy ? (R*)I.buf[3] : nullptr;
    A.force = nullptr;
    A.partial = I.partial;
    A.st = I.st;
    A.E_traj = I.E_traj;
    A.err_traj = I.err_traj;
    A.E_idx = B.E_idx;
    A.err_idx = B.err_idx;
    A.mode = MODE;
    A.with_energy = B.with_energy;
    A.arrest_update = B.arrest_update;
    A.init_state = B.init_state;
    A.prev_energy = B.prev_energy ? B.prev_energy[inst] : NAN;
    A.grad_raw = 0;
    A.exact_energy = 0;
    A.wait_cycles = B.wait_cycles;
    A.tx_extra = 0;
  }
  __syncthreads();
  flow_tile<TH, R, TX, TY, NT, TMA, MODE>(A, tm_phi, tm_vel, tm_l, blockIdx.x - I.tile0, I.ntiles, smem_raw, S, TMA);
}

// Copy each lattice's result back into the caller's buffers when the alternates hold
// it, and apply a pending arrest (V = 0).  grid.y = lattice.
template <typename R, int NF>
__global__ void batch_finish_kernel(const BatchInst* __restrict__ insts, int parity) {
  const BatchInst& I = insts[blockIdx.y];
  const bool arrest = I.st->arrest != 0;
  const bool copy = parity != 0;
  if (!copy && !arrest) return;
  R* dp = (R*)I.buf[0];
  R* dv = (R*)I.buf[1];
  const R* sp = (const R*)I.buf[2];
  const R* sv = (const R*)I.buf[3];
  const long long n = (long long)NF * I.G.N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    if (copy) dp[i] = sp[i];
    dv[i] = arrest ? (R)0 : (copy ? sv[i] : dv[i]);
  }
}

}  // namespace ssb
