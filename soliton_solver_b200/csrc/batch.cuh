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

// a lattice's buffers (BatchInst::buf) and halo-box TMA maps (BatchInst::tm, the
// buffers BATCH_TM_BUF names)
enum { BB_FIELD = 0, BB_VEL = 1, BB_CP = 2, BB_CV = 3, BB_L1 = 4, BB_L2 = 5, BB_T4 = 6, BB_COUNT = 7 };
enum { BT_FIELD = 0, BT_VEL = 1, BT_L1 = 2, BT_T4 = 3, BT_COUNT = 4 };
constexpr int BATCH_TM_BUF[BT_COUNT] = {BB_FIELD, BB_VEL, BB_L1, BB_T4};

struct BatchInst {
  CUtensorMap tm[BT_COUNT];
  Grid G;
  Phys P;
  void* buf[BB_COUNT];  // field, velocity, cP, cV, l1, l2 (four-kernel steps), T4
  StepState* st;
  double* partial;    // one slot per tile of this lattice
  double* E_traj;     // per-lattice trajectory rows
  double* err_traj;
  int tile0, ntiles;
};

struct BatchStep {
  int with_energy, arrest_update, init_state;
  int E_idx, err_idx;
  const double* prev_energy;  // device, one per lattice (NaN keeps E_last); read with init_state
  int scratch_out;            // stage 4 writes phi' and V' into l1 and l2 (timing)
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
  const CUtensorMap* tm_phi = &I.tm[MODE == M_S4 ? BT_T4 : BT_FIELD];
  const CUtensorMap* tm_vel = &I.tm[BT_VEL];
  const CUtensorMap* tm_l = &I.tm[BT_L1];
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
    A.phi = (const R*)I.buf[MODE == M_S4 ? BB_T4 : BB_FIELD];
    A.vel = (const R*)I.buf[BB_VEL];
    A.la = (const R*)I.buf[BB_L1];
    A.lb = (const R*)I.buf[BB_L2];
    A.cp = (const R*)I.buf[BB_CP];
    A.cv = (const R*)I.buf[BB_CV];
    A.out_l = MODE == M_S1 ? (R*)I.buf[BB_L1] : MODE == M_S2 ? (R*)I.buf[BB_L2] : nullptr;
    A.out_t4 = (R*)I.buf[BB_T4];
    A.out_cp = (R*)I.buf[BB_CP];
    A.out_cv = (R*)I.buf[BB_CV];
    A.out_eg = nullptr;
    A.phi_out = (R*)I.buf[B.scratch_out ? BB_L1 : BB_FIELD];
    A.vel_out = (R*)I.buf[B.scratch_out ? BB_L2 : BB_VEL];
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

// Apply each lattice's pending arrest (V = 0), left by the trailing energy pass, at the
// end of a call.  grid.y = lattice.
template <typename R, int NF>
__global__ void batch_finish_kernel(const BatchInst* __restrict__ insts) {
  const BatchInst& I = insts[blockIdx.y];
  if (I.st->arrest == 0) return;
  R* dv = (R*)I.buf[BB_VEL];
  const long long n = (long long)NF * I.G.N;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dv[i] = (R)0;
}

}  // namespace ssb
