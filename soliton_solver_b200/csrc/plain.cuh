// plain.cuh -- the "plain FP64" form of the flow step: the reference's own kernel
// structure on the GPU, used as the comparator the fused kernels are measured
// against.  Derivatives go through global buffers in the reference's x-contiguous
// layout (soliton_solver/core/utils.py:45-106), each RK stage is its own launch
// with (8, 8) thread blocks whose x index varies fastest (as numba's cuda.grid(2)),
// reductions are 1024-wide block trees whose partials are summed on the host, and
// the arrest decision is taken on the host (core/integrator.py:217-348).
#pragma once

#include "common.cuh"
#include "theories.cuh"

namespace ssb {

// value of component a at (x+dx, y+dy), 0 outside the lattice (never used unmasked)
struct GlobalAcc {
  const double* F;
  int X, Y, x, y;
  long long off;
  __device__ double operator()(int dx, int dy) const {
    const int gx = x + dx, gy = y + dy;
    if (gx < 0 || gx >= X || gy < 0 || gy >= Y) return 0.0;
    return F[off + (long long)gx * Y + gy];
  }
};

__device__ inline long long pl_d1(int coord, int field, int x, int y, const Grid& G) {
  return x + (long long)y * G.X + coord * G.N + field * G.N * 2;
}
__device__ inline long long pl_d2(int c1, int c2, int field, int x, int y, const Grid& G) {
  return x + (long long)y * G.X + c1 * G.N + c2 * G.N * 2 + field * G.N * 4;
}

// make_do_gradient_step_kernel (core/integrator.py:15-48): derivatives of every
// component written to d1/d2, read back by the theory's point function.
template <class TH>
__global__ void plain_gradient_kernel(double* l_out, const double* F, double* d1, double* d2, double* EG, Grid G,
                                      Phys P) {
  constexpr int NF = TH::NF;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= G.X || y >= G.Y) return;
  const Masks mk = site_masks(G, x, y);
  const Inv<double> iv(G);
  for (int a = 0; a < NF; ++a) {
    GlobalAcc acc{F, G.X, G.Y, x, y, (long long)a * G.N};
    double f, dx, dy, dxx, dyy, dxy;
    fill_jet_comp<double>(acc, mk, iv, f, dx, dy, dxx, dyy, dxy, true);
    d1[pl_d1(0, a, x, y, G)] = dx;
    d1[pl_d1(1, a, x, y, G)] = dy;
    d2[pl_d2(0, 0, a, x, y, G)] = dxx;
    d2[pl_d2(1, 1, a, x, y, G)] = dyy;
    d2[pl_d2(1, 0, a, x, y, G)] = dxy;
    d2[pl_d2(0, 1, a, x, y, G)] = dxy;
  }
  Jet<double, NF> J;
  const long long s = (long long)x * G.Y + y;
  for (int a = 0; a < NF; ++a) {
    J.f[a] = F[a * G.N + s];
    J.dx[a] = d1[pl_d1(0, a, x, y, G)];
    J.dy[a] = d1[pl_d1(1, a, x, y, G)];
    J.dxx[a] = d2[pl_d2(0, 0, a, x, y, G)];
    J.dyy[a] = d2[pl_d2(1, 1, a, x, y, G)];
    J.dxy[a] = d2[pl_d2(1, 0, a, x, y, G)];
  }
  double g[NF];
  TH::gradient(J, P, g);
  if (TH::HALO_ZERO && (x < G.halo || x > G.X - G.halo - 1 || y < G.halo || y > G.Y - G.halo - 1)) {
    for (int a = 0; a < NF; ++a) g[a] = 0.0;
  }
  if (TH::CONSTRAINED) {
    double lm = 0.0;
    for (int a = 0; a < TH::NMAG; ++a) lm += g[a] * J.f[a];
    for (int a = 0; a < TH::NMAG; ++a) g[a] -= lm * J.f[a];
  }
  for (int a = 0; a < NF; ++a) {
    EG[a * G.N + s] = g[a];
    l_out[a * G.N + s] = -G.dt * g[a];
  }
}

// compute_energy_kernel (e.g. theories/chiral_magnet/kernels.py:219-251)
template <class TH>
__global__ void plain_energy_kernel(double* en, const double* F, double* d1, Grid G, Phys P) {
  constexpr int NF = TH::NF;
  const int x = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  if (x >= G.X || y >= G.Y) return;
  const Masks mk = site_masks(G, x, y);
  const Inv<double> iv(G);
  for (int a = 0; a < NF; ++a) {
    GlobalAcc acc{F, G.X, G.Y, x, y, (long long)a * G.N};
    double f, dx, dy;
    fill_jet1_comp<double>(acc, mk, iv, f, dx, dy);
    d1[pl_d1(0, a, x, y, G)] = dx;
    d1[pl_d1(1, a, x, y, G)] = dy;
  }
  Jet1<double, NF> J;
  const long long s = (long long)x * G.Y + y;
  for (int a = 0; a < NF; ++a) {
    J.f[a] = F[a * G.N + s];
    J.dx[a] = d1[pl_d1(0, a, x, y, G)];
    J.dy[a] = d1[pl_d1(1, a, x, y, G)];
  }
  en[s] = TH::energy(J, P, G.dA);
}

// reduce_sum_kernel / reduce_max_kernel (core/utils.py:188-271)
__global__ void plain_reduce_kernel(const double* var, double* partial, long long size, int is_max) {
  __shared__ double sdata[1024];
  const int tid = threadIdx.x;
  const long long idx = blockIdx.x * (long long)blockDim.x + tid;
  double v = is_max ? -1.0e300 : 0.0;
  if (idx < size) v = var[idx];
  sdata[tid] = v;
  __syncthreads();
  for (int stride = blockDim.x / 2; stride > 0; stride /= 2) {
    if (tid < stride) {
      if (is_max) {
        if (sdata[tid] < sdata[tid + stride]) sdata[tid] = sdata[tid + stride];
      } else {
        sdata[tid] += sdata[tid + stride];
      }
    }
    __syncthreads();
  }
  if (tid == 0) partial[blockIdx.x] = sdata[0];
}

}  // namespace ssb
