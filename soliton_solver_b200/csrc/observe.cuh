// observe.cuh -- per-site diagnostic densities of the gauge theories (Simulation's
// output helpers), one thread per site with plain loads: these run once per output,
// not per flow step.
//
//   FD_HIGGS         |psi|^2 (components 2, 3)         ginzburg_landau_superconductor/kernels.py:218-272
//   FD_HIGGS1        |psi1|^2 (components 2, 3)        anisotropic_superconductor/kernels.py:315-369
//   FD_HIGGS2        |psi2|^2 (components 4, 5)        anisotropic_superconductor/kernels.py:372-426
//   FD_PHASE_DIFF    cos(arg psi1 - arg psi2)           anisotropic_superconductor/kernels.py:497-553
//   FD_SUPERCURRENT  (dxy A2 - dyy A1, dxy A1 - dxx A2) ginzburg_landau_superconductor/kernels.py:275-340,
//                    two planes of N sites              anisotropic_superconductor/kernels.py:429-494
//   FD_MAGNETIC      (dx A2 - dy A1) dA / (2 pi q)     anisotropic_superconductor/kernels.py:280-312
// Derivatives use the reference's masks (the mixed derivative's asymmetric ring
// included) through fill_jet_comp.
#pragma once

#include "common.cuh"

namespace ssb {

enum FieldDensityKind { FD_HIGGS = 0, FD_HIGGS1 = 1, FD_HIGGS2 = 2, FD_PHASE_DIFF = 3, FD_SUPERCURRENT = 4,
                        FD_MAGNETIC = 5 };

template <typename R>
__global__ void field_density_kernel(const R* __restrict__ phi, double* __restrict__ out, int kind, Grid G,
                                     double charge_q) {
  const long long N = G.N;
  const Inv<double> iv(G);
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < N; s += (long long)gridDim.x * blockDim.x) {
    const int gx = (int)(s / G.Y), gy = (int)(s - (long long)gx * G.Y);
    auto val = [&](int a) -> double { return (double)phi[a * N + s]; };
    if (kind == FD_HIGGS || kind == FD_HIGGS1 || kind == FD_HIGGS2) {
      const int a = kind == FD_HIGGS2 ? 4 : 2;
      const double re = val(a), im = val(a + 1);
      out[s] = __dadd_rn(__dmul_rn(re, re), __dmul_rn(im, im));
      continue;
    }
    if (kind == FD_PHASE_DIFF) {
      const double t1 = atan2(val(3), val(2));
      const double t2 = atan2(val(5), val(4));
      out[s] = cos(t1 - t2);
      continue;
    }
    // gauge-field derivatives (components 0 and 1): reads clamped to the lattice; a
    // derivative whose stencil leaves the lattice is masked to zero anyway
    const Masks m = site_masks(G, gx, gy);
    double f[2], dx[2], dy[2], dxx[2], dyy[2], dxy[2];
#pragma unroll
    for (int a = 0; a < 2; ++a) {
      const R* pa = phi + a * N;
      auto acc = [&](int ox, int oy) -> double {
        const int x = gx + ox, y = gy + oy;
        if (x < 0 || x >= G.X || y < 0 || y >= G.Y) return 0.0;
        return (double)pa[(long long)x * G.Y + y];
      };
      fill_jet_comp<double>(acc, m, iv, f[a], dx[a], dy[a], dxx[a], dyy[a], dxy[a], kind == FD_SUPERCURRENT);
    }
    if (kind == FD_SUPERCURRENT) {
      out[s] = dxy[1] - dyy[0];
      out[N + s] = dxy[0] - dxx[1];
    } else {
      out[s] = (dx[1] - dy[0]) * (G.dA / (2.0 * 3.14159265358979323846 * charge_q));
    }
  }
}

}  // namespace ssb
