// init.cuh -- initial-condition kernels of the four theories (ground state, the
// single-soliton ansatz, and inserting a soliton into an existing field).
//
// Restates theories/<theory>/initial_config.py of the reference per site in FP64:
// coordinates grid = (lsx x, lsy y) (create_grid_kernel), position / angle /
// profile functions, create_ground_state_kernel, create_initial_configuration_kernel,
// create_skyrmion_kernel (chiral magnet, baby Skyrme; stereographic composition with
// the field already there) and create_vortex_kernel (Abelian Higgs, s+id).  The
// reference's slot choices are kept (skyrmion number p_f[9] for the chiral magnet,
// p_f[8] for baby Skyrme; the s+id ground state reads u1, u2 from p_f[11], p_f[12]);
// the Abelian Higgs ansatz reads ainf from its packed slot p_f[10] (the reference reads
// p_f[11], past the end of the array).
#pragma once

namespace ssb {

enum InitMode { IM_GROUND = 0, IM_ANSATZ = 1, IM_INSERT = 2 };
enum Ansatz { AZ_NONE = 0, AZ_BLOCH = 1, AZ_NEEL = 2, AZ_ANTI = 3 };

struct InitArgs {
  int X, Y, nf, mode, ansatz, vortex, pxi, pxj;
  double rotation, vortex_number;
  double pf[32];  // the theory's packed p_f
};

constexpr double IC_TWO_PI = 2.0 * 3.141592653589793;

// angle (initial_config.py: angle): -orientation + atan2 in [0, 2 pi), or
// -orientation at the centre itself
__device__ inline double ic_angle(double r, double dx, double dy, double orientation) {
  const double theta = -orientation;
  if (r == 0.0) return theta;
  double ang = atan2(dy, dx);
  if (ang < 0.0) ang += IC_TWO_PI;
  return theta + ang;
}

__device__ inline double ic_profile_m(double r, double max_r) {
  if (r > max_r) return 0.0;
  const double t = 2.0 * r / max_r;
  return 3.141592653589793 * exp(-(t * t));
}

__device__ inline double ic_profile_s(double r, double max_r, double value) {
  if (r > max_r) return 1.0;
  return tanh(value * r);
}

// ansatz magnetisation; false for "no ansatz" (vacuum)
__device__ inline bool ic_ansatz_m(int ansatz, double fm, double th, double skN, double m[3]) {
  const double sf = sin(fm), cf = cos(fm), sa = sin(skN * th), ca = cos(skN * th);
  switch (ansatz) {
    case AZ_BLOCH: m[0] = -sf * sa; m[1] = sf * ca; m[2] = cf; return true;
    case AZ_NEEL: m[0] = sf * ca; m[1] = sf * sa; m[2] = cf; return true;
    case AZ_ANTI: m[0] = -sf * sa; m[1] = -sf * ca; m[2] = cf; return true;
  }
  return false;
}

// compute_norm_magnetization (chiral_magnet/kernels.py:48-84)
__device__ inline void ic_normalise(double m[3]) {
  double s = 0.0;
  for (int a = 0; a < 3; ++a) s += m[a] * m[a];
  s = sqrt(s);
  if (s == 0.0) return;
  for (int a = 0; a < 3; ++a) m[a] /= s;
}

// THEORY: 0 chiral magnet, 1 baby Skyrme, 2 Abelian Higgs, 3 s+id.  One thread per site.
template <int THEORY, typename R>
__global__ void init_kernel(R* __restrict__ F, R* __restrict__ V, const InitArgs A) {
  const long long N = (long long)A.X * A.Y;
  const long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (s >= N) return;
  const int x = (int)(s / A.Y), y = (int)(s - (long long)x * A.Y);
  const double* pf = A.pf;
  const double lsx = pf[2], lsy = pf[3];
  // Coordinates, centre and distance with explicitly rounded operations: the site at
  // the centre must give r == 0 exactly, as in the reference (a fused lsx*x - xc would
  // leave a residual that the ansatz then divides by max(r, 1e-12)).
  const double gx = __dmul_rn(lsx, (double)x), gy = __dmul_rn(lsy, (double)y);
  const double rmax = pf[0] > pf[1] ? pf[0] : pf[1];
  double out[6] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  double xc, yc;
  if (A.mode == IM_INSERT) {
    xc = __dmul_rn(lsx, (double)A.pxi);
    yc = __dmul_rn(lsy, (double)A.pxj);
  } else {
    xc = __dadd_rn(0.0, __dmul_rn(lsx, (double)(A.X - 1))) / 2.0;
    yc = __dadd_rn(0.0, __dmul_rn(lsy, (double)(A.Y - 1))) / 2.0;
  }
  const double dx = __dsub_rn(gx, xc), dy = __dsub_rn(gy, yc);
  const double r = sqrt(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)));

  if constexpr (THEORY == 0 || THEORY == 1) {
    const double skN = pf[THEORY == 0 ? 9 : 8];
    const double th = ic_angle(r, dx, dy, A.rotation);
    if (A.mode == IM_GROUND) {
      out[2] = 1.0;
    } else if (A.mode == IM_ANSATZ) {
      double m[3];
      if (ic_ansatz_m(A.ansatz, ic_profile_m(r, rmax / 10.0 * skN), th, skN, m)) {
        ic_normalise(m);
        out[0] = m[0]; out[1] = m[1]; out[2] = m[2];
      } else {
        out[2] = 1.0;
      }
    } else {  // create_skyrmion_kernel: stereographic composition with the field present
      double m[3];
      const bool any = skN == 0.0 ? ic_ansatz_m(A.ansatz, 2.0 * ic_profile_m(r, rmax / 10.0 * 2.0), th, 1.0, m)
                                  : ic_ansatz_m(A.ansatz, ic_profile_m(r, rmax / 10.0 * skN), th, skN, m);
      if (!any) { m[0] = 0.0; m[1] = 0.0; m[2] = 1.0; }
      const double eps = 1e-12;
      const double f0 = (double)F[s], f1 = (double)F[s + N], f2 = (double)F[s + 2 * N];
      const double den = fmax(1.0 + f2, eps);
      const double int_den = fmax(1.0 + m[2], eps);
      const double wr = f0 / den + m[0] / int_den, wi = f1 / den + m[1] / int_den;
      const double nw = wr * wr + wi * wi;
      double n[3] = {2.0 * wr / (1.0 + nw), 2.0 * wi / (1.0 + nw), (1.0 - nw) / (1.0 + nw)};
      ic_normalise(n);
      F[s] = (R)n[0];
      F[s + N] = (R)n[1];
      F[s + 2 * N] = (R)n[2];
      return;  // psi and the velocity are untouched
    }
  } else if constexpr (THEORY == 2) {
    const double th = ic_angle(r, dx, dy, 0.0);
    const double u1 = pf[8];
    if (A.mode == IM_GROUND) {
      out[2] = u1;
    } else if (A.mode == IM_ANSATZ) {
      const double ainf = pf[10];
      const double fs = ic_profile_s(r, rmax, 0.2);
      const double rr = r > 1e-12 ? r : 1e-12;
      out[0] = ainf * fs * sin(th) / rr;
      out[1] = -ainf * fs * cos(th) / rr;
      out[2] = u1 * fs * cos(A.vortex_number * th);
      out[3] = u1 * fs * sin(A.vortex_number * th);
    } else {  // create_vortex_kernel
      const double vn = pf[9];
      const double fs = ic_profile_s(r, rmax, 0.2);
      const double phase = (A.vortex ? -1.0 : 1.0) * th;
      const double ir = u1 * fs * cos(vn * phase), ii = u1 * fs * sin(vn * phase);
      const double o_r = (double)F[s + 2 * N], o_i = (double)F[s + 3 * N];
      F[s + 2 * N] = (R)((o_r * ir - o_i * ii) / u1);
      F[s + 3 * N] = (R)((o_r * ii + o_i * ir) / u1);
      return;
    }
  } else {  // s+id
    const double th = ic_angle(r, dx, dy, 0.0);
    if (A.mode == IM_GROUND) {
      const double u1 = pf[11], u2 = pf[12], td = pf[19];
      out[2] = u1;
      out[4] = u2 * cos(td);
      out[5] = u2 * sin(td);
    } else if (A.mode == IM_ANSATZ) {
      const double u1 = pf[17], u2 = pf[18], ainf = pf[22], v1 = pf[23], v2 = pf[24];
      const double fs = ic_profile_s(r, rmax, 1.0);
      const double rr = r > 1e-12 ? r : 1e-12;
      out[0] = ainf * fs * sin(th) / rr;
      out[1] = -ainf * fs * cos(th) / rr;
      out[2] = u1 * fs * cos(v1 * th);
      out[3] = u1 * fs * sin(v1 * th);
      out[4] = u2 * fs * cos(v2 * th);
      out[5] = u2 * fs * sin(v2 * th);
    } else {  // create_vortex_kernel
      const double vn = pf[21], ainf = pf[22];
      const double fs = ic_profile_s(r, rmax, 2.0);
      const double phase = (A.vortex ? -1.0 : 1.0) * th;
      const double rr = r > 1e-12 ? r : 1e-12;
      F[s] = (R)((double)F[s] - ainf * fs * sin(th) / rr);
      F[s + N] = (R)((double)F[s + N] + ainf * fs * cos(th) / rr);
      const double ir = fs * cos(vn * phase), ii = fs * sin(vn * phase);
      for (int a = 2; a <= 4; a += 2) {
        const double o_r = (double)F[s + a * N], o_i = (double)F[s + (a + 1) * N];
        F[s + a * N] = (R)(o_r * ir - o_i * ii);
        F[s + (a + 1) * N] = (R)(o_r * ii + o_i * ir);
      }
      return;
    }
  }
  for (int a = 0; a < A.nf; ++a) {
    F[s + a * N] = (R)out[a];
    if (V) V[s + a * N] = (R)0;
  }
}

}  // namespace ssb
