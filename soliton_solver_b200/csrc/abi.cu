// abi.cu -- C ABI of libsoliton_b200 (declared in include/soliton_b200.h).
#include <algorithm>
#include <atomic>
#include <cmath>
#include <type_traits>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <vector>

#include <cuda.h>
#include <cudaTypedefs.h>

#include "../../include/soliton_b200.h"
#include "common.cuh"
#include "flow.cuh"
#include "plain.cuh"
#include "batch.cuh"
#include "render.cuh"
#include "init.cuh"
#include "observe.cuh"
#include "adjoint.cuh"
#include "text.cuh"
#include "theories.cuh"

using namespace ssb;

namespace {

constexpr int TX = 16, TY = 64, NT = 256;  // fused tile: 16 x 64 sites, 256 threads
constexpr int TRAJ_CAP = 1024;              // device trajectory slots used by ss_step
constexpr size_t ALIGN = 256;
// TMA maps of a bound handle: halo boxes of the field, the velocity, l1 and T4 (l[2]),
// and centre boxes of cP and cV
enum { TM_FIELD = 0, TM_VEL = 1, TM_L1 = 2, TM_T4 = 3, TM_CP = 4, TM_CV = 5, TM_COUNT = 6 };

thread_local char g_err[512] = "";

int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

#define CK(call)                                                                        \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) return fail(SS_ERR_CUDA, "%s: %s", #call, cudaGetErrorString(e_)); \
  } while (0)

size_t align_up(size_t v) { return (v + ALIGN - 1) / ALIGN * ALIGN; }

// cuTensorMapEncodeTiled through the runtime's driver entry point (no libcuda link)
PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = (PFN_cuTensorMapEncodeTiled_v12000)p;
  }
  return fn;
}

// 3-D map over component planes (dims y, x, component) whose box is one staged
// tile: (TY + 8) x (TX + 4) x NF.  Fails (-> plain loads) when the buffer or its
// row pitch is not 16-byte aligned.
bool encode_tile_map(CUtensorMap* m, const void* ptr, size_t es, int X, int Y, int NF, bool centre = false,
                     int tx = TX, int ty = TY) {
  if (!ptr || ((uintptr_t)ptr) % 16 || ((size_t)Y * es) % 16) return false;
  auto fn = encode_fn();
  if (!fn) return false;
  cuuint64_t dims[3] = {(cuuint64_t)Y, (cuuint64_t)X, (cuuint64_t)NF};
  cuuint64_t strides[2] = {(cuuint64_t)Y * es, (cuuint64_t)X * Y * es};
  cuuint32_t box[3] = {(cuuint32_t)(centre ? ty : ty + 8), (cuuint32_t)(centre ? tx : tx + 4), (cuuint32_t)NF};
  cuuint32_t estr[3] = {1, 1, 1};
  CUresult r = fn(m, es == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 3,
                  const_cast<void*>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                  CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

}  // namespace

struct ss_handle {
  int theory = 0, precision = 0, nf = 0;
  double pf_raw[32] = {};  // the packed p_f as given (initial-condition kernels read it)
  Grid G{};
  Phys P{};
  size_t elem = 8;
  int nblocks = 0;        // fused tiles
  int plain_sum_blocks = 0, plain_max_blocks = 0;
  // bound buffers
  void* field = nullptr;
  void* vel = nullptr;
  char* ws = nullptr;
  size_t ws_bytes = 0;
  cudaStream_t stream = nullptr;
  // workspace carve (fused)
  StepState* st = nullptr;
  double* partial = nullptr;
  double* traj_E = nullptr;
  double* traj_err = nullptr;
  // fused flow buffers: l1, l2 (four-kernel steps only), T4; then cP and cV (stage 4's
  // inputs besides T4: phi + dt V + dt (l1 + l2 + l3)/6 and V + (l1 + 2 l2 + 2 l3)/6)
  void* l[4] = {nullptr, nullptr, nullptr, nullptr};
  void* cp_buf = nullptr;
  void* cv_buf = nullptr;
  // plain extras
  void* k[4] = {nullptr, nullptr, nullptr, nullptr};
  void* temp = nullptr;
  void* eg = nullptr;
  double* d1 = nullptr;
  double* d2 = nullptr;
  double* en = nullptr;
  double* entmp = nullptr;
  double E_last_host = NAN;
  std::vector<double> host_partial;
  // TMA maps of the bound buffers (index constants TM_*)
  CUtensorMap tm[TM_COUNT];
  bool tma = false;
  int num_sms = 148;
  // per flow mode: 1 = persistent pipelined kernel, 0 = one tile per CTA (autotuned)
  int use_pipe[N_FLOW_MODES] = {1, 1, 1, 1, 1, 1, 0};
  float tune_ms[N_FLOW_MODES][2] = {};
  int fuse23 = 1;  // stages 2 and 3 in one kernel (TMA staging only)
  long long wait_cycles = WAIT_CYCLES;
  mutable int inject_timeout = 0;  // test hook, consumed by the next flow launch
  cudaGraphExec_t graph = nullptr;  // captured n-step relaxation (ss_graph_create)
  const double* force = nullptr;    // FP64 flows: field added to the gradient rows (ss_set_forcing)
  // mapped page-locked staging of ss_step, written by the kernels themselves: the energy
  // and err trajectories of one chunk and the status of the call (allocated on the first
  // ss_step; host_stage_dev is its device address)
  double* host_stage = nullptr;
  double* host_stage_dev = nullptr;
  ~ss_handle() {
    if (graph) cudaGraphExecDestroy(graph);
    if (host_stage) cudaFreeHost(host_stage);
  }
};

namespace {

// ---------------------------------------------------------------------------
// workspace layout
// ---------------------------------------------------------------------------
size_t layout(ss_handle* h, char* base) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> char* {
    char* p = base ? base + off : nullptr;
    off = align_up(off + bytes);
    return p;
  };
  const size_t field_bytes = h->elem * (size_t)h->nf * (size_t)h->G.N;
  h->st = (StepState*)take(sizeof(StepState));
  const size_t np = (size_t)std::max(h->nblocks, std::max(h->plain_sum_blocks, h->plain_max_blocks));
  h->partial = (double*)take(np * sizeof(double));
  h->traj_E = (double*)take(TRAJ_CAP * sizeof(double));
  h->traj_err = (double*)take(TRAJ_CAP * sizeof(double));
  if (h->precision == SS_PLAIN_FP64) {
    for (int i = 0; i < 4; ++i) h->k[i] = take(field_bytes);
    for (int i = 0; i < 4; ++i) h->l[i] = take(field_bytes);
    h->temp = take(field_bytes);
    h->eg = take(field_bytes);
    h->d1 = (double*)take(2 * field_bytes);
    h->d2 = (double*)take(4 * field_bytes);
    h->en = (double*)take((size_t)h->G.N * sizeof(double));
    h->entmp = (double*)take((size_t)h->G.N * sizeof(double));
  } else {
    for (int i = 0; i < 3; ++i) h->l[i] = take(field_bytes);
    h->l[3] = nullptr;
    h->cp_buf = take(field_bytes);
    h->cv_buf = take(field_bytes);
  }
  return off;
}

// ---------------------------------------------------------------------------
// parameter decoding (packed arrays of each theory's pack_device_params)
// ---------------------------------------------------------------------------
int decode(ss_handle* h, int theory, const int32_t* p_i, int n_i, const double* p_f, int n_f) {
  static const int need_i[4] = {16, 20, 12, 14};
  static const int need_f[4] = {15, 14, 11, 25};
  static const int theory_nf[4] = {4, 3, 4, 6};
  if (theory < 0 || theory > 3) return fail(SS_ERR_ARG, "unknown theory id %d", theory);
  if (!p_i || !p_f) return fail(SS_ERR_ARG, "p_i/p_f must not be NULL");
  if (n_i < need_i[theory] || n_f < need_f[theory])
    return fail(SS_ERR_ARG, "packed params too short for theory %d: n_i=%d (need %d), n_f=%d (need %d)", theory, n_i,
                need_i[theory], n_f, need_f[theory]);
  for (int i = 0; i < n_f && i < 32; ++i) h->pf_raw[i] = p_f[i];
  Grid& G = h->G;
  G.X = p_i[0];
  G.Y = p_i[1];
  G.halo = p_i[2];
  const int nc = p_i[3], nf = p_i[4];
  if (G.X < 1 || G.Y < 1) return fail(SS_ERR_ARG, "xlen/ylen must be positive (got %d, %d)", G.X, G.Y);
  if (nc != 2) return fail(SS_ERR_ARG, "number_coordinates must be 2 (got %d)", nc);
  if (nf != theory_nf[theory])
    return fail(SS_ERR_ARG, "number_total_fields=%d but theory %d has %d components", nf, theory, theory_nf[theory]);
  if (G.halo < 2) return fail(SS_ERR_ARG, "halo must be >= 2 for the 5-point stencils (got %d)", G.halo);
  G.N = (long long)G.X * G.Y;
  if ((long long)p_i[5] != G.N || (long long)p_i[6] != G.N * nf)
    return fail(SS_ERR_ARG, "p_i[5]/p_i[6] (dim_grid/dim_fields) inconsistent with xlen*ylen*nf");
  G.killkinen = p_i[7] ? 1 : 0;
  G.unit_mag = p_i[9] ? 1 : 0;
  G.lsx = p_f[2];
  G.lsy = p_f[3];
  G.dA = p_f[4];
  G.dt = p_f[5];
  G.ihx = 1.0 / G.lsx;
  G.ihy = 1.0 / G.lsy;
  G.ihx2 = 1.0 / (G.lsx * G.lsx);
  G.ihy2 = 1.0 / (G.lsy * G.lsy);
  G.ih2dA = 1.0 / (2.0 * G.dA);
  if (!(G.lsx > 0) || !(G.lsy > 0) || !std::isfinite(G.lsx) || !std::isfinite(G.lsy) || !std::isfinite(G.dA) ||
      !std::isfinite(G.dt))
    return fail(SS_ERR_ARG, "lattice spacings / time step must be finite and positive");
  h->nf = nf;
  {
    const double c12 = 1.0 / 12.0, c23 = 2.0 / 3.0, c43 = 4.0 / 3.0;
    double* k = G.kd;
    k[GK_C23HX] = c23 * G.ihx;   k[GK_MC12HX] = -c12 * G.ihx;
    k[GK_C43HX2] = c43 * G.ihx2; k[GK_MC12HX2] = -c12 * G.ihx2;
    k[GK_C23HY] = c23 * G.ihy;   k[GK_MC12HY] = -c12 * G.ihy;
    k[GK_C43HY2] = c43 * G.ihy2; k[GK_MC12HY2] = -c12 * G.ihy2;
    k[GK_C43HD] = c43 * G.ih2dA; k[GK_MC12HD] = -c12 * G.ih2dA;
    k[GK_DT] = G.dt; k[GK_MDT] = -G.dt; k[GK_HDT] = 0.5 * G.dt; k[GK_DT6] = G.dt / 6.0; k[GK_SIXTH] = 1.0 / 6.0;
    for (int i = 0; i < 16; ++i) G.kf[i] = (float)G.kd[i];
  }
  Phys& P = h->P;
  memset(&P, 0, sizeof(P));
  switch (theory) {
    case SS_THEORY_CHIRAL_MAGNET: {
      if (p_i[10] != 3) return fail(SS_ERR_ARG, "chiral magnet needs number_magnetization_fields=3");
      P.c[0] = p_f[6];
      P.c[1] = p_f[7];
      P.c[2] = p_f[8];
      double D00 = 0, D01 = 0, D10 = 0, D11 = 0;  // chiral_magnet/kernels.py:151-160
      if (p_i[11]) {
        D00 = -1.0; D11 = -1.0;
      } else if (p_i[12]) {
        D01 = -1.0; D10 = 1.0;
      } else if (p_i[13]) {
        D00 = 1.0; D11 = -1.0;
      } else if (p_i[14]) {
        const double s = 0.7071067811865476;
        D00 = -s; D01 = -s; D10 = s; D11 = -s;
      }
      P.c[3] = D00; P.c[4] = D01; P.c[5] = D10; P.c[6] = D11;
      P.k[0] = p_i[15] ? 1 : 0;
      if (P.k[0] && !(P.c[2] != 0.0)) return fail(SS_ERR_ARG, "demag needs coup_mu != 0");
      break;
    }
    case SS_THEORY_BABY_SKYRME: {
      if (p_i[10] != 3) return fail(SS_ERR_ARG, "baby Skyrme needs number_magnetization_fields=3");
      P.c[0] = p_f[6];
      P.c[1] = p_f[7];
      for (int i = 0; i < 8; ++i) P.k[i] = p_i[11 + i] ? 1 : 0;
      P.k[8] = p_i[19];
      if (P.k[6] && P.k[8] < 1) return fail(SS_ERR_ARG, "broken potential needs N >= 1");
      break;
    }
    case SS_THEORY_GINZBURG_LANDAU: {
      P.c[0] = p_f[6];
      P.c[1] = p_f[7];
      P.c[2] = p_f[8];
      P.c[3] = p_f[9];
      if (!(P.c[0] != 0.0)) return fail(SS_ERR_ARG, "q must be nonzero");
      break;
    }
    case SS_THEORY_ANISOTROPIC: {
      for (int i = 0; i < 11; ++i) P.c[i] = p_f[6 + i];
      const double a1 = p_f[8], a2 = p_f[9], b1 = p_f[10], b2 = p_f[11], b3 = p_f[12], b4 = p_f[13];
      const double u1 = p_f[17], u2 = p_f[18], th = p_f[19];
      // vacuum energy density subtracted per site (anisotropic_superconductor/kernels.py:169)
      P.c[11] = a1 * u1 * u1 + a2 * u2 * u2 + b1 * u1 * u1 * u1 * u1 + b2 * u2 * u2 * u2 * u2 + b3 * u1 * u1 * u2 * u2 +
                2.0 * b4 * u1 * u1 * u2 * u2 * std::cos(2.0 * th);
      if (!(P.c[1] != 0.0)) return fail(SS_ERR_ARG, "Q must be nonzero");
      break;
    }
  }
  switch (theory) {
    case SS_THEORY_CHIRAL_MAGNET: ChiralMagnet::derive(P); break;
    case SS_THEORY_BABY_SKYRME: BabySkyrme::derive(P); break;
    case SS_THEORY_GINZBURG_LANDAU: GinzburgLandau::derive(P); break;
    case SS_THEORY_ANISOTROPIC: Anisotropic::derive(P); break;
  }
  for (int i = 0; i < 24; ++i) P.cf[i] = (float)P.c[i];
  return SS_OK;
}

int check_bound(const ss_handle* h) {
  if (!h) return fail(SS_ERR_ARG, "NULL handle");
  if (!h->ws) return fail(SS_ERR_STATE, "no workspace bound: call ss_bind first");
  return SS_OK;
}

// Opt a kernel into more than 48 KB of dynamic shared memory, once per device.
// `done` is owned by the caller's template instantiation.
template <class K>
void set_smem(K kernel, size_t bytes, unsigned long long& done) {
  if (bytes <= 32 * 1024) return;
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 64 && (done >> dev) & 1ULL) return;
  cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (dev < 64) done |= 1ULL << dev;
}

dim3 grid_1d(long long n) {
  long long b = (n + 255) / 256;
  if (b > 148 * 16) b = 148 * 16;
  if (b < 1) b = 1;
  return dim3((unsigned)b);
}

// ---------------------------------------------------------------------------
// per-(theory, precision) implementation
// ---------------------------------------------------------------------------
template <class TH, typename R>
struct Fused {
  static constexpr size_t BUF = tile_buf_bytes<R, TH::NF, TX, TY>();
  static inline unsigned long long smem_done_density = 0;

  // tma: use the TMA-staged instantiation (A.tm_* must describe A's buffers)
  static inline unsigned long long smem_done[2][N_FLOW_MODES] = {};

  // dynamic shared memory of flow_kernel: the staged buffers
  template <bool TMA_, int MODE>
  static constexpr size_t flow_smem() {
    return TMA_ ? flow_buffers(MODE) * BUF : BUF;
  }

  // threads of a one-tile CTA: 512 where the staged buffers leave room for only one CTA
  // per SM (above 113 KB: FP64 stages 3 and 2+3, and stage 2 of the six-component s+id
  // in FP64), else 256
  template <bool TMA_, int MODE>
  static constexpr int flow_threads() {
    return flow_smem<TMA_, MODE>() > 113 * 1024 ? 2 * NT : NT;
  }

  template <bool TMA_, int MODE>
  static int launch_mode(const ss_handle* h, const FlowArgs<R>& A) {
    constexpr int NTM = flow_threads<TMA_, MODE>();
    auto k = flow_kernel<TH, R, TX, TY, NTM, TMA_, MODE>;
    const size_t smem = flow_smem<TMA_, MODE>();
    set_smem(k, smem, smem_done[TMA_ ? 1 : 0][MODE]);
    k<<<h->nblocks, NTM, smem, h->stream>>>(A);
    CK(cudaGetLastError());
    return SS_OK;
  }

  template <bool TMA_>
  static int launch_tma(const ss_handle* h, const FlowArgs<R>& A) {
    switch (A.mode) {
      case M_GRAD: return launch_mode<TMA_, M_GRAD>(h, A);
      case M_S1: return launch_mode<TMA_, M_S1>(h, A);
      case M_S2: return launch_mode<TMA_, M_S2>(h, A);
      case M_S3: return launch_mode<TMA_, M_S3>(h, A);
      case M_S4: return launch_mode<TMA_, M_S4>(h, A);
      case M_ENERGY: return launch_mode<TMA_, M_ENERGY>(h, A);
      case M_S23:
        if constexpr (TMA_) return launch_mode<TMA_, M_S23>(h, A);
        else return fail(SS_ERR_ARG, "the fused stages 2+3 need TMA staging");
    }
    return fail(SS_ERR_ARG, "bad flow mode");
  }

  // persistent TMA-pipelined variant: FP32 fields and at least two ring slots; threads
  // and resident CTAs per SM from pipe_threads / pipe_ctas
  template <int MODE>
  static constexpr int pipe_stages() {
    const size_t slot = pipe_slot_bytes<R, TH::NF, TX, TY, MODE>();
    // dynamic shared memory left next to the static reduction arrays, per resident CTA
    const size_t budget = pipe_ctas<TH, MODE>() == 4 ? 50 * 1024 : 212 * 1024;
    const int n = (int)(budget / slot);
    return n > 4 ? 4 : n;
  }
  template <int MODE>
  static constexpr bool pipe_ok() {
    return sizeof(R) == 4 && pipe_stages<MODE>() >= 2;
  }
  static inline unsigned long long smem_done_pipe[N_FLOW_MODES] = {};

  template <int MODE>
  static int launch_pipe(const ss_handle* h, const FlowArgs<R>& A) {
    if constexpr (pipe_ok<MODE>()) {
      constexpr int S = pipe_stages<MODE>();
      constexpr int NTP = pipe_threads<TH, MODE>();
      auto k = flow_kernel_pipe<TH, R, TX, TY, NTP, MODE, S>;
      const size_t smem = S * pipe_slot_bytes<R, TH::NF, TX, TY, MODE>();
      set_smem(k, smem, smem_done_pipe[MODE]);
      const int grid = std::min(h->nblocks, pipe_ctas<TH, MODE>() * h->num_sms);
      k<<<grid, NTP, smem, h->stream>>>(A);
      CK(cudaGetLastError());
      return SS_OK;
    } else {
      return launch_mode<true, MODE>(h, A);
    }
  }

  static bool uses_pipe(int mode) {
    switch (mode) {
      case M_GRAD: return pipe_ok<M_GRAD>();
      case M_S1: return pipe_ok<M_S1>();
      case M_S2: return pipe_ok<M_S2>();
      case M_S3: return pipe_ok<M_S3>();
      case M_S4: return pipe_ok<M_S4>();
      case M_ENERGY: return pipe_ok<M_ENERGY>();
    }
    return false;
  }

  // tma: use the TMA-staged instantiations (A.tm_* must describe A's buffers)
  static int launch(const ss_handle* h, const FlowArgs<R>& A0, bool tma) {
    FlowArgs<R> A = A0;
    if (h->inject_timeout && tma) {
      A.tx_extra = 16;
      h->inject_timeout = 0;
    }
    if (!tma) return launch_tma<false>(h, A);
    // exact FP64 energies (observables) run one tile per CTA: the pipelined energy pass
    // of the packed-energy theories is built for the flow energy only
    if (!h->use_pipe[A.mode] || (A.mode == M_ENERGY && A.exact_energy && pipe_ctas<TH, M_ENERGY>() == 4))
      return launch_tma<true>(h, A);
    switch (A.mode) {
      case M_GRAD: return launch_pipe<M_GRAD>(h, A);
      case M_S1: return launch_pipe<M_S1>(h, A);
      case M_S2: return launch_pipe<M_S2>(h, A);
      case M_S3: return launch_pipe<M_S3>(h, A);
      case M_S4: return launch_pipe<M_S4>(h, A);
      case M_ENERGY: return launch_pipe<M_ENERGY>(h, A);
    }
    return fail(SS_ERR_ARG, "bad flow mode");
  }

  static FlowArgs<R> base_args(const ss_handle* h) {
    FlowArgs<R> A;
    memset(&A, 0, sizeof(A));
    A.wait_cycles = h->wait_cycles;
    A.G = h->G;
    A.P = h->P;
    A.st = h->st;
    A.partial = h->partial;
    A.force = h->force;
    A.E_idx = -1;
    A.err_idx = -1;
    A.prev_energy = NAN;
    return A;
  }

  // n flow steps of the bound buffers, in place; trajectories to device arrays (nullable)
  // status_out (nullable, device-visible): the finish kernel copies the call's status there
  static int step(ss_handle* h, int n, double prev, double* E_dev, double* err_dev, int* status_out = nullptr) {
    if (n <= 0) return SS_OK;
    R* field = (R*)h->field;
    R* vel = (R*)h->vel;
    R* l1 = (R*)h->l[0];
    R* l2 = (R*)h->l[1];
    R* t4 = (R*)h->l[2];
    R* cp = (R*)h->cp_buf;
    R* cv = (R*)h->cv_buf;
    FlowArgs<R> A = base_args(h);
    A.E_traj = E_dev;
    A.err_traj = err_dev;
    const bool tma = h->tma;
    const bool fused23 = tma && h->fuse23;
    A.vel = vel;
    A.la = l1;
    A.lb = l2;
    A.out_t4 = t4;
    A.out_cp = cp;
    A.out_cv = cv;
    A.cp = cp;
    A.cv = cv;
    A.phi_out = field;
    A.vel_out = vel;
    if (tma) {
      A.tm_vel = h->tm[TM_VEL];
      A.tm_l = h->tm[TM_L1];
      A.tm_cp = h->tm[TM_CP];
      A.tm_cv = h->tm[TM_CV];
    }
    for (int s = 0; s < n; ++s) {
      // S1: l1 = -dt G(phi); energy of phi (the previous step's result) + arrest test
      A.mode = M_S1;
      A.phi = field;
      A.out_l = l1;
      A.with_energy = s > 0;
      A.arrest_update = s > 0;
      A.E_idx = s - 1;
      A.init_state = s == 0;
      A.prev_energy = prev;
      if (tma) A.tm_phi = h->tm[TM_FIELD];
      int rc = launch(h, A, tma);
      if (rc) return rc;
      A.with_energy = 0;
      A.arrest_update = 0;
      A.init_state = 0;
      A.E_idx = -1;
      // S2, S3 (one fused kernel on TMA-staged buffers: one staging of phi, V, l1):
      // T4, cV, cP
      if (fused23) {
        A.mode = M_S23;
        if ((rc = launch(h, A, tma))) return rc;
      } else {
        A.mode = M_S2;
        A.out_l = l2;
        if ((rc = launch(h, A, tma))) return rc;
        A.mode = M_S3;
        if ((rc = launch(h, A, tma))) return rc;
      }
      A.out_l = nullptr;
      // S4: phi' and V' into the caller's buffers, err
      A.mode = M_S4;
      A.phi = t4;
      A.err_idx = s;
      if (tma) A.tm_phi = h->tm[TM_T4];
      if ((rc = launch(h, A, tma))) return rc;
      A.err_idx = -1;
    }
    // trailing energy of the final field + arrest test
    A.phi = field;
    A.mode = M_ENERGY;
    A.with_energy = 1;
    A.arrest_update = 1;
    A.E_idx = n - 1;
    if (tma) A.tm_phi = h->tm[TM_FIELD];
    int rc = launch(h, A, tma);
    if (rc) return rc;
    const long long nfN = (long long)h->nf * h->G.N;
    finish_kernel<R><<<grid_1d(nfN), 256, 0, h->stream>>>(vel, nfN, h->st, status_out);
    CK(cudaGetLastError());
    return SS_OK;
  }

  // Time both staging variants of every stage on the bound buffers and keep the faster
  // one.  Writes only workspace scratch: l1, l2, T4, cV, cP, and stage 4's phi' and V'
  // into the l1 and l2 buffers (stage 4 reads neither); stage 1's energy reduction
  // leaves the arrest state and the trajectories alone.
  static int autotune(ss_handle* h, int iters) {
    if (!h->tma) return SS_OK;
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    FlowArgs<R> A = base_args(h);
    A.vel = (const R*)h->vel;
    A.la = (const R*)h->l[0];
    A.lb = (const R*)h->l[1];
    A.out_t4 = (R*)h->l[2];
    A.out_cp = (R*)h->cp_buf;
    A.out_cv = (R*)h->cv_buf;
    A.cp = (const R*)h->cp_buf;
    A.cv = (const R*)h->cv_buf;
    A.phi_out = (R*)h->l[0];
    A.vel_out = (R*)h->l[1];
    A.tm_vel = h->tm[TM_VEL];
    A.tm_l = h->tm[TM_L1];
    A.tm_cp = h->tm[TM_CP];
    A.tm_cv = h->tm[TM_CV];
    auto set_mode = [&](int m) {
      A.mode = m;
      A.phi = m == M_S4 ? (const R*)h->l[2] : (const R*)h->field;
      A.tm_phi = h->tm[m == M_S4 ? TM_T4 : TM_FIELD];
      A.out_l = m == M_S1 ? (R*)h->l[0] : m == M_S2 ? (R*)h->l[1] : nullptr;
      A.with_energy = m == M_S1 ? 1 : 0;
    };
    auto time_mode = [&](float& out) -> int {
      int rc = launch(h, A, true);  // warm-up
      if (rc) return rc;
      CK(cudaEventRecord(e0, h->stream));
      for (int i = 0; i < iters && rc == SS_OK; ++i) rc = launch(h, A, true);
      CK(cudaEventRecord(e1, h->stream));
      CK(cudaEventSynchronize(e1));
      float ms = 0.f;
      CK(cudaEventElapsedTime(&ms, e0, e1));
      out = ms / iters;
      return rc;
    };
    const int modes[4] = {M_S1, M_S2, M_S3, M_S4};
    int rc = SS_OK;
    for (int mi = 0; mi < 4 && rc == SS_OK; ++mi) {
      const int m = modes[mi];
      if (m == M_S4) {  // stage 4's inputs from this field, whatever stage 3's variants
        set_mode(M_S3);
        if ((rc = launch(h, A, true))) break;
      }
      set_mode(m);
      // the one-tile-per-CTA variant always (its time enters the fusion decision below),
      // the pipelined one where it exists
      const bool pipe = uses_pipe(m);
      for (int v = 0; v < (pipe ? 2 : 1) && rc == SS_OK; ++v) {
        h->use_pipe[m] = v;
        rc = time_mode(h->tune_ms[m][v]);
      }
      h->use_pipe[m] = (pipe && h->tune_ms[m][1] <= h->tune_ms[m][0]) ? 1 : 0;
    }
    // the energy-only pass must reduce exactly like stage 1 (same grid and tile order)
    h->use_pipe[M_ENERGY] = h->use_pipe[M_S1];
    h->use_pipe[M_GRAD] = h->use_pipe[M_S2];
    // fused stages 2+3 against the two chosen stage kernels
    if (rc == SS_OK) {
      set_mode(M_S23);
      rc = time_mode(h->tune_ms[M_S23][1]);
      if (rc == SS_OK) {
        h->tune_ms[M_S23][0] = h->tune_ms[M_S2][h->use_pipe[M_S2]] + h->tune_ms[M_S3][h->use_pipe[M_S3]];
        h->fuse23 = h->tune_ms[M_S23][1] <= h->tune_ms[M_S23][0] ? 1 : 0;
      }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return rc;
  }

  static int gradient(ss_handle* h, const void* field, void* eg, void* l_out, int raw = 0) {
    FlowArgs<R> A = base_args(h);
    A.mode = M_GRAD;
    A.grad_raw = raw;
    A.phi = (const R*)field;
    A.out_eg = (R*)eg;
    A.out_l = (R*)l_out;
    const bool tma = encode_tile_map(&A.tm_phi, field, sizeof(R), h->G.X, h->G.Y, TH::NF);
    return launch(h, A, tma);
  }

  // dE_h/dphi / dA of the discrete energy sum (true rows, unprojected), optionally
  // minus the flow's functional derivative in the same rows (FP64 fields)
  static int energy_gradient_exact(ss_handle* h, const void* field, double* out, double* q, double* sub) {
    if (sub) {
      int rc = Fused<TH, double>::gradient(h, field, sub, nullptr, 1);
      if (rc) return rc;
    }
    exact_partials_kernel<TH, R><<<grid_1d(h->G.N), 256, 0, h->stream>>>((const R*)field, out, q, h->G, h->P);
    CK(cudaGetLastError());
    exact_transpose_kernel<double><<<grid_1d((long long)TH::NF * h->G.N), 256, 0, h->stream>>>(out, q, sub, TH::NF,
                                                                                              h->G);
    CK(cudaGetLastError());
    return SS_OK;
  }

  // the observable: exact FP64 stencil of the stored values for every precision
  static int energy(ss_handle* h, const void* field) {
    FlowArgs<R> A = base_args(h);
    A.mode = M_ENERGY;
    A.exact_energy = 1;
    A.phi = (const R*)field;
    A.with_energy = 1;
    const bool tma = encode_tile_map(&A.tm_phi, field, sizeof(R), h->G.X, h->G.Y, TH::NF);
    return launch(h, A, tma);
  }

  // FP64 energy of the sphere projection of `field` (element type R).  The FP64 copy
  // goes to the start of the l-buffer region, which holds at least 8 * nf * N bytes
  // for every precision (two FP32 l buffers, or one FP64 one) and is free between steps.
  static int energy_projected(ss_handle* h, const void* field) {
    double* copy = (double*)h->l[0];
    convert_kernel<R, double, TH::NF, TH::NMAG><<<grid_1d(h->G.N), 256, 0, h->stream>>>(
        (const R*)field, copy, h->G.N, TH::CONSTRAINED && h->G.unit_mag);
    CK(cudaGetLastError());
    return Fused<TH, double>::energy(h, copy);
  }

  static int density(ss_handle* h, const void* field, double* dens, bool reduce, int kind, int which) {
    auto k = density_kernel<TH, R, TX, TY, NT>;
    set_smem(k, BUF, smem_done_density);
    k<<<h->nblocks, NT, BUF, h->stream>>>((const R*)field, dens, reduce ? h->partial : nullptr, h->st, kind, which,
                                           h->G, h->P);
    CK(cudaGetLastError());
    return SS_OK;
  }

  static int rk4_stage(ss_handle* h, void* k_out, const void* vel, const void* l_in, void* temp, const void* field,
                       const void* k_prev, double factor) {
    const long long n = (long long)h->nf * h->G.N;
    rk4_stage_kernel<R><<<grid_1d(n), 256, 0, h->stream>>>((R*)k_out, (const R*)vel, (const R*)l_in, (R*)temp,
                                                           (const R*)field, (const R*)k_prev, (R)factor, (R)h->G.dt, n);
    CK(cudaGetLastError());
    return SS_OK;
  }

  static int rk4_finalize(ss_handle* h, void* vel, void* field, const void* const* k, const void* const* l) {
    rk4_finalize_kernel<R, TH::NF, TH::NMAG><<<grid_1d(h->G.N), 256, 0, h->stream>>>(
        (R*)vel, (R*)field, (const R*)k[0], (const R*)k[1], (const R*)k[2], (const R*)k[3], (const R*)l[0],
        (const R*)l[1], (const R*)l[2], (const R*)l[3], h->G.N, TH::CONSTRAINED && h->G.unit_mag);
    CK(cudaGetLastError());
    return SS_OK;
  }
};

template <class TH>
struct Plain {
  static dim3 blocks(const ss_handle* h) { return dim3((h->G.X + 7) / 8, (h->G.Y + 7) / 8); }

  static int gradient(ss_handle* h, const double* F, double* l_out, double* eg) {
    plain_gradient_kernel<TH><<<blocks(h), dim3(8, 8), 0, h->stream>>>(l_out, F, h->d1, h->d2, eg, h->G, h->P);
    CK(cudaGetLastError());
    return SS_OK;
  }

  static int reduce(ss_handle* h, const double* var, long long size, int is_max, double* out) {
    const int nb = (int)((size + 1023) / 1024);
    plain_reduce_kernel<<<nb, 1024, 0, h->stream>>>(var, h->partial, size, is_max);
    CK(cudaGetLastError());
    h->host_partial.resize(nb);
    CK(cudaMemcpyAsync(h->host_partial.data(), h->partial, nb * sizeof(double), cudaMemcpyDeviceToHost, h->stream));
    CK(cudaStreamSynchronize(h->stream));
    double r = is_max ? -INFINITY : 0.0;
    for (int i = 0; i < nb; ++i) r = is_max ? std::max(r, h->host_partial[i]) : r + h->host_partial[i];
    *out = r;
    return SS_OK;
  }

  // observables.compute_energy (e.g. theories/chiral_magnet/observables.py:15-57)
  static int energy(ss_handle* h, const double* F, double* out) {
    plain_energy_kernel<TH><<<blocks(h), dim3(8, 8), 0, h->stream>>>(h->en, F, h->d1, h->G, h->P);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->stream));
    CK(cudaMemcpyAsync(h->entmp, h->en, h->G.N * sizeof(double), cudaMemcpyDeviceToDevice, h->stream));
    int rc = reduce(h, h->entmp, h->G.N, 0, out);
    if (rc) return rc;
    CK(cudaMemsetAsync(h->entmp, 0, h->G.N * sizeof(double), h->stream));
    CK(cudaMemsetAsync(h->en, 0, h->G.N * sizeof(double), h->stream));
    return SS_OK;
  }

  // do_arrested_newton_flow (core/integrator.py:217-348), one host-driven step at a time
  static int step(ss_handle* h, int n, double prev, double* E_host, double* err_host) {
    double* F = (double*)h->field;
    double* V = (double*)h->vel;
    double** k = (double**)h->k;
    double** l = (double**)h->l;
    double* T = (double*)h->temp;
    double* EG = (double*)h->eg;
    const long long nfN = (long long)h->nf * h->G.N;
    double E = std::isnan(prev) ? h->E_last_host : prev;
    const double factors[4] = {0.0, 0.5, 0.5, 1.0};
    for (int s = 0; s < n; ++s) {
      for (int st = 0; st < 4; ++st) {
        const double* l_in = st == 0 ? V : l[st - 1];
        const double* k_prev = st == 0 ? F : k[st - 1];
        rk4_stage_kernel<double><<<grid_1d(nfN), 256, 0, h->stream>>>(k[st], V, l_in, T, F, k_prev, factors[st],
                                                                          h->G.dt, nfN);
        CK(cudaGetLastError());
        int rc = gradient(h, T, l[st], EG);
        if (rc) return rc;
      }
      rk4_finalize_kernel<double, TH::NF, TH::NMAG><<<grid_1d(h->G.N), 256, 0, h->stream>>>(
          V, F, k[0], k[1], k[2], k[3], l[0], l[1], l[2], l[3], h->G.N, TH::CONSTRAINED && h->G.unit_mag);
      CK(cudaGetLastError());
      CK(cudaStreamSynchronize(h->stream));
      double E_new = 0.0;
      int rc = energy(h, F, &E_new);
      if (rc) return rc;
      if (h->G.killkinen && E_new > E) {
        CK(cudaMemsetAsync(V, 0, nfN * sizeof(double), h->stream));
        CK(cudaStreamSynchronize(h->stream));
      }
      double err = 0.0;
      if ((rc = reduce(h, EG, nfN, 1, &err))) return rc;
      E = E_new;
      if (E_host) E_host[s] = E;
      if (err_host) err_host[s] = err;
      if (!std::isfinite(E)) {
        h->E_last_host = E;
        return fail(SS_ERR_NONFINITE, "non-finite energy at step %d", s);
      }
    }
    h->E_last_host = E;
    return SS_OK;
  }
};

// ---------------------------------------------------------------------------
// dispatch tables
// ---------------------------------------------------------------------------
template <class Fn>
int dispatch(const ss_handle* h, Fn&& fn) {
  switch (h->theory) {
    case SS_THEORY_CHIRAL_MAGNET: return fn((ChiralMagnet*)nullptr);
    case SS_THEORY_BABY_SKYRME: return fn((BabySkyrme*)nullptr);
    case SS_THEORY_GINZBURG_LANDAU: return fn((GinzburgLandau*)nullptr);
    case SS_THEORY_ANISOTROPIC: return fn((Anisotropic*)nullptr);
  }
  return fail(SS_ERR_ARG, "bad theory");
}

int read_state(ss_handle* h, StepState* out) {
  CK(cudaMemcpyAsync(out, h->st, sizeof(StepState), cudaMemcpyDeviceToHost, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  return SS_OK;
}

// error of a nonzero device status (read by the caller), which is cleared on the device
int status_error(ss_handle* h, int status) {
  const int zero = 0;
  CK(cudaMemcpyAsync(&h->st->status, &zero, sizeof(int), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  if (status == SS_ERR_TIMEOUT)
    return fail(SS_ERR_TIMEOUT, "a device-side wait timed out; re-bind the handle before further use");
  return fail(SS_ERR_NONFINITE, "a reduction produced a non-finite value");
}

int take_status(ss_handle* h) {
  StepState s;
  int rc = read_state(h, &s);
  if (rc) return rc;
  return s.status ? status_error(h, s.status) : SS_OK;
}

int fused_density(ss_handle* h, const void* field, double* dens, bool reduce, int kind, int which) {
  return dispatch(h, [&](auto* tag) -> int {
    using TH = std::remove_pointer_t<decltype(tag)>;
    if (h->precision == SS_FP32) return Fused<TH, float>::density(h, field, dens, reduce, kind, which);
    return Fused<TH, double>::density(h, field, dens, reduce, kind, which);
  });
}

bool theory_has_charge(int theory, int which) {
  switch (theory) {
    case SS_THEORY_CHIRAL_MAGNET: return ChiralMagnet::has_charge(which);
    case SS_THEORY_BABY_SKYRME: return BabySkyrme::has_charge(which);
    case SS_THEORY_GINZBURG_LANDAU: return GinzburgLandau::has_charge(which);
    case SS_THEORY_ANISOTROPIC: return Anisotropic::has_charge(which);
  }
  return false;
}

bool theory_has_coupling(int theory, int which) {
  switch (theory) {
    case SS_THEORY_CHIRAL_MAGNET: return ChiralMagnet::has_coupling(which);
    case SS_THEORY_BABY_SKYRME: return BabySkyrme::has_coupling(which);
    case SS_THEORY_GINZBURG_LANDAU: return GinzburgLandau::has_coupling(which);
    case SS_THEORY_ANISOTROPIC: return Anisotropic::has_coupling(which);
  }
  return false;
}

int scalar_result(ss_handle* h, double* out) {
  StepState s;
  int rc = read_state(h, &s);
  if (rc) return rc;
  *out = s.scalar;
  if (s.status) return take_status(h);
  return SS_OK;
}

}  // namespace

// ===========================================================================
// exported entry points
// ===========================================================================
extern "C" {

int ss_abi_version(void) { return SS_ABI_VERSION; }

const char* ss_status_string(int status) {
  switch (status) {
    case SS_OK: return "ok";
    case SS_ERR_ARG: return "invalid argument";
    case SS_ERR_CUDA: return "CUDA error";
    case SS_ERR_NONFINITE: return "non-finite value";
    case SS_ERR_STATE: return "invalid call order";
    case SS_ERR_WORKSPACE: return "workspace too small or misaligned";
    case SS_ERR_TIMEOUT: return "device-side wait timed out";
  }
  return "unknown status";
}

const char* ss_last_error(void) { return g_err; }

int ss_create(int theory, const int32_t* p_i, int n_i, const double* p_f, int n_f, int precision, ss_handle** out) {
  if (!out) return fail(SS_ERR_ARG, "out must not be NULL");
  *out = nullptr;
  if (precision != SS_FP64 && precision != SS_FP32 && precision != SS_PLAIN_FP64)
    return fail(SS_ERR_ARG, "unknown precision %d", precision);
  ss_handle* h = new ss_handle();
  h->theory = theory;
  h->precision = precision;
  int rc = decode(h, theory, p_i, n_i, p_f, n_f);
  if (rc) {
    delete h;
    return rc;
  }
  h->elem = precision == SS_FP32 ? 4 : 8;
  const long long tiles = (long long)((h->G.X + TX - 1) / TX) * ((h->G.Y + TY - 1) / TY);
  if (tiles > 0x7fffffffLL) {
    delete h;
    return fail(SS_ERR_ARG, "lattice too large");
  }
  h->nblocks = (int)tiles;
  h->plain_sum_blocks = (int)((h->G.N + 1023) / 1024);
  h->plain_max_blocks = (int)((h->G.N * h->nf + 1023) / 1024);
  *out = h;
  return SS_OK;
}

int ss_destroy(ss_handle* h) {
  delete h;
  return SS_OK;
}

int ss_workspace_bytes(const ss_handle* h, size_t* bytes) {
  if (!h || !bytes) return fail(SS_ERR_ARG, "NULL argument");
  ss_handle tmp = *h;
  tmp.graph = nullptr;  // the copy must not own the original's graph or staging
  tmp.host_stage = nullptr;
  tmp.host_stage_dev = nullptr;
  *bytes = layout(&tmp, nullptr);
  return SS_OK;
}

int ss_bind(ss_handle* h, void* field, void* velocity, void* workspace, size_t workspace_bytes, void* stream) {
  if (!h) return fail(SS_ERR_ARG, "NULL handle");
  if (!workspace) return fail(SS_ERR_ARG, "workspace must not be NULL");
  if (((uintptr_t)workspace) % ALIGN) return fail(SS_ERR_WORKSPACE, "workspace must be %zu-byte aligned", ALIGN);
  size_t need = 0;
  ss_workspace_bytes(h, &need);
  if (workspace_bytes < need) return fail(SS_ERR_WORKSPACE, "workspace has %zu bytes, needs %zu", workspace_bytes, need);
  h->field = field;
  h->vel = velocity;
  h->ws = (char*)workspace;
  h->ws_bytes = workspace_bytes;
  h->stream = (cudaStream_t)stream;
  layout(h, h->ws);
  StepState init;
  memset(&init, 0, sizeof(init));
  init.E_last = NAN;
  CK(cudaMemcpyAsync(h->st, &init, sizeof(init), cudaMemcpyHostToDevice, h->stream));
  CK(cudaStreamSynchronize(h->stream));
  h->E_last_host = NAN;
  h->tma = false;
  if (h->precision != SS_PLAIN_FP64 && field && velocity) {
    const void* bufs[TM_COUNT] = {field, velocity, h->l[0], h->l[2], h->cp_buf, h->cv_buf};
    bool ok = true;
    for (int i = 0; i < TM_COUNT && ok; ++i)
      ok = encode_tile_map(&h->tm[i], bufs[i], h->elem, h->G.X, h->G.Y, h->nf, i >= TM_CP);
    h->tma = ok;
  }
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) == cudaSuccess &&
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess && sms > 0)
    h->num_sms = sms;
  return SS_OK;
}

int ss_tma_enabled(const ss_handle* h) { return h && h->tma ? 1 : 0; }

int ss_autotune(ss_handle* h, int iters, float* ms_out) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (!h->field || !h->vel) return fail(SS_ERR_STATE, "no Field/Velocity bound");
  if (h->precision == SS_PLAIN_FP64) return SS_OK;
  if (iters < 1) iters = 1;
  rc = dispatch(h, [&](auto* tag) -> int {
    using TH = std::remove_pointer_t<decltype(tag)>;
    if (h->precision == SS_FP32) return Fused<TH, float>::autotune(h, iters);
    return Fused<TH, double>::autotune(h, iters);
  });
  if (rc) return rc;
  if (ms_out)
    for (int m = 0; m < N_FLOW_MODES; ++m) {
      ms_out[2 * m] = h->tune_ms[m][0];
      ms_out[2 * m + 1] = h->tune_ms[m][1];
    }
  return take_status(h);
}

int ss_debug_wait_timeout(ss_handle* h, long long wait_cycles, int inject) {
  if (!h) return fail(SS_ERR_ARG, "NULL handle");
  if (wait_cycles <= 0) return fail(SS_ERR_ARG, "wait_cycles must be positive");
  h->wait_cycles = wait_cycles;
  h->inject_timeout = inject ? 1 : 0;
  return SS_OK;
}

int ss_get_variant(const ss_handle* h, int mode) {
  if (!h || mode < 0 || mode > 6) return -1;
  if (mode == M_S23) return h->fuse23;
  return h->use_pipe[mode];
}

int ss_set_variant(ss_handle* h, int mode, int variant) {
  if (!h) return fail(SS_ERR_ARG, "NULL handle");
  if (mode < 0 || mode > 6 || mode == 5)
    return fail(SS_ERR_ARG, "mode %d: 0 (gradient), 1..4 (stages) or 6 (stages 2+3 fused); the energy pass follows "
                "stage 1", mode);
  if (variant != 0 && variant != 1) return fail(SS_ERR_ARG, "variant %d: 0 (one tile per CTA) or 1 (pipelined)", variant);
  if (h->precision == SS_PLAIN_FP64) return fail(SS_ERR_ARG, "the plain FP64 form has no staging variants");
  if (mode == M_S23) {  // 1: stages 2 and 3 in one kernel (used with TMA staging), 0: two kernels
    h->fuse23 = variant;
    return SS_OK;
  }
  if (variant == 1) {
    if (!h->tma) return fail(SS_ERR_STATE, "the pipelined variant needs TMA-staged buffers (bind first; rows of 16-byte multiples)");
    const bool ok = dispatch(h, [&](auto* tag) -> int {
      using TH = std::remove_pointer_t<decltype(tag)>;
      return h->precision == SS_FP32 ? Fused<TH, float>::uses_pipe(mode) : Fused<TH, double>::uses_pipe(mode);
    }) != 0;
    if (!ok) return fail(SS_ERR_ARG, "no pipelined variant of mode %d for this theory and precision", mode);
  }
  h->use_pipe[mode] = variant;
  if (mode == M_S1) h->use_pipe[M_ENERGY] = variant;  // the energy pass reduces exactly like stage 1
  return SS_OK;
}

int ss_step_async(ss_handle* h, int n_steps, double prev_energy, double* energy_traj_dev, double* err_traj_dev) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (n_steps < 0) return fail(SS_ERR_ARG, "n_steps must be >= 0");
  if (!h->field || !h->vel) return fail(SS_ERR_STATE, "no Field/Velocity bound");
  if (h->precision == SS_PLAIN_FP64)
    return fail(SS_ERR_ARG, "the plain FP64 form arrests on the host; use ss_step");
  return dispatch(h, [&](auto* tag) -> int {
    using TH = std::remove_pointer_t<decltype(tag)>;
    if (h->precision == SS_FP32) return Fused<TH, float>::step(h, n_steps, prev_energy, energy_traj_dev, err_traj_dev);
    return Fused<TH, double>::step(h, n_steps, prev_energy, energy_traj_dev, err_traj_dev);
  });
}

int ss_step(ss_handle* h, int n_steps, double prev_energy, double* energy_traj, double* err_traj) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (n_steps < 0) return fail(SS_ERR_ARG, "n_steps must be >= 0");
  if (!h->field || !h->vel) return fail(SS_ERR_STATE, "no Field/Velocity bound");
  if (h->precision == SS_PLAIN_FP64) {
    return dispatch(h, [&](auto* tag) -> int {
      using TH = std::remove_pointer_t<decltype(tag)>;
      return Plain<TH>::step(h, n_steps, prev_energy, energy_traj, err_traj);
    });
  }
  if (n_steps == 0) return take_status(h);
  // each chunk's trajectories and status are written by the kernels into mapped
  // page-locked memory: one synchronisation per chunk and no copies
  if (!h->host_stage) {
    CK(cudaHostAlloc((void**)&h->host_stage, 2 * TRAJ_CAP * sizeof(double) + 64, cudaHostAllocMapped));
    CK(cudaHostGetDevicePointer((void**)&h->host_stage_dev, h->host_stage, 0));
  }
  double* hE = h->host_stage;
  double* hErr = h->host_stage + TRAJ_CAP;
  volatile int* hstatus = reinterpret_cast<volatile int*>(h->host_stage + 2 * TRAJ_CAP);
  int* dstatus = reinterpret_cast<int*>(h->host_stage_dev + 2 * TRAJ_CAP);
  double prev = prev_energy;
  for (int done = 0; done < n_steps; done += TRAJ_CAP) {
    const int k = std::min(TRAJ_CAP, n_steps - done);
    *hstatus = -1;
    rc = dispatch(h, [&](auto* tag) -> int {
      using TH = std::remove_pointer_t<decltype(tag)>;
      double* dE = h->host_stage_dev;
      double* dErr = h->host_stage_dev + TRAJ_CAP;
      if (h->precision == SS_FP32) return Fused<TH, float>::step(h, k, prev, dE, dErr, dstatus);
      return Fused<TH, double>::step(h, k, prev, dE, dErr, dstatus);
    });
    if (rc) return rc;
    prev = NAN;
    CK(cudaStreamSynchronize(h->stream));
    if (energy_traj) memcpy(energy_traj + done, hE, k * sizeof(double));
    if (err_traj) memcpy(err_traj + done, hErr, k * sizeof(double));
    const int status = *hstatus;
    if (status < 0) return fail(SS_ERR_CUDA, "the step's status was not written");
    if (status) return status_error(h, status);
  }
  return SS_OK;
}

int ss_check_status(ss_handle* h) {
  int rc = check_bound(h);
  if (rc) return rc;
  return take_status(h);
}

int ss_gradient(ss_handle* h, const void* field, void* energy_gradient, void* l_out) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (!field) return fail(SS_ERR_ARG, "field must not be NULL");
  if (h->precision == SS_PLAIN_FP64) {
    return dispatch(h, [&](auto* tag) -> int {
      using TH = std::remove_pointer_t<decltype(tag)>;
      double* eg = energy_gradient ? (double*)energy_gradient : (double*)h->eg;
      double* l = l_out ? (double*)l_out : (double*)h->l[0];
      return Plain<TH>::gradient(h, (const double*)field, l, eg);
    });
  }
  return dispatch(h, [&](auto* tag) -> int {
    using TH = std::remove_pointer_t<decltype(tag)>;
    if (h->precision == SS_FP32) return Fused<TH, float>::gradient(h, field, energy_gradient, l_out);
    return Fused<TH, double>::gradient(h, field, energy_gradient, l_out);
  });
}

int ss_energy_gradient(ss_handle* h, const void* field, void* grad) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (!field || !grad) return fail(SS_ERR_ARG, "NULL argument");
  if (h->precision == SS_PLAIN_FP64) return fail(SS_ERR_ARG, "ss_energy_gradient needs SS_FP32 or SS_FP64");
  return dispatch(h, [&](auto* tag) -> int {
    using TH = std::remove_pointer_t<decltype(tag)>;
    if (h->precision == SS_FP32) return Fused<TH, float>::gradient(h, field, grad, nullptr, 1);
    return Fused<TH, double>::gradient(h, field, grad, nullptr, 1);
  });
}

int ss_energy_density(ss_handle* h, const void* field, double* density) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (!field || !density) return fail(SS_ERR_ARG, "NULL argument");
  return fused_density(h, field, density, false, D_ENERGY, 0);
}

int ss_energy(ss_handle* h, const void* field, double* out) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (!field || !out) return fail(SS_ERR_ARG, "NULL argument");
  if (h->precision == SS_PLAIN_FP64) {
    return dispatch(h, [&](auto* tag) -> int {
      using TH = std::remove_pointer_t<decltype(tag)>;
      return Plain<TH>::energy(h, (const double*)field, out);
    });
  }
  rc = dispatch(h, [&](auto* tag) -> int {
    using TH = std::remove_pointer_t<decltype(tag)>;
    if (h->precision == SS_FP32) return Fused<TH, float>::energy(h, field);
    return Fused<TH, double>::energy(h, field);
  });
  if (rc) return rc;
  return scalar_result(h, out);
}

namespace {
int launch_init(ss_handle* h, void* field, void* velocity, const InitArgs& A) {
  const long long N = (long long)A.X * A.Y;
  const unsigned blocks = (unsigned)((N + 255) / 256);
  auto go = [&](auto* tag) -> int {
    using R = std::remove_pointer_t<decltype(tag)>;
    R* F = (R*)field;
    R* V = (R*)velocity;
    switch (h->theory) {
      case 0: init_kernel<0, R><<<blocks, 256, 0, h->stream>>>(F, V, A); break;
      case 1: init_kernel<1, R><<<blocks, 256, 0, h->stream>>>(F, V, A); break;
      case 2: init_kernel<2, R><<<blocks, 256, 0, h->stream>>>(F, V, A); break;
      default: init_kernel<3, R><<<blocks, 256, 0, h->stream>>>(F, V, A); break;
    }
    CK(cudaGetLastError());
    return SS_OK;
  };
  return h->precision == SS_FP32 ? go((float*)nullptr) : go((double*)nullptr);
}

InitArgs init_args(const ss_handle* h, int mode) {
  InitArgs A;
  memset(&A, 0, sizeof(A));
  A.X = h->G.X;
  A.Y = h->G.Y;
  A.nf = h->nf;
  A.mode = mode;
  for (int i = 0; i < 32; ++i) A.pf[i] = h->pf_raw[i];
  return A;
}
}  // namespace

int ss_initialize(ss_handle* h, void* field, void* velocity, int mode, int ansatz, double rotation,
                  double vortex_number) {
  if (!h || !field) return fail(SS_ERR_ARG, "handle and field must not be NULL");
  if (mode != SS_INIT_GROUND && mode != SS_INIT_ANSATZ) return fail(SS_ERR_ARG, "unknown init mode %d", mode);
  if (ansatz < SS_ANSATZ_NONE || ansatz > SS_ANSATZ_ANTI) return fail(SS_ERR_ARG, "unknown ansatz %d", ansatz);
  InitArgs A = init_args(h, mode == SS_INIT_GROUND ? IM_GROUND : IM_ANSATZ);
  A.ansatz = ansatz;
  A.rotation = rotation;
  A.vortex_number = vortex_number;
  return launch_init(h, field, velocity, A);
}

int ss_insert_soliton(ss_handle* h, void* field, int pxi, int pxj, int ansatz, int vortex, double rotation) {
  if (!h || !field) return fail(SS_ERR_ARG, "handle and field must not be NULL");
  if (ansatz < SS_ANSATZ_NONE || ansatz > SS_ANSATZ_ANTI) return fail(SS_ERR_ARG, "unknown ansatz %d", ansatz);
  if (pxi < 0 || pxi >= h->G.X || pxj < 0 || pxj >= h->G.Y) return SS_OK;  // the reference's kernels ignore it
  InitArgs A = init_args(h, IM_INSERT);
  A.ansatz = ansatz;
  A.vortex = vortex ? 1 : 0;
  A.rotation = rotation;
  A.pxi = pxi;
  A.pxj = pxj;
  return launch_init(h, field, nullptr, A);
}

int ss_text_workspace_bytes(long long n, size_t* bytes) {
  if (!bytes || n < 0) return fail(SS_ERR_ARG, "bad arguments");
  const long long nb = (n + 1023) / 1024;
  *bytes = (size_t)(n + nb + 8) * sizeof(long long);
  return SS_OK;
}

int ss_format_text(const void* values, int precision, long long n, int digits, long long row, long long block,
                   char* out, size_t out_cap, long long* out_len, void* workspace, size_t workspace_bytes,
                   void* stream) {
  if (!values || !out_len || !workspace) return fail(SS_ERR_ARG, "values, out_len and workspace must not be NULL");
  if (precision != SS_FP32 && precision != SS_FP64) return fail(SS_ERR_ARG, "precision must be SS_FP32 or SS_FP64");
  if (n <= 0) return fail(SS_ERR_ARG, "n must be positive");
  if (digits < 1 || digits > TXT_MAX_P) return fail(SS_ERR_ARG, "digits must be 1..%d", TXT_MAX_P);
  if (row < 0 || block < 0) return fail(SS_ERR_ARG, "row and block must be >= 0");
  size_t need = 0;
  ss_text_workspace_bytes(n, &need);
  if (workspace_bytes < need) return fail(SS_ERR_WORKSPACE, "workspace of %zu bytes, need %zu", workspace_bytes, need);
  if ((reinterpret_cast<uintptr_t>(workspace) & 7u) != 0) return fail(SS_ERR_WORKSPACE, "workspace must be 8-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  const long long nb = (n + 1023) / 1024;
  long long* off = (long long*)workspace;
  long long* sums = off + n;
  long long* total = sums + nb;
  const TextLayout L{n, row, block, digits};
  const unsigned g256 = (unsigned)((n + 255) / 256);
  if (precision == SS_FP32) text_len_kernel<float><<<g256, 256, 0, st>>>((const float*)values, L, off);
  else text_len_kernel<double><<<g256, 256, 0, st>>>((const double*)values, L, off);
  scan_block_kernel<<<(unsigned)nb, 1024, 0, st>>>(off, n, sums);
  scan_sums_kernel<<<1, 1024, 0, st>>>(sums, nb, total);
  scan_add_kernel<<<(unsigned)nb, 1024, 0, st>>>(off, n, sums);
  CK(cudaGetLastError());
  long long len = 0;
  CK(cudaMemcpyAsync(&len, total, sizeof(len), cudaMemcpyDeviceToHost, st));
  CK(cudaStreamSynchronize(st));
  *out_len = len;
  if (!out) return SS_OK;  // size query
  if ((size_t)len > out_cap) return fail(SS_ERR_ARG, "text of %lld bytes does not fit the %zu-byte buffer", len, out_cap);
  if (precision == SS_FP32) text_write_kernel<float><<<g256, 256, 0, st>>>((const float*)values, L, off, out);
  else text_write_kernel<double><<<g256, 256, 0, st>>>((const double*)values, L, off, out);
  CK(cudaGetLastError());
  return SS_OK;
}

int ss_render_rgba(int kind, const void* src, int precision, int xlen, int ylen, double vmin, double vmax,
                   unsigned char* rgba, void* stream) {
  if (!src || !rgba) return fail(SS_ERR_ARG, "src and rgba must not be NULL");
  if (kind < SS_RENDER_JET || kind > SS_RENDER_MAGNETIZATION) return fail(SS_ERR_ARG, "unknown render kind %d", kind);
  if (precision != SS_FP32 && precision != SS_FP64)
    return fail(SS_ERR_ARG, "precision must be SS_FP32 or SS_FP64 (element type of src)");
  if (xlen <= 0 || ylen <= 0) return fail(SS_ERR_ARG, "xlen and ylen must be positive");
  if ((reinterpret_cast<uintptr_t>(rgba) & 3u) != 0) return fail(SS_ERR_ARG, "rgba must be 4-byte aligned");
  const dim3 grid((unsigned)((ylen + 31) / 32), (unsigned)((xlen + 31) / 32)), block(32, 8);
  if (grid.y > 65535u) return fail(SS_ERR_ARG, "xlen %d too large (at most %d)", xlen, 65535 * 32);
  cudaStream_t s = (cudaStream_t)stream;
  uint32_t* out = reinterpret_cast<uint32_t*>(rgba);
  auto go = [&](auto* tag) {
    using T = std::remove_pointer_t<decltype(tag)>;
    const T* p = (const T*)src;
    if (kind == SS_RENDER_JET) render_kernel<T, RK_JET><<<grid, block, 0, s>>>(p, xlen, ylen, vmin, vmax, out);
    else if (kind == SS_RENDER_GRAY) render_kernel<T, RK_GRAY><<<grid, block, 0, s>>>(p, xlen, ylen, vmin, vmax, out);
    else render_kernel<T, RK_MAGNETIZATION><<<grid, block, 0, s>>>(p, xlen, ylen, vmin, vmax, out);
  };
  if (precision == SS_FP32) go((float*)nullptr); else go((double*)nullptr);
  CK(cudaGetLastError());
  return SS_OK;
}

int ss_energy_projected(ss_handle* h, const void* field, double* out) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (!field || !out) return fail(SS_ERR_ARG, "NULL argument");
  rc = dispatch(h, [&](auto* tag) -> int {
    using TH = std::remove_pointer_t<decltype(tag)>;
    if (h->precision == SS_FP32) return Fused<TH, float>::energy_projected(h, field);
    return Fused<TH, double>::energy_projected(h, field);
  });
  if (rc) return rc;
  return scalar_result(h, out);
}

int ss_charge_density(ss_handle* h, const void* field, int which, double* density) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (!field || !density) return fail(SS_ERR_ARG, "NULL argument");
  if (!theory_has_charge(h->theory, which)) return fail(SS_ERR_ARG, "charge %d not defined for theory %d", which, h->theory);
  return fused_density(h, field, density, false, D_CHARGE, which);
}

int ss_charge(ss_handle* h, const void* field, int which, double* out) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (!field || !out) return fail(SS_ERR_ARG, "NULL argument");
  if (!theory_has_charge(h->theory, which)) return fail(SS_ERR_ARG, "charge %d not defined for theory %d", which, h->theory);
  rc = fused_density(h, field, nullptr, true, D_CHARGE, which);
  if (rc) return rc;
  return scalar_result(h, out);
}

int ss_coupling_grad(ss_handle* h, const void* field, int coupling, double* out) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (!field || !out) return fail(SS_ERR_ARG, "NULL argument");
  if (!theory_has_coupling(h->theory, coupling))
    return fail(SS_ERR_ARG, "coupling %d not defined for theory %d", coupling, h->theory);
  rc = fused_density(h, field, nullptr, true, D_COUPLING, coupling);
  if (rc) return rc;
  return scalar_result(h, out);
}

int ss_convert_field(ss_handle* h, const void* src, int src_precision, void* dst, int dst_precision, int project) {
  if (!h || !src || !dst) return fail(SS_ERR_ARG, "NULL argument");
  auto is_prec = [](int p) { return p == SS_FP32 || p == SS_FP64 || p == SS_PLAIN_FP64; };
  if (!is_prec(src_precision) || !is_prec(dst_precision)) return fail(SS_ERR_ARG, "unknown precision");
  const bool s32 = src_precision == SS_FP32, d32 = dst_precision == SS_FP32;
  if (src == dst && s32 != d32) return fail(SS_ERR_ARG, "in-place conversion needs equal element types");
  return dispatch(h, [&](auto* tag) -> int {
    using TH = std::remove_pointer_t<decltype(tag)>;
    const int norm = project && TH::CONSTRAINED && h->G.unit_mag;
    const dim3 g = grid_1d(h->G.N);
    if (s32 && d32) convert_kernel<float, float, TH::NF, TH::NMAG><<<g, 256, 0, h->stream>>>((const float*)src, (float*)dst, h->G.N, norm);
    else if (s32) convert_kernel<float, double, TH::NF, TH::NMAG><<<g, 256, 0, h->stream>>>((const float*)src, (double*)dst, h->G.N, norm);
    else if (d32) convert_kernel<double, float, TH::NF, TH::NMAG><<<g, 256, 0, h->stream>>>((const double*)src, (float*)dst, h->G.N, norm);
    else convert_kernel<double, double, TH::NF, TH::NMAG><<<g, 256, 0, h->stream>>>((const double*)src, (double*)dst, h->G.N, norm);
    CK(cudaGetLastError());
    return SS_OK;
  });
}

int ss_energy_gradient_exact(ss_handle* h, const void* field, double* out, int minus_stencil) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (!field || !out) return fail(SS_ERR_ARG, "NULL argument");
  if (h->precision == SS_PLAIN_FP64) return fail(SS_ERR_ARG, "ss_energy_gradient_exact needs SS_FP32 or SS_FP64");
  if (minus_stencil && h->precision != SS_FP64)
    return fail(SS_ERR_ARG, "the residual against the stencil gradient needs SS_FP64 fields");
  const size_t nfN = (size_t)h->nf * (size_t)h->G.N;
  const size_t q_bytes = align_up(2 * nfN * sizeof(double));
  const size_t need = q_bytes + (minus_stencil ? nfN * sizeof(double) : 0);
  char* region = (char*)h->l[0];
  if (!region || region + need > h->ws + h->ws_bytes)
    return fail(SS_ERR_WORKSPACE, "the workspace's flow buffers (%zu bytes) cannot hold the %zu bytes of scratch",
                (size_t)(h->ws + h->ws_bytes - region), need);
  double* q = (double*)region;
  double* sub = minus_stencil ? (double*)(region + q_bytes) : nullptr;
  return dispatch(h, [&](auto* tag) -> int {
    using TH = std::remove_pointer_t<decltype(tag)>;
    if (h->precision == SS_FP32) return Fused<TH, float>::energy_gradient_exact(h, field, out, q, sub);
    return Fused<TH, double>::energy_gradient_exact(h, field, out, q, sub);
  });
}

int ss_set_forcing(ss_handle* h, const double* force) {
  if (!h) return fail(SS_ERR_ARG, "NULL handle");
  if (force && h->precision != SS_FP64) return fail(SS_ERR_ARG, "a forcing needs SS_FP64 fields");
  if (((uintptr_t)force) % 16) return fail(SS_ERR_ARG, "the forcing must be 16-byte aligned");
  h->force = force;
  return SS_OK;
}

int ss_field_density(ss_handle* h, const void* field, int kind, double* out) {
  if (!h || !field || !out) return fail(SS_ERR_ARG, "NULL argument");
  const bool ah = h->theory == SS_THEORY_GINZBURG_LANDAU, sid = h->theory == SS_THEORY_ANISOTROPIC;
  const bool ok = (kind == SS_DENSITY_HIGGS && ah) || (kind == SS_DENSITY_SUPERCURRENT && (ah || sid)) ||
                  ((kind == SS_DENSITY_HIGGS1 || kind == SS_DENSITY_HIGGS2 || kind == SS_DENSITY_PHASE_DIFFERENCE ||
                    kind == SS_DENSITY_MAGNETIC_FIELD) && sid);
  if (!ok) return fail(SS_ERR_ARG, "density kind %d not defined for theory %d", kind, h->theory);
  const double q = ah ? h->P.c[0] : h->P.c[1];
  if (h->precision == SS_FP32)
    field_density_kernel<float><<<grid_1d(h->G.N), 256, 0, h->stream>>>((const float*)field, out, kind, h->G, q);
  else
    field_density_kernel<double><<<grid_1d(h->G.N), 256, 0, h->stream>>>((const double*)field, out, kind, h->G, q);
  CK(cudaGetLastError());
  return SS_OK;
}

int ss_rk4_stage(ss_handle* h, void* k_out, const void* velocity, const void* l_in, void* temp, const void* field,
                 const void* k_prev, double factor) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (!k_out || !velocity || !l_in || !temp || !field || !k_prev) return fail(SS_ERR_ARG, "NULL argument");
  return dispatch(h, [&](auto* tag) -> int {
    using TH = std::remove_pointer_t<decltype(tag)>;
    if (h->precision == SS_FP32) return Fused<TH, float>::rk4_stage(h, k_out, velocity, l_in, temp, field, k_prev, factor);
    return Fused<TH, double>::rk4_stage(h, k_out, velocity, l_in, temp, field, k_prev, factor);
  });
}

int ss_rk4_finalize(ss_handle* h, void* velocity, void* field, const void* k1, const void* k2, const void* k3,
                    const void* k4, const void* l1, const void* l2, const void* l3, const void* l4) {
  int rc = check_bound(h);
  if (rc) return rc;
  const void* k[4] = {k1, k2, k3, k4};
  const void* l[4] = {l1, l2, l3, l4};
  for (int i = 0; i < 4; ++i)
    if (!k[i] || !l[i]) return fail(SS_ERR_ARG, "NULL argument");
  if (!velocity || !field) return fail(SS_ERR_ARG, "NULL argument");
  return dispatch(h, [&](auto* tag) -> int {
    using TH = std::remove_pointer_t<decltype(tag)>;
    if (h->precision == SS_FP32) return Fused<TH, float>::rk4_finalize(h, velocity, field, k, l);
    return Fused<TH, double>::rk4_finalize(h, velocity, field, k, l);
  });
}

}  // extern "C"

// ===========================================================================
// Total energy without any allocation.
//
// Some callers cannot allocate device memory at the point where they need an
// energy: hosts whose memory manager owns the whole device and forbids further
// allocations (a framework's caching allocator or a fixed memory pool), and
// interactive loops (a viewer's per-frame callback) that must not call cudaMalloc
// or cudaFree because those synchronise the device and stall the frame.  For them
// ss_energy_noalloc keeps its scratch (the per-block partial sums and the
// reduction state) in the file-scope array below, which every GPU that loads
// this library holds until exit.
// ===========================================================================
namespace {

constexpr size_t NOALLOC_SCRATCH_BYTES = 512 * 1024;   // 256 B state + up to 65504 block partials
__device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];
// Device address of the array, per device.  Host threads calling concurrently on a
// device that has no entry yet may each look it up; they store the same address, and
// the atomic (relaxed ordering suffices) makes those concurrent stores well defined.
std::atomic<void*> g_noalloc_addr[64];

// Device address of the static scratch on the current device (looked up once per device,
// with that device current: in host code the array's name is only a host-side stand-in).
int noalloc_scratch(void** out) {
  int dev = -1;
  CK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) return fail(SS_ERR_ARG, "device ordinal %d out of range", dev);
  void* p = g_noalloc_addr[dev].load(std::memory_order_relaxed);
  if (!p) {
    CK(cudaGetSymbolAddress(&p, g_noalloc_scratch));
    g_noalloc_addr[dev].store(p, std::memory_order_relaxed);
  }
  *out = p;
  return SS_OK;
}

}  // namespace

extern "C" int ss_energy_noalloc(int theory, const int32_t* p_i, int n_i, const double* p_f, int n_f,
                                 int precision, const void* field, double* out, void* stream) {
  if (!field || !out) return fail(SS_ERR_ARG, "field and out must not be NULL");
  if (precision != SS_FP32 && precision != SS_FP64)
    return fail(SS_ERR_ARG, "ss_energy_noalloc supports SS_FP32 and SS_FP64 fields");
  ss_handle h;  // on the stack: decoding the parameters allocates nothing
  h.theory = theory;
  h.precision = precision;
  int rc = decode(&h, theory, p_i, n_i, p_f, n_f);
  if (rc) return rc;
  h.elem = precision == SS_FP32 ? 4 : 8;
  const long long tiles = (long long)((h.G.X + TX - 1) / TX) * ((h.G.Y + TY - 1) / TY);
  const size_t need = 256 + (size_t)tiles * sizeof(double);
  if (need > NOALLOC_SCRATCH_BYTES)
    return fail(SS_ERR_ARG,
                "lattice of %lld tiles (16 x 64 sites each) needs %zu bytes of scratch; the allocation-free "
                "entry point holds %zu (at most %zu tiles)",
                tiles, need, NOALLOC_SCRATCH_BYTES, (NOALLOC_SCRATCH_BYTES - 256) / sizeof(double));
  h.nblocks = (int)tiles;
  h.stream = (cudaStream_t)stream;
  void* scratch = nullptr;
  if ((rc = noalloc_scratch(&scratch))) return rc;
  h.st = (StepState*)scratch;
  h.partial = (double*)((char*)scratch + 256);
  // the last call's contents stay in the array: the reduction state must start at zero
  CK(cudaMemsetAsync(h.st, 0, sizeof(StepState), h.stream));
  rc = dispatch(&h, [&](auto* tag) -> int {
    using TH = std::remove_pointer_t<decltype(tag)>;
    if (precision == SS_FP32) {
      FlowArgs<float> A = Fused<TH, float>::base_args(&h);
      A.mode = M_ENERGY;
      A.exact_energy = 1;
      A.phi = (const float*)field;
      A.with_energy = 1;
      return Fused<TH, float>::template launch_mode<false, M_ENERGY>(&h, A);
    }
    FlowArgs<double> A = Fused<TH, double>::base_args(&h);
    A.mode = M_ENERGY;
    A.phi = (const double*)field;
    A.with_energy = 1;
    return Fused<TH, double>::template launch_mode<false, M_ENERGY>(&h, A);
  });
  if (rc) return rc;
  StepState s;
  CK(cudaMemcpyAsync(&s, h.st, sizeof(StepState), cudaMemcpyDeviceToHost, h.stream));
  CK(cudaStreamSynchronize(h.stream));
  *out = s.scalar;
  if (s.status) return fail(SS_ERR_NONFINITE, "the energy reduction produced a non-finite value");
  return SS_OK;
}


// ===========================================================================
// Batched lattices: many independent relaxations of one theory per launch
// ===========================================================================
// Tile shapes of the batched stage kernels (x rows, y columns, threads): the
// autotuner picks one per size class of lattices (ss_batch_autotune).  Shape 1 exists
// for TMA-staged FP32 batches.
constexpr int N_BATCH_SHAPES = 2;
constexpr int BSHAPE_TX[N_BATCH_SHAPES] = {16, 8};
constexpr int BSHAPE_TY[N_BATCH_SHAPES] = {64, 32};

struct ss_batch {
  int theory = 0, precision = 0, n = 0, nf = 0;
  size_t elem = 4;
  std::vector<ss_handle> inst;   // decoded parameters per lattice (host only)
  std::vector<int> shape;        // tile shape per lattice
  std::vector<int> max_tiles;    // tiles per lattice in its finest shape (partials are sized for it)
  int total_max = 0;             // sum of max_tiles: capacity of each tile list
  int group_tiles[N_BATCH_SHAPES] = {0, 0};  // tiles of the lattices of each shape
  bool tma = false;
  cudaStream_t stream = nullptr;
  char* ws = nullptr;
  BatchInst* d_insts = nullptr;
  int* d_tile_inst[N_BATCH_SHAPES] = {nullptr, nullptr};  // lattice of each tile, per shape group
  int* d_tune_tiles = nullptr;   // a single size class's tiles while the autotuner times it
  float tune_ms[64][N_BATCH_SHAPES] = {};  // autotuner: per size class (first 64) and shape
  double* d_prev = nullptr;
  std::vector<BatchInst> h_insts;
  std::vector<void*> fields, vels;
  long long wait_cycles = WAIT_CYCLES;
  cudaGraphExec_t graph = nullptr;
  // per-lattice step states and trajectory rows, contiguous in the workspace (lattice i:
  // d_st[i], d_E / d_err rows i * TRAJ_CAP), so that one copy returns each for all lattices
  StepState* d_st = nullptr;
  double* d_E = nullptr;
  double* d_err = nullptr;
  char* h_stage = nullptr;  // page-locked staging of those copies (first ss_batch_step)
  ~ss_batch() {
    if (graph) cudaGraphExecDestroy(graph);
    if (h_stage) cudaFreeHost(h_stage);
  }
};

namespace {

size_t batch_layout(ss_batch* b, char* base) {
  size_t off = 0;
  auto take = [&](size_t bytes) -> char* {
    char* p = base ? base + off : nullptr;
    off = align_up(off + bytes);
    return p;
  };
  b->d_insts = (BatchInst*)take(sizeof(BatchInst) * b->n);
  for (int g = 0; g < N_BATCH_SHAPES; ++g) b->d_tile_inst[g] = (int*)take(sizeof(int) * b->total_max);
  b->d_tune_tiles = (int*)take(sizeof(int) * b->total_max);
  b->d_prev = (double*)take(sizeof(double) * b->n);
  b->d_st = (StepState*)take(sizeof(StepState) * b->n);
  b->d_E = (double*)take(sizeof(double) * TRAJ_CAP * b->n);
  b->d_err = (double*)take(sizeof(double) * TRAJ_CAP * b->n);
  b->h_insts.assign(b->n, BatchInst{});
  for (int i = 0; i < b->n; ++i) {
    BatchInst& I = b->h_insts[i];
    const size_t fb = b->elem * (size_t)b->nf * (size_t)b->inst[i].G.N;
    I.st = b->d_st ? b->d_st + i : nullptr;
    I.partial = (double*)take(sizeof(double) * b->max_tiles[i]);
    I.E_traj = b->d_E ? b->d_E + (size_t)i * TRAJ_CAP : nullptr;
    I.err_traj = b->d_err ? b->d_err + (size_t)i * TRAJ_CAP : nullptr;
    for (int k = BB_CP; k < BB_COUNT; ++k) I.buf[k] = take(fb);
  }
  return off;
}

template <class TH, typename R>
struct Batched {
  // one launch over the tiles of `tile_inst` (lattices of one tile shape)
  template <int BTX, int BTY, int BNT, bool TMA_, int MODE>
  static int launch_shape(const ss_batch* b, const BatchStep& B, const int* tile_inst, int ntiles) {
    if (ntiles <= 0) return SS_OK;
    constexpr size_t BUF = tile_buf_bytes<R, TH::NF, BTX, BTY>();
    constexpr size_t smem = TMA_ ? flow_buffers(MODE) * BUF : BUF;
    constexpr int NTM = smem > 113 * 1024 ? 2 * BNT : BNT;  // as Fused::flow_threads
    auto k = batch_flow_kernel<TH, R, BTX, BTY, NTM, TMA_, MODE>;
    static unsigned long long smem_done = 0;  // one per instantiation
    set_smem(k, smem, smem_done);
    k<<<ntiles, NTM, smem, b->stream>>>(b->d_insts, tile_inst, B);
    CK(cudaGetLastError());
    return SS_OK;
  }
  // a stage over every shape group (shape 1: TMA-staged FP32 batches only)
  template <int MODE>
  static int launch(const ss_batch* b, const BatchStep& B) {
    int rc;
    if constexpr (MODE == M_S23) {  // needs TMA staging
      rc = launch_shape<16, 64, NT, true, MODE>(b, B, b->d_tile_inst[0], b->group_tiles[0]);
    } else {
      rc = b->tma ? launch_shape<16, 64, NT, true, MODE>(b, B, b->d_tile_inst[0], b->group_tiles[0])
                  : launch_shape<16, 64, NT, false, MODE>(b, B, b->d_tile_inst[0], b->group_tiles[0]);
    }
    if (rc) return rc;
    if constexpr (sizeof(R) == 4) {
      if (b->tma && b->group_tiles[1] > 0)
        rc = launch_shape<8, 32, 128, true, MODE>(b, B, b->d_tile_inst[1], b->group_tiles[1]);
    }
    return rc;
  }

  static int step(ss_batch* b, int n, bool use_prev) {
    if (n <= 0) return SS_OK;
    BatchStep B;
    memset(&B, 0, sizeof(B));
    B.wait_cycles = b->wait_cycles;
    int rc;
    for (int s = 0; s < n; ++s) {
      B.with_energy = s > 0;
      B.arrest_update = s > 0;
      B.init_state = s == 0;
      B.prev_energy = (s == 0 && use_prev) ? b->d_prev : nullptr;
      B.E_idx = s - 1;
      B.err_idx = -1;
      if ((rc = launch<M_S1>(b, B))) return rc;
      B.with_energy = B.arrest_update = B.init_state = 0;
      B.prev_energy = nullptr;
      B.E_idx = -1;
      if (b->tma) {  // stages 2 and 3 fused (one staging of phi, V, l1)
        if ((rc = launch<M_S23>(b, B))) return rc;
      } else {
        if ((rc = launch<M_S2>(b, B))) return rc;
        if ((rc = launch<M_S3>(b, B))) return rc;
      }
      B.err_idx = s;
      if ((rc = launch<M_S4>(b, B))) return rc;  // in place
      B.err_idx = -1;
    }
    B.with_energy = B.arrest_update = 1;
    B.E_idx = n - 1;
    if ((rc = launch<M_ENERGY>(b, B))) return rc;
    batch_finish_kernel<R, TH::NF><<<dim3(64, b->n), 256, 0, b->stream>>>(b->d_insts);
    CK(cudaGetLastError());
    return SS_OK;
  }

  // The stage launches of one step with every reduction, trajectory and arrest update
  // off: reads the current fields, writes only workspace scratch (l1, l2, T4, cV, cP,
  // and stage 4's phi' and V' into l1 and l2).
  static int timing_step(ss_batch* b) {
    BatchStep B;
    memset(&B, 0, sizeof(B));
    B.wait_cycles = b->wait_cycles;
    B.E_idx = -1;
    B.err_idx = -1;
    int rc = launch<M_S1>(b, B);
    if (!rc) rc = b->tma ? launch<M_S23>(b, B) : launch<M_S2>(b, B);
    if (!rc && !b->tma) rc = launch<M_S3>(b, B);
    B.scratch_out = 1;
    if (!rc) rc = launch<M_S4>(b, B);
    return rc;
  }
};

template <class Fn>
int batch_dispatch(const ss_batch* b, Fn&& fn) {
  switch (b->theory) {
    case SS_THEORY_CHIRAL_MAGNET: return fn((ChiralMagnet*)nullptr);
    case SS_THEORY_BABY_SKYRME: return fn((BabySkyrme*)nullptr);
    case SS_THEORY_GINZBURG_LANDAU: return fn((GinzburgLandau*)nullptr);
    case SS_THEORY_ANISOTROPIC: return fn((Anisotropic*)nullptr);
  }
  return fail(SS_ERR_ARG, "bad theory");
}

// tiles of a lattice in tile shape `shape`
long long batch_tiles(const Grid& G, int shape) {
  return (long long)((G.X + BSHAPE_TX[shape] - 1) / BSHAPE_TX[shape]) * ((G.Y + BSHAPE_TY[shape] - 1) / BSHAPE_TY[shape]);
}

// TMA maps of lattice i for its current tile shape (buffers already set); false when
// a buffer or its row pitch is not 16-byte aligned
bool batch_encode(ss_batch* b, int i) {
  BatchInst& I = b->h_insts[i];
  const int sh = b->shape[i];
  bool ok = true;
  for (int k = 0; k < BT_COUNT && ok; ++k)
    ok = encode_tile_map(&I.tm[k], I.buf[BATCH_TM_BUF[k]], b->elem, I.G.X, I.G.Y, b->nf, false, BSHAPE_TX[sh],
                         BSHAPE_TY[sh]);
  return ok;
}

// Rebuild the per-shape tile lists from the lattices with include[i] (all when null),
// set each lattice's tile range and copy the descriptors and lists to the device.
int batch_upload(ss_batch* b, const std::vector<char>* include) {
  std::vector<int> lists[N_BATCH_SHAPES];
  for (int i = 0; i < b->n; ++i) {
    BatchInst& I = b->h_insts[i];
    const int sh = b->shape[i];
    I.ntiles = (int)batch_tiles(I.G, sh);
    if (include && !(*include)[i]) {
      I.tile0 = 0;
      continue;
    }
    I.tile0 = (int)lists[sh].size();
    lists[sh].insert(lists[sh].end(), (size_t)I.ntiles, i);
  }
  for (int g = 0; g < N_BATCH_SHAPES; ++g) {
    b->group_tiles[g] = (int)lists[g].size();
    if (!lists[g].empty())
      CK(cudaMemcpyAsync(b->d_tile_inst[g], lists[g].data(), sizeof(int) * lists[g].size(), cudaMemcpyHostToDevice,
                         b->stream));
  }
  CK(cudaMemcpyAsync(b->d_insts, b->h_insts.data(), sizeof(BatchInst) * b->n, cudaMemcpyHostToDevice, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return SS_OK;
}

}  // namespace

extern "C" {

int ss_batch_create(int theory, int n_lattices, const int32_t* p_i, int n_i, const double* p_f, int n_f,
                    int precision, ss_batch** out) {
  if (!out) return fail(SS_ERR_ARG, "out must not be NULL");
  *out = nullptr;
  if (n_lattices < 1) return fail(SS_ERR_ARG, "n_lattices must be >= 1");
  if (precision != SS_FP32 && precision != SS_FP64) return fail(SS_ERR_ARG, "batches support SS_FP32 and SS_FP64");
  ss_batch* b = new ss_batch();
  b->theory = theory;
  b->precision = precision;
  b->n = n_lattices;
  b->elem = precision == SS_FP32 ? 4 : 8;
  b->inst.resize(n_lattices);
  long long total = 0;
  for (int i = 0; i < n_lattices; ++i) {
    ss_handle& h = b->inst[i];
    int rc = decode(&h, theory, p_i + (size_t)i * n_i, n_i, p_f + (size_t)i * n_f, n_f);
    if (rc) {
      char msg[sizeof(g_err)];
      snprintf(msg, sizeof(msg), "%s", g_err);
      delete b;
      return fail(rc, "lattice %d: %s", i, msg);
    }
    // partials and tile lists are sized for the finest shape the precision may use
    const long long t = std::max(batch_tiles(h.G, 0), precision == SS_FP32 ? batch_tiles(h.G, 1) : 0LL);
    b->max_tiles.push_back((int)std::min(t, 0x7fffffffLL));
    total += t;
  }
  if (total > 0x7fffffffLL) {
    delete b;
    return fail(SS_ERR_ARG, "batch too large");
  }
  b->total_max = (int)total;
  b->shape.assign(n_lattices, 0);
  b->nf = b->inst[0].nf;
  *out = b;
  return SS_OK;
}

int ss_batch_destroy(ss_batch* b) {
  delete b;
  return SS_OK;
}

int ss_batch_workspace_bytes(const ss_batch* b, size_t* bytes) {
  if (!b || !bytes) return fail(SS_ERR_ARG, "NULL argument");
  ss_batch tmp = *b;
  tmp.graph = nullptr;  // the copy must not own the original's graph or staging
  tmp.h_stage = nullptr;
  *bytes = batch_layout(&tmp, nullptr);
  return SS_OK;
}

int ss_batch_bind(ss_batch* b, void* const* fields, void* const* velocities, void* workspace, size_t workspace_bytes,
                  void* stream) {
  if (!b || !fields || !velocities || !workspace) return fail(SS_ERR_ARG, "NULL argument");
  if (((uintptr_t)workspace) % ALIGN) return fail(SS_ERR_WORKSPACE, "workspace must be %zu-byte aligned", ALIGN);
  size_t need = 0;
  ss_batch_workspace_bytes(b, &need);
  if (workspace_bytes < need) return fail(SS_ERR_WORKSPACE, "workspace has %zu bytes, needs %zu", workspace_bytes, need);
  b->ws = (char*)workspace;
  b->stream = (cudaStream_t)stream;
  batch_layout(b, b->ws);
  b->fields.assign(fields, fields + b->n);
  b->vels.assign(velocities, velocities + b->n);
  bool tma = true;
  for (int i = 0; i < b->n; ++i) {
    BatchInst& I = b->h_insts[i];
    if (!fields[i] || !velocities[i]) return fail(SS_ERR_ARG, "lattice %d: NULL field or velocity", i);
    I.G = b->inst[i].G;
    I.P = b->inst[i].P;
    I.buf[0] = fields[i];
    I.buf[1] = velocities[i];
    if (tma) tma = batch_encode(b, i);
  }
  b->tma = tma;
  if (!tma) b->shape.assign(b->n, 0);  // the small shape is built for TMA staging only
  StepState init;
  memset(&init, 0, sizeof(init));
  init.E_last = NAN;
  const std::vector<StepState> inits(b->n, init);  // pageable: staged before the call returns
  CK(cudaMemcpyAsync(b->d_st, inits.data(), sizeof(StepState) * b->n, cudaMemcpyHostToDevice, b->stream));
  return batch_upload(b, nullptr);
}

int ss_batch_step(ss_batch* b, int n_steps, const double* prev_energy, double* energy_traj, double* err_traj) {
  if (!b || !b->ws) return fail(SS_ERR_STATE, "batch not bound");
  if (n_steps < 0) return fail(SS_ERR_ARG, "n_steps must be >= 0");
  if (prev_energy)
    CK(cudaMemcpyAsync(b->d_prev, prev_energy, sizeof(double) * b->n, cudaMemcpyHostToDevice, b->stream));
  bool use_prev = prev_energy != nullptr;
  // trajectories (k columns of every lattice's row) and the step states come back through
  // page-locked staging: one 2-D copy each, one synchronisation per chunk
  const size_t nn = (size_t)b->n;
  if (!b->h_stage)
    CK(cudaHostAlloc((void**)&b->h_stage, 2 * nn * TRAJ_CAP * sizeof(double) + nn * sizeof(StepState),
                     cudaHostAllocDefault));
  double* hE = reinterpret_cast<double*>(b->h_stage);
  double* hErr = hE + nn * TRAJ_CAP;
  StepState* hst = reinterpret_cast<StepState*>(hErr + nn * TRAJ_CAP);
  for (int done = 0; done < n_steps; done += TRAJ_CAP) {
    const int k = std::min(TRAJ_CAP, n_steps - done);
    int rc = batch_dispatch(b, [&](auto* tag) -> int {
      using TH = std::remove_pointer_t<decltype(tag)>;
      if (b->precision == SS_FP32) return Batched<TH, float>::step(b, k, use_prev);
      return Batched<TH, double>::step(b, k, use_prev);
    });
    if (rc) return rc;
    use_prev = false;
    const size_t row = k * sizeof(double), pitch = TRAJ_CAP * sizeof(double);
    if (energy_traj) CK(cudaMemcpy2DAsync(hE, row, b->d_E, pitch, row, nn, cudaMemcpyDeviceToHost, b->stream));
    if (err_traj) CK(cudaMemcpy2DAsync(hErr, row, b->d_err, pitch, row, nn, cudaMemcpyDeviceToHost, b->stream));
    CK(cudaStreamSynchronize(b->stream));
    for (size_t i = 0; i < nn; ++i) {
      if (energy_traj) memcpy(energy_traj + i * n_steps + done, hE + i * k, row);
      if (err_traj) memcpy(err_traj + i * n_steps + done, hErr + i * k, row);
    }
  }
  CK(cudaMemcpyAsync(hst, b->d_st, nn * sizeof(StepState), cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  int worst = 0;
  for (size_t i = 0; i < nn; ++i) {
    if (hst[i].status) {
      worst = hst[i].status;
      const int zero = 0;
      CK(cudaMemcpy(&b->d_st[i].status, &zero, sizeof(int), cudaMemcpyHostToDevice));
    }
  }
  if (worst == SS_ERR_TIMEOUT) return fail(SS_ERR_TIMEOUT, "a device-side wait timed out; re-bind the batch");
  if (worst) return fail(SS_ERR_NONFINITE, "a lattice's energy became non-finite");
  return SS_OK;
}

int ss_batch_tma_enabled(const ss_batch* b) { return b && b->tma ? 1 : 0; }

int ss_batch_get_shape(const ss_batch* b, int lattice) {
  if (!b || lattice < 0 || lattice >= b->n) return -1;
  return b->shape[lattice];
}

int ss_batch_set_shape(ss_batch* b, int lattice, int shape) {
  if (!b || !b->ws) return fail(SS_ERR_STATE, "batch not bound");
  if (lattice < 0 || lattice >= b->n) return fail(SS_ERR_ARG, "lattice %d out of range", lattice);
  if (shape < 0 || shape >= N_BATCH_SHAPES) return fail(SS_ERR_ARG, "tile shape %d: 0 (16 x 64) or 1 (8 x 32)", shape);
  if (shape != 0 && (!b->tma || b->precision != SS_FP32))
    return fail(SS_ERR_ARG, "the 8 x 32 tile shape needs TMA-staged FP32 lattices");
  b->shape[lattice] = shape;
  if (!batch_encode(b, lattice)) return fail(SS_ERR_CUDA, "tensor map of lattice %d", lattice);
  return batch_upload(b, nullptr);
}

int ss_batch_autotune(ss_batch* b, int iters, float* ms_out) {
  if (!b || !b->ws) return fail(SS_ERR_STATE, "batch not bound");
  if (iters < 1) iters = 1;
  if (ms_out)
    for (int i = 0; i < 2 * b->n; ++i) ms_out[i] = 0.f;
  if (!b->tma || b->precision != SS_FP32) return SS_OK;  // one tile shape only
  // size classes: lattices of equal extents
  std::vector<int> cls(b->n, -1);
  std::vector<std::pair<int, int>> keys;
  for (int i = 0; i < b->n; ++i) {
    const std::pair<int, int> k(b->inst[i].G.X, b->inst[i].G.Y);
    size_t c = 0;
    while (c < keys.size() && keys[c] != k) ++c;
    if (c == keys.size()) keys.push_back(k);
    cls[i] = (int)c;
  }
  cudaEvent_t e0, e1;
  CK(cudaEventCreate(&e0));
  CK(cudaEventCreate(&e1));
  std::vector<float> ms(keys.size() * N_BATCH_SHAPES, 0.f);
  int rc = SS_OK;
  for (size_t c = 0; c < keys.size() && rc == SS_OK; ++c) {
    std::vector<char> inc(b->n, 0);
    for (int i = 0; i < b->n; ++i) inc[i] = cls[i] == (int)c;
    for (int sh = 0; sh < N_BATCH_SHAPES && rc == SS_OK; ++sh) {
      for (int i = 0; i < b->n; ++i)
        if (inc[i]) {
          b->shape[i] = sh;
          batch_encode(b, i);
        }
      if ((rc = batch_upload(b, &inc))) break;
      auto time_steps = [&](int n) -> int {
        return batch_dispatch(b, [&](auto* tag) -> int {
          using TH = std::remove_pointer_t<decltype(tag)>;
          for (int k = 0; k < n; ++k) {
            const int r = Batched<TH, float>::timing_step(b);
            if (r) return r;
          }
          return SS_OK;
        });
      };
      if ((rc = time_steps(1))) break;  // warm-up
      if (cudaEventRecord(e0, b->stream) != cudaSuccess) { rc = fail(SS_ERR_CUDA, "cudaEventRecord"); break; }
      if ((rc = time_steps(iters))) break;
      if (cudaEventRecord(e1, b->stream) != cudaSuccess || cudaEventSynchronize(e1) != cudaSuccess) {
        rc = fail(SS_ERR_CUDA, "timing the batch's tile shapes");
        break;
      }
      float t = 0.f;
      cudaEventElapsedTime(&t, e0, e1);
      ms[c * N_BATCH_SHAPES + sh] = t / iters;
    }
    const int best = ms[c * N_BATCH_SHAPES + 1] < ms[c * N_BATCH_SHAPES] ? 1 : 0;
    for (int i = 0; i < b->n; ++i)
      if (inc[i]) {
        b->shape[i] = rc == SS_OK ? best : 0;
        batch_encode(b, i);
      }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  const int up = batch_upload(b, nullptr);
  if (rc) return rc;
  if (up) return up;
  if (ms_out)
    for (int i = 0; i < b->n; ++i)
      for (int sh = 0; sh < N_BATCH_SHAPES; ++sh) ms_out[2 * i + sh] = ms[cls[i] * N_BATCH_SHAPES + sh];
  // the timing steps ran the stages with every state update off; only the ticket and
  // err slots they reset were touched
  return SS_OK;
}

}  // extern "C"


// ===========================================================================
// CUDA graphs of whole relaxations
// ===========================================================================
namespace {

// Capture `issue` (which launches on *stream_slot) on a private stream into a graph.
template <class Issue>
int capture_graph(cudaStream_t* stream_slot, cudaGraphExec_t* out, Issue&& issue) {
  cudaStream_t cs;
  CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
  cudaStream_t saved = *stream_slot;
  *stream_slot = cs;
  cudaGraph_t g = nullptr;
  int rc = SS_OK;
  cudaError_t e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed);
  if (e == cudaSuccess) {
    rc = issue();
    cudaError_t e2 = cudaStreamEndCapture(cs, &g);
    if (rc == SS_OK && e2 != cudaSuccess) rc = fail(SS_ERR_CUDA, "cudaStreamEndCapture: %s", cudaGetErrorString(e2));
  } else {
    rc = fail(SS_ERR_CUDA, "cudaStreamBeginCapture: %s", cudaGetErrorString(e));
  }
  *stream_slot = saved;
  if (rc == SS_OK) {
    if (*out) cudaGraphExecDestroy(*out);
    *out = nullptr;
    e = cudaGraphInstantiate(out, g, 0);
    if (e != cudaSuccess) rc = fail(SS_ERR_CUDA, "cudaGraphInstantiate: %s", cudaGetErrorString(e));
  }
  if (g) cudaGraphDestroy(g);
  cudaStreamDestroy(cs);
  return rc;
}

}  // namespace

extern "C" {

int ss_graph_create(ss_handle* h, int n_steps, double* energy_traj_dev, double* err_traj_dev) {
  int rc = check_bound(h);
  if (rc) return rc;
  if (n_steps < 1) return fail(SS_ERR_ARG, "n_steps must be >= 1");
  if (h->precision == SS_PLAIN_FP64) return fail(SS_ERR_ARG, "the plain FP64 form arrests on the host");
  return capture_graph(&h->stream, &h->graph,
                       [&]() { return ss_step_async(h, n_steps, NAN, energy_traj_dev, err_traj_dev); });
}

int ss_graph_launch(ss_handle* h) {
  if (!h || !h->graph) return fail(SS_ERR_STATE, "no graph captured: call ss_graph_create");
  CK(cudaGraphLaunch(h->graph, h->stream));
  return SS_OK;
}

int ss_batch_graph_create(ss_batch* b, int n_steps) {
  if (!b || !b->ws) return fail(SS_ERR_STATE, "batch not bound");
  if (n_steps < 1 || n_steps > TRAJ_CAP) return fail(SS_ERR_ARG, "n_steps must be in 1..%d", TRAJ_CAP);
  return capture_graph(&b->stream, &b->graph, [&]() {
    return batch_dispatch(b, [&](auto* tag) -> int {
      using TH = std::remove_pointer_t<decltype(tag)>;
      if (b->precision == SS_FP32) return Batched<TH, float>::step(b, n_steps, false);
      return Batched<TH, double>::step(b, n_steps, false);
    });
  });
}

int ss_batch_graph_launch(ss_batch* b) {
  if (!b || !b->graph) return fail(SS_ERR_STATE, "no graph captured: call ss_batch_graph_create");
  CK(cudaGraphLaunch(b->graph, b->stream));
  return SS_OK;
}

int ss_batch_trajectory(ss_batch* b, int n_steps, double* energy_traj, double* err_traj) {
  if (!b || !b->ws) return fail(SS_ERR_STATE, "batch not bound");
  if (n_steps < 0 || n_steps > TRAJ_CAP) return fail(SS_ERR_ARG, "n_steps must be in 0..%d", TRAJ_CAP);
  const size_t row = n_steps * sizeof(double), pitch = TRAJ_CAP * sizeof(double);
  if (n_steps > 0 && energy_traj)
    CK(cudaMemcpy2DAsync(energy_traj, row, b->d_E, pitch, row, b->n, cudaMemcpyDeviceToHost, b->stream));
  if (n_steps > 0 && err_traj)
    CK(cudaMemcpy2DAsync(err_traj, row, b->d_err, pitch, row, b->n, cudaMemcpyDeviceToHost, b->stream));
  CK(cudaStreamSynchronize(b->stream));
  return SS_OK;
}

}  // extern "C"
