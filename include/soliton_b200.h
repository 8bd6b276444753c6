/*
 * soliton_b200.h -- C ABI of the B200-native soliton_solver flow backend.
 *
 * The library (libsoliton_b200.so) implements, as hand-written sm_100a CUDA
 * kernels, the per-theory energy-gradient stencils, the arrested-Newton-flow
 * RK4 step with unit-norm re-projection, and the energy / topological-charge
 * reductions of soliton_solver, for the Chiral magnet, Baby Skyrme model,
 * Ginzburg-Landau (Abelian Higgs) and anisotropic s+id superconductor theories.
 *
 * Conventions
 *  - Every function returns an int status (SS_OK == 0).  ss_last_error() gives a
 *    thread-local message for the last failing call.
 *  - Parameters are the reference's packed arrays: p_i (int32) and p_f (float64)
 *    exactly as produced by each theory's pack_device_params
 *    (soliton_solver/core/params.py:229-249 plus the theory's params.py).
 *  - Buffers are device pointers owned by the caller.  Fields use the reference
 *    layout idx = y + x*ylen + a*xlen*ylen (soliton_solver/core/utils.py:17-42)
 *    in the handle's element type (double for SS_FP64 / SS_PLAIN_FP64, float for
 *    SS_FP32).  Densities are always double.
 *  - The library never allocates device memory: the caller provides a workspace
 *    of ss_workspace_bytes() bytes through ss_bind().
 *  - Work is issued on the stream given to ss_bind() (a cudaStream_t, NULL for the
 *    legacy default stream).  Functions that return host scalars synchronise that
 *    stream; the *_async variants do not.
 */
#ifndef SOLITON_B200_H
#define SOLITON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SS_ABI_VERSION 1

/* status codes */
#define SS_OK 0
#define SS_ERR_ARG 1          /* bad argument, unsupported parameter combination */
#define SS_ERR_CUDA 2         /* a CUDA runtime call failed */
#define SS_ERR_NONFINITE 3    /* a reduction produced NaN or Inf */
#define SS_ERR_STATE 4        /* call out of order (e.g. no workspace bound) */
#define SS_ERR_WORKSPACE 5    /* workspace too small or misaligned */
#define SS_ERR_TIMEOUT 6      /* a bounded device-side wait expired (kernel returned early) */

/* theories (THEORY_SPEC names of the reference theory packages) */
#define SS_THEORY_CHIRAL_MAGNET 0   /* theories/chiral_magnet */
#define SS_THEORY_BABY_SKYRME 1     /* theories/baby_skyrme */
#define SS_THEORY_GINZBURG_LANDAU 2 /* theories/ginzburg_landau_superconductor */
#define SS_THEORY_ANISOTROPIC 3     /* theories/anisotropic_superconductor (s+id) */

/* precision / method */
#define SS_FP64 0       /* fused single-pass-per-stage kernels, FP64 fields */
#define SS_FP32 1       /* fused kernels, FP32 fields, FP64 energy/charge reductions */
#define SS_PLAIN_FP64 2 /* reference-structured FP64 form: derivative buffers, one
                           launch per RK stage, host-side arrest */

/* charges */
#define SS_CHARGE_SKYRMION 0 /* m.(dx m x dy m) dA/4pi : chiral magnet, baby Skyrme */
#define SS_CHARGE_MAGNETIC 1 /* -div m dA : chiral magnet */
#define SS_CHARGE_VORTEX 2   /* (dx A2 - dy A1) dA/(2 pi q) : Ginzburg-Landau, s+id */

/* couplings for ss_coupling_grad (partial derivatives of E at fixed field).  The
 * chiral magnet's physical constants enter only through the reduced couplings
 * coup_K = K J/D^2, coup_h = M B J/D^2, coup_mu = mu0 M^2 J/D^2; the host applies
 * the chain rule for dE/dB, dE/dK, dE/dD. */
#define SS_COUPLING_KAPPA 0   /* baby Skyrme kappa */
#define SS_COUPLING_MPI 1     /* baby Skyrme mpi */
#define SS_COUPLING_LAMBDA 2  /* Ginzburg-Landau Lambda */
#define SS_COUPLING_COUP_K 3  /* chiral magnet coup_K (p_f[6]) */
#define SS_COUPLING_COUP_H 4  /* chiral magnet coup_h (p_f[7]) */
#define SS_COUPLING_COUP_MU 5 /* chiral magnet coup_mu (p_f[8]) */

/* colormaps for ss_render_rgba */
#define SS_RENDER_JET 0           /* core/colormaps.py render_jet_density_to_rgba */
#define SS_RENDER_GRAY 1          /* core/colormaps.py render_gray_density_to_rgba */
#define SS_RENDER_MAGNETIZATION 2 /* core/colormaps.py render_magnetization_to_rgba */

/* diagnostic densities for ss_field_density (gauge theories) */
#define SS_DENSITY_HIGGS 0            /* |psi|^2: Ginzburg-Landau compute_norm_higgs_kernel */
#define SS_DENSITY_HIGGS1 1           /* |psi1|^2: s+id compute_norm_higgs1_kernel */
#define SS_DENSITY_HIGGS2 2           /* |psi2|^2: s+id compute_norm_higgs2_kernel */
#define SS_DENSITY_PHASE_DIFFERENCE 3 /* cos(arg psi1 - arg psi2): s+id compute_phase_difference_kernel */
#define SS_DENSITY_SUPERCURRENT 4     /* 2 planes: dxy A2 - dyy A1, dxy A1 - dxx A2 (both gauge theories) */
#define SS_DENSITY_MAGNETIC_FIELD 5   /* (dx A2 - dy A1) dA/(2 pi Q): s+id compute_magnetic_field_kernel */

/* initial conditions (ss_initialize, ss_insert_soliton) */
#define SS_INIT_GROUND 0   /* create_ground_state_kernel */
#define SS_INIT_ANSATZ 1   /* create_initial_configuration_kernel */
#define SS_ANSATZ_NONE 0   /* chiral magnet / baby Skyrme ansatz flags (ansatz_bloch, ansatz_neel, ansatz_anti) */
#define SS_ANSATZ_BLOCH 1
#define SS_ANSATZ_NEEL 2
#define SS_ANSATZ_ANTI 3

typedef struct ss_handle ss_handle;
typedef struct ss_batch ss_batch;

int ss_abi_version(void);
const char *ss_status_string(int status);
const char *ss_last_error(void);

/* Create a solver handle for one lattice.  Replaces Simulation.__init__'s
 * parameter resolution and packing (soliton_solver/core/simulation.py:43-115). */
int ss_create(int theory, const int32_t *p_i, int n_i, const double *p_f, int n_f, int precision,
              ss_handle **out);
int ss_destroy(ss_handle *h);
/* Bytes of caller-owned device workspace ss_bind() needs (five field-sized flow
 * buffers: l1, l2, the stage-4 field T4 and stage 4's two accumulated inputs; reduction
 * partials and the device-side step state). */
int ss_workspace_bytes(const ss_handle *h, size_t *bytes);
/* Bind the caller's Field and Velocity buffers, the workspace and the stream. */
int ss_bind(ss_handle *h, void *field, void *velocity, void *workspace, size_t workspace_bytes,
            void *stream);

/* n_steps arrested-Newton-flow RK4 steps of the bound Field/Velocity.
 * Replaces Simulation.step / do_arrested_newton_flow
 * (soliton_solver/core/simulation.py:388-409, core/integrator.py:217-348).
 * energy_traj[s] / err_traj[s] (host, nullable) receive E after step s and the
 * signed maximum of the stage-4 energy gradient of step s.  prev_energy is the
 * energy the first step's arrest test compares against; pass NaN to continue from
 * the energy the previous ss_step call left on the device.  Steps run in chunks of
 * 1024; a non-finite energy or a timed-out wait ends the call after the chunk in
 * which it happened (the trajectories up to there are written).  The first call
 * page-locks a 16 KB host staging buffer, held until ss_destroy. */
int ss_step(ss_handle *h, int n_steps, double prev_energy, double *energy_traj, double *err_traj);
/* As ss_step but without a host synchronisation: the trajectories go to device
 * arrays of n_steps doubles (nullable) and the status of the device-side checks is
 * reported by the next synchronising call or ss_check_status(). */
int ss_step_async(ss_handle *h, int n_steps, double prev_energy, double *energy_traj_dev,
                  double *err_traj_dev);
/* Synchronise the bound stream and return the status the device-side checks set. */
int ss_check_status(ss_handle *h);
/* 1 when the bound Field/Velocity/workspace buffers are staged by TMA tensor maps
 * (row pitch and base 16-byte aligned), 0 when the plain-load path is used. */
int ss_tma_enabled(const ss_handle *h);
/* Autotuner: times, on the bound buffers, the two TMA staging variants of each flow
 * stage (persistent CTAs walking tiles through a shared-memory ring, or one tile per
 * CTA) over `iters` launches and keeps the faster one, then times stages 2 and 3 fused
 * into one kernel (one staging of phi, V, l1) against the two chosen kernels.  Writes
 * only workspace scratch.  ms_out (nullable, 14 floats) receives [mode][variant]
 * times for modes 0..6 (mode 6: [two kernels, fused]). */
int ss_autotune(ss_handle *h, int iters, float *ms_out);
/* Variant chosen for a flow mode (0..5): 1 pipelined, 0 one tile per CTA; mode 6: 1 if
 * stages 2 and 3 run fused; -1 bad args. */
int ss_get_variant(const ss_handle *h, int mode);
/* Pin the staging variant of a flow mode instead of autotuning it: mode 0 (gradient)
 * or 1..4 (stages; stage 1 also sets the energy pass, whose per-CTA partials must
 * match it), variant 0 (one tile per CTA) or 1 (pipelined; needs TMA-staged bound
 * buffers and FP32 fields); mode 6: 1 runs stages 2 and 3 as one kernel (with TMA
 * staging), 0 as two.  For reproducible runs and for profiling a known kernel set.
 * No reference counterpart (tuning control). */
int ss_set_variant(ss_handle *h, int mode, int variant);
/* Failure-detection hook.  Sets the bound (clock64 cycles, default 2e9) of every
 * device-side mbarrier wait of this handle's kernels; with inject != 0 the next
 * TMA-staged stage kernel's barrier expects 16 bytes more than its loads deliver,
 * so its bounded wait expires: the kernel records SS_ERR_TIMEOUT, waits the bound
 * again for its own copies and returns without computing.  No fault, trap or
 * unbounded spin is involved; after SS_ERR_TIMEOUT re-bind the handle. */
int ss_debug_wait_timeout(ss_handle *h, long long wait_cycles, int inject);

/* One gradient evaluation of an arbitrary field buffer: energy_gradient (nullable)
 * receives the theory's projected dE/dphi, l_out (nullable) receives -dt*dE/dphi.
 * Replaces theory.kernels.do_gradient_step_kernel(l_out, Field, d1, d2, EG, p_i, p_f)
 * (core/integrator.py:15-48 with e.g. theories/chiral_magnet/kernels.py:398-511). */
int ss_gradient(ss_handle *h, const void *field, void *energy_gradient, void *l_out);
/* Functional derivative dE/dphi of the energy density at every site (element type
 * of the handle): the same stencil as the flow's gradient but without the unit-norm
 * projection and without the chiral magnet's halo zeroing, and with the demag psi
 * row converted from the flow's -coup_mu dE/dpsi to dE/dpsi.  dA times this is the
 * gradient of the total energy up to O(h^4) and boundary terms; it is the backward
 * of the autograd energy.  No reference counterpart (new capability). */
int ss_energy_gradient(ss_handle *h, const void *field, void *grad);
/* Per-site energy x dA (double).  Replaces compute_energy_kernel
 * (e.g. theories/chiral_magnet/kernels.py:219-251). */
int ss_energy_density(ss_handle *h, const void *field, double *density);
/* Total energy, fixed-order compensated FP64 sum.  Replaces observables.compute_energy
 * (e.g. theories/chiral_magnet/observables.py:15-57). */
int ss_energy(ss_handle *h, const void *field, double *out);
/* Total FP64 energy (as ss_energy) of the field with each site's unit-vector
 * components divided by their FP64 norm: the normalisation of the reference's RK4
 * finalize (core/integrator.py:151-189) applied in FP64 before
 * observables.compute_energy.  For an FP32 field it removes the bias of m3 rounding to 1
 * where |m_perp| < 2.4e-4 (|m|^2 - 1 = |m_perp|^2 there); for theories without a
 * unit-vector constraint it equals the FP64 energy of the field.  Uses the l-buffer
 * part of the bound workspace.  No reference counterpart (new observable). */
int ss_energy_projected(ss_handle *h, const void *field, double *out);

/* Initial configuration of the handle's theory into field (and velocity, nullable:
 * set to zero), element type of the handle, on the bound stream (asynchronous).
 * SS_INIT_GROUND: the vacuum of create_ground_state_kernel.  SS_INIT_ANSATZ: the
 * single soliton of create_initial_configuration_kernel at the lattice centre —
 * chiral magnet / baby Skyrme: `ansatz` (SS_ANSATZ_*) rotated by `rotation`, with the
 * skyrmion number of the packed params; Abelian Higgs: winding `vortex_number`; s+id:
 * the packed windings.  Reference quirks kept: the s+id ground state reads u1, u2 from
 * p_f[11], p_f[12]; one bug repaired: the Abelian Higgs ansatz reads ainf from its packed
 * slot p_f[10] (the reference reads one past the array).  Replaces
 * theories/<theory>/initial_config.py create_ground_state_kernel and
 * create_initial_configuration_kernel (e.g. chiral_magnet/initial_config.py:117-283);
 * the chiral magnet's and baby Skyrme's initialize(mode="initial") cannot run in the
 * reference (one argument short). */
int ss_initialize(ss_handle *h, void *field, void *velocity, int mode, int ansatz, double rotation,
                  double vortex_number);
/* Add one soliton centred on lattice point (pxi, pxj) to the field in place:
 * chiral magnet / baby Skyrme: the `ansatz` skyrmion composed stereographically with
 * the field there (create_skyrmion_kernel, chiral_magnet/initial_config.py:285-386);
 * Abelian Higgs / s+id: a vortex (`vortex` != 0: phase -theta, else +theta) multiplied
 * into the condensates (create_vortex_kernel, ginzburg_landau_superconductor/
 * initial_config.py:259-313, anisotropic_superconductor/initial_config.py:282-347).
 * A point outside the lattice leaves the field unchanged, as in the reference. */
int ss_insert_soliton(ss_handle *h, void *field, int pxi, int pxj, int ansatz, int vortex, double rotation);

/* Plain-text formatting of n values on the device, byte for byte as the reference's
 * .dat writers (core/io.py:44-240): each value as Python's format(v, ".{digits}g")
 * (exact decimal conversion, round half to even, "g" presentation, "nan", "inf",
 * "-0"), followed by a tab; a newline after every `row` values and another after
 * every `block` values (0: none).  output_field_dat is row = ylen, block = xlen*ylen;
 * output_density_data_dat row = ylen, block = 0; output_iteration_data_dat row =
 * block = 0.  values: device array of SS_FP32 or SS_FP64 (`precision`); digits 1..40.
 * workspace: device scratch of ss_text_workspace_bytes(n) bytes, 8-byte aligned.  With
 * out == NULL only *out_len (the text's length) is computed; otherwise the text is
 * written to the device buffer out (out_cap bytes) and *out_len set.  Synchronises
 * the stream once (to read the length).  Replaces output_field_dat,
 * output_density_data_dat and output_iteration_data_dat's formatting loops. */
int ss_text_workspace_bytes(long long n, size_t *bytes);
int ss_format_text(const void *values, int precision, long long n, int digits, long long row, long long block,
                   char *out, size_t out_cap, long long *out_len, void *workspace, size_t workspace_bytes,
                   void *stream);

/* Headless RGBA image of a lattice into a caller-owned device buffer of ylen*xlen*4
 * bytes (4-byte aligned; pixel (y, x) at byte 4*(y*xlen + x), R G B A), the bytes
 * the reference's viewer writes into its GL pixel buffer, without a graphics context.
 * SS_RENDER_JET / SS_RENDER_GRAY: src is a density indexed y + x*ylen, normalised by
 * vmin/vmax; SS_RENDER_MAGNETIZATION: src holds the planes m1, m2, m3 (stride
 * xlen*ylen; vmin/vmax unused).  precision (SS_FP32 or SS_FP64) is src's element
 * type; the arithmetic is FP64.  Asynchronous on `stream`.  Replaces
 * render_jet_density_to_rgba, render_gray_density_to_rgba and
 * render_magnetization_to_rgba (soliton_solver/core/colormaps.py:94-267). */
int ss_render_rgba(int kind, const void *src, int precision, int xlen, int ylen, double vmin, double vmax,
                   unsigned char *rgba, void *stream);
/* Charge densities / totals.  Replace compute_skyrmion_number_kernel,
 * compute_magnetic_charge_kernel, compute_vortex_number_kernel and the matching
 * observables.compute_* (e.g. theories/chiral_magnet/kernels.py:294-395,
 * theories/ginzburg_landau_superconductor/kernels.py:181-215). */
int ss_charge_density(ss_handle *h, const void *field, int which, double *density);
int ss_charge(ss_handle *h, const void *field, int which, double *out);
/* Copy of a field of the handle's lattice and theory from src (SS_FP32 or SS_FP64 /
 * SS_PLAIN_FP64 elements, `src_precision`) into dst (`dst_precision`), on the handle's
 * stream (asynchronous; needs no workspace).  With project != 0, each site's
 * unit-vector components are divided by their FP64 norm first (theories with the
 * constraint and unit_magnetization set; the normalisation of the reference's RK4
 * finalize, core/integrator.py:151-189); the result is rounded once to dst's type.
 * Used to hand a relaxation from FP32 to FP64 fields and back.  In place only for
 * equal element types.  No reference counterpart (the reference is FP64 only). */
int ss_convert_field(ss_handle *h, const void *src, int src_precision, void *dst, int dst_precision, int project);
/* Exact derivative of the discrete energy sum E_h = dA sum_s e(phi, Dx phi, Dy phi)
 * (the reference's compute_energy_kernel summed, e.g. theories/chiral_magnet/
 * kernels.py:125-251) with respect to every field value, divided by dA, into `out`
 * (double, nf planes of N, true rows: dE/dpsi for the demag field, unprojected, no halo
 * zeroing): de/dphi(t) - D1x[mask de/d(dx phi)](t) - D1y[mask de/d(dy phi)](t), the
 * partials of the energy point by forward-mode dual numbers.  The flow's stencil
 * gradient equals it only to O(h^4); with minus_stencil != 0 (SS_FP64 handles) `out`
 * receives that difference (out minus ss_energy_gradient's result).  Uses the flow
 * buffers of the bound workspace as scratch (not during a step).  No reference
 * counterpart (the adjoint's discretisation correction). */
int ss_energy_gradient_exact(ss_handle *h, const void *field, double *out, int minus_stencil);
/* Add a fixed field `force` (device, double, nf planes of N in the true rows of
 * ss_energy_gradient, 16-byte aligned; NULL removes it) to the flow's gradient rows in
 * every stage of the following steps, before the halo zeroing and the unit-norm
 * projection; the stage-4 err includes it.  SS_FP64 handles only.  A graph captured
 * before the call keeps its old forcing.  With force = the residual of
 * ss_energy_gradient_exact at a relaxed field, the flow relaxes to the stationary point
 * of the discrete energy sum itself, to O(h^8).  No reference counterpart. */
int ss_set_forcing(ss_handle *h, const double *force);
/* Diagnostic density of `field` (element type of the handle) into the device array
 * `out` (double; N sites, 2 N for SS_DENSITY_SUPERCURRENT: the x plane, then the y
 * plane), asynchronous on the handle's stream; needs no workspace.  Replaces the
 * Simulation helpers compute_higgs_density, compute_higgs1_density,
 * compute_higgs2_density, compute_phase_difference_density, supercurrent and
 * magnetic_field (soliton_solver/core/simulation.py:211-300,301-318,370-386) and the
 * kernels they launch (theories/ginzburg_landau_superconductor/kernels.py:218-340,
 * theories/anisotropic_superconductor/kernels.py:280-553). */
int ss_field_density(ss_handle *h, const void *field, int kind, double *out);
/* Partial derivative dE/dc of the discrete energy with respect to a coupling at
 * fixed field.  At a relaxed (stationary) field this is dE_min/dc by the envelope
 * theorem.  No reference counterpart: a new capability of this backend. */
int ss_coupling_grad(ss_handle *h, const void *field, int coupling, double *out);

/* Total energy of `field` (SS_FP32 or SS_FP64 elements, reference layout) with no
 * handle and no allocation of any kind.  No counterpart in the reference: it exists
 * for callers that cannot allocate device memory when they need the energy — a host
 * whose memory manager owns the whole device and forbids further allocations, or an
 * interactive loop (a viewer's per-frame callback) that must not call cudaMalloc or
 * cudaFree, which synchronise the device.  Its scratch (reduction state and one FP64
 * partial per 16 x 64-site tile) lives in a 512 KiB static device array that every
 * GPU loading the library holds until exit, so lattices of at most 65504 tiles are
 * accepted (4096 x 4096 needs 16384); larger ones get SS_ERR_ARG.  The first call
 * on a device looks up the array's device address (cudaGetSymbolAddress, with that
 * device current): make that first call before any stream capture.  All calls share
 * the array and the kernel runs on `stream` (a cudaStream_t, NULL for the legacy
 * default stream): calls that overlap on the GPU race; each call clears the
 * reduction state before use.  The call synchronises `stream` and returns the
 * result in *out. */
int ss_energy_noalloc(int theory, const int32_t *p_i, int n_i, const double *p_f, int n_f, int precision,
                      const void *field, double *out, void *stream);

/* The reference's RK4 building blocks on arbitrary buffers (element type of the
 * handle).  ss_rk4_stage replaces do_rk4_step_kernel (core/integrator.py:51-96):
 * k_out = dt*(velocity + factor*l_in), temp = field + factor*k_prev.
 * ss_rk4_finalize replaces the theory's do_rk4_kernel / do_rk4_kernel_no_constraint
 * (core/integrator.py:99-189). */
int ss_rk4_stage(ss_handle *h, void *k_out, const void *velocity, const void *l_in, void *temp,
                 const void *field, const void *k_prev, double factor);
int ss_rk4_finalize(ss_handle *h, void *velocity, void *field, const void *k1, const void *k2,
                    const void *k3, const void *k4, const void *l1, const void *l2, const void *l3,
                    const void *l4);

/* ---- batches: many independent lattices of one theory ----------------------
 * The lattices may differ in size, couplings and state; each keeps its own arrest
 * flag and energy.  One launch per RK stage covers every lattice's tiles.  No
 * reference counterpart (the reference runs one lattice per Simulation); each
 * lattice's step is exactly ss_step's.
 * p_i / p_f hold n_lattices packed arrays of n_i / n_f entries back to back. */
int ss_batch_create(int theory, int n_lattices, const int32_t *p_i, int n_i, const double *p_f, int n_f,
                    int precision, ss_batch **out);
int ss_batch_destroy(ss_batch *b);
int ss_batch_workspace_bytes(const ss_batch *b, size_t *bytes);
/* fields[i] / velocities[i]: device buffers of lattice i (caller-owned). */
int ss_batch_bind(ss_batch *b, void *const *fields, void *const *velocities, void *workspace,
                  size_t workspace_bytes, void *stream);
/* n_steps steps of every lattice.  prev_energy (host, n_lattices, nullable: continue
 * from the device state) seeds each first arrest test; energy_traj / err_traj (host,
 * nullable) receive lattice-major [i * n_steps + s] trajectories.  The first call
 * page-locks a host staging buffer of 16 KB per lattice, held until ss_batch_destroy. */
int ss_batch_step(ss_batch *b, int n_steps, const double *prev_energy, double *energy_traj, double *err_traj);
int ss_batch_tma_enabled(const ss_batch *b);
/* Tile shapes of the batched stage kernels, chosen per size class of lattices (the
 * lattices of equal extents): shape 0 tiles 16 x 64 sites per 256-thread CTA (three
 * resident per SM), shape 1 tiles 8 x 32 per 128-thread CTA (six per SM; TMA-staged
 * FP32 batches only).  ss_batch_autotune times one step's stage launches of each size
 * class in each shape (`iters` steps, after one warm-up; only workspace scratch is
 * written) and keeps the faster; ms_out (nullable, 2 n floats) receives, per lattice,
 * its class's step time in shape 0 and 1 (zeros when only shape 0 applies).  Lattices
 * of different shapes are launched as one kernel per shape and stage.  Results do not
 * depend on the shape up to the order of the per-tile energy partials.  No reference
 * counterpart. */
int ss_batch_autotune(ss_batch *b, int iters, float *ms_out);
int ss_batch_get_shape(const ss_batch *b, int lattice);
int ss_batch_set_shape(ss_batch *b, int lattice, int shape);

/* ---- CUDA graphs ---------------------------------------------------------------
 * ss_graph_create captures n_steps of ss_step_async(h, n_steps, NaN, ...) — every
 * stage launch and the closing arrest kernel — into a CUDA graph on a
 * private stream; ss_graph_launch replays it on the bound stream (each replay
 * continues from the device state).  The batch versions capture n_steps (at most
 * 1024) of every lattice; ss_batch_trajectory copies the last replay's per-lattice
 * trajectories to the host.  No reference counterpart. */
int ss_graph_create(ss_handle *h, int n_steps, double *energy_traj_dev, double *err_traj_dev);
int ss_graph_launch(ss_handle *h);
int ss_batch_graph_create(ss_batch *b, int n_steps);
int ss_batch_graph_launch(ss_batch *b);
int ss_batch_trajectory(ss_batch *b, int n_steps, double *energy_traj, double *err_traj);

#ifdef __cplusplus
}
#endif

#endif /* SOLITON_B200_H */
