/* pfdd_b200.h -- C ABI of the B200 Ginzburg-Landau stepper (libpfdd_b200.so).
 *
 * The library advances the PFDD Ginzburg-Landau relaxation that the reference
 * runs inside its FFT style object, driven step by step from SolveGL::iterate
 * (src/solve_GL.cpp:70-158).  One call to pfdd_gpu_advance replaces, per GL
 * iteration, the reference's sequence
 *     init_loop -> gradient -> App::core_energy -> prep_forward ->
 *     internal_energy -> prep_backward -> update_order_parameter ->
 *     prepare_next_itr
 * (src/solve_GL.cpp:92-124, src/fft_fftw_slab.cpp:1628-1862).
 *
 * Conventions (all as in the reference):
 *   - grid nx*ny*nz, z fastest: site r = k + j*nz + i*ny*nz
 *     (src/fft_fftw_slab.cpp:1763-1766);
 *   - slip-system fields are stacked: value of system a at site r is at
 *     [r + a*N], N = nx*ny*nz;
 *   - the order parameter is complex (xi[0][2*(r+a*N)] = Re, +1 = Im in the
 *     reference, src/fft.h:48); this ABI takes/returns Re and Im planes;
 *   - stresses are in units of the shear modulus (the deck's `sigma` values,
 *     src/app.cpp:325-381);
 *   - elastic constants in Pa, b in m, GSFE energies in J/m^2
 *     (src/material.cpp:41-156).
 *
 * Every entry point returns a pfdd_status (0 = success, < 0 = error) and never
 * exits the process or throws across the boundary; pfdd_gpu_last_error gives
 * the message.  (The reference reports errors through Error::all/one, which
 * print and call exit/MPI_Abort, src/error.cpp:34-69.)
 *
 * A handle is thread-compatible: calls on one handle must not overlap; calls
 * on different handles may run concurrently from different host threads.
 */
#ifndef PFDD_B200_H
#define PFDD_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef int pfdd_status;
enum {
  PFDD_OK = 0,
  PFDD_EINVAL = -1,        /* bad argument / descriptor */
  PFDD_ENOMEM = -2,        /* device or host allocation failed */
  PFDD_ECUDA = -3,         /* CUDA runtime error */
  PFDD_EUNSUPPORTED = -4,  /* size/model combination not built */
  PFDD_EDIVERGED = -5,     /* non-finite order parameter detected */
  PFDD_ENODEVICE = -6,     /* no usable sm_100 device */
  PFDD_ESTATE = -7,        /* call not valid in the handle's current state */
  PFDD_ETIMEOUT = -8       /* a bounded device-side wait ran out (the step was abandoned) */
};

#define PFDD_MAX_SLIP 12

/* Arithmetic of the step. */
enum { PFDD_FP64 = 0, PFDD_FP32 = 1 };

/* How the imaginary part of the complex order parameter is carried.
 * The reference's forward and inverse transforms are complex-to-complex and
 * its B(k) table is indexed so that B at index -k differs from B at k on the
 * Nyquist planes (src/fft_fftw_slab.cpp:280-337 maps index n/2 to -1/2); a
 * real xi therefore grows an imaginary part there, which feeds back into the
 * real part.  PFDD_IMAG_FULL carries Im xi as a second real field and is
 * exact in every case (masks included).  PFDD_IMAG_NYQUIST carries only the
 * Nyquist-plane spectrum of Im xi, which is exact when no obstacle mask is
 * set and the initial Im xi is zero.  PFDD_IMAG_AUTO picks NYQUIST when it
 * is exact, else FULL. */
enum { PFDD_IMAG_AUTO = 0, PFDD_IMAG_FULL = 1, PFDD_IMAG_NYQUIST = 2 };

/* GSFE core models, numbered as App::core_energy dispatches them
 * (src/app.cpp:663-672), plus one model with no reference counterpart. */
enum {
  PFDD_CORE_PERFECT = 1,     /* core_energy_perfect   src/fft_fftw_slab.cpp:1130-1191 */
  PFDD_CORE_EXTENDED = 2,    /* core_energy_extended  src/fft_fftw_slab.cpp:1243-1354 */
  PFDD_CORE_SINE = 3,        /* core_energy_sine      src/fft_fftw_slab.cpp:1360-1418 */
  PFDD_CORE_PYRII = 4,       /* core_energy_pyrII     src/fft_fftw_slab.cpp:1429-1493 */
  PFDD_CORE_BCC_PERFECT = 5, /* core_energy_bcc_perfect src/fft_fftw_slab.cpp:1070-1125, with the
                                edge/screw angle from FFTW_Slab::gradient :869-1065 */
  PFDD_CORE_USFE_ANGLE = 6,  /* core_energy_USFE_angle_tau src/fft_fftw_slab.cpp:1500-1545: the
                                amplitude follows sigma_rot[2][1] of each stress state through
                                `usfe_fit` and `angle_to_110`; the `An` field is not read */
  PFDD_CORE_MPEA = 7,        /* core_energy_mpea      src/fft_fftw_slab.cpp:1196-1235 */
  PFDD_CORE_SINE_FIELD = 103 /* sine GSFE with a per-site multiplier on isf and usf
                                (random-alloy fields); no reference counterpart,
                                equals PFDD_CORE_SINE when the multiplier is 1 */
};

/* One simulation instance: what FFTW_Slab::setup consumes
 * (rotate_stress, frec, stiffness, Bmatrix: src/fft_fftw_slab.cpp:111-119). */
typedef struct {
  int nx, ny, nz;              /* FFT::nx, ny, nz */
  int n_slip;                  /* FFT::slip_systems (1..PFDD_MAX_SLIP) */
  double four[3][3];           /* FFT::four, reciprocal basis (src/app.cpp:383-444) */
  double prim[3][3];           /* FFT::prim, normalised primitive vectors (src/fft.cpp:96-135) */
  double xn[PFDD_MAX_SLIP][3]; /* slip normals after App::set_slip */
  double xb[PFDD_MAX_SLIP][3]; /* Burgers vectors after App::set_slip */
  double C44, C12, C11;        /* Material elastic constants, Pa */
  double dslip, b;             /* Material::dslip, Material::b (m) */
  double cd_dt;                /* App::CD * App::timestep */
  int core_flag;               /* PFDD_CORE_* */
  double isf, usf, An;         /* J/m^2 */
  double c[7];                 /* c0 c1 c2 c3 c4 a1 a3 (extended core), J/m^2 */
  double aa[5], bb[4];         /* aa0..aa4, bb1..bb4 (pyrII core), J/m^2 */
  const double *site_gsfe;     /* per-site [S*N]: A_mpea (J/m^2) for MPEA, the
                                  multiplier for SINE_FIELD; else NULL.  Copied. */
  const double *xo;            /* obstacle mask [S*N] (nonzero = frozen), or NULL. Copied. */
  double sigma[3][3];          /* App::sigma at the first stress state (units of mu) */
  double dsigma[3][3];         /* App::deltasig added after each stress state */
  /* Non-Schmid resolved shear stress: App::set_nonSchmid (src/app.cpp:446-459)
   * selects FFTW_Slab::resolSS_non_Schmid (src/fft_fftw_slab.cpp:774-840)
   * over resolSS_Schmid (:737-769) through App::resolSS (src/app.cpp:654-658).
   * The reference sizes its projection tables for three systems, so
   * non_schmid = 1 needs n_slip <= 3. */
  int non_schmid;              /* App::non_Schmid: 0 = Schmid, 1 = non-Schmid */
  double angle_to_110;         /* App::angle_to_110, degrees (also read by core model 6) */
  double w1, w2, w3;           /* App::w1, w2, w3 */
  double usfe_fit[5];          /* Material::a_slope, a_b, b_b, c_slope, c_b (core model 6;
                                  the Ta and Fe presets, src/material.cpp:713-717, :766-770) */
} pfdd_instance_desc;

typedef struct {
  int precision;       /* PFDD_FP64 or PFDD_FP32 */
  int imag_mode;       /* PFDD_IMAG_* */
  int device;          /* CUDA device ordinal */
  int use_graphs;      /* capture multi-step advance in a CUDA graph (1 = yes) */
  int check_finite;    /* scan for non-finite xi after each advance (1 = yes) */
} pfdd_options;

typedef struct {
  double xinorm;       /* sqrt(sum |dxi|^2) of the last step (src/fft_fftw_slab.cpp:1787-1789) */
  double xiave;        /* sum of Re xi after the last step (ibid.) */
  int steps_done;      /* GL iterations performed by this call */
  int converged;       /* 1 if xinorm < tol ended the stress state early */
} pfdd_step_stats;

typedef struct pfdd_gpu pfdd_gpu;

/* Create a handle for n_instances independent instances (each may have its
 * own grid size, slip systems and material), allocate device memory, compute
 * the per-instance constants in FP64 and upload the initial state xi = 0.
 * Replaces FFTW_Slab::init/setup (src/fft_fftw_slab.cpp:52-119). */
pfdd_status pfdd_gpu_create(const pfdd_instance_desc *descs, int n_instances,
                            const pfdd_options *opt, pfdd_gpu **out);

/* Set instance `inst`'s order parameter from host planes xi_re, xi_im
 * ([S*N] each, reference site order; xi_im may be NULL = 0).  Replaces the
 * xi/data_fftw fill of initial_sxtal_* (src/fft_fftw_slab.cpp:2196-3247). */
pfdd_status pfdd_gpu_set_state(pfdd_gpu *h, int inst, const double *xi_re, const double *xi_im);

/* Same, from the reference's interleaved layout xi[0][2*(r + a*N) + {0,1}]. */
pfdd_status pfdd_gpu_set_state_interleaved(pfdd_gpu *h, int inst, const double *xi);

/* Copy instance `inst`'s order parameter to host planes ([S*N] each; either
 * pointer may be NULL).  The host refills FFT::xi from it for dumps
 * (src/app_fcc.cpp:320-502 reads xi through compute_mean_xi). */
pfdd_status pfdd_gpu_get_state(pfdd_gpu *h, int inst, double *xi_re, double *xi_im);

/* Same, into the reference's interleaved layout. */
pfdd_status pfdd_gpu_get_state_interleaved(pfdd_gpu *h, int inst, double *xi);

/* Run the SolveGL::iterate loop (src/solve_GL.cpp:80-156) on every instance:
 * `stress_states` outer iterations, each recomputing the resolved shear
 * stress (rotate_stress + resolSS_Schmid, src/fft_fftw_slab.cpp:242-274,
 * 737-769) and running up to `n_steps` GL iterations; a stress state ends
 * early when xinorm < tol (tol <= 0 disables the test); sigma += dsigma after
 * each stress state.  stats (may be NULL) receives one record per instance. */
pfdd_status pfdd_gpu_advance(pfdd_gpu *h, int n_steps, int stress_states, double tol,
                             pfdd_step_stats *stats);

/* Per-step xinorm/xiave history of instance `inst` for the last advance call
 * (every GL iteration of every stress state, in order):
 * up to `cap` records are written to xinorm[] / xiave[]; *count gets the
 * number of steps recorded. */
pfdd_status pfdd_gpu_step_history(pfdd_gpu *h, int inst, double *xinorm, double *xiave, int cap,
                                  int *count);

/* Total energy of the current state, per unit site, FP64 with compensated
 * summation: elastic 1/2 <xi, L xi>, core sum f(xi), applied -sum tau_a xi_a.
 * The reference accumulates E_core but never reduces or reports it
 * (src/fft_fftw_slab.cpp:1399); these are the terms whose gradient is the
 * drift of update_order_parameter (src/fft_fftw_slab.cpp:1773).  For core
 * model 5 the core term is sum usf' cof(theta) sin^2(pi xi) as
 * core_energy_bcc_perfect accumulates it (:1119), whose force holds cof fixed;
 * for core model 2 it is the fcore of each plane of three systems (:1320).
 * Core model 4 returns PFDD_EUNSUPPORTED. */
pfdd_status pfdd_gpu_energy(pfdd_gpu *h, int inst, double *e_elastic, double *e_core,
                            double *e_applied);

/* Strain and stress fields of instance `inst`'s current state, as the
 * reference's strain/stress diagnostics compute them when data_fftw holds the
 * forward transform of that state: FFTW_Slab::strain with Fmatrix,
 * stressfree_strain, total_average_strain and stress
 * (src/fft_fftw_slab.cpp:644-732, 3252-3553; called by DiagStress::compute,
 * src/diag_stress.cpp:43-62, and DumpText, src/dump_text.cpp:296-324).
 * eps and sigma (each 9*N doubles or NULL) receive component (i, j) at
 * (3 i + j) * N in the z-fastest site order: the real parts of data_eps and
 * data_sigma.  ave_eps[9] and ave_sigma[9] (or NULL) receive the box averages
 * (FFT::ave_eps, FFT::ave_sigma).  The applied stress is that of the stress
 * state the last pfdd_gpu_advance stepped with (the reference outputs inside
 * its GL loop, before sigma += dsigma).  The spectrum buffer is reused, so the
 * next pfdd_gpu_advance opens with a fresh forward transform. */
pfdd_status pfdd_gpu_strain_stress(pfdd_gpu *h, int inst, double *eps, double *sigma, double *ave_eps,
                                   double *ave_sigma);

/* FFTW_Slab::project_core_energy (src/fft_fftw_slab.cpp:1550-1624; called
 * after each GL iteration when non_Schmid is set, src/solve_GL.cpp:121-122)
 * on instance `inst`'s current state.  delta ([n_planes*N], z-fastest site
 * order) receives Re xi_p for one or two slip systems, else the projection
 * sum_c (Re xi_3p b_0c + Re xi_3p+1 b_1c + Re xi_3p+2 b_2c) b_1c.  ddelta
 * ([n_planes*nx] or NULL) receives the forward difference along x of delta on
 * the line j = ny/2, k = nz/2, zero at the last x (dx = 1, one rank).
 * n_planes is App::num_planes: at most n_slip for one or two systems, at most
 * n_slip/3 otherwise (beyond that the reference reads past its array). */
pfdd_status pfdd_gpu_core_profile(pfdd_gpu *h, int inst, int n_planes, double *delta, double *ddelta);

/* Pick each batched group's x-pencil tile width (the number of (ky, kz)
 * columns a CTA transforms along x) by timing every width the grid divides
 * into and shared memory holds, `reps` launches each, on this device; the
 * fastest is kept (chosen[n_instances] receives it, or NULL).  No counterpart
 * in the reference (FFTW's planner measures its own plans,
 * src/fft_fftw_slab.cpp:125-134).  Valid between calls; the state is kept. */
pfdd_status pfdd_gpu_autotune(pfdd_gpu *h, int reps, int *chosen);

/* Asynchronous snapshot of instance `inst`'s order parameter for output
 * (the reference's dumps and diagnostics read fft->xi between GL iterations,
 * src/output.cpp:79-188, src/dump_text.cpp:296-324): the state is converted
 * to FP64 planes in device memory on the stepping stream, then copied to re
 * and im ([S*N] each, either may be NULL) on a second stream, so the next
 * pfdd_gpu_advance overlaps the copy.  Host buffers stay untouched by the
 * caller until pfdd_gpu_snapshot_wait; they must be page-locked
 * (cudaHostAlloc / cudaHostRegister) for the copy to overlap (pageable memory
 * works, with the copy finishing inside begin). */
pfdd_status pfdd_gpu_snapshot_begin(pfdd_gpu *h, int inst, double *re, double *im);
pfdd_status pfdd_gpu_snapshot_wait(pfdd_gpu *h, int inst);

/* ---- Conductivity sub-problem (SolveGLCond, src/solve_GL+cond.cpp:70-150) ----
 * A complex scalar order parameter condxi relaxed by its own GL iteration:
 * forwardcond, divcurrent (a = i k_y/k^2 c, b = k_y^2/k^2 c),
 * backwardcond (unnormalised inverse transforms of a and b, then
 * j_y = sigma(y) (E_y - a/eps0) and the assembly of the driving term with
 * the y-derivative of the layer conductivity) and update_conduct_order_param
 * (src/fft_fftw_slab.cpp:1699-1741, 1795-1834, 1999-2186).  It reads none of
 * the dislocation fields.  SolveGLCond's loop leaves after its first
 * iteration in every stress state (the `break` after the unbraced `if` at
 * src/solve_GL+cond.cpp:132-140), so a binding calls pfdd_gpu_cond_step with
 * n_iters = 1 once per stress state, beside pfdd_gpu_advance(h, 1, 1, ...). */

/* Members of one layer material (Material, src/material.h:44-56). */
typedef struct {
  double condsigma;          /* S/m at 300 K */
  double alpha_resistivity;  /* 1/K */
  double mfpel;              /* electron mean free path, m */
  double alpha_mfpel;        /* 1/K */
  double dlayer;             /* layer thickness, m */
  double Rgrain;             /* grain-boundary reflection */
  double beta_disloc;        /* resistivity per dislocation density, Ohm m^3 */
  double rho_disloc;         /* dislocation density, 1/m^2 */
  int Ngrains;               /* grains per layer */
  int Nlayers;               /* read from material A only */
  double pinterface;         /* read from material A only */
} pfdd_cond_material;

/* The per-y conductivity backwardcond builds (src/fft_fftw_slab.cpp:2064-2156):
 * A and B layers alternate along y (A.Nlayers periods of thicknesses from the
 * dlayer volume fraction, with the reference's integer division of ny by
 * Nlayers); sigma_layer[ny] is the temperature-corrected layer conductivity,
 * sigma_eff[ny] adds interface, grain-boundary and dislocation resistivity.
 * Host-only; PFDD_EINVAL when the layer period rounds to zero cells. */
pfdd_status pfdd_cond_layers(const pfdd_cond_material *A, const pfdd_cond_material *B, int ny,
                             double temperature, double *sigma_eff, double *sigma_layer);

typedef struct {
  const double *sigma_eff;     /* [ny], copied */
  const double *sigma_layer;   /* [ny], copied (needs ny >= 2) */
  double El_y;                 /* Material::El[1] of material A, V/m */
  double epsilonzero;          /* Material::epsilonzero */
  double timestep;             /* App::timestep (the update uses 1e-22 * timestep) */
} pfdd_cond_desc;

typedef struct {
  double condxinorm;    /* FFT::condxinorm of the iteration */
  double condxiave;     /* FFT::condxiave */
  double conductivity;  /* <j_y> / El_y of the iteration's backwardcond */
} pfdd_cond_stats;

/* Give instance `inst` a conductivity field (condxi = 0, FFTW_Slab::allocate
 * :162-173) on its grid; calling it again replaces the tables and zeroes condxi. */
pfdd_status pfdd_gpu_cond_enable(pfdd_gpu *h, int inst, const pfdd_cond_desc *d);
/* condxi from / to host planes [N] each (im may be NULL = 0 on set, skipped on get). */
pfdd_status pfdd_gpu_cond_set_state(pfdd_gpu *h, int inst, const double *re, const double *im);
pfdd_status pfdd_gpu_cond_get_state(pfdd_gpu *h, int inst, double *re, double *im);
/* n_iters iterations of the conductivity sub-problem; stats[n_iters] or NULL. */
pfdd_status pfdd_gpu_cond_step(pfdd_gpu *h, int inst, int n_iters, pfdd_cond_stats *stats);

/* No counterpart in the reference (a hand-written adjoint of the GL step).
 * Gradients of a loss L(Re xi_N), xi_N = instance `inst` after n_steps GL
 * iterations from its current state at the current stress state, with
 * respect to the GSFE parameters and the applied stress, seeded with
 * dL/dRe xi_N; any final-state loss has that seed.
 *
 * pfdd_gpu_adjoint_forward runs the n_steps and keeps them as a tape: the
 * state every ckpt_every steps (with the Nyquist carrier of Im xi) and every
 * state of the last segment, on the device in the compute precision; the
 * instance ends at xi_N, as after pfdd_gpu_advance(h, n_steps, 1, 0, .), so
 * the caller can read xi_N (pfdd_gpu_get_state) to form its seed.
 * pfdd_gpu_adjoint_backward then recomputes each earlier segment from its
 * checkpoint and runs the adjoint steps
 *   lam_n = lam_{n+1} - CD dt (L lam_{n+1} + f''(xi_n) lam_{n+1}),
 * L the self-adjoint elastic operator, masked sites frozen, from
 * lam_N = dL_dxiN.  It may run several seeds on one tape; the tape is
 * dropped when the instance's state changes (advance, set_state, load)
 * (PFDD_ESTATE without one).  ckpt_every >= n_steps keeps every state and
 * recomputes nothing.
 *   dL_dxiN     host [S*N] dL/dRe xi_N (reference site order)
 *   dL_dparams  [2] or NULL: sine / sine-field cores dL/d(isf, usf); perfect
 *               / USFE dL/d(An, -); MPEA (0, 0)  (J/m^2)
 *   dL_dsigma   [6] or NULL: dL/d(sigma xx yy zz xy xz yz), deck units (stress / mu)
 * A non-finite gradient returns PFDD_EDIVERGED.  Core models 2, 4 and 5 have
 * no adjoint (PFDD_EUNSUPPORTED).  pfdd_gpu_adjoint is both calls in one,
 * for a seed known beforehand. */
pfdd_status pfdd_gpu_adjoint_forward(pfdd_gpu *h, int inst, int n_steps, int ckpt_every);
pfdd_status pfdd_gpu_adjoint_backward(pfdd_gpu *h, int inst, const double *dL_dxiN, double *dL_dparams,
                                      double *dL_dsigma);
pfdd_status pfdd_gpu_adjoint(pfdd_gpu *h, int inst, int n_steps, int ckpt_every, const double *dL_dxiN,
                             double *dL_dparams, double *dL_dsigma);

/* Set instance `inst`'s current applied stress (units of mu), replacing the
 * device's copy; dsigma is kept.  The host side of the reference owns sigma
 * (App::sigma, src/app.cpp:325-381, incremented by SolveGL::iterate after each
 * stress state, src/solve_GL.cpp:150-155): a binding that advances one stress
 * state in several chunks (output steps in between) sets it before each chunk,
 * since pfdd_gpu_advance adds dsigma when a stress state ends. */
pfdd_status pfdd_gpu_set_stress(pfdd_gpu *h, int inst, const double sigma[3][3]);

/* ---- Binary checkpoints for resume ----
 * No counterpart in the reference, which keeps no resumable state (its only
 * copies are the in-memory temp_stor_data / reset_data pair,
 * src/fft_fftw_slab.cpp:1891-1925, and the six-digit text dumps,
 * src/dump_text.cpp:361-400).  A checkpoint holds one instance's device state
 * as it is stepped (fields in the compute precision, the Nyquist carrier of
 * Im xi in frequency order, the device's sigma and dsigma), so a handle created from the same
 * descriptor and options that loads it continues bit for bit as the writer
 * would have.  The file is a 256-byte little-endian header with FNV-1a 64
 * checksums of itself and of the payload, then the payload; reading refuses a
 * file whose magic, version, sizes or checksums do not match (PFDD_EINVAL). */
typedef struct {
  int nx, ny, nz, n_slip;
  int fields;                  /* real fields carried: n_slip, or 2 n_slip with the full Im carrier */
  int precision;               /* PFDD_FP64 / PFDD_FP32 of the stored values */
  int imag_mode;               /* PFDD_IMAG_FULL or PFDD_IMAG_NYQUIST */
  int advanced;                /* 1: sigma is one dsigma past the last stress state stepped */
  size_t field_bytes, carrier_bytes;
  double sigma[3][3], dsigma[3][3];
  unsigned long long steps;    /* GL iterations the writer had run (informational) */
} pfdd_checkpoint_info;

/* The file format alone (host only, no device): write a checkpoint from
 * host buffers, or read one (fields == carrier == NULL: the header only). */
pfdd_status pfdd_checkpoint_write(const char *path, const pfdd_checkpoint_info *info, const void *fields,
                                  const void *carrier);
pfdd_status pfdd_checkpoint_read(const char *path, pfdd_checkpoint_info *info, void *fields, size_t field_cap,
                                 void *carrier, size_t carrier_cap);

/* Save instance `inst`'s state to `path`; load it back into an instance of
 * the same grid, slip systems, precision and carrier mode (PFDD_EINVAL
 * otherwise, the instance unchanged). */
pfdd_status pfdd_gpu_checkpoint_save(pfdd_gpu *h, int inst, const char *path);
pfdd_status pfdd_gpu_checkpoint_load(pfdd_gpu *h, int inst, const char *path);

/* Resolved shear stresses tau[S] of instance `inst` at the current stress state. */
pfdd_status pfdd_gpu_tau(pfdd_gpu *h, int inst, double *tau);

/* Run all later work of the handle on a caller-owned cudaStream_t (passed as
 * void* so this header needs no CUDA include); NULL returns to the handle's
 * own stream.  Lets a caller order the stepper against its own work and
 * bracket it with its own events. */
pfdd_status pfdd_gpu_set_stream(pfdd_gpu *h, void *stream);

/* Kernel classes of a run of GL iterations, in launch order: the forward
 * plane pass that opens the run (once), then per iteration the x-pencil pass,
 * the plane pass (inverse transforms + update, fused with the next
 * iteration's forward transforms) and the reduction. */
enum { PFDD_K_FWD_PLANES = 0, PFDD_K_XPENCIL = 1, PFDD_K_STEP_PLANES = 2, PFDD_K_FINALIZE = 3, PFDD_NKERNELS = 4 };

/* Advance n_steps GL iterations (one stress state, no tolerance test) with a
 * CUDA event pair around every launch and return the device time per
 * iteration of each kernel class in kernel_ms[PFDD_NKERNELS] (summed over
 * instances; the opening forward pass is divided by n_steps), and the number
 * of kernel launches one iteration makes (the run adds one stress-state and
 * one opening launch per batched group).  The state advances exactly as with
 * pfdd_gpu_advance. */
pfdd_status pfdd_gpu_profile(pfdd_gpu *h, int n_steps, double *kernel_ms, int *launches_per_step);

/* Number of instances, and the device bytes the handle holds. */
pfdd_status pfdd_gpu_info(pfdd_gpu *h, int *n_instances, size_t *device_bytes);

/* Last error message of the handle (or of the last failed create when h is NULL). */
const char *pfdd_gpu_last_error(pfdd_gpu *h);

/* Release the handle and all its device memory. */
void pfdd_gpu_destroy(pfdd_gpu *h);

/* Size of the device array behind pfdd_gl_step_noalloc (16 MiB per GPU). */
#define PFDD_STATIC_SCRATCH_BYTES (16u << 20)

/* No counterpart in the reference.  One FP64 GL iteration of one instance
 * (Re and Im carried as full fields, so the result is the reference's) that
 * allocates nothing, for callers that cannot call cudaMalloc: host codes whose
 * runtime hands out all device memory through its own pool (a direct
 * cudaMalloc would fragment it or exceed the pool's reservation), and
 * long-running or real-time hosts that must not allocate after start-up
 * (an allocation can block on the device or fail at an arbitrary time).
 *   d_xi_in, d_xi_out  caller-owned DEVICE arrays of 2*S*N doubles: the S Re
 *                      planes, then the S Im planes (reference site order);
 *                      they must not alias
 *   h_stats            NULL, or host double[2] receiving {xinorm, xiave}; when
 *                      given, the call waits for the step and reports
 *                      PFDD_EDIVERGED / PFDD_ETIMEOUT, otherwise it returns
 *                      after enqueueing on `stream` (a cudaStream_t, NULL =
 *                      legacy default stream) and reports neither: the next
 *                      call clears the device flags unread
 * All scratch (half spectrum, partial sums, tables) lives in one file-scope
 * device array of PFDD_STATIC_SCRATCH_BYTES that every GPU loading the library
 * holds until exit; a grid needing more (e.g. above 64^3 with 3 systems)
 * returns PFDD_EINVAL and computes nothing -- use pfdd_gpu_create for those.
 * The first call on a device (with that device current) looks up the array's
 * device address and caches it for the process, so make it before any stream
 * capture; cudaDeviceReset between calls is not supported (the cached address
 * would be stale).  Calls share the array and it keeps the last call's
 * contents; calls whose GPU work overlaps race on it.  The descriptor's mask, per-site
 * GSFE field and dsigma are not used (xo and site_gsfe must be NULL); tau is
 * taken at `sigma`. */
pfdd_status pfdd_gl_step_noalloc(const pfdd_instance_desc *desc, const double *d_xi_in, double *d_xi_out,
                                 double *h_stats, void *stream);

/* Library version string. */
const char *pfdd_gpu_version(void);

#ifdef __cplusplus
}
#endif

#endif /* PFDD_B200_H */
