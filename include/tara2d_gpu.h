/* tara2d_gpu.h -- C ABI of the B200 (sm_100a) pseudo-spectral RHS + time-step
 * path of TARA2D.
 *
 * Two layers:
 *
 * 1. Drop-in entry points with the reference's Fortran calling convention
 *    (gfortran mangling: lowercase name + '_', every argument by reference,
 *    arrays are the caller's column-major complex(8) (Nh,Ny) buffers in host
 *    memory, Nh = Nx/2+1).  Linking the library in place of the reference's
 *    objects makes the drivers' `call derive2coh(...)` etc. run on the GPU.
 *    Physical parameters are read from the COMMON /comm/ block exactly as the
 *    reference subroutines read it (this library defines `comm_` with default
 *    visibility, so a Fortran program's own COMMON block takes precedence).
 *    They return nothing (like the Fortran subroutines); the status of the
 *    last call is available from tara_legacy_status().
 *
 * 2. A session API (bind(C) style, explicit parameters, int status) that
 *    keeps the spectral state resident in HBM and advances it many steps per
 *    call; host arrays are copied only when the caller asks for them.
 *
 * Array convention for every double* "field" argument: interleaved
 * (re, im) pairs of a Fortran complex(8) (Nh,Ny) array, i.e. element
 * (i,j) (1-based) at 2*((i-1) + Nh*(j-1)).
 *
 * Threading: a session is not re-entrant; use one host thread per session.
 * All sessions of a process share the current CUDA device.
 */
#ifndef TARA2D_GPU_H
#define TARA2D_GPU_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---------------------------------------------------- */
#define TARA_OK 0
#define TARA_EINVAL (-1)       /* bad argument (size, pointer, model, stepper) */
#define TARA_ECUDA (-2)        /* a CUDA runtime call failed (see tara_last_error) */
#define TARA_ENAN (-3)         /* a non-finite value was found by a check */
#define TARA_ETIMEOUT (-4)     /* a bounded device wait ran out */
#define TARA_ENOMEM (-5)       /* device allocation failed */
#define TARA_EUNSUPPORTED (-6) /* grid size or mode not built */
#define TARA_ECFL (-7)         /* the time step exceeds the CFL limit (tara_set_cfl) */

/* ---- models ------------------------------------------------------------ */
#define TARA_MODEL_COH 1 /* compressible isothermal hydro (nk, ukx, uky): derive2coh */
#define TARA_MODEL_COM 2 /* compressible MHD (rho, rho_ux, rho_uy, E, Bx, By): derive2com */
#define TARA_MODEL_CSH 3 /* incompressible vorticity (omega): derive2csh */
#define TARA_MODEL_CSS 4 /* screened vorticity (omega): derive2css */

#define TARA_FP64 0 /* FFTs, products and state in double precision */
#define TARA_FP32 1 /* FFTs, products and state in single precision (FP64-accurate tables) */

#define TARA_STEP_AB2 0   /* Adams-Bashforth 2 (src/ab2coh.f95, src/ab2com.f95) */
#define TARA_STEP_RK4 1   /* classical RK4 of the coupled system (new) */
#define TARA_STEP_EULER 2 /* forward Euler (src/euler2coh.f95) */

/* Physical parameters.  Lx, Ly are the box lengths as the drivers hold them
 * after `Lx = Lx*pi` (src/main2coh.f95:102); kx = 2*pi*(i-1)/Lx. */
typedef struct {
  double Lx, Ly, pi, dt;
  double mux, muy, ms, CS;            /* hydro: COMMON /comm/ of src/main2coh.f95:29 */
  double spheat, mu, mu_0, eta, kf, A; /* MHD: COMMON /comm/ of src/main2com.f95:43 (+CS, ms) */
  double nu, alpha, lambda;           /* vorticity models */
  int fix_curlB; /* 0: curl B as the reference builds it (src/derive2com.f95:186-187), 1: corrected */
  int reserved[7];
} tara_params;

typedef struct tara_session tara_session;

/* ---- session API -------------------------------------------------------
 * Replaces the time loops of src/main2coh.f95:266-316 and
 * src/main2com.f95:352-423 (derive + stepper + copy-back per step). */

/* Nx, Ny in {16,32,64,128,256,384,512,1024,2048,4096}. */
int tara_open(tara_session** out, int model, int Nx, int Ny, int precision, const tara_params* p);
int tara_close(tara_session* s);
int tara_set_params(tara_session* s, const tara_params* p);
/* Number of fields of the session's model (3, 6, 1, 1). */
int tara_num_fields(const tara_session* s);
/* State <-> host, reference layout.  `fields` holds tara_num_fields pointers. */
int tara_set_state(tara_session* s, const double* const* fields);
int tara_get_state(tara_session* s, double* const* fields);
/* AB2 history (the *_dt_old arrays of the drivers); zero after tara_open. */
int tara_set_history(tara_session* s, const double* const* fields);
int tara_get_history(tara_session* s, double* const* fields);
/* Right-hand side of the current state (what derive2coh/derive2com return). */
int tara_rhs(tara_session* s, double* const* out);
/* Advance nsteps; asynchronous on the session's stream. */
int tara_step(tara_session* s, int stepper, int nsteps);
int tara_synchronize(tara_session* s);
/* Advance nsteps and return their device time (CUDA events on the session
 * stream, synchronised on both sides). */
int tara_time_steps(tara_session* s, int stepper, int nsteps, float* ms);
/* Kernel launches one step of the given stepper issues. */
int tara_launches_per_step(const tara_session* s, int stepper);
/* Device time of reps plain 2D transforms of nfields fields (1 .. min(6,
 * fields of the model)) on device-resident buffers, the transforms that
 * replace FFTW's dfftw_execute of an r2c / c2r plan (src/derive2com.f95:70-248):
 * inverse = 1: c2r of the state fields into real fields (normalised by
 * Nx Ny, as the drivers divide after every c2r); inverse = 0: r2c of those
 * real fields into work fields (the state is left as it is).  CUDA events on
 * the session stream; *ms is the total of the reps. */
int tara_time_transforms(tara_session* s, int inverse, int nfields, int reps, float* ms);
/* Steps are replayed from CUDA graphs of two steps each (captured on first
 * use per stepper, dropped on tara_set_params); on = 0 launches every kernel
 * from the host instead.  Default: on. */
int tara_set_graphs(tara_session* s, int on);

/* ---- time-step control and state checks (no counterpart in the reference,
 * whose drivers step a fixed dt from the INI file, src/main2com.f95:183-193,
 * and check nothing) ----
 * CFL control, computed on the device in FP64 at the first RHS evaluation of
 * every step from the real-space fields the row pass forms anyway:
 *   rate = max over the grid of (|ux| + c)/dx + (|uy| + c)/dy,
 *   c = CS (hydro) or sqrt(CS^2 + |B|^2/rho) (MHD, fast magnetosonic speed),
 *   dt_cfl = cfl / rate.
 *   TARA_CFL_CHECK: a step whose configured dt exceeds dt_cfl is not taken
 *     (the state stays as it is) and the session reports TARA_ECFL at its
 *     next synchronising call; every stepper.
 *   TARA_CFL_ADAPT: every step uses dt = min(configured dt, dt_cfl); RK4 and
 *     Euler only (AB2's weights assume a constant step); a step whose dt_cfl
 *     falls below 1e-6 of the configured dt is not taken (TARA_ECFL).
 * A rate that is not finite stops the step the same way with TARA_ENAN.
 * Hydro and MHD models; the vorticity models return TARA_EUNSUPPORTED. */
#define TARA_CFL_OFF 0
#define TARA_CFL_CHECK 1
#define TARA_CFL_ADAPT 2
int tara_set_cfl(tara_session* s, int mode, double cfl);
/* Model time advanced by the steps since tara_open (or tara_set_time), and
 * the dt of the last step (the configured dt when the CFL control is off). */
int tara_get_time(tara_session* s, double* t, double* dt_last);
int tara_set_time(tara_session* s, double t);
/* State checks: tara_set_state and tara_set_history check every uploaded
 * value, and every tara_step call checks the state it leaves, for values
 * that are not finite (TARA_ENAN, reported by the call or, for the
 * asynchronous tara_step, by the next synchronising call). */
/* Limit, in ns, of every bounded wait of the session's TMA kernels (default
 * 1 s); a wait that runs out stops its kernel and the session reports
 * TARA_ETIMEOUT. */
int tara_set_wait_limit(tara_session* s, long long limit_ns);
/* Self-test of the bounded wait those kernels use: one CTA waits on an
 * mbarrier that expects 16 bytes no copy delivers (no copy is issued), with
 * the given limit (1 us .. 10 s).  Returns what the kernel reports,
 * TARA_ETIMEOUT when the wait ran out as it must, and the time waited. */
int tara_selftest_bounded_wait(long long limit_ns, long long* waited_ns);

/* ---- diagnostics, computed on the device from the resident state ----
 * Values (all sums in FP64 whatever the precision; the last two are 0):
 *   MHD   (src/main2com.f95:587-604, the Energy.dat line after `time`):
 *         Energy = <|u|^2>, B_Field = <|B|^2>, C2 = <omega^2>, C3 = <j^2>,
 *         div_B_Tot = <div B>, then the cross-helicity <u.B>
 *   hydro (src/main2coh.f95:321-429): Energy/2, y_Energy/2, C0, C1, C2, C3
 *         (C_n = <omega^n>)
 * E(k): tara_num_shells() shells, E(k) = sum over floor(|k| + 1/2) = k of
 * (|ux_k|^2 + |uy_k|^2)/2/(NxNy)^2 (modes 0 < kx index < Nx/2 counted twice).
 * Vorticity models: TARA_EUNSUPPORTED. */
#define TARA_DIAG_VALUES 8
int tara_num_shells(tara_session* s);
int tara_diagnostics(tara_session* s, double* out, int nout, double* Ek, int nbins);
/* nrec records of TARA_DIAG_VALUES + tara_num_shells() doubles: the first of
 * the current state, then one after every `every` steps (nsteps = (nrec - 1)
 * * every in all).  Records stay on the device until the run ends. */
int tara_run_recorded(tara_session* s, int stepper, int every, int nrec, double* rec);

/* ---- real space and the drivers' output files ----
 * Real fields are real(8) (Nx,Ny) host arrays (x fastest).
 * tara_get_state_real: every state field after c2r / (Nx Ny), as the drivers
 * form them before their diagnostics (src/main2com.f95:446-480).
 * tara_get_vorticity_real: omega = c2r(i kx uy_k - i ky ux_k)/(Nx Ny), u the
 * velocity (src/main2coh.f95:321-360; MHD: u = (rho u)/rho, src/main2com.f95:500-540).
 * tara_set_state_real: the state from real fields by the device r2c, the
 * drivers' initial-condition path (src/main2com.f95:257-262).
 * tara_write_snapshot: the drivers' grid file (`fort.NNNNNNNN`,
 * src/main2com.f95:603-609, src/main2coh.f95:414-418), list-directed.
 * tara_format_list_directed: one list-directed record of n REAL(8) values
 * as gfortran writes them (for Energy.dat lines); returns its length. */
int tara_get_state_real(tara_session* s, double* const* fields);
int tara_get_vorticity_real(tara_session* s, double* omega);
int tara_set_state_real(tara_session* s, const double* const* fields);
int tara_write_snapshot(tara_session* s, const char* path);
int tara_format_list_directed(const double* v, int n, char* out, int cap);

/* ---- seeded initial conditions built on the device ----
 * The benchmark configurations' ICs, replacing the drivers' host-side IC
 * construction and r2c (src/main2coh.f95:141-222, src/main2com.f95:230-300).
 * A solenoidal random-phase field has psi_k = a(|k|) e^{2 pi i U} on every
 * half-spectrum mode, a = sqrt(E(|k|)/|k|^3), U a counter-based uniform of
 * (seed, stream, mode) (layout and generator: tara2d_b200/csrc/ic.cu; the
 * host restatement tara2d_b200.initial.hashed_state gives the same state).
 *   TARA_IC_RANDOM_PHASE, hydro: u with E(k) ~ k^4 exp(-(k/k0)^2) and
 *     <|u|^2>/2 = e1; density 1 + e2 N(0,1).
 *   TARA_IC_RANDOM_PHASE, MHD: rho = 1, u and B as above with energies e1, e2.
 *   TARA_IC_ORSZAG_TANG, MHD: u = (-sin y, sin x), B = (-sin y, sin 2x), rho = 1,
 *     plus random-phase perturbations with E(k) ~ k on kmin <= |k| <= kmax of
 *     rms e1 (u) and e2 (B).
 * MHD: P = CS^2 rho, E = P/(spheat-1) + rho|u|^2/2 + |B|^2/2.  The state is
 * replaced; the AB2 history is left as it is.  Vorticity models:
 * TARA_EUNSUPPORTED. */
#define TARA_IC_RANDOM_PHASE 1
#define TARA_IC_ORSZAG_TANG 2
typedef struct {
  int kind;
  int reserved0;
  unsigned long long seed;
  double k0, e1, e2, kmin, kmax;
  double reserved[3];
} tara_ic;
int tara_set_state_random(tara_session* s, const tara_ic* ic);

/* ---- tracer particles (src/main2csh.f95:93-96, 187-268), vorticity models ----
 * np particles at (xp, yp) (host arrays, updated in place).  nsteps > 0:
 * nsteps times, one step of the state (stepper) and then, as the driver does,
 * one forward-Euler move of every particle by dt with the velocity of the new
 * state, positions wrapped into (0, Lx] x (0, Ly].  nsteps = 0: only the
 * velocities at the particles.  vxp, vyp (may be NULL) receive the last
 * velocities; a position that is not finite gets NaN velocities and stays.
 * Velocity: u = c2r(i ky psi_k)/(NxNy), v = c2r(-i kx psi_k)/(NxNy),
 * psi_k = omega_k/(k^2 + lambda) (lambda = 0 for csh), interpolated
 * bilinearly in the particle's grid cell with the reference's formula and
 * operation order (no fused multiply-add); in the last column / row the far
 * corner is x = Lx / y = Ly as in the reference, and the far grid values are
 * those of column / row 1 (the reference reads past its arrays there).
 * Other models: TARA_EUNSUPPORTED. */
int tara_tracers_run(tara_session* s, int stepper, int nsteps, int np, double* xp, double* yp, double* vxp,
                     double* vyp);

/* ---- binary checkpoint / restart (no counterpart in the reference, whose
 * drivers always start from an initial condition: src/main2com.f95:215-343,
 * src/main2coh.f95:176-257) ----
 * tara_checkpoint_write: state, AB2/Euler history, model, grid, parameters
 * and the caller's step count and time to one binary file (FP64 whatever the
 * precision; written to path.tmp, then renamed over path).
 * tara_checkpoint_read: restores parameters, state and history into a session
 * of the same model and grid (the precision may differ) and returns the
 * stored step and time (either pointer may be NULL).  TARA_EINVAL with
 * tara_last_error() set for a missing, truncated or corrupted file (checksum)
 * or a model/grid mismatch.  Layout: tara2d_b200/csrc/checkpoint.cu. */
int tara_checkpoint_write(tara_session* s, const char* path, long long step, double time);
int tara_checkpoint_read(tara_session* s, const char* path, long long* step, double* time);

/* ---- learned subgrid closure of the MHD path (no counterpart in the
 * reference) ----
 * A CNN of four periodic 3x3 convolutions (5 -> 32 -> 32 -> 32 -> 4 channels,
 * GELU after the first three; BF16 weights, FP32 accumulation; activations
 * FP32, TF32 into the tensor-core convolutions) maps the filtered coarse fields (rho - 1, ux, uy, Bx, By) on
 * Nc x Nc to the subgrid stress (tau_xx, tau_xy, tau_yy) and EMF, each
 * normalised by the channel means/scales of tara_closure_get_norm.
 * Training pairs are made on the device from an FP64 MHD session on Nf x Nf
 * (Nc divides Nf) by a sharp spectral filter:
 *   tau_ij = filter(rho u_i u_j + B^2/2 d_ij - B_i B_j) - (same of the filtered state)
 *   EMF    = filter(uy Bx - ux By) - (same of the filtered state).
 * Attached to an FP64 MHD session on Nc x Nc, the RHS adds
 * -(i kx tau_x. + i ky tau_.y) to the momentum and -i ky EMF / +i kx EMF to
 * Bx / By, masked like the resolved fluxes.  Training and a coarse run must
 * not overlap in time (they share the closure's buffers). */
typedef struct tara_closure tara_closure;
int tara_closure_open(tara_closure** out, int Nc, int capacity, int batch_max, unsigned long long seed);
int tara_closure_close(tara_closure* c);
int tara_closure_num_params(void);
int tara_closure_count(const tara_closure* c);
int tara_closure_add_pair(tara_closure* c, tara_session* fine);
/* The same from the current state of member `member` of an ensemble: an FP64
 * MHD member whose grid the closure grid divides (so a batch of DNS runs
 * advanced together as one ensemble produces the training data). */
struct tara_ensemble;
int tara_closure_add_pair_member(tara_closure* c, struct tara_ensemble* e, int member);
int tara_closure_get_pair(tara_closure* c, int idx, float* in5, float* out4);
int tara_closure_get_norm(const tara_closure* c, float* norm18); /* mean_in[5] std_in[5] mean_out[4] std_out[4] */
int tara_closure_set_norm(tara_closure* c, const float* norm18);
int tara_closure_fit_norm(tara_closure* c, int first, int count);
int tara_closure_train(tara_closure* c, int first, int count, int epochs, int batch, float lr, float* epoch_loss);
int tara_closure_eval_loss(tara_closure* c, int first, int count, float* loss);
int tara_closure_get_params(tara_closure* c, float* w);
int tara_closure_set_params(tara_closure* c, const float* w);
int tara_closure_forward(tara_closure* c, const float* in, int B, float* out);
int tara_closure_backward(tara_closure* c, const float* in, const float* dout, int B, float* grad);
/* The 32 -> 32 convolutions (forward and input gradient) run on the tensor
 * cores (tcgen05 MMAs with TF32 activations, FP32 accumulation in tensor
 * memory) when on != 0 (the default) and the plane width is a multiple of
 * 128; on = 0 runs every convolution on CUDA cores with FP32 activations. */
int tara_closure_set_tensor_cores(tara_closure* c, int on);
/* TARA_ETIMEOUT if a bounded wait of a tensor-core convolution ran out since
 * the last check (also reported by forward/backward/train/eval_loss). */
int tara_closure_status(tara_closure* c);
/* Device time per call of the network on B samples (ms): forward, and
 * forward + backward. */
int tara_closure_time_cnn(tara_closure* c, int B, int reps, float* ms_forward, float* ms_backward);
int tara_session_attach_closure(tara_session* s, tara_closure* c); /* c = NULL detaches */
/* Where an attached closure is evaluated in RK4 steps.
 * TARA_CLOSURE_EVERY_RHS (the default): every RHS evaluation, each RK4 stage
 * with the closure of its own input.  TARA_CLOSURE_ONCE_PER_STEP: at the
 * first stage of each step only; stages 2-4 reuse its stress/EMF spectra
 * (first order in time for the subgrid term, a quarter of its cost).  AB2,
 * Euler and single RHS calls evaluate it once per RHS in both modes.  Holds
 * across detach/attach; TARA_EINVAL for another mode value. */
#define TARA_CLOSURE_EVERY_RHS 0
#define TARA_CLOSURE_ONCE_PER_STEP 1
int tara_session_set_closure_mode(tara_session* s, int mode);
int tara_filter_state(tara_session* fine, tara_session* coarse);

/* ---- batched ensembles (no counterpart in the reference, whose drivers run
 * one grid per process) ----
 * n independent runs, member m a hydro (*2coh, src/derive2coh.f95) or MHD
 * (*2com, src/derive2com.f95) run on an N[m] x N[m] grid (N in {128, 256,
 * 384, 512}) with its own parameters params[m] (hydro: mux, muy, CS, dt; MHD:
 * mu, eta, CS, dt with A = 0 and fix_curlB = 0; members of one grid size
 * share Lx, Ly, pi), advanced together: each step is three persistent
 * launches over every hydro member (column inverse, row pass, column forward
 * with the AB2/Euler update) and one over every MHD member (a cooperative
 * launch whose phases, separated by grid-wide barriers, are the first row
 * pass, d(uy)/dy, the second row pass and the column forward with the update
 * and the y-inverse of the new state; a column inverse first where the state
 * was just set), replayed from a CUDA graph.  Each member is bit-identical to a session run
 * of it.  State arrays are complex(8) (Nh,Ny) host arrays as for sessions,
 * tara_ens_num_fields(e, m) of them (3 hydro, 6 MHD); AB2 history starts at
 * zero.  FP32 or FP64 fields; diagnostics sum in FP64. */
typedef struct tara_ensemble tara_ensemble;
/* every member runs `model` (TARA_MODEL_COH or TARA_MODEL_COM) */
int tara_ens_open(tara_ensemble** out, int model, int n, const int* N, const tara_params* params, int precision);
/* member m runs models[m] */
int tara_ens_open_mixed(tara_ensemble** out, int n, const int* models, const int* N, const tara_params* params,
                        int precision);
int tara_ens_close(tara_ensemble* e);
int tara_ens_size(const tara_ensemble* e);
int tara_ens_num_fields(const tara_ensemble* e, int member);
int tara_ens_set_state(tara_ensemble* e, int member, const double* const* fields);
int tara_ens_get_state(tara_ensemble* e, int member, double* const* fields);
int tara_ens_get_history(tara_ensemble* e, int member, double* const* fields);
int tara_ens_step(tara_ensemble* e, int stepper, int nsteps); /* TARA_STEP_AB2 or TARA_STEP_EULER */
int tara_ens_time_steps(tara_ensemble* e, int stepper, int nsteps, float* ms);
/* Tuning of the hydro phases: {values per thread of the column inverse, the
 * row pass and the column forward pass (8 or 16), CTAs per SM of each
 * persistent grid (0 = as many as fit)}.  Default {16, 16, 16, 0, 0, 0}.
 * The MHD phases keep the sessions' values per thread. */
int tara_ens_set_tuning(tara_ensemble* e, const int* tuning6);
int tara_ens_get_tuning(const tara_ensemble* e, int* tuning6);
/* Times every candidate per phase on this ensemble (reps steps each, state
 * and history restored afterwards) and keeps the fastest; chosen6 and
 * best_ms3 (ms per step of each phase) may be NULL. */
int tara_ens_autotune(tara_ensemble* e, int stepper, int reps, int* chosen6, float* best_ms3);
int tara_ens_num_shells(tara_ensemble* e, int member);
int tara_ens_diagnostics(tara_ensemble* e, int member, double* out, int nout, double* Ek, int nbins);
/* Advance nsteps with a CUDA event recorded before every kernel; returns, per
 * kernel kind (index 0..TARA_NUM_KERNEL_KINDS-1, see tara_kernel_name), the
 * summed device time in ms and the number of launches, plus the total. */
#define TARA_NUM_KERNEL_KINDS 12
int tara_profile_steps(tara_session* s, int stepper, int nsteps, double* kernel_ms, int* kernel_launches,
                       float* total_ms);
const char* tara_kernel_name(int kind);
/* Page-lock (pin) a host range for fast host<->device copies, and undo it. */
int tara_host_register(void* p, size_t bytes);
int tara_host_unregister(void* p);
/* PCI bus id ("0000:xx:yy.z") of the current CUDA device. */
int tara_device_pci_bus_id(char* out, int len);
/* Select the CUDA device of the calling thread for later tara_open calls. */
int tara_set_device(int dev);
/* Sticky error of the session (first failure), TARA_OK if none. */
int tara_status(const tara_session* s);
/* Description of the last error of the calling thread ("" if none). */
const char* tara_last_error(void);

/* Explicit-parameter RHS / stepper calls on host arrays (the bind(C)
 * entry points an iso_c_binding shim calls).  Each copies in, computes on
 * the GPU and copies out; the grid context is cached between calls. */
int tara_derive2coh(const tara_params* p, int Nx, int Ny, const double* nk, const double* ukx,
                    const double* uky, double* dn_dt, double* dux_dt, double* duy_dt);
int tara_derive2com(const tara_params* p, int Nx, int Ny, const double* const* state6,
                    double* const* rhs6);

/* Hydro right-hand side that allocates nothing (no counterpart in the
 * reference; it is an addition for hosts that must not allocate device
 * memory from the solver, e.g. a program whose own pool allocator already
 * holds all device memory, or a time-critical loop that cannot afford an
 * allocation's latency and implicit synchronisation).  Same result as
 * tara_derive2coh, but inputs and outputs are device buffers the caller owns
 * (complex(8) (Nh,Ny), no padding) and every temporary lives in one static
 * device workspace of about 6 MB reserved when the library loads.
 * Nx, Ny must be 16, 32, 64, 128 or 256; anything larger returns
 * TARA_EINVAL.  All calls share the workspace, so calls that overlap on the
 * GPU race; calls on one stream are ordered.  The host-side preparation of
 * a call (grid tables, kept while Nx, Ny, Lx, Ly and pi stay the same) is
 * serialised by a lock, so concurrent calls from several host threads are
 * safe on the host side.  The call runs no TMA tile loads and no bounded
 * device waits: its return value is its whole status.  The first call on a
 * device looks up the workspace address and should come before any stream
 * capture.  `stream` is a cudaStream_t (NULL: the default stream). */
int tara_derive2coh_noalloc(const tara_params* p, int Nx, int Ny, const double* nk, const double* ukx,
                            const double* uky, double* dn_dt, double* dux_dt, double* duy_dt, void* stream);

/* ---- drop-in Fortran entry points (reference signatures) ---------------- */
/* src/derive2coh.f95:6-7 */
void derive2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                 const double* time, double* nk, double* ukx, double* uky, double* dn_dt_old,
                 double* dux_dt_old, double* duy_dt_old, double* dn_dt_new, double* dux_dt_new,
                 double* duy_dt_new);
/* src/ab2coh.f95:5-6 */
void ab2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
             const double* time, double* nk, double* ukx, double* uky, double* nk_new,
             double* ukx_new, double* uky_new, double* dn_dt_old, double* dux_dt_old,
             double* duy_dt_old, double* dn_dt_new, double* dux_dt_new, double* duy_dt_new);
/* src/euler2coh.f95:6 */
void euler2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                const double* time, double* nk, double* ukx, double* uky, double* nk_new,
                double* ukx_new, double* uky_new, double* dn_dt, double* dux_dt, double* duy_dt);
/* src/pcnk2coh.f95:6, src/pcukx2coh.f95:6, src/pcuky2coh.f95:6 */
void pc_nk2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                const double* time, double* nk, double* nk_new, double* ukx, double* uky,
                double* dn_dt, double* dux_dt, double* duy_dt);
void pc_ukx2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                 const double* time, double* nk, double* ukx, double* ukx_new, double* uky,
                 double* dn_dt, double* dux_dt, double* duy_dt);
void pc_uky2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                 const double* time, double* nk, double* ukx, double* uky, double* uky_new,
                 double* dn_dt, double* dux_dt, double* duy_dt);
/* src/rk4nk2coh.f95:6, src/rk4ukx2coh.f95:6, src/rk4uky2coh.f95:6 */
void rk4_nk2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                 const double* time, double* nk, double* nk_new, double* ukx, double* uky,
                 double* dn_dt, double* dux_dt, double* duy_dt);
void rk4_ukx2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                  const double* time, double* nk, double* ukx, double* ukx_new, double* uky,
                  double* dn_dt, double* dux_dt, double* duy_dt);
void rk4_uky2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                  const double* time, double* nk, double* ukx, double* uky, double* uky_new,
                  double* dn_dt, double* dux_dt, double* duy_dt);
/* src/derive2com.f95:6-8 (derivatives interleaved old/new per field) */
void derive2com_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                 const double* time, double* rho_k, double* rho_ux_k, double* rho_uy_k,
                 double* E_k, double* Bx_k, double* By_k, double* d_rho_k_dt_old,
                 double* d_rho_k_dt_new, double* d_rho_ux_k_dt_old, double* d_rho_ux_k_dt_new,
                 double* d_rho_uy_k_dt_old, double* d_rho_uy_k_dt_new, double* d_E_k_dt_old,
                 double* d_E_k_dt_new, double* d_Bx_k_dt_old, double* d_Bx_k_dt_new,
                 double* d_By_k_dt_old, double* d_By_k_dt_new);
/* src/ab2com.f95:6-9 */
void ab2com_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
             const double* time, double* rho_k, double* rho_ux_k, double* rho_uy_k, double* E_k,
             double* Bx_k, double* By_k, double* rho_k_new, double* rho_ux_k_new,
             double* rho_uy_k_new, double* E_k_new, double* Bx_k_new, double* By_k_new,
             double* d_rho_k_dt_old, double* d_rho_k_dt_new, double* d_rho_ux_k_dt_old,
             double* d_rho_ux_k_dt_new, double* d_rho_uy_k_dt_old, double* d_rho_uy_k_dt_new,
             double* d_E_k_dt_old, double* d_E_k_dt_new, double* d_Bx_k_dt_old,
             double* d_Bx_k_dt_new, double* d_By_k_dt_old, double* d_By_k_dt_new);

/* Incompressible vorticity models.  These take their parameters as
 * arguments, not from COMMON.  derive2csh_/derive2css_ use the reference's
 * pi = 3.1428 (a default-real literal), with Lx = Ly = 2 pi for csh.
 * derive2csh_ replaces src/derive2csh.f95:3 and writes dt_omegak_new;
 * ab2csh_ replaces src/ab2csh.f95:3 and writes omegak_new. */
void derive2csh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* nu,
                 const double* time, double* omegak, double* omegak_new, double* dt_omegak_old,
                 double* dt_omegak_new);
void ab2csh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* nu,
             const double* time, const double* dt, double* omegak, double* omegak_new,
             double* dt_omegak_old, double* dt_omegak_new);
/* Screened model.  derive2css_ replaces src/derive2css.f95:6 and ab2css_
 * replaces src/ab2css.f95:6.  rk42css_ replaces src/rk42css.f95:6, which reads
 * uninitialised stage derivatives; here it takes one classical RK4 step and
 * writes omegak_new only.  The reference never sets Lx, Ly and lambda in
 * derive2css; they come from tara_set_css_box (default 2 pi, 2 pi, 10, the
 * driver's values at src/main2css.f95:78-87). */
void derive2css_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* alpha,
                 const double* nu, const double* time, double* omegak, double* omegak_new,
                 double* dt_omegak_old, double* dt_omegak_new);
void ab2css_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* alpha,
             const double* nu, const double* time, const double* dt, double* omegak,
             double* omegak_new, double* dt_omegak_old, double* dt_omegak_new);
void rk42css_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* alpha,
              const double* nu, const double* time, const double* dt, double* omegak,
              double* omegak_new, double* dt_omegak_old, double* dt_omegak_new);
int tara_set_css_box(double Lx, double Ly, double lambda);

/* Status of the last drop-in call of the calling thread. */
int tara_legacy_status(void);
/* Semantics of pc_*2coh_ / rk4_*2coh_:
 *   TARA_LEGACY_REFERENCE (default): what the reference computes -- every
 *     stage reads the unchanged argument derivative, so the update equals
 *     (predict+correct)*dt/2 resp. dt/6*(k1+2k2+2k3+k4) with all k equal
 *     (src/pcnk2coh.f95:31, src/rk4nk2coh.f95:33-54).  The reference's
 *     inner derive2coh calls write only subroutine-local arrays and are not
 *     repeated.
 *   TARA_LEGACY_CORRECT: stage derivatives are recomputed (other fields
 *     frozen), and the last RK4 stage is taken at dt. */
#define TARA_LEGACY_REFERENCE 0
#define TARA_LEGACY_CORRECT 1
int tara_set_legacy_mode(int mode);

/* COMMON /comm/ storage used by the drop-in entry points (11 doubles:
 * hydro units read Lx,Ly,mux,muy,ms,CS,dt; MHD units read
 * Lx,Ly,spheat,mu,ms,CS,mu_0,eta,dt,kf,A).  The 3D MHD units read the 3D
 * driver's block (src/main3com.f95:56): two integer(4) (iret, thread_num) in
 * the first 8 bytes, then time_max,Lx,Ly,Lz,dx,dy,dz,spheat,mu,ms,CS,mu_0,
 * eta,dt,kf as comm_[1..15]. */
extern double comm_[16];

/* ---------------------------------------------------------------------------
 * 3D compressible MHD (src/derive3com.f95:5-1047, src/ab3com.f95:6-66), FP64.
 *
 * Spectral fields are the reference's complex(8) (Nh,Ny,Nz) arrays,
 * Nh = Nx/2+1, as interleaved (re, im) doubles; the 8 fields are, in order,
 * rho, rho ux, rho uy, rho uz, E, Bx, By, Bz.  Nx, Ny, Nz in
 * {16, 32, 64, 128, 256, 512}.  The reference's constants are kept: the
 * momentum and induction equations diffuse with 1/450 (not mu), the energy
 * equation adds mu (div u)^2, eta enters only the energy flux, and ab3com
 * leaves E unchanged.
 * ------------------------------------------------------------------------- */
typedef struct tara3d tara3d;
typedef struct {
  double pi, Lx, Ly, Lz;  /* box lengths as the reference holds them (already times pi) */
  double mu, CS, eta, dt; /* COMMON /comm/ mu, CS, eta, dt of src/main3com.f95:56 */
  double reserved[8];
} tara3d_params;

/* One device-resident 3D state; AB2 history starts at zero (the reference's
 * d_*_dt_old before the first step). */
int tara3d_open(tara3d** out, int Nx, int Ny, int Nz, const tara3d_params* p);
int tara3d_close(tara3d* s);
int tara3d_set_params(tara3d* s, const tara3d_params* p);
/* host <-> device, 8 fields of Nh*Ny*Nz complex(8) each */
int tara3d_set_state(tara3d* s, const double* const fields[8]);
int tara3d_get_state(tara3d* s, double* const fields[8]);
int tara3d_set_history(tara3d* s, const double* const d_old[8]);
/* derive3com of the current state into host arrays (state unchanged) */
int tara3d_rhs(tara3d* s, double* const d_new[8]);
/* nsteps of derive3com + ab3com + history shift (src/main3com.f95:548-600) */
int tara3d_step(tara3d* s, int nsteps);
/* the same, timed on the device with CUDA events (milliseconds in *ms) */
int tara3d_time_steps(tara3d* s, int nsteps, float* ms);
/* kernel launches of one step */
int tara3d_launches_per_step(tara3d* s);

/* Drop-in replacements (gfortran names) of the 3D subroutines; parameters
 * from comm_ as laid out above.  Status in tara_legacy_status(). */
void derive3com_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nz, const int32_t* Nh,
                 const double* pi, const double* time, double* rho_k, double* rho_ux_k,
                 double* rho_uy_k, double* rho_uz_k, double* E_k, double* Bx_k, double* By_k,
                 double* Bz_k, double* d_rho_k_dt_old, double* d_rho_k_dt_new,
                 double* d_rho_ux_k_dt_old, double* d_rho_ux_k_dt_new, double* d_rho_uy_k_dt_old,
                 double* d_rho_uy_k_dt_new, double* d_rho_uz_k_dt_old, double* d_rho_uz_k_dt_new,
                 double* d_E_k_dt_old, double* d_E_k_dt_new, double* d_Bx_k_dt_old,
                 double* d_Bx_k_dt_new, double* d_By_k_dt_old, double* d_By_k_dt_new,
                 double* d_Bz_k_dt_old, double* d_Bz_k_dt_new);
void ab3com_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nz, const int32_t* Nh,
             const double* pi, const double* time, double* rho_k, double* rho_ux_k, double* rho_uy_k,
             double* rho_uz_k, double* E_k, double* Bx_k, double* By_k, double* Bz_k,
             double* rho_k_new, double* rho_ux_k_new, double* rho_uy_k_new, double* rho_uz_k_new,
             double* E_k_new, double* Bx_k_new, double* By_k_new, double* Bz_k_new,
             double* d_rho_k_dt_old, double* d_rho_k_dt_new, double* d_rho_ux_k_dt_old,
             double* d_rho_ux_k_dt_new, double* d_rho_uy_k_dt_old, double* d_rho_uy_k_dt_new,
             double* d_rho_uz_k_dt_old, double* d_rho_uz_k_dt_new, double* d_E_k_dt_old,
             double* d_E_k_dt_new, double* d_Bx_k_dt_old, double* d_Bx_k_dt_new,
             double* d_By_k_dt_old, double* d_By_k_dt_new, double* d_Bz_k_dt_old,
             double* d_Bz_k_dt_new);

#ifdef __cplusplus
}
#endif
#endif
