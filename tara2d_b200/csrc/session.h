// The session object behind the C ABI's opaque tara_session handle: one grid
// whose state stays in HBM, with its own stream.  The precision-specific
// implementation (SessionT<double|float>) lives in api.cu.
#pragma once
#include <cuda_runtime.h>
#include "prof.h"
#include "../../include/tara2d_gpu.h"

struct tara_session {
  int model = 0, precision = 0, Nx = 0, Ny = 0, Nh = 0, nf = 0;
  tara_params p{};
  cudaStream_t st = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  int status = TARA_OK;
  tara::Prof prof;
  virtual ~tara_session() {
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (st) cudaStreamDestroy(st);
  }
  virtual int init() = 0;
  virtual int apply_params() = 0;
  virtual int set_fields(int which, const double* const* h) = 0;  // which: 0 state, 1 history
  virtual int get_fields(int which, double* const* h) = 0;
  virtual int rhs_to_host(double* const* out) = 0;
  virtual int step(int stepper, int n) = 0;
  virtual int launches(int stepper) const = 0;
  int fail_if(int s) {
    if (s != TARA_OK && status == TARA_OK) status = s;
    return s;
  }
  // Device status word: TARA_ETIMEOUT when a kernel's bounded wait ran out
  // (the word is cleared after it has been reported).
  virtual int device_status() = 0;
  // elementwise stepper on host fields (drop-in ab2/euler/pc/rk4 entry points);
  // nfld fields, each out = stepper(u, d1, d2)
  virtual int elementwise(int mode, int nfld, const double* const* u, const double* const* d1,
                          const double* const* d2, double* const* out) = 0;
  // per-field PC / RK4 with the other hydro fields frozen (TARA_LEGACY_CORRECT)
  virtual int frozen_field_step(bool rk4, int which, const double* const* f, const double* d,
                                double* out) = 0;
  virtual int num_shells() = 0;
  virtual void set_graphs(bool on) = 0;
  // what = 0: the nf state fields in real space (c2r / NxNy); 1: vorticity
  virtual int real_fields(int what, double* const* h) = 0;
  virtual int set_state_real(const double* const* h) = 0;
  // the state from a seeded initial condition built on the device
  virtual int set_state_random(const tara_ic* ic) = 0;
  // tracer particles (host arrays of np): nsteps steps of the state, each
  // followed by one particle move with the new state's velocity (nsteps = 0:
  // only the velocities at the particles)
  virtual int tracers_run(int stepper, int nsteps, int np, double* xp, double* yp, double* vxp, double* vyp) = 0;
  // nrec diagnostics records of the state, one before the first step and one
  // after every `every` steps (nsteps = (nrec - 1) * every), into rec
  // (host, nrec * (TARA_DIAG_VALUES + num_shells()) doubles)
  virtual int run_recorded(int stepper, int every, int nrec, double* rec) = 0;
  // device time of reps plain 2D c2r (inverse) or r2c of nfields fields
  virtual int time_transforms(int inverse, int nfields, int reps, float* ms) = 0;
  // for the closure code: the grid (const tara::Grid<T>*), state field q
  // (tara::Cx<T>*), and the closure whose term the MHD RHS adds (NULL: none)
  virtual const void* grid_ptr() const = 0;
  virtual void* state_ptr(int q) = 0;
  virtual int attach_closure(tara_closure* c) = 0;
  virtual int set_closure_mode(int mode) = 0;  // TARA_CLOSURE_*
  // the state was changed from outside the stepping kernels: drop what was
  // derived from it
  virtual void invalidate_derived() = 0;
  // CFL control (TARA_CFL_*), model time, bounded-wait limit
  virtual int set_cfl(int mode, double number) = 0;
  virtual int get_time(double* t, double* dt) = 0;
  virtual int set_time(double t) = 0;
  virtual int set_wait_limit(long long ns) = 0;
};
