// C ABI: sessions (state resident in HBM) and the drop-in Fortran entry
// points with the reference's calling convention.
#include <cstdio>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <tuple>
#include <vector>
#include "models.h"
#include "closure.h"
#include "diag.cuh"
#include "output.h"
#include "ic.cuh"
#include "tracers.cuh"
#include "realspace.cuh"
#include "session.h"

using namespace tara;

extern "C" {
double comm_[16] = {0};
}

namespace {

// host complex(8) (Nh,Ny) <-> device [Ny][ld] Cx<float>
__global__ void k_f64_to_f32(const double2* __restrict__ src, Cx<float>* dst, int Nh, int ld, int Ny) {
  size_t n = (size_t)Nh * Ny;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    int j = (int)(q / Nh), i = (int)(q % Nh);
    double2 v = src[q];
    dst[(size_t)j * ld + i] = cx<float>((float)v.x, (float)v.y);
  }
}
__global__ void k_f32_to_f64(const Cx<float>* src, double2* __restrict__ dst, int Nh, int ld, int Ny) {
  size_t n = (size_t)Nh * Ny;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    int j = (int)(q / Nh), i = (int)(q % Nh);
    Cx<float> v = src[(size_t)j * ld + i];
    dst[q] = make_double2((double)v.x, (double)v.y);
  }
}

// elementwise steppers on [Ny][ld] fields
enum : int { EW_AB2 = 0, EW_EULER = 1, EW_PC_REF = 2, EW_RK4_REF = 3, EW_AXPY = 4, EW_PC = 5 };
template <class T> struct EwArgs {
  int mode, nf, Nh, ld, Ny;
  T dt, alpha;
  const Cx<T>* u[6];
  const Cx<T>* d1[6];
  const Cx<T>* d2[6];
  Cx<T>* out[6];
};
// Operation order: ab2coh.f95:22, euler2coh.f95:104, pcnk2coh.f95:32, rk4nk2coh.f95:54.
template <class T>
__global__ void k_elementwise(const EwArgs<T> a) {
  const size_t n = (size_t)a.Nh * a.Ny;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const size_t o = (q / a.Nh) * a.ld + (q % a.Nh);
    for (int f = 0; f < a.nf; f++) {
      const Cx<T> u = a.u[f][o], d = a.d1[f][o];
      Cx<T> r;
      switch (a.mode) {
        case EW_AB2: r = u + rmul(a.dt, rmul((T)1.5, d) - rmul((T)0.5, a.d2[f][o])); break;
        case EW_EULER: r = u + rmul(a.dt, d); break;
        case EW_PC_REF: case EW_PC: {
          const Cx<T> s = d + (a.mode == EW_PC ? a.d2[f][o] : d);
          r = u + cx<T>(s.x * a.dt / (T)2, s.y * a.dt / (T)2);
          break;
        }
        case EW_RK4_REF: {
          const Cx<T> s = ((d + rmul((T)2, d)) + rmul((T)2, d)) + d;
          r = u + rmul(a.alpha, s);  // alpha = dt/6
          break;
        }
        default: r = u + rmul(a.alpha, d); break;  // EW_AXPY
      }
      a.out[f][o] = r;
    }
  }
}

int nfields_of(int model) {
  switch (model) {
    case TARA_MODEL_COH: return 3;
    case TARA_MODEL_COM: return 6;
    case TARA_MODEL_CSH: case TARA_MODEL_CSS: return 1;
    default: return 0;
  }
}

}  // namespace

namespace {

template <class T>
struct SessionT : tara_session {
  Grid<T> g;
  FieldPool<T> u, unew, dold, acc, us, us2, tmp;
  FieldPool<double> stage;  // FP32 sessions: FP64 staging of host transfers
  CohWork<T> cw;
  ComWork<T> mw;
  VortWork<T> vw;
  CohParamsT<T> cohp{};
  ComParamsT<T> comp{};
  VortParamsT<T> vortp{};
  DiagWork<T> dw;

  ~SessionT() override {
    if (st) cudaStreamSynchronize(st);
    drop_graphs();
    g.release(); u.release(); unew.release(); dold.release(); acc.release(); us.release(); us2.release();
    tmp.release(); dw.release(); closf.release();
    if (cfl_dev) cudaFree(cfl_dev);
    if (rbuf) cudaFree(rbuf);
    if (rstage) cudaFree(rstage);
    stage.release(); cw.release(); mw.release(); vw.release();
  }

  int init() override {
    TARA_TRY(g.init(Nx, Ny, p.Lx, p.Ly, p.pi, st));
    g.prof = &prof;
    TARA_TRY(u.alloc(g, nf, st));
    TARA_TRY(dold.alloc(g, nf, st));
    TARA_TRY(acc.alloc(g, nf, st));
    TARA_TRY(us.alloc(g, nf, st));
    TARA_TRY(us2.alloc(g, nf, st));
    TARA_TRY(unew.alloc(g, nf, st));
    TARA_TRY(tmp.alloc(g, nf, st));
    if (cudaMalloc(&cfl_dev, sizeof(CflDev)) != cudaSuccess) {
      cfl_dev = nullptr;
      set_error("cudaMalloc of the CFL state failed");
      return TARA_ENOMEM;
    }
    TARA_CUDA_TRY(cudaMemsetAsync(cfl_dev, 0, sizeof(CflDev), st));
    if (sizeof(T) != sizeof(double)) {
      // staging as complex128 [Ny][Nh] (host layout, no pitch)
      stage.elems = (size_t)Nh * Ny;
      stage.count = 1;
      if (cudaMalloc(&stage.base, stage.elems * sizeof(Cx<double>)) != cudaSuccess) {
        stage.base = nullptr;
        set_error("cudaMalloc of staging buffer failed");
        return TARA_ENOMEM;
      }
    }
    switch (model) {
      case TARA_MODEL_COH: TARA_TRY(cw.alloc(g, st)); break;
      case TARA_MODEL_COM: TARA_TRY(mw.alloc(g, st)); break;
      default: TARA_TRY(vw.alloc(g, st)); break;
    }
    TARA_TRY(apply_params());
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    return TARA_OK;
  }

  int apply_params() override {
    drop_graphs();
    h_for = nullptr;
    if (p.Lx != g.Lx || p.Ly != g.Ly || p.pi != g.pi) {
      // wavenumber tables depend on Lx, Ly and pi
      TARA_CUDA_TRY(cudaStreamSynchronize(st));
      g.release();
      TARA_TRY(g.init(Nx, Ny, p.Lx, p.Ly, p.pi, st));
      g.prof = &prof;
    }
    cohp.mux = (T)p.mux;
    cohp.muy = (T)p.muy;
    cohp.cs2 = (T)(p.CS * p.CS);
    comp.mu = (T)p.mu;
    comp.eta = (T)p.eta;
    comp.cs2 = (T)(p.CS * p.CS);
    comp.kf = (T)p.kf;
    comp.A = (T)p.A;
    comp.fix_curlB = p.fix_curlB;
    vortp.nu = (T)p.nu;
    vortp.alpha = (T)p.alpha;
    vortp.lambda = (T)p.lambda;
    vortp.screened = model == TARA_MODEL_CSS;
    return TARA_OK;
  }

  FieldPool<T>& pool(int which) { return which == 0 ? u : dold; }

  int device_status() override {
    int v = 0;
    TARA_CUDA_TRY(cudaMemcpyAsync(&v, g.tb.status, sizeof(int), cudaMemcpyDeviceToHost, st));
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    if (v != TARA_OK) {
      const int zero = 0;
      cudaMemcpyAsync(g.tb.status, &zero, sizeof(int), cudaMemcpyHostToDevice, st);
      cudaStreamSynchronize(st);
      switch (v) {
        case TARA_ENAN: set_error("a value that is not finite was found (state, history or CFL rate)"); break;
        case TARA_ECFL: set_error("the time step exceeds the CFL limit; the step was not taken"); break;
        default: set_error("a bounded wait for a TMA tile load ran out in a kernel"); break;
      }
      return v;
    }
    return TARA_OK;
  }

  // ---- CFL control (first RHS of every step) and time
  CflDev* cfl_dev = nullptr;
  int cfl_mode = CFL_OFF;
  double cfl_number = 0.0;
  double t_off = 0.0;   // model time of the steps taken with the CFL control off
  CflCfg cur_cfl{};     // settings of the RHS being launched
  CflCfg cfl_cfg() const {
    if (cfl_mode == CFL_OFF) return CflCfg{};
    CflCfg c{};
    c.dev = cfl_dev;
    c.mode = cfl_mode;
    c.number = cfl_number;
    c.dt = p.dt;
    c.idx = (double)Nx / p.Lx;
    c.idy = (double)Ny / p.Ly;
    c.cs2 = p.CS * p.CS;
    return c;
  }
  int set_cfl(int mode, double number) override {
    if (model != TARA_MODEL_COH && model != TARA_MODEL_COM) {
      set_error("the CFL control is defined for the hydro and MHD models");
      return TARA_EUNSUPPORTED;
    }
    if (mode != CFL_OFF && mode != CFL_CHECK && mode != CFL_ADAPT) { set_error("unknown CFL mode"); return TARA_EINVAL; }
    if (mode != CFL_OFF && !(number > 0.0)) { set_error("the CFL number must be positive"); return TARA_EINVAL; }
    drop_graphs();  // the graphs hold the CFL settings in their kernel arguments
    cfl_mode = mode;
    cfl_number = number;
    return TARA_OK;
  }
  int get_time(double* t, double* dt) override {
    CflDev d{};
    TARA_CUDA_TRY(cudaMemcpyAsync(&d, cfl_dev, sizeof(CflDev), cudaMemcpyDeviceToHost, st));
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    if (t) *t = t_off + d.t;
    if (dt) *dt = cfl_mode == CFL_OFF ? p.dt : d.dt;
    return TARA_OK;
  }
  int set_time(double t) override {
    double td = 0.0;
    TARA_CUDA_TRY(cudaMemcpyAsync(&td, &cfl_dev->t, sizeof(double), cudaMemcpyDeviceToHost, st));
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    t_off = t - td;
    return TARA_OK;
  }
  int set_wait_limit(long long ns) override {
    if (ns < 1000) { set_error("wait limit below 1 us"); return TARA_EINVAL; }
    drop_graphs();
    g.tb.wait_ns = (unsigned long long)ns;
    return TARA_OK;
  }
  // TARA_ENAN into the status word when a value of these fields is not finite
  int check_finite(FieldPool<T>& f) {
    Cx<T>* q[6];
    for (int k = 0; k < nf; k++) q[k] = f[k];
    return launch_finite_check(g, q, nf, st);
  }

  int h2d(const double* h, Cx<T>* d) {
    if (!h) { set_error("null host field pointer"); return TARA_EINVAL; }
    if constexpr (sizeof(T) == sizeof(double)) {
      TARA_CUDA_TRY(cudaMemcpy2DAsync(d, g.ld * sizeof(Cx<T>), h, Nh * sizeof(Cx<double>),
                                      Nh * sizeof(Cx<double>), Ny, cudaMemcpyHostToDevice, st));
    } else {
      TARA_CUDA_TRY(cudaMemcpyAsync(stage.base, h, stage.elems * sizeof(Cx<double>),
                                    cudaMemcpyHostToDevice, st));
      k_f64_to_f32<<<512, 256, 0, st>>>(reinterpret_cast<const double2*>(stage.base),
                                        reinterpret_cast<Cx<float>*>(d), Nh, g.ld, Ny);
      TARA_CUDA_TRY(cudaGetLastError());
    }
    return TARA_OK;
  }
  int d2h(const Cx<T>* d, double* h) {
    if (!h) { set_error("null host field pointer"); return TARA_EINVAL; }
    if constexpr (sizeof(T) == sizeof(double)) {
      TARA_CUDA_TRY(cudaMemcpy2DAsync(h, Nh * sizeof(Cx<double>), d, g.ld * sizeof(Cx<T>),
                                      Nh * sizeof(Cx<double>), Ny, cudaMemcpyDeviceToHost, st));
    } else {
      k_f32_to_f64<<<512, 256, 0, st>>>(reinterpret_cast<const Cx<float>*>(d),
                                        reinterpret_cast<double2*>(stage.base), Nh, g.ld, Ny);
      TARA_CUDA_TRY(cudaGetLastError());
      TARA_CUDA_TRY(cudaMemcpyAsync(h, stage.base, stage.elems * sizeof(Cx<double>),
                                    cudaMemcpyDeviceToHost, st));
    }
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    return TARA_OK;
  }

  int set_fields(int which, const double* const* h) override {
    if (!h) { set_error("null field array"); return TARA_EINVAL; }
    if (which == 0) h_for = nullptr;
    for (int f = 0; f < nf; f++) TARA_TRY(h2d(h[f], pool(which)[f]));
    TARA_TRY(check_finite(pool(which)));
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    return device_status();
  }
  int get_fields(int which, double* const* h) override {
    if (!h) { set_error("null field array"); return TARA_EINVAL; }
    for (int f = 0; f < nf; f++) TARA_TRY(d2h(pool(which)[f], h[f]));
    return device_status();
  }

  int rhs(Cx<T>* const* in, const StepArgs<T>& s) {
    switch (model) {
      case TARA_MODEL_COH:
        cohp.cfl = cur_cfl;
        return coh_rhs(g, cw, cohp, in, s, st);
      case TARA_MODEL_COM: {
        if constexpr (sizeof(T) == sizeof(double)) {
          // the learned closure's stress/EMF spectra for this RHS input; once
          // per step, RK4 stages 1-3 keep those of stage 0
          if (clos && (clos_mode == TARA_CLOSURE_EVERY_RHS || s.mode != STEP_RK4 || s.stage == 0)) {
            Cx<double>* out4[4] = {closf[0], closf[1], closf[2], closf[3]};
            TARA_TRY(closure_terms(clos, g, in, out4, st));
          }
        }
        // the column-inverse pass runs only when mw.H does not already hold
        // the y-inverse of this input; stepping RHS write it for the next input
        comp.skip_inv = h_for == (const void*)in[0];
        comp.fuse_inv = s.mode != STEP_RHS;
        comp.cfl = cur_cfl;
        const int r = com_rhs(g, mw, comp, in, s, st);
        if (s.mode == STEP_RHS) h_for = in[0];
        else if (s.mode == STEP_RK4 && s.stage < 3) h_for = s.us[0];
        else h_for = s.unew[0];
        return r;
      }
      default: return vort_rhs(g, vw, vortp, in, s, st);
    }
  }

  // MHD: the field set whose y-inverse mw.H holds (nullptr: none)
  const void* h_for = nullptr;
  void invalidate_derived() override { h_for = nullptr; }

  // learned closure (MHD, FP64 sessions of the closure's coarse grid)
  tara_closure* clos = nullptr;
  int clos_mode = TARA_CLOSURE_EVERY_RHS;
  FieldPool<T> closf;
  int set_closure_mode(int mode) override {
    if (mode != TARA_CLOSURE_EVERY_RHS && mode != TARA_CLOSURE_ONCE_PER_STEP) {
      set_error("closure mode must be TARA_CLOSURE_EVERY_RHS or TARA_CLOSURE_ONCE_PER_STEP");
      return TARA_EINVAL;
    }
    if (mode != clos_mode) drop_graphs();  // captured steps hold the closure launches of the old mode
    clos_mode = mode;
    return TARA_OK;
  }
  const void* grid_ptr() const override { return &g; }
  void* state_ptr(int q) override { return q >= 0 && q < nf ? (void*)u[q] : nullptr; }
  int attach_closure(tara_closure* c) override {
    drop_graphs();
    if (!c) {
      clos = nullptr;
      comp.closure = 0;
      return TARA_OK;
    }
    if (model != TARA_MODEL_COM || sizeof(T) != sizeof(double) || Nx != Ny || Nx != closure_grid(c)) {
      set_error("a closure attaches to an FP64 MHD session on its coarse grid");
      return TARA_EINVAL;
    }
    if (!closf.base) TARA_TRY(closf.alloc(g, 4, st));
    clos = c;
    comp.closure = 1;
    for (int q = 0; q < 4; q++) comp.clos[q] = closf[q];
    return TARA_OK;
  }
  StepArgs<T> base_args(int mode) {
    StepArgs<T> s{};
    s.mode = mode;
    s.dt = (T)p.dt;
    s.scale = (cfl_mode != CFL_OFF && mode != STEP_RHS) ? &cfl_dev->scale : nullptr;
    for (int f = 0; f < nf; f++) {
      s.out[f] = tmp[f];
      s.u[f] = u[f];
      s.unew[f] = unew[f];
      s.dold[f] = dold[f];
      s.acc[f] = acc[f];
      s.us[f] = us[f];
    }
    return s;
  }
  int rhs_to_host(double* const* out) override {
    if (!out) { set_error("null field array"); return TARA_EINVAL; }
    Cx<T>* in[6];
    for (int f = 0; f < nf; f++) in[f] = u[f];
    TARA_TRY(rhs(in, base_args(STEP_RHS)));
    for (int f = 0; f < nf; f++) TARA_TRY(d2h(tmp[f], out[f]));
    return device_status();
  }
  // One step reads the state from `u` and writes the new state to `unew`
  // (the RHS of one field reads other fields of its input state, so no
  // kernel may update a state it also reads); the two are swapped after the
  // step.  RK4 stage inputs alternate between us and us2 for the same reason.
  // CUDA graphs of two steps (after which u and unew are back in place), one
  // per (stepper, buffer holding the state); kernel arguments are baked in,
  // so a parameter change drops them.
  struct StepGraph {
    int stepper = -1;
    const void* ubase = nullptr;
    bool hv = false;  // MHD: captured with mw.H holding the inverse of the state
    cudaGraphExec_t exec = nullptr;
  };
  StepGraph graphs[6];
  void drop_graphs() {
    for (auto& gr : graphs) {
      if (gr.exec) cudaGraphExecDestroy(gr.exec);
      gr = StepGraph{};
    }
  }
  cudaGraphExec_t pair_graph(int stepper) {
    for (auto& gr : graphs)
      if (gr.exec && gr.stepper == stepper && gr.ubase == u.base && gr.hv == (h_for == (const void*)u[0]))
        return gr.exec;
    StepGraph* slot = nullptr;
    for (auto& gr : graphs)
      if (!gr.exec) { slot = &gr; break; }
    if (!slot) { drop_graphs(); slot = &graphs[0]; }
    const void* ub = u.base;
    const FieldPool<T> u0 = u, unew0 = unew;
    const void* h0 = h_for;
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal) != cudaSuccess) return nullptr;
    int r = launch_steps(stepper, 2);
    cudaError_t e = cudaStreamEndCapture(st, &graph);
    u = u0;  // nothing ran while capturing
    unew = unew0;
    h_for = h0;
    cudaGetLastError();
    cudaGraphExec_t exec = nullptr;
    if (r == TARA_OK && e == cudaSuccess && graph && cudaGraphInstantiate(&exec, graph, 0) != cudaSuccess) exec = nullptr;
    if (graph) cudaGraphDestroy(graph);
    cudaGetLastError();
    if (!exec) return nullptr;
    slot->stepper = stepper;
    slot->ubase = ub;
    slot->hv = h0 == (const void*)u[0];
    slot->exec = exec;
    return exec;
  }
  bool use_graphs = true;
  void set_graphs(bool on) override {
    use_graphs = on;
    if (!on) drop_graphs();
  }

  int step(int stepper, int n) override {
    if (stepper != TARA_STEP_AB2 && stepper != TARA_STEP_EULER && stepper != TARA_STEP_RK4) {
      set_error("unknown stepper");
      return TARA_EINVAL;
    }
    if (cfl_mode == CFL_ADAPT && stepper == TARA_STEP_AB2) {
      set_error("the adaptive CFL step needs RK4 or Euler (AB2's weights assume a constant dt)");
      return TARA_EINVAL;
    }
    TARA_TRY(step_launch(stepper, n));
    if (cfl_mode == CFL_OFF) t_off += n * p.dt;
    // the state this call leaves must be finite (reported at the next
    // synchronising call)
    return n > 0 ? check_finite(u) : TARA_OK;
  }
  int step_launch(int stepper, int n) {
    int done = 0;
    if (model == TARA_MODEL_COM && n >= 1 && h_for != (const void*)u[0]) {
      // one step with the column-inverse pass; after it mw.H holds the inverse
      // of the state, as the graphs (captured in that condition) assume
      TARA_TRY(launch_steps(stepper, 1));
      done = 1;
    }
    if (use_graphs && !prof.on && n - done >= 2) {
      cudaGraphExec_t ex = pair_graph(stepper);
      if (ex) {
        // capture swapped u/unew twice: the state is back in the same buffer
        // (and mw.H, for MHD, again holds its inverse)
        for (; done + 2 <= n; done += 2) TARA_CUDA_TRY(cudaGraphLaunch(ex, st));
      }
    }
    return launch_steps(stepper, n - done);
  }
  int launch_steps(int stepper, int n) {
    for (int t = 0; t < n; t++) {
      Cx<T>* in_u[6];
      for (int f = 0; f < nf; f++) in_u[f] = u[f];
      if (stepper == TARA_STEP_AB2 || stepper == TARA_STEP_EULER) {
        cur_cfl = cfl_cfg();
        const int r = rhs(in_u, base_args(stepper == TARA_STEP_AB2 ? STEP_AB2 : STEP_EULER));
        cur_cfl = CflCfg{};
        TARA_TRY(r);
      } else {
        // classical RK4; weights and stage offsets as in the oracle:
        // acc = u + (w dt/6) k1 ; us = u + (c dt) k ; u_new = acc + (dt/6) k4
        const double w[4] = {1.0, 2.0, 2.0, 1.0}, c[3] = {0.5, 0.5, 1.0};
        FieldPool<T>* ping[2] = {&us, &us2};
        for (int s = 0; s < 4; s++) {
          StepArgs<T> a = base_args(STEP_RK4);
          a.stage = s;
          a.wa = (T)(w[s] * p.dt / 6.0);
          a.cs = s < 3 ? (T)(c[s] * p.dt) : (T)0;
          Cx<T>* in[6];
          for (int f = 0; f < nf; f++) {
            in[f] = s == 0 ? u[f] : (*ping[(s - 1) & 1])[f];
            a.us[f] = (*ping[s & 1])[f];
          }
          cur_cfl = s == 0 ? cfl_cfg() : CflCfg{};
          const int r = rhs(in, a);
          cur_cfl = CflCfg{};
          TARA_TRY(r);
        }
      }
      std::swap(u, unew);
    }
    return TARA_OK;
  }
  void ew(int mode, int nfld, Cx<T>* const* u, Cx<T>* const* d1, Cx<T>* const* d2,
          Cx<T>* const* out, T alpha) {
    EwArgs<T> a{};
    a.mode = mode; a.nf = nfld; a.Nh = Nh; a.ld = g.ld; a.Ny = Ny;
    a.dt = (T)p.dt; a.alpha = alpha;
    for (int f = 0; f < nfld; f++) { a.u[f] = u[f]; a.d1[f] = d1[f]; a.d2[f] = d2[f]; a.out[f] = out[f]; }
    k_elementwise<T><<<592, 256, 0, st>>>(a);
  }
  int elementwise(int mode, int nfld, const double* const* u, const double* const* d1,
                  const double* const* d2, double* const* out) override {
    if (!u || !d1 || !d2 || !out) { set_error("null field array"); return TARA_EINVAL; }
    h_for = nullptr;
    Cx<T>* du[6];
    Cx<T>* dd1[6];
    Cx<T>* dd2[6];
    for (int f = 0; f < nfld; f++) {
      du[f] = acc[f]; dd1[f] = tmp[f]; dd2[f] = us[f];
      TARA_TRY(h2d(u[f], du[f]));
      TARA_TRY(h2d(d1[f], dd1[f]));
      if (mode == EW_AB2) TARA_TRY(h2d(d2[f], dd2[f]));
    }
    ew(mode, nfld, du, dd1, dd2, du, (T)(p.dt / 6.0));
    TARA_CUDA_TRY(cudaGetLastError());
    for (int f = 0; f < nfld; f++) TARA_TRY(d2h(du[f], out[f]));
    return TARA_OK;
  }
  int frozen_field_step(bool rk4, int w, const double* const* f, const double* d, double* out) override {
    if (model != TARA_MODEL_COH || w < 0 || w > 2) { set_error("bad field"); return TARA_EINVAL; }
    for (int q = 0; q < 3; q++) TARA_TRY(h2d(f[q], u[q]));
    TARA_TRY(h2d(d, dold[w]));  // k1
    const size_t fb = g.field_bytes();
    Cx<T>* in_s[6] = {us[0], us[1], us[2]};
    Cx<T>* uw[1] = {u[w]};
    Cx<T>* usw[1] = {us[w]};
    Cx<T>* accw[1] = {acc[w]};
    Cx<T>* kw[1] = {tmp[w]};
    Cx<T>* k1[1] = {dold[w]};
    for (int q = 0; q < 3; q++) TARA_CUDA_TRY(cudaMemcpyAsync(us[q], u[q], fb, cudaMemcpyDeviceToDevice, st));
    if (!rk4) {
      // predictor u + dt*k1, corrector with the refreshed derivative
      ew(EW_AXPY, 1, uw, k1, k1, usw, (T)p.dt);
      TARA_TRY(rhs(in_s, base_args(STEP_RHS)));
      ew(EW_PC, 1, uw, k1, kw, accw, (T)0);
    } else {
      const double c[3] = {0.5, 0.5, 1.0}, wgt[4] = {1.0, 2.0, 2.0, 1.0};
      ew(EW_AXPY, 1, uw, k1, k1, accw, (T)(wgt[0] * p.dt / 6.0));
      Cx<T>* kprev[1] = {dold[w]};
      for (int s = 0; s < 3; s++) {
        ew(EW_AXPY, 1, uw, kprev, kprev, usw, (T)(c[s] * p.dt));
        TARA_TRY(rhs(in_s, base_args(STEP_RHS)));
        ew(EW_AXPY, 1, accw, kw, kw, accw, (T)(wgt[s + 1] * p.dt / 6.0));
        kprev[0] = tmp[w];
      }
    }
    TARA_CUDA_TRY(cudaGetLastError());
    return d2h(acc[w], out);
  }
  int launches(int stepper) const override {
    int per = model == TARA_MODEL_COH ? kCohLaunches : model == TARA_MODEL_COM ? kComLaunches : kVortLaunches;
    return stepper == TARA_STEP_RK4 ? 4 * per : per;
  }

  // real-space buffers: nf + 3 fields of Nx*Ny values, and FP64 staging
  T* rbuf = nullptr;
  double* rstage = nullptr;
  int ensure_real() {
    if (rbuf) return TARA_OK;
    const size_t nn = (size_t)Nx * Ny;
    if (cudaMalloc(&rbuf, (nf + 3) * nn * sizeof(T)) != cudaSuccess ||
        cudaMalloc(&rstage, nn * sizeof(double)) != cudaSuccess) {
      set_error("cudaMalloc of real-space buffers failed");
      return TARA_ENOMEM;
    }
    return TARA_OK;
  }
  FieldPool<T>& workpool() { return model == TARA_MODEL_COH ? cw.H : model == TARA_MODEL_COM ? mw.H : vw.H; }
  int real_fields(int what, double* const* h) override {
    if (!h) { set_error("null field array"); return TARA_EINVAL; }
    TARA_TRY(ensure_real());
    h_for = nullptr;  // the transforms use the work pool
    const size_t nn = (size_t)Nx * Ny;
    T* r[9];
    for (int q = 0; q < nf + 3; q++) r[q] = rbuf + q * nn;
    Cx<T>* st_[6];
    Cx<T>* wk[8];
    for (int q = 0; q < nf; q++) st_[q] = u[q];
    // one work field per transformed field (pools hold >= nf, >= 4 fields)
    const int nw = workpool().count < 8 ? workpool().count : 8;
    for (int q = 0; q < 8; q++) wk[q] = q < nw ? workpool()[q] : nullptr;
    if (nw < nf || nw < 3) { set_error("work pool too small"); return TARA_EINVAL; }
    int nout = 0;
    if (what == 0) {
      TARA_TRY(state_to_real(g, nf, st_, r, wk, st));
      nout = nf;
    } else if (what == 1) {
      Cx<T>* w3[3] = {tmp[0], tmp[1], model == TARA_MODEL_COM ? tmp[2] : wk[2]};
      TARA_TRY(vorticity_real(g, model, st_, r[0], r + nf, w3, st));
      nout = 1;
    } else {
      set_error("unknown real-space field set");
      return TARA_EINVAL;
    }
    for (int q = 0; q < nout; q++) {
      if (!h[q]) { set_error("null host field pointer"); return TARA_EINVAL; }
      if constexpr (sizeof(T) == sizeof(double)) {
        TARA_CUDA_TRY(cudaMemcpyAsync(h[q], r[q], nn * sizeof(double), cudaMemcpyDeviceToHost, st));
      } else {
        copy_from_real(r[q], rstage, nn, st);
        TARA_CUDA_TRY(cudaMemcpyAsync(h[q], rstage, nn * sizeof(double), cudaMemcpyDeviceToHost, st));
      }
      TARA_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return device_status();
  }
  int set_state_real(const double* const* h) override {
    if (!h) { set_error("null field array"); return TARA_EINVAL; }
    TARA_TRY(ensure_real());
    h_for = nullptr;
    const size_t nn = (size_t)Nx * Ny;
    const T* r[6];
    Cx<T>* st_[6];
    Cx<T>* wk[6];
    for (int q = 0; q < nf; q++) {
      if (!h[q]) { set_error("null host field pointer"); return TARA_EINVAL; }
      T* d = rbuf + q * nn;
      if constexpr (sizeof(T) == sizeof(double)) {
        TARA_CUDA_TRY(cudaMemcpyAsync(d, h[q], nn * sizeof(double), cudaMemcpyHostToDevice, st));
      } else {
        TARA_CUDA_TRY(cudaMemcpyAsync(rstage, h[q], nn * sizeof(double), cudaMemcpyHostToDevice, st));
        copy_to_real(rstage, d, nn, st);
      }
      r[q] = d;
      st_[q] = u[q];
      wk[q] = workpool()[q];
    }
    TARA_TRY(real_to_state(g, nf, r, st_, wk, st));
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    return device_status();
  }

  int set_state_random(const tara_ic* ic) override {
    if (!ic) { set_error("null initial-condition description"); return TARA_EINVAL; }
    TARA_TRY(ensure_real());
    h_for = nullptr;
    const size_t nn = (size_t)Nx * Ny;
    T* r[9];
    for (int q = 0; q < nf + 3; q++) r[q] = rbuf + q * nn;
    if (workpool().count < nf || workpool().count < 4) { set_error("work pool too small"); return TARA_EINVAL; }
    Cx<T>* wk[6];
    for (int q = 0; q < 6; q++) wk[q] = q < workpool().count ? workpool()[q] : nullptr;
    TARA_TRY(ic_random_state<T>(g, model, p, *ic, r, wk, st));
    const T* rc[6];
    Cx<T>* st_[6];
    for (int q = 0; q < nf; q++) {
      rc[q] = r[q];
      st_[q] = u[q];
    }
    TARA_TRY(real_to_state(g, nf, rc, st_, wk, st));
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    return device_status();
  }

  int tracers_run(int stepper, int nsteps, int np, double* xp, double* yp, double* vxp, double* vyp) override {
    if (model != TARA_MODEL_CSH && model != TARA_MODEL_CSS) {
      set_error("tracer particles move with the velocity of the vorticity models");
      return TARA_EUNSUPPORTED;
    }
    if (np < 0 || nsteps < 0 || (np > 0 && (!xp || !yp))) { set_error("bad tracer arguments"); return TARA_EINVAL; }
    if (np == 0) return step(stepper, nsteps);
    TARA_TRY(ensure_real());
    if (workpool().count < 4) { set_error("work pool too small"); return TARA_EINVAL; }
    const size_t nn = (size_t)Nx * Ny;
    T* ux = rbuf + nn;  // real fields 1 and 2 of nf + 3 >= 4
    T* uy = rbuf + 2 * nn;
    Cx<T>* wk[4] = {workpool()[0], workpool()[1], workpool()[2], workpool()[3]};
    double* d = nullptr;
    if (cudaMalloc(&d, 4 * (size_t)np * sizeof(double)) != cudaSuccess) {
      set_error("cudaMalloc of the tracer arrays failed");
      return TARA_ENOMEM;
    }
    double *dx = d, *dy = d + np, *dvx = d + 2 * (size_t)np, *dvy = d + 3 * (size_t)np;
    const T lam = model == TARA_MODEL_CSS ? vortp.lambda : (T)0;
    int r = TARA_OK;
    if (cudaMemcpyAsync(dx, xp, np * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess ||
        cudaMemcpyAsync(dy, yp, np * sizeof(double), cudaMemcpyHostToDevice, st) != cudaSuccess) {
      set_error("tracer upload failed");
      r = TARA_ECUDA;
    }
    if (r == TARA_OK && nsteps == 0) {
      r = tracer_velocity_real<T>(g, u[0], lam, ux, uy, wk, st);
      if (r == TARA_OK) r = tracers_update<T>(g, ux, uy, np, dx, dy, dvx, dvy, p.dt, false, st);
    }
    for (int k = 0; k < nsteps && r == TARA_OK; k++) {
      r = step(stepper, 1);  // the new state is u
      if (r == TARA_OK) r = tracer_velocity_real<T>(g, u[0], lam, ux, uy, wk, st);
      if (r == TARA_OK) r = tracers_update<T>(g, ux, uy, np, dx, dy, dvx, dvy, p.dt, true, st);
    }
    if (r == TARA_OK) {
      const size_t b = np * sizeof(double);
      if (cudaMemcpyAsync(xp, dx, b, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          cudaMemcpyAsync(yp, dy, b, cudaMemcpyDeviceToHost, st) != cudaSuccess ||
          (vxp && cudaMemcpyAsync(vxp, dvx, b, cudaMemcpyDeviceToHost, st) != cudaSuccess) ||
          (vyp && cudaMemcpyAsync(vyp, dvy, b, cudaMemcpyDeviceToHost, st) != cudaSuccess)) {
        set_error("tracer download failed");
        r = TARA_ECUDA;
      }
    }
    cudaStreamSynchronize(st);
    cudaFree(d);
    return r == TARA_OK ? device_status() : r;
  }

  int time_transforms(int inverse, int nfields, int reps, float* ms) override {
    if (nfields < 1 || nfields > nf || nfields > 6 || reps < 1 || !ms) {
      set_error("bad transform timing request");
      return TARA_EINVAL;
    }
    TARA_TRY(ensure_real());
    h_for = nullptr;  // the transforms use the work pool
    if (workpool().count < nfields) { set_error("work pool too small"); return TARA_EINVAL; }
    const size_t nn = (size_t)Nx * Ny;
    T* r[6];
    const T* rc[6];
    const Cx<T>* uc[6];
    Cx<T>* sp[6];
    Cx<T>* wk[6];
    for (int q = 0; q < nfields; q++) {
      r[q] = rbuf + q * nn;
      rc[q] = r[q];
      uc[q] = u[q];
      sp[q] = tmp[q];
      wk[q] = workpool()[q];
    }
    // real fields to transform forward: the state's own c2r
    if (!inverse) TARA_TRY(c2r_fields<T>(g, nfields, uc, r, wk, true, st));
    TARA_CUDA_TRY(cudaStreamSynchronize(st));
    TARA_CUDA_TRY(cudaEventRecord(ev0, st));
    for (int k = 0; k < reps; k++) {
      if (inverse) TARA_TRY(c2r_fields<T>(g, nfields, uc, r, wk, true, st));
      else TARA_TRY(r2c_fields<T>(g, nfields, rc, sp, wk, st));
    }
    TARA_CUDA_TRY(cudaEventRecord(ev1, st));
    TARA_CUDA_TRY(cudaEventSynchronize(ev1));
    TARA_CUDA_TRY(cudaEventElapsedTime(ms, ev0, ev1));
    return device_status();
  }

  int num_shells() override { return diag_num_shells(Nx, Ny, p.Lx, p.Ly, p.pi); }
  int record(double* drec) {
    h_for = nullptr;  // the diagnostics use the work pool
    if (!dw.mem || dw.nbins != num_shells()) {
      dw.release();
      TARA_TRY(dw.alloc(g, st));
    }
    Cx<T>* state[6];
    for (int f = 0; f < nf; f++) state[f] = u[f];
    if (model == TARA_MODEL_COM) return diag_record(model, g, dw, state, mw.H, mw.X, tmp, drec, st);
    return diag_record(model, g, dw, state, cw.H, cw.X, tmp, drec, st);
  }
  int run_recorded(int stepper, int every, int nrec, double* rec) override {
    if (!rec || nrec < 1 || every < 0 || (nrec > 1 && every < 1)) { set_error("bad record request"); return TARA_EINVAL; }
    if (model != TARA_MODEL_COM && model != TARA_MODEL_COH) {
      set_error("diagnostics are defined for the hydro and MHD models");
      return TARA_EUNSUPPORTED;
    }
    const size_t per = (size_t)kDiagOut + (size_t)num_shells();
    double* d = nullptr;
    if (cudaMalloc(&d, per * nrec * sizeof(double)) != cudaSuccess) {
      set_error("cudaMalloc of the diagnostics records failed");
      return TARA_ENOMEM;
    }
    int r = TARA_OK;
    for (int k = 0; k < nrec && r == TARA_OK; k++) {
      if (k > 0) r = step(stepper, every);
      if (r == TARA_OK) r = record(d + per * k);
    }
    if (r == TARA_OK && cudaMemcpyAsync(rec, d, per * nrec * sizeof(double), cudaMemcpyDeviceToHost, st) != cudaSuccess)
      r = TARA_ECUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess && r == TARA_OK) r = TARA_ECUDA;
    if (r == TARA_ECUDA) set_error(std::string("diagnostics: ") + cudaGetErrorString(cudaGetLastError()));
    cudaFree(d);
    if (r != TARA_OK) return r;
    return device_status();
  }
};

tara_session* make_session(int precision) {
  if (precision == TARA_FP32) return new SessionT<float>();
  return new SessionT<double>();
}

thread_local int g_legacy_status = TARA_OK;
int g_legacy_mode = TARA_LEGACY_REFERENCE;
std::mutex g_legacy_mu;
std::map<std::tuple<int, int, int>, std::unique_ptr<tara_session>> g_legacy;

}  // namespace

namespace tara {
// status word of the drop-in entry points (tara_legacy_status)
void set_legacy_status(int s) { g_legacy_status = s; }
}  // namespace tara

// ======================================================================
// session API
// ======================================================================
extern "C" {

const char* tara_last_error(void) { return tara::last_error(); }

int tara_open(tara_session** out, int model, int Nx, int Ny, int precision, const tara_params* p) {
  if (!out || !p) { set_error("null argument"); return TARA_EINVAL; }
  *out = nullptr;
  int nf = nfields_of(model);
  if (!nf) { set_error("unknown model"); return TARA_EINVAL; }
  if (precision != TARA_FP64 && precision != TARA_FP32) { set_error("unknown precision"); return TARA_EINVAL; }
  if (!supported_length(Nx) || !supported_length(Ny)) {
    set_error("grid size not supported (Nx, Ny in {16,32,64,128,256,384,512,1024,2048,4096})");
    return TARA_EUNSUPPORTED;
  }
  std::unique_ptr<tara_session> s(make_session(precision));
  s->model = model; s->precision = precision; s->Nx = Nx; s->Ny = Ny; s->Nh = Nx / 2 + 1; s->nf = nf;
  s->p = *p;
  if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&s->ev0) != cudaSuccess || cudaEventCreate(&s->ev1) != cudaSuccess) {
    set_error(std::string("CUDA initialisation failed: ") + cudaGetErrorString(cudaGetLastError()));
    return TARA_ECUDA;
  }
  int r = s->init();
  if (r != TARA_OK) return r;
  *out = s.release();
  return TARA_OK;
}

int tara_close(tara_session* s) {
  if (!s) return TARA_EINVAL;
  delete s;
  return TARA_OK;
}

int tara_set_params(tara_session* s, const tara_params* p) {
  if (!s || !p) return TARA_EINVAL;
  s->p = *p;
  return s->fail_if(s->apply_params());
}

int tara_num_fields(const tara_session* s) { return s ? s->nf : 0; }

int tara_set_state(tara_session* s, const double* const* f) { return s ? s->fail_if(s->set_fields(0, f)) : TARA_EINVAL; }
int tara_get_state(tara_session* s, double* const* f) { return s ? s->fail_if(s->get_fields(0, f)) : TARA_EINVAL; }
int tara_set_history(tara_session* s, const double* const* f) { return s ? s->fail_if(s->set_fields(1, f)) : TARA_EINVAL; }
int tara_get_history(tara_session* s, double* const* f) { return s ? s->fail_if(s->get_fields(1, f)) : TARA_EINVAL; }
int tara_rhs(tara_session* s, double* const* out) { return s ? s->fail_if(s->rhs_to_host(out)) : TARA_EINVAL; }

int tara_step(tara_session* s, int stepper, int nsteps) {
  if (!s || nsteps < 0) return TARA_EINVAL;
  return s->fail_if(s->step(stepper, nsteps));
}
int tara_synchronize(tara_session* s) {
  if (!s) return TARA_EINVAL;
  cudaError_t e = cudaStreamSynchronize(s->st);
  if (e != cudaSuccess) {
    set_error(std::string("cudaStreamSynchronize: ") + cudaGetErrorString(e));
    return s->fail_if(TARA_ECUDA);
  }
  return s->fail_if(s->device_status());
}
int tara_time_steps(tara_session* s, int stepper, int nsteps, float* ms) {
  if (!s || !ms || nsteps < 0) return TARA_EINVAL;
  if (cudaStreamSynchronize(s->st) != cudaSuccess) return s->fail_if(TARA_ECUDA);
  cudaEventRecord(s->ev0, s->st);
  int r = s->step(stepper, nsteps);
  if (r != TARA_OK) return s->fail_if(r);
  cudaEventRecord(s->ev1, s->st);
  cudaError_t e = cudaEventSynchronize(s->ev1);
  if (e != cudaSuccess) {
    set_error(std::string("cudaEventSynchronize: ") + cudaGetErrorString(e));
    return s->fail_if(TARA_ECUDA);
  }
  cudaEventElapsedTime(ms, s->ev0, s->ev1);
  r = s->device_status();
  if (r != TARA_OK) return s->fail_if(r);
  return TARA_OK;
}
int tara_profile_steps(tara_session* s, int stepper, int nsteps, double* kernel_ms, int* kernel_launches,
                       float* total_ms) {
  if (!s || !kernel_ms || !kernel_launches || nsteps < 0) return TARA_EINVAL;
  for (int k = 0; k < TARA_NUM_KERNEL_KINDS; k++) { kernel_ms[k] = 0; kernel_launches[k] = 0; }
  if (cudaStreamSynchronize(s->st) != cudaSuccess) return s->fail_if(TARA_ECUDA);
  Prof& pr = s->prof;
  pr.cap = nsteps * (s->launches(stepper) * 2 + 8) + 8;
  pr.ev = new cudaEvent_t[pr.cap];
  pr.kind = new int[pr.cap];
  int made = 0, r = TARA_OK;
  for (; made < pr.cap; made++)
    if (cudaEventCreate(&pr.ev[made]) != cudaSuccess) { r = TARA_ECUDA; break; }
  if (r == TARA_OK) {
    pr.n = 0;
    pr.on = 1;
    cudaEventRecord(s->ev0, s->st);
    r = s->step(stepper, nsteps);
    cudaEventRecord(s->ev1, s->st);
    pr.on = 0;
    if (r == TARA_OK && cudaEventSynchronize(s->ev1) != cudaSuccess) r = TARA_ECUDA;
    if (r == TARA_OK) {
      if (total_ms) cudaEventElapsedTime(total_ms, s->ev0, s->ev1);
      for (int i = 0; i + 1 < pr.n; i++) {
        const int k = pr.kind[i];
        if (k == KK_END) continue;
        float ms = 0;
        cudaEventElapsedTime(&ms, pr.ev[i], pr.ev[i + 1]);
        kernel_ms[k] += ms;
        kernel_launches[k] += 1;
      }
    }
  }
  for (int i = 0; i < made; i++) cudaEventDestroy(pr.ev[i]);
  delete[] pr.ev;
  delete[] pr.kind;
  pr.ev = nullptr;
  pr.kind = nullptr;
  pr.cap = pr.n = 0;
  if (r != TARA_OK) set_error("profiling run failed");
  return s->fail_if(r);
}
const char* tara_kernel_name(int kind) { return kernel_kind_name(kind); }

int tara_host_register(void* p, size_t bytes) {
  cudaError_t e = cudaHostRegister(p, bytes, cudaHostRegisterDefault);
  if (e != cudaSuccess) {
    set_error(std::string("cudaHostRegister: ") + cudaGetErrorString(e));
    return TARA_ECUDA;
  }
  return TARA_OK;
}
int tara_host_unregister(void* p) {
  cudaError_t e = cudaHostUnregister(p);
  if (e != cudaSuccess) {
    set_error(std::string("cudaHostUnregister: ") + cudaGetErrorString(e));
    return TARA_ECUDA;
  }
  return TARA_OK;
}
int tara_set_device(int dev) {
  cudaError_t e = cudaSetDevice(dev);
  if (e != cudaSuccess) {
    set_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return TARA_ECUDA;
  }
  return TARA_OK;
}
int tara_device_pci_bus_id(char* out, int len) {
  int dev = 0;
  if (!out || len < 13) return TARA_EINVAL;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetPCIBusId(out, len, dev) != cudaSuccess) {
    set_error("cudaDeviceGetPCIBusId failed");
    return TARA_ECUDA;
  }
  return TARA_OK;
}

int tara_launches_per_step(const tara_session* s, int stepper) { return s ? s->launches(stepper) : 0; }
int tara_time_transforms(tara_session* s, int inverse, int nfields, int reps, float* ms) {
  return s ? s->fail_if(s->time_transforms(inverse, nfields, reps, ms)) : TARA_EINVAL;
}

int tara_get_state_real(tara_session* s, double* const* fields) {
  return s ? s->fail_if(s->real_fields(0, fields)) : TARA_EINVAL;
}
int tara_get_vorticity_real(tara_session* s, double* omega) {
  if (!s || !omega) return TARA_EINVAL;
  double* o[1] = {omega};
  return s->fail_if(s->real_fields(1, o));
}
int tara_set_state_real(tara_session* s, const double* const* fields) {
  return s ? s->fail_if(s->set_state_real(fields)) : TARA_EINVAL;
}
int tara_set_state_random(tara_session* s, const tara_ic* ic) {
  return s ? s->fail_if(s->set_state_random(ic)) : TARA_EINVAL;
}
int tara_tracers_run(tara_session* s, int stepper, int nsteps, int np, double* xp, double* yp, double* vxp,
                     double* vyp) {
  return s ? s->fail_if(s->tracers_run(stepper, nsteps, np, xp, yp, vxp, vyp)) : TARA_EINVAL;
}

// The drivers' grid files: one line per grid point, x outer, y inner, as
// list-directed records (src/main2com.f95:603-609: x, y, rho, ux, uy, P, E,
// Bx, By; src/main2coh.f95:414-418: x, y, omega, n, ux, uy).
int tara_write_snapshot(tara_session* s, const char* path) {
  if (!s || !path) return TARA_EINVAL;
  if (s->model != TARA_MODEL_COM && s->model != TARA_MODEL_COH) {
    set_error("grid files are written for the hydro and MHD models");
    return TARA_EUNSUPPORTED;
  }
  const size_t nn = (size_t)s->Nx * s->Ny;
  std::vector<double> f((size_t)(s->nf + 1) * nn);
  double* fp[7];
  for (int q = 0; q <= s->nf; q++) fp[q] = f.data() + q * nn;
  int r = s->real_fields(0, fp);
  if (r == TARA_OK && s->model == TARA_MODEL_COH) r = s->real_fields(1, fp + s->nf);
  if (r != TARA_OK) return s->fail_if(r);
  FILE* out = std::fopen(path, "w");
  if (!out) { set_error(std::string("cannot open ") + path); return TARA_EINVAL; }
  const double dx = s->p.Lx / (double)s->Nx, dy = s->p.Ly / (double)s->Ny, cs2 = s->p.CS * s->p.CS;
  std::string line;
  double v[9];
  for (int i = 0; i < s->Nx; i++)
    for (int j = 0; j < s->Ny; j++) {
      const size_t k = (size_t)j * s->Nx + i;
      v[0] = 0.0 + (double)i * dx;
      v[1] = 0.0 + (double)j * dy;
      int n;
      if (s->model == TARA_MODEL_COM) {
        const double rho = fp[0][k];
        v[2] = rho; v[3] = fp[1][k] / rho; v[4] = fp[2][k] / rho; v[5] = cs2 * rho;
        v[6] = fp[3][k]; v[7] = fp[4][k]; v[8] = fp[5][k];
        n = 9;
      } else {
        v[2] = fp[3][k]; v[3] = fp[0][k]; v[4] = fp[1][k]; v[5] = fp[2][k];
        n = 6;
      }
      line.clear();
      list_directed_append(line, v, n);
      line += '\n';
      std::fwrite(line.data(), 1, line.size(), out);
    }
  const bool ok = std::fclose(out) == 0;
  if (!ok) { set_error(std::string("write to ") + path + " failed"); return TARA_EINVAL; }
  return TARA_OK;
}

int tara_set_graphs(tara_session* s, int on) {
  if (!s) return TARA_EINVAL;
  s->set_graphs(on != 0);
  return TARA_OK;
}
int tara_set_cfl(tara_session* s, int mode, double cfl) { return s ? s->fail_if(s->set_cfl(mode, cfl)) : TARA_EINVAL; }
int tara_get_time(tara_session* s, double* t, double* dt_last) {
  return s ? s->fail_if(s->get_time(t, dt_last)) : TARA_EINVAL;
}
int tara_set_time(tara_session* s, double t) { return s ? s->fail_if(s->set_time(t)) : TARA_EINVAL; }
int tara_set_wait_limit(tara_session* s, long long limit_ns) {
  return s ? s->fail_if(s->set_wait_limit(limit_ns)) : TARA_EINVAL;
}
int tara_num_shells(tara_session* s) { return s ? s->num_shells() : 0; }
int tara_diagnostics(tara_session* s, double* out, int nout, double* Ek, int nbins) {
  if (!s || (!out && nout > 0) || (!Ek && nbins > 0) || nout < 0 || nbins < 0) return TARA_EINVAL;
  const int ns = s->num_shells();
  if (nout > TARA_DIAG_VALUES || nbins > ns) { set_error("more values requested than computed"); return TARA_EINVAL; }
  std::vector<double> rec((size_t)TARA_DIAG_VALUES + ns);
  int r = s->run_recorded(TARA_STEP_RK4, 0, 1, rec.data());
  if (r != TARA_OK) return s->fail_if(r);
  for (int k = 0; k < nout; k++) out[k] = rec[k];
  for (int k = 0; k < nbins; k++) Ek[k] = rec[TARA_DIAG_VALUES + k];
  return TARA_OK;
}
int tara_run_recorded(tara_session* s, int stepper, int every, int nrec, double* rec) {
  if (!s) return TARA_EINVAL;
  if (stepper != TARA_STEP_AB2 && stepper != TARA_STEP_EULER && stepper != TARA_STEP_RK4) {
    set_error("unknown stepper");
    return TARA_EINVAL;
  }
  return s->fail_if(s->run_recorded(stepper, every, nrec, rec));
}
int tara_status(const tara_session* s) { return s ? s->status : TARA_EINVAL; }

}  // extern "C"

// ======================================================================
// drop-in entry points
// ======================================================================
namespace {

// Cached FP64 session per (model, Nx, Ny) for the per-call entry points.
// Caller holds g_legacy_mu.
tara_session* legacy_session(int model, int Nx, int Ny, const tara_params& p, int& status) {
  auto key = std::make_tuple(model, Nx, Ny);
  auto it = g_legacy.find(key);
  if (it != g_legacy.end()) {
    tara_session* s = it->second.get();
    s->p = p;
    status = s->apply_params();
    return status == TARA_OK ? s : nullptr;
  }
  tara_session* s = nullptr;
  status = tara_open(&s, model, Nx, Ny, TARA_FP64, &p);
  if (status != TARA_OK) return nullptr;
  g_legacy[key].reset(s);
  return s;
}

tara_params coh_params_from_comm(double pi) {
  // COMMON /comm/ Lx,Ly,mux,muy,ms,CS,dt   (src/derive2coh.f95:30)
  tara_params p{};
  p.Lx = comm_[0]; p.Ly = comm_[1]; p.mux = comm_[2]; p.muy = comm_[3];
  p.ms = comm_[4]; p.CS = comm_[5]; p.dt = comm_[6]; p.pi = pi;
  return p;
}
tara_params com_params_from_comm(double pi) {
  // COMMON /comm/ Lx,Ly,spheat,mu,ms,CS,mu_0,eta,dt,kf,A   (src/derive2com.f95:48)
  tara_params p{};
  p.Lx = comm_[0]; p.Ly = comm_[1]; p.spheat = comm_[2]; p.mu = comm_[3]; p.ms = comm_[4];
  p.CS = comm_[5]; p.mu_0 = comm_[6]; p.eta = comm_[7]; p.dt = comm_[8]; p.kf = comm_[9];
  p.A = comm_[10]; p.pi = pi;
  return p;
}

bool check_dims(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh) {
  if (!Nx || !Ny || !Nh || *Nh != *Nx / 2 + 1) {
    set_error("inconsistent Nx/Ny/Nh");
    g_legacy_status = TARA_EINVAL;
    return false;
  }
  return true;
}

void legacy_derive(int model, int Nx, int Ny, const tara_params& p, const double* const* in,
                   double* const* out) {
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  int st = TARA_OK;
  tara_session* s = legacy_session(model, Nx, Ny, p, st);
  if (s) st = s->set_fields(0, in);
  if (st == TARA_OK) st = s->rhs_to_host(out);
  g_legacy_status = st;
}

void legacy_elementwise(int model, int Nx, int Ny, const tara_params& p, int mode, int nfld,
                        const double* const* u, const double* const* d1, const double* const* d2,
                        double* const* out) {
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  int st = TARA_OK;
  tara_session* s = legacy_session(model, Nx, Ny, p, st);
  if (s) st = s->elementwise(mode, nfld, u, d1, d2, out);
  g_legacy_status = st;
}

}  // namespace

extern "C" {

int tara_legacy_status(void) { return g_legacy_status; }
int tara_set_legacy_mode(int mode) {
  if (mode != TARA_LEGACY_REFERENCE && mode != TARA_LEGACY_CORRECT) return TARA_EINVAL;
  g_legacy_mode = mode;
  return TARA_OK;
}

int tara_derive2coh(const tara_params* p, int Nx, int Ny, const double* nk, const double* ukx,
                    const double* uky, double* dn_dt, double* dux_dt, double* duy_dt) {
  if (!p) return TARA_EINVAL;
  const double* in[3] = {nk, ukx, uky};
  double* out[3] = {dn_dt, dux_dt, duy_dt};
  legacy_derive(TARA_MODEL_COH, Nx, Ny, *p, in, out);
  return g_legacy_status;
}
int tara_derive2com(const tara_params* p, int Nx, int Ny, const double* const* state6,
                    double* const* rhs6) {
  if (!p || !state6 || !rhs6) return TARA_EINVAL;
  legacy_derive(TARA_MODEL_COM, Nx, Ny, *p, state6, rhs6);
  return g_legacy_status;
}

void derive2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                 const double* time, double* nk, double* ukx, double* uky, double* dn_dt_old,
                 double* dux_dt_old, double* duy_dt_old, double* dn_dt_new, double* dux_dt_new,
                 double* duy_dt_new) {
  (void)time; (void)dn_dt_old; (void)dux_dt_old; (void)duy_dt_old;
  if (!check_dims(Nx, Ny, Nh)) return;
  const double* in[3] = {nk, ukx, uky};
  double* out[3] = {dn_dt_new, dux_dt_new, duy_dt_new};
  legacy_derive(TARA_MODEL_COH, *Nx, *Ny, coh_params_from_comm(*pi), in, out);
}

void ab2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
             const double* time, double* nk, double* ukx, double* uky, double* nk_new,
             double* ukx_new, double* uky_new, double* dn_dt_old, double* dux_dt_old,
             double* duy_dt_old, double* dn_dt_new, double* dux_dt_new, double* duy_dt_new) {
  (void)time;
  if (!check_dims(Nx, Ny, Nh)) return;
  const double* u[3] = {nk, ukx, uky};
  const double* dn[3] = {dn_dt_new, dux_dt_new, duy_dt_new};
  const double* dol[3] = {dn_dt_old, dux_dt_old, duy_dt_old};
  double* out[3] = {nk_new, ukx_new, uky_new};
  legacy_elementwise(TARA_MODEL_COH, *Nx, *Ny, coh_params_from_comm(*pi), EW_AB2, 3, u, dn, dol, out);
}

void euler2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                const double* time, double* nk, double* ukx, double* uky, double* nk_new,
                double* ukx_new, double* uky_new, double* dn_dt, double* dux_dt, double* duy_dt) {
  (void)time;
  if (!check_dims(Nx, Ny, Nh)) return;
  const double* u[3] = {nk, ukx, uky};
  const double* d[3] = {dn_dt, dux_dt, duy_dt};
  double* out[3] = {nk_new, ukx_new, uky_new};
  legacy_elementwise(TARA_MODEL_COH, *Nx, *Ny, coh_params_from_comm(*pi), EW_EULER, 3, u, d, d, out);
}

}  // extern "C"

namespace {
// pc_*2coh / rk4_*2coh: advance field `which` (0 nk, 1 ukx, 2 uky).
void legacy_pc_rk4(bool rk4, int which, const int32_t* Nx, const int32_t* Ny, const int32_t* Nh,
                   const double* pi, double* nk, double* ukx, double* uky, double* out,
                   double* dn_dt, double* dux_dt, double* duy_dt) {
  if (!check_dims(Nx, Ny, Nh)) return;
  const double* f[3] = {nk, ukx, uky};
  const double* d[3] = {dn_dt, dux_dt, duy_dt};
  tara_params p = coh_params_from_comm(*pi);
  if (g_legacy_mode == TARA_LEGACY_REFERENCE) {
    const double* u1[1] = {f[which]};
    const double* d1[1] = {d[which]};
    double* o1[1] = {out};
    legacy_elementwise(TARA_MODEL_COH, *Nx, *Ny, p, rk4 ? EW_RK4_REF : EW_PC_REF, 1, u1, d1, d1, o1);
    return;
  }
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  int st = TARA_OK;
  tara_session* s = legacy_session(TARA_MODEL_COH, *Nx, *Ny, p, st);
  if (s) st = s->frozen_field_step(rk4, which, f, d[which], out);
  g_legacy_status = st;
}
}  // namespace

extern "C" {
void pc_nk2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                const double* time, double* nk, double* nk_new, double* ukx, double* uky,
                double* dn_dt, double* dux_dt, double* duy_dt) {
  (void)time;
  legacy_pc_rk4(false, 0, Nx, Ny, Nh, pi, nk, ukx, uky, nk_new, dn_dt, dux_dt, duy_dt);
}
void pc_ukx2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                 const double* time, double* nk, double* ukx, double* ukx_new, double* uky,
                 double* dn_dt, double* dux_dt, double* duy_dt) {
  (void)time;
  legacy_pc_rk4(false, 1, Nx, Ny, Nh, pi, nk, ukx, uky, ukx_new, dn_dt, dux_dt, duy_dt);
}
void pc_uky2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                 const double* time, double* nk, double* ukx, double* uky, double* uky_new,
                 double* dn_dt, double* dux_dt, double* duy_dt) {
  (void)time;
  legacy_pc_rk4(false, 2, Nx, Ny, Nh, pi, nk, ukx, uky, uky_new, dn_dt, dux_dt, duy_dt);
}
void rk4_nk2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                 const double* time, double* nk, double* nk_new, double* ukx, double* uky,
                 double* dn_dt, double* dux_dt, double* duy_dt) {
  (void)time;
  legacy_pc_rk4(true, 0, Nx, Ny, Nh, pi, nk, ukx, uky, nk_new, dn_dt, dux_dt, duy_dt);
}
void rk4_ukx2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                  const double* time, double* nk, double* ukx, double* ukx_new, double* uky,
                  double* dn_dt, double* dux_dt, double* duy_dt) {
  (void)time;
  legacy_pc_rk4(true, 1, Nx, Ny, Nh, pi, nk, ukx, uky, ukx_new, dn_dt, dux_dt, duy_dt);
}
void rk4_uky2coh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                  const double* time, double* nk, double* ukx, double* uky, double* uky_new,
                  double* dn_dt, double* dux_dt, double* duy_dt) {
  (void)time;
  legacy_pc_rk4(true, 2, Nx, Ny, Nh, pi, nk, ukx, uky, uky_new, dn_dt, dux_dt, duy_dt);
}

void derive2com_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
                 const double* time, double* rho_k, double* rho_ux_k, double* rho_uy_k,
                 double* E_k, double* Bx_k, double* By_k, double* d_rho_k_dt_old,
                 double* d_rho_k_dt_new, double* d_rho_ux_k_dt_old, double* d_rho_ux_k_dt_new,
                 double* d_rho_uy_k_dt_old, double* d_rho_uy_k_dt_new, double* d_E_k_dt_old,
                 double* d_E_k_dt_new, double* d_Bx_k_dt_old, double* d_Bx_k_dt_new,
                 double* d_By_k_dt_old, double* d_By_k_dt_new) {
  (void)time; (void)d_rho_k_dt_old; (void)d_rho_ux_k_dt_old; (void)d_rho_uy_k_dt_old;
  (void)d_E_k_dt_old; (void)d_Bx_k_dt_old; (void)d_By_k_dt_old;
  if (!check_dims(Nx, Ny, Nh)) return;
  const double* in[6] = {rho_k, rho_ux_k, rho_uy_k, E_k, Bx_k, By_k};
  double* out[6] = {d_rho_k_dt_new, d_rho_ux_k_dt_new, d_rho_uy_k_dt_new, d_E_k_dt_new,
                    d_Bx_k_dt_new, d_By_k_dt_new};
  legacy_derive(TARA_MODEL_COM, *Nx, *Ny, com_params_from_comm(*pi), in, out);
}

void ab2com_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* pi,
             const double* time, double* rho_k, double* rho_ux_k, double* rho_uy_k, double* E_k,
             double* Bx_k, double* By_k, double* rho_k_new, double* rho_ux_k_new,
             double* rho_uy_k_new, double* E_k_new, double* Bx_k_new, double* By_k_new,
             double* d_rho_k_dt_old, double* d_rho_k_dt_new, double* d_rho_ux_k_dt_old,
             double* d_rho_ux_k_dt_new, double* d_rho_uy_k_dt_old, double* d_rho_uy_k_dt_new,
             double* d_E_k_dt_old, double* d_E_k_dt_new, double* d_Bx_k_dt_old,
             double* d_Bx_k_dt_new, double* d_By_k_dt_old, double* d_By_k_dt_new) {
  (void)time;
  if (!check_dims(Nx, Ny, Nh)) return;
  const double* u[6] = {rho_k, rho_ux_k, rho_uy_k, E_k, Bx_k, By_k};
  const double* dn[6] = {d_rho_k_dt_new, d_rho_ux_k_dt_new, d_rho_uy_k_dt_new, d_E_k_dt_new,
                         d_Bx_k_dt_new, d_By_k_dt_new};
  const double* dol[6] = {d_rho_k_dt_old, d_rho_ux_k_dt_old, d_rho_uy_k_dt_old, d_E_k_dt_old,
                          d_Bx_k_dt_old, d_By_k_dt_old};
  double* out[6] = {rho_k_new, rho_ux_k_new, rho_uy_k_new, E_k_new, Bx_k_new, By_k_new};
  legacy_elementwise(TARA_MODEL_COM, *Nx, *Ny, com_params_from_comm(*pi), EW_AB2, 6, u, dn, dol, out);
}

}  // extern "C"

// ---------------------------------------------------------------- vorticity
namespace {
// Box of derive2css, whose Lx, Ly and lambda are never set in the reference
// (src/derive2css.f95:12, 24, 32); the driver's values (src/main2css.f95:78-87)
// are the defaults.
double g_css_Lx = 2.0 * 3.14159265358979323846, g_css_Ly = 2.0 * 3.14159265358979323846, g_css_lambda = 10.0;

// real(kind=8), parameter :: pi = 3.1428   (a default-real literal;
// src/derive2csh.f95:16, src/derive2css.f95:15)
const double kVortPi = (double)3.1428f;

tara_params csh_params(double nu, double dt) {
  tara_params p{};
  p.pi = kVortPi;
  p.Lx = 2.0 * kVortPi;  // src/derive2csh.f95:20-21
  p.Ly = 2.0 * kVortPi;
  p.nu = nu;
  p.dt = dt;
  return p;
}
tara_params css_params(double alpha, double nu, double dt) {
  tara_params p{};
  p.pi = kVortPi;
  p.Lx = g_css_Lx;
  p.Ly = g_css_Ly;
  p.lambda = g_css_lambda;
  p.alpha = alpha;
  p.nu = nu;
  p.dt = dt;
  return p;
}
}  // namespace

extern "C" {

int tara_set_css_box(double Lx, double Ly, double lambda) {
  if (!(Lx > 0) || !(Ly > 0)) { set_error("box lengths must be positive"); return TARA_EINVAL; }
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  g_css_Lx = Lx;
  g_css_Ly = Ly;
  g_css_lambda = lambda;
  return TARA_OK;
}

void derive2csh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* nu, const double* time,
                 double* omegak, double* omegak_new, double* dt_omegak_old, double* dt_omegak_new) {
  (void)time; (void)omegak_new; (void)dt_omegak_old;
  if (!check_dims(Nx, Ny, Nh)) return;
  const double* in[1] = {omegak};
  double* out[1] = {dt_omegak_new};
  legacy_derive(TARA_MODEL_CSH, *Nx, *Ny, csh_params(*nu, 0.0), in, out);
}
void ab2csh_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* nu, const double* time,
             const double* dt, double* omegak, double* omegak_new, double* dt_omegak_old, double* dt_omegak_new) {
  (void)time;
  if (!check_dims(Nx, Ny, Nh)) return;
  const double* u[1] = {omegak};
  const double* dn[1] = {dt_omegak_new};
  const double* dol[1] = {dt_omegak_old};
  double* out[1] = {omegak_new};
  legacy_elementwise(TARA_MODEL_CSH, *Nx, *Ny, csh_params(*nu, *dt), EW_AB2, 1, u, dn, dol, out);
}
void derive2css_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* alpha, const double* nu,
                 const double* time, double* omegak, double* omegak_new, double* dt_omegak_old,
                 double* dt_omegak_new) {
  (void)time; (void)omegak_new; (void)dt_omegak_old;
  if (!check_dims(Nx, Ny, Nh)) return;
  const double* in[1] = {omegak};
  double* out[1] = {dt_omegak_new};
  legacy_derive(TARA_MODEL_CSS, *Nx, *Ny, css_params(*alpha, *nu, 0.0), in, out);
}
void ab2css_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* alpha, const double* nu,
             const double* time, const double* dt, double* omegak, double* omegak_new, double* dt_omegak_old,
             double* dt_omegak_new) {
  (void)time;
  if (!check_dims(Nx, Ny, Nh)) return;
  const double* u[1] = {omegak};
  const double* dn[1] = {dt_omegak_new};
  const double* dol[1] = {dt_omegak_old};
  double* out[1] = {omegak_new};
  legacy_elementwise(TARA_MODEL_CSS, *Nx, *Ny, css_params(*alpha, *nu, *dt), EW_AB2, 1, u, dn, dol, out);
}
// src/rk42css.f95:6-52 reads its stage derivatives from an uninitialised
// local; this entry point takes one classical RK4 step of derive2css instead
// and writes omegak_new only.
void rk42css_(const int32_t* Nx, const int32_t* Ny, const int32_t* Nh, const double* alpha, const double* nu,
              const double* time, const double* dt, double* omegak, double* omegak_new, double* dt_omegak_old,
              double* dt_omegak_new) {
  (void)time; (void)dt_omegak_old; (void)dt_omegak_new;
  if (!check_dims(Nx, Ny, Nh)) return;
  std::lock_guard<std::mutex> lk(g_legacy_mu);
  int st = TARA_OK;
  tara_session* s = legacy_session(TARA_MODEL_CSS, *Nx, *Ny, css_params(*alpha, *nu, *dt), st);
  const double* in[1] = {omegak};
  double* out[1] = {omegak_new};
  if (s) st = s->set_fields(0, in);
  if (st == TARA_OK) st = s->step(TARA_STEP_RK4, 1);
  if (st == TARA_OK) st = s->get_fields(0, out);
  g_legacy_status = st;
}

}  // extern "C"
