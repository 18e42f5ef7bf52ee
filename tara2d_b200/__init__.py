"""tara2d_b200 -- B200 (sm_100a) pseudo-spectral RHS + time-step path of TARA2D.

The compute path is the CUDA shared library ``_lib/libtara2d_b200.so`` (C ABI
in ``include/tara2d_gpu.h``).  This module is a thin ctypes binding with the
same array convention as the reference's Fortran: a ``complex(8) (Nh,Ny)``
array is a C-contiguous numpy ``complex128`` array of shape ``(Ny, Nh)``.

There is no CPU fallback: if the library is missing or no CUDA device is
usable, calls raise.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import initial  # noqa: F401  (seeded initial conditions)

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libtara2d_b200.so")

OK, EINVAL, ECUDA, ENAN, ETIMEOUT, ENOMEM, EUNSUPPORTED, ECFL = 0, -1, -2, -3, -4, -5, -6, -7
CFL_OFF, CFL_CHECK, CFL_ADAPT = 0, 1, 2
MODEL_COH, MODEL_COM, MODEL_CSH, MODEL_CSS = 1, 2, 3, 4
FP64, FP32 = 0, 1
STEP_AB2, STEP_RK4, STEP_EULER = 0, 1, 2
CLOSURE_EVERY_RHS, CLOSURE_ONCE_PER_STEP = 0, 1
LEGACY_REFERENCE, LEGACY_CORRECT = 0, 1
SUPPORTED_N = (16, 32, 64, 128, 256, 384, 512, 1024, 2048, 4096)
NUM_KERNEL_KINDS = 12
DIAG_VALUES = 8
NFIELDS = {MODEL_COH: 3, MODEL_COM: 6, MODEL_CSH: 1, MODEL_CSS: 1}
PI = 3.14159265358979323846
# pi of the vorticity subroutines: real(kind=8), parameter :: pi = 3.1428, a
# default-real literal (src/derive2csh.f95:16, src/derive2css.f95:15)
VORT_PI = float(np.float32(3.1428))


class TaraError(RuntimeError):
    def __init__(self, msg: str, status: int = 0):
        super().__init__(msg)
        self.status = status


class IcDesc(C.Structure):
    """tara_ic (include/tara2d_gpu.h): a seeded initial condition built on the device."""
    _fields_ = [("kind", C.c_int), ("reserved0", C.c_int), ("seed", C.c_ulonglong), ("k0", C.c_double),
                ("e1", C.c_double), ("e2", C.c_double), ("kmin", C.c_double), ("kmax", C.c_double),
                ("reserved", C.c_double * 3)]


IC_RANDOM_PHASE, IC_ORSZAG_TANG = 1, 2


class Params(C.Structure):
    """tara_params (include/tara2d_gpu.h)."""
    _fields_ = [(n, C.c_double) for n in
                ("Lx", "Ly", "pi", "dt", "mux", "muy", "ms", "CS", "spheat", "mu", "mu_0", "eta",
                 "kf", "A", "nu", "alpha", "lambda_")] + \
               [("fix_curlB", C.c_int), ("reserved", C.c_int * 7)]

    @classmethod
    def make(cls, **kw) -> "Params":
        p = cls()
        p.Lx = p.Ly = 2.0 * PI
        p.pi = PI
        for k, v in kw.items():
            setattr(p, "lambda_" if k == "lambda" else k, v)
        return p


_lib = None


def lib():
    """The loaded CUDA library (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise TaraError(f"CUDA library not built: {LIB_PATH} (run python -m tara2d_b200.build)")
        L = C.CDLL(LIB_PATH)
        P, I, D = C.c_void_p, C.c_int, C.c_double
        PP = C.POINTER(C.c_void_p)
        L.tara_last_error.restype = C.c_char_p
        L.tara_open.argtypes = [C.POINTER(C.c_void_p), I, I, I, I, C.POINTER(Params)]
        L.tara_close.argtypes = [P]
        L.tara_set_params.argtypes = [P, C.POINTER(Params)]
        L.tara_num_fields.argtypes = [P]
        for n in ("tara_set_state", "tara_get_state", "tara_set_history", "tara_get_history", "tara_rhs"):
            getattr(L, n).argtypes = [P, PP]
        L.tara_step.argtypes = [P, I, I]
        L.tara_synchronize.argtypes = [P]
        L.tara_time_steps.argtypes = [P, I, I, C.POINTER(C.c_float)]
        L.tara_launches_per_step.argtypes = [P, I]
        L.tara_status.argtypes = [P]
        L.tara_derive2coh.argtypes = [C.POINTER(Params), I, I, P, P, P, P, P, P]
        L.tara_derive2com.argtypes = [C.POINTER(Params), I, I, PP, PP]
        L.tara_set_legacy_mode.argtypes = [I]
        L.tara_profile_steps.argtypes = [P, I, I, C.POINTER(C.c_double), C.POINTER(C.c_int), C.POINTER(C.c_float)]
        L.tara_kernel_name.restype = C.c_char_p
        L.tara_kernel_name.argtypes = [I]
        L.tara_host_register.argtypes = [P, C.c_size_t]
        L.tara_host_unregister.argtypes = [P]
        L.tara_device_pci_bus_id.argtypes = [C.c_char_p, I]
        L.tara_set_device.argtypes = [I]
        L.tara_set_graphs.argtypes = [P, I]
        L.tara_closure_open.argtypes = [C.POINTER(C.c_void_p), I, I, I, C.c_ulonglong]
        L.tara_closure_close.argtypes = [P]
        L.tara_closure_count.argtypes = [P]
        L.tara_closure_add_pair.argtypes = [P, P]
        L.tara_closure_get_pair.argtypes = [P, I, P, P]
        L.tara_closure_get_norm.argtypes = [P, P]
        L.tara_closure_set_norm.argtypes = [P, P]
        L.tara_closure_fit_norm.argtypes = [P, I, I]
        L.tara_closure_train.argtypes = [P, I, I, I, I, C.c_float, P]
        L.tara_closure_eval_loss.argtypes = [P, I, I, C.POINTER(C.c_float)]
        L.tara_closure_get_params.argtypes = [P, P]
        L.tara_closure_set_params.argtypes = [P, P]
        L.tara_closure_forward.argtypes = [P, P, I, P]
        L.tara_closure_backward.argtypes = [P, P, P, I, P]
        L.tara_closure_set_tensor_cores.argtypes = [P, I]
        L.tara_closure_add_pair_member.argtypes = [P, P, I]
        L.tara_closure_status.argtypes = [P]
        L.tara_closure_time_cnn.argtypes = [P, I, I, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.tara_session_attach_closure.argtypes = [P, P]
        L.tara_session_set_closure_mode.argtypes = [P, C.c_int]
        L.tara_filter_state.argtypes = [P, P]
        L.tara_get_state_real.argtypes = [P, PP]
        L.tara_set_state_real.argtypes = [P, PP]
        L.tara_get_vorticity_real.argtypes = [P, P]
        L.tara_write_snapshot.argtypes = [P, C.c_char_p]
        L.tara_checkpoint_write.argtypes = [P, C.c_char_p, C.c_longlong, D]
        L.tara_set_state_random.argtypes = [P, C.POINTER(IcDesc)]
        L.tara_tracers_run.argtypes = [P, I, I, I, P, P, P, P]
        L.tara_checkpoint_read.argtypes = [P, C.c_char_p, C.POINTER(C.c_longlong), C.POINTER(C.c_double)]
        L.tara_format_list_directed.argtypes = [P, I, C.c_char_p, I]
        L.tara_ens_open.argtypes = [C.POINTER(C.c_void_p), I, I, P, C.POINTER(Params), I]
        L.tara_ens_open_mixed.argtypes = [C.POINTER(C.c_void_p), I, P, P, C.POINTER(Params), I]
        L.tara_ens_num_fields.argtypes = [P, I]
        L.tara_ens_close.argtypes = [P]
        for n in ("tara_ens_set_state", "tara_ens_get_state", "tara_ens_get_history"):
            getattr(L, n).argtypes = [P, I, PP]
        L.tara_ens_step.argtypes = [P, I, I]
        L.tara_ens_time_steps.argtypes = [P, I, I, C.POINTER(C.c_float)]
        L.tara_ens_set_tuning.argtypes = [P, P]
        L.tara_ens_get_tuning.argtypes = [P, P]
        L.tara_ens_autotune.argtypes = [P, I, I, P, P]
        L.tara_ens_num_shells.argtypes = [P, I]
        L.tara_ens_diagnostics.argtypes = [P, I, P, I, P, I]
        L.tara_ens_size.argtypes = [P]
        L.tara3d_open.argtypes = [C.POINTER(C.c_void_p), I, I, I, C.POINTER(Params3D)]
        L.tara3d_close.argtypes = [P]
        L.tara3d_set_params.argtypes = [P, C.POINTER(Params3D)]
        for n in ("tara3d_set_state", "tara3d_get_state", "tara3d_set_history", "tara3d_rhs"):
            getattr(L, n).argtypes = [P, PP]
        L.tara3d_step.argtypes = [P, I]
        L.tara3d_time_steps.argtypes = [P, I, C.POINTER(C.c_float)]
        L.tara3d_launches_per_step.argtypes = [P]
        L.tara_num_shells.argtypes = [P]
        L.tara_diagnostics.argtypes = [P, P, I, P, I]
        L.tara_run_recorded.argtypes = [P, I, I, I, P]
        L.tara_set_css_box.argtypes = [D, D, D]
        L.tara_set_cfl.argtypes = [P, I, D]
        L.tara_get_time.argtypes = [P, C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.tara_set_time.argtypes = [P, D]
        L.tara_set_wait_limit.argtypes = [P, C.c_longlong]
        L.tara_time_transforms.argtypes = [P, I, I, I, C.POINTER(C.c_float)]
        L.tara_selftest_bounded_wait.argtypes = [C.c_longlong, C.POINTER(C.c_longlong)]
        _lib = L
    return _lib


def last_error() -> str:
    return lib().tara_last_error().decode()


def check(status: int, what: str = "") -> None:
    if status != OK:
        raise TaraError(f"{what} failed with status {status}: {last_error()}", status)


def selftest_bounded_wait(limit_ns: int):
    """tara_selftest_bounded_wait: (status, ns waited) of a kernel whose
    bounded mbarrier wait must run out (status ETIMEOUT)."""
    waited = C.c_longlong()
    st = lib().tara_selftest_bounded_wait(int(limit_ns), C.byref(waited))
    return st, waited.value


def _ptrs(arrs):
    return (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])


class Params3D(C.Structure):
    """tara3d_params: pi, box lengths (already times pi), and mu, CS, eta, dt of
    the 3D driver's COMMON /comm/ (src/main3com.f95:56)."""
    _fields_ = [(n, C.c_double) for n in ("pi", "Lx", "Ly", "Lz", "mu", "CS", "eta", "dt")] + \
               [("reserved", C.c_double * 8)]

    @classmethod
    def make(cls, **kw):
        p = cls()
        for k, v in kw.items():
            setattr(p, k, v)
        return p


class Mhd3:
    """3D compressible MHD (src/derive3com.f95, src/ab3com.f95) with the state in
    HBM.  Fields: rho, rho ux, rho uy, rho uz, E, Bx, By, Bz, each a complex
    (Nz, Ny, Nx/2+1) array (the reference's Fortran (Nh,Ny,Nz) layout)."""

    NF = 8

    def __init__(self, Nx: int, Ny: int, Nz: int, params: Params3D):
        self.Nx, self.Ny, self.Nz = Nx, Ny, Nz
        self.Nh = Nx // 2 + 1
        self.params = params
        h = C.c_void_p()
        check(lib().tara3d_open(C.byref(h), Nx, Ny, Nz, C.byref(params)), "tara3d_open")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().tara3d_close(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _shape(self):
        return (self.Nz, self.Ny, self.Nh)

    def _in(self, fields):
        if len(fields) != self.NF:
            raise ValueError("8 fields expected")
        arrs = [np.ascontiguousarray(f, dtype=np.complex128) for f in fields]
        for a in arrs:
            if a.shape != self._shape():
                raise ValueError(f"field shape {a.shape}, expected {self._shape()}")
        return arrs, (C.c_void_p * self.NF)(*[a.ctypes.data for a in arrs])

    def _out(self):
        arrs = [np.empty(self._shape(), dtype=np.complex128) for _ in range(self.NF)]
        return arrs, (C.c_void_p * self.NF)(*[a.ctypes.data for a in arrs])

    def set_params(self, params: Params3D) -> None:
        check(lib().tara3d_set_params(self._h, C.byref(params)), "tara3d_set_params")
        self.params = params

    def set_state(self, fields) -> None:
        arrs, ptrs = self._in(fields)
        check(lib().tara3d_set_state(self._h, ptrs), "tara3d_set_state")

    def set_history(self, fields) -> None:
        arrs, ptrs = self._in(fields)
        check(lib().tara3d_set_history(self._h, ptrs), "tara3d_set_history")

    def get_state(self):
        arrs, ptrs = self._out()
        check(lib().tara3d_get_state(self._h, ptrs), "tara3d_get_state")
        return arrs

    def rhs(self):
        """derive3com of the current state (d/dt of the 8 fields)."""
        arrs, ptrs = self._out()
        check(lib().tara3d_rhs(self._h, ptrs), "tara3d_rhs")
        return arrs

    def step(self, nsteps: int = 1) -> None:
        """nsteps of derive3com + ab3com + history shift (src/main3com.f95:548-600)."""
        check(lib().tara3d_step(self._h, nsteps), "tara3d_step")

    def time_steps(self, nsteps: int) -> float:
        ms = C.c_float()
        check(lib().tara3d_time_steps(self._h, nsteps, C.byref(ms)), "tara3d_time_steps")
        return ms.value

    def launches_per_step(self) -> int:
        return lib().tara3d_launches_per_step(self._h)


class Session:
    """A grid whose spectral state stays in HBM (tara_open ... tara_close)."""

    def __init__(self, model: int, Nx: int, Ny: int, params: Params, precision: int = FP64):
        self.model, self.Nx, self.Ny, self.precision = model, Nx, Ny, precision
        self.Nh = Nx // 2 + 1
        self.nf = NFIELDS[model]
        self.params = params
        h = C.c_void_p()
        check(lib().tara_open(C.byref(h), model, Nx, Ny, precision, C.byref(params)), "tara_open")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().tara_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _fields_in(self, fields):
        arrs = [np.ascontiguousarray(f, dtype=np.complex128) for f in fields]
        assert len(arrs) == self.nf and all(a.shape == (self.Ny, self.Nh) for a in arrs)
        return arrs

    def _fields_out(self):
        return [np.zeros((self.Ny, self.Nh), dtype=np.complex128) for _ in range(self.nf)]

    def set_params(self, params: Params) -> None:
        self.params = params
        check(lib().tara_set_params(self._h, C.byref(params)), "tara_set_params")

    def set_state(self, fields) -> None:
        a = self._fields_in(fields)
        check(lib().tara_set_state(self._h, _ptrs(a)), "tara_set_state")

    def set_cfl(self, mode: int, cfl: float = 0.0) -> None:
        """CFL control (CFL_OFF, CFL_CHECK, CFL_ADAPT) with CFL number cfl."""
        check(lib().tara_set_cfl(self._h, mode, cfl), "tara_set_cfl")

    def set_closure_mode(self, mode: int) -> None:
        """Where an attached closure is evaluated in RK4 steps:
        CLOSURE_EVERY_RHS (default) or CLOSURE_ONCE_PER_STEP (stages 2-4
        reuse the first stage's subgrid spectra)."""
        check(lib().tara_session_set_closure_mode(self._h, mode), "tara_session_set_closure_mode")

    def time(self):
        """(model time advanced so far, dt of the last step)."""
        t, dt = C.c_double(), C.c_double()
        check(lib().tara_get_time(self._h, C.byref(t), C.byref(dt)), "tara_get_time")
        return t.value, dt.value

    def set_time(self, t: float) -> None:
        check(lib().tara_set_time(self._h, t), "tara_set_time")

    def time_transforms(self, inverse: int, nfields: int, reps: int) -> float:
        """Device ms of reps plain 2D c2r (inverse = 1) or r2c of nfields fields."""
        ms = C.c_float()
        check(lib().tara_time_transforms(self._h, inverse, nfields, reps, C.byref(ms)), "tara_time_transforms")
        return ms.value

    def set_wait_limit(self, ns: int) -> None:
        check(lib().tara_set_wait_limit(self._h, int(ns)), "tara_set_wait_limit")

    def get_state(self):
        out = self._fields_out()
        check(lib().tara_get_state(self._h, _ptrs(out)), "tara_get_state")
        return out

    def get_state_into(self, out) -> None:
        """Copy the state into caller-owned (e.g. pinned) (Ny, Nh) complex128 arrays."""
        assert len(out) == self.nf and all(a.flags.c_contiguous and a.dtype == np.complex128 for a in out)
        check(lib().tara_get_state(self._h, _ptrs(out)), "tara_get_state")

    def set_history(self, fields) -> None:
        a = self._fields_in(fields)
        check(lib().tara_set_history(self._h, _ptrs(a)), "tara_set_history")

    def get_history(self):
        out = self._fields_out()
        check(lib().tara_get_history(self._h, _ptrs(out)), "tara_get_history")
        return out

    def rhs(self):
        out = self._fields_out()
        check(lib().tara_rhs(self._h, _ptrs(out)), "tara_rhs")
        return out

    def step(self, stepper: int, nsteps: int) -> None:
        check(lib().tara_step(self._h, stepper, nsteps), "tara_step")

    def synchronize(self) -> None:
        check(lib().tara_synchronize(self._h), "tara_synchronize")

    def time_steps(self, stepper: int, nsteps: int) -> float:
        ms = C.c_float()
        check(lib().tara_time_steps(self._h, stepper, nsteps, C.byref(ms)), "tara_time_steps")
        return ms.value

    def launches_per_step(self, stepper: int) -> int:
        return lib().tara_launches_per_step(self._h, stepper)

    def _real_out(self, n):
        return [np.zeros((self.Ny, self.Nx), dtype=np.float64) for _ in range(n)]

    def get_state_real(self):
        """Every state field in real space (c2r / (Nx Ny)), arrays of shape (Ny, Nx)."""
        out = self._real_out(self.nf)
        check(lib().tara_get_state_real(self._h, _ptrs(out)), "tara_get_state_real")
        return out

    def get_vorticity_real(self):
        out = self._real_out(1)[0]
        check(lib().tara_get_vorticity_real(self._h, out.ctypes.data), "tara_get_vorticity_real")
        return out

    def set_state_real(self, fields) -> None:
        """State from real-space fields (shape (Ny, Nx)) by the device r2c."""
        a = [np.ascontiguousarray(f, dtype=np.float64) for f in fields]
        assert len(a) == self.nf and all(x.shape == (self.Ny, self.Nx) for x in a)
        check(lib().tara_set_state_real(self._h, _ptrs(a)), "tara_set_state_real")

    def write_snapshot(self, path: str) -> None:
        """The drivers' grid file (fort.NNNNNNNN) of the current state."""
        check(lib().tara_write_snapshot(self._h, os.fsencode(path)), "tara_write_snapshot")

    def set_state_random(self, kind: int, seed: int, k0: float = 4.0, e1: float = 0.5, e2: float = 0.01,
                         kmin: float = 0.0, kmax: float = 0.0) -> None:
        """State from a seeded initial condition built on the device
        (IC_RANDOM_PHASE: hydro u energy e1 and density noise e2, or MHD
        kinetic / magnetic energies e1, e2; IC_ORSZAG_TANG (MHD): perturbation
        rms e1 (u), e2 (B) on kmin <= |k| <= kmax).  The host restatement
        initial.hashed_state builds the same state."""
        d = IcDesc(kind=kind, seed=seed, k0=k0, e1=e1, e2=e2, kmin=kmin, kmax=kmax)
        check(lib().tara_set_state_random(self._h, C.byref(d)), "tara_set_state_random")

    def tracers_run(self, stepper: int, nsteps: int, xp, yp):
        """Tracer particles (vorticity models): nsteps state steps, each followed
        by one Euler move of the particles with the new velocity; xp, yp are
        float64 arrays updated in place.  Returns the last velocities (vx, vy)."""
        for a in (xp, yp):
            if not (isinstance(a, np.ndarray) and a.dtype == np.float64 and a.flags.c_contiguous):
                raise TaraError("tracer positions must be contiguous float64 arrays")
        n = int(xp.size)
        if yp.size != n:
            raise TaraError("xp and yp differ in length")
        vx, vy = np.zeros(n), np.zeros(n)
        check(lib().tara_tracers_run(self._h, stepper, nsteps, n, xp.ctypes.data, yp.ctypes.data, vx.ctypes.data,
                                     vy.ctypes.data), "tara_tracers_run")
        return vx, vy

    def checkpoint(self, path: str, step: int = 0, time: float = 0.0) -> None:
        """Binary checkpoint of state, history, parameters, step and time
        (format: tara2d_b200.checkpoint)."""
        check(lib().tara_checkpoint_write(self._h, os.fsencode(path), int(step), float(time)),
              "tara_checkpoint_write")

    def restore(self, path: str):
        """Restore parameters, state and history from a checkpoint of the same
        model and grid; returns its (step, time)."""
        step, time = C.c_longlong(), C.c_double()
        check(lib().tara_checkpoint_read(self._h, os.fsencode(path), C.byref(step), C.byref(time)),
              "tara_checkpoint_read")
        from .checkpoint import read_header
        h = read_header(path)
        for k, v in h["params"].items():
            setattr(self.params, "lambda_" if k == "lambda" else k, v)
        self.params.fix_curlB = h["fix_curlB"]
        return step.value, time.value

    def set_graphs(self, on: bool) -> None:
        """Replay steps from CUDA graphs (default) or launch every kernel from the host."""
        check(lib().tara_set_graphs(self._h, 1 if on else 0), "tara_set_graphs")

    def num_shells(self) -> int:
        return lib().tara_num_shells(self._h)

    def diagnostics(self):
        """(values[DIAG_VALUES], E(k)[num_shells]) of the current state, computed on the device."""
        out = np.zeros(DIAG_VALUES)
        ek = np.zeros(self.num_shells())
        check(lib().tara_diagnostics(self._h, out.ctypes.data, DIAG_VALUES, ek.ctypes.data, ek.size),
              "tara_diagnostics")
        return out, ek

    def run_recorded(self, stepper: int, every: int, nrec: int):
        """Records of the state before the first step and after every `every`
        steps: (values[nrec, DIAG_VALUES], E(k)[nrec, num_shells])."""
        ns = self.num_shells()
        rec = np.zeros((nrec, DIAG_VALUES + ns))
        check(lib().tara_run_recorded(self._h, stepper, every, nrec, rec.ctypes.data), "tara_run_recorded")
        return rec[:, :DIAG_VALUES], rec[:, DIAG_VALUES:]

    def profile_steps(self, stepper: int, nsteps: int):
        """Per-kernel device time: {name: (total_ms, launches)} and the total ms."""
        n = NUM_KERNEL_KINDS
        ms = (C.c_double * n)()
        cnt = (C.c_int * n)()
        tot = C.c_float()
        check(lib().tara_profile_steps(self._h, stepper, nsteps, ms, cnt, C.byref(tot)), "tara_profile_steps")
        out = {}
        for k in range(n):
            if cnt[k]:
                out[lib().tara_kernel_name(k).decode()] = (ms[k], cnt[k])
        return out, tot.value

    @property
    def status(self) -> int:
        return lib().tara_status(self._h)


# ---- drop-in Fortran entry points (reference calling convention) ----------
_COH = ("Lx", "Ly", "mux", "muy", "ms", "CS", "dt")
_COM = ("Lx", "Ly", "spheat", "mu", "ms", "CS", "mu_0", "eta", "dt", "kf", "A")


def set_comm(values) -> None:
    """Write the COMMON /comm/ block the drop-in entry points read."""
    comm = (C.c_double * 16).in_dll(lib(), "comm_")
    for i, v in enumerate(values):
        comm[i] = float(v)


def comm_coh(p: Params):
    return [getattr(p, n) for n in _COH]


def comm_com(p: Params):
    return [getattr(p, n) for n in _COM]


def _i32(v):
    return C.byref(C.c_int32(v))


def _d(v):
    return C.byref(C.c_double(v))


class Closure:
    """Learned subgrid closure (tara_closure_*): the CNN, its normalisation and
    a device-resident dataset of (filtered fields, subgrid stress/EMF) pairs
    on an Nc x Nc grid."""

    def __init__(self, Nc: int, capacity: int, batch_max: int = 16, seed: int = 0):
        self.Nc, self.capacity, self.batch_max = Nc, capacity, batch_max
        h = C.c_void_p()
        check(lib().tara_closure_open(C.byref(h), Nc, capacity, batch_max, seed), "tara_closure_open")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().tara_closure_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def set_tensor_cores(self, on: bool) -> None:
        """32 -> 32 convolutions on the tensor cores (default) or all on CUDA cores."""
        check(lib().tara_closure_set_tensor_cores(self._h, int(bool(on))), "tara_closure_set_tensor_cores")

    def time_cnn(self, B: int = 1, reps: int = 20):
        """Device ms per network call on B samples: (forward, forward + backward)."""
        f, b = C.c_float(), C.c_float()
        check(lib().tara_closure_time_cnn(self._h, B, reps, C.byref(f), C.byref(b)), "tara_closure_time_cnn")
        return f.value, b.value

    @staticmethod
    def num_params() -> int:
        return lib().tara_closure_num_params()

    @property
    def count(self) -> int:
        return lib().tara_closure_count(self._h)

    def add_pair(self, fine: "Session") -> None:
        check(lib().tara_closure_add_pair(self._h, fine._h), "tara_closure_add_pair")

    def add_pair_member(self, ens: "Ensemble", member: int) -> None:
        """A training pair from the current state of an FP64 MHD ensemble member."""
        check(lib().tara_closure_add_pair_member(self._h, ens._h, member), "tara_closure_add_pair_member")

    def get_pair(self, idx: int):
        n = self.Nc
        a = np.zeros((5, n, n), np.float32)
        b = np.zeros((4, n, n), np.float32)
        check(lib().tara_closure_get_pair(self._h, idx, a.ctypes.data, b.ctypes.data), "tara_closure_get_pair")
        return a, b

    def get_norm(self):
        v = np.zeros(18, np.float32)
        check(lib().tara_closure_get_norm(self._h, v.ctypes.data), "tara_closure_get_norm")
        return v

    def set_norm(self, v) -> None:
        v = np.ascontiguousarray(v, dtype=np.float32)
        assert v.size == 18
        check(lib().tara_closure_set_norm(self._h, v.ctypes.data), "tara_closure_set_norm")

    def fit_norm(self, first: int = 0, count: int = None) -> None:
        count = self.count - first if count is None else count
        check(lib().tara_closure_fit_norm(self._h, first, count), "tara_closure_fit_norm")

    def train(self, first: int, count: int, epochs: int, batch: int = 8, lr: float = 1e-3):
        losses = np.zeros(max(epochs, 1), np.float32)
        check(lib().tara_closure_train(self._h, first, count, epochs, batch, C.c_float(lr), losses.ctypes.data),
              "tara_closure_train")
        return losses[:epochs]

    def eval_loss(self, first: int, count: int) -> float:
        v = C.c_float()
        check(lib().tara_closure_eval_loss(self._h, first, count, C.byref(v)), "tara_closure_eval_loss")
        return v.value

    def get_params(self):
        w = np.zeros(self.num_params(), np.float32)
        check(lib().tara_closure_get_params(self._h, w.ctypes.data), "tara_closure_get_params")
        return w

    def set_params(self, w) -> None:
        w = np.ascontiguousarray(w, dtype=np.float32)
        assert w.size == self.num_params()
        check(lib().tara_closure_set_params(self._h, w.ctypes.data), "tara_closure_set_params")

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32)
        out = np.zeros((x.shape[0], 4, self.Nc, self.Nc), np.float32)
        check(lib().tara_closure_forward(self._h, x.ctypes.data, x.shape[0], out.ctypes.data), "tara_closure_forward")
        return out

    def backward(self, x, dout):
        x = np.ascontiguousarray(x, dtype=np.float32)
        dout = np.ascontiguousarray(dout, dtype=np.float32)
        g = np.zeros(self.num_params(), np.float32)
        check(lib().tara_closure_backward(self._h, x.ctypes.data, dout.ctypes.data, x.shape[0], g.ctypes.data),
              "tara_closure_backward")
        return g


def attach_closure(session: "Session", closure) -> None:
    """Add the closure's subgrid terms to the MHD RHS of `session` (None detaches)."""
    check(lib().tara_session_attach_closure(session._h, closure._h if closure is not None else None),
          "tara_session_attach_closure")


def filter_state(fine: "Session", coarse: "Session") -> None:
    """coarse state = sharp spectral filter of the fine state."""
    check(lib().tara_filter_state(fine._h, coarse._h), "tara_filter_state")


def format_list_directed(values) -> str:
    """One Fortran list-directed record of REAL(8) values, as gfortran writes it."""
    v = np.ascontiguousarray(values, dtype=np.float64).ravel()
    buf = C.create_string_buffer(32 * v.size + 8)
    n = lib().tara_format_list_directed(v.ctypes.data, v.size, buf, len(buf))
    if n < 0:
        raise TaraError(f"tara_format_list_directed failed: {last_error()}")
    return buf.value.decode()


class Ensemble:
    """Independent hydro and/or MHD runs of mixed grid sizes advanced together
    (tara_ens_open / tara_ens_open_mixed ... tara_ens_close).  sizes[m] in
    {128, 256, 384, 512}; params[m] is a Params (or one Params for every
    member); model is MODEL_COH or MODEL_COM for every member, or a list with
    one model per member."""

    def __init__(self, sizes, params, precision: int = FP32, model=MODEL_COH):
        self.sizes = [int(n) for n in sizes]
        n = len(self.sizes)
        if isinstance(params, Params):
            params = [params] * n
        self.params = list(params)
        arr = (Params * n)(*self.params)
        ns = (C.c_int * n)(*self.sizes)
        h = C.c_void_p()
        if isinstance(model, (list, tuple)):
            self.models = [int(x) for x in model]
            assert len(self.models) == n
            ms = (C.c_int * n)(*self.models)
            check(lib().tara_ens_open_mixed(C.byref(h), n, ms, ns, arr, precision), "tara_ens_open_mixed")
        else:
            self.models = [int(model)] * n
            check(lib().tara_ens_open(C.byref(h), int(model), n, ns, arr, precision), "tara_ens_open")
        self._h = h

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().tara_ens_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __len__(self):
        return len(self.sizes)

    def _out(self, m):
        if not 0 <= m < len(self.sizes):
            raise TaraError(f"no ensemble member {m}")
        N = self.sizes[m]
        nf = lib().tara_ens_num_fields(self._h, m)
        return [np.zeros((N, N // 2 + 1), dtype=np.complex128) for _ in range(nf)]

    def set_state(self, m: int, fields) -> None:
        N = self.sizes[m]
        a = [np.ascontiguousarray(f, dtype=np.complex128) for f in fields]
        nf = lib().tara_ens_num_fields(self._h, m)
        if len(a) != nf or not all(x.shape == (N, N // 2 + 1) for x in a):
            raise TaraError(f"member {m} takes {nf} fields of shape {(N, N // 2 + 1)}")
        check(lib().tara_ens_set_state(self._h, m, _ptrs(a)), "tara_ens_set_state")

    def get_state(self, m: int):
        out = self._out(m)
        check(lib().tara_ens_get_state(self._h, m, _ptrs(out)), "tara_ens_get_state")
        return out

    def get_history(self, m: int):
        out = self._out(m)
        check(lib().tara_ens_get_history(self._h, m, _ptrs(out)), "tara_ens_get_history")
        return out

    def step(self, stepper: int, nsteps: int) -> None:
        check(lib().tara_ens_step(self._h, stepper, nsteps), "tara_ens_step")

    def time_steps(self, stepper: int, nsteps: int) -> float:
        ms = C.c_float()
        check(lib().tara_ens_time_steps(self._h, stepper, nsteps, C.byref(ms)), "tara_ens_time_steps")
        return ms.value

    def set_tuning(self, tuning) -> None:
        t = (C.c_int * 6)(*tuning)
        check(lib().tara_ens_set_tuning(self._h, t), "tara_ens_set_tuning")

    def get_tuning(self):
        t = (C.c_int * 6)()
        check(lib().tara_ens_get_tuning(self._h, t), "tara_ens_get_tuning")
        return list(t)

    def autotune(self, stepper: int = STEP_AB2, reps: int = 3):
        """Pick the fastest tuning per phase; returns (tuning, ms per step of each phase)."""
        t = (C.c_int * 6)()
        ms = (C.c_float * 3)()
        check(lib().tara_ens_autotune(self._h, stepper, reps, t, ms), "tara_ens_autotune")
        return list(t), list(ms)

    def diagnostics(self, m: int):
        ns = lib().tara_ens_num_shells(self._h, m)
        out = np.zeros(DIAG_VALUES)
        ek = np.zeros(ns)
        check(lib().tara_ens_diagnostics(self._h, m, out.ctypes.data, DIAG_VALUES, ek.ctypes.data, ns),
              "tara_ens_diagnostics")
        return out, ek


def legacy_call(name: str, Nx: int, Ny: int, pi: float, time: float, arrays) -> int:
    """Call a drop-in entry point (e.g. 'derive2coh_') with Fortran-style
    arguments: Nx, Ny, Nh, pi, time by reference, then the arrays in the
    reference's order.  Returns tara_legacy_status()."""
    fn = getattr(lib(), name)
    args = [_i32(Nx), _i32(Ny), _i32(Nx // 2 + 1), _d(pi), _d(time)]
    for a in arrays:
        assert a.dtype == np.complex128 and a.flags.c_contiguous
        args.append(C.c_void_p(a.ctypes.data))
    fn(*args)
    return lib().tara_legacy_status()


def set_legacy_mode(mode: int) -> None:
    check(lib().tara_set_legacy_mode(mode), "tara_set_legacy_mode")


def pin(a: np.ndarray) -> None:
    """Page-lock a numpy array's memory (fast DMA for set_state/get_state)."""
    check(lib().tara_host_register(C.c_void_p(a.ctypes.data), a.nbytes), "tara_host_register")


def unpin(a: np.ndarray) -> None:
    check(lib().tara_host_unregister(C.c_void_p(a.ctypes.data)), "tara_host_unregister")


def set_device(dev: int) -> None:
    check(lib().tara_set_device(int(dev)), "tara_set_device")


def device_pci_bus_id() -> str:
    buf = C.create_string_buffer(64)
    check(lib().tara_device_pci_bus_id(buf, 64), "tara_device_pci_bus_id")
    return buf.value.decode()
