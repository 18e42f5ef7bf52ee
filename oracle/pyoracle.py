"""ctypes binding of the CPU oracle (oracle/_build/liboracle.so).

TEST INFRASTRUCTURE ONLY: the oracle is the checker for the CUDA path, never
part of it.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg import this module.

Array convention: a Fortran ``complex(8) (Nh,Ny)`` array is a C-contiguous
numpy ``complex128`` array of shape ``(Ny, Nh)`` (index ``[j, i]``); a Fortran
``real(8) (Nx,Ny)`` array is ``float64`` of shape ``(Ny, Nx)``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_build", "liboracle.so")

_lib = None


class CohParams(C.Structure):
    """COMMON /comm/ of the hydro units (src/main2coh.f95:29)."""
    _fields_ = [(n, C.c_double) for n in ("Lx", "Ly", "mux", "muy", "ms", "CS", "dt")]


class ComParams(C.Structure):
    """COMMON /comm/ of the MHD units (src/main2com.f95:43) + defect switch."""
    _fields_ = [(n, C.c_double) for n in
                ("Lx", "Ly", "spheat", "mu", "ms", "CS", "mu_0", "eta", "dt", "kf", "A")] + \
               [("fix_curlB", C.c_int)]


class Com3Params(C.Structure):
    """3D MHD: Lx, Ly, Lz (already times pi) and mu, CS, eta, dt of COMMON /comm/
    (src/main3com.f95:56)."""
    _fields_ = [(n, C.c_double) for n in ("Lx", "Ly", "Lz", "mu", "CS", "eta", "dt")]


def build() -> None:
    """Build the oracle (and, with the reference checkout present, its FFTW)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        _lib = C.CDLL(LIB_PATH)
        P = C.c_void_p
        i, d = C.c_int, C.c_double
        L = _lib
        L.ora_derive2coh.argtypes = [i, i, i, d, d, C.POINTER(CohParams), P, P, P, P, P, P]
        L.ora_ab2coh.argtypes = [i, i, i, C.POINTER(CohParams)] + [P] * 12
        L.ora_euler2coh.argtypes = [i, i, i, C.POINTER(CohParams)] + [P] * 9
        L.ora_pc2coh.argtypes = [i, i, i, i, d, d, C.POINTER(CohParams)] + [P] * 7
        L.ora_rk42coh.argtypes = [i, i, i, i, d, d, C.POINTER(CohParams)] + [P] * 7
        L.ora_rk4coh.argtypes = [i, i, i, d, d, C.POINTER(CohParams), P, P, P]
        L.ora_derive2com.argtypes = [i, i, i, d, d, C.POINTER(ComParams)] + [P] * 12
        L.ora_ab2com.argtypes = [i, i, i, C.POINTER(ComParams), P, P, P, P]
        L.ora_rk4com.argtypes = [i, i, i, d, d, C.POINTER(ComParams), P]
        L.ora_derive2csh.argtypes = [i, i, i, d, d, P, P]
        L.ora_ab2csh.argtypes = [i, i, i, d, P, P, P, P]
        L.ora_derive2css.argtypes = [i, i, i, d, d, d, d, d, d, P, P]
        L.ora_ab2css.argtypes = [i, i, i, d, P, P, P, P]
        L.ora_r2c_2d.argtypes = [i, i, P, P]
        L.ora_c2r_2d.argtypes = [i, i, P, P]
        L.ora_run_coh.argtypes = [i, i, d, C.POINTER(CohParams), i, i, P, P, P, P, P, P]
        L.ora_run_com.argtypes = [i, i, d, C.POINTER(ComParams), i, i, P, P]
        L.ora_diag_com.argtypes = [i, i, d, C.POINTER(ComParams), P, P]
        L.ora_diag_coh.argtypes = [i, i, d, C.POINTER(CohParams), P, P, P, P]
        L.ora_num_shells.argtypes = [i, i, d, d, d]
        L.ora_num_shells.restype = i
        L.ora_spectrum_coh.argtypes = [i, i, d, C.POINTER(CohParams), P, P, i, P]
        L.ora_spectrum_com.argtypes = [i, i, d, C.POINTER(ComParams), P, i, P]
        L.ora_derive3com.argtypes = [i, i, i, d, C.POINTER(Com3Params), P, P]
        L.ora_ab3com.argtypes = [i, i, i, d, P, P, P, P]
        L.ora_run3com.argtypes = [i, i, i, d, C.POINTER(Com3Params), i, P, P]
        L.ora_set_threads.argtypes = [i]
        L.ora_get_threads.restype = i
    return _lib


PI = 3.14159265358979323846


def _p(a: np.ndarray):
    assert a.flags.c_contiguous
    return a.ctypes.data_as(C.c_void_p)


def _cz(shape):
    return np.zeros(shape, dtype=np.complex128)


def _ptr_array(arrs):
    arr = (C.c_void_p * len(arrs))(*[a.ctypes.data for a in arrs])
    return arr


def set_threads(n: int) -> None:
    lib().ora_set_threads(int(n))


def r2c_2d(a: np.ndarray) -> np.ndarray:
    Ny, Nx = a.shape
    a = np.ascontiguousarray(a, dtype=np.float64)
    out = _cz((Ny, Nx // 2 + 1))
    lib().ora_r2c_2d(Nx, Ny, _p(a), _p(out))
    return out


def c2r_2d(X: np.ndarray, Nx: int) -> np.ndarray:
    Ny = X.shape[0]
    X = np.ascontiguousarray(X, dtype=np.complex128)
    out = np.zeros((Ny, Nx), dtype=np.float64)
    lib().ora_c2r_2d(Nx, Ny, _p(X), _p(out))
    return out


def derive2coh(Nx, Ny, P: CohParams, nk, ukx, uky, pi=PI, time=0.0):
    Nh = Nx // 2 + 1
    ins = [np.ascontiguousarray(a, dtype=np.complex128) for a in (nk, ukx, uky)]
    outs = [_cz((Ny, Nh)) for _ in range(3)]
    lib().ora_derive2coh(Nx, Ny, Nh, pi, time, C.byref(P), *[_p(a) for a in ins], *[_p(a) for a in outs])
    return outs


def ab2coh(Nx, Ny, P: CohParams, state, d_old, d_new):
    Nh = Nx // 2 + 1
    st = [np.ascontiguousarray(a, dtype=np.complex128) for a in state]
    do = [np.ascontiguousarray(a, dtype=np.complex128) for a in d_old]
    dn = [np.ascontiguousarray(a, dtype=np.complex128) for a in d_new]
    out = [_cz((Ny, Nh)) for _ in range(3)]
    lib().ora_ab2coh(Nx, Ny, Nh, C.byref(P), *[_p(a) for a in st], *[_p(a) for a in out],
                     *[_p(a) for a in do], *[_p(a) for a in dn])
    return out


def euler2coh(Nx, Ny, P: CohParams, state, d):
    Nh = Nx // 2 + 1
    st = [np.ascontiguousarray(a, dtype=np.complex128) for a in state]
    dd = [np.ascontiguousarray(a, dtype=np.complex128) for a in d]
    out = [_cz((Ny, Nh)) for _ in range(3)]
    lib().ora_euler2coh(Nx, Ny, Nh, C.byref(P), *[_p(a) for a in st], *[_p(a) for a in out],
                        *[_p(a) for a in dd])
    return out


def pc2coh(which, Nx, Ny, P, state, d, pi=PI, time=0.0):
    Nh = Nx // 2 + 1
    st = [np.ascontiguousarray(a, dtype=np.complex128) for a in state]
    dd = [np.ascontiguousarray(a, dtype=np.complex128) for a in d]
    out = _cz((Ny, Nh))
    lib().ora_pc2coh(which, Nx, Ny, Nh, pi, time, C.byref(P), *[_p(a) for a in st], _p(out),
                     *[_p(a) for a in dd])
    return out


def rk42coh(which, Nx, Ny, P, state, d, pi=PI, time=0.0):
    Nh = Nx // 2 + 1
    st = [np.ascontiguousarray(a, dtype=np.complex128) for a in state]
    dd = [np.ascontiguousarray(a, dtype=np.complex128) for a in d]
    out = _cz((Ny, Nh))
    lib().ora_rk42coh(which, Nx, Ny, Nh, pi, time, C.byref(P), *[_p(a) for a in st], _p(out),
                      *[_p(a) for a in dd])
    return out


def rk4coh(Nx, Ny, P, state, pi=PI, time=0.0):
    Nh = Nx // 2 + 1
    st = [np.array(a, dtype=np.complex128, order="C") for a in state]
    lib().ora_rk4coh(Nx, Ny, Nh, pi, time, C.byref(P), *[_p(a) for a in st])
    return st


def derive2com(Nx, Ny, P: ComParams, state, pi=PI, time=0.0):
    Nh = Nx // 2 + 1
    st = [np.ascontiguousarray(a, dtype=np.complex128) for a in state]
    outs = [_cz((Ny, Nh)) for _ in range(6)]
    lib().ora_derive2com(Nx, Ny, Nh, pi, time, C.byref(P), *[_p(a) for a in st], *[_p(a) for a in outs])
    return outs


def ab2com(Nx, Ny, P: ComParams, state, d_old, d_new):
    Nh = Nx // 2 + 1
    st = [np.ascontiguousarray(a, dtype=np.complex128) for a in state]
    do = [np.ascontiguousarray(a, dtype=np.complex128) for a in d_old]
    dn = [np.ascontiguousarray(a, dtype=np.complex128) for a in d_new]
    out = [_cz((Ny, Nh)) for _ in range(6)]
    lib().ora_ab2com(Nx, Ny, Nh, C.byref(P), _ptr_array(st), _ptr_array(out), _ptr_array(do), _ptr_array(dn))
    return out


def rk4com(Nx, Ny, P: ComParams, state, pi=PI, time=0.0):
    Nh = Nx // 2 + 1
    st = [np.array(a, dtype=np.complex128, order="C") for a in state]
    lib().ora_rk4com(Nx, Ny, Nh, pi, time, C.byref(P), _ptr_array(st))
    return st


def derive2csh(Nx, Ny, nu, omegak, time=0.0):
    Nh = Nx // 2 + 1
    w = np.ascontiguousarray(omegak, dtype=np.complex128)
    out = _cz((Ny, Nh))
    lib().ora_derive2csh(Nx, Ny, Nh, nu, time, _p(w), _p(out))
    return out


def derive2css(Nx, Ny, alpha, nu, Lx, Ly, lam, omegak, time=0.0):
    Nh = Nx // 2 + 1
    w = np.ascontiguousarray(omegak, dtype=np.complex128)
    out = _cz((Ny, Nh))
    lib().ora_derive2css(Nx, Ny, Nh, alpha, nu, time, Lx, Ly, lam, _p(w), _p(out))
    return out


def ab2csh(Nx, Ny, dt, w, d_old, d_new):
    Nh = Nx // 2 + 1
    a = [np.ascontiguousarray(x, dtype=np.complex128) for x in (w, d_old, d_new)]
    out = _cz((Ny, Nh))
    lib().ora_ab2csh(Nx, Ny, Nh, dt, _p(a[0]), _p(out), _p(a[1]), _p(a[2]))
    return out


def run_coh(Nx, Ny, P: CohParams, stepper, nsteps, state, d_old=None, pi=PI):
    Nh = Nx // 2 + 1
    st = [np.array(a, dtype=np.complex128, order="C") for a in state]
    do = [np.array(a, dtype=np.complex128, order="C") for a in d_old] if d_old is not None else \
        [_cz((Ny, Nh)) for _ in range(3)]
    lib().ora_run_coh(Nx, Ny, pi, C.byref(P), stepper, nsteps, *[_p(a) for a in st], *[_p(a) for a in do])
    return st, do


def run_com(Nx, Ny, P: ComParams, stepper, nsteps, state, d_old=None, pi=PI):
    Nh = Nx // 2 + 1
    st = [np.array(a, dtype=np.complex128, order="C") for a in state]
    do = [np.array(a, dtype=np.complex128, order="C") for a in d_old] if d_old is not None else \
        [_cz((Ny, Nh)) for _ in range(6)]
    lib().ora_run_com(Nx, Ny, pi, C.byref(P), stepper, nsteps, _ptr_array(st), _ptr_array(do))
    return st, do


def diag_com(Nx, Ny, P: ComParams, state, pi=PI):
    st = [np.ascontiguousarray(a, dtype=np.complex128) for a in state]
    out = np.zeros(6)
    lib().ora_diag_com(Nx, Ny, pi, C.byref(P), _ptr_array(st), _p(out))
    return out


def diag_coh(Nx, Ny, P: CohParams, state, pi=PI):
    st = [np.ascontiguousarray(a, dtype=np.complex128) for a in state]
    out = np.zeros(6)
    lib().ora_diag_coh(Nx, Ny, pi, C.byref(P), *[_p(a) for a in st], _p(out))
    return out


def num_shells(Nx, Ny, Lx=2 * PI, Ly=2 * PI, pi=PI):
    return lib().ora_num_shells(Nx, Ny, pi, Lx, Ly)


def spectrum_coh(Nx, Ny, P: CohParams, ukx, uky, pi=PI):
    n = num_shells(Nx, Ny, P.Lx, P.Ly, pi)
    a = [np.ascontiguousarray(x, dtype=np.complex128) for x in (ukx, uky)]
    out = np.zeros(n)
    lib().ora_spectrum_coh(Nx, Ny, pi, C.byref(P), _p(a[0]), _p(a[1]), n, _p(out))
    return out


def spectrum_com(Nx, Ny, P: ComParams, state, pi=PI):
    n = num_shells(Nx, Ny, P.Lx, P.Ly, pi)
    st = [np.ascontiguousarray(a, dtype=np.complex128) for a in state]
    out = np.zeros(n)
    lib().ora_spectrum_com(Nx, Ny, pi, C.byref(P), _ptr_array(st), n, _p(out))
    return out


# ---------------------------------------------------------------- tracers
def vort_velocity_real(omegak: np.ndarray, Nx: int, Ny: int, Lx: float, Ly: float, pi: float, lam: float = 0.0):
    """Real (ux, uy) of a vorticity spectrum as src/main2csh.f95:122-173 forms
    them: psi = omega/(kx^2 + ky^2 [+ lambda]) (0 at k = 0), ukx = i ky psi,
    uky = -i kx psi, c2r (the reference's FFTW) / (Nx Ny)."""
    Nh = Nx // 2 + 1
    kx = 2.0 * pi * np.arange(Nh, dtype=np.float64) / Lx
    j = np.arange(Ny, dtype=np.float64)
    ky = np.where(np.arange(Ny) < Ny // 2, 2.0 * pi * j / Ly, 2.0 * pi * (j - Ny) / Ly)
    KX, KY = np.meshgrid(kx, ky)
    den = KX * KX + KY * KY + lam
    den[0, 0] = 1.0
    psi = omegak / den
    psi[0, 0] = 0.0
    ux = c2r_2d(1j * KY * psi, Nx) / (Nx * Ny)
    uy = c2r_2d(-1j * KX * psi, Nx) / (Nx * Ny)
    return ux, uy


def _tracer_cell(p, d, L, N):
    m = np.trunc(p / d).astype(np.int64) + 1          # aint(p/d) + 1
    m = np.clip(m, 1, N + 1)
    p0 = (m - 1).astype(np.float64) * d              # x(m)
    p1 = np.where(m == N, L, m.astype(np.float64) * d)   # x(m+1), Lx in the last column
    return (m - 1) % N, m % N, p0, p1


def tracer_velocity(ux, uy, xp, yp, Lx, Ly):
    """Bilinear velocity at (xp, yp) in (0, Lx] x (0, Ly] (src/main2csh.f95:187-242,
    products and sums in the reference's order); in the last column / row the
    far grid values are those of column / row 1 (periodic)."""
    Ny, Nx = ux.shape
    dx, dy = Lx / float(Nx), Ly / float(Ny)
    h = 1.0 / (dx * dy)
    i0, i1, x0, x1 = _tracer_cell(xp, dx, Lx, Nx)
    j0, j1, y0, y1 = _tracer_cell(yp, dy, Ly, Ny)
    ax, bx, ay, by = x1 - xp, xp - x0, y1 - yp, yp - y0

    def interp(u):
        v = u[j0, i0] * ax * ay * h
        v = v + u[j0, i1] * bx * ay * h
        v = v + u[j1, i0] * ax * by * h
        return v + u[j1, i1] * bx * by * h
    return interp(ux), interp(uy)


def tracer_move(xp, yp, vx, vy, dt, Lx, Ly):
    """One forward-Euler move with the wrap of src/main2csh.f95:244-256."""
    xn = xp + vx * dt
    yn = yp + vy * dt
    xn = xn - np.trunc(xn / Lx).astype(np.int64).astype(np.float64) * Lx
    xn = np.where(xn <= 0.0, xn + Lx, xn)
    yn = yn - np.trunc(yn / Ly).astype(np.int64).astype(np.float64) * Ly
    yn = np.where(yn <= 0.0, yn + Ly, yn)
    return xn, yn


# ------------------------------------------------------------------ 3D MHD
def derive3com(Nx, Ny, Nz, P: Com3Params, state, pi=PI):
    """src/derive3com.f95:5-1047: d/dt of (rho, rho ux, rho uy, rho uz, E, Bx, By, Bz),
    each a complex (Nz, Ny, Nx/2+1) array (the Fortran (Nh,Ny,Nz) layout)."""
    Nh = Nx // 2 + 1
    st = [np.ascontiguousarray(a, dtype=np.complex128) for a in state]
    out = [_cz((Nz, Ny, Nh)) for _ in range(8)]
    lib().ora_derive3com(Nx, Ny, Nz, pi, C.byref(P), _ptr_array(st), _ptr_array(out))
    return out


def ab3com(Nx, Ny, Nz, dt, state, d_old, d_new):
    """src/ab3com.f95:44-61 (E unchanged)."""
    Nh = Nx // 2 + 1
    st = [np.ascontiguousarray(a, dtype=np.complex128) for a in state]
    do = [np.ascontiguousarray(a, dtype=np.complex128) for a in d_old]
    dn = [np.ascontiguousarray(a, dtype=np.complex128) for a in d_new]
    out = [_cz((Nz, Ny, Nh)) for _ in range(8)]
    lib().ora_ab3com(Nx, Ny, Nz, dt, _ptr_array(st), _ptr_array(out), _ptr_array(do), _ptr_array(dn))
    return out


def run3com(Nx, Ny, Nz, P: Com3Params, nsteps, state, d_old=None, pi=PI):
    """nsteps of the time loop of src/main3com.f95:536-600 (AB2, history from zero)."""
    Nh = Nx // 2 + 1
    st = [np.array(a, dtype=np.complex128, order="C") for a in state]
    do = [np.array(a, dtype=np.complex128, order="C") for a in d_old] if d_old is not None else \
        [_cz((Nz, Ny, Nh)) for _ in range(8)]
    lib().ora_run3com(Nx, Ny, Nz, pi, C.byref(P), nsteps, _ptr_array(st), _ptr_array(do))
    return st, do
