"""CUDA vorticity path (*2csh unscreened, *2css screened) against the CPU
oracle, through the C ABI.

Tolerances: FP64 relative L2 <= 1e-12 for one RHS evaluation and <= 1e-11
after short AB2/RK4 runs (the two paths differ only by FFT rounding); FP32
relative L2 <= 2e-5 for one RHS evaluation."""
import ctypes as C

import numpy as np
import pytest

from tests.gpu_common import rel_l2
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu

PI = 3.14159265358979323846
VPI = float(np.float32(3.1428))  # real(kind=8), parameter :: pi = 3.1428 (default-real literal)
SIZES = [(16, 16), (64, 64), (128, 64), (32, 128), (256, 256), (384, 384), (1024, 32)]


def csh_params(tara, nu=1e-3, dt=1e-3):
    return tara.Params.make(pi=VPI, Lx=2 * VPI, Ly=2 * VPI, nu=nu, dt=dt)


def css_params(tara, alpha=1.0, nu=1e-3, lam=10.0, dt=1e-3, Lx=2 * PI, Ly=2 * PI):
    return tara.Params.make(pi=VPI, Lx=Lx, Ly=Ly, nu=nu, alpha=alpha, dt=dt, **{"lambda": lam})


def noise(Nx, Ny, seed):
    rng = np.random.default_rng(seed)
    Nh = Nx // 2 + 1
    return rng.standard_normal((Ny, Nh)) + 1j * rng.standard_normal((Ny, Nh))


@pytest.mark.parametrize("Nx,Ny", SIZES)
def test_derive2csh_session(tara, oracle, Nx, Ny):
    w = I.vorticity_random_phase(Nx, Ny, seed=Nx + 3 * Ny)
    ref = oracle.derive2csh(Nx, Ny, 1e-3, w[0])
    with tara.Session(tara.MODEL_CSH, Nx, Ny, csh_params(tara)) as s:
        s.set_state(w)
        got = s.rhs()[0]
    assert rel_l2(got, ref) <= 1e-12, rel_l2(got, ref)


@pytest.mark.parametrize("Nx,Ny", SIZES)
def test_derive2css_session(tara, oracle, Nx, Ny):
    w = I.vorticity_random_phase(Nx, Ny, seed=Nx + 5 * Ny)
    ref = oracle.derive2css(Nx, Ny, 0.7, 2e-3, 2 * PI, 2 * PI, 10.0, w[0])
    with tara.Session(tara.MODEL_CSS, Nx, Ny, css_params(tara, alpha=0.7, nu=2e-3)) as s:
        s.set_state(w)
        got = s.rhs()[0]
    assert rel_l2(got, ref) <= 1e-12, rel_l2(got, ref)


@pytest.mark.parametrize("model", ["csh", "css"])
def test_non_hermitian_input(tara, oracle, model):
    """Arbitrary complex input: the kx = 0 / Nyquist columns are not
    Hermitian and the k = 0 mode is non-zero."""
    Nx, Ny = 64, 32
    w = noise(Nx, Ny, 7)
    if model == "csh":
        ref = oracle.derive2csh(Nx, Ny, 1e-2, w)
        p, m = csh_params(tara, nu=1e-2), tara.MODEL_CSH
    else:
        ref = oracle.derive2css(Nx, Ny, 1.3, 1e-2, 3.0, 5.0, 2.5, w)
        p, m = css_params(tara, alpha=1.3, nu=1e-2, lam=2.5, Lx=3.0, Ly=5.0), tara.MODEL_CSS
    with tara.Session(m, Nx, Ny, p) as s:
        s.set_state([w])
        got = s.rhs()[0]
    assert rel_l2(got, ref) <= 1e-12, rel_l2(got, ref)


def test_ab2_run_csh(tara, oracle):
    Nx = Ny = 128
    dt, nu, nsteps = 2e-3, 1e-3, 25
    w = I.vorticity_random_phase(Nx, Ny, seed=5)[0]
    ref, d_old = w.copy(), np.zeros_like(w)
    for _ in range(nsteps):
        d = oracle.derive2csh(Nx, Ny, nu, ref)
        ref = oracle.ab2csh(Nx, Ny, dt, ref, d_old, d)
        d_old = d
    with tara.Session(tara.MODEL_CSH, Nx, Ny, csh_params(tara, nu=nu, dt=dt)) as s:
        s.set_state([w])
        s.step(tara.STEP_AB2, nsteps)
        got = s.get_state()[0]
        hist = s.get_history()[0]
    assert rel_l2(got, ref) <= 1e-11, rel_l2(got, ref)
    assert rel_l2(hist, d_old) <= 1e-11


def _rk4_oracle(oracle, Nx, Ny, w, dt, nsteps, rhs):
    """Classical RK4 with the session's operation order:
    acc = u + (dt/6) k1, u_s = u + c_s dt k_s, acc += (w_s dt/6) k_s, u_new = acc + (dt/6) k4."""
    wts, cs = (1.0, 2.0, 2.0, 1.0), (0.5, 0.5, 1.0)
    u = w.copy()
    for _ in range(nsteps):
        k = rhs(u)
        acc = u + (wts[0] * dt / 6.0) * k
        us = u + (cs[0] * dt) * k
        for s in range(1, 4):
            k = rhs(us)
            if s < 3:
                acc = acc + (wts[s] * dt / 6.0) * k
                us = u + (cs[s] * dt) * k
            else:
                u = acc + (wts[s] * dt / 6.0) * k
    return u


def test_rk4_run_css(tara, oracle):
    Nx = Ny = 64
    dt, nu, alpha, lam, nsteps = 2e-3, 1e-3, 1.0, 10.0, 10
    w = I.vorticity_random_phase(Nx, Ny, seed=9)[0]
    ref = _rk4_oracle(oracle, Nx, Ny, w, dt, nsteps,
                      lambda u: oracle.derive2css(Nx, Ny, alpha, nu, 2 * PI, 2 * PI, lam, u))
    with tara.Session(tara.MODEL_CSS, Nx, Ny, css_params(tara, alpha=alpha, nu=nu, lam=lam, dt=dt)) as s:
        s.set_state([w])
        s.step(tara.STEP_RK4, nsteps)
        got = s.get_state()[0]
    assert rel_l2(got, ref) <= 1e-11, rel_l2(got, ref)


def test_fp32_rhs(tara, oracle):
    Nx = Ny = 256
    w = I.vorticity_random_phase(Nx, Ny, seed=13)
    ref = oracle.derive2csh(Nx, Ny, 1e-3, w[0])
    with tara.Session(tara.MODEL_CSH, Nx, Ny, csh_params(tara), precision=tara.FP32) as s:
        s.set_state(w)
        got = s.rhs()[0]
    assert rel_l2(got, ref) <= 2e-5, rel_l2(got, ref)


# ----------------------------------------------------------- drop-in symbols
def _i(v):
    return C.byref(C.c_int32(v))


def _d(v):
    return C.byref(C.c_double(v))


def _a(x):
    assert x.dtype == np.complex128 and x.flags.c_contiguous
    return C.c_void_p(x.ctypes.data)


def test_dropin_csh(tara, oracle):
    L = tara.lib()
    Nx, Ny = 64, 64
    Nh = Nx // 2 + 1
    nu, dt = 1e-3, 1e-3
    w = np.ascontiguousarray(I.vorticity_random_phase(Nx, Ny, seed=2)[0])
    d_old = np.ascontiguousarray(oracle.derive2csh(Nx, Ny, nu, 0.9 * w))
    w_new = np.zeros_like(w)
    d_new = np.zeros_like(w)
    L.derive2csh_(_i(Nx), _i(Ny), _i(Nh), _d(nu), _d(0.0), _a(w), _a(w_new), _a(d_old), _a(d_new))
    assert L.tara_legacy_status() == 0, tara.last_error()
    ref = oracle.derive2csh(Nx, Ny, nu, w)
    assert rel_l2(d_new, ref) <= 1e-12
    L.ab2csh_(_i(Nx), _i(Ny), _i(Nh), _d(nu), _d(0.0), _d(dt), _a(w), _a(w_new), _a(d_old), _a(d_new))
    assert L.tara_legacy_status() == 0, tara.last_error()
    ref_w = oracle.ab2csh(Nx, Ny, dt, w, d_old, d_new)
    assert rel_l2(w_new, ref_w) <= 1e-14


def test_dropin_css(tara, oracle):
    L = tara.lib()
    Nx, Ny = 32, 64
    Nh = Nx // 2 + 1
    alpha, nu, dt, lam = 1.0, 1e-3, 1e-3, 4.0
    assert L.tara_set_css_box(C.c_double(2 * PI), C.c_double(2 * PI), C.c_double(lam)) == 0
    try:
        w = np.ascontiguousarray(I.vorticity_random_phase(Nx, Ny, seed=3)[0])
        d_old = np.ascontiguousarray(oracle.derive2css(Nx, Ny, alpha, nu, 2 * PI, 2 * PI, lam, 1.1 * w))
        w_new = np.zeros_like(w)
        d_new = np.zeros_like(w)
        L.derive2css_(_i(Nx), _i(Ny), _i(Nh), _d(alpha), _d(nu), _d(0.0), _a(w), _a(w_new), _a(d_old),
                      _a(d_new))
        assert L.tara_legacy_status() == 0, tara.last_error()
        assert rel_l2(d_new, oracle.derive2css(Nx, Ny, alpha, nu, 2 * PI, 2 * PI, lam, w)) <= 1e-12
        L.ab2css_(_i(Nx), _i(Ny), _i(Nh), _d(alpha), _d(nu), _d(0.0), _d(dt), _a(w), _a(w_new), _a(d_old),
                  _a(d_new))
        assert L.tara_legacy_status() == 0, tara.last_error()
        assert rel_l2(w_new, oracle.ab2csh(Nx, Ny, dt, w, d_old, d_new)) <= 1e-14
        L.rk42css_(_i(Nx), _i(Ny), _i(Nh), _d(alpha), _d(nu), _d(0.0), _d(dt), _a(w), _a(w_new), _a(d_old),
                   _a(d_new))
        assert L.tara_legacy_status() == 0, tara.last_error()
        ref = _rk4_oracle(oracle, Nx, Ny, w, dt, 1,
                          lambda u: oracle.derive2css(Nx, Ny, alpha, nu, 2 * PI, 2 * PI, lam, u))
        assert rel_l2(w_new, ref) <= 1e-12
    finally:
        L.tara_set_css_box(C.c_double(2 * PI), C.c_double(2 * PI), C.c_double(10.0))
