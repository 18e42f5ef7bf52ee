"""CUDA MHD path (*2com) against the CPU oracle, through the C ABI.

FP64 tolerances: one RHS evaluation, relative L2 <= 1e-10 per field (the
energy equation carries E ~ CS^2 rho/(gamma-1) ~ 1.5e4 with O(1) fluxes, so
its derivative is the most cancellation-prone); short runs <= 1e-10."""
import os

import numpy as np
import pytest

from tests.gpu_common import com_kw, oracle_com_params, rel_l2
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu


def compressive(st, seed, amp=1e-3):
    """Adds seeded compressive (non-solenoidal) noise on every mode so that
    every field's derivative, d(rho)/dt included, is far above rounding (an
    Orszag-Tang state with solenoidal perturbations has div(rho u) = 0 and
    d(rho)/dt is pure rounding noise in both codes)."""
    rng = np.random.default_rng(seed)
    out = []
    for a in st:
        s = np.abs(a).max()
        out.append(a + amp * s * (rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape)) / a.size ** 0.5)
    return out


@pytest.mark.parametrize("Nx,Ny", [(16, 16), (32, 32), (64, 64), (128, 64), (64, 128), (256, 256), (384, 384),
                                   (1024, 1024)])
def test_derive2com_session(tara, oracle, Nx, Ny):
    kw = com_kw()
    st = compressive(I.com_orszag_tang(Nx, Ny, seed=Nx + 3 * Ny, kmin=2.0, kmax=min(16.0, Nx / 4.0)), Nx)
    ref = oracle.derive2com(Nx, Ny, oracle_com_params(oracle, kw), st)
    with tara.Session(tara.MODEL_COM, Nx, Ny, tara.Params.make(**kw)) as s:
        s.set_state(st)
        got = s.rhs()
    for q, (g, r) in enumerate(zip(got, ref)):
        assert rel_l2(g, r) <= 1e-10, (q, rel_l2(g, r))


@pytest.mark.parametrize("fix,A", [(1, 0.0), (0, 0.25), (1, 0.25)])
def test_derive2com_switches(tara, oracle, fix, A):
    Nx = Ny = 64
    kw = com_kw(fix_curlB=fix, A=A, kf=2.0)
    st = compressive(I.com_random_phase(Nx, Ny, seed=5, k0=4.0), 6)
    ref = oracle.derive2com(Nx, Ny, oracle_com_params(oracle, kw), st)
    with tara.Session(tara.MODEL_COM, Nx, Ny, tara.Params.make(**kw)) as s:
        s.set_state(st)
        got = s.rhs()
    for q, (g, r) in enumerate(zip(got, ref)):
        assert rel_l2(g, r) <= 1e-10, (q, rel_l2(g, r))


def test_derive2com_dropin_symbol(tara, oracle):
    Nx, Ny = 32, 32
    kw = com_kw(mu=1e-3, eta=2e-4)
    rng = np.random.default_rng(3)
    st = I.com_orszag_tang(Nx, Ny, seed=2, kmin=2, kmax=8)
    st = [a + 1e-3 * (rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape)) for a in st]
    ref = oracle.derive2com(Nx, Ny, oracle_com_params(oracle, kw), st)
    p = tara.Params.make(**kw)
    tara.set_comm(tara.comm_com(p))
    z = lambda: np.zeros((Ny, Nx // 2 + 1), np.complex128)
    d = [[z(), z()] for _ in range(6)]  # (old, new) per field, interleaved like the reference
    args = [np.ascontiguousarray(a) for a in st] + [x for pair in d for x in pair]
    assert tara.legacy_call("derive2com_", Nx, Ny, kw["pi"], 0.0, args) == 0, tara.last_error()
    for q in range(6):
        assert rel_l2(d[q][1], ref[q]) <= 1e-10, (q, rel_l2(d[q][1], ref[q]))


def test_golden_fixture_derive2com(tara):
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "derive2com_16.npz"))
    with tara.Session(tara.MODEL_COM, 16, 16, tara.Params.make(**com_kw())) as s:
        s.set_state(list(g["state"]))
        got = s.rhs()
    for a, b in zip(got, g["rhs"]):
        assert rel_l2(a, b) <= 1e-10


@pytest.mark.parametrize("stepper", [0, 1])
def test_mhd_steps_vs_oracle(tara, oracle, stepper):
    Nx = Ny = 64
    kw = com_kw(dt=5e-5)
    st = I.com_orszag_tang(Nx, Ny, seed=8, kmin=2, kmax=8)
    n = 20
    ref, _ = oracle.run_com(Nx, Ny, oracle_com_params(oracle, kw), stepper, n, st)
    with tara.Session(tara.MODEL_COM, Nx, Ny, tara.Params.make(**kw)) as s:
        s.set_state(st)
        s.step(stepper, n)
        got = s.get_state()
    for q, (g, r) in enumerate(zip(got, ref)):
        assert rel_l2(g, r) <= 1e-10, (q, rel_l2(g, r))


def test_dropin_ab2com(tara, oracle):
    Nx, Ny = 32, 16
    kw = com_kw()
    P = oracle_com_params(oracle, kw)
    st = I.com_orszag_tang(Nx, Ny, seed=1, kmin=2, kmax=6)
    dn = oracle.derive2com(Nx, Ny, P, st)
    do = oracle.derive2com(Nx, Ny, P, [a * 1.01 for a in st])
    tara.set_comm(tara.comm_com(tara.Params.make(**kw)))
    z = lambda: np.zeros((Ny, Nx // 2 + 1), np.complex128)
    new = [z() for _ in range(6)]
    inter = [x for q in range(6) for x in (np.ascontiguousarray(do[q]), np.ascontiguousarray(dn[q]))]
    assert tara.legacy_call("ab2com_", Nx, Ny, kw["pi"], 0.0, [np.ascontiguousarray(a) for a in st] + new + inter) == 0
    ref = oracle.ab2com(Nx, Ny, P, st, do, dn)
    for g, r in zip(new, ref):
        assert rel_l2(g, r) <= 1e-15
