"""Seeded initial conditions built on the device (tara_set_state_random)
against the host restatement of the same counter-based generator
(tara2d_b200.initial.hashed_state).  FP64: relative L2 <= 1e-12 per field
(the two sides differ in FFT and math-function rounding only); FP32:
<= 2e-6."""
import numpy as np
import pytest

from tests.gpu_common import coh_kw, com_kw, rel_l2
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("Nx,Ny,prec", [(128, 128, 0), (128, 64, 0), (256, 256, 1)])
def test_hydro_random_phase(tara, Nx, Ny, prec):
    kw = coh_kw()
    ref = I.hashed_state(1, Nx, Ny, I.IC_RANDOM_PHASE, seed=11, k0=4.0, e1=0.5, e2=0.01)
    with tara.Session(tara.MODEL_COH, Nx, Ny, tara.Params.make(**kw), precision=prec) as s:
        s.set_state_random(tara.IC_RANDOM_PHASE, 11, k0=4.0, e1=0.5, e2=0.01)
        got = s.get_state()
    tol = 1e-12 if prec == 0 else 2e-6
    for a, b in zip(got, ref):
        assert rel_l2(a, b) <= tol


@pytest.mark.parametrize("N", [64, 384])
def test_mhd_random_phase(tara, N):
    kw = com_kw()
    ref = I.hashed_state(2, N, N, I.IC_RANDOM_PHASE, seed=4, k0=6.0, e1=0.5, e2=0.5, CS=kw["CS"],
                         spheat=kw["spheat"])
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**kw)) as s:
        s.set_state_random(tara.IC_RANDOM_PHASE, 4, k0=6.0, e1=0.5, e2=0.5)
        got = s.get_state()
    for a, b in zip(got, ref):
        assert rel_l2(a, b) <= 1e-12


def test_mhd_orszag_tang(tara):
    """The 1024^2 workload's initial state (Orszag-Tang + 1e-3 perturbation on
    8 <= |k| <= 16), built at 256^2."""
    N = 256
    kw = com_kw()
    ref = I.hashed_state(2, N, N, I.IC_ORSZAG_TANG, seed=0, e1=1e-3, e2=1e-3, kmin=8.0, kmax=16.0,
                         CS=kw["CS"], spheat=kw["spheat"])
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**kw)) as s:
        s.set_state_random(tara.IC_ORSZAG_TANG, 0, e1=1e-3, e2=1e-3, kmin=8.0, kmax=16.0)
        got = s.get_state()
        vals, _ = s.diagnostics()
    for a, b in zip(got, ref):
        assert rel_l2(a, b) <= 1e-12
    # <|u|^2> of u = (-sin y, sin x) + perturbation: 1 + 1e-6 up to cross terms
    assert abs(vals[0] - 1.0) < 1e-3


def test_repeatable_and_seeded(tara):
    N = 64
    with tara.Session(tara.MODEL_COH, N, N, tara.Params.make(**coh_kw())) as s:
        s.set_state_random(tara.IC_RANDOM_PHASE, 5)
        a = s.get_state()
        s.set_state_random(tara.IC_RANDOM_PHASE, 5)
        b = s.get_state()
        s.set_state_random(tara.IC_RANDOM_PHASE, 6)
        c = s.get_state()
    assert all(np.array_equal(x, y) for x, y in zip(a, b))
    assert not np.array_equal(a[1], c[1])


def test_rejected_requests(tara):
    with tara.Session(tara.MODEL_CSH, 64, 64, tara.Params.make(nu=1e-3)) as s:
        with pytest.raises(tara.TaraError):
            s.set_state_random(tara.IC_RANDOM_PHASE, 1)
    with tara.Session(tara.MODEL_COH, 64, 64, tara.Params.make(**coh_kw())) as s:
        with pytest.raises(tara.TaraError):
            s.set_state_random(tara.IC_ORSZAG_TANG, 1)
        with pytest.raises(tara.TaraError):
            s.set_state_random(7, 1)
