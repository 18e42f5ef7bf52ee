"""On-device diagnostics (Energy.dat values and E(k)) against the oracle, and
full runs with diagnostics recorded on the device.

Tolerances: one evaluation, FP64: relative error <= 1e-10 per value (div B,
which is rounding noise around 0, to 1e-12 absolute) and relative L2 <= 1e-10
for E(k); recorded runs: fields relative L2 <= 1e-10 after 100 RK4 steps and
every diagnostic within 1e-6 relative over the run."""
import numpy as np
import pytest

from tests.gpu_common import com_kw, coh_kw, oracle_com_params, oracle_coh_params, rel_l2
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu


def _close(got, ref, rtol, atol=0.0):
    return abs(got - ref) <= rtol * abs(ref) + atol


@pytest.mark.parametrize("Nx,Ny", [(16, 16), (64, 64), (128, 64), (256, 256), (384, 384)])
def test_diag_com(tara, oracle, Nx, Ny):
    kw = com_kw()
    st = I.com_random_phase(Nx, Ny, seed=Nx + Ny)
    P = oracle_com_params(oracle, kw)
    ref = oracle.diag_com(Nx, Ny, P, st)
    ref_ek = oracle.spectrum_com(Nx, Ny, P, st)
    with tara.Session(tara.MODEL_COM, Nx, Ny, tara.Params.make(**kw)) as s:
        s.set_state(st)
        vals, ek = s.diagnostics()
    assert ek.shape == ref_ek.shape
    for k in (0, 1, 2, 3, 5):
        assert _close(vals[k], ref[k], 1e-10), (k, vals[k], ref[k])
    assert _close(vals[4], ref[4], 0.0, 1e-12), (vals[4], ref[4])
    assert rel_l2(ek, ref_ek) <= 1e-10, rel_l2(ek, ref_ek)


@pytest.mark.parametrize("Nx,Ny", [(16, 16), (64, 64), (128, 256), (512, 512)])
def test_diag_coh(tara, oracle, Nx, Ny):
    kw = coh_kw()
    st = I.coh_random_phase(Nx, Ny, seed=2 * Nx + Ny)
    P = oracle_coh_params(oracle, kw)
    ref = oracle.diag_coh(Nx, Ny, P, st)
    ref_ek = oracle.spectrum_coh(Nx, Ny, P, st[1], st[2])
    with tara.Session(tara.MODEL_COH, Nx, Ny, tara.Params.make(**kw)) as s:
        s.set_state(st)
        vals, ek = s.diagnostics()
    for k in (0, 1, 2, 4):
        assert _close(vals[k], ref[k], 1e-10), (k, vals[k], ref[k])
    # C1 = <omega> and C3 = <omega^3> are near-cancelling sums
    scale = np.sqrt(ref[4])
    assert _close(vals[3], ref[3], 0.0, 1e-12 * scale)
    assert _close(vals[5], ref[5], 0.0, 1e-10 * scale ** 3)
    assert rel_l2(ek, ref_ek) <= 1e-10, rel_l2(ek, ref_ek)


def test_diag_com_fp32(tara, oracle):
    Nx = Ny = 256
    kw = com_kw()
    st = I.com_random_phase(Nx, Ny, seed=1)
    P = oracle_com_params(oracle, kw)
    ref = oracle.diag_com(Nx, Ny, P, st)
    ref_ek = oracle.spectrum_com(Nx, Ny, P, st)
    with tara.Session(tara.MODEL_COM, Nx, Ny, tara.Params.make(**kw), precision=tara.FP32) as s:
        s.set_state(st)
        vals, ek = s.diagnostics()
    for k in (0, 1, 2, 3):
        assert _close(vals[k], ref[k], 1e-5), (k, vals[k], ref[k])
    assert rel_l2(ek, ref_ek) <= 1e-5


def test_diag_unsupported_model(tara):
    with tara.Session(tara.MODEL_CSH, 32, 32, tara.Params.make(nu=1e-3)) as s:
        with pytest.raises(tara.TaraError):
            s.diagnostics()


def _oracle_record(oracle, Nx, Ny, P, st):
    return oracle.diag_com(Nx, Ny, P, st), oracle.spectrum_com(Nx, Ny, P, st)


@pytest.mark.parametrize("N,nsteps,every", [(256, 100, 20), (1024, 100, 50)])
def test_recorded_mhd_rk4_run(tara, oracle, N, nsteps, every):
    """The MHD Orszag-Tang workload (perturbed) under RK4: state after 100
    steps and the diagnostics along the way, against the oracle's run."""
    kw = com_kw()
    P = oracle_com_params(oracle, kw)
    st0 = I.com_orszag_tang(N, N, seed=7)
    nrec = nsteps // every + 1
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**kw)) as s:
        s.set_state(st0)
        vals, eks = s.run_recorded(tara.STEP_RK4, every, nrec)
        got = s.get_state()
    st = [a.copy() for a in st0]
    d_old = None
    for k in range(nrec):
        if k > 0:
            st, d_old = oracle.run_com(N, N, P, 1, every, st, d_old)
        ref, ref_ek = _oracle_record(oracle, N, N, P, st)
        for q in (0, 1, 2, 3, 5):
            assert _close(vals[k, q], ref[q], 1e-6), (k, q, vals[k, q], ref[q])
        assert abs(vals[k, 4] - ref[4]) <= 1e-10
        assert rel_l2(eks[k], ref_ek) <= 1e-6
    for g, r in zip(got, st):
        assert rel_l2(g, r) <= 1e-10, rel_l2(g, r)


def test_recorded_hydro_ab2_run(tara, oracle):
    N, every, nrec = 128, 25, 5
    kw = coh_kw(dt=1e-3)
    P = oracle_coh_params(oracle, kw)
    st0 = I.coh_random_phase(N, N, seed=12)
    with tara.Session(tara.MODEL_COH, N, N, tara.Params.make(**kw)) as s:
        s.set_state(st0)
        vals, eks = s.run_recorded(tara.STEP_AB2, every, nrec)
    st, d_old = [a.copy() for a in st0], None
    for k in range(nrec):
        if k > 0:
            st, d_old = oracle.run_coh(N, N, P, 0, every, st, d_old)
        ref = oracle.diag_coh(N, N, P, st)
        ref_ek = oracle.spectrum_coh(N, N, P, st[1], st[2])
        for q in (0, 1, 2, 4):
            assert _close(vals[k, q], ref[q], 1e-6), (k, q)
        assert rel_l2(eks[k], ref_ek) <= 1e-6
