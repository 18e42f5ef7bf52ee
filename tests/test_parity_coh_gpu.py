"""CUDA hydro path (*2coh) against the CPU oracle, through the C ABI.

Tolerances (FP64): relative L2 <= 1e-12 for one RHS evaluation and for short
runs; the oracle and the CUDA path differ only by FFT rounding."""
import numpy as np
import pytest

from tests.gpu_common import coh_kw, oracle_coh_params, rel_l2
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu

SIZES = [(16, 16), (32, 32), (64, 64), (128, 128), (64, 32), (32, 128), (256, 256), (384, 384), (512, 128),
         (1024, 64)]


@pytest.mark.parametrize("Nx,Ny", SIZES)
def test_derive2coh_session(tara, oracle, Nx, Ny):
    kw = coh_kw()
    st = I.coh_random_phase(Nx, Ny, seed=Nx * 7 + Ny)
    ref = oracle.derive2coh(Nx, Ny, oracle_coh_params(oracle, kw), *st)
    with tara.Session(tara.MODEL_COH, Nx, Ny, tara.Params.make(**kw)) as s:
        s.set_state(st)
        got = s.rhs()
    for g, r in zip(got, ref):
        assert rel_l2(g, r) <= 1e-12, rel_l2(g, r)


def test_derive2coh_dropin_symbol_non_hermitian(tara, oracle):
    """derive2coh_ with the Fortran calling convention and COMMON /comm/,
    on inputs whose kx=0/Nyquist columns are not Hermitian."""
    Nx, Ny = 32, 32
    kw = coh_kw(mux=2e-3, muy=1e-3)
    rng = np.random.default_rng(11)
    st = [rng.standard_normal((Ny, Nx // 2 + 1)) + 1j * rng.standard_normal((Ny, Nx // 2 + 1)) for _ in range(3)]
    st[0][0, 0] += 40 * Nx * Ny
    ref = oracle.derive2coh(Nx, Ny, oracle_coh_params(oracle, kw), *st)
    p = tara.Params.make(**kw)
    tara.set_comm(tara.comm_coh(p))
    outs = [np.zeros((Ny, Nx // 2 + 1), np.complex128) for _ in range(6)]
    ins = [np.ascontiguousarray(a) for a in st]
    status = tara.legacy_call("derive2coh_", Nx, Ny, kw["pi"], 0.0, ins + outs)
    assert status == 0, tara.last_error()
    for g, r in zip(outs[3:], ref):
        assert rel_l2(g, r) <= 1e-12, rel_l2(g, r)


def test_golden_fixture_derive2coh(tara):
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "derive2coh_16.npz"))
    with tara.Session(tara.MODEL_COH, 16, 16, tara.Params.make(**coh_kw())) as s:
        s.set_state([g["nk"], g["ukx"], g["uky"]])
        got = s.rhs()
    for a, k in zip(got, ("dn", "dux", "duy")):
        assert rel_l2(a, g[k]) <= 1e-12


@pytest.mark.parametrize("stepper,ostep", [(0, 0), (2, 2), (1, 1)])
def test_time_stepping_vs_oracle(tara, oracle, stepper, ostep):
    Nx = Ny = 64
    kw = coh_kw(dt=2e-3)
    st = I.coh_random_phase(Nx, Ny, seed=21)
    nsteps = 20
    ref, _ = oracle.run_coh(Nx, Ny, oracle_coh_params(oracle, kw), ostep, nsteps, st)
    with tara.Session(tara.MODEL_COH, Nx, Ny, tara.Params.make(**kw)) as s:
        s.set_state(st)
        s.step(stepper, nsteps)
        got = s.get_state()
        assert s.status == 0
    for g, r in zip(got, ref):
        assert rel_l2(g, r) <= 1e-11, rel_l2(g, r)


def test_dropin_steppers(tara, oracle):
    Nx, Ny = 32, 16
    kw = coh_kw(dt=1e-3)
    P = oracle_coh_params(oracle, kw)
    st = I.coh_random_phase(Nx, Ny, seed=4)
    d_new = oracle.derive2coh(Nx, Ny, P, *st)
    d_old = oracle.derive2coh(Nx, Ny, P, *[a * 0.9 for a in st])
    tara.set_comm(tara.comm_coh(tara.Params.make(**kw)))
    z = lambda: np.zeros((Ny, Nx // 2 + 1), np.complex128)
    # ab2coh_(..., nk,ukx,uky, nk_new,ukx_new,uky_new, 3x d_old, 3x d_new)
    new = [z(), z(), z()]
    assert tara.legacy_call("ab2coh_", Nx, Ny, kw["pi"], 0.0, list(st) + new + list(d_old) + list(d_new)) == 0
    ref = oracle.ab2coh(Nx, Ny, P, st, d_old, d_new)
    for g, r in zip(new, ref):
        assert np.array_equal(g, r) or rel_l2(g, r) <= 1e-15
    new = [z(), z(), z()]
    assert tara.legacy_call("euler2coh_", Nx, Ny, kw["pi"], 0.0, list(st) + new + list(d_new)) == 0
    ref = oracle.euler2coh(Nx, Ny, P, st, d_new)
    for g, r in zip(new, ref):
        assert rel_l2(g, r) <= 1e-15
    tara.set_legacy_mode(tara.LEGACY_REFERENCE)
    names = {"pc": ("pc_nk2coh_", "pc_ukx2coh_", "pc_uky2coh_"), "rk4": ("rk4_nk2coh_", "rk4_ukx2coh_", "rk4_uky2coh_")}
    for kind, fns in names.items():
        for w, fn in enumerate(fns):
            out = z()
            nk, ukx, uky = [np.ascontiguousarray(a) for a in st]
            order = {0: [nk, out, ukx, uky], 1: [nk, ukx, out, uky], 2: [nk, ukx, uky, out]}[w]
            assert tara.legacy_call(fn, Nx, Ny, kw["pi"], 0.0, order + list(d_new)) == 0
            ref = (oracle.pc2coh if kind == "pc" else oracle.rk42coh)(w, Nx, Ny, P, st, d_new)
            assert rel_l2(out, ref) <= 1e-15, (fn, rel_l2(out, ref))


def test_fp32_mode_error_bound(tara, oracle):
    Nx = Ny = 128
    kw = coh_kw()
    st = I.coh_random_phase(Nx, Ny, seed=3)
    ref = oracle.derive2coh(Nx, Ny, oracle_coh_params(oracle, kw), *st)
    with tara.Session(tara.MODEL_COH, Nx, Ny, tara.Params.make(**kw), precision=tara.FP32) as s:
        s.set_state(st)
        got = s.rhs()
    for g, r in zip(got, ref):
        assert rel_l2(g, r) <= 1e-4, rel_l2(g, r)
