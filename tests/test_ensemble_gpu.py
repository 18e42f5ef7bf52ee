"""Batched ensembles against single-grid sessions and the oracle.

With the sessions' values per thread (the default tuning) every member runs
exactly the session's arithmetic, so states must be bit-identical to a
session run of that member.  After autotuning (other FFT radix plans) the
tolerance is FP32: relative L2 <= 1e-5 against the session after a few steps;
FP64 ensembles match the oracle to <= 1e-11."""
import numpy as np
import pytest

from tests.gpu_common import coh_kw, oracle_coh_params, rel_l2
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu

SIZES = [128, 256, 384, 512, 128, 256]
NUS = [1e-3, 3e-4, 2e-3, 1e-4, 5e-3, 1e-2]


def _members(tara, dt=2e-4):
    params = [tara.Params.make(**coh_kw(mux=nu, muy=nu, dt=dt)) for nu in NUS]
    states = [I.coh_random_phase(N, N, seed=10 + m, k0=2.0 + m) for m, N in enumerate(SIZES)]
    return params, states


def _session_run(tara, N, p, st, nsteps, precision):
    with tara.Session(tara.MODEL_COH, N, N, p, precision=precision) as s:
        s.set_state(st)
        s.step(tara.STEP_AB2, nsteps)
        return s.get_state(), s.get_history(), s.diagnostics()


@pytest.mark.parametrize("precision", [1, 0])
def test_members_bit_identical_to_sessions(tara, precision):
    params, states = _members(tara)
    nsteps = 7  # graph pairs plus one host-launched step
    with tara.Ensemble(SIZES, params, precision=precision) as e:
        assert e.get_tuning() == [16, 16, 16, 0, 0, 0]
        for m, st in enumerate(states):
            e.set_state(m, st)
        e.step(tara.STEP_AB2, 3)
        e.step(tara.STEP_AB2, nsteps - 3)
        got = [(e.get_state(m), e.get_history(m), e.diagnostics(m)) for m in range(len(SIZES))]
    for m, N in enumerate(SIZES):
        ref_state, ref_hist, (ref_vals, ref_ek) = _session_run(tara, N, params[m], states[m], nsteps, precision)
        st, hist, (vals, ek) = got[m]
        for a, b in zip(st + hist, ref_state + ref_hist):
            assert np.array_equal(a, b), (m, N, rel_l2(a, b))
        assert np.allclose(vals, ref_vals, rtol=1e-12, atol=0)
        assert np.allclose(ek, ref_ek, rtol=1e-12, atol=1e-300)


def test_autotune_keeps_state_and_stays_close(tara):
    params, states = _members(tara)
    with tara.Ensemble(SIZES, params, precision=tara.FP32) as e:
        for m, st in enumerate(states):
            e.set_state(m, st)
        e.step(tara.STEP_AB2, 2)
        before = [e.get_state(m) + e.get_history(m) for m in range(len(SIZES))]
        tuning, ms = e.autotune(tara.STEP_AB2, reps=2)
        assert tuning[0] in (8, 16) and tuning[1] in (8, 16) and tuning[2] in (8, 16)
        assert all(t >= 0 for t in tuning[3:]) and all(x > 0 for x in ms)
        after = [e.get_state(m) + e.get_history(m) for m in range(len(SIZES))]
        for a, b in zip(before, after):
            for x, y in zip(a, b):
                assert np.array_equal(x, y)
        e.set_tuning([8, 8, 8, 1, 1, 1])
        e.step(tara.STEP_AB2, 5)
        got = [e.get_state(m) for m in range(len(SIZES))]
    for m, N in enumerate(SIZES):
        ref, _, _ = _session_run(tara, N, params[m], states[m], 7, tara.FP32)
        for a, b in zip(got[m], ref):
            assert rel_l2(a, b) <= 1e-5, (m, rel_l2(a, b))


def test_fp64_members_vs_oracle(tara, oracle):
    sizes = [128, 256]
    kws = [coh_kw(mux=1e-3, muy=1e-3, dt=2e-4), coh_kw(mux=2e-3, muy=2e-3, dt=2e-4)]
    states = [I.coh_random_phase(N, N, seed=3 + m) for m, N in enumerate(sizes)]
    with tara.Ensemble(sizes, [tara.Params.make(**k) for k in kws], precision=tara.FP64) as e:
        e.set_tuning([8, 8, 8, 0, 0, 0])
        for m, st in enumerate(states):
            e.set_state(m, st)
        e.step(tara.STEP_AB2, 10)
        got = [e.get_state(m) for m in range(2)]
    for m, N in enumerate(sizes):
        ref, _ = oracle.run_coh(N, N, oracle_coh_params(oracle, kws[m]), 0, 10, states[m])
        for a, b in zip(got[m], ref):
            assert rel_l2(a, b) <= 1e-11, rel_l2(a, b)


def test_ensemble_errors(tara):
    p = tara.Params.make(**coh_kw())
    with pytest.raises(tara.TaraError):
        tara.Ensemble([100], p)
    with pytest.raises(tara.TaraError):
        tara.Ensemble([128], p, model=tara.MODEL_CSH)  # ensembles run the hydro and MHD models
    with tara.Ensemble([128], p) as e:
        with pytest.raises(tara.TaraError):
            e.step(tara.STEP_RK4, 1)
        with pytest.raises(tara.TaraError):
            e.set_tuning([12, 16, 16, 0, 0, 0])
        with pytest.raises(tara.TaraError):
            e.get_state(1)
        bufs = [np.zeros((128, 65), np.complex128) for _ in range(3)]
        ptrs = (tara.C.c_void_p * 3)(*[b.ctypes.data for b in bufs])
        assert tara.lib().tara_ens_get_state(e._h, 1, ptrs) == tara.EINVAL


def test_config_ensemble_of_256_runs(tara):
    """The 256-member ensemble (sizes, viscosities and k0 drawn as in the
    ensemble workload) steps; sampled members stay finite with their kinetic
    energy within 10% of the start after 20 steps of dt = 1e-4."""
    mem = I.ensemble_members(256, seed=1)
    params = [tara.Params.make(**coh_kw(mux=d["nu"], muy=d["nu"], dt=1e-4)) for d in mem]
    with tara.Ensemble([d["N"] for d in mem], params) as e:
        for m, d in enumerate(mem):
            e.set_state(m, I.coh_random_phase(d["N"], d["N"], seed=d["seed"], k0=d["k0"]))
        e0 = [e.diagnostics(m)[0][0] for m in range(0, 256, 17)]
        e.step(tara.STEP_AB2, 20)
        e1 = [e.diagnostics(m)[0][0] for m in range(0, 256, 17)]
    assert all(np.isfinite(x) for x in e1)
    assert all(abs(b - a) < 0.1 * a for a, b in zip(e0, e1))
