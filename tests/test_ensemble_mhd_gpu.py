"""MHD (*2com) members in batched ensembles, alone and mixed with hydro
members, against single-grid sessions and the oracle.

The MHD phase kernels run the sessions' device code with the sessions'
values per thread, so every member's state, AB2 history and diagnostics must
be bit-identical to a session run of that member (the same steps, the same
calls in between).  FP64 members also match the oracle's AB2 run of
src/derive2com.f95 + src/ab2com.f95 to relative L2 <= 1e-10 per field (the
MHD tolerance of the single-grid parity tests: E carries ~1e4 with O(1)
fluxes)."""
import numpy as np
import pytest

from tests.gpu_common import coh_kw, com_kw, oracle_com_params, rel_l2
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu

SIZES = [128, 256, 384, 512, 128]
MUS = [1e-3, 5e-4, 2e-3, 1e-3, 5e-3]


def _com_members(tara, sizes=SIZES, mus=MUS, dt=1e-5, CS=10.0):
    kws = [com_kw(mu=mu, eta=0.5 * mu, dt=dt, CS=CS) for mu in mus]
    params = [tara.Params.make(**k) for k in kws]
    states = [I.com_random_phase(N, N, seed=20 + m, k0=3.0 + m, CS=CS) for m, N in enumerate(sizes)]
    return kws, params, states


def _session(tara, model, N, p, st, precision, plan):
    """Runs `plan` (a list of step counts, or "diag" for a diagnostics call
    in between) on a session; returns state, history, last diagnostics."""
    with tara.Session(model, N, N, p, precision=precision) as s:
        s.set_state(st)
        diag = None
        for item in plan:
            if item == "diag":
                diag = s.diagnostics()
            else:
                s.step(tara.STEP_AB2, item)
        return s.get_state(), s.get_history(), s.diagnostics() if diag is None else diag


def _same(got, ref, tag):
    for a, b in zip(got, ref):
        assert np.array_equal(a, b), (tag, rel_l2(a, b))


@pytest.mark.parametrize("precision", [1, 0])
def test_mhd_members_bit_identical_to_sessions(tara, precision):
    _, params, states = _com_members(tara)
    with tara.Ensemble(SIZES, params, precision=precision, model=tara.MODEL_COM) as e:
        assert all(len(e.get_state(m)) == 6 for m in range(len(SIZES)))
        for m, st in enumerate(states):
            e.set_state(m, st)
        e.step(tara.STEP_AB2, 3)  # first step (column inverse), one captured pair
        e.step(tara.STEP_AB2, 4)  # two pairs
        got = [(e.get_state(m), e.get_history(m), e.diagnostics(m)) for m in range(len(SIZES))]
    for m, N in enumerate(SIZES):
        ref_st, ref_h, (ref_v, ref_ek) = _session(tara, tara.MODEL_COM, N, params[m], states[m], precision, [3, 4])
        st, h, (v, ek) = got[m]
        _same(st + h, ref_st + ref_h, (m, N))
        assert np.allclose(v, ref_v, rtol=1e-12, atol=0)
        assert np.allclose(ek, ref_ek, rtol=1e-12, atol=1e-300)


def test_mixed_hydro_mhd_bit_identical(tara):
    """Hydro and MHD members of every size in one ensemble (FP32, as the
    ensemble configuration runs)."""
    sizes = [256, 128, 384, 512, 128, 384]
    models = [tara.MODEL_COH, tara.MODEL_COM, tara.MODEL_COM, tara.MODEL_COH, tara.MODEL_COH, tara.MODEL_COM]
    params, states = [], []
    for m, (N, mod) in enumerate(zip(sizes, models)):
        if mod == tara.MODEL_COH:
            params.append(tara.Params.make(**coh_kw(mux=1e-3 * (m + 1), muy=1e-3 * (m + 1), dt=2e-4)))
            states.append(I.coh_random_phase(N, N, seed=40 + m, k0=2.0 + m))
        else:
            params.append(tara.Params.make(**com_kw(mu=1e-3 * (m + 1), eta=1e-3, dt=1e-5, CS=10.0)))
            states.append(I.com_random_phase(N, N, seed=40 + m, k0=3.0, CS=10.0))
    with tara.Ensemble(sizes, params, precision=tara.FP32, model=models) as e:
        for m, st in enumerate(states):
            e.set_state(m, st)
        e.step(tara.STEP_AB2, 5)
        got = [(e.get_state(m), e.get_history(m)) for m in range(len(sizes))]
    for m, (N, mod) in enumerate(zip(sizes, models)):
        ref_st, ref_h, _ = _session(tara, mod, N, params[m], states[m], tara.FP32, [5])
        _same(got[m][0] + got[m][1], ref_st + ref_h, (m, N, mod))


def test_diagnostics_between_steps(tara):
    """A diagnostics call uses the members' work fields; the next step must
    redo the column inverse, as a session does."""
    sizes, mus = [256, 128], [1e-3, 2e-3]
    _, params, states = _com_members(tara, sizes, mus)
    plan = [3, "diag", 4]
    with tara.Ensemble(sizes, params, precision=tara.FP64, model=tara.MODEL_COM) as e:
        for m, st in enumerate(states):
            e.set_state(m, st)
        e.step(tara.STEP_AB2, 3)
        mid = [e.diagnostics(m) for m in range(2)]
        e.step(tara.STEP_AB2, 4)
        got = [e.get_state(m) + e.get_history(m) for m in range(2)]
    for m, N in enumerate(sizes):
        ref_st, ref_h, (ref_v, _) = _session(tara, tara.MODEL_COM, N, params[m], states[m], tara.FP64, plan)
        _same(got[m], ref_st + ref_h, m)
        assert np.allclose(mid[m][0], ref_v, rtol=1e-12, atol=0)


def test_mhd_euler_bit_identical(tara):
    _, params, states = _com_members(tara, [256], [1e-3])
    with tara.Ensemble([256], params, precision=tara.FP64, model=tara.MODEL_COM) as e:
        e.set_state(0, states[0])
        e.step(tara.STEP_EULER, 5)
        got = e.get_state(0)
    with tara.Session(tara.MODEL_COM, 256, 256, params[0], precision=tara.FP64) as s:
        s.set_state(states[0])
        s.step(tara.STEP_EULER, 5)
        ref = s.get_state()
    _same(got, ref, "euler")


def test_fp64_mhd_members_vs_oracle(tara, oracle):
    sizes, mus = [128, 256], [1e-3, 2e-3]
    kws, params, states = _com_members(tara, sizes, mus)
    with tara.Ensemble(sizes, params, precision=tara.FP64, model=tara.MODEL_COM) as e:
        for m, st in enumerate(states):
            e.set_state(m, st)
        e.step(tara.STEP_AB2, 10)
        got = [e.get_state(m) for m in range(2)]
    for m, N in enumerate(sizes):
        ref, _ = oracle.run_com(N, N, oracle_com_params(oracle, kws[m]), 0, 10, states[m])
        for q, (a, b) in enumerate(zip(got[m], ref)):
            assert rel_l2(a, b) <= 1e-10, (m, q, rel_l2(a, b))


def test_autotune_leaves_mhd_members_unchanged(tara):
    """Autotuning times the hydro phases only; afterwards every member
    (hydro and MHD) continues bit-identically to a session run."""
    sizes = [128, 256]
    models = [tara.MODEL_COH, tara.MODEL_COM]
    params = [tara.Params.make(**coh_kw(dt=2e-4)), tara.Params.make(**com_kw(dt=1e-5, CS=10.0))]
    states = [I.coh_random_phase(128, 128, seed=5), I.com_random_phase(256, 256, seed=6, CS=10.0)]
    with tara.Ensemble(sizes, params, precision=tara.FP32, model=models) as e:
        for m, st in enumerate(states):
            e.set_state(m, st)
        e.step(tara.STEP_AB2, 2)
        e.autotune(tara.STEP_AB2, reps=1)
        e.set_tuning([16, 16, 16, 0, 0, 0])  # the sessions' values per thread again
        e.step(tara.STEP_AB2, 3)
        got = [e.get_state(m) + e.get_history(m) for m in range(2)]
    for m, N in enumerate(sizes):
        ref_st, ref_h, _ = _session(tara, models[m], N, params[m], states[m], tara.FP32, [2, 3])
        _same(got[m], ref_st + ref_h, m)


def test_mhd_ensemble_errors(tara):
    p = tara.Params.make(**com_kw(A=1.0))
    with pytest.raises(tara.TaraError):
        tara.Ensemble([128], p, model=tara.MODEL_COM)  # forcing is not run in ensembles
    with pytest.raises(tara.TaraError):
        tara.Ensemble([128], tara.Params.make(**com_kw(fix_curlB=1)), model=tara.MODEL_COM)
    with pytest.raises(tara.TaraError):
        tara.Ensemble([128], tara.Params.make(**com_kw()), model=[tara.MODEL_COM + 5])
    with tara.Ensemble([128, 128], tara.Params.make(**com_kw()), model=[tara.MODEL_COH, tara.MODEL_COM]) as e:
        assert tara.lib().tara_ens_num_fields(e._h, 0) == 3
        assert tara.lib().tara_ens_num_fields(e._h, 1) == 6
        with pytest.raises(tara.TaraError):
            e.set_state(1, I.coh_random_phase(128, 128, seed=1))  # 3 fields for an MHD member


def test_closure_pairs_from_ensemble_members(tara):
    """Training pairs of the learned closure taken from FP64 MHD ensemble
    members (a batch of fine runs stepped together) are bit-identical to pairs
    taken from sessions holding the same states."""
    sizes, mus = [256, 128], [1e-3, 2e-3]
    _, params, states = _com_members(tara, sizes, mus)
    nsteps = 4
    with tara.Ensemble(sizes, params, precision=tara.FP64, model=tara.MODEL_COM) as e, \
            tara.Closure(64, 4) as c_ens, tara.Closure(64, 4) as c_ses:
        for m, st in enumerate(states):
            e.set_state(m, st)
        e.step(tara.STEP_AB2, nsteps)
        for m in range(2):
            c_ens.add_pair_member(e, m)
        for m, N in enumerate(sizes):
            with tara.Session(tara.MODEL_COM, N, N, params[m], precision=tara.FP64) as s:
                s.set_state(states[m])
                s.step(tara.STEP_AB2, nsteps)
                c_ses.add_pair(s)
        assert c_ens.count == 2 and c_ses.count == 2
        for m in range(2):
            for a, b in zip(c_ens.get_pair(m), c_ses.get_pair(m)):
                assert np.array_equal(a, b), m
        with pytest.raises(tara.TaraError):  # hydro or FP32 members give no pairs
            with tara.Ensemble([128], tara.Params.make(**com_kw()), precision=tara.FP32,
                               model=tara.MODEL_COM) as e32:
                c_ens.add_pair_member(e32, 0)
