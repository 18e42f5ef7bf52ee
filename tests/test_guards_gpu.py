"""Time-step control and failure detection of the sessions (no counterpart in
the reference, whose drivers step a fixed dt and check nothing).

* CFL control: the device's FP64 rate max((|ux| + c)/dx + (|uy| + c)/dy)
  (c = CS for hydro, sqrt(CS^2 + |B|^2/rho) for MHD) against the same rate of
  the oracle's real-space fields (relative 1e-12); adaptive RK4 / Euler runs
  against the oracle stepped with the same dt sequence (fields relative L2
  <= 1e-10, time relative 1e-12); the check mode leaves the state untouched
  and reports TARA_ECFL, and is bit-identical to an uncontrolled run below
  the limit.
* Non-finite values: host-injected NaN / inf in tara_set_state and
  tara_set_history give TARA_ENAN; a state that overflows while stepping is
  reported by the next synchronising call; the session works afterwards.
* Bounded waits: the self-test kernel's mbarrier wait (the wait of the TMA
  kernels, with a 1 ms limit) runs out and reports TARA_ETIMEOUT without a
  hang, and the context stays usable.  No GPU is faulted or hung by any of
  these tests: the failures are made on the host (injected values) or by a
  wait that nothing completes, with a limit."""
import numpy as np
import pytest

from tests.gpu_common import PI, coh_kw, com_kw, oracle_coh_params, oracle_com_params, rel_l2
from tests.test_parity_com_gpu import compressive
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu


def _real(oracle, a, Nx):
    Ny = a.shape[0]
    return oracle.c2r_2d(a, Nx) / (Nx * Ny)


def rate_com(oracle, st, Nx, Ny, CS, L=2 * PI):
    rho, mx, my, bx, by = (_real(oracle, st[q], Nx) for q in (0, 1, 2, 4, 5))
    ux, uy = mx / rho, my / rho
    c = np.sqrt(CS * CS + (bx * bx + by * by) / rho)
    return np.max((np.abs(ux) + c) * (Nx / L) + (np.abs(uy) + c) * (Ny / L))


def rate_coh(oracle, st, Nx, Ny, CS, L=2 * PI):
    ux, uy = _real(oracle, st[1], Nx), _real(oracle, st[2], Nx)
    return np.max((np.abs(ux) + CS) * (Nx / L) + (np.abs(uy) + CS) * (Ny / L))


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_cfl_rate_com(tara, oracle, prec):
    N, C = 128, 0.5
    kw = com_kw(dt=1.0)  # far above the limit: the step takes dt_cfl
    st = I.com_random_phase(N, N, seed=21)
    want = C / rate_com(oracle, st, N, N, kw["CS"])
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**kw),
                      precision=tara.FP64 if prec == "fp64" else tara.FP32) as s:
        s.set_state(st)
        s.set_cfl(tara.CFL_ADAPT, C)
        s.step(tara.STEP_RK4, 1)
        t, dt = s.time()
    tol = 1e-12 if prec == "fp64" else 1e-5
    assert abs(dt - want) <= tol * want, (dt, want)
    assert t == dt


def test_cfl_rate_coh(tara, oracle):
    N, C = 128, 0.4
    kw = coh_kw(dt=1.0)
    st = I.coh_random_phase(N, N, seed=22)
    want = C / rate_coh(oracle, st, N, N, kw["CS"])
    with tara.Session(tara.MODEL_COH, N, N, tara.Params.make(**kw)) as s:
        s.set_state(st)
        s.set_cfl(tara.CFL_ADAPT, C)
        s.step(tara.STEP_EULER, 1)
        t, dt = s.time()
    assert abs(dt - want) <= 1e-12 * want, (dt, want)


def test_cfl_adaptive_rk4_run_com(tara, oracle):
    """20 adaptive RK4 steps on a state whose CFL limit is below the
    configured dt, against the oracle stepped with the dt sequence the rate
    of its own state gives."""
    N, C, nsteps = 64, 0.8, 20
    kw = com_kw(dt=1e-2, CS=10.0)  # dt_cfl is about 3.6e-3 here
    st0 = I.com_random_phase(N, N, seed=23, CS=10.0)
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**kw)) as s:
        s.set_state(st0)
        s.set_cfl(tara.CFL_ADAPT, C)
        s.step(tara.STEP_RK4, nsteps)
        got = s.get_state()
        t_got, dt_got = s.time()
    st, t = [a.copy() for a in st0], 0.0
    limited = 0
    for _ in range(nsteps):
        dt = min(kw["dt"], C / rate_com(oracle, st, N, N, kw["CS"]))
        limited += dt < kw["dt"]
        P = oracle_com_params(oracle, dict(kw, dt=dt))
        st, _ = oracle.run_com(N, N, P, 1, 1, st)
        t += dt
    assert limited == nsteps  # every step was limited by the CFL condition
    assert abs(t_got - t) <= 1e-12 * t, (t_got, t)
    for g, r in zip(got, st):
        assert rel_l2(g, r) <= 1e-10, rel_l2(g, r)


def test_cfl_adaptive_euler_run_coh(tara, oracle):
    N, C, nsteps = 64, 0.3, 15
    kw = coh_kw(dt=0.05)
    st0 = I.coh_random_phase(N, N, seed=24)
    with tara.Session(tara.MODEL_COH, N, N, tara.Params.make(**kw)) as s:
        s.set_state(st0)
        s.set_cfl(tara.CFL_ADAPT, C)
        s.step(tara.STEP_EULER, nsteps)
        got = s.get_state()
        t_got, _ = s.time()
    st, t, d_old = [a.copy() for a in st0], 0.0, None
    for _ in range(nsteps):
        dt = min(kw["dt"], C / rate_coh(oracle, st, N, N, kw["CS"]))
        P = oracle_coh_params(oracle, dict(kw, dt=dt))
        st, d_old = oracle.run_coh(N, N, P, 2, 1, st, d_old)
        t += dt
    assert abs(t_got - t) <= 1e-12 * t
    for g, r in zip(got, st):
        assert rel_l2(g, r) <= 1e-11, rel_l2(g, r)


def test_cfl_check_mode(tara):
    """Above the limit no step is taken (state bit-identical, time unchanged,
    TARA_ECFL); below it the controlled run is bit-identical to the plain one."""
    N = 128
    st0 = I.com_orszag_tang(N, N, seed=3)
    # the acoustic limit at 128^2 with CS = 100 is about 4e-4 (CFL number 1)
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**com_kw(dt=2e-3))) as s:
        s.set_state(st0)
        s.set_cfl(tara.CFL_CHECK, 1.0)
        s.step(tara.STEP_RK4, 3)
        with pytest.raises(tara.TaraError) as ei:
            s.synchronize()
        assert ei.value.status == tara.ECFL
        got = s.get_state()
        assert s.time()[0] == 0.0
    for g, r in zip(got, st0):
        assert np.array_equal(g, r)
    out = {}
    for mode in (tara.CFL_OFF, tara.CFL_CHECK):
        with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**com_kw(dt=5e-5))) as s:
            s.set_state(st0)
            if mode:
                s.set_cfl(mode, 1.0)
            s.step(tara.STEP_RK4, 10)
            out[mode] = (s.get_state(), s.time())
    for a, b in zip(out[tara.CFL_OFF][0], out[tara.CFL_CHECK][0]):
        assert np.array_equal(a, b)
    assert abs(out[tara.CFL_CHECK][1][0] - 10 * 5e-5) <= 1e-15


def test_cfl_rejections(tara):
    with tara.Session(tara.MODEL_COM, 32, 32, tara.Params.make(**com_kw())) as s:
        s.set_state(I.com_random_phase(32, 32, seed=1))
        s.set_cfl(tara.CFL_ADAPT, 0.5)
        with pytest.raises(tara.TaraError):
            s.step(tara.STEP_AB2, 1)
        with pytest.raises(tara.TaraError):
            s.set_cfl(tara.CFL_ADAPT, -1.0)
    with tara.Session(tara.MODEL_CSH, 32, 32, tara.Params.make(nu=1e-3)) as s:
        with pytest.raises(tara.TaraError) as ei:
            s.set_cfl(tara.CFL_CHECK, 0.5)
        assert ei.value.status == tara.EUNSUPPORTED


@pytest.mark.parametrize("model", ["com", "coh"])
@pytest.mark.parametrize("bad", [np.nan, np.inf])
def test_set_state_rejects_nonfinite(tara, model, bad):
    N = 64
    if model == "com":
        m, kw, st = tara.MODEL_COM, com_kw(), I.com_random_phase(N, N, seed=5)
    else:
        m, kw, st = tara.MODEL_COH, coh_kw(), I.coh_random_phase(N, N, seed=5)
    with tara.Session(m, N, N, tara.Params.make(**kw)) as s:
        s.set_state(st)
        bad_st = [a.copy() for a in st]
        bad_st[-1][7, 3] = complex(bad, 0.0)
        with pytest.raises(tara.TaraError) as ei:
            s.set_state(bad_st)
        assert ei.value.status == tara.ENAN
        with pytest.raises(tara.TaraError) as ei:
            s.set_history(bad_st)
        assert ei.value.status == tara.ENAN


def test_overflow_while_stepping_is_reported(tara, oracle):
    N = 64
    kw = com_kw()
    st = I.com_random_phase(N, N, seed=6)
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**kw)) as s:
        s.set_state([a * 1e300 for a in st])  # finite, but its fluxes overflow
        s.step(tara.STEP_RK4, 2)
        with pytest.raises(tara.TaraError) as ei:
            s.synchronize()
        assert ei.value.status == tara.ENAN
        # the session works again with a sound state
        s.set_state(st)
        s.step(tara.STEP_RK4, 1)
        s.synchronize()
        got = s.get_state()
    ref = oracle.rk4com(N, N, oracle_com_params(oracle, kw), st)
    for g, r in zip(got, ref):
        assert rel_l2(g, r) <= 1e-10


def test_bounded_wait_runs_out(tara, oracle):
    st, waited = tara.selftest_bounded_wait(1_000_000)  # 1 ms
    assert st == tara.ETIMEOUT, (st, tara.last_error())
    assert 1_000_000 <= waited < 1_000_000_000, waited
    # the context is still usable: a RHS against the oracle (compressive
    # noise, so that d(rho)/dt is not rounding noise)
    N = 64
    kw = com_kw()
    s0 = compressive(I.com_random_phase(N, N, seed=8), 8)
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**kw)) as s:
        s.set_wait_limit(2_000_000_000)
        s.set_state(s0)
        got = s.rhs()
    ref = oracle.derive2com(N, N, oracle_com_params(oracle, kw), s0)
    for g, r in zip(got, ref):
        assert rel_l2(g, r) <= 1e-10
    assert tara.selftest_bounded_wait(10)[0] == tara.EINVAL
