"""Full runs of the benchmark configurations against the oracle's own runs
(fixtures made by tests/golden/make_runs.py from the C restatement of the
reference over its FFTW; the reference's drivers record the same quantities:
src/main2coh.f95:266-431, src/main2com.f95:352-623).

Tolerances (FP64 path): every recorded diagnostic within 1e-6 relative over
the whole run, E(k) within 1e-6 (relative L2 over the shells) at every
record, fields (the modes |kx|, |ky| <= 32) within 1e-10 relative L2 after
100 steps; quantities that are rounding noise around zero (hydro C1 = <omega>,
MHD <div B>) to an absolute bound.  The 4096^2 FP32 run is compared with the
same FP64 oracle run at the tolerances of the precision mode."""
import os

import numpy as np
import pytest

from tests.gpu_common import coh_kw, com_kw, rel_l2
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def low_modes(fields, K=32):
    out = []
    for a in fields:
        Ny = a.shape[0]
        out.append(a[np.r_[0:K + 1, Ny - K:Ny], :K + 1])
    return np.array(out)


def rel_fields(got, ref):
    return max(rel_l2(g, r) for g, r in zip(got, ref))


def test_config1_hydro_128_ab2_1000_steps(tara):
    """128^2 hydro, AB2, dt = 1e-4, nu = 1e-3, 1000 steps, Energy.dat values
    after every step (src/main2coh.f95:428-429)."""
    fx = np.load(os.path.join(GOLD, "run_coh128_ab2.npz"))
    N, nsteps, ek_every = int(fx["N"]), int(fx["nsteps"]), int(fx["ek_every"])
    kw = coh_kw(dt=float(fx["dt"]), mux=float(fx["nu"]), muy=float(fx["nu"]), CS=float(fx["CS"]))
    st0 = I.coh_random_phase(N, N, seed=int(fx["seed"]))
    with tara.Session(tara.MODEL_COH, N, N, tara.Params.make(**kw)) as s:
        s.set_state(st0)
        vals, eks = s.run_recorded(tara.STEP_AB2, 1, nsteps + 1)
        final = s.get_state()
    ref = fx["diag"]
    rel = np.abs(vals[:, [0, 1, 2, 4, 5]] - ref[:, [0, 1, 2, 4, 5]]) / np.abs(ref[:, [0, 1, 2, 4, 5]])
    assert rel.max() <= 1e-6, rel.max(axis=0)
    scale = np.sqrt(ref[:, 4])
    assert np.all(np.abs(vals[:, 3] - ref[:, 3]) <= 1e-12 * scale)
    for k in range(ref.shape[0] // ek_every + 1):
        assert rel_l2(eks[k * ek_every], fx["ek"][k]) <= 1e-6, k
    assert rel_fields(low_modes(final), fx["final_low"]) <= 1e-10


def _com_records(tara, N, kw, st0, every, nrec_parts, precision):
    """Records every `every` RK4 steps, run in parts of nrec_parts[i] records
    after the first; returns (vals, eks, states after each part)."""
    vals, eks, states = [], [], []
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**kw), precision=precision) as s:
        s.set_state(st0)
        for i, n in enumerate(nrec_parts):
            v, e = s.run_recorded(tara.STEP_RK4, every, n + 1)
            vals.append(v if i == 0 else v[1:])
            eks.append(e if i == 0 else e[1:])
            states.append(s.get_state())
    return np.concatenate(vals), np.concatenate(eks), states


def _check_com_diag(vals, eks, fx, rtol, rtol_w2=None, ek_tol=None):
    ref = fx["diag"]
    q = [0, 1, 2, 3, 5]  # energy, <B^2>, <omega^2>, <j^2>, <u.B>
    rel = np.abs(vals[:, q] - ref[:, q]) / np.abs(ref[:, q])
    lim = np.full(len(q), rtol)
    if rtol_w2 is not None:
        lim[2] = rtol_w2
    assert np.all(rel.max(axis=0) <= lim), rel.max(axis=0)
    assert np.all(np.abs(vals[:, 4] - ref[:, 4]) <= 1e-10)
    for k in range(ref.shape[0]):
        assert rel_l2(eks[k], fx["ek"][k]) <= (ek_tol or rtol), k
    return rel.max(axis=0)


def test_config2_mhd_1024_rk4_2000_steps(tara):
    """1024^2 MHD (perturbed Orszag-Tang), RK4, dt = 5e-5, nu = eta = 5e-4,
    2000 steps, diagnostics every 100 (the Energy.dat cadence of
    src/main2com.f95:615-617, plus <u.B> and E(k))."""
    fx = np.load(os.path.join(GOLD, "run_com1024_rk4.npz"))
    N, every, nsteps = int(fx["N"]), int(fx["every"]), int(fx["nsteps"])
    kw = com_kw(dt=float(fx["dt"]), mu=float(fx["mu"]), eta=float(fx["eta"]), CS=float(fx["CS"]))
    st0 = I.com_orszag_tang(N, N, seed=int(fx["seed"]))
    vals, eks, states = _com_records(tara, N, kw, st0, every, [1, nsteps // every - 1], tara.FP64)
    _check_com_diag(vals, eks, fx, 1e-6)
    steps = list(fx["field_steps"])
    assert steps == [100, 2000]
    assert rel_fields(low_modes(states[0]), fx["fields_low"][0]) <= 1e-10
    assert rel_fields(low_modes(states[1]), fx["fields_low"][1]) <= 1e-8


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_config5_mhd_4096_rk4_first_50_steps_vs_fp64_oracle(tara, prec):
    """4096^2 MHD, nu = eta = 2e-5, E(k) ~ k^4 exp(-(k/6)^2), dt = 1.5e-5
    (below the acoustic CFL limit), the first 50 RK4 steps against the FP64
    oracle: FP64 to the FP64 tolerances; FP32 bulk (FP64 reductions) with
    fields within 2e-4, energy, <B^2>, <j^2>, <u.B> and E(k) within 1e-5 and
    <omega^2> within 1e-4."""
    fx = np.load(os.path.join(GOLD, "run_com4096_rk4.npz"))
    N, every, nsteps = int(fx["N"]), int(fx["every"]), int(fx["nsteps"])
    kw = com_kw(dt=float(fx["dt"]), mu=float(fx["mu"]), eta=float(fx["eta"]), CS=float(fx["CS"]))
    st0 = I.com_random_phase(N, N, seed=int(fx["seed"]), k0=float(fx["k0"]))
    fp64 = prec == "fp64"
    vals, eks, states = _com_records(tara, N, kw, st0, every, [1, nsteps // every - 1],
                                     tara.FP64 if fp64 else tara.FP32)
    if fp64:
        rel = _check_com_diag(vals, eks, fx, 1e-9)
        ftol, ntol = 1e-10, 1e-10
    else:
        rel = _check_com_diag(vals, eks, fx, 1e-5, rtol_w2=1e-4)
        ftol, ntol = 2e-4, 1e-4
    assert list(fx["field_steps"]) == [10, 50]
    e10 = rel_fields(low_modes(states[0]), fx["fields_low"][0])
    e50 = rel_fields(low_modes(states[1]), fx["fields_low"][1])
    norms = np.array([np.vdot(a, a).real for a in states[1]])
    en = np.max(np.abs(norms - fx["final_norm2"]) / fx["final_norm2"])
    print(f"4096^2 {prec} vs FP64 oracle: diag rel {rel}, fields@10 {e10:.2e}, fields@50 {e50:.2e}, "
          f"|field|^2@50 {en:.2e}")
    assert e10 <= ftol and e50 <= ftol, (e10, e50)
    assert en <= ntol, en
