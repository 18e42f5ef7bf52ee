"""Binary checkpoint / restart through the C ABI (tara_checkpoint_write /
tara_checkpoint_read).

A run checkpointed after k steps and restored into a fresh session continues
as the uninterrupted run: exactly for hydro (AB2 needs the stored history);
for MHD to rounding (relative L2 <= 1e-13 after 4 RK4 steps), because the
first RHS after a restore does the y-inverse of its input in the separate
column-inverse pass, whose FFT factorisation differs from the one fused into
the stepping column pass.  Files written by the library and by the host
module tara2d_b200.checkpoint are read by the other."""
import numpy as np
import pytest

from tests.gpu_common import coh_kw, com_kw, rel_l2
from tara2d_b200 import checkpoint as ck
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu


def test_hydro_ab2_restart_is_exact(tara, tmp_path):
    N = 64
    kw = coh_kw()
    p = tmp_path / "h.ck"
    with tara.Session(tara.MODEL_COH, N, N, tara.Params.make(**kw)) as s:
        s.set_state(I.coh_random_phase(N, N, seed=3))
        s.step(tara.STEP_AB2, 5)
        s.checkpoint(str(p), step=5, time=5 * kw["dt"])
        s.step(tara.STEP_AB2, 4)
        ref = s.get_state()
    other = dict(kw, dt=kw["dt"] * 3)  # the restore brings back dt as well
    with tara.Session(tara.MODEL_COH, N, N, tara.Params.make(**other)) as s:
        assert s.restore(str(p)) == (5, 5 * kw["dt"])
        assert s.params.dt == kw["dt"]
        s.step(tara.STEP_AB2, 4)
        got = s.get_state()
    for a, b in zip(got, ref):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("prec", [0, 1])
def test_mhd_rk4_restart(tara, tmp_path, prec):
    N = 64
    p = tmp_path / "m.ck"
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**com_kw()), precision=prec) as s:
        s.set_state(I.com_orszag_tang(N, N, seed=1))
        s.step(tara.STEP_RK4, 3)
        s.checkpoint(str(p), step=3, time=0.5)
        s.step(tara.STEP_RK4, 4)
        ref = s.get_state()
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**com_kw(eta=1e-2)), precision=prec) as s:
        assert s.restore(str(p)) == (3, 0.5)
        assert s.params.eta == com_kw()["eta"]
        s.step(tara.STEP_RK4, 4)
        got = s.get_state()
    tol = 1e-13 if prec == 0 else 1e-6
    for a, b in zip(got, ref):
        assert rel_l2(a, b) <= tol


def test_library_file_matches_host_reader(tara, tmp_path):
    N = 32
    p = tmp_path / "r.ck"
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**com_kw(fix_curlB=1))) as s:
        s.set_state(I.com_random_phase(N, N, seed=5))
        s.step(tara.STEP_AB2, 2)
        s.checkpoint(str(p), step=2, time=1e-4)
        st, hi = s.get_state(), s.get_history()
    r = ck.read(p)
    assert (r["model"], r["precision"], r["Nx"], r["Ny"], r["nf"], r["fix_curlB"]) == (tara.MODEL_COM, 0, N, N, 6, 1)
    assert (r["step"], r["time"]) == (2, 1e-4)
    assert r["params"]["mu"] == com_kw()["mu"] and r["params"]["CS"] == com_kw()["CS"]
    for a, b in zip(r["state"] + r["history"], st + hi):
        assert np.array_equal(a, b)


def test_host_written_file_restores(tara, tmp_path):
    N = 32
    kw = coh_kw()
    st = I.coh_random_phase(N, N, seed=9)
    hi = [0.5 * a for a in I.coh_random_phase(N, N, seed=10)]
    p = tmp_path / "w.ck"
    ck.write(p, tara.MODEL_COH, 0, N, N, st, hi, step=40, time=4e-3,
             params={k: kw[k] for k in ("Lx", "Ly", "pi", "dt", "mux", "muy", "ms", "CS")})
    with tara.Session(tara.MODEL_COH, N, N, tara.Params.make(**kw)) as s:
        assert s.restore(str(p)) == (40, 4e-3)
        for a, b in zip(s.get_state() + s.get_history(), st + hi):
            assert np.array_equal(a, b)


def test_restore_errors(tara, tmp_path):
    N = 32
    p = tmp_path / "x.ck"
    with tara.Session(tara.MODEL_COH, N, N, tara.Params.make(**coh_kw())) as s:
        s.set_state(I.coh_random_phase(N, N, seed=1))
        s.checkpoint(str(p))
        with pytest.raises(tara.TaraError, match="cannot open"):
            s.restore(str(tmp_path / "missing.ck"))
        raw = bytearray(p.read_bytes())
        raw[5000] ^= 1
        (tmp_path / "bad.ck").write_bytes(bytes(raw))
        with pytest.raises(tara.TaraError, match="checksum"):
            s.restore(str(tmp_path / "bad.ck"))
    with tara.Session(tara.MODEL_COH, 64, N, tara.Params.make(**coh_kw())) as s:
        with pytest.raises(tara.TaraError, match="grid"):
            s.restore(str(p))
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**com_kw())) as s:
        with pytest.raises(tara.TaraError, match="grid"):
            s.restore(str(p))


def test_fp64_checkpoint_into_fp32_session(tara, tmp_path):
    N = 64
    p = tmp_path / "c.ck"
    st = I.com_orszag_tang(N, N, seed=2)
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**com_kw())) as s:
        s.set_state(st)
        s.checkpoint(str(p))
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**com_kw()), precision=1) as s:
        s.restore(str(p))
        for a, b in zip(s.get_state(), st):
            assert rel_l2(a, b) <= 1e-7
