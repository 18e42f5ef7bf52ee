"""Real-space state, vorticity, initial conditions set on the device, and the
drivers' output files, against the oracle's FFTW transforms.

Tolerances (FP64): relative L2 <= 1e-13 for transforms of the state; the grid
files print 17 significant digits, so their columns match to <= 1e-15."""
import os

import numpy as np
import pytest

from tests.gpu_common import com_kw, coh_kw, oracle_com_params, rel_l2
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("Nx,Ny", [(64, 64), (128, 32), (384, 384)])
def test_state_real_round_trip(tara, oracle, Nx, Ny):
    st = I.com_random_phase(Nx, Ny, seed=2)
    with tara.Session(tara.MODEL_COM, Nx, Ny, tara.Params.make(**com_kw())) as s:
        s.set_state(st)
        real = s.get_state_real()
        for r, a in zip(real, st):
            ref = oracle.c2r_2d(a, Nx) / (Nx * Ny)
            assert rel_l2(r, ref) <= 1e-13
        s.set_state_real([2.0 * r for r in real])
        back = s.get_state()
    for b, a in zip(back, st):
        ref = oracle.r2c_2d(2.0 * oracle.c2r_2d(a, Nx) / (Nx * Ny))
        assert rel_l2(b, ref) <= 1e-13


def test_orszag_tang_from_real_fields(tara):
    """The MHD initial state set from real-space fields on the device equals
    the host-transformed one (the reference's IC path)."""
    N = 128
    x = np.arange(N) * 2 * np.pi / N
    X, Y = np.meshgrid(x, x)
    rho = np.ones((N, N))
    ux, uy, bx, by = -np.sin(Y), np.sin(X), -np.sin(Y), np.sin(2 * X)
    ref = I.com_state(rho, ux, uy, bx, by, CS=100.0)
    P = 100.0 ** 2 * rho
    E = P / (5.0 / 3.0 - 1.0) + 0.5 * rho * (ux ** 2 + uy ** 2) + 0.5 * (bx ** 2 + by ** 2)
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**com_kw())) as s:
        s.set_state_real([rho, rho * ux, rho * uy, E, bx, by])
        got = s.get_state()
    for g, r in zip(got, ref):
        assert rel_l2(g, r) <= 1e-13


@pytest.mark.parametrize("model", ["coh", "com"])
def test_vorticity(tara, oracle, model):
    N = 64
    if model == "coh":
        st = I.coh_random_phase(N, N, seed=5)
        kw, m = coh_kw(), tara.MODEL_COH
        uxk, uyk = st[1], st[2]
    else:
        st = I.com_random_phase(N, N, seed=5)
        kw, m = com_kw(), tara.MODEL_COM
        rho = oracle.c2r_2d(st[0], N) / N ** 2
        uxk = oracle.r2c_2d(oracle.c2r_2d(st[1], N) / N ** 2 / rho)
        uyk = oracle.r2c_2d(oracle.c2r_2d(st[2], N) / N ** 2 / rho)
    k = np.fft.fftfreq(N, 1.0 / N)
    KX, KY = np.meshgrid(k[:N // 2 + 1], k)
    KX[:, -1] = N // 2  # the kx Nyquist column carries +N/2
    ref = oracle.c2r_2d(1j * KX * uyk - 1j * KY * uxk, N) / N ** 2
    with tara.Session(m, N, N, tara.Params.make(**kw)) as s:
        s.set_state(st)
        got = s.get_vorticity_real()
    assert rel_l2(got, ref) <= 1e-13


def test_grid_file_mhd(tara, oracle, tmp_path):
    N = 32
    kw = com_kw()
    st = I.com_random_phase(N, N, seed=8)
    path = str(tmp_path / "fort.00100000")
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**kw)) as s:
        s.set_state(st)
        s.write_snapshot(path)
    d = np.loadtxt(path, converters=None)
    assert d.shape == (N * N, 9)
    real = [oracle.c2r_2d(a, N) / N ** 2 for a in st]
    # x outer, y inner: line i*N + j holds grid point (x_i, y_j)
    i, j = np.divmod(np.arange(N * N), N)
    dx = 2 * np.pi / N
    assert np.array_equal(d[:, 0], i * dx) and np.array_equal(d[:, 1], j * dx)
    rho = real[0][j, i]
    cols = [rho, real[1][j, i] / rho, real[2][j, i] / rho, 100.0 ** 2 * rho, real[3][j, i], real[4][j, i],
            real[5][j, i]]
    for c, ref in zip(d[:, 2:].T, cols):
        assert rel_l2(c, ref) <= 1e-13


def test_driver_files(tara, oracle, tmp_path):
    from tara2d_b200 import driver
    N = 64
    kw = com_kw(dt=5e-5)
    st = I.com_orszag_tang(N, N, seed=1)
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**kw)) as s:
        s.set_state(st)
        recs = driver.run(s, tara.STEP_RK4, 40, 10, str(tmp_path), snapshot_every=20)
    e = np.loadtxt(tmp_path / "Energy.dat")
    assert e.shape == (5, 6)
    assert np.allclose(e[:, 0], np.arange(5) * 10 * 5e-5, rtol=0, atol=1e-15)
    ref = oracle.diag_com(N, N, oracle_com_params(oracle, kw), st)
    assert abs(e[0, 1] - ref[0]) <= 1e-12 * ref[0] and abs(e[0, 2] - ref[1]) <= 1e-12 * ref[1]
    assert sorted(os.listdir(tmp_path)) == ["Cross_Helicity.dat", "Energy.dat", "Energy_Spectra.dat",
                                            "fort.00100000", "fort.00100020", "fort.00100040"]
    h = np.loadtxt(tmp_path / "Cross_Helicity.dat")
    assert np.allclose(h[:, 1], [r[1][5] for r in recs], rtol=1e-15)
    sp = np.loadtxt(tmp_path / "Energy_Spectra.dat")
    assert sp.shape[1] == 3 and sp.shape[0] == 5 * len(recs[0][2])
