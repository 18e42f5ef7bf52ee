"""Pins the CPU oracle: against the reference's FFTW fixtures, an independent
numpy restatement, and analytic known answers (no GPU needed)."""
import os

import numpy as np
import pytest

from tests import numpy_ref as R
from tara2d_b200 import initial as I

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def coh_params(O, **kw):
    d = dict(Lx=2 * O.PI, Ly=2 * O.PI, mux=1e-3, muy=1e-3, ms=1.0, CS=3.77, dt=1e-4)
    d.update(kw)
    return O.CohParams(**d)


def com_params(O, fix=0, **kw):
    d = dict(Lx=2 * O.PI, Ly=2 * O.PI, spheat=5.0 / 3.0, mu=5e-4, ms=1.0, CS=100.0, mu_0=1.0, eta=5e-4,
             dt=5e-5, kf=1.0, A=0.0, fix_curlB=fix)
    d.update(kw)
    return O.ComParams(**d)


def test_fftw_fixture_reproduced(oracle):
    g = np.load(os.path.join(GOLD, "fftw_16x12.npz"))
    assert np.array_equal(oracle.r2c_2d(g["real_in"]), g["r2c_out"])
    assert np.array_equal(oracle.c2r_2d(g["spec_in"], 16), g["c2r_out"])


def test_fftw_c2r_semantics_non_hermitian(oracle):
    """FFTW's 2D c2r = complex inverse along y of every column, then c2r
    along x keeping only Re of the kx=0 and Nyquist bins."""
    g = np.load(os.path.join(GOLD, "fftw_16x12.npz"))
    np.testing.assert_allclose(R.c2r(g["spec_in"], 16), g["c2r_out"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(np.fft.rfft2(g["real_in"]), g["r2c_out"], atol=1e-12, rtol=0)


def test_golden_rhs_reproduced(oracle):
    g = np.load(os.path.join(GOLD, "derive2coh_16.npz"))
    d = oracle.derive2coh(16, 16, coh_params(oracle), g["nk"], g["ukx"], g["uky"])
    for a, k in zip(d, ("dn", "dux", "duy")):
        assert np.array_equal(a, g[k])
    g = np.load(os.path.join(GOLD, "derive2com_16.npz"))
    d = oracle.derive2com(16, 16, com_params(oracle), list(g["state"]))
    for a, b in zip(d, g["rhs"]):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("Nx,Ny", [(16, 16), (32, 32), (64, 32), (32, 64)])
def test_derive2coh_vs_numpy(oracle, Nx, Ny):
    st = I.coh_random_phase(Nx, Ny, seed=Nx + Ny)
    d = oracle.derive2coh(Nx, Ny, coh_params(oracle), *st)
    dn = R.derive2coh(Nx, Ny, dict(Lx=2 * oracle.PI, Ly=2 * oracle.PI, mux=1e-3, muy=1e-3, CS=3.77), *st)
    for a, b in zip(d, dn):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


def test_derive2coh_non_hermitian_input(oracle):
    rng = np.random.default_rng(5)
    Nx = Ny = 16
    st = [rng.standard_normal((Ny, 9)) + 1j * rng.standard_normal((Ny, 9)) for _ in range(3)]
    st[0][0, 0] += 40 * Nx * Ny
    d = oracle.derive2coh(Nx, Ny, coh_params(oracle), *st)
    dn = R.derive2coh(Nx, Ny, dict(Lx=2 * oracle.PI, Ly=2 * oracle.PI, mux=1e-3, muy=1e-3, CS=3.77), *st)
    for a, b in zip(d, dn):
        assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max()


@pytest.mark.parametrize("fix", [0, 1])
def test_derive2com_vs_numpy(oracle, fix):
    sm = I.com_orszag_tang(32, 32, seed=1)
    d = oracle.derive2com(32, 32, com_params(oracle, fix), sm)
    dn = R.derive2com(32, 32, dict(Lx=2 * oracle.PI, Ly=2 * oracle.PI, mu=5e-4, eta=5e-4, CS=100.0,
                                   fix_curlB=fix, A=0.0, kf=1.0), sm)
    for a, b in zip(d, dn):
        scale = max(np.abs(b).max(), 1e-300)
        assert np.abs(a - b).max() <= 1e-10 * scale


def test_derive2com_forcing_grid(oracle):
    sm = I.com_orszag_tang(16, 16, seed=2)
    P = com_params(oracle, A=0.3, kf=1.0)
    d = oracle.derive2com(16, 16, P, sm)
    dn = R.derive2com(16, 16, dict(Lx=2 * oracle.PI, Ly=2 * oracle.PI, mu=5e-4, eta=5e-4, CS=100.0,
                                   fix_curlB=0, A=0.3, kf=1.0), sm)
    for a, b in zip(d, dn):
        assert np.abs(a - b).max() <= 1e-10 * max(np.abs(b).max(), 1e-300)


def test_viscous_decay_single_mode(oracle):
    """Nonlinearity off (a single uniform-density shear mode u=(A sin 3y, 0)
    has u.grad u = 0): du/dt = -nu k^2 u exactly on the retained mode."""
    Nx = Ny = 32
    X, Y = I.grid(Nx, Ny)
    A = 0.1
    st = [np.fft.rfft2(np.ones((Ny, Nx))), np.fft.rfft2(A * np.sin(3 * Y)), np.fft.rfft2(0 * X)]
    P = coh_params(oracle, mux=2e-3, muy=2e-3, CS=1.0)
    d = oracle.derive2coh(Nx, Ny, P, *st)
    np.testing.assert_allclose(d[1], -2e-3 * 9.0 * st[1], atol=1e-12 * Nx * Ny)
    assert np.abs(d[0]).max() < 1e-10 and np.abs(d[2]).max() < 1e-10


def test_mhd_mass_conservation(oracle):
    sm = I.com_orszag_tang(32, 32, seed=3)
    st, _ = oracle.run_com(32, 32, com_params(oracle), 1, 5, sm)
    assert abs(st[0][0, 0] - sm[0][0, 0]) <= 1e-12 * abs(sm[0][0, 0])


def test_mask_integer_form():
    """The host cut-off table equals the integer form 36(kx^2+ky^2) >= (Nx+Ny)^2
    for every configured N (the FP64 formula has no near-ties there)."""
    for N in (128, 256, 384, 512, 1024, 2048, 4096):
        kx = np.arange(N // 2 + 1)
        ky = np.where(np.arange(N) < N // 2, np.arange(N), np.arange(N) - N)
        KX, KY = np.meshgrid(kx, ky)
        KXf = 2.0 * I.PI * KX / (2 * I.PI)
        KYf = 2.0 * I.PI * KY.astype(float) / (2 * I.PI)
        fp = np.sqrt(KXf * KXf + KYf * KYf) >= ((N + N) / 2.0) / 3.0
        it = 36 * (KX * KX + KY * KY) >= (2 * N) ** 2
        assert np.array_equal(fp, it), N


def test_bug_compatible_rk4_pc_are_euler_like(oracle):
    Nx = Ny = 16
    st = I.coh_random_phase(Nx, Ny, seed=9)
    P = coh_params(oracle)
    d = oracle.derive2coh(Nx, Ny, P, *st)
    for w in range(3):
        r = oracle.rk42coh(w, Nx, Ny, P, st, d)
        np.testing.assert_allclose(r, st[w] + P.dt * d[w], rtol=1e-14, atol=1e-14 * np.abs(st[w]).max())
        p = oracle.pc2coh(w, Nx, Ny, P, st, d)
        np.testing.assert_allclose(p, st[w] + P.dt * d[w], rtol=1e-14, atol=1e-14 * np.abs(st[w]).max())
