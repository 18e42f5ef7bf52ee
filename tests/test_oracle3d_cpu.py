"""The oracle's 3D MHD restatement (derive3com / ab3com, src/derive3com.f95:5-1047,
src/ab3com.f95:6-66) against an independent numpy restatement with numpy's FFT,
plus known answers: a uniform state has a zero RHS, the k = 0 modes of mass,
momentum and B never change, ab3com leaves E as it is."""
import numpy as np
import pytest

from oracle import pyoracle as O
from tara2d_b200 import initial

PI = O.PI


def params(dt=1e-4):
    return O.Com3Params(Lx=2 * PI, Ly=2 * PI, Lz=2 * PI, mu=0.01, CS=10.0, eta=0.005, dt=dt)


def state3(Nx, Ny, Nz, seed=0, noise=1e-3):
    """Smooth fields + small broadband noise, as spectra (Nz, Ny, Nx/2+1)."""
    return initial.mhd3_state(Nx, Ny, Nz, seed=seed, noise=noise)


def wavenumbers(Nx, Ny, Nz, P, pi=PI):
    Nh = Nx // 2 + 1
    kx = np.array([2.0 * pi * i / P.Lx for i in range(Nh)])
    ky = np.array([2.0 * pi * (j if j < Ny // 2 else j - Ny) / P.Ly for j in range(Ny)])
    kz = np.array([2.0 * pi * (k if k < Nz // 2 else k - Nz) / P.Lz for k in range(Nz)])
    return np.meshgrid(kz, ky, kx, indexing="ij")[::-1]  # KX, KY, KZ on (Nz, Ny, Nh)


def np_derive3com(Nx, Ny, Nz, P, st, pi=PI):
    """numpy restatement of src/derive3com.f95 (FFT: numpy's pocketfft)."""
    s, ax = (Nz, Ny, Nx), (0, 1, 2)
    c2r = lambda a: np.fft.irfftn(a, s=s, axes=ax)  # normalised like the reference's c2r / (Nx Ny Nz)
    r2c = lambda a: np.fft.rfftn(a, axes=ax)
    KX, KY, KZ = wavenumbers(Nx, Ny, Nz, P, pi)
    rho, rux, ruy, ruz, E, Bx, By, Bz = [c2r(a) for a in st]
    ux, uy, uz = rux / rho, ruy / rho, ruz / rho
    uk = [r2c(ux), r2c(uy), r2c(uz)]
    ik = lambda k, a: 1j * k * a
    dux = c2r(ik(KX, uk[0]))
    duy = c2r(ik(KY, uk[1]))
    duz = c2r(ik(KZ, uk[2]))
    dBx_dy, dBx_dz = c2r(ik(KY, st[5])), c2r(ik(KZ, st[5]))
    dBy_dx, dBy_dz = c2r(ik(KX, st[6])), c2r(ik(KZ, st[6]))
    dBz_dx, dBz_dy = c2r(ik(KX, st[7])), c2r(ik(KY, st[7]))
    cxB, cyB, czB = dBz_dy - dBy_dz, dBz_dx - dBx_dz, dBy_dx - dBx_dy
    B2 = Bx * Bx + By * By + Bz * Bz
    Pp = P.CS * P.CS * rho
    H = E + Pp + B2 / 2
    Mx = [rux * ux + Pp + B2 / 2 - Bx * Bx, rux * uy - Bx * By, rux * uz - Bx * Bz]
    My = [rux * uy - Bx * By, ruy * uy + Pp + B2 / 2 - By * By, ruy * uz - By * Bz]
    Mz = [ruz * ux - Bz * Bx, ruz * uy - Bz * By, ruz * uz + Pp + B2 / 2 - Bz * Bz]
    En = [H * ux - ux * Bx * Bx - uy * Bx * By - uz * Bx * Bz - P.eta * (By * czB + Bz * cyB),
          H * uy - ux * Bx * By - uy * By * By - uz * By * Bz + P.eta * (Bx * czB - Bz * cxB),
          H * uz - ux * Bz * Bx - uy * Bz * By - uz * Bz * Bz + P.eta * (Bx * cyB + By * cxB)]
    EV = (dux + duy + duz) ** 2
    Mag = [ux * By - uy * Bx, ux * Bz - uz * Bx, uy * Bz - uz * By]
    K = (KX, KY, KZ)
    div = lambda F: sum(ik(K[c], r2c(F[c])) for c in range(3))
    k2 = KX * KX + KY * KY + KZ * KZ
    mask = np.sqrt(k2) < ((Nx + Ny + Nz) / 3.0) / 3.0
    mg = [r2c(m) for m in Mag]
    out = [-(ik(KX, st[1]) + ik(KY, st[2]) + ik(KZ, st[3])),
           -div(Mx) - k2 * uk[0] / 450.0,
           -div(My) - k2 * uk[1] / 450.0,
           -div(Mz) - k2 * uk[2] / 450.0,
           -div(En) + P.mu * r2c(EV),
           (ik(KY, mg[0]) + ik(KZ, mg[1])) - k2 * st[5] / 450.0,
           -(ik(KX, mg[0]) - ik(KZ, mg[2])) - k2 * st[6] / 450.0,
           -(ik(KX, mg[1]) + ik(KY, mg[2])) - k2 * st[7] / 450.0]
    return [np.where(mask, o, 0) for o in out]


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("Nx,Ny,Nz", [(16, 16, 16), (16, 8, 32), (32, 16, 8)])
def test_derive3com_matches_numpy(Nx, Ny, Nz):
    P = params()
    st = state3(Nx, Ny, Nz, seed=Nx + Ny + Nz)
    got = O.derive3com(Nx, Ny, Nz, P, st)
    ref = np_derive3com(Nx, Ny, Nz, P, st)
    for q in range(8):
        assert rel(got[q], ref[q]) <= 1e-12, (q, rel(got[q], ref[q]))


def test_derive3com_matches_numpy_unequal_box():
    """Lx, Ly, Lz all different (wavenumbers 2 pi i / L per direction)."""
    Nx, Ny, Nz = 16, 32, 16
    P = O.Com3Params(Lx=2 * PI, Ly=4 * PI, Lz=PI, mu=0.02, CS=5.0, eta=0.01, dt=1e-4)
    st = state3(Nx, Ny, Nz, seed=9)
    got = O.derive3com(Nx, Ny, Nz, P, st)
    ref = np_derive3com(Nx, Ny, Nz, P, st)
    for q in range(8):
        assert rel(got[q], ref[q]) <= 1e-12, (q, rel(got[q], ref[q]))


def test_uniform_state_has_zero_rhs():
    N = 16
    Nh = N // 2 + 1
    st = [np.zeros((N, N, Nh), complex) for _ in range(8)]
    NN = N ** 3
    st[0][0, 0, 0] = 1.0 * NN
    st[4][0, 0, 0] = 5.0 * NN
    st[5][0, 0, 0] = 0.3 * NN
    st[7][0, 0, 0] = -0.2 * NN
    d = O.derive3com(N, N, N, params(), st)
    assert all(np.abs(a).max() == 0 for a in d)


def test_ab3com_keeps_E_and_the_mean_modes():
    N = 16
    P = params(dt=2e-4)
    st0 = state3(N, N, N, seed=3)
    st, hist = O.run3com(N, N, N, P, 3, st0)
    assert np.array_equal(st[4], st0[4])  # E_k_new = E_k (src/ab3com.f95:52)
    for q in (0, 1, 2, 3, 5, 6, 7):  # k = 0: every divergence and k^2 term vanishes
        assert st[q][0, 0, 0] == st0[q][0, 0, 0]
    assert not all(np.array_equal(st[q], st0[q]) for q in (0, 1, 5))


def test_ab3com_formula():
    N = 8
    rng = np.random.default_rng(1)
    shape = (N, N, N // 2 + 1)
    z = lambda: rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    u, dn, do = [z() for _ in range(8)], [z() for _ in range(8)], [z() for _ in range(8)]
    out = O.ab3com(N, N, N, 1e-3, u, do, dn)
    for q in range(8):
        ref = u[q] if q == 4 else u[q] + (1.5 * dn[q] - 0.5 * do[q]) * 1e-3
        assert np.array_equal(out[q], ref)


@pytest.mark.parametrize("N", [16, 32])
def test_bench_mask_share_matches_the_oracle(N):
    """The unmasked share f in bench.py's 3D byte model is the share of modes
    the oracle's RHS does not zero (the momentum RHS is nonzero on every kept
    mode except k = 0, where its divergence and k^2 terms vanish)."""
    import bench
    d = O.derive3com(N, N, N, params(), state3(N, N, N, seed=N))
    nonzero = np.count_nonzero(d[1])
    assert nonzero + 1 == round(bench.mhd3_unmasked_fraction(N) * d[1].size)
