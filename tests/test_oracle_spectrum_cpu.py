"""The oracle's shell spectrum E(k) against independent facts (CPU only):
Parseval (sum_k E(k) = <|u|^2>/2 from the real-space diagnostics) and a single
Fourier mode landing in its shell."""
import numpy as np

from tara2d_b200 import initial as I

PI = 3.14159265358979323846


def test_spectrum_sums_to_half_energy_com(oracle):
    Nx, Ny = 64, 48
    P = oracle.ComParams(Lx=2 * PI, Ly=2 * PI, spheat=5 / 3, mu=5e-4, ms=1.0, CS=100.0, mu_0=1.0, eta=5e-4,
                         dt=5e-5, kf=1.0, A=0.0, fix_curlB=0)
    st = I.com_random_phase(Nx, Ny, seed=3)
    ek = oracle.spectrum_com(Nx, Ny, P, st)
    d = oracle.diag_com(Nx, Ny, P, st)
    assert ek.size == oracle.num_shells(Nx, Ny)
    assert abs(ek.sum() - d[0] / 2) <= 1e-13 * d[0]


def test_spectrum_sums_to_half_energy_coh(oracle):
    Nx = Ny = 64
    P = oracle.CohParams(Lx=2 * PI, Ly=2 * PI, mux=1e-3, muy=1e-3, ms=1.0, CS=3.77, dt=1e-4)
    st = I.coh_random_phase(Nx, Ny, seed=8)
    ek = oracle.spectrum_coh(Nx, Ny, P, st[1], st[2])
    d = oracle.diag_coh(Nx, Ny, P, st)
    assert abs(ek.sum() - d[0]) <= 1e-13 * d[0]  # d[0] is Energy/(2 NxNy) = <|u|^2>/2


def test_single_mode_shell(oracle):
    Nx = Ny = 32
    P = oracle.CohParams(Lx=2 * PI, Ly=2 * PI, mux=0, muy=0, ms=1.0, CS=1.0, dt=1e-4)
    y, x = np.meshgrid(np.arange(Ny) * 2 * PI / Ny, np.arange(Nx) * 2 * PI / Nx, indexing="ij")
    ux = np.cos(3 * x + 4 * y)  # |k| = 5, <ux^2> = 1/2
    uxk = oracle.r2c_2d(ux)
    ek = oracle.spectrum_coh(Nx, Ny, P, uxk, np.zeros_like(uxk))
    assert abs(ek[5] - 0.25) < 1e-14
    assert abs(ek.sum() - 0.25) < 1e-14
