"""Host restatement of the counter-based seeded initial conditions
(tara2d_b200.initial.hashed_*): known answer of the splitmix64 finaliser,
uniform range, and the properties of the states it builds.  The device
generator is compared with it in tests/test_ic_gpu.py."""
import numpy as np

from tara2d_b200 import initial as I


def test_splitmix64_known_answer():
    """splitmix64 seeded with 0 first returns mix(0x9E3779B97F4A7C15) =
    0xE220A8397B1DCDAF (the published generator's first output)."""
    z = np.array([0x9E3779B97F4A7C15], dtype=np.uint64)
    assert int(I.splitmix64_mix(z)[0]) == 0xE220A8397B1DCDAF


def test_uniforms():
    u = I.hashed_uniform(7, 1, np.arange(200000))
    assert u.min() >= 0.0 and u.max() < 1.0
    assert abs(u.mean() - 0.5) < 5e-3 and abs(u.var() - 1 / 12) < 2e-3
    assert not np.array_equal(u, I.hashed_uniform(8, 1, np.arange(200000)))
    assert not np.array_equal(u, I.hashed_uniform(7, 2, np.arange(200000)))
    assert np.array_equal(u[1000:1010], I.hashed_uniform(7, 1, np.arange(1000, 1010)))


def test_hydro_state():
    N = 64
    st = I.hashed_state(1, N, N, I.IC_RANDOM_PHASE, seed=3, k0=4.0, e1=0.5, e2=0.01)
    n, ux, uy = (np.fft.irfft2(a, s=(N, N)) for a in st)
    assert abs(0.5 * np.mean(ux * ux + uy * uy) - 0.5) < 1e-13
    assert abs(np.std(n - 1.0) - 0.01) < 1e-3
    KX, KY = I._half_k(N, N, 2 * I.PI, 2 * I.PI, I.PI)
    div = KX * st[1] + KY * st[2]
    assert np.max(np.abs(div)) <= 1e-9 * np.max(np.abs(st[1]))


def test_orszag_tang_state():
    N = 64
    st = I.hashed_state(2, N, N, I.IC_ORSZAG_TANG, seed=1, e1=1e-3, e2=1e-3, kmin=8.0, kmax=16.0)
    rho, mx, my, E, bx, by = (np.fft.irfft2(a, s=(N, N)) for a in st)
    X, Y = I.grid(N, N)
    assert np.allclose(rho, 1.0)
    du = np.sqrt(np.mean((mx + np.sin(Y)) ** 2 + (my - np.sin(X)) ** 2))
    db = np.sqrt(np.mean((bx + np.sin(Y)) ** 2 + (by - np.sin(2 * X)) ** 2))
    assert abs(du - 1e-3) < 1e-12 and abs(db - 1e-3) < 1e-12
