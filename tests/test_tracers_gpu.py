"""Tracer particles of the vorticity driver (tara_tracers_run) against the
oracle's restatement of src/main2csh.f95:122-173 (velocity) and :187-256
(interpolation, move, wrap), with the oracle's FFTW velocity field.  The
interpolation arithmetic is the same on both sides; the velocity fields
differ by FFT rounding, so velocities and positions agree to 1e-12.
Particles sit at random, on grid lines, in the last column / row and at
x = Lx exactly (the periodic seam, where the reference reads past its
arrays and this build wraps to column / row 1)."""
import numpy as np
import pytest

from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu

VPI = float(np.float32(3.1428))


def csh(tara, nu=1e-3, dt=1e-3):
    return tara.Params.make(pi=VPI, Lx=2 * VPI, Ly=2 * VPI, nu=nu, dt=dt)


def particles(Nx, Ny, Lx, Ly, seed=0, n=2000):
    rng = np.random.default_rng(seed)
    dx, dy = Lx / Nx, Ly / Ny
    x = list(rng.uniform(0, Lx, n))
    y = list(rng.uniform(0, Ly, n))
    special_x = [Lx, Lx - 1e-13, (Nx - 0.5) * dx, 3 * dx, dx, 1e-12, 0.5 * dx]
    special_y = [Ly, 0.25 * dy, Ly - 1e-13, (Ny - 0.5) * dy, 7 * dy, Ly, 1e-12]
    x += special_x
    y += special_y
    return np.array(x), np.array(y)


@pytest.mark.parametrize("Nx,Ny", [(64, 64), (128, 64)])
def test_velocity_at_particles(tara, oracle, Nx, Ny):
    p = csh(tara)
    Lx = Ly = 2 * VPI
    w = I.vorticity_random_phase(Nx, Ny, seed=3)
    xp, yp = particles(Nx, Ny, Lx, Ly)
    x0, y0 = xp.copy(), yp.copy()
    with tara.Session(tara.MODEL_CSH, Nx, Ny, p) as s:
        s.set_state(w)
        vx, vy = s.tracers_run(tara.STEP_AB2, 0, xp, yp)
        wk = s.get_state()[0]
    assert np.array_equal(xp, x0) and np.array_equal(yp, y0)  # no move without steps
    ux, uy = oracle.vort_velocity_real(wk, Nx, Ny, Lx, Ly, VPI)
    rx, ry = oracle.tracer_velocity(ux, uy, x0, y0, Lx, Ly)
    scale = max(np.abs(ux).max(), np.abs(uy).max())
    assert np.abs(vx - rx).max() <= 1e-12 * scale
    assert np.abs(vy - ry).max() <= 1e-12 * scale


def test_particles_move_with_the_new_state(tara, oracle):
    N, steps = 64, 4
    p = csh(tara, dt=2e-3)
    Lx = Ly = 2 * VPI
    w = I.vorticity_random_phase(N, N, seed=5)
    xp, yp = particles(N, N, Lx, Ly, seed=1, n=500)
    rx, ry = xp.copy(), yp.copy()
    with tara.Session(tara.MODEL_CSH, N, N, p) as s:
        s.set_state(w)
        vx, vy = s.tracers_run(tara.STEP_AB2, steps, xp, yp)
    with tara.Session(tara.MODEL_CSH, N, N, p) as s:
        s.set_state(w)
        for _ in range(steps):
            s.step(tara.STEP_AB2, 1)
            ux, uy = oracle.vort_velocity_real(s.get_state()[0], N, N, Lx, Ly, VPI)
            rvx, rvy = oracle.tracer_velocity(ux, uy, rx, ry, Lx, Ly)
            rx, ry = oracle.tracer_move(rx, ry, rvx, rvy, 2e-3, Lx, Ly)
    assert np.all((xp > 0) & (xp <= Lx) & (yp > 0) & (yp <= Ly))
    assert np.abs(xp - rx).max() <= 1e-12 and np.abs(yp - ry).max() <= 1e-12
    assert np.abs(vx - rvx).max() <= 1e-11 and np.abs(vy - rvy).max() <= 1e-11


def test_screened_model(tara, oracle):
    N = 64
    p = tara.Params.make(pi=VPI, Lx=2 * np.pi, Ly=2 * np.pi, nu=1e-3, alpha=1.0, dt=1e-3, **{"lambda": 10.0})
    w = I.vorticity_random_phase(N, N, seed=7)
    xp, yp = particles(N, N, 2 * np.pi, 2 * np.pi, seed=2, n=300)
    with tara.Session(tara.MODEL_CSS, N, N, p) as s:
        s.set_state(w)
        vx, vy = s.tracers_run(tara.STEP_AB2, 0, xp, yp)
        wk = s.get_state()[0]
    ux, uy = oracle.vort_velocity_real(wk, N, N, 2 * np.pi, 2 * np.pi, VPI, lam=10.0)
    rx, ry = oracle.tracer_velocity(ux, uy, xp, yp, 2 * np.pi, 2 * np.pi)
    scale = max(np.abs(ux).max(), np.abs(uy).max())
    assert np.abs(vx - rx).max() <= 1e-12 * scale and np.abs(vy - ry).max() <= 1e-12 * scale


def test_positions_outside_the_box(tara, oracle):
    N = 32
    Lx = Ly = 2 * VPI
    xp = np.array([-0.5, Lx + 0.25, 1e300, np.nan, 1.0])
    yp = np.array([1.0, 2.0, 1.0, 1.0, -3 * Ly + 0.5])
    with tara.Session(tara.MODEL_CSH, N, N, csh(tara)) as s:
        s.set_state(I.vorticity_random_phase(N, N, seed=1))
        vx, vy = s.tracers_run(tara.STEP_AB2, 0, xp, yp)
        wk = s.get_state()[0]
    ux, uy = oracle.vort_velocity_real(wk, N, N, Lx, Ly, VPI)
    wx = np.array([Lx - 0.5, 0.25, 1.0])
    wy = np.array([1.0, 2.0, 0.5])
    rx, ry = oracle.tracer_velocity(ux, uy, wx, wy, Lx, Ly)
    assert np.allclose(vx[[0, 1, 4]], rx, rtol=0, atol=1e-12) and np.allclose(vy[[0, 1, 4]], ry, rtol=0, atol=1e-12)
    assert np.isnan(vx[2]) and np.isnan(vy[3])


def test_other_models_refuse(tara):
    from tests.gpu_common import coh_kw
    with tara.Session(tara.MODEL_COH, 32, 32, tara.Params.make(**coh_kw())) as s:
        with pytest.raises(tara.TaraError):
            s.tracers_run(tara.STEP_AB2, 1, np.array([1.0]), np.array([1.0]))
