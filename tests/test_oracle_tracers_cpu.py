"""Known answers for the oracle's restatement of the vorticity driver's tracer
step (src/main2csh.f95:187-256): a field that is bilinear inside a cell is
reproduced exactly there, a constant field everywhere (the seam included),
and the move wraps positions into (0, L] as the reference's int() rule does."""
import numpy as np

from oracle import pyoracle as O


def test_bilinear_field_reproduced_inside_cells():
    Nx, Ny, Lx, Ly = 16, 12, 2.0, 3.0
    x = np.arange(Nx) * (Lx / Nx)
    y = np.arange(Ny) * (Ly / Ny)
    X, Y = np.meshgrid(x, y)
    f = lambda a, b: 0.3 + 1.7 * a - 0.4 * b + 0.9 * a * b  # noqa: E731
    u = f(X, Y)
    rng = np.random.default_rng(0)
    xp = rng.uniform(0, x[-1], 200)   # interior cells only (no seam)
    yp = rng.uniform(0, y[-1], 200)
    vx, vy = O.tracer_velocity(u, 2 * u, xp, yp, Lx, Ly)
    assert np.abs(vx - f(xp, yp)).max() < 1e-12
    assert np.abs(vy - 2 * f(xp, yp)).max() < 1e-12


def test_constant_field_everywhere_including_seam():
    Nx, Ny, Lx, Ly = 8, 8, 2 * np.pi, 2 * np.pi
    u = np.full((Ny, Nx), 2.5)
    xp = np.array([Lx, Lx - 1e-9, 7.5 * Lx / Nx, 1e-12, 3.0])
    yp = np.array([Ly, 1.0, Ly - 1e-9, Ly, 7.9 * Ly / Ny])
    vx, _ = O.tracer_velocity(u, u, xp, yp, Lx, Ly)
    assert np.abs(vx - 2.5).max() < 1e-12


def test_periodic_neighbour_at_the_seam():
    """In the last column the far values are column 1's: a field that is 0 in
    the last column and 1 in the first gives x-weighted values in between."""
    Nx, Ny, Lx, Ly = 4, 4, 4.0, 4.0
    u = np.zeros((Ny, Nx))
    u[:, 0] = 1.0
    vx, _ = O.tracer_velocity(u, u, np.array([3.25, 3.5, 4.0]), np.array([1.5, 1.5, 1.5]), Lx, Ly)
    assert np.allclose(vx, [0.25, 0.5, 1.0], rtol=0, atol=1e-14)


def test_move_and_wrap():
    Lx = Ly = 2.0
    x, y = O.tracer_move(np.array([1.9, 0.1, 1.0, 2.0]), np.array([1.0, 1.0, 1.9, 1.0]),
                         np.array([1.0, -2.0, 0.0, 0.0]), np.array([0.0, 0.0, 3.0, 0.0]), 0.2, Lx, Ly)
    assert np.allclose(x, [0.1, 1.7, 1.0, 2.0], rtol=0, atol=1e-14)   # 2.1 -> 0.1; -0.3 -> 1.7; L stays L
    assert np.allclose(y, [1.0, 1.0, 0.5, 1.0], rtol=0, atol=1e-14)   # 2.5 -> 0.5
    assert np.all((x > 0) & (x <= Lx))
