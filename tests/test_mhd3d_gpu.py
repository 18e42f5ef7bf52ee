"""3D compressible MHD on the device (tara3d_*, derive3com_ / ab3com_) against the
oracle's restatement of src/derive3com.f95 and src/ab3com.f95 over the
reference's FFTW: RHS and 10 AB2 steps within rel L2 1e-10 per field (FP64),
the drop-in entry points through the COMMON /comm/ layout of
src/main3com.f95:56, ab3com bit for bit, and at 256^3 the size-independent
properties (E untouched by ab3com, k = 0 modes of mass / momentum / B
conserved exactly, finite state)."""
import ctypes as C

import numpy as np
import pytest

from tara2d_b200 import initial


def state3(Nx, Ny, Nz, seed=0, noise=1e-3):
    return initial.mhd3_state(Nx, Ny, Nz, seed=seed, noise=noise)


pytestmark = pytest.mark.gpu

PI = 3.14159265358979323846


def p3(tara, dt=1e-4):
    return tara.Params3D.make(pi=PI, Lx=2 * PI, Ly=2 * PI, Lz=2 * PI, mu=0.01, CS=10.0, eta=0.005, dt=dt)


def op3(oracle, dt=1e-4):
    return oracle.Com3Params(Lx=2 * PI, Ly=2 * PI, Lz=2 * PI, mu=0.01, CS=10.0, eta=0.005, dt=dt)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("Nx,Ny,Nz", [(16, 16, 16), (32, 16, 64), (64, 32, 16), (64, 64, 64), (128, 128, 128)])
def test_rhs_matches_oracle(tara, oracle, Nx, Ny, Nz):
    st = state3(Nx, Ny, Nz, seed=Nx * 7 + Nz)
    ref = oracle.derive3com(Nx, Ny, Nz, op3(oracle), st)
    with tara.Mhd3(Nx, Ny, Nz, p3(tara)) as s:
        s.set_state(st)
        got = s.rhs()
        back = s.get_state()
    for q in range(8):
        assert rel(got[q], ref[q]) <= 1e-10, (q, rel(got[q], ref[q]))
        assert np.array_equal(back[q], st[q])  # the RHS leaves the state as it is


def test_rhs_unequal_box(tara, oracle):
    """Lx, Ly, Lz all different: the wavenumber tables and the mask cut-off of
    the flux z pass (which guesses from 2 pi / Lz) on a non-cubic box."""
    Nx, Ny, Nz = 32, 16, 64
    box = dict(Lx=2 * PI, Ly=4 * PI, Lz=PI, mu=0.02, CS=5.0, eta=0.01, dt=1e-4)
    st = state3(Nx, Ny, Nz, seed=21)
    ref = oracle.derive3com(Nx, Ny, Nz, oracle.Com3Params(**box), st)
    with tara.Mhd3(Nx, Ny, Nz, tara.Params3D.make(pi=PI, **box)) as s:
        s.set_state(st)
        got = s.rhs()
    for q in range(8):
        assert rel(got[q], ref[q]) <= 1e-10, (q, rel(got[q], ref[q]))


def test_ab2_steps_match_oracle(tara, oracle):
    N, n = 32, 10
    st0 = state3(N, N, N, seed=11)
    ref, ref_h = oracle.run3com(N, N, N, op3(oracle, dt=2e-4), n, st0)
    with tara.Mhd3(N, N, N, p3(tara, dt=2e-4)) as s:
        s.set_state(st0)
        s.step(n)
        got = s.get_state()
    for q in range(8):
        assert rel(got[q], ref[q]) <= 1e-10, (q, rel(got[q], ref[q]))
    assert np.array_equal(got[4], st0[4])


def test_history_is_used(tara, oracle):
    """A given d_old enters the first step as in src/ab3com.f95:47."""
    N = 16
    st0 = state3(N, N, N, seed=5)
    h0 = state3(N, N, N, seed=6)
    ref, _ = oracle.run3com(N, N, N, op3(oracle), 2, st0, d_old=h0)
    with tara.Mhd3(N, N, N, p3(tara)) as s:
        s.set_state(st0)
        s.set_history(h0)
        s.step(2)
        got = s.get_state()
    for q in range(8):
        assert rel(got[q], ref[q]) <= 1e-10, (q, rel(got[q], ref[q]))


def _set_comm(tara, P):
    comm = (C.c_double * 16).in_dll(tara.lib(), "comm_")
    raw = (C.c_double * 16)()
    # iret, thread_num (integer(4)) in the first 8 bytes, then
    # time_max,Lx,Ly,Lz,dx,dy,dz,spheat,mu,ms,CS,mu_0,eta,dt,kf   (src/main3com.f95:56)
    vals = {2: P.Lx, 3: P.Ly, 4: P.Lz, 8: 1.0, 9: P.mu, 10: 1.0, 11: P.CS, 12: 1.0, 13: P.eta, 14: P.dt, 15: 1.0}
    for k, v in vals.items():
        raw[k] = v
    C.memmove(comm, raw, C.sizeof(raw))


def test_dropin_entry_points(tara, oracle):
    Nx, Ny, Nz = 32, 16, 16
    Nh = Nx // 2 + 1
    P = op3(oracle, dt=3e-4)
    _set_comm(tara, P)
    L = tara.lib()
    i32 = lambda v: C.byref(C.c_int32(v))
    dbl = lambda v: C.byref(C.c_double(v))
    st = [np.ascontiguousarray(a) for a in state3(Nx, Ny, Nz, seed=2)]
    d_old = [np.ascontiguousarray(a) for a in state3(Nx, Ny, Nz, seed=4)]
    d_new = [np.zeros((Nz, Ny, Nh), complex) for _ in range(8)]
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    pairs = []
    for q in range(8):
        pairs += [ptr(d_old[q]), ptr(d_new[q])]
    L.derive3com_(i32(Nx), i32(Ny), i32(Nz), i32(Nh), dbl(PI), dbl(0.0), *[ptr(a) for a in st], *pairs)
    assert L.tara_legacy_status() == 0
    ref = oracle.derive3com(Nx, Ny, Nz, P, st)
    for q in range(8):
        assert rel(d_new[q], ref[q]) <= 1e-10, q
    new = [np.zeros((Nz, Ny, Nh), complex) for _ in range(8)]
    L.ab3com_(i32(Nx), i32(Ny), i32(Nz), i32(Nh), dbl(PI), dbl(0.0), *[ptr(a) for a in st], *[ptr(a) for a in new],
              *pairs)
    assert L.tara_legacy_status() == 0
    ref_new = oracle.ab3com(Nx, Ny, Nz, P.dt, st, d_old, d_new)
    for q in range(8):
        assert np.array_equal(new[q], ref_new[q]), q  # same rounding as written
    # inconsistent Nh is refused, not computed
    L.derive3com_(i32(Nx), i32(Ny), i32(Nz), i32(Nh + 1), dbl(PI), dbl(0.0), *[ptr(a) for a in st], *pairs)
    assert L.tara_legacy_status() != 0


def test_unsupported_sizes_refused(tara):
    for dims in [(48, 16, 16), (16, 16, 1024), (8, 16, 16)]:
        with pytest.raises(tara.TaraError):
            tara.Mhd3(*dims, p3(tara))


def test_full_size_conservation(tara):
    """256^3, 5 AB2 steps: E untouched, the k = 0 modes of rho, rho u and B
    unchanged bit for bit (their RHS is exactly zero), every value finite."""
    N = 256
    st0 = state3(N, N, N, seed=1, noise=1e-4)
    with tara.Mhd3(N, N, N, p3(tara, dt=1e-4)) as s:
        s.set_state(st0)
        s.step(5)
        got = s.get_state()
    assert np.array_equal(got[4], st0[4])
    for q in (0, 1, 2, 3, 5, 6, 7):
        assert got[q][0, 0, 0] == st0[q][0, 0, 0]
        assert np.isfinite(got[q]).all()
        assert not np.array_equal(got[q], st0[q])
