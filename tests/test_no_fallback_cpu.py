"""Without a usable CUDA device the product entry points fail loudly: opening a
2D session, a 3D session or calling a drop-in RHS raises / reports an error
instead of computing anything on the host (there is no CPU fallback).
Skipped where a GPU is present."""
import ctypes as C

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.skipif(torch.cuda.is_available(), reason="a CUDA device is present")


def test_sessions_refuse_without_a_device(tara):
    with pytest.raises(tara.TaraError):
        tara.Session(tara.MODEL_COM, 32, 32, tara.Params.make(Lx=2 * tara.PI, Ly=2 * tara.PI, pi=tara.PI, dt=1e-4))
    with pytest.raises(tara.TaraError):
        tara.Mhd3(16, 16, 16, tara.Params3D.make(pi=tara.PI, Lx=2 * tara.PI, Ly=2 * tara.PI, Lz=2 * tara.PI))


def test_dropin_reports_an_error_without_a_device(tara):
    Nx = Ny = Nz = 16
    Nh = Nx // 2 + 1
    L = tara.lib()
    i32 = lambda v: C.byref(C.c_int32(v))
    dbl = lambda v: C.byref(C.c_double(v))
    st = [np.ones((Nz, Ny, Nh), complex) for _ in range(8)]
    out = [np.full((Nz, Ny, Nh), 7.0 + 0j) for _ in range(16)]
    ptr = lambda a: a.ctypes.data_as(C.c_void_p)
    L.derive3com_(i32(Nx), i32(Ny), i32(Nz), i32(Nh), dbl(tara.PI), dbl(0.0), *[ptr(a) for a in st],
                  *[ptr(a) for a in out])
    assert L.tara_legacy_status() != 0
    assert all(np.all(a == 7.0) for a in out)  # nothing written
