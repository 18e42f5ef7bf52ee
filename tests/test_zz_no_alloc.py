"""tara_derive2coh_noalloc: the hydro right-hand side for hosts that must not
allocate device memory from the solver (for example a program whose pool
allocator already owns all device memory, or a time-critical loop that cannot
afford an allocation).  It must give the same result as the regular entry
point tara_derive2coh, on two calls in a row (the calls share one static
workspace, so the second call must not see stale data from the first).

The device buffers for inputs and outputs are allocated here by the test
(torch), standing in for memory the caller already owns.

This file is collected last on purpose."""
import ctypes as C

import numpy as np
import pytest

from tests.gpu_common import coh_kw, rel_l2
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu


def _noalloc(T, p, Nx, Ny, dev_in, dev_out):
    fn = T.lib().tara_derive2coh_noalloc
    fn.argtypes = [C.POINTER(T.Params), C.c_int, C.c_int] + [C.c_void_p] * 7
    ptrs = [C.c_void_p(t.data_ptr()) for t in dev_in + dev_out]
    return fn(C.byref(p), Nx, Ny, *ptrs, None)


@pytest.mark.parametrize("Nx,Ny", [(64, 64), (256, 128)])
def test_noalloc_matches_regular_entry_point_twice(tara, Nx, Ny):
    import torch
    T = tara
    T.set_device(0)
    kw = coh_kw()
    p = T.Params.make(**kw)
    Nh = Nx // 2 + 1
    for call, seed in enumerate((101, 202)):
        st = I.coh_random_phase(Nx, Ny, seed=seed)
        # regular entry point (host arrays, cached workspace allocated by the library)
        ref = [np.zeros((Ny, Nh), np.complex128) for _ in range(3)]
        ins = [np.ascontiguousarray(a) for a in st]
        T.lib().tara_derive2coh.argtypes = [C.POINTER(T.Params), C.c_int, C.c_int] + [C.c_void_p] * 6
        assert T.lib().tara_derive2coh(C.byref(p), Nx, Ny, *[C.c_void_p(a.ctypes.data) for a in ins + ref]) == 0
        # no-allocation entry point on device buffers owned by the caller
        dev_in = [torch.from_numpy(a).to("cuda:0") for a in ins]
        dev_out = [torch.full((Ny, Nh), complex(float("nan"), float("nan")), dtype=torch.complex128,
                              device="cuda:0") for _ in range(3)]
        torch.cuda.synchronize()
        status = _noalloc(T, p, Nx, Ny, dev_in, dev_out)
        assert status == 0, T.last_error()
        torch.cuda.synchronize()
        got = [t.cpu().numpy() for t in dev_out]
        for g, r in zip(got, ref):
            assert rel_l2(g, r) <= 1e-12, (call, rel_l2(g, r))


def test_noalloc_rejects_sizes_beyond_workspace(tara):
    import torch
    T = tara
    T.set_device(0)
    p = T.Params.make(**coh_kw())
    N = 512
    bufs = [torch.zeros((N, N // 2 + 1), dtype=torch.complex128, device="cuda:0") for _ in range(6)]
    status = _noalloc(T, p, N, N, bufs[:3], bufs[3:])
    assert status == T.EINVAL
    assert "256" in T.last_error()
