"""tara_derive2coh_noalloc: the hydro right-hand side for hosts that must not
allocate device memory from the solver (for example a program whose pool
allocator already owns all device memory, or a time-critical loop that cannot
afford an allocation).  It must give the same result as the regular entry
point tara_derive2coh and as the oracle's derive2coh, on two calls in a row
(the calls share one static workspace, so the second call must not see stale
data from the first), allocate nothing on the device after its first call
(which loads the library's device code and workspace), and stay correct when
several host threads call it at once on one stream.

Tolerance: relative L2 <= 1e-12 per field against both references (FP64).

The device buffers for inputs and outputs are allocated here by the test
(torch), standing in for memory the caller already owns.

This file is collected last on purpose."""
import ctypes as C
import json
import os
import subprocess
import sys
import threading

import numpy as np
import pytest

from tests.gpu_common import coh_kw, oracle_coh_params, rel_l2
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _noalloc(T, p, Nx, Ny, dev_in, dev_out, stream=None):
    fn = T.lib().tara_derive2coh_noalloc
    fn.argtypes = [C.POINTER(T.Params), C.c_int, C.c_int] + [C.c_void_p] * 7
    ptrs = [C.c_void_p(t.data_ptr()) for t in dev_in + dev_out]
    return fn(C.byref(p), Nx, Ny, *ptrs, stream)


def _regular(T, p, Nx, Ny, ins):
    Nh = Nx // 2 + 1
    ref = [np.zeros((Ny, Nh), np.complex128) for _ in range(3)]
    T.lib().tara_derive2coh.argtypes = [C.POINTER(T.Params), C.c_int, C.c_int] + [C.c_void_p] * 6
    assert T.lib().tara_derive2coh(C.byref(p), Nx, Ny, *[C.c_void_p(a.ctypes.data) for a in ins + ref]) == 0
    return ref


@pytest.mark.parametrize("Nx,Ny", [(16, 16), (32, 256), (64, 64), (256, 128), (256, 256)])
def test_noalloc_matches_regular_entry_point_and_oracle_twice(tara, oracle, Nx, Ny):
    import torch
    T = tara
    T.set_device(0)
    kw = coh_kw()
    p = T.Params.make(**kw)
    P = oracle_coh_params(oracle, kw)
    Nh = Nx // 2 + 1
    for call, seed in enumerate((101, 202)):
        ins = [np.ascontiguousarray(a) for a in I.coh_random_phase(Nx, Ny, seed=seed + Nx + Ny)]
        ref = _regular(T, p, Nx, Ny, ins)
        ora = oracle.derive2coh(Nx, Ny, P, *ins)
        dev_in = [torch.from_numpy(a).to("cuda:0") for a in ins]
        dev_out = [torch.full((Ny, Nh), complex(float("nan"), float("nan")), dtype=torch.complex128,
                              device="cuda:0") for _ in range(3)]
        torch.cuda.synchronize()
        status = _noalloc(T, p, Nx, Ny, dev_in, dev_out)
        assert status == 0, T.last_error()
        torch.cuda.synchronize()
        got = [t.cpu().numpy() for t in dev_out]
        for g, r, o in zip(got, ref, ora):
            assert rel_l2(g, r) <= 1e-12, (call, rel_l2(g, r))
            assert rel_l2(g, o) <= 1e-12, (call, rel_l2(g, o))


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


def test_noalloc_concurrent_host_threads_one_stream(tara, oracle):
    """Two host threads alternate grid sizes on the default stream (ordered on
    the GPU): the host-side table preparation is serialised by the library,
    so every call sees its own tables."""
    import torch
    T = tara
    T.set_device(0)
    kw = coh_kw()
    p = T.Params.make(**kw)
    P = oracle_coh_params(oracle, kw)
    jobs = {}
    for N in (64, 128):
        ins = [np.ascontiguousarray(a) for a in I.coh_random_phase(N, N, seed=N)]
        jobs[N] = (ins, oracle.derive2coh(N, N, P, *ins),
                   [torch.from_numpy(a).to("cuda:0") for a in ins])
    torch.cuda.synchronize()
    errors = []

    def worker(N):
        ins, ora, dev_in = jobs[N]
        for _ in range(6):
            out = [torch.empty((N, N // 2 + 1), dtype=torch.complex128, device="cuda:0") for _ in range(3)]
            if _noalloc(T, p, N, N, dev_in, out) != 0:
                errors.append((N, "status"))
                return
            torch.cuda.synchronize()
            for g, o in zip(out, ora):
                e = rel_l2(g.cpu().numpy(), o)
                if not e <= 1e-12:
                    errors.append((N, e))
    th = [threading.Thread(target=worker, args=(N,)) for N in (64, 128)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors


_FRESH = r"""
import ctypes as C, json, sys
import numpy as np, torch
sys.path.insert(0, sys.argv[1])
import tara2d_b200 as T
from tara2d_b200 import initial as I
from tests.gpu_common import coh_kw
lib = C.CDLL(T.LIB_PATH)
fn = lib.tara_derive2coh_noalloc
fn.argtypes = [C.POINTER(T.Params), C.c_int, C.c_int] + [C.c_void_p] * 7
N = 128
p = T.Params.make(**coh_kw())
outs, free = [], []
torch.cuda.init()
ins = [[torch.from_numpy(np.ascontiguousarray(a)).to("cuda:0") for a in I.coh_random_phase(N, N, seed=s)]
       for s in (5, 6, 7)]
res = [[torch.empty((N, N // 2 + 1), dtype=torch.complex128, device="cuda:0") for _ in range(3)] for _ in range(3)]
torch.cuda.synchronize()
alloc0 = (torch.cuda.memory_allocated(), torch.cuda.memory_reserved())
status = []
for k in range(3):
    status.append(fn(C.byref(p), N, N, *[C.c_void_p(t.data_ptr()) for t in ins[k] + res[k]], None))
    torch.cuda.synchronize()
    free.append(torch.cuda.mem_get_info()[0])
alloc1 = (torch.cuda.memory_allocated(), torch.cuda.memory_reserved())
np.save(sys.argv[2], np.array([[t.cpu().numpy() for t in r] for r in res]))
print(json.dumps({"status": status, "free": free, "alloc0": alloc0, "alloc1": alloc1}))
"""


def test_noalloc_first_call_in_fresh_process_allocates_nothing(tara, oracle, tmp_path):
    """In a fresh process whose first library call is the no-allocation entry
    point: torch's allocator statistics do not move, the device's free memory
    is the same after the second and third calls as after the first (which
    loads the library's device code and static workspace), and the results
    match the oracle."""
    out = tmp_path / "res.npy"
    r = subprocess.run([sys.executable, "-c", _FRESH, ROOT, str(out)], capture_output=True, text=True,
                       timeout=600, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-3000:]
    info = json.loads(r.stdout.strip().splitlines()[-1])
    assert info["status"] == [0, 0, 0], info
    assert info["alloc0"] == info["alloc1"], info
    assert info["free"][1] == info["free"][0] and info["free"][2] == info["free"][0], info
    res = np.load(out)
    kw = coh_kw()
    P = oracle_coh_params(oracle, kw)
    N = 128
    for k, s in enumerate((5, 6, 7)):
        ora = oracle.derive2coh(N, N, P, *I.coh_random_phase(N, N, seed=s))
        for g, o in zip(res[k], ora):
            assert rel_l2(g, o) <= 1e-12, (k, rel_l2(g, o))
