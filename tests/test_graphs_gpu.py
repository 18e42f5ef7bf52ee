"""Steps replayed from CUDA graphs give bit-identical states to steps launched
kernel by kernel, for every model and stepper, odd step counts and parameter
changes between batches."""
import numpy as np
import pytest

from tests.gpu_common import coh_kw, com_kw
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu


def _run(tara, model, N, kw, st, stepper, batches, graphs, precision=0, change=None):
    with tara.Session(model, N, N, tara.Params.make(**kw), precision=precision) as s:
        s.set_graphs(graphs)
        s.set_state(st)
        for b, n in enumerate(batches):
            if change is not None and b == 1:
                s.set_params(tara.Params.make(**change))
            s.step(stepper, n)
        return s.get_state(), s.get_history()


def _cases(tara):
    vk = dict(pi=tara.VORT_PI, Lx=2 * tara.VORT_PI, Ly=2 * tara.VORT_PI, nu=1e-3, dt=1e-3)
    return [
        (tara.MODEL_COH, 64, coh_kw(dt=1e-3), I.coh_random_phase(64, 64, seed=1)),
        (tara.MODEL_COM, 64, com_kw(), I.com_random_phase(64, 64, seed=2)),
        (tara.MODEL_CSH, 64, vk, I.vorticity_random_phase(64, 64, seed=3)),
    ]


@pytest.mark.parametrize("case", [0, 1, 2])
@pytest.mark.parametrize("stepper", [0, 1, 2])
def test_graph_replay_is_bit_identical(tara, case, stepper):
    model, N, kw, st = _cases(tara)[case]
    batches = [5, 2, 3]  # odd counts leave the state in the other buffer between batches
    a_state, a_hist = _run(tara, model, N, kw, st, stepper, batches, True)
    b_state, b_hist = _run(tara, model, N, kw, st, stepper, batches, False)
    for x, y in zip(a_state + a_hist, b_state + b_hist):
        assert np.array_equal(x, y)


def test_graphs_follow_parameter_changes(tara):
    N = 64
    kw = com_kw()
    st = I.com_random_phase(N, N, seed=4)
    change = com_kw(dt=2.5e-5, mu=1e-3)
    a, _ = _run(tara, tara.MODEL_COM, N, kw, st, 1, [4, 4], True, change=change)
    b, _ = _run(tara, tara.MODEL_COM, N, kw, st, 1, [4, 4], False, change=change)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_graphs_fp32(tara):
    N = 128
    kw = com_kw()
    st = I.com_random_phase(N, N, seed=5)
    a, _ = _run(tara, tara.MODEL_COM, N, kw, st, 1, [6], True, precision=tara.FP32)
    b, _ = _run(tara, tara.MODEL_COM, N, kw, st, 1, [6], False, precision=tara.FP32)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)
