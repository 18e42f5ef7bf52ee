"""The closure CNN's tensor-core convolutions (tcgen05, kind::tf32) against
PyTorch references of the same network.

On planes whose width is a multiple of 128 every convolution (the four
layers forward and the input gradients) runs as tcgen05 MMAs whose
activations enter rounded to TF32 (round to nearest, ties away from zero:
what cvt.rna.tf32.f32 does) while the BF16 weights are exact in TF32 and
accumulation is FP32.  Tolerances:
  * forward against a PyTorch FP32 network whose inputs to every
    convolution are rounded to TF32 the same way: relative L2 <= 1e-4 (the
    accumulation order differs, and a value that lands within an FP32 ulp of
    a TF32 rounding boundary before a later layer may round to the other
    neighbour, one TF32 ulp (2^-11) away);
  * forward against plain FP32 PyTorch and against the CUDA-core path of the
    same closure: <= 3e-3 (the TF32 rounding of the activations);
  * parameter gradients against plain FP32 PyTorch: <= 1e-2 per layer (the
    input-gradient convolutions also take TF32 inputs)."""
import numpy as np
import pytest

from tests.gpu_common import rel_l2
from tests.test_closure_gpu import _layers, _random_params, _unflatten

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
F = torch.nn.functional


def _tf32(t):
    """FP32 -> TF32 (10-bit mantissa), round to nearest with ties away from zero."""
    b = t.contiguous().view(torch.int32)
    r = ((b & 0x7FFFFFFF) + 0x1000) & 0x7FFFE000
    return (r | (b & -0x80000000)).view(torch.float32)


def _net(w, x, tf32_inputs):
    h = torch.tensor(x)
    for (W, b), (_, _, act) in zip(_unflatten(w), _layers()):
        Wq = W.to(torch.bfloat16).to(torch.float32)
        bq = b.to(torch.bfloat16).to(torch.float32)
        if tf32_inputs:
            h = _tf32(h)
        h = F.conv2d(F.pad(h, (1, 1, 1, 1), mode="circular"), Wq, bq)
        if act:
            h = F.gelu(h)
    return h.numpy()


@pytest.mark.parametrize("N", [128, 256])
def test_tensor_core_forward(tara, N):
    w = _random_params(tara, 11)
    x = np.random.default_rng(12).standard_normal((2, 5, N, N)).astype(np.float32)
    with tara.Closure(N, 1, batch_max=2) as c:
        c.set_params(w)
        got = c.forward(x)
        c.set_tensor_cores(False)
        cuda_cores = c.forward(x)
    emulated = _net(w, x, True)
    plain = _net(w, x, False)
    assert rel_l2(got, emulated) <= 1e-4, rel_l2(got, emulated)
    assert rel_l2(got, plain) <= 3e-3, rel_l2(got, plain)
    assert rel_l2(cuda_cores, plain) <= 1e-5, rel_l2(cuda_cores, plain)
    assert not np.array_equal(got, cuda_cores)  # the tensor-core path ran
    assert rel_l2(got, cuda_cores) <= 3e-3


def test_tensor_core_gradients(tara):
    N = 128
    w = _random_params(tara, 13)
    rng = np.random.default_rng(14)
    x = rng.standard_normal((2, 5, N, N)).astype(np.float32)
    dout = rng.standard_normal((2, 4, N, N)).astype(np.float32)
    with tara.Closure(N, 1, batch_max=2) as c:
        c.set_params(w)
        got = c.backward(x, dout)
    h = torch.tensor(x)
    q = []
    for (W, b), (_, _, act) in zip(_unflatten(w), _layers()):
        Wq = W.to(torch.bfloat16).to(torch.float32).clone().requires_grad_(True)
        bq = b.to(torch.bfloat16).to(torch.float32).clone().requires_grad_(True)
        q.append((Wq, bq))
        h = F.conv2d(F.pad(h, (1, 1, 1, 1), mode="circular"), Wq, bq)
        if act:
            h = F.gelu(h)
    (h * torch.tensor(dout)).sum().backward()
    ref = np.concatenate([np.concatenate([W.grad.numpy().ravel(), b.grad.numpy().ravel()]) for W, b in q])
    o = 0
    for ci, co, _ in _layers():
        n = co * ci * 9 + co
        assert rel_l2(got[o:o + n], ref[o:o + n]) <= 1e-2, (ci, co, rel_l2(got[o:o + n], ref[o:o + n]))
        o += n
    assert tara.lib().tara_closure_status(c._h) == tara.EINVAL  # closed handle is refused


def test_tensor_core_time(tara):
    """Both paths time on the device; report, and check they give a time."""
    with tara.Closure(256, 1, batch_max=1) as c:
        c.set_params(_random_params(tara, 15))
        tc = c.time_cnn(1, 10)
        c.set_tensor_cores(False)
        cc = c.time_cnn(1, 10)
    assert all(t > 0 for t in tc + cc)
    print(f"CNN 256^2 B=1: tensor cores fwd {tc[0]:.3f} ms, fwd+bwd {tc[1]:.3f} ms; "
          f"CUDA cores fwd {cc[0]:.3f} ms, fwd+bwd {cc[1]:.3f} ms")
