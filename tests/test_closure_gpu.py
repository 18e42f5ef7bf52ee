"""Learned closure: the hand-written CNN kernels against a PyTorch FP32
reference of the same network (weights rounded to BF16, circular padding),
the device-made training pairs against a numpy restatement over the
oracle's FFTW transforms, the closure term inside the MHD RHS, and training.

Tolerances: CNN forward relative L2 <= 1e-5 and parameter gradients <= 1e-4
(FP32 accumulation in a different order); training pairs <= 1e-5 (stored in
FP32); the closure term in the RHS <= 1e-5 (its FP32 network input may round
differently from one computed over the oracle's transforms); the filtered
state is exact to rounding (<= 1e-15)."""
import numpy as np
import pytest

from tests.gpu_common import com_kw, rel_l2
from tests.test_parity_com_gpu import compressive
from tara2d_b200 import initial as I

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
F = torch.nn.functional


def _layers():
    return [(5, 32, True), (32, 32, True), (32, 32, True), (32, 4, False)]


def _unflatten(w):
    out, o = [], 0
    for ci, co, _ in _layers():
        W = torch.tensor(w[o:o + co * ci * 9].reshape(co, ci, 3, 3))
        o += co * ci * 9
        b = torch.tensor(w[o:o + co])
        o += co
        out.append((W, b))
    return out


def _torch_net(w, x, grad=False):
    ps = _unflatten(w)
    q = []
    for W, b in ps:
        Wq = W.to(torch.bfloat16).to(torch.float32).clone().requires_grad_(grad)
        bq = b.to(torch.bfloat16).to(torch.float32).clone().requires_grad_(grad)
        q.append((Wq, bq))
    h = torch.tensor(x)
    for (W, b), (_, _, act) in zip(q, _layers()):
        h = F.conv2d(F.pad(h, (1, 1, 1, 1), mode="circular"), W, b)
        if act:
            h = F.gelu(h)
    return h, q


def _random_params(tara, seed, scale=0.15):
    rng = np.random.default_rng(seed)
    return (scale * rng.standard_normal(tara.Closure.num_params())).astype(np.float32)


def test_cnn_forward_matches_torch(tara):
    with tara.Closure(32, 1, batch_max=2) as c:
        w = _random_params(tara, 1)
        c.set_params(w)
        x = np.random.default_rng(2).standard_normal((2, 5, 32, 32)).astype(np.float32)
        got = c.forward(x)
    ref, _ = _torch_net(w, x)
    assert rel_l2(got, ref.numpy()) <= 1e-5, rel_l2(got, ref.numpy())


def test_cnn_gradients_match_torch(tara):
    with tara.Closure(32, 1, batch_max=2) as c:
        w = _random_params(tara, 3)
        c.set_params(w)
        rng = np.random.default_rng(4)
        x = rng.standard_normal((2, 5, 32, 32)).astype(np.float32)
        dout = rng.standard_normal((2, 4, 32, 32)).astype(np.float32)
        got = c.backward(x, dout)
    out, q = _torch_net(w, x, grad=True)
    (out * torch.tensor(dout)).sum().backward()
    ref = np.concatenate([np.concatenate([W.grad.numpy().ravel(), b.grad.numpy().ravel()]) for W, b in q])
    o = 0
    for ci, co, _ in _layers():
        n = co * ci * 9 + co
        assert rel_l2(got[o:o + n], ref[o:o + n]) <= 1e-4, (ci, co, rel_l2(got[o:o + n], ref[o:o + n]))
        o += n


def _filter(a, Nf, Nc):
    out = np.zeros((Nc, Nc // 2 + 1), np.complex128)
    for jc in range(Nc):
        if jc == Nc // 2:
            continue
        jf = jc if jc < Nc // 2 else jc + (Nf - Nc)
        out[jc, :Nc // 2] = a[jf, :Nc // 2]
    return out * (Nc * Nc) / (Nf * Nf)


def _fluxes(rho, mx, my, bx, by):
    ux, uy = mx / rho, my / rho
    B2 = bx * bx + by * by
    return [mx * ux + B2 / 2 - bx * bx, mx * uy - bx * by, my * uy + B2 / 2 - by * by, uy * bx - by * ux]


def test_training_pair_and_filter(tara, oracle):
    Nf, Nc = 128, 32
    st = compressive(I.com_random_phase(Nf, Nf, seed=6, k0=10.0), 7)
    with tara.Session(tara.MODEL_COM, Nf, Nf, tara.Params.make(**com_kw())) as fine, \
            tara.Session(tara.MODEL_COM, Nc, Nc, tara.Params.make(**com_kw())) as coarse, \
            tara.Closure(Nc, 2) as c:
        fine.set_state(st)
        c.add_pair(fine)
        assert c.count == 1
        gin, gout = c.get_pair(0)
        tara.filter_state(fine, coarse)
        filt = coarse.get_state()
    for g, a in zip(filt, st):
        assert rel_l2(g, _filter(a, Nf, Nc)) <= 1e-15
    R = [oracle.c2r_2d(a, Nf) / Nf ** 2 for a in st]
    Ff = _fluxes(R[0], R[1], R[2], R[4], R[5])
    fl = [oracle.c2r_2d(_filter(oracle.r2c_2d(f), Nf, Nc), Nc) / Nc ** 2 for f in Ff]
    Rc = [oracle.c2r_2d(_filter(st[k], Nf, Nc), Nc) / Nc ** 2 for k in (0, 1, 2, 4, 5)]
    Fc = _fluxes(*Rc)
    tau = [a - b for a, b in zip(fl, Fc)]
    inp = [Rc[0] - 1.0, Rc[1] / Rc[0], Rc[2] / Rc[0], Rc[3], Rc[4]]
    for k in range(5):
        assert rel_l2(gin[k], inp[k]) <= 1e-5, (k, rel_l2(gin[k], inp[k]))
    for k in range(4):
        assert rel_l2(gout[k], tau[k]) <= 1e-5, (k, rel_l2(gout[k], tau[k]))


def test_closure_term_in_rhs(tara, oracle):
    N = 32
    st = compressive(I.com_random_phase(N, N, seed=9), 3)
    norm = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 1e-3, 0.3, 0.3, 0.4, 0.4,
                     1e-3, -2e-3, 5e-4, 1e-4, 2e-2, 1e-2, 3e-2, 5e-3], np.float32)
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**com_kw())) as s, tara.Closure(N, 1) as c:
        c.set_params(_random_params(tara, 5, 0.2))
        c.set_norm(norm)
        s.set_state(st)
        plain = s.rhs()
        tara.attach_closure(s, c)
        closed = s.rhs()
        s.step(tara.STEP_RK4, 3)  # graph capture with the closure attached
        tara.attach_closure(s, None)
        s.set_state(st)
        again = s.rhs()
        mi, si, mo, so = norm[:5], norm[5:10], norm[10:14], norm[14:18]
        R = [oracle.c2r_2d(st[k], N) / N ** 2 for k in (0, 1, 2, 4, 5)]
        x = np.stack([R[0] - 1.0, R[1] / R[0], R[2] / R[0], R[3], R[4]]).astype(np.float32)
        x = ((x - mi[:, None, None]) / si[:, None, None])[None].astype(np.float32)
        out = c.forward(x)[0].astype(np.float64)
    tau = [oracle.r2c_2d(out[k] * so[k] + mo[k]) for k in range(4)]
    k = np.fft.fftfreq(N, 1.0 / N)
    KX, KY = np.meshgrid(np.arange(N // 2 + 1, dtype=np.float64), k)
    keep = np.sqrt(KX ** 2 + KY ** 2) < (N + N) / 2 / 3
    term = [0 * tau[0], -(1j * KX * tau[0] + 1j * KY * tau[1]), -(1j * KX * tau[1] + 1j * KY * tau[2]),
            0 * tau[0], -1j * KY * tau[3], 1j * KX * tau[3]]
    for f in range(6):
        d = closed[f] - plain[f]
        t = term[f] * keep
        if f in (0, 3):
            assert np.array_equal(closed[f], plain[f])
        else:
            assert rel_l2(d, t) <= 1e-5, (f, rel_l2(d, t))
    for a, b in zip(again, plain):
        assert np.array_equal(a, b)


def test_training_reduces_the_loss(tara):
    Nf, Nc = 128, 32
    kw = com_kw(mu=1e-3, eta=1e-3, dt=1e-4)
    with tara.Session(tara.MODEL_COM, Nf, Nf, tara.Params.make(**kw)) as fine, tara.Closure(Nc, 24, 8, seed=3) as c:
        fine.set_state(I.com_random_phase(Nf, Nf, seed=2, k0=8.0))
        for _ in range(24):
            fine.step(tara.STEP_RK4, 2)
            c.add_pair(fine)
        c.fit_norm(0, 24)
        before = c.eval_loss(0, 24)
        losses = c.train(0, 24, epochs=40, batch=8, lr=2e-3)
        after = c.eval_loss(0, 24)
    assert np.all(np.isfinite(losses))
    assert after < 0.5 * before, (before, after, losses[-5:])


def _rk4_host(s, u0, dt, term):
    """One classical RK4 step built from single RHS calls of session `s`
    (closure detached): k_i = rhs(stage input) + term(stage index, input)."""
    def f(i, u):
        s.set_state(u)
        r = s.rhs()
        t = term(i, u)
        return [a + b for a, b in zip(r, t)]
    k1 = f(0, u0)
    k2 = f(1, [a + 0.5 * dt * b for a, b in zip(u0, k1)])
    k3 = f(2, [a + 0.5 * dt * b for a, b in zip(u0, k2)])
    k4 = f(3, [a + dt * b for a, b in zip(u0, k3)])
    return [a + dt / 6.0 * (b + 2.0 * c + 2.0 * d + e) for a, b, c, d, e in zip(u0, k1, k2, k3, k4)]


@pytest.mark.parametrize("mode", ["every_rhs", "once_per_step"])
def test_closure_mode_in_rk4_steps(tara, mode):
    """An RK4 step with the closure attached against the classical RK4 step
    built on the host from single RHS evaluations: every RHS evaluation adds
    the closure term of its own stage input (CLOSURE_EVERY_RHS), or all four
    stages add the term of the step's input (CLOSURE_ONCE_PER_STEP).  The
    step increments agree to relative L2 <= 1e-9 per field (FP64; the fused
    stepper rounds in another order), the two modes differ by far more than
    that, and four captured single steps equal one call of four steps."""
    N, dt = 32, 2e-4
    st = compressive(I.com_random_phase(N, N, seed=9), 3)
    norm = np.array([0.0, 0.0, 0.0, 0.0, 0.0, 1e-3, 0.3, 0.3, 0.4, 0.4,
                     1e-3, -2e-3, 5e-4, 1e-4, 2e-2, 1e-2, 3e-2, 5e-3], np.float32)
    want = tara.CLOSURE_EVERY_RHS if mode == "every_rhs" else tara.CLOSURE_ONCE_PER_STEP
    with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**com_kw(dt=dt))) as s, tara.Closure(N, 1) as c:
        c.set_params(_random_params(tara, 5, 0.2))
        c.set_norm(norm)

        def closure_term(u):
            s.set_state(u)
            plain = s.rhs()
            tara.attach_closure(s, c)
            closed = s.rhs()
            tara.attach_closure(s, None)
            return [a - b for a, b in zip(closed, plain)]

        c0 = closure_term(st)
        ref = {"every_rhs": _rk4_host(s, st, dt, lambda i, u: closure_term(u)),
               "once_per_step": _rk4_host(s, st, dt, lambda i, u: c0)}
        s.set_closure_mode(want)
        tara.attach_closure(s, c)
        s.set_state(st)
        s.step(tara.STEP_RK4, 1)
        got = s.get_state()
        s.set_state(st)
        for _ in range(4):
            s.step(tara.STEP_RK4, 1)
        four_single = s.get_state()
        s.set_state(st)
        s.step(tara.STEP_RK4, 4)
        four = s.get_state()
        with pytest.raises(tara.TaraError):
            s.set_closure_mode(2)
        tara.attach_closure(s, None)
    other = "once_per_step" if mode == "every_rhs" else "every_rhs"
    for f in (1, 2, 4, 5):  # the fields the closure acts on
        inc = got[f] - st[f]
        err = rel_l2(inc, ref[mode][f] - st[f])
        gap = rel_l2(ref[other][f] - st[f], ref[mode][f] - st[f])
        assert err <= 1e-9, (f, err)
        assert gap > 1e3 * max(err, 1e-12), (f, err, gap)
    for a, b in zip(four_single, four):
        assert np.array_equal(a, b)


def test_closure_mode_leaves_ab2_unchanged(tara):
    """AB2 has one RHS evaluation per step: both closure modes give the same
    bits."""
    N = 32
    st = compressive(I.com_random_phase(N, N, seed=11), 3)
    out = []
    with tara.Closure(N, 1) as c:
        c.set_params(_random_params(tara, 6, 0.2))
        for mode in (tara.CLOSURE_EVERY_RHS, tara.CLOSURE_ONCE_PER_STEP):
            with tara.Session(tara.MODEL_COM, N, N, tara.Params.make(**com_kw())) as s:
                s.set_closure_mode(mode)
                tara.attach_closure(s, c)
                s.set_state(st)
                s.step(tara.STEP_AB2, 5)
                out.append(s.get_state() + s.get_history())
                tara.attach_closure(s, None)
    for a, b in zip(*out):
        assert np.array_equal(a, b)
