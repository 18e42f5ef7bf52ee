"""Generates the full-run fixtures in tests/golden/ from the CPU oracle.

    python tests/golden/make_runs.py [coh128] [com1024] [com4096]

Each fixture is the oracle's own run of one workload (the C restatement of
the reference's RHS, stepper and diagnostics over the reference's FFTW, see
oracle/tara_oracle.c), recorded the way the reference's drivers record it:

* ``run_coh128_ab2.npz``: 2D isothermal hydro (src/derive2coh.f95 +
  src/ab2coh.f95, time loop src/main2coh.f95:266-431), 128^2, AB2,
  dt = 1e-4, nu = 1e-3, CS = 3.77, 1000 steps from the seeded random-phase
  state (E(k) ~ k^4 exp(-(k/4)^2), total energy 0.5, 1% density noise).
  The Energy.dat quantities after every step (1001 records) and E(k) every
  10 steps.
* ``run_com1024_rk4.npz``: 2D MHD (src/derive2com.f95, coupled RK4, time
  loop src/main2com.f95:352-623), 1024^2, dt = 5e-5, nu = eta = 5e-4,
  CS = 100, 2000 steps from the perturbed Orszag-Tang state; the Energy.dat
  quantities, <u.B> and E(k) every 100 steps, and the modes |kx|, |ky| <= 32
  of every field after 100 and 2000 steps.
* ``run_com4096_rk4.npz``: the 4096^2 MHD workload (nu = eta = 2e-5,
  E(k) ~ k^4 exp(-(k/6)^2), dt = 1.5e-5 under the acoustic CFL limit),
  FP64, the first 50 RK4 steps: diagnostics and E(k) every 10 steps, the
  modes |kx|, |ky| <= 32 of every field after 10 and 50 steps, and the
  squared L2 norm of every field after 50 steps.

The 1024^2 run takes about an hour on 8 cores, the 4096^2 run about as long.
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as O  # noqa: E402
from tara2d_b200 import initial as I  # noqa: E402

KBLOCK = 32
# oracle stepper codes (oracle/tara_oracle.h)
AB2, RK4 = 0, 1


def coh_params():
    return O.CohParams(Lx=2 * O.PI, Ly=2 * O.PI, mux=1e-3, muy=1e-3, ms=1.0, CS=3.77, dt=1e-4)


def com_params(mu, eta, dt):
    return O.ComParams(Lx=2 * O.PI, Ly=2 * O.PI, spheat=5.0 / 3.0, mu=mu, ms=1.0, CS=100.0, mu_0=1.0,
                       eta=eta, dt=dt, kf=1.0, A=0.0, fix_curlB=0)


def low_modes(fields, K=KBLOCK):
    """Modes 0 <= kx <= K, |ky| <= K of each (Ny, Nh) spectral field, ky in
    FFT order (0..K, then -K..-1)."""
    out = []
    for a in fields:
        Ny = a.shape[0]
        rows = np.r_[0:K + 1, Ny - K:Ny]
        out.append(a[rows, :K + 1])
    return np.array(out)


def make_coh128():
    N, nsteps, ek_every = 128, 1000, 10
    P = coh_params()
    st = I.coh_random_phase(N, N, seed=1)
    diag = [O.diag_coh(N, N, P, st)]
    eks = [O.spectrum_coh(N, N, P, st[1], st[2])]
    d_old = None
    for n in range(1, nsteps + 1):
        st, d_old = O.run_coh(N, N, P, AB2, 1, st, d_old)
        diag.append(O.diag_coh(N, N, P, st))
        if n % ek_every == 0:
            eks.append(O.spectrum_coh(N, N, P, st[1], st[2]))
    np.savez_compressed(os.path.join(HERE, "run_coh128_ab2.npz"), N=N, seed=1, dt=1e-4, nu=1e-3, CS=3.77,
                        nsteps=nsteps, ek_every=ek_every, diag=np.array(diag), ek=np.array(eks),
                        final_low=low_modes(st))


def _run_com(N, seed_state, P, nsteps, every, field_steps, name, extra):
    st = seed_state
    diag = [O.diag_com(N, N, P, st)]
    eks = [O.spectrum_com(N, N, P, st)]
    fields = {}
    d_old = None
    t0 = time.time()
    for n in range(every, nsteps + 1, every):
        st, d_old = O.run_com(N, N, P, RK4, every, st, d_old)
        diag.append(O.diag_com(N, N, P, st))
        eks.append(O.spectrum_com(N, N, P, st))
        if n in field_steps:
            fields[n] = low_modes(st)
        print(f"{name}: step {n} ({time.time() - t0:.0f} s)", flush=True)
    norms = np.array([np.vdot(a, a).real for a in st])
    np.savez_compressed(os.path.join(HERE, name), N=N, nsteps=nsteps, every=every, mu=P.mu, eta=P.eta,
                        dt=P.dt, CS=P.CS, diag=np.array(diag), ek=np.array(eks),
                        field_steps=np.array(sorted(fields)),
                        fields_low=np.array([fields[k] for k in sorted(fields)]), final_norm2=norms, **extra)


def make_com1024():
    N = 1024
    P = com_params(5e-4, 5e-4, 5e-5)
    st = I.com_orszag_tang(N, N, seed=7)
    _run_com(N, st, P, 2000, 100, (100, 2000), "run_com1024_rk4.npz", dict(seed=7))


def make_com4096():
    N = 4096
    P = com_params(2e-5, 2e-5, 1.5e-5)
    st = I.com_random_phase(N, N, seed=11, k0=6.0)
    _run_com(N, st, P, 50, 10, (10, 50), "run_com4096_rk4.npz", dict(seed=11, k0=6.0))


def main(argv):
    which = argv or ["coh128", "com1024", "com4096"]
    for w in which:
        {"coh128": make_coh128, "com1024": make_com1024, "com4096": make_com4096}[w]()


if __name__ == "__main__":
    main(sys.argv[1:])
