"""Generates the golden fixtures in tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

The FFT fixtures are outputs of the reference's own FFTW 3.3.9 (compiled from
its sources by oracle/Makefile) on seeded inputs, including a spectrum whose
kx = 0 / Nyquist columns are not Hermitian (it pins the c2r semantics the CUDA
path reproduces).  The RHS fixtures are outputs of the oracle's restatement of
src/derive2coh.f95 and src/derive2com.f95 on seeded states.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import pyoracle as O  # noqa: E402
from tara2d_b200 import initial as I  # noqa: E402


def coh_params():
    return O.CohParams(Lx=2 * O.PI, Ly=2 * O.PI, mux=1e-3, muy=1e-3, ms=1.0, CS=3.77, dt=1e-4)


def com_params(fix=0):
    return O.ComParams(Lx=2 * O.PI, Ly=2 * O.PI, spheat=5.0 / 3.0, mu=5e-4, ms=1.0, CS=100.0, mu_0=1.0,
                       eta=5e-4, dt=5e-5, kf=1.0, A=0.0, fix_curlB=fix)


def main():
    rng = np.random.default_rng(20261203)
    Nx, Ny = 16, 12
    a = rng.standard_normal((Ny, Nx))
    X = rng.standard_normal((Ny, Nx // 2 + 1)) + 1j * rng.standard_normal((Ny, Nx // 2 + 1))
    np.savez(os.path.join(HERE, "fftw_16x12.npz"), real_in=a, r2c_out=O.r2c_2d(a), spec_in=X,
             c2r_out=O.c2r_2d(X, Nx))
    st = I.coh_random_phase(16, 16, seed=7)
    d = O.derive2coh(16, 16, coh_params(), *st)
    np.savez(os.path.join(HERE, "derive2coh_16.npz"), nk=st[0], ukx=st[1], uky=st[2], dn=d[0], dux=d[1], duy=d[2])
    sm = I.com_orszag_tang(16, 16, seed=7, amp=1e-2, kmin=2, kmax=5)
    # compressive noise on every mode, so that d(rho)/dt is not rounding noise
    sm = [a + 1e-3 * np.abs(a).max() * (rng.standard_normal(a.shape) + 1j * rng.standard_normal(a.shape))
          for a in sm]
    dm = O.derive2com(16, 16, com_params(0), sm)
    np.savez(os.path.join(HERE, "derive2com_16.npz"), state=np.array(sm), rhs=np.array(dm))


if __name__ == "__main__":
    main()
