"""Shared helpers of the GPU parity tests."""
import numpy as np

PI = 3.14159265358979323846


def rel_l2(a, b):
    a = np.asarray(a)
    b = np.asarray(b)
    den = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (den if den > 0 else 1.0)


def coh_kw(**kw):
    d = dict(Lx=2 * PI, Ly=2 * PI, pi=PI, mux=1e-3, muy=1e-3, ms=1.0, CS=3.77, dt=1e-4)
    d.update(kw)
    return d


def com_kw(**kw):
    d = dict(Lx=2 * PI, Ly=2 * PI, pi=PI, spheat=5.0 / 3.0, mu=5e-4, ms=1.0, CS=100.0, mu_0=1.0, eta=5e-4,
             dt=5e-5, kf=1.0, A=0.0, fix_curlB=0)
    d.update(kw)
    return d


def oracle_coh_params(O, kw):
    return O.CohParams(**{k: kw[k] for k in ("Lx", "Ly", "mux", "muy", "ms", "CS", "dt")})


def oracle_com_params(O, kw):
    return O.ComParams(**{k: kw[k] for k in ("Lx", "Ly", "spheat", "mu", "ms", "CS", "mu_0", "eta", "dt", "kf",
                                              "A", "fix_curlB")})
