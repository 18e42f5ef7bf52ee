"""Seeded initial conditions of the benchmark configurations (host side).

The reference's drivers build their initial states on the host and transform
them with FFTW r2c (src/main2coh.f95:141-222, src/main2com.f95:230-300); the
benchmark configurations replace the reference's point-vortex / uniform-B
profiles with seeded random-phase and Orszag-Tang states, built here with
numpy (PCG64 via ``numpy.random.default_rng(seed)``).  The same arrays feed the
GPU path and the CPU oracle.

Arrays: real fields (Ny, Nx) float64; spectral state (Ny, Nh) complex128 =
unnormalised r2c of the real field (the reference's convention).
"""
from __future__ import annotations

import numpy as np

PI = 3.14159265358979323846


def grid(Nx: int, Ny: int, Lx: float = 2 * PI, Ly: float = 2 * PI):
    """x_i = (i-1) dx, y_j = (j-1) dy (src/main2coh.f95:142-145)."""
    x = np.arange(Nx) * (Lx / Nx)
    y = np.arange(Ny) * (Ly / Ny)
    return np.meshgrid(x, y)  # X[j, i], Y[j, i]


def _kgrid_full(Nx, Ny, Lx=2 * PI, Ly=2 * PI):
    kx = np.fft.fftfreq(Nx, d=1.0 / Nx) * (2 * PI / Lx)
    ky = np.fft.fftfreq(Ny, d=1.0 / Ny) * (2 * PI / Ly)
    return np.meshgrid(kx, ky)


def r2c(a: np.ndarray) -> np.ndarray:
    return np.fft.rfft2(a)


def solenoidal_random(Nx, Ny, rng, spectrum, kmin=0.0, kmax=np.inf, Lx=2 * PI, Ly=2 * PI):
    """Random-phase divergence-free (ux, uy) with shell spectrum E(k) ~ spectrum(k).

    u = (d psi/dy, -d psi/dx), as the reference builds ukx = i ky psi,
    uky = -i kx psi (src/main2coh.f95:198-200)."""
    KX, KY = _kgrid_full(Nx, Ny, Lx, Ly)
    K = np.sqrt(KX ** 2 + KY ** 2)
    amp = np.zeros_like(K)
    sel = (K > 0) & (K >= kmin) & (K <= kmax)
    # E(k) ~ 2 pi k * k^2 |psi|^2 / 2  =>  |psi| ~ sqrt(E(k)/k^3)
    amp[sel] = np.sqrt(spectrum(K[sel]) / K[sel] ** 3)
    phase = rng.uniform(0.0, 2 * PI, size=K.shape)
    psik = amp * np.exp(1j * phase)
    psi = np.real(np.fft.ifft2(psik))
    psik = np.fft.fft2(psi)
    ux = np.real(np.fft.ifft2(1j * KY * psik))
    uy = np.real(np.fft.ifft2(-1j * KX * psik))
    return ux, uy


def _normalise(ux, uy, energy):
    e = 0.5 * np.mean(ux * ux + uy * uy)
    s = np.sqrt(energy / e) if e > 0 else 0.0
    return ux * s, uy * s


def coh_random_phase(Nx=128, Ny=128, seed=0, k0=4.0, energy=0.5, noise=0.01):
    """Hydro state (nk, ukx, uky): solenoidal u with E(k) ~ k^4 exp(-(k/k0)^2),
    total energy `energy`; density 1 + noise*N(0,1)."""
    rng = np.random.default_rng(seed)
    ux, uy = solenoidal_random(Nx, Ny, rng, lambda k: k ** 4 * np.exp(-(k / k0) ** 2))
    ux, uy = _normalise(ux, uy, energy)
    n = 1.0 + noise * rng.standard_normal((Ny, Nx))
    return [r2c(n), r2c(ux), r2c(uy)]


def ensemble_members(n=256, seed=0, sizes=(128, 256, 384, 512), nu_range=(1e-4, 1e-2), k0_range=(2.0, 8.0)):
    """Seeded ensemble of hydro runs: grid size uniform over `sizes`, viscosity
    log-uniform over `nu_range`, IC peak wavenumber k0 uniform over `k0_range`,
    and a seed per member.  Returns a list of dicts (N, nu, k0, seed)."""
    rng = np.random.default_rng(seed)
    out = []
    for m in range(n):
        out.append(dict(N=int(rng.choice(sizes)),
                        nu=float(np.exp(rng.uniform(np.log(nu_range[0]), np.log(nu_range[1])))),
                        k0=float(rng.uniform(*k0_range)), seed=int(rng.integers(0, 2 ** 31 - 1))))
    return out


def com_state(rho, ux, uy, Bx, By, CS, spheat=5.0 / 3.0):
    """Conservative MHD state (rho, rho ux, rho uy, E, Bx, By) in k-space with
    P = CS^2 rho and E = P/(spheat-1) + rho u^2/2 + B^2/2 (src/main2com.f95:247-255)."""
    P = CS * CS * rho
    E = P / (spheat - 1.0) + 0.5 * rho * (ux ** 2 + uy ** 2) + 0.5 * (Bx ** 2 + By ** 2)
    return [r2c(rho), r2c(rho * ux), r2c(rho * uy), r2c(E), r2c(Bx), r2c(By)]


def com_orszag_tang(Nx=1024, Ny=1024, seed=0, amp=1e-3, kmin=8.0, kmax=16.0, CS=100.0):
    """u = (-sin y, sin x), B = (-sin y, sin 2x), rho = 1, plus seeded
    random-phase solenoidal perturbations of rms `amp` on kmin <= |k| <= kmax
    in u and in B."""
    rng = np.random.default_rng(seed)
    X, Y = grid(Nx, Ny)
    ux, uy = -np.sin(Y), np.sin(X)
    Bx, By = -np.sin(Y), np.sin(2.0 * X)
    flat = lambda k: np.ones_like(k) * k  # E(k) ~ k : equal energy per mode
    pux, puy = solenoidal_random(Nx, Ny, rng, flat, kmin, kmax)
    pbx, pby = solenoidal_random(Nx, Ny, rng, flat, kmin, kmax)
    for a, b in ((pux, puy), (pbx, pby)):
        rms = np.sqrt(np.mean(a * a + b * b))
        if rms > 0:
            a *= amp / rms
            b *= amp / rms
    rho = np.ones((Ny, Nx))
    return com_state(rho, ux + pux, uy + puy, Bx + pbx, By + pby, CS)


def com_random_phase(Nx, Ny, seed=0, k0=6.0, ekin=0.5, emag=0.5, CS=100.0):
    """MHD state with random-phase u and B, both E(k) ~ k^4 exp(-(k/k0)^2)."""
    rng = np.random.default_rng(seed)
    spec = lambda k: k ** 4 * np.exp(-(k / k0) ** 2)
    ux, uy = _normalise(*solenoidal_random(Nx, Ny, rng, spec), ekin)
    bx, by = _normalise(*solenoidal_random(Nx, Ny, rng, spec), emag)
    return com_state(np.ones((Ny, Nx)), ux, uy, bx, by, CS)


def vorticity_random_phase(Nx, Ny, seed=0, k0=4.0, energy=0.5):
    """omega_k = i kx uy_k - i ky ux_k of a random-phase solenoidal field."""
    rng = np.random.default_rng(seed)
    ux, uy = _normalise(*solenoidal_random(Nx, Ny, rng, lambda k: k ** 4 * np.exp(-(k / k0) ** 2)), energy)
    KX, KY = _kgrid_full(Nx, Ny)
    w = np.real(np.fft.ifft2(1j * KX * np.fft.fft2(uy) - 1j * KY * np.fft.fft2(ux)))
    return [r2c(w)]


# ---------------------------------------------------------------------------
# Counter-based seeded initial conditions: the host restatement of the
# device generator (tara_set_state_random, csrc/ic.cu).  Every random value
# is a function of (seed, stream, index) only, so host and device build the
# same state; FFTs and math functions differ only in rounding.
IC_RANDOM_PHASE, IC_ORSZAG_TANG = 1, 2
_M1, _M2 = np.uint64(0xBF58476D1CE4E5B9), np.uint64(0x94D049BB133111EB)
_C1, _C2 = np.uint64(0xD1B54A32D192ED03), np.uint64(0x9E3779B97F4A7C15)


def splitmix64_mix(z):
    """The splitmix64 finaliser (S. Vigna): xor-shift 30, multiply, xor-shift 27,
    multiply, xor-shift 31, modulo 2**64 (uint64 arrays)."""
    z = np.asarray(z, dtype=np.uint64)
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def hashed_uniform(seed: int, stream: int, index) -> np.ndarray:
    """u in [0, 1): mix(mix(seed ^ stream*C1) + (index+1)*C2) >> 11, times 2**-53."""
    key = splitmix64_mix(np.array([seed], dtype=np.uint64) ^ (np.array([stream], dtype=np.uint64) * _C1))
    idx = np.asarray(index, dtype=np.uint64)
    v = splitmix64_mix(key + (idx + np.uint64(1)) * _C2)
    return (v >> np.uint64(11)).astype(np.float64) * 2.0 ** -53


def _half_k(Nx, Ny, Lx, Ly, pi):
    Nh = Nx // 2 + 1
    kx = 2.0 * pi * np.arange(Nh, dtype=np.float64) / Lx
    j = np.arange(Ny, dtype=np.float64)
    ky = np.where(np.arange(Ny) < Ny // 2, 2.0 * pi * j / Ly, 2.0 * pi * (j - Ny) / Ly)
    return np.meshgrid(kx, ky)  # (Ny, Nh)


def hashed_solenoidal(Nx, Ny, seed, stream, peaked, k0, kmin=0.0, kmax=np.inf, Lx=2 * PI, Ly=2 * PI, pi=PI):
    """(u, v, mean(u^2 + v^2)) of the random-phase streamfunction of stream
    `stream`: psi_k = a e^{2 pi i U(seed, stream, j*Nh + i)} on the half spectrum,
    a = sqrt(E(k)/k^3), E = k^4 exp(-(k/k0)^2) (peaked) or k."""
    KX, KY = _half_k(Nx, Ny, Lx, Ly, pi)
    Nh = Nx // 2 + 1
    K = np.sqrt(KX * KX + KY * KY)
    amp = np.zeros_like(K)
    sel = (K > 0) & (K >= kmin) & (K <= kmax)
    k = K[sel]
    e = k * k * k * k * np.exp(-(k / k0) * (k / k0)) if peaked else k
    amp[sel] = np.sqrt(e / (k * k * k))
    th = 2.0 * PI * hashed_uniform(seed, stream, np.arange(Ny * Nh)).reshape(Ny, Nh)
    px, py = amp * np.cos(th), amp * np.sin(th)
    u = np.fft.irfft2((-KY * py) + 1j * (KY * px), s=(Ny, Nx))
    v = np.fft.irfft2((KX * py) + 1j * (-KX * px), s=(Ny, Nx))
    return u, v, float(np.sum(u * u + v * v)) / (Nx * Ny)


def hashed_state(model, Nx, Ny, kind, seed, k0=4.0, e1=0.5, e2=0.01, kmin=0.0, kmax=np.inf, Lx=2 * PI,
                 Ly=2 * PI, pi=PI, CS=100.0, spheat=5.0 / 3.0):
    """Spectral state of the device initial condition `kind` (model 1: hydro,
    2: MHD), the same as tara_set_state_random builds (see include/tara2d_gpu.h)."""
    ot = kind == IC_ORSZAG_TANG
    lo, hi = (kmin, kmax) if ot else (0.0, np.inf)

    def scale(msq, e):
        if not msq > 0:
            return 0.0
        return e / np.sqrt(msq) if ot else np.sqrt(e / (0.5 * msq))

    u, v, msq = hashed_solenoidal(Nx, Ny, seed, 1, not ot, k0, lo, hi, Lx, Ly, pi)
    su = scale(msq, e1)
    if model == 1:
        n = Nx * Ny
        k = np.arange(n, dtype=np.uint64)
        u1 = 1.0 - hashed_uniform(seed, 3, 2 * k)
        u2 = hashed_uniform(seed, 3, 2 * k + np.uint64(1))
        g = (np.sqrt(-2.0 * np.log(u1)) * np.cos(2.0 * PI * u2)).reshape(Ny, Nx)
        return [r2c(1.0 + e2 * g), r2c(su * u), r2c(su * v)]
    bu, bv, msq = hashed_solenoidal(Nx, Ny, seed, 2, not ot, k0, lo, hi, Lx, Ly, pi)
    sb = scale(msq, e2)
    ux, uy, bx, by = su * u, su * v, sb * bu, sb * bv
    if ot:
        X, Y = grid(Nx, Ny, Lx, Ly)
        ux, uy, bx, by = ux - np.sin(Y), uy + np.sin(X), bx - np.sin(Y), by + np.sin(2.0 * X)
    return com_state(np.ones((Ny, Nx)), ux, uy, bx, by, CS, spheat)


def mhd3_state(Nx, Ny, Nz, seed=0, noise=1e-3):
    """Seeded 3D MHD state for the 3D path (src/derive3com.f95): smooth fields
    (rho ~ 1, |u|, |B| ~ 0.1, E ~ 10) plus Gaussian noise of amplitude `noise`
    on every grid point, as the spectra of rho, rho ux, rho uy, rho uz, E, Bx,
    By, Bz, each complex (Nz, Ny, Nx/2+1) (the reference's (Nh,Ny,Nz) layout)."""
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(Nz) * 2 * np.pi / Nz, np.arange(Ny) * 2 * np.pi / Ny,
                          np.arange(Nx) * 2 * np.pi / Nx, indexing="ij", sparse=True)
    n = lambda: noise * rng.standard_normal((Nz, Ny, Nx))
    rho = 1 + 0.1 * np.sin(x + 0.3) * np.cos(y) + n()
    ux = 0.1 * np.sin(z) + 0.05 * np.cos(x + y) + n()
    uy = 0.1 * np.cos(x) + n()
    uz = 0.1 * np.sin(y + 2 * x) + n()
    out = [np.fft.rfftn(rho), np.fft.rfftn(rho * ux), np.fft.rfftn(rho * uy), np.fft.rfftn(rho * uz)]
    del ux, uy, uz
    out.append(np.fft.rfftn(10 + 0.1 * np.cos(x) + n()))
    out.append(np.fft.rfftn(0.1 * np.cos(z) + n()))
    out.append(np.fft.rfftn(0.1 * np.sin(x + z) + n()))
    out.append(np.fft.rfftn(0.05 * np.cos(y) + n()))
    return out
