"""Independent numpy (pocketfft) restatement of the reference RHS routines.

Used by the tests to cross-check the C oracle, which in turn is the checker
for the CUDA path.  Follows src/derive2coh.f95:6-265 and
src/derive2com.f95:6-426 with vectorised numpy; the 2D c2r keeps the
semantics FFTW implements (complex inverse along y for every kx column, then
a c2r along x that keeps only the real parts of the kx=0 and kx=Nx/2 bins).

Arrays: spectral (Ny, Nh) complex, real (Ny, Nx) float -- the C-order view of
the Fortran column-major (Nh,Ny) / (Nx,Ny) arrays.
"""
import numpy as np

PI = 3.14159265358979323846


def r2c(a):
    return np.fft.rfft2(a)


def c2r(X, Nx):
    H = np.fft.ifft(X, axis=0) * X.shape[0]
    H = H.copy()
    H[:, 0] = H[:, 0].real
    if Nx % 2 == 0:
        H[:, -1] = H[:, -1].real
    return np.fft.irfft(H, n=Nx, axis=1) * Nx


def wavenumbers(Nx, Ny, Lx, Ly, pi=PI):
    Nh = Nx // 2 + 1
    i = np.arange(Nh, dtype=np.float64)
    j = np.arange(Ny)
    kx = 2.0 * pi * i / Lx
    ky = np.where(j < Ny // 2, 2.0 * pi * j / Ly, 2.0 * pi * (j - Ny).astype(np.float64) / Ly)
    KX, KY = np.meshgrid(kx, ky)
    return KX, KY


def mask(Nx, Ny, KX, KY):
    return np.sqrt(KX * KX + KY * KY) >= ((Nx + Ny) / 2.0) / 3.0


def derive2coh(Nx, Ny, P, nk, ukx, uky, pi=PI):
    KX, KY = wavenumbers(Nx, Ny, P["Lx"], P["Ly"], pi)
    NN = float(Nx) * float(Ny)
    f = lambda X: c2r(X, Nx) / NN
    n, ux, uy = f(nk), f(ukx), f(uky)
    dndx, dndy = f(1j * KX * nk), f(1j * KY * nk)
    duxdx, duxdy = f(1j * KX * ukx), f(1j * KY * ukx)
    duydx, duydy = f(1j * KX * uky), f(1j * KY * uky)
    d2uxdx2, d2uxdy2 = f(KX * KX * ukx), f(KY * KY * ukx)
    d2uydx2, d2uydy2 = f(KX * KX * uky), f(KY * KY * uky)
    NLn = ux * dndx + uy * dndy + n * (duxdx + duydy)
    NLx = ux * duxdx + uy * duxdy
    NLy = ux * duydx + uy * duydy
    M = mask(Nx, Ny, KX, KY)
    g = lambda a: np.where(M, 0.0, r2c(a))
    nlx = g(NLx) + (P["mux"] * g(d2uxdx2 / n) + P["muy"] * g(d2uxdy2 / n)) + P["CS"] ** 2 * g(dndx / n)
    nly = g(NLy) + (P["mux"] * g(d2uydx2 / n) + P["muy"] * g(d2uydy2 / n)) + P["CS"] ** 2 * g(dndy / n)
    return -g(NLn), -nlx, -nly


def derive2com(Nx, Ny, P, st, pi=PI):
    rho_k, rux_k, ruy_k, E_k, Bx_k, By_k = st
    KX, KY = wavenumbers(Nx, Ny, P["Lx"], P["Ly"], pi)
    NN = float(Nx) * float(Ny)
    f = lambda X: c2r(X, Nx) / NN
    rho, rux, ruy, E, Bx, By = (f(a) for a in st)
    ux, uy = rux / rho, ruy / rho
    B2 = Bx * Bx + By * By
    ux_k, uy_k = r2c(ux), r2c(uy)
    dux = f(1j * KX * ux_k)
    duy = f(1j * KY * uy_k)
    if P.get("fix_curlB", 0):
        dBxdy, dBydx = f(1j * KY * Bx_k), f(1j * KX * By_k)
    else:
        dBxdy, dBydx = dux / NN, duy / NN
    curl = dBydx - dBxdy
    Pr = P["CS"] * P["CS"] * rho
    Mx1 = rux * ux + Pr + B2 / 2.0 - Bx * Bx
    Mx2 = rux * uy - Bx * By
    My2 = ruy * uy + Pr + B2 / 2.0 - By * By
    Ex = (E + Pr + B2 / 2.0) * ux - ux * Bx * Bx - uy * Bx * By - P["eta"] * By * curl
    Ey = (E + Pr + B2 / 2.0) * uy - ux * Bx * By - uy * By * By + P["eta"] * Bx * curl
    EV = (dux + duy) ** 2
    Magx = uy * Bx - By * ux
    M = mask(Nx, Ny, KX, KY)
    z = lambda a: np.where(M, 0.0, a)
    mu, eta = P["mu"], P["eta"]
    K2 = KX * KX + KY * KY
    d_rho = -(z(1j * KX * rux_k) + z(1j * KY * ruy_k))
    d_rux = -(z(1j * KX * r2c(Mx1)) + z(1j * KY * r2c(Mx2))) - mu * z(K2 * ux_k)
    d_ruy = -(z(1j * KX * r2c(Mx2)) + z(1j * KY * r2c(My2))) - mu * z(K2 * uy_k)
    d_E = -(z(1j * KX * r2c(Ex)) + z(1j * KY * r2c(Ey))) + mu * z(r2c(EV))
    Mk = r2c(Magx)
    d_Bx = -z(1j * KY * Mk) - eta * z(K2 * Bx_k)
    d_By = z(1j * KX * Mk) - eta * z(K2 * By_k)
    if P.get("A", 0.0) != 0.0:
        x = np.arange(Nx) * (P["Lx"] / Nx)
        y = np.arange(Ny) * (P["Ly"] / Ny)
        X, Y = np.meshgrid(x, y)
        d_rux = d_rux + r2c(-rho * P["A"] * np.sin(P["kf"] * Y))
        d_ruy = d_ruy + r2c(rho * P["A"] * np.sin(P["kf"] * X))
    return [d_rho, d_rux, d_ruy, d_E, d_Bx, d_By]
