"""Seeded synthetic inputs in the reference's host layouts.

The reference draws its initial conditions with GSL and FFTW at start-up
(INITIALCONDITIONS/*); those routines are outside the timed loop.  Benchmarks and
tests instead generate links, electric fields and mode sets here, once, and
hand the same arrays to the GPU path and to the CPU checkers.

Layouts (SU(2), reference conventions):
  links  float64[V, 3, 4]   U = u3 + i u_k sigma_k       (LATTICE/GaugeLinks.cpp:27-36)
  efield float64[V, 3, 3]   E^a_mu                        (LATTICE/ElectricFields.cpp:36-42)
  modes  complex128[M, V, Nc, 4]  colour-major spinors    (FERMIONS/FermionField.cpp:8-9)
with site = x + N0*(y + N1*z).
"""
from __future__ import annotations

import numpy as np


def volume(N) -> int:
    return int(N[0]) * int(N[1]) * int(N[2])


def su2_exp(alpha: np.ndarray, c: float = 1.0) -> np.ndarray:
    """exp(i c alpha^a sigma^a / 2) as (u0, u1, u2, u3) (SUNc/SU2/AlgebraOperations.cpp:37-56)."""
    a = np.asarray(alpha, dtype=np.float64) * c
    d = np.sqrt((a * a).sum(-1, keepdims=True))
    safe = np.where(d == 0.0, 1.0, d)
    vec = np.where(d == 0.0, 0.0, np.sin(0.5 * d) * a / safe)
    return np.concatenate([vec, np.cos(0.5 * d)], axis=-1)


def random_links(N, sigma: float, seed: int) -> np.ndarray:
    """Links exp(i A^a sigma^a / 2) with A^a ~ N(0, sigma^2), independently per link."""
    rng = np.random.default_rng(seed)
    A = rng.normal(0.0, sigma, size=(volume(N), 3, 3))
    return np.ascontiguousarray(su2_exp(A))


def random_efield(N, sigma: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.ascontiguousarray(rng.normal(0.0, sigma, size=(volume(N), 3, 3)))


def unit_links(N) -> np.ndarray:
    U = np.zeros((volume(N), 3, 4))
    U[..., 3] = 1.0
    return U


def mode_count(N, Nc: int = 2) -> int:
    """All modes of the complete plane-wave basis: 2 particle x Nc x 2 spin x V (MPI/ModePartition.cpp:19)."""
    return 4 * Nc * volume(N)


def u1_flux(N, n_b: int) -> np.ndarray:
    """Constant magnetic field along z with n_b flux quanta through the (x, y)
    plane, as QED::SetConstantMagneticField (QED/QED.cpp:62-84): complex
    [N1, N0, 2] phases of the x and y links, U_y(x, y) = exp(-2 pi i n_b x / (N0 N1)),
    U_x = 1 except on the last x column, U_x(N0 - 1, y) = exp(2 pi i n_b y N0 / (N0 N1))."""
    N0, N1 = int(N[0]), int(N[1])
    x = np.arange(N0)[None, :]
    y = np.arange(N1)[:, None]
    u = np.ones((N1, N0, 2), np.complex128)
    u[:, :, 1] = np.exp(-2j * np.pi * n_b * x / (N0 * N1)) * np.ones((N1, 1))
    u[:, N0 - 1, 0] = np.exp(2j * np.pi * n_b * y[:, 0] * N0 / (N0 * N1))
    return u


# ------------------------------------------------------------------- SU(3) --
# Links of three colours are 9 complex numbers per link, U_ij at i + 3j
# (SUNc/SU3/GroupOperations.cpp:4-12): complex128[V, 3, 9]; E has the 8
# components of t^a = lambda^a / 2 per link: float64[V, 3, 8].

def su3_matrix_form(alpha: np.ndarray) -> np.ndarray:
    """t^a alpha^a as complex (..., 3, 3) (MatrixForm, SU3/AlgebraOperations.cpp:89-105)."""
    a = np.asarray(alpha, dtype=np.float64)
    r3 = 1.0 / np.sqrt(3.0)
    A = np.zeros(a.shape[:-1] + (3, 3), dtype=np.complex128)
    A[..., 0, 0] = 0.5 * (a[..., 2] + a[..., 7] * r3)
    A[..., 1, 1] = -0.5 * (a[..., 2] - a[..., 7] * r3)
    A[..., 2, 2] = -a[..., 7] * r3
    A[..., 1, 0] = 0.5 * (a[..., 0] + 1j * a[..., 1])
    A[..., 2, 0] = 0.5 * (a[..., 3] + 1j * a[..., 4])
    A[..., 2, 1] = 0.5 * (a[..., 5] + 1j * a[..., 6])
    A[..., 0, 1] = np.conj(A[..., 1, 0])
    A[..., 0, 2] = np.conj(A[..., 2, 0])
    A[..., 1, 2] = np.conj(A[..., 2, 1])
    return A


def su3_pack(M: np.ndarray) -> np.ndarray:
    """(..., 3, 3) matrices -> (..., 9) in the reference order i + 3j."""
    return np.ascontiguousarray(np.swapaxes(M, -1, -2).reshape(M.shape[:-2] + (9,)))


def su3_unpack(u: np.ndarray) -> np.ndarray:
    """(..., 9) in the order i + 3j -> (..., 3, 3) matrices."""
    return np.swapaxes(np.asarray(u).reshape(u.shape[:-1] + (3, 3)), -1, -2)


def su3_exp(alpha: np.ndarray, c: float = 1.0) -> np.ndarray:
    """exp(i c t^a alpha^a), (..., 3, 3), through the eigensystem of t^a alpha^a."""
    lam, vec = np.linalg.eigh(su3_matrix_form(alpha))
    return np.einsum("...ij,...j,...kj->...ik", vec, np.exp(1j * c * lam), np.conj(vec))


def random_links_su3(N, sigma: float, seed: int) -> np.ndarray:
    """Links exp(i A^a t^a) with A^a ~ N(0, sigma^2), independently per link: complex128[V, 3, 9]."""
    rng = np.random.default_rng(seed)
    A = rng.normal(0.0, sigma, size=(volume(N), 3, 8))
    return su3_pack(su3_exp(A))


def random_efield_su3(N, sigma: float, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return np.ascontiguousarray(rng.normal(0.0, sigma, size=(volume(N), 3, 8)))


def unit_links_su3(N) -> np.ndarray:
    return su3_pack(np.broadcast_to(np.eye(3, dtype=np.complex128), (volume(N), 3, 3, 3)).copy())


def embed_su2_links(U2: np.ndarray) -> np.ndarray:
    """SU(2) links (u0, u1, u2, u3) in the upper-left block of SU(3) (sigma_k -> lambda_k)."""
    u = np.asarray(U2)
    M = np.zeros(u.shape[:-1] + (3, 3), dtype=np.complex128)
    M[..., 0, 0] = u[..., 3] + 1j * u[..., 2]
    M[..., 0, 1] = u[..., 1] + 1j * u[..., 0]
    M[..., 1, 0] = -u[..., 1] + 1j * u[..., 0]
    M[..., 1, 1] = u[..., 3] - 1j * u[..., 2]
    M[..., 2, 2] = 1.0
    return su3_pack(M)


def embed_su2_efield(E2: np.ndarray) -> np.ndarray:
    E = np.zeros(np.asarray(E2).shape[:-1] + (8,))
    E[..., :3] = E2
    return E


# -------------------------------------------------------- quasi-particles --
_MASK64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def _mix64(z: np.ndarray) -> np.ndarray:
    """SplitMix64 finaliser (Steele, Lea and Flood, OOPSLA 2014) on uint64 arrays."""
    with np.errstate(over="ignore"):
        z = z + np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def counter_gaussians(N, ncomp: int, seed: int) -> np.ndarray:
    """The counter-based complex Gaussians of ovl_set_quasi_particles (include/ovl.h):
    for counter n = (kx + N0 (ky + N1 kz)) ncomp + a, key = mix64(seed ^ mix64(n)),
    u_j = ((mix64(key + j) >> 11) + 1) 2^-53, Box-Muller pairs (u0, u1), (u2, u3).
    Returns g[kx, ky, kz, a, (c1, c2), (re, im)] of unit normal variables."""
    N = tuple(int(n) for n in N)
    kx, ky, kz = np.meshgrid(*[np.arange(n) for n in N], indexing="ij")
    site = (kx + N[0] * (ky + N[1] * kz)).astype(np.uint64)
    n = site[..., None] * np.uint64(ncomp) + np.arange(ncomp, dtype=np.uint64)
    key = _mix64(np.uint64(seed) ^ _mix64(n))
    with np.errstate(over="ignore"):
        u = [((_mix64(key + np.uint64(j)) >> np.uint64(11)) + np.uint64(1)).astype(np.float64) * 2.0 ** -53
             for j in range(4)]
    g = np.empty(N + (ncomp, 2, 2))
    for pair in range(2):
        r = np.sqrt(-2.0 * np.log(u[2 * pair]))
        g[..., pair, 0] = r * np.cos(2.0 * np.pi * u[2 * pair + 1])
        g[..., pair, 1] = r * np.sin(2.0 * np.pi * u[2 * pair + 1])
    return g


def quasi_particles(N, n0: float, qs: float, seed: int, n_colours: int = 2, generator: str = "numpy"):
    """Quasi-particle gauge fields, InitialConditions::SetQuasiParticles
    (INITIALCONDITIONS/SetQuasiParticles.cpp:28-157) for a = 1, Minkowski metric:
    per lattice momentum p_mu = -i (1 - e^{-2 pi i k_mu / N_mu}) (LATTICE/Momenta.cpp:4-8),
    two transverse polarisations xi_1, xi_2 from the base vector
    (1/sqrt3, 1/sqrt2, 1/sqrt6) (MISC/MinkowskiWaveVectors.cpp:7-44), occupancy
    f(p) = n0 / sqrt(p^2/Qs^2 + 0.1) below Qs, zero above; per colour component
    complex Gaussians c_1, c_2 (variance 1); A(p) = sqrt(f V) (c_1 xi_1 + c_2 xi_2),
    E(p) = sqrt(f V) i omega (c_1 xi_1 + c_2 xi_2); the unnormalised inverse FFT
    (FFTW_BACKWARD), A(x) = 2 Re A / V, E(x) = 2 Re E / V, and U = exp(-i A^a t^a).

    The reference draws c_1, c_2 from its GSL generator in (kx, ky, kz, a) order;
    here numpy's generator draws them in the same order (generator "numpy"), so
    the fields follow the same distribution but are not the same numbers, or
    the counter-based generator of the device version (generator "counter",
    counter_gaussians), which then gives the device's fields.  Returns (links, E) in the
    layouts of Context.set_links / set_efield; restore Gauss's law afterwards
    (Context.gauss_restore), as the reference does.
    """
    N = tuple(int(n) for n in N)
    ncomp = n_colours * n_colours - 1
    rng = np.random.default_rng(seed)
    k = np.meshgrid(*[np.arange(n) for n in N], indexing="ij")  # (kx, ky, kz)
    cdp = [-1j * (1.0 - np.exp(-2j * np.pi * k[m] / N[m])) for m in range(3)]
    p2 = sum(np.abs(c) ** 2 for c in cdp)
    omega = np.sqrt(p2)
    pv = [np.sign(c.real) * np.abs(c) for c in cdp]
    psq = sum(v * v for v in pv)
    # a mode on |p| = Qs is not occupied; the margin keeps rounding from deciding it
    occ = np.where(psq < (1.0 - 1e-12) * qs * qs, n0 / np.sqrt(psq / (qs * qs) + 0.1), 0.0)
    base = np.array([1 / np.sqrt(3.0), 1 / np.sqrt(2.0), 1 / (np.sqrt(2.0) * np.sqrt(3.0))])
    safe = np.where(p2 > 0, p2, 1.0)
    bdp = base[0] * cdp[0] + base[1] * cdp[1] + base[2] * cdp[2]
    norm = np.sqrt(np.abs(base @ base - (bdp * np.conj(bdp)).real / safe))
    norm = np.where(p2 > 0, norm, 1.0)
    om = np.where(p2 > 0, omega, 1.0)
    xi1 = [np.where(p2 > 0, (base[m] - bdp * np.conj(cdp[m]) / safe) / (norm * np.sqrt(2.0 * om)), 0.0) for m in range(3)]
    xi2 = [np.where(p2 > 0, (cdp[(m + 1) % 3] * np.conj(xi1[(m + 2) % 3]) - cdp[(m + 2) % 3] * np.conj(xi1[(m + 1) % 3])) / om,
                    0.0) for m in range(3)]
    # complex Gaussians c_1, c_2 per (kx, ky, kz, a), drawn in that loop order
    g = rng.normal(size=N + (ncomp, 2, 2)) if generator == "numpy" else counter_gaussians(N, ncomp, seed)
    c = (g[..., 0] + 1j * g[..., 1]) / np.sqrt(2.0)  # [..., a, (c1, c2)]
    V = N[0] * N[1] * N[2]
    amp = np.sqrt(occ) * np.sqrt(V)
    A = np.empty((3,) + N + (ncomp,), complex)
    E = np.empty_like(A)
    for m in range(3):
        mode = c[..., 0] * xi1[m][..., None] + c[..., 1] * xi2[m][..., None]
        A[m] = amp[..., None] * mode
        E[m] = amp[..., None] * 1j * omega[..., None] * mode
    # unnormalised backward transform over (x, y, z) times 1/V: numpy's ifftn; then 2 Re
    Ax = 2.0 * np.fft.ifftn(A, axes=(1, 2, 3)).real
    Ex = 2.0 * np.fft.ifftn(E, axes=(1, 2, 3)).real
    # [mu, x, y, z, a] -> [site = x + N0 (y + N1 z), mu, a]
    Ax = np.transpose(Ax, (3, 2, 1, 0, 4)).reshape(V, 3, ncomp)
    Ex = np.ascontiguousarray(np.transpose(Ex, (3, 2, 1, 0, 4)).reshape(V, 3, ncomp))
    if n_colours == 2:
        return np.ascontiguousarray(su2_exp(Ax, -1.0)), Ex
    return su3_pack(su3_exp(Ax, -1.0)), Ex
