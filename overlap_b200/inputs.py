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
