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
