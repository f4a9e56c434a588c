"""Input generators (overlap_b200/inputs.py) on the CPU: the quasi-particle
initial condition of SetQuasiParticles.cpp, whose reference implementation
needs FFTW and GSL (absent here), is checked by the properties its
construction guarantees."""
import numpy as np

from overlap_b200.inputs import quasi_particles, su3_unpack, volume


def _backward_divergence(E, N):
    """sum_mu E_mu(x) - E_mu(x - mu) per site and colour component."""
    V = volume(N)
    F = E.reshape(N[2], N[1], N[0], 3, -1)  # [z, y, x, mu, a]
    div = np.zeros(F.shape[:3] + F.shape[4:])
    for mu, ax in ((0, 2), (1, 1), (2, 0)):
        div += F[..., mu, :] - np.roll(F[..., mu, :], 1, axis=ax)
    return div.reshape(V, -1)


def test_quasi_particle_fields_are_transverse_and_special_unitary():
    N = (8, 6, 10)
    U, E = quasi_particles(N, 4.0, 1.0, seed=3)
    assert U.shape == (volume(N), 3, 4) and E.shape == (volume(N), 3, 3)
    assert np.abs(np.sum(U * U, axis=-1) - 1.0).max() < 1e-14
    # polarisations orthogonal to the lattice momentum: E is divergence-free
    assert np.abs(_backward_divergence(E, N)).max() < 1e-13 * max(1.0, np.abs(E).max())
    U3, E3 = quasi_particles(N, 4.0, 1.0, seed=3, n_colours=3)
    M = su3_unpack(U3)
    assert np.abs(M @ np.conj(np.swapaxes(M, -1, -2)) - np.eye(3)).max() < 1e-13
    assert np.abs(np.linalg.det(M) - 1).max() < 1e-13
    assert np.abs(_backward_divergence(E3, N)).max() < 1e-13 * max(1.0, np.abs(E3).max())


def test_quasi_particle_electric_energy_follows_the_occupancy():
    """<sum_x E^2> = 2 (Nc^2 - 1) sum_p f(p) omega(p): each occupied mode
    carries omega f in E^2 per colour component (two polarisations of norm
    1/(2 omega) each, E(p) = i omega A(p), 2 Re of the transform)."""
    N = (16, 16, 16)
    n0, qs = 4.0, 1.0
    k = np.meshgrid(*[np.arange(n) for n in N], indexing="ij")
    cdp = [-1j * (1.0 - np.exp(-2j * np.pi * k[m] / N[m])) for m in range(3)]
    omega = np.sqrt(sum(np.abs(c) ** 2 for c in cdp))
    psq = sum((np.sign(c.real) * np.abs(c)) ** 2 for c in cdp)
    f = np.where(psq < qs * qs, n0 / np.sqrt(psq / qs ** 2 + 0.1), 0.0)
    want = 2 * 3 * np.sum(f * omega)
    for generator in ("numpy", "counter"):  # numpy's generator, and the device version's counter-based one
        got = np.mean([np.sum(quasi_particles(N, n0, qs, seed=s, generator=generator)[1] ** 2) for s in range(24)])
        assert abs(got / want - 1) < 0.1, generator
    # nothing above Qs: no occupied mode, no field
    U, E = quasi_particles(N, n0, 1e-3, seed=1)
    assert np.abs(E).max() == 0.0 and np.abs(U[..., 3] - 1).max() == 0.0


def test_counter_generator_gives_independent_unit_normals():
    """The counter-based Gaussians of the device's quasi-particles: mean 0,
    variance 1, uncorrelated between neighbouring counters, and a function of
    (seed, momentum, component) only."""
    from overlap_b200.inputs import counter_gaussians

    g = counter_gaussians((16, 16, 16), 8, 11).reshape(-1)
    assert abs(g.mean()) < 0.01 and abs(g.var() - 1.0) < 0.01
    assert abs(np.corrcoef(g[:-1], g[1:])[0, 1]) < 0.01
    a = counter_gaussians((4, 4, 4), 3, 5)
    assert np.array_equal(a, counter_gaussians((4, 4, 4), 3, 5))
    assert not np.array_equal(a, counter_gaussians((4, 4, 4), 3, 6))
