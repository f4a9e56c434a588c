"""The overlap eigenmodes in the U(1) background on the device
(ovl_set_qed_eigenmodes, InitialConditions::SetOverlapQEDEigenfunctions)
against the Hamiltonian the reference's own code builds
(OverlapQEDEigenfunctions::Setup's construction, run in the reference build by
ovlref_qed_hamiltonian: U(1)-only links in colour (0,0), Ritz bounds, one
Zolotarev overlap application per basis vector).

The reference's sign function is a rational approximation on its Ritz
interval, the device's the exact sign of h_W's eigenvalues, so the matrices
agree to the reference's approximation (a few 1e-8 here, bound 1e-6).
Eigenvectors are compared through what does not depend on the phase or the
basis of a degenerate level: the projector onto the negative-energy modes, and
each mode's residual as an eigenvector of the reference's matrix."""
import numpy as np
import pytest

from _oracle import have_reference, ptr, reference
from overlap_b200 import Context
from overlap_b200.inputs import u1_flux, volume

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not have_reference("overlap"), reason="reference overlap build not present")]

TOL = 1e-6
M_F, M_DW, DT = 0.05, 1.4, 0.05


def reference_hamiltonian(N, n_b):
    V = volume(N)
    D = 8 * V
    R = reference("overlap")
    R.ovlref_init(*N, 1, 0, M_F, 1.0, M_DW, 6.0, DT, 1.0, 7)
    buf, b = np.zeros(2 * D * D), np.zeros(2)
    R.ovlref_qed_hamiltonian(n_b, ptr(buf), ptr(b))
    return buf.view(np.complex128).reshape(D, D).T  # column-major -> [row, column]


@pytest.mark.parametrize("N,n_b", [((4, 4, 4), 2), ((4, 3, 5), 1)])
def test_qed_eigenmodes_match_the_reference_hamiltonian(N, n_b):
    V = volume(N)
    D = 8 * V
    H_ref = reference_hamiltonian(N, n_b)
    with Context(N=N, n_modes=D, fermion="overlap", precision="fp64", m_fermion=M_F, m_dw=M_DW, dt=DT) as ctx:
        ctx.set_u1(u1_flux(N, n_b))
        w, bad, H = ctx.set_qed_eigenmodes(hamiltonian=True)
        psi, mid = ctx.get_modes()
    assert bad == 0
    assert np.max(np.abs(H - H.conj().T)) < 1e-12
    assert np.max(np.abs(H - H_ref)) < TOL
    w_ref, v_ref = np.linalg.eigh(0.5 * (H_ref + H_ref.conj().T))
    assert np.max(np.abs(w - w_ref)) < TOL
    assert np.all(w[:D // 2] < 0) and np.all(w[D // 2:] > 0)
    # the modes as D-vectors in the reference's index site + V (spin + 4 colour)
    vecs = np.transpose(psi, (0, 2, 3, 1)).reshape(D, D).T / np.sqrt(V)  # [component, mode]: [mode][colour][spin][site]
    g = np.arange(D)
    col = np.where(g % 2 == 0, D // 2 + g // 2, D // 2 - 1 - g // 2)  # particles up, antiparticles down
    omega = w[col]
    res = np.linalg.norm(H_ref @ vecs - vecs * omega[None, :], axis=0)
    assert np.max(res) < 10 * TOL
    assert np.max(np.abs(vecs.conj().T @ vecs - np.eye(D))) < 1e-12
    # the negative-energy projector (the antiparticle modes) against the reference's
    neg = vecs[:, g % 2 == 1]
    P_ref = v_ref[:, :D // 2] @ v_ref[:, :D // 2].conj().T
    assert np.max(np.abs(neg @ neg.conj().T - P_ref)) < 10 * TOL
    # psimid = psi e^{-i omega dt / 2}
    phase = np.exp(-0.5j * omega * DT)
    assert np.max(np.abs(mid - psi * phase[:, None, None, None])) < 1e-13


def test_qed_eigenmodes_of_a_rank_slice_and_limits():
    """A context holding global modes 100-163 gets the same modes as the full
    basis; a context with modes beyond the basis is refused."""
    N = (4, 4, 4)
    D = 8 * volume(N)
    kw = dict(N=N, fermion="overlap", precision="fp64", m_fermion=M_F, m_dw=M_DW, dt=DT)
    with Context(n_modes=D, **kw) as ctx:
        ctx.set_u1(u1_flux(N, 2))
        w_full, _ = ctx.set_qed_eigenmodes()
        full = ctx.get_modes(100, 64)[0]
    with Context(n_modes=64, first_mode=100, **kw) as ctx:
        ctx.set_u1(u1_flux(N, 2))
        w, bad = ctx.set_qed_eigenmodes()
        part = ctx.get_modes()[0]
    assert bad == 0 and np.array_equal(w, w_full)
    # the same diagonalisation on the same matrix: the same vectors
    assert np.max(np.abs(part - full)) < 1e-12
    with Context(n_modes=64, first_mode=D - 32, **kw) as ctx:
        with pytest.raises(Exception):
            ctx.set_qed_eigenmodes()
