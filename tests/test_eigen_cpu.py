"""Subspace eigenvalues (the 1e-5 Ha eigenvalue check is oracle vs GPU: the
reference prints none).  CPU tests of the shared diagonalisation and of
the H|psi> scaling it assumes (C2 = -f_i H|psi_i>, f_i = 2)."""
import numpy as np

from amdkiit_b200 import configs
from amdkiit_b200.engine import subspace_eigenvalues
from oracle.oracle import Oracle
from tests.helpers import oracle_eigenvalues, start_coefficients


def _real_bands(rng, n, ng):
    c = rng.normal(size=(n, ng)) + 1j * rng.normal(size=(n, ng))
    c[:, 0] = c[:, 0].real
    return c


def test_eigenvalues_invariant_under_band_rotation():
    """A real orthogonal mix of the bands (and of H|bands>) spans the same
    subspace: same eigenvalues.  Also H = diag(e) on orthonormal bands."""
    rng = np.random.default_rng(3)
    n, ng = 6, 400
    c = _real_bands(rng, n, ng)
    # orthonormalise in the Gamma-point inner product
    s = 2.0 * np.real(np.conj(c) @ c.T) - np.outer(c[:, 0].real, c[:, 0].real)
    c = np.linalg.solve(np.linalg.cholesky(s), c)
    e = np.sort(rng.normal(size=n))
    hc = e[:, None] * c
    assert np.allclose(subspace_eigenvalues(c, hc), e, atol=1e-12)
    q, _ = np.linalg.qr(rng.normal(size=(n, n)))
    assert np.allclose(subspace_eigenvalues(q @ c, q @ hc), e, atol=1e-12)
    # non-orthonormal bands: the generalised problem gives the same values
    m = np.eye(n) + 0.1 * rng.normal(size=(n, n))
    assert np.allclose(subspace_eigenvalues(m @ c, m @ hc), e, atol=1e-10)


def test_band_energy_identity():
    """2 sum_i e_i = E_kin + E_nl + integral V_pot rho at any orthonormal C0:
    checks the -C2/2 scaling of H|psi> against the energies."""
    s = configs.small_water()
    o = Oracle(s, 0)
    g = o.gvectors()
    o.set_wfn(start_coefficients(g["hg"][: o.ngpw], o.d("tpiba"), o.nstate))
    assert o.ortho() == 0
    ev = oracle_eigenvalues(o)
    o.call("e_total")
    rho, v = o.real_grid("rho"), o.real_grid("v_pot")
    rhs = o.d("eke") + o.d("enl") + o.d("omega") / rho.size * np.sum(rho * v)
    assert abs(2.0 * ev.sum() - rhs) < 1e-9 * abs(rhs)
