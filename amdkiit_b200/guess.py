"""Seeded initial wavefunction used by every configuration of the library.

The reference starts from an atomic-orbital guess (wfn_initialize.f90:4);
the library starts every run from seeded complex Gaussian coefficients damped
by 1/(1+|G|^2) (|G|^2 in bohr^-2), with Im c(G=0) = 0, which the caller then
orthonormalises (ortho_gs, wfn_initialize.f90:448-499).
"""
import numpy as np


def initial_coefficients(hg_bohr2: np.ndarray, nstate: int, seed: int = 1234) -> np.ndarray:
    """(nstate, ngpw) complex128; hg_bohr2 = |G|^2 of the PW sphere in bohr^-2."""
    rng = np.random.default_rng(seed)
    ngpw = hg_bohr2.shape[0]
    re = rng.standard_normal((nstate, ngpw))
    im = rng.standard_normal((nstate, ngpw))
    c = (re + 1j * im) / (1.0 + hg_bohr2)[None, :]
    c[:, 0] = c[:, 0].real
    return np.ascontiguousarray(c)
