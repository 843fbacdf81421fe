"""Host logic of the BOMD driver that needs no GPU: the always-stable
predictor weights (Kolafa, J. Comput. Chem. 25, 335 (2004))."""
import numpy as np
import pytest

from amdkiit_b200.md import aspc_coefficients


def test_aspc_known_weights():
    assert np.allclose(aspc_coefficients(1), [1.0])
    assert np.allclose(aspc_coefficients(2), [2.0, -1.0])
    assert np.allclose(aspc_coefficients(3), [2.5, -2.0, 0.5])
    assert np.allclose(aspc_coefficients(4), [2.8, -2.8, 1.2, -0.2])
    assert np.allclose(aspc_coefficients(5), [3.0, -24 / 7, 27 / 14, -4 / 7, 1 / 14])


@pytest.mark.parametrize("n", range(2, 9))
def test_aspc_weights_extrapolate_linear_trajectories_exactly(n):
    w = aspc_coefficients(n)
    t = -np.arange(n, dtype=float)  # C0(t), C0(t-dt), ... at t = 0, -1, ...
    assert abs(w.sum() - 1.0) < 1e-12
    assert abs(w @ t - 1.0) < 1e-12  # a(t) = t is predicted at t = +1
