"""The restated functionals (libxc is not vendored by the reference): the
potentials must be the derivatives of the energy density, checked by central
finite differences, and limiting values must match the closed forms."""
import math

import numpy as np
import pytest

from oracle.oracle import xc_point

RHOS = [1e-5, 3e-4, 0.01, 0.1, 0.7, 3.0]


@pytest.mark.parametrize("xc", [0, 1, 2])
@pytest.mark.parametrize("rho", RHOS)
def test_vrho_is_derivative(xc, rho):
    sigma = 0.3 * rho ** (8.0 / 3.0) if xc == 2 else 0.0
    h = 1e-6 * rho
    ep = xc_point(xc, rho + h, sigma)[0]
    em = xc_point(xc, rho - h, sigma)[0]
    v = xc_point(xc, rho, sigma)[1]
    assert abs((ep - em) / (2 * h) - v) < 1e-6 * max(1.0, abs(v))


@pytest.mark.parametrize("rho", RHOS)
@pytest.mark.parametrize("s2", [0.01, 0.5, 4.0])
def test_vsigma_is_derivative(rho, s2):
    kf = (3 * math.pi ** 2 * rho) ** (1 / 3)
    sigma = s2 * 4 * kf * kf * rho * rho
    h = 1e-3 * sigma
    ep = xc_point(2, rho, sigma + h)[0]
    em = xc_point(2, rho, sigma - h)[0]
    vs = xc_point(2, rho, sigma)[2]
    assert abs((ep - em) / (2 * h) - vs) < 1e-5 * abs(vs)


def test_slater_exchange_closed_form():
    # PZ = Slater + PZ81 correlation; at high density correlation is small
    rho = 1.0
    ex = -0.75 * (3 / math.pi) ** (1 / 3) * rho ** (4 / 3)
    e = xc_point(1, rho, 0.0)[0]
    assert ex - 0.1 < e < ex


def test_pbe_reduces_to_lda_exchange_plus_pw92():
    # at sigma = 0 PBE is Slater exchange + PW92 correlation; compare with PZ81 loosely
    for rho in (0.01, 0.1, 1.0):
        e_pbe = xc_point(2, rho, 0.0)[0]
        e_pz = xc_point(1, rho, 0.0)[0]
        assert abs(e_pbe - e_pz) < 2e-3 * abs(e_pz)


def test_teter93_matches_pz_at_moderate_density():
    for rho in (0.01, 0.1, 1.0):
        assert abs(xc_point(0, rho, 0)[0] - xc_point(1, rho, 0)[0]) < 3e-3 * abs(xc_point(1, rho, 0)[0])
