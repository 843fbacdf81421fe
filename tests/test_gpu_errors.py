"""Failure detection on the GPU path, with no GPU fault: the status codes of
the C-ABI for inputs the reference STOPs on or cannot handle, and a context
that stays usable after each of them.

- a band of zeros makes the overlap singular: ortho_gs's Cholesky meets a
  zero pivot (UINV STOPs there, wfn_initialize.f90:514-528) -> NOT_SPD;
- a NaN coefficient reaches the total energy -> NONFINITE;
- a CG step number below 1 -> BADARG."""
import numpy as np
import pytest

from amdkiit_b200 import configs
from amdkiit_b200.engine import FP64, MIXED, AmdkError, Engine
from tests.helpers import start_coefficients

pytestmark = pytest.mark.gpu


def _engine(prec):
    s = configs.small_water()
    e = Engine(s, prec)
    g = e.gvectors()
    c = start_coefficients(g["hg"][: e.ngpw], 2 * np.pi / s.alat, e.nstate)
    return e, c


def _usable(e, c):
    e.set_wfn(c)
    e.ortho()
    en, gm, _ = e.scf_iteration(1, 1e-6)
    assert np.isfinite(en["etotal"]) and np.isfinite(gm)


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_singular_overlap_is_not_spd(prec):
    e, c = _engine(prec)
    bad = c.copy()
    bad[1] = 0.0
    e.set_wfn(bad)
    with pytest.raises(AmdkError, match=r"\(-4\)"):
        e.ortho()
    _usable(e, c)


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_nan_coefficient_is_nonfinite(prec):
    e, c = _engine(prec)
    e.set_wfn(c)
    e.ortho()
    bad = e.get_wfn()
    bad[0, 3] = np.nan
    e.set_wfn(bad)
    e.density()
    e.potential()
    with pytest.raises(AmdkError, match=r"\(-5\)"):
        e.energy()
    _usable(e, c)


def test_step_below_one_is_badarg():
    e, c = _engine(FP64)
    e.set_wfn(c)
    e.ortho()
    with pytest.raises(AmdkError, match=r"\(-1\)"):
        e.scf_iteration(0, 1e-6)
    _usable(e, c)
