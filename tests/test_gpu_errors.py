"""Failure detection on the GPU path, with no GPU fault: the status codes of
the C-ABI for inputs the reference STOPs on or cannot handle, and a context
that stays usable after each of them.

- a band of zeros makes the overlap singular: ortho_gs's Cholesky meets a
  zero pivot (UINV STOPs there, wfn_initialize.f90:514-528) -> NOT_SPD;
- a NaN coefficient reaches the total energy -> NONFINITE;
- a CG step number below 1 -> BADARG;
- the int8 tensor-core kernels' pipeline waits made to give up at once (a
  test-only limit, amdk_options.reserved[0]; the waits that drain a block's
  own copies and MMAs keep their full limit) -> TIMEOUT, NaN in the Gram
  product, C0 left as it was, and the context goes on with the FP64
  products;
- the same for the FP64 tensor-core kernels (amdk_options.reserved[1]): the
  density and potential computed afterwards in that context equal those of
  a fresh context."""
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


def test_slice_pipeline_wait_expiry_is_timeout():
    """64 bands (16 waters): the orthonormalisation's Gram and rotation run
    on the int8 slice kernels, whose pipeline waits give up at once here."""
    s = configs.cluster(16, 18.0, 916, ecut=20.0)
    e = Engine(s, MIXED, wait_limit=-1)
    g = e.gvectors()
    c = start_coefficients(g["hg"][: e.ngpw], 2 * np.pi / s.alat, e.nstate)
    e.set_wfn(c)
    with pytest.raises(AmdkError, match=r"\(-6\)"):
        e.ortho()
    # the Gram product wrote NaN; the call stopped before rotating C0
    assert np.isnan(e.get("overlap")).any()
    assert np.array_equal(e.get_wfn(), c)
    # the same context with FP64 products (no slice kernel) runs normally
    e.set_precision(FP64)
    _usable(e, c)


def test_fp64_pipeline_wait_expiry_is_timeout():
    s = configs.small_water()
    e = Engine(s, FP64, fp64_wait_limit=-1)
    g = e.gvectors()
    c = start_coefficients(g["hg"][: e.ngpw], 2 * np.pi / s.alat, e.nstate)
    e.set_wfn(c)
    with pytest.raises(AmdkError, match=r"\(-6\)"):
        e.ortho()
    assert np.isnan(e.get("overlap")).any()
    assert np.array_equal(e.get_wfn(), c)
    # kernels other than the products still run and give the same results
    e.density()
    e.potential()
    ref = Engine(s, FP64)
    ref.set_wfn(c)
    ref.density()
    ref.potential()
    for name in ("rho", "v_pot"):
        assert np.array_equal(e.get(name), ref.get(name)), name
