"""Integer-slice tensor-core GEMMs (int8 tcgen05, four 7-bit digits per
value, exact int32 accumulation) of the mixed path against the DGEMM/DTRMM
path on the same wavefunctions: the orthonormalisation, two CG iterations
(Lambda, C2 -= C0 Lambda, S, C0 U^-1) and a converged energy.  Each operand
value keeps 28 bits relative to its band's largest, so single products are
FP32-accurate or better; the bars below are FP32-level (the mixed path's
FFTs are FP32) and the converged energy, after the FP64 refinement, is held
to the FP64 path's 1e-7 Ha/atom."""
import numpy as np
import pytest

from amdkiit_b200 import configs
from amdkiit_b200.engine import FP64, MIXED, Engine
from amdkiit_b200.inputs import XC_PBE
from tests.helpers import start_coefficients

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def engines(system, monkeypatch, prec=MIXED):
    """(DGEMM engine, slice-GEMM engine, the default) on the same start."""
    monkeypatch.setenv("AMDK_NO_SLICE", "1")
    ref = Engine(system, prec)
    monkeypatch.delenv("AMDK_NO_SLICE")
    e = Engine(system, prec)
    g = ref.gvectors()
    c = start_coefficients(g["hg"][: ref.ngpw], 2 * np.pi / system.alat, ref.nstate, 5)
    for x in (ref, e):
        x.set_wfn(c)
    return ref, e


# the slice products are used from 64 bands (16 molecules) to 128 (water32)
SYSTEMS = {"cluster16": lambda: configs.cluster(16, 18.0, 916, ecut=20.0),
           "water32": configs.water32}


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_slice_ortho_matches_dgemm(name, monkeypatch):
    ref, e = engines(SYSTEMS[name](), monkeypatch)
    for x in (ref, e):
        x.ortho()
    assert rel(e.get_wfn(), ref.get_wfn()) < 1e-5


@pytest.mark.parametrize("name", ["cluster16", "water32"])
def test_slice_cg_iteration_matches_dgemm(name, monkeypatch):
    """From a random start (ill-conditioned overlap, large gradient)."""
    ref, e = engines(SYSTEMS[name](), monkeypatch)
    for x in (ref, e):
        x.ortho()
    for it in (1, 2):
        ra = ref.scf_iteration(it, 1e-7)
        rb = e.scf_iteration(it, 1e-7)
        assert abs(ra[1] - rb[1]) < 1e-3 * abs(ra[1]), it
        assert abs(ra[0]["etotal"] - rb[0]["etotal"]) < 2e-5 * abs(ra[0]["etotal"]), it
    assert rel(e.get("c2"), ref.get("c2")) < 1e-3
    assert rel(e.get_wfn(), ref.get_wfn()) < 1e-5


def test_slice_near_convergence_matches_dgemm(monkeypatch):
    """Near convergence (C0 orthonormal to rounding, small gradient) the
    slice GEMMs change the energy of a water32 CG iteration by far less than
    1e-6 Ha/atom and the gradient maximum by far less than its value."""
    s = configs.water32()
    ref, e = engines(s, monkeypatch)
    ref.ortho()
    ref.wfn_opt(300, 2e-5)
    ref.set_precision(MIXED)
    c = ref.get_wfn()
    for x in (ref, e):
        x.set_wfn(c)
        x.ortho()
    for it in (1, 2, 3):
        ra = ref.scf_iteration(it, 1e-7)
        rb = e.scf_iteration(it, 1e-7)
        assert abs(ra[0]["etotal"] - rb[0]["etotal"]) < 1e-7 * s.nat, it
        assert abs(ra[1] - rb[1]) < 1e-2 * abs(ra[1]), it


def test_slice_fp64_engine_keeps_dgemm(monkeypatch):
    """The FP64 path never takes the slice GEMMs: bit-identical results."""
    ref, e = engines(configs.small_water(), monkeypatch, prec=FP64)
    for x in (ref, e):
        x.ortho()
    assert np.array_equal(e.get_wfn(), ref.get_wfn())


def test_slice_mixed_converged_energy_matches_fp64(monkeypatch):
    s = configs.cluster(16, 18.0, 916, ecut=20.0)
    ref, e = engines(s, monkeypatch)
    e64 = Engine(s, FP64)
    e64.set_wfn(ref.get_wfn())
    for x in (e, e64):
        x.ortho()
    n64, en64, _ = e64.wfn_opt(400, 1e-7)
    nmx, enmx, _ = e.wfn_opt(400, 1e-7)
    assert n64 < 400 and nmx < 400
    assert abs(enmx["etotal"] - en64["etotal"]) < 1e-7 * s.nat
    assert np.max(np.abs(e.get("force") - e64.get("force"))) < 1e-5
