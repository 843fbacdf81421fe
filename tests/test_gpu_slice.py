"""Integer-slice tensor-core GEMMs (int8 tcgen05, four 7-bit digits per
value, exact int32 accumulation) of the mixed path against the DGEMM/DTRMM
path on the same wavefunctions: the orthonormalisation, one CG iteration
(Lambda, C2 -= C0 Lambda, S, C0 U^-1) and a converged energy."""
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
    monkeypatch.delenv("AMDK_SLICE", raising=False)
    ref = Engine(system, prec)
    monkeypatch.setenv("AMDK_SLICE", "1")
    e = Engine(system, prec)
    monkeypatch.delenv("AMDK_SLICE")
    g = ref.gvectors()
    c = start_coefficients(g["hg"][: ref.ngpw], 2 * np.pi / system.alat, ref.nstate, 5)
    for x in (ref, e):
        x.set_wfn(c)
    return ref, e


SYSTEMS = {"water1": lambda: configs.small_water(xc=XC_PBE),
           "cluster5": lambda: configs.cluster(5, 18.0, 905, ecut=20.0),
           "water32": configs.water32}


@pytest.mark.parametrize("name", list(SYSTEMS))
def test_slice_ortho_matches_dgemm(name, monkeypatch):
    ref, e = engines(SYSTEMS[name](), monkeypatch)
    for x in (ref, e):
        x.ortho()
    assert rel(e.get_wfn(), ref.get_wfn()) < 1e-7


@pytest.mark.parametrize("name", ["water1", "water32"])
def test_slice_cg_iteration_matches_dgemm(name, monkeypatch):
    ref, e = engines(SYSTEMS[name](), monkeypatch)
    for x in (ref, e):
        x.ortho()
    for it in (1, 2):
        ra = ref.scf_iteration(it, 1e-7)
        rb = e.scf_iteration(it, 1e-7)
        assert abs(ra[1] - rb[1]) < 1e-6 * abs(ra[1]), it
        assert abs(ra[0]["etotal"] - rb[0]["etotal"]) < 1e-8 * abs(ra[0]["etotal"]), it
    assert rel(e.get("c2"), ref.get("c2")) < 1e-6
    assert rel(e.get_wfn(), ref.get_wfn()) < 1e-7


def test_slice_fp64_engine_keeps_dgemm(monkeypatch):
    """The FP64 path never takes the slice GEMMs: bit-identical results."""
    ref, e = engines(configs.small_water(), monkeypatch, prec=FP64)
    for x in (ref, e):
        x.ortho()
    assert np.array_equal(e.get_wfn(), ref.get_wfn())


def test_slice_mixed_converged_energy_matches_fp64(monkeypatch):
    s = configs.small_water(xc=XC_PBE)
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
