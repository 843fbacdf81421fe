"""Integer setup work is bit-exact: the library's G half-sphere order (with
the EPSGX tie-break, gvectors.f90:231-252), grid indices and the compressed
ray maps (fft_interface.f90:262-343) against the oracle, without a GPU."""
import numpy as np
import pytest

from amdkiit_b200 import configs
from amdkiit_b200.engine import host_gvectors
from oracle.oracle import Oracle
from tests.helpers import load_fixture

SYSTEMS = {
    "water1_mt": lambda: load_fixture("water1_mt"),
    "si_fcc_mt": lambda: load_fixture("si_fcc_mt"),
    "small_water": configs.small_water,
    "water1": configs.water1,
    "si64": configs.si64,
    "water32": configs.water32,
    "o2_angstrom_cell": lambda: load_fixture("o2_singlet"),
    "h2_upf_90": lambda: load_fixture("h2_upf"),
}


@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_gvectors_bit_exact(name):
    s = SYSTEMS[name]()
    g = host_gvectors(s)
    o = Oracle(s, 0).gvectors()
    for k in ("ngpw", "ngrho", "ngrays", "nhrays", "nr"):
        assert g[k] == o[k], k
    for k in ("inyh", "mapp", "mapm"):
        assert np.array_equal(g[k], o[k]), k
    # the floating point tables are recomputed identically (same operations)
    assert np.array_equal(g["hg"], o["hg"])
    assert np.array_equal(g["gvec"], o["gvec"])


def test_gsphere_properties():
    """Sorted by |G|, PW sphere first, G=0 first, maps inside the ray buffer."""
    s = configs.water1()
    g = host_gvectors(s)
    hg = g["hg"]
    assert hg[0] == 0.0 and np.all(np.diff(hg) >= -1e-12 * hg[1:])
    assert hg[: g["ngpw"]].max() <= hg[g["ngpw"]:].min()
    n1 = g["nr"][0] + (g["nr"][0] + 1) % 2
    assert g["mapp"].min() >= 1 and g["mapp"].max() <= g["nhrays"] * n1
    assert g["mapp"][0] == g["mapm"][0]
    assert len(np.unique(g["mapp"])) == g["ngrho"]
