"""Several systems iterated together (amdk_ensemble_iteration: each CG
segment of all members as one CUDA graph launch of the members' own segment
graphs) give bit for bit what each system gives iterated alone, in both
precisions (launch shapes from the model, AMDK_NO_TUNE=1, so both sides
sum in the same order)."""
import numpy as np
import pytest

from amdkiit_b200 import configs
from amdkiit_b200.engine import FP64, MIXED, Engine, Ensemble
from tests.helpers import start_coefficients

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prec", [FP64, MIXED])
def test_ensemble_matches_members_alone(prec, monkeypatch):
    monkeypatch.setenv("AMDK_NO_TUNE", "1")
    systems = [configs.cluster(n, L, 500 + n, ecut=30.0) for n, L in ((1, 12.0), (3, 13.5), (2, 14.0))]
    alone, together, starts = [], [], []
    for s in systems:
        a, b = Engine(s, prec), Engine(s, prec)
        g = a.gvectors()
        c = start_coefficients(g["hg"][: a.ngpw], 2 * np.pi / s.alat, a.nstate)
        for e in (a, b):
            e.set_wfn(c)
            e.ortho()
        alone.append(a)
        together.append(b)
    ens = Ensemble(together)
    for it in range(1, 9):
        # a loose cutoff turns the forces segment on after a few iterations
        ref = [e.scf_iteration(it, 5e-2) for e in alone]
        en, gm, cv = ens.iteration([it] * len(systems), 5e-2)
        for i in range(len(systems)):
            assert en[i]["etotal"] == ref[i][0]["etotal"] and gm[i] == ref[i][1], (it, i)
    assert ens.last_ms() > 0
    for a, b in zip(alone, together):
        assert np.array_equal(a.get_wfn(), b.get_wfn())
        assert np.array_equal(a.get("force"), b.get("force"))
    ens.close()
