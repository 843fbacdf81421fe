"""Golden outputs of the CPU restatement (the oracle) at full size.

For the reference's 32-water run (water32_mt.npz: MT psp, Teter93, 80 Ry,
108^3, 128 bands) the oracle is converged from the seeded start the tests use
(tests/helpers.start_coefficients) to GEMAX < the reference's GRAD_CUTOFF
(1e-6), and its total energy and components, ionic forces and subspace
eigenvalues are written to oracle_water32_mt.json.  About 40 minutes on 8
cores.  The 2-water run (water2_mt, 8 bands, GRAD_CUTOFF 1e-7) takes a few
minutes.  Run from the repository root:
    python tests/golden/make_oracle_fixtures.py [water32_mt|water2_mt]
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle.oracle import Oracle  # noqa: E402
from tests.helpers import load_fixture, oracle_eigenvalues, start_coefficients  # noqa: E402

GCUT = {"water32_mt": 1e-6, "water2_mt": 1e-7}


def main(name="water32_mt"):
    s = load_fixture(name)
    o = Oracle(s, 0)
    g = o.gvectors()
    o.set_wfn(start_coefficients(g["hg"][: o.ngpw], o.d("tpiba"), o.nstate))
    assert o.ortho() == 0
    t0 = time.time()
    for it in range(1, 601):
        conv = o.scf_iteration(it, GCUT[name])
        print(it, f"{time.time() - t0:.0f}s", o.d("gemax"), o.d("etotal"), flush=True)
        if conv:
            break
    assert conv == 1, "no convergence"
    out = dict(system=name, gcut=GCUT[name], iterations=it, energies=o.energies(),
               forces=np.concatenate([o.force()[i, :k] for i, k in enumerate(s.na)]).tolist())
    out["eigenvalues"] = oracle_eigenvalues(o).tolist()
    with open(os.path.join(HERE, f"oracle_{name}.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("energy", out["energies"]["etotal"], "iterations", it)


if __name__ == "__main__":
    main(*sys.argv[1:])
