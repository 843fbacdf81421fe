"""Golden outputs of the CPU restatement (the oracle) at full size.

Each system is converged by the oracle from the seeded start the tests use
(tests/helpers.start_coefficients) to GEMAX < its gradient cutoff, and its
total energy and components, ionic forces and subspace eigenvalues are
written to oracle_<name>.json.  Systems:
  water32_mt  the reference's 32-water run (MT psp, Teter93, 80 Ry, 108^3,
              128 bands), GRAD_CUTOFF 1e-6; about 40 minutes on 8 cores
  water2_mt   the reference's 2-water run (8 bands), 1e-7; a few minutes
  water32     the 32-water benchmark system (GTH, PBE, 70 Ry, 100^3, 128
              bands), 1e-6; about an hour on 8 cores
  water1      the single-water benchmark system (GTH, LDA-PZ, 70 Ry, 64^3,
              4 bands), CG to 1e-7 then forces; a minute
  o2_triplet  the reference's open-shell O2 triplet (MT psp, Teter93, 80 Ry,
              60^3, 5 + 7 bands), 1e-7; a minute
Run from the repository root:
    python tests/golden/make_oracle_fixtures.py <name>
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
from amdkiit_b200 import configs  # noqa: E402
from tests.helpers import load_fixture, oracle_eigenvalues, start_coefficients  # noqa: E402

GCUT = {"water32_mt": 1e-6, "water2_mt": 1e-7, "water32": 1e-6, "water1": 1e-7, "o2_triplet": 1e-7}


def system(name):
    """The reference runs come from their npz fixtures, the benchmark systems
    from amdkiit_b200.configs."""
    if name.endswith("_mt") or name.startswith("o2_"):
        return load_fixture(name)
    return configs.BY_NAME[name]()


def main(name="water32_mt"):
    s = system(name)
    o = Oracle(s, 0)
    g = o.gvectors()
    o.set_wfn(start_coefficients(g["hg"][: o.ngpw], o.d("tpiba"), o.nstate))
    assert o.ortho() == 0
    t0 = time.time()
    for it in range(1, 2001):
        conv = o.scf_iteration(it, GCUT[name])
        print(it, f"{time.time() - t0:.0f}s", o.d("gemax"), o.d("etotal"), flush=True)
        if conv:
            break
    assert conv == 1, "no convergence"
    out = dict(system=name, gcut=GCUT[name], iterations=it, energies=o.energies(),
               forces=np.concatenate([o.force()[i, :k] for i, k in enumerate(s.na)]).tolist())
    out["eigenvalues"] = oracle_eigenvalues(o, s.multiplicity).tolist()
    with open(os.path.join(HERE, f"oracle_{name}.json"), "w") as f:
        json.dump(out, f, indent=1)
    print("energy", out["energies"]["etotal"], "iterations", it)


if __name__ == "__main__":
    main(*sys.argv[1:])
