"""Shared helpers for the tests: golden fixtures and paired oracle/engine runs."""
from __future__ import annotations

import json
import os

import numpy as np

from amdkiit_b200.guess import initial_coefficients
from amdkiit_b200.inputs import Species, System

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def golden():
    with open(os.path.join(GOLDEN, "golden.json")) as f:
        return json.load(f)


def load_fixture(name: str) -> System:
    d = np.load(os.path.join(GOLDEN, name + ".npz"))
    species, pos = [], []
    for i in range(int(d["nsp"])):
        z, zv, kind, lmax, l_local, skip, tkb, upf_lmax = d[f"sp{i}_meta"]
        kw = {}
        for k in ("rr", "vr", "rps", "rab", "vloc", "beta", "beta_l", "dij"):
            if f"sp{i}_{k}" in d:
                kw[k] = d[f"sp{i}_{k}"]
        species.append(Species(label=str(d[f"sp{i}_label"]), z=int(z), zv=float(zv), kind=int(kind),
                               lmax=int(lmax), l_local=int(l_local), skip=int(skip), tkb=bool(tkb),
                               upf_lmax=int(upf_lmax), **kw))
        pos.append(d[f"pos{i}"])
    mult = int(d["multiplicity"]) if "multiplicity" in d else 0
    return System(a_cell=d["a_cell"], alat=float(d["alat"]), symmetry=int(d["symmetry"]), ecut=float(d["ecut"]),
                  species=species, positions=pos, xc=int(d["xc"]), name=name, multiplicity=mult)


def start_coefficients(hg_pw: np.ndarray, tpiba: float, nstate: int, seed: int = 1234) -> np.ndarray:
    return initial_coefficients(hg_pw * tpiba * tpiba, nstate, seed)


class OracleEngine:
    """The CPU restatement behind the small Engine interface BOMD uses."""

    def __init__(self, system, seed: int = 1234):
        from oracle.oracle import Oracle
        self.system = system
        self.o = Oracle(system, 0)
        g = self.o.gvectors()
        self.o.set_wfn(start_coefficients(g["hg"][: self.o.ngpw], self.o.d("tpiba"), self.o.nstate, seed))

    def ortho(self):
        assert self.o.ortho() == 0

    def set_positions(self, atco):
        self.o.set_positions(atco)

    def wfn_opt(self, max_step, gcut):
        n = self.o.wfn_opt(max_step, gcut)
        return n, {"etotal": self.o.d("etotal")}, self.o.d("gemax")

    def get(self, name):
        assert name == "force"
        return self.o.force()


def oracle_eigenvalues(o, multiplicity: int = 0) -> np.ndarray:
    """Subspace eigenvalues (Ha) at the oracle's current C0: the stages of one
    iteration up to H|psi> (C2 = -f_i H|psi_i>, f_i = 2, or 1 open shell),
    then the same diagonalisation the engine uses (per spin block when open
    shell, spin 1 first)."""
    from amdkiit_b200.engine import subspace_eigenvalues
    for r in ("eval_density", "rhor2g", "eval_pot", "cal_vpot_ex", "pp_energy", "vpsi", "fnonloc"):
        o.call(r)
    if multiplicity > 0:
        nu = (o.nstate - (multiplicity - 1)) // 2
        c, hc = o.c0(), -o.c2()
        return np.concatenate([subspace_eigenvalues(c[:nu], hc[:nu]), subspace_eigenvalues(c[nu:], hc[nu:])])
    return subspace_eigenvalues(o.c0(), -0.5 * o.c2())


def golden_oracle(name: str) -> dict:
    """Converged oracle outputs at full size (tests/golden/make_oracle_fixtures.py)."""
    with open(os.path.join(GOLDEN, f"oracle_{name}.json")) as f:
        return json.load(f)
