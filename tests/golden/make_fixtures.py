"""Generate the golden fixtures from the reference's committed test runs.

Reads AMDKIIT's tests/<case>/ directories (input.yaml, xyz, pseudopotential
files and the amdkiit.out of the committed run) and writes, per case,
  <case>.npz   the parsed system (cell, positions, pseudopotential tables)
  golden.json  the energies the reference printed (eprint.f90:1-14), the
               per-rank G-vector tables summed over ranks (gvectors.f90:315-325),
               and for the 32-water MD run every tenth frame of its trajectory
               and its per-step energies
Run from the repository root:  python tests/golden/make_fixtures.py /path/to/AMDKIIT
"""
from __future__ import annotations

import json
import os
import re
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from amdkiit_b200.inputs import load_reference_input  # noqa: E402

CASES = {
    "water1_mt": "tests/1_water/wf_opt",
    "water2_mt": "tests/2_water/wf_opt",
    "water32_mt": "tests/32_water/wf_opt",
    "si_fcc_mt": "tests/bulk_si/single_point",
    # open shell (LSD): O2 singlet and triplet, MT psp, Teter93
    "o2_singlet": "tests/O2/singlet_sp_cube",
    "o2_triplet": "tests/O2/triplet_sp_cube",
}
KEYS = {"TOTAL ENERGY": "etotal", "KINETIC ENERGY": "eke", "ELECTROSTATIC ENERGY": "estat",
        "SELF ENERGY CONTRIBUTION": "eself", "OVERLAP ENERGY CONTRIBUTION": "esr", "LOCAL PP ENERGY": "eloc",
        "NON LOCAL PP ENERGY": "enl", "EXCHANGE CORRELATION ENERGY": "exc"}


def parse_out(path):
    txt = open(path).read()
    e = {}
    for k, v in KEYS.items():
        m = re.findall(r"#\s+%s\s+=\s+([-0-9.]+)" % re.escape(k), txt)
        if m:
            e[v] = float(m[-1])
    rows = re.findall(r"^\s+\d+\s+(\d+)\s+(\d+)\s+\d+\s+(\d+)\s+(\d+)\s+(\d+)\s+(\d+)\s+\d+\s*$", txt, re.M)
    g = {}
    if rows:
        a = np.array(rows, dtype=np.int64)
        g = dict(ngpw=int(a[:, 0].sum()), ngrho=int(a[:, 1].sum()), ny=int(a[0, 2]), nz=int(a[0, 3]),
                 ngrays=int(a[:, 4].sum()), nhrays=int(a[:, 5].sum()))
    iters = re.findall(r"^#\s+(\d+)\s+-?[0-9.]+\s", txt, re.M)
    return e, g, (int(iters[-1]) if iters else None)


def parse_md_start_forces(path):
    """The ionic forces of the converged start of an MD run: the first
    ATOM / COORDINATES / FORCES table after END OF FORCES INITIALIZATION
    (molecular_dynamics.f90:92-95 prints it, 4 significant figures)."""
    txt = open(path).read()
    txt = txt[txt.index("END OF FORCES INITIALIZATION"):]
    num = r"(-?[0-9.]+(?:E[-+]?\d+)?)"
    rows = re.findall(r"^\s+(\d+)\s+([A-Z][a-z]?)" + (r"\s+" + num) * 6 + r"\s*$", txt, re.M)
    out, seen = [], set()
    for r in rows:
        i = int(r[0])
        if i in seen:
            break
        seen.add(i)
        out.append([float(v) for v in r[2:]])
    a = np.array(out)
    return a[:, :3], a[:, 3:]


# cases whose committed run left only the per-iteration energy file (no
# amdkiit.out): the last line of SP_ENERGY.dat is the converged total energy
ENERGY_ONLY = {"h2_upf": ("tests/H2_upf", "SP_ENERGY.dat")}


def parse_sp_energy(path):
    """Last line of SP_ENERGY.dat: iteration, E_tot (6 decimals), time."""
    last = [ln for ln in open(path).read().split("\n") if ln.strip()][-1]
    return float(last.split()[1])


# G-sphere / ray counts only (none at present)
GSPHERE_ONLY = {}

MD_FORCES = {"water32_mt": "tests/32_water/md", "water1_mt": "tests/1_water/md"}
GEO_GRADIENTS = {"water1_mt": "tests/1_water/geo_opt/atom_force.dat",
                 "water2_mt": "tests/2_water/geo_opt/atom_force.dat",
                 "si_fcc_mt": "tests/bulk_si/geo_opt/atom_force.dat"}


# the committed MD run whose trajectory the BOMD driver is compared with:
# frames kept (every MD_FRAME_STRIDE-th, and frame 1, which with frame 0
# fixes the initial velocities), all MD_ENERGY.dat rows
MD_TRAJECTORY = {"water32_mt": "tests/32_water/md"}
MD_FRAME_STRIDE = 10


def parse_md_trajectory(dirname):
    """MD_TRAJECTORY.xyz (write_md_trajectory, md_tools.f90:152-172: per
    frame the atom count, 'MD STEP= n', then per atom the symbol, position
    (Angstrom) and velocity (a.u.), 6 decimals) and MD_ENERGY.dat
    (write_md_energy, md_tools.f90:174-184: step, temperature, KS energy,
    KS + kinetic energy, CPU time)."""
    lines = open(os.path.join(dirname, "MD_TRAJECTORY.xyz")).read().split("\n")
    frames = {}
    i = 0
    while i < len(lines) and lines[i].strip():
        nat = int(lines[i].split()[0])
        step = int(lines[i + 1].split()[-1])
        rows = [ln.split() for ln in lines[i + 2:i + 2 + nat]]
        frames[step] = dict(symbols=[r[0] for r in rows], pos=[[float(v) for v in r[1:4]] for r in rows],
                            vel=[[float(v) for v in r[4:7]] for r in rows])
        i += 2 + nat
    keep = sorted(k for k in frames if k % MD_FRAME_STRIDE == 0 or k == 1)
    energy = [[float(v) for v in ln.split()[:4]]
              for ln in open(os.path.join(dirname, "MD_ENERGY.dat")).read().split("\n") if ln.strip()]
    return dict(symbols=frames[0]["symbols"], frames={str(k): frames[k]["pos"] for k in keep},
                vel0=frames[0]["vel"], energy=energy, nsteps=max(frames))


def parse_first_gradient(path):
    """The first block of a geometry optimisation's atom_force.dat: atom
    count, ENERGY= E step, then one line per atom with dE/dR (Ha/bohr, 16
    digits), at the run's input geometry."""
    lines = open(path).read().split("\n")
    nat = int(lines[0].split()[0])
    energy = float(lines[1].split()[1])
    grad = [[float(v) for v in ln.split()[1:4]] for ln in lines[2:2 + nat]]
    return energy, grad


def save_system(path, s):
    d = dict(a_cell=s.a_cell, alat=s.alat, symmetry=s.symmetry, ecut=s.ecut, xc=s.xc, nsp=len(s.species),
             multiplicity=s.multiplicity)
    for i, (sp, pos) in enumerate(zip(s.species, s.positions)):
        d[f"pos{i}"] = pos
        d[f"sp{i}_meta"] = np.array([sp.z, sp.zv, sp.kind, sp.lmax, sp.l_local, sp.skip, int(sp.tkb), sp.upf_lmax])
        d[f"sp{i}_label"] = np.array(sp.label)
        for k in ("rr", "vr", "rps", "rab", "vloc", "beta", "beta_l", "dij"):
            v = getattr(sp, k)
            if v is not None:
                d[f"sp{i}_{k}"] = v
    np.savez_compressed(path, **d)


def main(root):
    golden = {}
    for name, rel in CASES.items():
        d = os.path.join(root, rel)
        s = load_reference_input(d)
        save_system(os.path.join(HERE, name + ".npz"), s)
        e, g, it = parse_out(os.path.join(d, "amdkiit.out"))
        golden[name] = dict(energies=e, gvectors=g, iterations=it, source=rel + "/amdkiit.out")
        if name in MD_FORCES:
            # the MD run starts from the same input geometry; its first force
            # table is the converged force at that geometry
            md = MD_FORCES[name] + "/amdkiit.out"
            pos, frc = parse_md_start_forces(os.path.join(root, md))
            golden[name]["md_start"] = dict(positions=pos.tolist(), forces=frc.tolist(), source=md)
        if name in MD_TRAJECTORY:
            tr = parse_md_trajectory(os.path.join(root, MD_TRAJECTORY[name]))
            tr["source"] = MD_TRAJECTORY[name] + "/MD_TRAJECTORY.xyz, MD_ENERGY.dat"
            golden[name]["md_trajectory"] = tr
        if name in GEO_GRADIENTS:
            # the geometry optimisation starts from the same input; its first
            # gradient is taken at the converged start geometry
            en, grad = parse_first_gradient(os.path.join(root, GEO_GRADIENTS[name]))
            golden[name]["geo_start"] = dict(energy=en, gradient=grad, source=GEO_GRADIENTS[name])
        print(name, e.get("etotal"), g)
    for name, rel in GSPHERE_ONLY.items():
        s = load_reference_input(os.path.join(root, rel))
        save_system(os.path.join(HERE, name + ".npz"), s)
        _, g, _ = parse_out(os.path.join(root, rel, "amdkiit.out"))
        golden[name] = dict(gvectors=g, source=rel + "/amdkiit.out")
        print(name, g)
    for name, (rel, efile) in ENERGY_ONLY.items():
        s = load_reference_input(os.path.join(root, rel))
        save_system(os.path.join(HERE, name + ".npz"), s)
        golden[name] = dict(energies={"etotal": parse_sp_energy(os.path.join(root, rel, efile))},
                            energy_decimals=6, source=rel + "/" + efile)
        print(name, golden[name]["energies"]["etotal"])
    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(golden, f, indent=1, sort_keys=True)


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_fixtures.py <path to the AMDKIIT checkout>")
    main(sys.argv[1])
