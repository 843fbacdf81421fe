"""Write the benchmark systems in the reference's own input form.

For each configuration this writes a directory that AMDKIIT's Fortran driver
reads as it reads its committed tests: ``input.yaml`` (the keys of
``source/yamlread.f90``: TASK, INITIALIZATION, OPTIMIZATION, DYNAMICS,
SYMMETRY, CUTOFF, CELL, INPUT, SPECIES, DFT), ``input_coordinate.xyz`` (each
species a contiguous run, ``yamlread.f90:360-419``) and, once, the GTH
pseudopotentials as UPF v2 files in ``pseudo/`` laid out line by line the way
``source/readupf.f90`` parses them:

- ``PP_HEADER``: one attribute per line in the reader's order
  (``readupf.f90:131-179``), ``l_max`` the highest projector channel (0 for a
  local-only species), ``number_of_proj`` 0 for H;
- ``PP_MESH`` (``PP_R``, ``PP_RAB``) and ``PP_LOCAL`` (in Ry: the reader halves
  it, ``readupf.f90:411``);
- ``PP_NONLOCAL``: ``PP_BETA.n`` (r p_l(r)) with its attribute lines in the
  order ``readupf.f90:258-275`` reads them, then ``PP_DIJ`` = 2 h (Ry, halved by
  the reader, ``readupf.f90:347``) on the line after the last beta, or right
  after ``<PP_NONLOCAL>`` when there is none (``readupf.f90:318``);
- ``PP_PSWFC``: pseudo-atomic orbitals for the reference's ATOMIC initial
  guess (GTH potentials have none: normalised Gaussians r^(l+1) exp(-a r^2)
  per valence shell stand in, used only as that starting point), and
  ``PP_RHOATOM`` = sum of occupation x chi^2.

The arrays are written with 17 significant digits, so
``inputs.load_reference_input`` reads back the same System as
``configs.py`` builds (``tests/test_reference_inputs.py``).

    python -m amdkiit_b200.write_inputs <output directory>
"""
from __future__ import annotations

import math
import os
import sys
from typing import Dict, List

import numpy as np

from . import configs
from .inputs import XC_PBE, XC_PZ, XC_TETER93, Species, System

# valence shells of the pseudo-atomic orbitals: (label, l, occupation, Gaussian exponent in bohr^-2)
SHELLS = {"H": [("1S", 0, 1.0, 0.35)], "O": [("2S", 0, 2.0, 0.8), ("2P", 1, 4.0, 0.6)],
          "Si": [("3S", 0, 2.0, 0.25), ("3P", 1, 2.0, 0.2)]}
_XC_KEYS = {XC_PZ: ("XC_LDA_X", "XC_LDA_C_PZ"), XC_PBE: ("XC_GGA_X_PBE", "XC_GGA_C_PBE")}
_LETTER = "SPDF"


def _fmt(a, per_line: int = 4) -> str:
    vals = ["%.16e" % v for v in np.asarray(a, dtype=float)]
    return "\n".join("    ".join(vals[i:i + per_line]) for i in range(0, len(vals), per_line))


def _chi(r: np.ndarray, l: int, a: float) -> np.ndarray:
    """r R(r) with R = N r^l exp(-a r^2), normalised: int (r R)^2 dr = 1."""
    norm2 = math.gamma(l + 1.5) / (2.0 * (2.0 * a) ** (l + 1.5))
    return r ** (l + 1) * np.exp(-a * r * r) / math.sqrt(norm2)


def upf_text(sp: Species) -> str:
    """A GTH species (inputs.gth_species arrays) as a UPF v2 file for readupf.f90."""
    r, n, nb = sp.rr, sp.mesh, sp.nbeta
    shells = SHELLS[sp.label]
    lmax = sp.upf_lmax - 1
    head = [
        '<UPF version="2.0.1">',
        "<PP_INFO>",
        "GTH pseudopotential (Goedecker-Teter-Hutter 1996, Hartwigsen-Goedecker-Hutter 1998)",
        "tabulated on r_i = rmin exp(i dx); written by amdkiit_b200.write_inputs",
        "</PP_INFO>",
        "<PP_HEADER",
        'generated="amdkiit_b200.write_inputs"',
        'author="amdkiit_b200"',
        'date="000000"',
        'comment="GTH"',
        'element="%s"' % sp.label,
        'pseudo_type="NC"',
        'relativistic="scalar"',
        'is_ultrasoft="F"',
        'is_paw="F"',
        'is_coulomb="F"',
        'has_so="F"',
        'has_wfc="F"',
        'has_gipaw="F"',
        'paw_as_gipaw="F"',
        'core_correction="F"',
        'functional="GTH"',
        'z_valence="%.1f"' % sp.zv,
        'total_psenergy="0.0"',
        'wfc_cutoff="0.0"',
        'rho_cutoff="0.0"',
        'l_max="%d"' % lmax,
        'l_max_rho="%d"' % (2 * lmax),
        'l_local="-1"',
        'mesh_size="%d"' % n,
        'number_of_wfc="%d"' % len(shells),
        'number_of_proj="%d"/>' % nb,
    ]
    out = head + ["<PP_MESH>", '<PP_R type="real" size="%d" columns="4">' % n, _fmt(r), "</PP_R>",
                  '<PP_RAB type="real" size="%d" columns="4">' % n, _fmt(sp.rab), "</PP_RAB>", "</PP_MESH>",
                  '<PP_LOCAL type="real" size="%d" columns="4">' % n, _fmt(2.0 * sp.vloc), "</PP_LOCAL>",
                  "<PP_NONLOCAL>"]
    for k in range(nb):
        out += ["<PP_BETA.%d" % (k + 1), 'type="real"', 'size="%d"' % n, 'columns="4"', 'index="%d"' % (k + 1),
                'label="%d%s"' % (k + 1, _LETTER[int(sp.beta_l[k])]),
                'angular_momentum="%d"' % int(sp.beta_l[k]), 'cutoff_radius_index="%d"' % n,
                'cutoff_radius="%.16e" >' % r[-1], _fmt(sp.beta[k]), "</PP_BETA.%d>" % (k + 1)]
    dij = np.asarray(sp.dij, dtype=float)[: nb * nb]
    out += ['<PP_DIJ type="real" size="%d" columns="4">' % (nb * nb), _fmt(dij) if nb else "0.0", "</PP_DIJ>",
            "</PP_NONLOCAL>", "<PP_PSWFC>"]
    rho = np.zeros(n)
    for k, (lab, l, occ, a) in enumerate(shells):
        chi = _chi(r, l, a)
        rho += occ * chi * chi
        out += ["<PP_CHI.%d" % (k + 1), 'type="real"', 'size="%d"' % n, 'columns="4"', 'index="%d"' % (k + 1),
                'occupation="%.3f"' % occ, 'pseudo_energy="0.0"', 'label="%s"' % lab, 'l="%d" >' % l, _fmt(chi),
                "</PP_CHI.%d>" % (k + 1)]
    out += ["</PP_PSWFC>", '<PP_RHOATOM type="real" size="%d" columns="4">' % n, _fmt(rho), "</PP_RHOATOM>",
            "</UPF>", ""]
    return "\n".join(out)


def yaml_text(s: System, task: str, pp_files: Dict[str, str], extra: List[str]) -> str:
    """input.yaml with the keys and defaults of yamlread.f90 (bohr units)."""
    if s.symmetry != 1:
        raise ValueError("only cubic benchmark cells are written")
    lines = ["TASK: %s" % task, "INITIALIZATION:", "  WAVEFUNCTION: ATOMIC", "OPTIMIZATION:", "  WAVEFUNCTION:",
             "    MINIMIZER: CONJUGATE_GRADIENT", "    MAX_STEPS: 800", "    GRAD_CUTOFF: %s" % extra[0]]
    lines += extra[1:]
    L = s.a_cell
    lines += ["SYMMETRY: CUBIC", "CUTOFF:", "  VALUE: %r" % float(s.ecut), "  UNIT: RYDBERG", "CELL:", "  UNIT: BOHR",
              "  DIMENSION:"] + ["    - %r" % float(L[k, k]) for k in range(3)] + \
             ["  ANGLE:", "    - 90", "    - 90", "    - 90", "INPUT:", "  COORDINATES_FILE: input_coordinate.xyz",
              "  UNIT: BOHR", "SPECIES:"]
    for i, sp in enumerate(s.species):
        top = max([int(l) for l in sp.beta_l] or [0])
        lines += ["  LABEL%d:" % (i + 1), "    ATOM: %s" % sp.label, "    PP_FILE: %s" % pp_files[sp.label],
                  "    PP_SCHEME: NONE", "    LMAX: %s" % _LETTER[top], "    LOCAL: 0"]
    if s.xc == XC_TETER93:
        lines += ["DFT:", "   XC: XC_LDA_XC_TETER93"]
    else:
        x, c = _XC_KEYS[s.xc]
        lines += ["DFT:", "   EXCHANGE: %s" % x, "   CORRELATION: %s" % c]
    return "\n".join(lines) + "\n"


def xyz_text(s: System) -> str:
    out = ["%d" % s.nat, "%s (bohr)" % s.name]
    for sp, p in zip(s.species, s.positions):
        for x in p:
            out.append("%s %r %r %r" % (sp.label, float(x[0]), float(x[1]), float(x[2])))
    return "\n".join(out) + "\n"


def benchmark_inputs() -> Dict[str, tuple]:
    """name -> (System, TASK, [GRAD_CUTOFF, extra yaml lines]) for the five configurations."""
    run = {"cfg0_water1": (configs.water1(), "WAVEFUNCTION_OPTIMIZATION", ["1.0E-007"]),
           "cfg1_si64": (configs.si64(), "WAVEFUNCTION_OPTIMIZATION", ["1.0E-006"]),
           "cfg3_water32": (configs.water32(), "MOLECULAR_DYNAMICS",
                            ["1.0E-006", "DYNAMICS:", "  TEMPERATURE: 300", "  MAX_STEPS: 200", "  TIMESTEP: 0.5"]),
           "cfg4_water128": (configs.water128(), "GEOMETRY_OPTIMIZATION",
                             ["1.0E-006", "  GEOMETRY:", "    MINIMIZER: LBFGS", "    MAX_STEPS: 100",
                              "    GRAD_CUTOFF: 5.0E-004"])}
    for k, s in enumerate(configs.ensemble()):
        run["cfg2_cluster%02d" % k] = (s, "WAVEFUNCTION_OPTIMIZATION", ["1.0E-006"])
    return run


def write_all(root: str) -> List[str]:
    """Write every configuration under root (one directory each) and the
    pseudopotentials under root/pseudo; returns the directories."""
    pseudo = os.path.join(root, "pseudo")
    os.makedirs(pseudo, exist_ok=True)
    written, dirs = set(), []
    for name, (s, task, extra) in benchmark_inputs().items():
        d = os.path.join(root, name)
        os.makedirs(d, exist_ok=True)
        files = {}
        for sp in s.species:
            fn = "%s_GTH.upf" % sp.label
            if fn not in written:
                with open(os.path.join(pseudo, fn), "w") as f:
                    f.write(upf_text(sp))
                written.add(fn)
            files[sp.label] = "../pseudo/" + fn
        with open(os.path.join(d, "input.yaml"), "w") as f:
            f.write(yaml_text(s, task, files, extra))
        with open(os.path.join(d, "input_coordinate.xyz"), "w") as f:
            f.write(xyz_text(s))
        dirs.append(d)
    return dirs


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python -m amdkiit_b200.write_inputs <output directory>")
    for d in write_all(sys.argv[1]):
        print(d)
