"""Input side of the driver: the reference's input formats and the seeded systems.

This mirrors what AMDKIIT's Fortran driver does before its first SCF
iteration (``source/init_module.f90:3-162``): it reads the YAML input
(``source/yamlread.f90``), the xyz coordinates (``yamlread.f90:360-419``), the
pseudopotential files (``source/readpsp.f90``, ``source/readupf.f90``) and
builds the cell (``source/set_cell.f90:4-131``).  GTH pseudopotentials, which
the reference can only read as UPF v2 files, are tabulated here on a
logarithmic mesh into the same arrays the UPF reader fills.

Units follow the reference: bohr and Hartree, cutoffs in Rydberg.
"""
from __future__ import annotations

import math
import os
import re
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

ANGS2BOHR = 1.0 / 0.529177210859          # constants.f90:19
AMU_AU = 1822.888485                      # constants.f90:8

XC_TETER93, XC_PZ, XC_PBE = 0, 1, 2
PP_PSP, PP_UPF = 0, 1

# atomic masses by Z (system_data_types.f90:128-148, first 20 elements)
_ATWT = [1.00797, 4.0026, 6.939, 9.0122, 10.811, 12.01115, 14.0067, 15.9994,
         18.9984, 20.183, 22.9898, 24.312, 26.9815, 28.086, 30.9738, 32.064,
         35.453, 39.948, 39.102, 40.080]
_SYMBOLS = ["H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg",
            "Al", "Si", "P", "S", "Cl", "Ar", "K", "Ca"]


def atomic_mass(z: int) -> float:
    return _ATWT[z - 1]


def symbol_to_z(sym: str) -> int:
    return _SYMBOLS.index(sym.strip().capitalize()) + 1


@dataclass
class Species:
    """One species in the form the reference holds after reading its PP file."""
    label: str
    z: int
    zv: float
    kind: int                        # PP_PSP or PP_UPF
    rr: np.ndarray                   # radial mesh
    # numeric psp (readpsp.f90): vr[l], rps[l] for l < lmax; lmax/l_local/skip 1-based
    vr: Optional[np.ndarray] = None
    rps: Optional[np.ndarray] = None
    lmax: int = 0
    l_local: int = 0
    skip: int = 0
    tkb: bool = False
    # UPF-like (readupf.f90): rab, vloc in Ha, beta = r*p(r), dij in Ry
    rab: Optional[np.ndarray] = None
    vloc: Optional[np.ndarray] = None
    beta: Optional[np.ndarray] = None
    beta_l: Optional[np.ndarray] = None
    dij: Optional[np.ndarray] = None
    upf_lmax: int = 0

    @property
    def mesh(self) -> int:
        return int(self.rr.shape[0])

    @property
    def nbeta(self) -> int:
        return 0 if self.beta is None else int(self.beta.shape[0])


@dataclass
class System:
    """A periodic system: cell, species, positions, cutoff, functional."""
    a_cell: np.ndarray               # 3x3, lattice vectors as columns (bohr)
    alat: float                      # a_lattice (bohr)
    symmetry: int                    # 1 cubic, 2 fcc
    ecut: float                      # wavefunction cutoff (Ry)
    species: List[Species]
    positions: List[np.ndarray]      # per species (na, 3) in bohr
    xc: int
    nstate: int = 0                  # 0: derived from the valence charge
    name: str = ""
    multiplicity: int = 0            # 0: closed shell; m >= 1: open shell (LSD) of multiplicity m

    @property
    def na(self) -> List[int]:
        return [int(p.shape[0]) for p in self.positions]

    @property
    def na_max(self) -> int:
        return max(self.na)

    @property
    def nat(self) -> int:
        return sum(self.na)

    def atco(self) -> np.ndarray:
        """Positions as the reference's atco(3, na_max, nsp), Fortran order."""
        a = np.zeros((len(self.species), self.na_max, 3))
        for i, p in enumerate(self.positions):
            a[i, : p.shape[0], :] = p
        return np.ascontiguousarray(a)

    def with_positions(self, atco: np.ndarray) -> "System":
        pos = [np.array(atco[i, :n, :]) for i, n in enumerate(self.na)]
        return System(self.a_cell.copy(), self.alat, self.symmetry, self.ecut,
                      self.species, pos, self.xc, self.nstate, self.name, self.multiplicity)


# --------------------------------------------------------------------------
# cell (set_cell.f90:4-131)
# --------------------------------------------------------------------------
def set_vec(a: float, b: float, c: float, symmetry: str) -> np.ndarray:
    s = symmetry.strip().upper()
    if s == "CUBIC":
        return np.diag([a, b, c]).astype(float)
    if s == "FCC":
        cols = [[-a / 2.0, 0.0, a / 2.0], [0.0, a / 2.0, a / 2.0], [-a / 2.0, a / 2.0, 0.0]]
        return np.array(cols, dtype=float).T
    raise ValueError(f"lattice {symmetry} is not supported (cubic and fcc only)")


_SYM_ID = {"CUBIC": 1, "FCC": 2}


# --------------------------------------------------------------------------
# pseudopotential files
# --------------------------------------------------------------------------
def _lval(s: str) -> int:
    return {"S": 0, "P": 1, "D": 2, "F": 3, "G": 4, "H": 5}.get(s.strip().upper(), -1)


def read_psp(path: str, lmax_letter: str, kleinman_bylander: bool, label: str = "") -> Species:
    """CPMD numeric pseudopotential (readpsp.f90:11-67) with the LMAX/LOCAL/SKIP
    conventions of yamlread.f90:244-314 (LOCAL defaults to LMAX)."""
    lmax = _lval(lmax_letter)
    l_local = lmax
    skip = -1
    if kleinman_bylander and 0 <= l_local <= lmax:
        l_local += 1
    else:
        l_local = lmax + 1
    if kleinman_bylander and 0 <= skip <= lmax:
        skip += 1
    else:
        skip = lmax + 2
    lmax += 1
    with open(path) as f:
        lines = f.read().splitlines()

    def find(tag, start=0):
        for i in range(start, len(lines)):
            if "&" + tag in lines[i]:
                return i
        raise ValueError(f"{path}: no &{tag} block")

    ia = find("ATOM")
    vals = {}
    for k in range(ia + 1, ia + 5):
        key, _, val = lines[k].partition("=")
        vals[key.strip()] = val.strip()
    z = int(vals["Z"].split()[0])
    zv = float(vals["ZV"].split()[0])
    ip = find("POTENTIAL", find("INFO"))
    mesh = int(lines[ip + 1].split()[0])
    pot = np.array([[float(x) for x in lines[ip + 2 + i].split()[: lmax + 1]] for i in range(mesh)])
    iw = find("WAVEFUNCTION", ip)
    meshw = int(lines[iw + 1].split()[0])
    wf = np.array([[float(x) for x in lines[iw + 2 + i].split()[: lmax + 1]] for i in range(meshw)])
    if meshw != mesh:
        raise ValueError(f"{path}: incompatible meshes {meshw} {mesh}")
    return Species(label=label or _SYMBOLS[z - 1], z=z, zv=zv, kind=PP_PSP, rr=pot[:, 0].copy(),
                   vr=np.ascontiguousarray(pot[:, 1:].T), rps=np.ascontiguousarray(wf[:, 1:].T),
                   lmax=lmax, l_local=l_local, skip=skip, tkb=kleinman_bylander)


def _upf_block(text: str, tag: str) -> str:
    m = re.search(r"<%s\b[^>]*>(.*?)</%s>" % (re.escape(tag), re.escape(tag)), text, re.S)
    if not m:
        raise ValueError(f"UPF block {tag} missing")
    return m.group(1)


def _upf_attr(text: str, tag: str, attr: str) -> str:
    m = re.search(r"<%s\b([^>]*)>" % re.escape(tag), text, re.S)
    if not m:
        raise ValueError(f"UPF tag {tag} missing")
    a = re.search(r'%s\s*=\s*"([^"]*)"' % attr, m.group(1))
    if not a:
        raise ValueError(f"UPF attribute {tag}.{attr} missing")
    return a.group(1).strip()


def read_upf(path: str, label: str = "") -> Species:
    """UPF v2 (readupf.f90:19-85, 237-356): mesh, PP_LOCAL (halved to Ha),
    PP_BETA.n with angular_momentum, PP_DIJ (kept in Ry; halved when used)."""
    text = open(path).read()
    element = _upf_attr(text, "PP_HEADER", "element")
    zv = float(_upf_attr(text, "PP_HEADER", "z_valence"))
    l_max = int(_upf_attr(text, "PP_HEADER", "l_max"))
    mesh = int(_upf_attr(text, "PP_HEADER", "mesh_size"))
    nbeta = int(_upf_attr(text, "PP_HEADER", "number_of_proj"))
    arr = lambda s: np.array([float(x) for x in s.split()])[:mesh]
    r = arr(_upf_block(text, "PP_R"))
    rab = arr(_upf_block(text, "PP_RAB"))
    vloc = arr(_upf_block(text, "PP_LOCAL")) * 0.5
    betas, ls = [], []
    for nb in range(1, nbeta + 1):
        betas.append(arr(_upf_block(text, f"PP_BETA.{nb}")))
        ls.append(int(_upf_attr(text, f"PP_BETA.{nb}", "angular_momentum")))
    dij = np.array([float(x) for x in _upf_block(text, "PP_DIJ").split()][: nbeta * nbeta]) if nbeta else np.zeros(1)
    z = symbol_to_z(element)
    return Species(label=label or element, z=z, zv=zv, kind=PP_UPF, rr=r, rab=rab, vloc=vloc,
                   beta=np.array(betas).reshape(nbeta, mesh) if nbeta else np.zeros((0, mesh)),
                   beta_l=np.array(ls, dtype=np.int32), dij=dij, upf_lmax=l_max + 1)


def gth_species(symbol: str, zion: float, rloc: float, c: Sequence[float],
                projectors: Sequence[tuple], rmin: float = 1.0e-4, rmax: float = 24.0,
                dx: float = 0.004) -> Species:
    """Tabulate a GTH/HGH pseudopotential into the UPF arrays.

    V_loc(r) = -Z/r erf(r/(sqrt2 rloc)) + exp(-r^2/(2 rloc^2)) sum_i C_i (r/rloc)^(2i-2)
    p_l(r)   = sqrt2 r^l exp(-r^2/(2 r_l^2)) / (r_l^(l+3/2) sqrt(Gamma(l+3/2)))
    (Goedecker, Teter, Hutter, PRB 54, 1703 (1996); Hartwigsen, Goedecker,
    Hutter, PRB 58, 3641 (1998)).  UPF stores beta = r p(r) and D = 2h (Ry).
    The mesh is r_i = rmin exp(i dx), rab = r dx.
    """
    n = int(math.log(rmax / rmin) / dx) + 1
    r = rmin * np.exp(dx * np.arange(n))
    rab = r * dx
    x = r / rloc
    vl = -zion / r * np.array([math.erf(v) for v in r / (math.sqrt(2.0) * rloc)])
    poly = np.zeros_like(r)
    for i, ci in enumerate(c):
        poly += ci * x ** (2 * i)
    vl += np.exp(-0.5 * x * x) * poly
    betas, ls, hs = [], [], []
    for (l, rl, h) in projectors:
        p = math.sqrt(2.0) * r ** l * np.exp(-r * r / (2.0 * rl * rl)) / (rl ** (l + 1.5) * math.sqrt(math.gamma(l + 1.5)))
        betas.append(r * p)
        ls.append(l)
        hs.append(h)
    nb = len(betas)
    dij = np.zeros(max(nb * nb, 1))
    for i, h in enumerate(hs):
        dij[i * nb + i] = 2.0 * h
    lmax = max(ls) if ls else 0
    return Species(label=symbol, z=symbol_to_z(symbol), zv=float(zion), kind=PP_UPF, rr=r, rab=rab,
                   vloc=vl, beta=np.array(betas).reshape(nb, n) if nb else np.zeros((0, n)),
                   beta_l=np.array(ls, dtype=np.int32), dij=dij, upf_lmax=lmax + 1)


# --------------------------------------------------------------------------
# reference input directory (input.yaml + xyz + PP files)
# --------------------------------------------------------------------------
def read_xyz(path: str, fact: float):
    """readcoordinate (yamlread.f90:360-419): species are contiguous runs."""
    lines = open(path).read().splitlines()
    labels, pos = [], []
    for ln in lines[2:]:
        t = ln.split()
        if len(t) < 4:
            continue
        labels.append(t[0])
        pos.append([float(v) * fact for v in t[1:4]])
    order, groups = [], {}
    prev = None
    for lab, p in zip(labels, pos):
        if lab != prev:
            order.append(lab)
            groups[len(order) - 1] = []
        groups[len(order) - 1].append(p)
        prev = lab
    return order, [np.array(groups[i]) for i in range(len(order))]


def load_reference_input(directory: str, yaml_name: str = "input.yaml") -> System:
    import yaml
    cfg = yaml.safe_load(open(os.path.join(directory, yaml_name)))
    cell = cfg["CELL"]
    dims = [float(v) for v in cell["DIMENSION"]]
    if cell.get("UNIT", "BOHR").strip().upper() == "ANGSTROM":
        dims = [d * ANGS2BOHR for d in dims]
    sym = str(cfg.get("SYMMETRY", "CUBIC")).strip().upper()
    a_cell = set_vec(dims[0], dims[1], dims[2], sym)
    ecut = 80.0
    if isinstance(cfg.get("CUTOFF"), dict):
        ecut = float(cfg["CUTOFF"].get("VALUE", 80.0))
    inp = cfg["INPUT"]
    fact = ANGS2BOHR if inp.get("UNIT", "BOHR").strip().upper() == "ANGSTROM" else 1.0
    labels, pos = read_xyz(os.path.join(directory, inp["COORDINATES_FILE"]), fact)
    species = []
    for i, lab in enumerate(labels):
        d = cfg["SPECIES"][f"LABEL{i + 1}"]
        ppf = os.path.join(directory, d["PP_FILE"])
        if "upf" in d["PP_FILE"]:
            species.append(read_upf(ppf, label=lab))
        else:
            kb = "KLEINMAN" in str(d.get("PP_SCHEME", "NONE")).upper()
            species.append(read_psp(ppf, str(d["LMAX"]), kb, label=lab))
    dft = cfg.get("DFT", {})
    xcs = " ".join(str(dft.get(k, "")) for k in ("EXCHANGE", "CORRELATION", "XC")).upper()
    if "TETER93" in xcs:
        xc = XC_TETER93
    elif "PBE" in xcs:
        xc = XC_PBE
    else:
        xc = XC_PZ
    # INITIALIZATION: OPEN_SHELL (Fortran logical) and MULTIPLICITY (yamlread.f90:70-73)
    init = cfg.get("INITIALIZATION") or {}
    open_shell = str(init.get("OPEN_SHELL", ".FALSE.")).strip().upper() in (".TRUE.", "TRUE", "T", ".T.")
    mult = int(init.get("MULTIPLICITY", 1)) if open_shell else 0
    return System(a_cell=a_cell, alat=dims[0], symmetry=_SYM_ID[sym], ecut=ecut, species=species,
                  positions=pos, xc=xc, name=os.path.basename(os.path.normpath(directory)), multiplicity=mult)
