"""The seeded benchmark systems (synthetic stand-ins for the reference inputs).

All use GTH-form norm-conserving pseudopotentials tabulated into the UPF
arrays (inputs.gth_species), cubic cells, Gamma point:

  water1   1 H2O, 12 bohr box, O centred, O-H 1.81 bohr, 104.5 deg; LDA (PZ),
           70 Ry, 64^3 grid, 4 doubly occupied bands
  si64     64-atom diamond Si (2x2x2 of a = 10.26 bohr), atoms displaced by
           a seeded uniform +-0.05 bohr; LDA, 30 Ry, 72^3 grid, 128 bands
  water32  32 H2O at 1 g/cm^3 (18.63 bohr), seeded rigid molecules with
           O-O >= 2.5 A; PBE, 70 Ry, 100^3 grid, 128 bands
  water128 128 H2O at 1 g/cm^3 (29.58 bohr), as water32 and perturbed by a
           seeded +-0.1 bohr; PBE, 70 Ry, 160^3 grid, 512 bands
  cluster  a water cluster of n molecules in its own cubic box (the members
           of the batched ensemble), LDA, 70 Ry
"""
from __future__ import annotations

import math
from typing import List, Optional

import numpy as np

from .inputs import ANGS2BOHR, XC_PBE, XC_PZ, System, gth_species

OH = 1.81                      # bohr
HOH = math.radians(104.5)


def gth_oxygen():
    return gth_species("O", 6.0, 0.25, [-16.6, 2.4], [(0, 0.22, 18.3)])


def gth_hydrogen():
    return gth_species("H", 1.0, 0.20, [-4.18, 0.73], [])


def gth_silicon():
    return gth_species("Si", 4.0, 0.44, [-7.34], [(0, 0.42, 5.9), (1, 0.48, 2.7)])


def _water_local(rot: np.ndarray) -> np.ndarray:
    """O and the two H of a rigid water in the molecule frame, rotated."""
    h1 = OH * np.array([math.sin(HOH / 2), math.cos(HOH / 2), 0.0])
    h2 = OH * np.array([-math.sin(HOH / 2), math.cos(HOH / 2), 0.0])
    return np.array([np.zeros(3), h1, h2]) @ rot.T


def _random_rotation(rng) -> np.ndarray:
    q = rng.standard_normal(4)
    q /= np.linalg.norm(q)
    a, b, c, d = q
    return np.array([[a * a + b * b - c * c - d * d, 2 * (b * c - a * d), 2 * (b * d + a * c)],
                     [2 * (b * c + a * d), a * a - b * b + c * c - d * d, 2 * (c * d - a * b)],
                     [2 * (b * d - a * c), 2 * (c * d + a * b), a * a - b * b - c * c + d * d]])


def _water_box(nmol: int, L: float, seed: int, dmin_angstrom: float, periodic: bool = True,
               margin: float = 0.0) -> List[np.ndarray]:
    rng = np.random.default_rng(seed)
    dmin = dmin_angstrom * ANGS2BOHR
    oxy, hyd = [], []
    tries = 0
    while len(oxy) < nmol:
        tries += 1
        if tries > 200000:
            raise RuntimeError("could not place the water molecules")
        o = rng.uniform(margin, L - margin, 3)
        ok = True
        for p in oxy:
            d = o - p
            if periodic:
                d -= L * np.round(d / L)
            if np.linalg.norm(d) < dmin:
                ok = False
                break
        if not ok:
            continue
        m = _water_local(_random_rotation(rng)) + o
        oxy.append(m[0])
        hyd.extend([m[1], m[2]])
    return [np.array(oxy), np.array(hyd)]


def water1(ecut: float = 70.0) -> System:
    L = 12.0
    o = np.array([L / 2, L / 2, L / 2])
    m = _water_local(np.eye(3)) + o
    return System(a_cell=np.diag([L, L, L]), alat=L, symmetry=1, ecut=ecut,
                  species=[gth_oxygen(), gth_hydrogen()], positions=[m[:1], m[1:]], xc=XC_PZ, name="water1")


def si64(ecut: float = 30.0, seed: int = 7) -> System:
    a = 10.26
    basis = np.array([[0, 0, 0], [0, .5, .5], [.5, 0, .5], [.5, .5, 0],
                      [.25, .25, .25], [.25, .75, .75], [.75, .25, .75], [.75, .75, .25]])
    pos = []
    for i in range(2):
        for j in range(2):
            for k in range(2):
                for b in basis:
                    pos.append((np.array([i, j, k]) + b) * a)
    pos = np.array(pos)
    rng = np.random.default_rng(seed)
    pos = pos + rng.uniform(-0.05, 0.05, pos.shape)
    L = 2 * a
    return System(a_cell=np.diag([L, L, L]), alat=L, symmetry=1, ecut=ecut, species=[gth_silicon()],
                  positions=[pos], xc=XC_PZ, name="si64")


def water32(ecut: float = 70.0, seed: int = 32, xc: int = XC_PBE) -> System:
    L = 18.63
    pos = _water_box(32, L, seed, 2.5)
    return System(a_cell=np.diag([L, L, L]), alat=L, symmetry=1, ecut=ecut,
                  species=[gth_oxygen(), gth_hydrogen()], positions=pos, xc=xc, name="water32")


def water128(ecut: float = 70.0, seed: int = 128) -> System:
    L = 29.58
    pos = _water_box(128, L, seed, 2.5)
    rng = np.random.default_rng(seed + 1)
    pos = [p + rng.uniform(-0.1, 0.1, p.shape) for p in pos]
    return System(a_cell=np.diag([L, L, L]), alat=L, symmetry=1, ecut=ecut,
                  species=[gth_oxygen(), gth_hydrogen()], positions=pos, xc=XC_PBE, name="water128")


def cluster(nmol: int, L: float, seed: int, ecut: float = 70.0) -> System:
    pos = _water_box(nmol, L, seed, 2.6, periodic=False, margin=2.5)
    return System(a_cell=np.diag([L, L, L]), alat=L, symmetry=1, ecut=ecut,
                  species=[gth_oxygen(), gth_hydrogen()], positions=pos, xc=XC_PZ, name=f"cluster{nmol}")


def ensemble(seed: int = 16) -> List[System]:
    """16 independent clusters of 1-8 molecules, boxes of 12-16 bohr."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(16):
        n = int(rng.integers(1, 9))
        L = float(rng.uniform(12.0, 16.0))
        out.append(cluster(n, L, seed * 100 + k))
    return out


def small_water(ecut: float = 30.0, xc: int = XC_PZ) -> System:
    """1 H2O in a 10 bohr box at a low cutoff: the quick parity case."""
    L = 10.0
    o = np.array([L / 2 + 0.13, L / 2 - 0.07, L / 2 + 0.21])
    m = _water_local(_random_rotation(np.random.default_rng(3))) + o
    return System(a_cell=np.diag([L, L, L]), alat=L, symmetry=1, ecut=ecut,
                  species=[gth_oxygen(), gth_hydrogen()], positions=[m[:1], m[1:]], xc=xc, name="small_water")


BY_NAME = {"water1": water1, "si64": si64, "water32": water32, "water128": water128, "small_water": small_water}
