"""Born-Oppenheimer MD driver (velocity Verlet) on top of the GPU engine.

Restates the outer loop of molecular_dynamics.f90:5-136 with
update_velver.f90:14-51: half kick, drift, new structure factors and
ortho_gs, a full wavefunction optimisation to GRAD_CUTOFF, ionic forces
from the last CG iteration, half kick.  Units: bohr, Hartree, atomic time;
constants from constants.f90:6-8.

Option outside the reference (off by default): extrapolate=True predicts
each step's starting wavefunction from the last `predictor_points`
converged ones (C0 <- sum_j w_j C0(t-j dt) [C0(t-j dt)^T C0(t)], then
ortho_gs; weights of Kolafa's always-stable predictor, linear
extrapolation 2 C0(t) - C0(t-dt)[...] for two points) instead of
restarting from C0(t) as molecular_dynamics.f90:106-109 does; the converged
state and the trajectory are the same to the SCF tolerance, the number of
SCF iterations per step drops.

Velocities and the centre-of-mass shift (outside the hot path):
- by default velocities are drawn per atom from a seeded Maxwell-Boltzmann
  distribution; md_tools.f90:19-44 instead draws one random triple w for
  all atoms (v = sigma_s w for every atom of species s, then the linear
  momentum is removed and the velocities rescaled to the temperature), and
  its seed is not applied (random.f90:15-17), so its w cannot be
  reproduced: `reference_velocities(w)` restates init_vel for a given w;
- by default no centre-of-mass shift after the drift; com_shift=True
  restates shift_com (md_tools.f90:116-149, called at
  molecular_dynamics.f90:100): all atoms translated so that the sum of the
  positions divided by na_max keeps its starting value (a uniform
  translation, which changes no energy beyond the grid's egg-box effect).
"""
from __future__ import annotations

import time

import numpy as np

from .inputs import AMU_AU, atomic_mass

AU_TO_FS = 2.418884326505e-2
KBOLTZ = 0.316681534e-5


class BOMD:
    def __init__(self, engine, temperature: float = 300.0, dt_fs: float = 0.5, seed: int = 2024,
                 gcut: float = 1e-6, max_scf: int = 800, extrapolate: bool = False,
                 predictor_points: int = 2, com_shift: bool = False):
        self.e = engine
        self.extrapolate = extrapolate
        self.predictor_points = predictor_points
        s = engine.system
        self.system = s
        self.dt = dt_fs / AU_TO_FS
        self.gcut = gcut
        self.max_scf = max_scf
        self.mass = np.zeros((len(s.species), s.na_max))
        for i, sp in enumerate(s.species):
            self.mass[i, : s.na[i]] = atomic_mass(sp.z) * AMU_AU
        self.mask = self.mass > 0
        self.pos = s.atco()
        self.com_shift = com_shift
        self.com0 = self._com(self.pos)
        self.ndof = 3 * s.nat - 3
        self.vel = self._init_velocities(temperature, seed)
        self.force = None
        self.energy = None
        self.scf_iterations = []
        self.step_wall = []   # host wall clock of each step of run(), s

    def _init_velocities(self, temperature, seed):
        rng = np.random.default_rng(seed)
        v = np.zeros_like(self.pos)
        sig = np.zeros_like(self.mass)
        sig[self.mask] = np.sqrt(temperature * KBOLTZ / self.mass[self.mask])
        v[self.mask] = rng.standard_normal((int(self.mask.sum()), 3)) * sig[self.mask][:, None]
        p = (self.mass[..., None] * v).sum(axis=(0, 1)) / self.mass.sum()
        v[self.mask] -= p
        t = self.temperature(v)
        if t > 0:
            v *= np.sqrt(temperature / t)
        return v

    def reference_velocities(self, w, temperature: float = 300.0):
        """init_vel (md_tools.f90:19-48) with its random triple's vector w
        given: every atom of species s gets sigma_s w, sigma_s =
        sqrt(T k_B / m_s); then remove_lin_momentum (md_tools.f90:87-114)
        and rescale_atvel to the temperature."""
        w = np.asarray(w, dtype=np.float64)
        v = np.zeros_like(self.pos)
        sig = np.zeros_like(self.mass)
        sig[self.mask] = np.sqrt(temperature * KBOLTZ / self.mass[self.mask])
        v[self.mask] = sig[self.mask][:, None] * w[None, :]
        p = (self.mass[..., None] * v).sum(axis=(0, 1)) / self.mass.sum()
        v[self.mask] -= p
        v *= np.sqrt(temperature / self.temperature(v))
        return v

    def _com(self, pos):
        """get_com (md_tools.f90:116-131): the sum of the positions over all
        atoms divided by na_max."""
        return pos[self.mask].sum(axis=0) / self.system.na_max

    def kinetic(self, v=None):
        v = self.vel if v is None else v
        return 0.5 * float((self.mass[..., None] * v * v).sum())

    def temperature(self, v=None):
        return 2.0 * self.kinetic(v) / (self.ndof * KBOLTZ)

    def _scf(self):
        """wfn_opt (do_opt.f90:51-138) from the current wavefunction."""
        n, en, gm = self.e.wfn_opt(self.max_scf, self.gcut)
        self.scf_iterations.append(n)
        self.energy = en["etotal"]
        # forces are evaluated in every CG iteration once GEMAX < 3 gcut
        # (CHK_TFOR); a first-iteration convergence has none yet
        self.force = self.e.get("force") if n > 1 else self.e.ionic_forces()
        return n

    def start(self):
        """Forces at the initial geometry (molecular_dynamics.f90:56-60)."""
        self.e.set_positions(self.pos)
        if self.extrapolate:
            self.e.set_predictor(self.predictor_points)
            self.e.clear_history()
        self.e.ortho()
        return self._scf()

    def step(self):
        """One velocity-Verlet step (molecular_dynamics.f90:96-118)."""
        if self.force is None:
            self.start()
        a = np.zeros_like(self.vel)
        a[self.mask] = self.force[self.mask] / self.mass[self.mask][:, None]
        self.vel += 0.5 * self.dt * a
        self.pos = self.pos + self.vel * self.dt
        if self.com_shift:
            self.pos[self.mask] -= self._com(self.pos) - self.com0
        self.e.set_positions(self.pos)
        if self.extrapolate:
            self.e.extrapolate()
        self.e.ortho()
        n = self._scf()
        a[self.mask] = self.force[self.mask] / self.mass[self.mask][:, None]
        self.vel += 0.5 * self.dt * a
        return n

    def total_energy(self):
        return self.energy + self.kinetic()

    def run(self, nsteps: int, callback=None):
        t0 = time.perf_counter()
        for i in range(nsteps):
            t = time.perf_counter()
            n = self.step()
            self.step_wall.append(time.perf_counter() - t)
            if callback:
                callback(i, n, self.energy, self.total_energy(), self.temperature())
        return time.perf_counter() - t0


def aspc_coefficients(npoints: int):
    """Weights of Kolafa's always-stable predictor with npoints = K + 2 points,
    most recent first (J. Comput. Chem. 25, 335 (2004)):
    B_j = (-1)^(j+1) j binom(2K+4, K+2-j) / binom(2K+2, K+1).  The engine
    computes the same weights for amdk_wfn_set_predictor(coef=NULL)."""
    from math import comb
    if npoints <= 1:
        return np.ones(1)
    k = npoints - 2
    return np.array([(-1) ** (j + 1) * j * comb(2 * k + 4, k + 2 - j) / comb(2 * k + 2, k + 1)
                     for j in range(1, npoints + 1)])
