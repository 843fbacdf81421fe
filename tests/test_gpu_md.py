"""Forces and dynamics on the GPU path.

- central finite differences of the GPU total energy (delta = 1e-3 bohr) on
  random atom components against the analytic ionic forces (e_sr + POTFOR +
  NLFOR) and the backward entry: within 1e-4 Ha/bohr;
- velocity-Verlet BOMD steps on the GPU follow the oracle's trajectory
  (same start, same driver): energies within 1e-8 Ha, positions within
  1e-8 bohr per step; the total-energy fluctuation is the integrator's
  (it shrinks as dt^2)."""
import numpy as np
import pytest

from amdkiit_b200 import configs
from amdkiit_b200.engine import FP64, Engine
from amdkiit_b200.inputs import XC_PBE
from amdkiit_b200.md import BOMD
from tests.helpers import OracleEngine, start_coefficients

pytestmark = pytest.mark.gpu


def _engine(system):
    e = Engine(system, FP64)
    g = e.gvectors()
    tp = 2 * np.pi / system.alat
    e.set_wfn(start_coefficients(g["hg"][: e.ngpw], tp, e.nstate))
    e.ortho()
    return e


def _energy_at(e, atco, c0):
    e.set_positions(atco)
    e.set_wfn(c0)
    e.ortho()
    n, en, gm = e.wfn_opt(600, 1e-9)
    return en["etotal"]


def test_forces_match_finite_differences():
    s = configs.small_water(xc=XC_PBE)
    e = _engine(s)
    n, en, gm = e.wfn_opt(600, 1e-9)
    f = e.ionic_forces()
    grad = e.backward()                   # dE/dR from the backward entry
    assert np.max(np.abs(grad + f)) < 1e-12
    c0 = e.get_wfn()
    x0 = s.atco()
    rng = np.random.default_rng(5)
    comps = [(0, 0, int(rng.integers(3))), (1, 0, int(rng.integers(3))), (1, 1, int(rng.integers(3)))]
    d = 1e-3
    for (isp, ia, k) in comps:
        xp = x0.copy(); xp[isp, ia, k] += d
        xm = x0.copy(); xm[isp, ia, k] -= d
        ep = _energy_at(e, xp, c0)
        em = _energy_at(e, xm, c0)
        fd = -(ep - em) / (2 * d)
        assert abs(fd - f[isp, ia, k]) < 1e-4, (isp, ia, k, fd, f[isp, ia, k])


def test_bomd_follows_oracle_trajectory():
    s = configs.small_water()
    e = _engine(s)
    md_g = BOMD(e, temperature=300.0, dt_fs=0.5, seed=3, gcut=1e-7)
    md_o = BOMD(OracleEngine(s), temperature=300.0, dt_fs=0.5, seed=3, gcut=1e-7)
    md_g.start()
    md_o.start()
    assert abs(md_g.total_energy() - md_o.total_energy()) < 1e-8
    for _ in range(4):
        md_g.step()
        md_o.step()
        assert abs(md_g.total_energy() - md_o.total_energy()) < 1e-8
        assert np.max(np.abs(md_g.pos - md_o.pos)) < 1e-8
    assert abs(md_g.total_energy() - md_o.total_energy()) < 1e-8


def test_bomd_energy_error_scales_with_timestep():
    s = configs.small_water()
    drift = []
    for dt in (0.5, 0.25):
        e = _engine(s)
        md = BOMD(e, temperature=300.0, dt_fs=dt, seed=3, gcut=1e-7)
        md.start()
        e0 = md.total_energy()
        worst = 0.0
        for _ in range(int(round(1.5 / dt))):
            md.step()
            worst = max(worst, abs(md.total_energy() - e0))
        drift.append(worst)
    assert drift[1] < 0.5 * drift[0]
    assert drift[0] < 1e-3


def test_bomd_predictor_keeps_trajectory_and_saves_iterations():
    """The wavefunction predictor (an option outside the reference driver)
    reaches the same states to the SCF tolerance in fewer iterations."""
    s = configs.small_water()
    runs = {}
    for x in (False, True):
        e = _engine(s)
        md = BOMD(e, temperature=300.0, dt_fs=0.5, seed=3, gcut=1e-7, extrapolate=x)
        md.start()
        for _ in range(6):
            md.step()
        runs[x] = md
    assert np.max(np.abs(runs[True].pos - runs[False].pos)) < 1e-6
    assert abs(runs[True].total_energy() - runs[False].total_energy()) < 1e-7
    assert np.mean(runs[True].scf_iterations[3:]) < np.mean(runs[False].scf_iterations[3:])


def test_bomd_higher_order_predictor():
    """Always-stable predictor weights over 4 points and explicit weights
    reach the same trajectory as the reference driver to the SCF tolerance;
    explicit (2, -1) weights are the default linear predictor bit for bit."""
    s = configs.small_water()
    runs = {}
    for key, x, npts, coef in (("ref", False, 2, None), ("aspc4", True, 4, None), ("lin", True, 2, None),
                               ("lin_w", True, 2, [2.0, -1.0]), ("poly3", True, 3, [3.0, -3.0, 1.0])):
        e = _engine(s)
        md = BOMD(e, temperature=300.0, dt_fs=0.5, seed=3, gcut=1e-7, extrapolate=x, predictor_points=npts)
        md.start()
        if coef is not None:
            e.set_predictor(npts, coef)
        for _ in range(6):
            md.step()
        runs[key] = (md, e.get_wfn())
    ref = runs["ref"][0]
    for key in ("aspc4", "lin", "poly3"):
        md = runs[key][0]
        assert np.max(np.abs(md.pos - ref.pos)) < 1e-6, key
        assert abs(md.total_energy() - ref.total_energy()) < 1e-7, key
        assert np.mean(md.scf_iterations[3:]) < np.mean(ref.scf_iterations[3:]), key
    assert runs["lin"][0].scf_iterations == runs["lin_w"][0].scf_iterations
    assert np.array_equal(runs["lin"][1], runs["lin_w"][1])
