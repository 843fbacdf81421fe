"""Host logic of the BOMD driver that needs no GPU: the always-stable
predictor weights (Kolafa, J. Comput. Chem. 25, 335 (2004)), and the
velocity-Verlet step against the reference's own 32-water MD run."""
import numpy as np
import pytest

from amdkiit_b200.md import aspc_coefficients


def test_aspc_known_weights():
    assert np.allclose(aspc_coefficients(1), [1.0])
    assert np.allclose(aspc_coefficients(2), [2.0, -1.0])
    assert np.allclose(aspc_coefficients(3), [2.5, -2.0, 0.5])
    assert np.allclose(aspc_coefficients(4), [2.8, -2.8, 1.2, -0.2])
    assert np.allclose(aspc_coefficients(5), [3.0, -24 / 7, 27 / 14, -4 / 7, 1 / 14])


@pytest.mark.parametrize("n", range(2, 9))
def test_aspc_weights_extrapolate_linear_trajectories_exactly(n):
    w = aspc_coefficients(n)
    t = -np.arange(n, dtype=float)  # C0(t), C0(t-dt), ... at t = 0, -1, ...
    assert abs(w.sum() - 1.0) < 1e-12
    assert abs(w @ t - 1.0) < 1e-12  # a(t) = t is predicted at t = +1


class _ForcesOnly:
    """Engine stand-in that returns fixed forces (the reference's printed
    start forces) for the driver's first step."""

    def __init__(self, system, force):
        self.system = system
        self.force = force

    def set_positions(self, atco):
        pass

    def ortho(self):
        pass

    def wfn_opt(self, max_step, gcut):
        return 2, {"etotal": 0.0}, 0.0

    def get(self, name):
        return self.force


def test_first_step_lands_on_reference_frame_1():
    """The driver's velocity-Verlet step with shift_com (molecular_dynamics.f90:
    96-100), the reference's start forces (printed to 4 figures) and the
    initial velocities of init_vel recovered from the reference's frames 0 and
    1 reproduce its frame 1 and its printed frame-0 velocities of the 32-water
    MD run (tests/32_water/md) to the printed digits."""
    from amdkiit_b200.inputs import ANGS2BOHR
    from amdkiit_b200.md import BOMD
    from tests.helpers import golden, load_fixture
    s = load_fixture("water32_mt")
    g = golden()["water32_mt"]
    tr = g["md_trajectory"]
    rows = [(i, a) for i, n in enumerate(s.na) for a in range(n)]
    f = np.array(g["md_start"]["forces"])
    force = np.zeros((len(s.species), s.na_max, 3))
    for (i, a), v in zip(rows, f):
        force[i, a] = v
    md = BOMD(_ForcesOnly(s, force), temperature=300.0, dt_fs=0.5, com_shift=True)
    md.force = force
    fr0 = np.array(tr["frames"]["0"]) * ANGS2BOHR
    fr1 = np.array(tr["frames"]["1"]) * ANGS2BOHR
    m = np.array([md.mass[i, a] for i, a in rows])
    d = (fr1 - fr0) / md.dt - 0.5 * md.dt * f / m[:, None]
    z = np.array([s.species[i].z for i, _ in rows])
    w = d[z == 1].mean(axis=0) - d[z == 8].mean(axis=0)
    md.vel = md.reference_velocities(w / np.linalg.norm(w))
    v0 = np.array([md.vel[i, a] for i, a in rows]) / ANGS2BOHR
    assert np.max(np.abs(v0 - np.array(tr["vel0"]))) < 6e-7  # printed to 1e-6
    assert abs(md.temperature() - 300.0) < 1e-9
    md.step()
    x1 = np.array([md.pos[i, a] for i, a in rows])
    assert np.max(np.abs(x1 - fr1)) < 3e-6  # bohr; printed to 1e-6 A
