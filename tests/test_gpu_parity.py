"""GPU parity: every stage of one CG iteration through the C-ABI against the
CPU restatement on the same inputs, then whole SCF runs.

Tolerances (FP64 path): the GPU FFTs and reductions round differently from
the oracle's, so real-space and G-space arrays agree to ~1e-12 relative;
we test 1e-10 relative to the array's max.  Energies: 1e-9 Ha per stage.
After convergence: |dE| <= 1e-6 Ha/atom and |dF| <= 1e-4 Ha/bohr (the
build's correctness bar), in practice far tighter."""
import numpy as np
import pytest

from amdkiit_b200 import configs
from amdkiit_b200.engine import FP64, Engine
from amdkiit_b200.inputs import XC_PBE
from oracle.oracle import Oracle
from tests.helpers import golden, golden_oracle, load_fixture, oracle_eigenvalues, start_coefficients

pytestmark = pytest.mark.gpu


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def pair(system, seed=1234, batch=0):
    o = Oracle(system, 0)
    e = Engine(system, FP64, pair_batch=batch)
    g = o.gvectors()
    c = start_coefficients(g["hg"][: o.ngpw], o.d("tpiba"), o.nstate, seed)
    o.set_wfn(c)
    e.set_wfn(c)
    return o, e


SYSTEMS = {
    "small_water_pz": lambda: configs.small_water(),
    "small_water_pbe": lambda: configs.small_water(xc=XC_PBE),
    "si_fcc_mt": lambda: load_fixture("si_fcc_mt"),
    "si64_low": lambda: configs.si64(ecut=12.0),
}


@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_one_iteration_stage_by_stage(name):
    s = SYSTEMS[name]()
    o, e = pair(s)
    # tables built on the device
    ng = e.ngrho
    assert rel(e.get("vps")[:, :ng], o.arr("vps", (len(s.species), ng))) < 1e-12
    assert rel(e.get("eigrxvps"), o.arr("eigrxvps", (ng,), np.complex128)) < 1e-11
    assert rel(e.get("eigrxrhos"), o.arr("eigrxrhos", (ng,), np.complex128)) < 1e-11
    # ortho_gs
    assert o.ortho() == 0
    e.ortho()
    assert rel(e.get_wfn(), o.c0()) < 1e-11
    # eval_density + rhor2g
    o.call("eval_density")
    o.call("rhor2g")
    e.density()
    assert rel(e.get("rho"), o.real_grid("rho")) < 1e-11
    assert rel(e.get("rho_g"), o.arr("rho_g", (ng,), np.complex128)) < 1e-11
    # eval_pot + cal_vpot_ex
    o.call("eval_pot")
    o.call("cal_vpot_ex")
    e.potential()
    assert rel(e.get("v_pot"), o.real_grid("v_pot")) < 1e-10
    # pp_energy + e_total
    o.call("pp_energy")
    o.call("e_total")
    en = e.energy()
    eo = o.energies()
    for k in ("etotal", "eke", "estat", "eloc", "enl", "exc", "esr", "eself"):
        assert abs(en[k] - eo[k]) < 1e-9, (k, en[k], eo[k])
    # vpsi + fnonloc
    o.call("vpsi")
    o.call("fnonloc")
    e.apply_h()
    assert rel(e.get("c2"), o.c2()) < 1e-10
    # forces (Lambda) + GEMAX
    o.call("forces")
    gm = e.gradient()
    assert rel(e.get("c2"), o.c2()) < 1e-10
    c2o = o.c2()
    nocc = int(np.sum(o.arr("occ", (o.nstate,)) > 1e-5))
    assert abs(gm - np.abs(c2o[:nocc]).max()) < 1e-12 * max(gm, 1.0)
    # PCG (first step) + ortho
    o.call("pcg", 1)
    e.pcg(1)
    assert rel(e.get_wfn(), o.c0()) < 1e-10
    assert o.ortho() == 0
    e.ortho()
    assert rel(e.get_wfn(), o.c0()) < 1e-10


@pytest.mark.parametrize("name", sorted(SYSTEMS))
def test_scf_iterations_track_oracle(name):
    s = SYSTEMS[name]()
    o, e = pair(s)
    o.ortho()
    e.ortho()
    for it in range(1, 26):
        ro = o.scf_iteration(it, 1e-7)
        en, gm, conv = e.scf_iteration(it, 1e-7)
        assert abs(en["etotal"] - o.d("etotal")) < 1e-8, it
        assert abs(gm - o.d("gemax")) < 1e-8 * max(1.0, gm), it
    assert rel(e.get_wfn(), o.c0()) < 1e-6


@pytest.mark.parametrize("batch", [1, 3, 0])
def test_pair_batch_does_not_change_results(batch):
    s = configs.small_water()
    o, e = pair(s, batch=batch)
    e.ortho()
    e.density()
    ref = Engine(s, FP64, pair_batch=1)
    ref.set_wfn(e.get_wfn())
    ref.density()
    assert rel(e.get("rho"), ref.get("rho")) < 1e-13


def test_converged_energy_and_forces_match_oracle():
    s = configs.small_water(xc=XC_PBE)
    o, e = pair(s)
    o.ortho()
    e.ortho()
    no = o.wfn_opt(400, 1e-7)
    ne, en, gm = e.wfn_opt(400, 1e-7)
    assert 0 < no < 400 and ne < 400
    assert abs(en["etotal"] - o.d("etotal")) < 1e-6 * s.nat
    fo = o.force()
    fe = e.ionic_forces()
    assert np.max(np.abs(fe - fo)) < 1e-4
    # forces are present (tfor) and the net force is small for a free molecule
    assert np.abs(fo).max() > 1e-3


def test_fft_sphere_roundtrip_and_numpy():
    s = configs.small_water()
    e = Engine(s, FP64)
    g = e.gvectors()
    rng = np.random.default_rng(0)
    coef = (rng.standard_normal(e.ngrho) + 1j * rng.standard_normal(e.ngrho)) / (1 + g["hg"])
    coef[0] = coef[0].real
    _, grid = e.fft_sphere(-1, coef=coef)
    n1, n2, n3 = e.nr
    nh = np.array([n1 // 2 + 1, n2 // 2 + 1, n3 // 2 + 1])
    mil = g["inyh"] - nh[None, :]
    full = np.zeros((n3, n2, n1), complex)
    full[mil[:, 2] % n3, mil[:, 1] % n2, mil[:, 0] % n1] = coef
    full[(-mil[:, 2]) % n3, (-mil[:, 1]) % n2, (-mil[:, 0]) % n1] = np.conj(coef)
    full[0, 0, 0] = coef[0]
    ref = np.fft.ifftn(full) * full.size
    assert rel(grid, ref) < 1e-12
    back, _ = e.fft_sphere(+1, grid=grid)
    assert rel(back, coef) < 1e-12


def test_reference_energy_on_gpu():
    """The 1-water reference run (tests/1_water/wf_opt: MT psp, Teter93,
    80 Ry, 108^3) through the GPU path: E_tot within 1e-6 Ha/atom, forces
    within 1e-5 Ha/bohr of the reference's start gradient."""
    s = load_fixture("water1_mt")
    e = Engine(s, FP64)
    g = e.gvectors()
    tp = 2 * np.pi / s.alat
    e.set_wfn(start_coefficients(g["hg"][: e.ngpw], tp, e.nstate))
    e.ortho()
    n, en, gm = e.wfn_opt(600, 1e-7)
    ref = golden()["water1_mt"]["energies"]
    assert abs(en["etotal"] - ref["etotal"]) < 1e-6 * s.nat
    assert abs(en["esr"] - ref["esr"]) < 1e-9 and abs(en["eself"] - ref["eself"]) < 1e-9
    # forces against the reference's geometry-optimisation start gradient
    # (tests/1_water/geo_opt/atom_force.dat, same input geometry)
    f = e.ionic_forces()
    f = np.concatenate([f[i, :k] for i, k in enumerate(s.na)])
    grad = np.array(golden()["water1_mt"]["geo_start"]["gradient"])
    assert np.max(np.abs(f + grad)) < 1e-5


def test_reference_water32_on_gpu():
    """The 32-water reference runs (tests/32_water: MT psp, Teter93, 80 Ry,
    108^3, 128 bands, GRAD_CUTOFF 1e-6) through the GPU path: E_tot of
    wf_opt within 1e-6 Ha/atom, and the ionic forces at convergence within
    1e-4 Ha/bohr of the first force table of the MD run, which starts from
    the same geometry (4 printed significant figures)."""
    s = load_fixture("water32_mt")
    e = Engine(s, FP64)
    g = e.gvectors()
    tp = 2 * np.pi / s.alat
    e.set_wfn(start_coefficients(g["hg"][: e.ngpw], tp, e.nstate))
    e.ortho()
    n, en, gm = e.wfn_opt(600, 1e-6)
    assert gm < 1e-6
    ref = golden()["water32_mt"]
    assert abs(en["etotal"] - ref["energies"]["etotal"]) < 1e-6 * s.nat
    f = e.ionic_forces()
    f = np.concatenate([f[i, :k] for i, k in enumerate(s.na)])
    assert np.max(np.abs(f - np.array(ref["md_start"]["forces"]))) < 1e-4
    # subspace eigenvalues against the oracle converged from the same start
    # (tests/golden/make_oracle_fixtures.py): within 1e-5 Ha
    orc = golden_oracle("water32_mt")
    assert np.max(np.abs(e.eigenvalues() - np.array(orc["eigenvalues"]))) < 1e-5
    e.close()


def test_reference_water2_on_gpu():
    """The 2-water reference run (tests/2_water/wf_opt, 8 bands, default
    GRAD_CUTOFF 1e-7) through the GPU path: E_tot within 1e-6 Ha/atom, and
    the subspace eigenvalues within 1e-5 Ha of the oracle converged from the
    same start (tests/golden/make_oracle_fixtures.py)."""
    s = load_fixture("water2_mt")
    e = Engine(s, FP64)
    g = e.gvectors()
    tp = 2 * np.pi / s.alat
    e.set_wfn(start_coefficients(g["hg"][: e.ngpw], tp, e.nstate))
    e.ortho()
    n, en, gm = e.wfn_opt(600, 1e-7)
    assert gm < 1e-7
    assert abs(en["etotal"] - golden()["water2_mt"]["energies"]["etotal"]) < 1e-6 * s.nat
    orc = golden_oracle("water2_mt")
    assert np.max(np.abs(e.eigenvalues() - np.array(orc["eigenvalues"]))) < 1e-5
    e.close()


@pytest.mark.parametrize("name", ["small_water_pbe", "si_fcc_mt"])
def test_eigenvalues_match_oracle(name):
    """Subspace eigenvalues from the GPU's H|psi> and from the oracle's at the
    same orthonormalised start agree to 1e-10 Ha."""
    s = SYSTEMS[name]()
    o, e = pair(s)
    assert o.ortho() == 0
    e.ortho()
    d = np.max(np.abs(e.eigenvalues() - oracle_eigenvalues(o)))
    assert d < 1e-10


def test_set_precision_switches_pair_transforms():
    """A mixed-precision engine switched to FP64 pair transforms reproduces
    the FP64 engine's density; switched back it is FP32-accurate again."""
    from amdkiit_b200.engine import MIXED
    s = configs.small_water()
    o, ref = pair(s)
    ref.ortho()
    c = ref.get_wfn()
    ref.density()
    rho64 = ref.get("rho")
    e = Engine(s, MIXED)
    e.set_wfn(c)
    e.density()
    rho_mx = e.get("rho")
    assert 1e-12 < rel(rho_mx, rho64) < 1e-5
    e.set_precision(FP64)
    e.density()
    assert rel(e.get("rho"), rho64) < 1e-12
    e.set_precision(MIXED)
    e.density()
    assert rel(e.get("rho"), rho_mx) < 1e-14


def test_mixed_with_fp64_refinement_matches_fp64_energy():
    """wfn_opt on a mixed engine ends with FP64 pair transforms: its energy
    and forces agree with the FP64 engine's at convergence far inside the
    1e-6 Ha/atom and 1e-4 Ha/bohr bars."""
    from amdkiit_b200.engine import MIXED
    s = configs.small_water(xc=XC_PBE)
    _, e64 = pair(s)
    emx = Engine(s, MIXED)
    emx.set_wfn(e64.get_wfn())
    e64.ortho()
    emx.ortho()
    n64, en64, _ = e64.wfn_opt(400, 1e-7)
    nmx, enmx, _ = emx.wfn_opt(400, 1e-7)
    assert n64 < 400 and nmx < 400
    assert emx.pair_precision == MIXED
    assert abs(enmx["etotal"] - en64["etotal"]) < 1e-7 * s.nat
    assert np.max(np.abs(emx.get("force") - e64.get("force"))) < 1e-5


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_slab_path_matches_pencil_path(prec, monkeypatch):
    """The slab transforms (used for grids the pencil kernels do not take)
    give the pencil path's density and H|psi> on the same wavefunction."""
    from amdkiit_b200.engine import MIXED
    p = FP64 if prec == "fp64" else MIXED
    tol = 1e-12 if prec == "fp64" else 1e-5
    s = configs.small_water(xc=XC_PBE)
    o, ref = pair(s)
    ref.ortho()
    c = ref.get_wfn()
    a = Engine(s, p)
    monkeypatch.setenv("AMDK_NO_PENCIL", "1")
    b = Engine(s, p)
    for e in (a, b):
        e.set_wfn(c)
        e.density()
        e.potential()
        e.energy()
        e.apply_h()
    assert rel(b.get("rho"), a.get("rho")) < tol
    assert rel(b.get("c2"), a.get("c2")) < tol


def test_graph_replay_matches_eager(monkeypatch):
    """CG iterations replayed from CUDA graphs (the default from the second
    iteration on) give the eager launches' energies, gradients and C0, with
    and without the ionic forces segment."""
    s = configs.small_water(xc=XC_PBE)
    # measured launch shapes could differ between the two engines and change
    # the summation order; the model's choice is deterministic
    monkeypatch.setenv("AMDK_NO_TUNE", "1")
    o, ref = pair(s)
    c = ref.get_wfn()
    monkeypatch.setenv("AMDK_NO_GRAPHS", "1")
    eager = Engine(s, FP64)
    monkeypatch.delenv("AMDK_NO_GRAPHS")
    for e in (ref, eager):
        e.set_wfn(c)
        e.ortho()
    for it in range(1, 9):
        # a loose cutoff turns the forces segment on after a few iterations
        a = ref.scf_iteration(it, 5e-2)
        b = eager.scf_iteration(it, 5e-2)
        assert a[0]["etotal"] == b[0]["etotal"] and a[1] == b[1], it
    assert np.array_equal(ref.get_wfn(), eager.get_wfn())
    assert np.array_equal(ref.get("force"), eager.get("force"))


def test_graph_replay_with_profiling():
    """Profiled intervals recorded inside captured graphs are timed."""
    s = configs.small_water()
    o, e = pair(s)
    e.ortho()
    e.scf_iteration(1, 1e-7)
    e.profile(True)
    for it in range(2, 6):
        e.scf_iteration(it, 1e-7)
        assert e.last_iteration_ms() > 0
    got = [e.profile_get(k) for k in e.KERNELS]
    e.profile(False)
    assert all(n >= 4 and ms > 0 for n, ms, _ in got), got


@pytest.mark.parametrize("nmol", [1, 2, 5, 7, 8, 12, 16])
def test_ortho_matches_oracle_across_band_counts(nmol):
    """ortho_gs for band counts that are and are not multiples of the
    Cholesky kernel's 16-column blocks (4 to 64 bands)."""
    s = configs.cluster(nmol, 18.0, 900 + nmol, ecut=20.0)
    o, e = pair(s)
    assert o.ortho() == 0
    e.ortho()
    assert rel(e.get_wfn(), o.c0()) < 1e-11


def test_density_independent_of_measured_launch_shape(monkeypatch):
    """The density pair-group count is measured at first use; whatever it
    picks, the density equals the model choice's to rounding."""
    s = configs.water32()
    monkeypatch.setenv("AMDK_NO_TUNE", "1")
    ref = Engine(s, FP64)
    monkeypatch.delenv("AMDK_NO_TUNE")
    e = Engine(s, FP64)
    g = ref.gvectors()
    c = start_coefficients(g["hg"][: ref.ngpw], 2 * np.pi / s.alat, ref.nstate, 7)
    for x in (ref, e):
        x.set_wfn(c)
        x.ortho()
        x.density()
    assert rel(e.get("rho"), ref.get("rho")) < 1e-13


def test_side_stream_overlap_matches_single_stream(monkeypatch):
    """The C0-only work on the side stream (the default) leaves every result
    of the iteration unchanged."""
    monkeypatch.setenv("AMDK_NO_TUNE", "1")
    s = configs.small_water(xc=XC_PBE)
    o, a = pair(s)
    c = a.get_wfn()
    monkeypatch.setenv("AMDK_NO_OVERLAP", "1")
    b = Engine(s, FP64)
    monkeypatch.delenv("AMDK_NO_OVERLAP")
    for e in (a, b):
        e.set_wfn(c)
        e.ortho()
    for it in range(1, 7):
        ra = a.scf_iteration(it, 1e-7)
        rb = b.scf_iteration(it, 1e-7)
        assert ra[0] == rb[0] and ra[1] == rb[1], it
    assert np.array_equal(a.get_wfn(), b.get_wfn())
