"""Host logic of Engine.wfn_opt that needs no GPU: when a mixed-precision
engine hands the CG iterations over to FP64 (GEMAX below max(gcut, 1e-6), or
no new GEMAX minimum for MIXED_STALL iterations once GEMAX is within
MIXED_STALL_ZONE of that threshold) and that it then iterates in FP64 to
gcut.  The engine's GPU calls are replaced by a scripted GEMAX sequence."""
from amdkiit_b200 import engine as eng
from amdkiit_b200.engine import FP64, MIXED, Engine


def scripted(gemax_mixed, gemax_fp64):
    """An Engine whose scf_iteration returns the next scripted GEMAX of the
    current pair precision; records the precision of every iteration."""
    e = object.__new__(Engine)
    e.precision = MIXED
    e.pair_precision = MIXED
    e.trace = []
    it = {MIXED: iter(gemax_mixed), FP64: iter(gemax_fp64)}

    def set_precision(p):
        e.pair_precision = p

    def scf_iteration(i, gcut):
        g = next(it[e.pair_precision])
        e.trace.append((e.pair_precision, g))
        return {"etotal": -1.0}, g, g < gcut

    e.set_precision = set_precision
    e.scf_iteration = scf_iteration
    return e


def test_hand_over_at_the_mixed_threshold_then_fp64_to_gcut():
    e = scripted([1e-3, 1e-4, 5e-6, 8e-7, 5e-7], [3e-7, 2e-7, 9e-8, 5e-8])
    n, en, g = e.wfn_opt(100, 1e-7)
    precs = [p for p, _ in e.trace]
    assert precs == [MIXED] * 4 + [FP64] * 3  # 8e-7 < 1e-6 hands over
    assert g == 9e-8 and n == 7
    assert e.pair_precision == MIXED  # restored for the next geometry


def test_loose_gcut_keeps_one_fp64_iteration():
    e = scripted([1e-3, 5e-7, 1e-7], [4e-7, 3e-7])
    n, en, g = e.wfn_opt(100, 1e-6)
    assert [p for p, _ in e.trace] == [MIXED, MIXED, FP64]
    assert n == 3 and g == 4e-7


def test_hand_over_when_mixed_gemax_stalls():
    stall = [2e-6] + [3e-6] * eng.MIXED_STALL + [1e-9]
    e = scripted(stall, [5e-7, 9e-8])
    n, en, g = e.wfn_opt(200, 1e-7)
    precs = [p for p, _ in e.trace]
    assert precs.count(MIXED) == 1 + eng.MIXED_STALL
    assert precs[-2:] == [FP64, FP64] and g == 9e-8


def test_no_refinement_requested():
    e = scripted([1e-3, 5e-8], [])
    n, en, g = e.wfn_opt(100, 1e-7, refine=False)
    assert [p for p, _ in e.trace] == [MIXED, MIXED] and n == 2


def test_plateau_far_above_the_threshold_stays_mixed():
    """A plateau at 1e-4 (the CG's own, as on bulk Si in FP64) does not hand
    over: only GEMAX below the threshold does."""
    plateau = [1e-3] + [2e-4] * (3 * eng.MIXED_STALL) + [5e-7]
    e = scripted(plateau, [9e-8])
    n, en, g = e.wfn_opt(400, 1e-7)
    precs = [p for p, _ in e.trace]
    assert precs.count(MIXED) == len(plateau) and precs[-1] == FP64
