"""The FP64 tensor-core products (csrc/dgemm.cuh) and the Cholesky against
numpy in FP64, on band counts that cover one and several 64 x 64 output
tiles, partial tiles, band chunks of 128 in the rotation, the symmetric
(upper-tile) Gram, and above 144 bands the blocked factorisation (160 and
300 bands: two and three blocks of 128):

- the overlap S = 2 Re C0^T C0 - Re c0(0) Re c0(0)^T of ortho_gs
  (wfn_initialize.f90:481-482), read back with amdk_get_array("overlap");
- the orthonormalised C0 = C0 U^{-1}, S = U^T U (wfn_initialize.f90:485)."""
import numpy as np
import pytest

from amdkiit_b200 import configs
from amdkiit_b200.engine import FP64, MIXED, AmdkError, Engine
from tests.helpers import start_coefficients

pytestmark = pytest.mark.gpu


def _overlap(c):
    re0 = c[:, 0].real
    return 2.0 * (c.conj() @ c.T).real - np.outer(re0, re0)


def _check_overlap(e, c):
    """The upper triangle of the device overlap (column-major; the G = 0
    correction is applied to the upper triangle only, which is all the
    Cholesky reads, as DSYRK + DGER leave it in the reference)."""
    S = _overlap(c)
    Sg = e.get("overlap").reshape(e.nstate, e.nstate).T  # Sg[i, j] = S(i, j)
    err = np.triu(np.abs(Sg - S))
    i, j = np.unravel_index(np.argmax(err), err.shape)
    assert err.max() < 1e-12 * np.abs(S).max(), f"overlap: max error {err.max():.3e} at ({i}, {j}) of {S.shape}"


CASES = [(1, 12.0, 501, 30.0, FP64), (3, 13.5, 503, 30.0, FP64), (2, 14.0, 502, 30.0, FP64), (5, 15.2, 705, 16.0, MIXED),
         (16, 18.1, 716, 16.0, FP64), (18, 18.4, 718, 16.0, FP64), (33, 20.5, 733, 16.0, FP64),
         # above 144 bands: the blocked Cholesky and inverse (blocks of 128)
         (40, 22.0, 740, 16.0, FP64), (75, 26.0, 775, 14.0, MIXED)]


@pytest.mark.parametrize("nwat,box,seed,ecut,prec", CASES)
def test_overlap_and_rotation_match_numpy(nwat, box, seed, ecut, prec):
    s = configs.cluster(nwat, box, seed, ecut=ecut)
    e = Engine(s, prec)
    g = e.gvectors()
    c = start_coefficients(g["hg"][: e.ngpw], 2 * np.pi / s.alat, e.nstate)
    e.set_wfn(c)
    failed = None
    try:
        e.ortho()
    except AmdkError as ex:  # report the overlap's error first
        failed = ex
    _check_overlap(e, c)
    if failed:
        raise failed
    U = np.linalg.cholesky(_overlap(c)).T  # S = U^T U, U upper
    ref = np.linalg.solve(U.T, c)  # rows: sum_b Uinv[b, j] c[b] = (U^-T c)[j]
    ref[:, 0] = ref[:, 0].real
    got = e.get_wfn()
    d = np.abs(got - ref).max() / np.abs(ref).max()
    assert d < 1e-11, f"C0 U^-1: relative error {d:.3e}"


def test_several_contexts_alive():
    """Contexts created side by side (as an ensemble's members are), each
    orthonormalising its own start."""
    engines = []
    for nwat, box, seed, ecut, prec in CASES[:3]:
        s = configs.cluster(nwat, box, seed, ecut=ecut)
        pair = [Engine(s, FP64), Engine(s, FP64)]
        engines += pair
        g = pair[0].gvectors()
        c = start_coefficients(g["hg"][: pair[0].ngpw], 2 * np.pi / s.alat, pair[0].nstate)
        for e in pair:
            e.set_wfn(c)
            failed = None
            try:
                e.ortho()
            except AmdkError as ex:
                failed = ex
            _check_overlap(e, c)
            if failed:
                raise failed
