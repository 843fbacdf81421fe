"""The slab decomposition's kernels on the GPU (amdk_slab_*): nranks ranks
held by one process (slab.LocalExchange moves the exchange buffers; every
rank's launches run one after the other on one stream, none waits on
another), against the oracle's vpsi and eval_density on the whole grid
(wfn_initialize.f90:283-362, density.f90:19-90).

Bars: FP64 1e-10 relative to the array's max, mixed (FP32 transforms) 1e-5."""
import numpy as np
import pytest

from amdkiit_b200 import configs
from amdkiit_b200.engine import FP64, MIXED, AmdkError, Engine
from amdkiit_b200.slab import LocalExchange, Slab, SlabLayout, apply_local_h, density
from oracle.oracle import Oracle
from tests.helpers import start_coefficients

pytestmark = pytest.mark.gpu

_REF = {}


def _reference(name):
    """Oracle C0 (orthonormal), V(r), vpsi's C2 and rho(r) of the system."""
    if name not in _REF:
        s = configs.small_water() if name == "small_water" else configs.water32()
        o = Oracle(s, 0)
        g = o.gvectors()
        o.set_wfn(start_coefficients(g["hg"][: o.ngpw], o.d("tpiba"), o.nstate, 21))
        assert o.ortho() == 0
        o.call("eval_density")
        o.call("rhor2g")
        o.call("eval_pot")
        o.call("cal_vpot_ex")
        o.call("vpsi")
        _REF[name] = (s, o.c0(), o.real_grid("v_pot"), o.c2(), o.real_grid("rho"))
    return _REF[name]


def _run(name, prec, nranks):
    import torch
    s, c0, v, c2_ref, rho_ref = _reference(name)
    e = Engine(s, prec)
    slabs = [Slab(e, nranks, r) for r in range(nranks)]
    lay = SlabLayout.of(s, nranks)
    for r, sl in enumerate(slabs):
        assert np.array_equal(sl.local_g, lay.local_g(r))
        assert sl.plane0 == lay.plane0[r] and sl.nplane == lay.plane0[r + 1] - lay.plane0[r]
    assert sum(sl.ngpw_local for sl in slabs) == e.ngpw
    assert sum(sl.gzero_local >= 0 for sl in slabs) == 1
    c0s = [torch.from_numpy(np.ascontiguousarray(c0[:, sl.local_g])).cuda() for sl in slabs]
    vs = [torch.from_numpy(np.ascontiguousarray(v[:, :, sl.plane0:sl.plane0 + sl.nplane])).cuda() for sl in slabs]
    c2s = [torch.zeros_like(c) for c in c0s]
    rhos = [torch.zeros_like(x) for x in vs]
    apply_local_h(slabs, LocalExchange(), c0s, vs, c2s)
    density(slabs, LocalExchange(), c0s, rhos)
    torch.cuda.synchronize()
    c2 = np.zeros_like(c0)
    rho = np.zeros_like(rho_ref)
    for sl, c2l, rl in zip(slabs, c2s, rhos):
        c2[:, sl.local_g] = c2l.cpu().numpy()
        rho[:, :, sl.plane0:sl.plane0 + sl.nplane] = rl.cpu().numpy()
    dc2 = np.abs(c2 - c2_ref).max() / np.abs(c2_ref).max()
    drho = np.abs(rho - rho_ref).max() / np.abs(rho_ref).max()
    for sl in slabs:
        sl.close()
    return dc2, drho


@pytest.mark.parametrize("prec", [FP64, MIXED])
@pytest.mark.parametrize("nranks", [1, 2, 3, 4])
def test_slab_small_water_matches_oracle(nranks, prec):
    dc2, drho = _run("small_water", prec, nranks)
    bar = 1e-10 if prec == FP64 else 1e-5
    assert dc2 < bar and drho < bar, (dc2, drho)


@pytest.mark.parametrize("prec,nranks", [(FP64, 2), (MIXED, 2), (MIXED, 8)])
def test_slab_water32_matches_oracle(prec, nranks):
    dc2, drho = _run("water32", prec, nranks)
    bar = 1e-10 if prec == FP64 else 1e-5
    print(prec, nranks, dc2, drho)
    assert dc2 < bar and drho < bar, (dc2, drho)


def test_slab_bad_arguments():
    s = configs.small_water()
    e = Engine(s, FP64)
    with pytest.raises(AmdkError):
        Slab(e, 2, 2)
    with pytest.raises(AmdkError):
        Slab(e, 17, 0)
    sl = Slab(e, 2, 0)
    import torch
    buf = torch.zeros(8, dtype=torch.float64, device="cuda")
    with pytest.raises(AmdkError):
        sl.pairs_out(buf, 1, 1, buf)  # odd band0
    with pytest.raises(AmdkError):
        sl.pairs_out(buf, 0, e.nstate, buf)  # pairs beyond the bands


@pytest.mark.parametrize("name,prec,nranks", [("small_water", FP64, 3), ("water32", MIXED, 4)])
def test_slab_local_h_from_c0_matches_oracle(name, prec, nranks):
    """The whole local part of H|psi> from a distributed C0 alone: rho(r) by
    the slab transforms, the slabs gathered into rho, the potential of that
    density (amdk_set_density + amdk_potential), each rank's V slab, then
    V(r)psi by the slab transforms; against the oracle's eval_density,
    eval_pot, cal_vpot_ex and vpsi from the same C0."""
    import torch
    from amdkiit_b200.slab import local_h_from_c0
    s, c0, v_ref, c2_ref, rho_ref = _reference(name)
    e = Engine(s, prec)
    slabs = [Slab(e, nranks, r) for r in range(nranks)]
    c0s = [torch.from_numpy(np.ascontiguousarray(c0[:, sl.local_g])).cuda() for sl in slabs]
    c2s = [torch.zeros_like(c) for c in c0s]
    rhos, vs = local_h_from_c0(e, slabs, LocalExchange(), c0s, c2s)
    torch.cuda.synchronize()
    c2 = np.zeros_like(c0)
    rho = np.zeros_like(rho_ref)
    v = np.zeros_like(v_ref)
    for sl, c2l, rl, vl in zip(slabs, c2s, rhos, vs):
        c2[:, sl.local_g] = c2l.cpu().numpy()
        rho[:, :, sl.plane0:sl.plane0 + sl.nplane] = rl.cpu().numpy()
        v[:, :, sl.plane0:sl.plane0 + sl.nplane] = vl.cpu().numpy()
    bar = 1e-10 if prec == FP64 else 1e-5
    errs = [np.abs(a - b).max() / np.abs(b).max() for a, b in ((rho, rho_ref), (v, v_ref), (c2, c2_ref))]
    print(name, prec, nranks, errs)
    assert max(errs) < bar, errs
    for sl in slabs:
        sl.close()


@pytest.mark.parametrize("name,nranks", [("small_water", 1), ("small_water", 3), ("water32", 4)])
def test_slab_gram_matches_numpy(name, nranks):
    """The band-space Gram product of a slab-decomposed pair of band arrays
    (each rank's share by the FP64 tensor cores, then the all-reduce): the
    overlap S of ortho_gs (wfn_initialize.f90:481-482) from C0 alone, and
    2 Re C0^H C2 - Re c0(0) Re c2(0) with C2 of vpsi, within 1e-12 of numpy."""
    import torch
    from amdkiit_b200.slab import gram
    s, c0, _, c2, _ = _reference(name)
    e = Engine(s, FP64)
    slabs = [Slab(e, nranks, r) for r in range(nranks)]
    n = e.nstate
    a_s = [torch.from_numpy(np.ascontiguousarray(c0[:, sl.local_g])).cuda() for sl in slabs]
    b_s = [torch.from_numpy(np.ascontiguousarray(c2[:, sl.local_g])).cuda() for sl in slabs]

    def ref(a, b):
        return 2.0 * (a.conj() @ b.T).real - np.outer(a[:, 0].real, b[:, 0].real)

    for got, want in ((gram(slabs, LocalExchange(), a_s, a_s, n)[0], ref(c0, c0)),
                      (gram(slabs, LocalExchange(), a_s, b_s, n)[0], ref(c0, c2))):
        err = np.abs(got.cpu().numpy() - want).max() / np.abs(want).max()
        print(name, nranks, err)
        assert err < 1e-12, err
    for sl in slabs:
        sl.close()
