"""Slab decomposition of the band-pair transforms, host side (no GPU).

- the partition (amdk_slab_layout, the library's host code): every G vector
  owned once, +G and -G rays with one owner, G counts balanced, contiguous
  plane ranges as distribute_YZplanes makes them (gvectors.f90:80-108);
- the driver (amdkiit_b200/slab.py) over two gloo ranks, with the library's
  kernels replaced by a numpy stand-in that keeps the library's buffer
  layouts (send [kx][pair][local ray] in rank order, receive blocks [plane]
  [pair][ray of the source]) and the all-to-all done by torch.distributed:
  the local H|psi> (vpsi) and rho(r) of every rank, gathered, equal the same
  transforms done on the whole grid in one process to round-off."""
import os
import socket

import numpy as np
import pytest

from amdkiit_b200 import configs
from amdkiit_b200.engine import host_gvectors
from amdkiit_b200.slab import LocalExchange, SlabLayout, TorchExchange, apply_local_h, density


def _grid_index(inyh, nr):
    """(kx, ky, kz) of +G and of -G for each G of the list (inyh 1-based centred)."""
    nh = np.array([n // 2 + 1 for n in nr])
    i = inyh - nh
    kp = np.mod(i, nr)
    km = np.mod(-i, nr)
    return kp, km


@pytest.mark.parametrize("nranks", [1, 2, 3, 4, 8])
def test_layout_partition(nranks):
    s = configs.water32()
    g = host_gvectors(s)
    lay = SlabLayout.of(s, nranks)
    ngpw, nr = g["ngpw"], np.array(g["nr"])
    assert lay.g_owner.shape == (ngpw,) and lay.g_owner.min() == 0 and lay.g_owner.max() == nranks - 1
    kp, km = _grid_index(g["inyh"][:ngpw], nr)
    # one owner per ray, whether the ray holds +G or -G positions
    owner_of = {}
    for o, a, b in zip(lay.g_owner, map(tuple, kp[:, 1:]), map(tuple, km[:, 1:])):
        for ray in (a, b):
            assert owner_of.setdefault(ray, o) == o
    # mirror rays together
    for (ky, kz), o in owner_of.items():
        assert owner_of[((-ky) % nr[1], (-kz) % nr[2])] == o
    counts = np.bincount(lay.g_owner, minlength=nranks)
    assert counts.max() <= 1.02 * ngpw / nranks + 2 * nr[0]
    p0 = lay.plane0
    assert p0[0] == 0 and p0[-1] == nr[0] and np.all(np.diff(p0) >= 1)
    assert np.all(p0 == (np.arange(nranks + 1) * nr[0]) // nranks)


def test_layout_rejects_bad_nranks():
    s = configs.small_water()
    with pytest.raises(ValueError):
        SlabLayout.of(s, 0)
    with pytest.raises(ValueError):
        SlabLayout.of(s, 17)


# ----------------------------------------------------------------- stand-in
class NumpySlab:
    """The library's four slab calls in numpy, same buffer layouts (torch CPU
    tensors for the exchange buffers, complex128 arrays for C0/C2)."""

    def __init__(self, system, nranks, rank):
        import torch
        self.torch = torch
        g = host_gvectors(system)
        lay = SlabLayout.of(system, nranks)
        self.nr = np.array(g["nr"])
        n1 = self.nr[0]
        ngpw = g["ngpw"]
        self.nranks, self.rank = nranks, rank
        self.tpiba2 = (2 * np.pi / system.alat) ** 2
        kp, km = _grid_index(g["inyh"][:ngpw], self.nr)
        # rays of every rank: sorted (ky, kz) of their +G and -G positions
        self.rays = []
        for o in range(nranks):
            sel = lay.g_owner == o
            keys = {tuple(r) for r in kp[sel, 1:]} | {tuple(r) for r in km[sel, 1:]}
            self.rays.append(sorted(keys))
        self.local_g = lay.local_g(rank)
        self.ngpw_local = len(self.local_g)
        ridx = {k: j for j, k in enumerate(self.rays[rank])}
        self.kp = kp[self.local_g]
        self.km = km[self.local_g]
        self.rp = np.array([ridx[tuple(k)] for k in self.kp[:, 1:]])
        self.rm = np.array([ridx[tuple(k)] for k in self.km[:, 1:]])
        self.hg = g["hg"][self.local_g]
        self.gzero = int(np.flatnonzero(self.local_g == 0)[0]) if 0 in self.local_g else -1
        self.plane0 = int(lay.plane0[rank])
        self.nplane = int(lay.plane0[rank + 1] - lay.plane0[rank])
        self.planes = np.diff(lay.plane0)
        self.nray_local = len(self.rays[rank])
        zv = sum(sp.zv * n for sp, n in zip(system.species, system.na))
        self.nstate = int(round(zv)) // 2
        self.occ = np.full(self.nstate, 2.0)
        self.omega = g["omega"]
        self.send_elems = [int(self.planes[r]) * self.nray_local for r in range(nranks)]
        self.recv_elems = [self.nplane * len(self.rays[s]) for s in range(nranks)]

    def send_counts(self, npairs):
        return [2 * npairs * e for e in self.send_elems]

    def recv_counts(self, npairs):
        return [2 * npairs * e for e in self.recv_elems]

    def new_send(self, npairs):
        return self.torch.zeros(sum(self.send_counts(npairs)), dtype=self.torch.float64)

    @staticmethod
    def _c(t):
        return t.numpy().view(np.complex128)

    def pairs_out(self, c0, band0, T, send):
        n1, R = self.nr[0], self.nray_local
        lines = np.zeros((T, R, n1), np.complex128)
        for t in range(T):
            a = c0[band0 + 2 * t]
            b = c0[band0 + 2 * t + 1] if band0 + 2 * t + 1 < self.nstate else np.zeros_like(a)
            lines[t, self.rm, self.km[:, 0]] = np.conj(a) + 1j * np.conj(b)
            lines[t, self.rp, self.kp[:, 0]] = a + 1j * b  # G = 0: the +G value
        x = np.fft.ifft(lines, axis=2) * n1  # backward: exp(+i G x)
        self._c(send)[:] = x.transpose(2, 0, 1).ravel()  # [kx][t][ray]

    def _planes(self, recv, T):
        n2, n3 = self.nr[1], self.nr[2]
        buf = self._c(recv)
        P = np.zeros((self.nplane, T, n2, n3), np.complex128)
        off = 0
        for s in range(self.nranks):
            rs = self.rays[s]
            blk = buf[off:off + self.nplane * T * len(rs)].reshape(self.nplane, T, len(rs))
            ky = np.array([k[0] for k in rs], int)
            kz = np.array([k[1] for k in rs], int)
            P[:, :, ky, kz] = blk
            off += blk.size
        return np.fft.ifft2(P, axes=(2, 3)) * (n2 * n3)

    def planes_vpsi(self, recv, T, v):
        n2, n3 = self.nr[1], self.nr[2]
        psi = self._planes(recv, T)
        vx = np.transpose(v, (2, 1, 0))  # [kz][ky][xl] -> [xl][ky][kz]
        F = np.fft.fft2(psi * vx[:, None], axes=(2, 3))
        buf = self._c(recv)
        off = 0
        for s in range(self.nranks):
            rs = self.rays[s]
            ky = np.array([k[0] for k in rs], int)
            kz = np.array([k[1] for k in rs], int)
            n = self.nplane * T * len(rs)
            buf[off:off + n] = F[:, :, ky, kz].ravel()
            off += n

    def planes_density(self, recv, band0, T, rho, accumulate):
        psi = self._planes(recv, T)
        p = band0 // 2
        r = np.zeros((self.nplane,) + tuple(self.nr[1:]))
        for t in range(T):
            wa = self.occ[2 * (p + t)] / self.omega
            wb = self.occ[2 * (p + t) + 1] / self.omega if 2 * (p + t) + 1 < self.nstate else 0.0
            r += wa * psi[:, t].real ** 2 + wb * psi[:, t].imag ** 2
        r = np.transpose(r, (2, 1, 0))
        if accumulate:
            rho += r
        else:
            rho[:] = r

    def pairs_in(self, back, c0, band0, T, c2):
        n1, R = self.nr[0], self.nray_local
        x = self._c(back).reshape(n1, T, R).transpose(1, 2, 0)
        f = np.fft.fft(x, axis=2) / np.prod(self.nr)
        for t in range(T):
            vp = f[t, self.rp, self.kp[:, 0]]
            vm = f[t, self.rm, self.km[:, 0]]
            fp, fm = vp + vm, vp - vm
            kin = self.tpiba2 * self.hg
            for band, val in ((band0 + 2 * t, fp.real + 1j * fm.imag), (band0 + 2 * t + 1, fp.imag - 1j * fm.real)):
                if band < self.nstate:
                    fi = self.occ[band] * 0.5 or 1.0
                    c2[band] = -fi * (kin * c0[band] + val)


def _full_reference(system, c0, v):
    """The same transforms on the whole grid in one process."""
    s = NumpySlab(system, 1, 0)
    T = (s.nstate + 1) // 2
    send = s.new_send(T)
    s.pairs_out(c0, 0, T, send)
    rho = np.zeros(tuple(s.nr[::-1]))
    s.planes_density(send.clone(), 0, T, rho, False)
    s.planes_vpsi(send, T, v)
    c2 = np.zeros_like(c0)
    s.pairs_in(send, c0, 0, T, c2)
    return c2, rho


def _inputs(system):
    rng = np.random.default_rng(5)
    g = host_gvectors(system)
    s = NumpySlab(system, 1, 0)
    c0 = rng.normal(size=(s.nstate, g["ngpw"])) + 1j * rng.normal(size=(s.nstate, g["ngpw"]))
    c0[:, 0] = c0[:, 0].real
    v = rng.normal(size=tuple(np.array(g["nr"])[::-1]))
    return c0, v


def _rank_run(rank, nranks, port, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks)
    try:
        system = configs.small_water()
        c0, v = _inputs(system)
        s = NumpySlab(system, nranks, rank)
        c0l = np.ascontiguousarray(c0[:, s.local_g])
        vl = np.ascontiguousarray(v[:, :, s.plane0:s.plane0 + s.nplane])
        c2l = np.zeros_like(c0l)
        rho = np.zeros_like(vl)
        ex = TorchExchange()
        apply_local_h([s], ex, [c0l], [vl], [c2l])
        density([s], ex, [c0l], [rho])
        q.put((rank, s.local_g, c2l, s.plane0, rho))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def test_two_gloo_ranks_match_one_process():
    import torch.multiprocessing as mp
    system = configs.small_water()
    c0, v = _inputs(system)
    c2_ref, rho_ref = _full_reference(system, c0, v)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_run, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    c2 = np.zeros_like(c0)
    rho = np.zeros_like(rho_ref)
    for rank, lg, c2l, p0, rl in res:
        c2[:, lg] = c2l
        rho[:, :, p0:p0 + rl.shape[2]] = rl
    assert np.abs(c2 - c2_ref).max() < 1e-12 * np.abs(c2_ref).max()
    assert np.abs(rho - rho_ref).max() < 1e-12 * np.abs(rho_ref).max()


@pytest.mark.parametrize("nranks", [3, 4])
def test_local_exchange_matches_one_process(nranks):
    """Several ranks in one process (LocalExchange), as the GPU test runs them."""
    system = configs.small_water()
    c0, v = _inputs(system)
    c2_ref, rho_ref = _full_reference(system, c0, v)
    slabs = [NumpySlab(system, nranks, r) for r in range(nranks)]
    c0s = [np.ascontiguousarray(c0[:, s.local_g]) for s in slabs]
    vs = [np.ascontiguousarray(v[:, :, s.plane0:s.plane0 + s.nplane]) for s in slabs]
    c2s = [np.zeros_like(c) for c in c0s]
    rhos = [np.zeros_like(x) for x in vs]
    apply_local_h(slabs, LocalExchange(), c0s, vs, c2s)
    density(slabs, LocalExchange(), c0s, rhos)
    c2 = np.zeros_like(c0)
    rho = np.zeros_like(rho_ref)
    for s, c2l, rl in zip(slabs, c2s, rhos):
        c2[:, s.local_g] = c2l
        rho[:, :, s.plane0:s.plane0 + s.nplane] = rl
    assert np.abs(c2 - c2_ref).max() < 1e-12 * np.abs(c2_ref).max()
    assert np.abs(rho - rho_ref).max() < 1e-12 * np.abs(rho_ref).max()


def test_stand_in_matches_oracle_vpsi_and_density():
    """The stand-in's layouts carry the reference's vpsi and eval_density
    (the oracle, density.f90:19-90, wfn_initialize.f90:283-362) on small
    water, so the multi-rank checks above check those transforms."""
    from oracle.oracle import Oracle
    from tests.helpers import start_coefficients
    system = configs.small_water()
    o = Oracle(system, 0)
    g = o.gvectors()
    o.set_wfn(start_coefficients(g["hg"][: o.ngpw], o.d("tpiba"), o.nstate, 11))
    assert o.ortho() == 0
    c0 = o.c0()
    o.call("eval_density")
    o.call("rhor2g")
    o.call("eval_pot")
    o.call("cal_vpot_ex")
    o.call("vpsi")
    c2_ref, rho_ref, v = o.c2(), o.real_grid("rho"), o.real_grid("v_pot")
    slabs = [NumpySlab(system, 2, r) for r in range(2)]
    c0s = [np.ascontiguousarray(c0[:, s.local_g]) for s in slabs]
    vs = [np.ascontiguousarray(v[:, :, s.plane0:s.plane0 + s.nplane]) for s in slabs]
    c2s = [np.zeros_like(c) for c in c0s]
    rhos = [np.zeros_like(x) for x in vs]
    apply_local_h(slabs, LocalExchange(), c0s, vs, c2s)
    density(slabs, LocalExchange(), c0s, rhos)
    c2 = np.zeros_like(c0)
    rho = np.zeros_like(rho_ref)
    for s, c2l, rl in zip(slabs, c2s, rhos):
        c2[:, s.local_g] = c2l
        rho[:, :, s.plane0:s.plane0 + s.nplane] = rl
    assert np.abs(c2 - c2_ref).max() < 1e-11 * np.abs(c2_ref).max()
    assert np.abs(rho - rho_ref).max() < 1e-11 * np.abs(rho_ref).max()


def _gather_rank(rank, nranks, port, q):
    import torch
    import torch.distributed as dist
    from amdkiit_b200.slab import plane_ranges
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=nranks)
    try:
        full = np.arange(5 * 4 * 9, dtype=np.float64).reshape(5, 4, 9)
        p0 = plane_ranges(9, nranks)
        mine = torch.from_numpy(np.ascontiguousarray(full[:, :, p0[rank]:p0[rank + 1]]))
        got = TorchExchange().gather_planes([mine], p0)[0].numpy()
        q.put((rank, bool(np.array_equal(got, full))))
    finally:
        dist.destroy_process_group()


def test_density_slabs_gathered_over_gloo():
    """The all-gather of the ranks' x-plane slabs (uneven plane counts: 9
    planes over 2 ranks) rebuilds the whole grid on every rank, as the
    potential between the two passes of a distributed H|psi> needs."""
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=300) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert all(ok for _, ok in res), res


def test_local_exchange_gathers_planes():
    import torch
    from amdkiit_b200.slab import plane_ranges
    full = np.random.default_rng(3).normal(size=(6, 5, 11))
    p0 = plane_ranges(11, 3)
    parts = [torch.from_numpy(np.ascontiguousarray(full[:, :, p0[r]:p0[r + 1]])) for r in range(3)]
    for got in LocalExchange().gather_planes(parts, p0):
        assert np.array_equal(got.numpy(), full)


def test_local_exchange_all_reduce():
    import torch
    parts = [torch.full((3, 3), float(r + 1)) for r in range(4)]
    for got in LocalExchange().all_reduce(parts):
        assert torch.equal(got, torch.full((3, 3), 10.0))
