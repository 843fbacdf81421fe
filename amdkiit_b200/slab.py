"""Slab decomposition of the band-pair transforms over several processes.

The reference distributes every 3D FFT over its MPI ranks as x-rays in G
space and contiguous ranges of x planes in real space, with an all-to-all
between the x pass and the y/z passes (fft_interface.f90:109-119 forward,
:129-137 backward; the exchange is MPI_trans through FFT_COMM, :500-511; the
plane ranges come from distribute_YZplanes, gvectors.f90:80-108, the ray
assignment from gvectors.f90:150-166).  Here each rank owns

- the plane-wave G vectors on its rays (rays in mirror pairs {(ky, kz),
  (-ky, -kz)}, so that both +G and -G of an owned G lie on the rank's rays
  and the pack/unpack of a band pair needs no remote coefficient), with its
  share of C0 and C2 as [nstate][ngpw_local] arrays;
- the x planes [plane0, plane0 + nplane) of the real-space grid, with its
  slab of V(r) and rho(r) as [kz][ky][x] arrays (x over the local planes).

One pass over a batch of band pairs is four library calls around two
all-to-alls:

    pairs_out   pack + backward x pass of the local rays, written straight
                into the send buffer in destination-rank order
    all-to-all  (NCCL over NVLink between GPUs)
    planes_*    y/z passes of the local planes, reading each source rank's
                block of the receive buffer in place; V(r)psi (in place)
                or the density sums
    all-to-all  (the same counts, reversed; V(r)psi only)
    pairs_in    forward x pass + unpack of the local G: C2 = -f (G^2/2 C0
                + FFT(V psi)), vpsi without fnonloc (wfn_initialize.f90:
                283-362)

so the exchange is fused with the pack and the unpack: no kernel copies the
ray data into or out of a staging layout.  The potential between the two
passes (`local_h_from_c0`) is computed on every rank from the gathered
density (the slabs' planes all-gathered, 8 MB at water32): the density-sphere
fields stay replicated.  The band-space products that
follow (Gram matrices, projections, norms) are sums over G and take an
all-reduce of the local sums, as the reference's are (mympi.f90).

`Exchange` objects implement the all-to-all for a list of ranks held by this
process: `TorchExchange` (one rank per process, torch.distributed, NCCL on
GPUs, gloo on the CPU) and `LocalExchange` (several ranks in one process,
the exchange as copies; it runs the ranks' launches one after the other on
one device, no launch waits on another).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Sequence

import numpy as np

from .engine import FP64, _check, load_library, system_struct
from .inputs import System

MAXRANKS = 16


class _SlabInfo(C.Structure):
    _fields_ = [("nranks", C.c_int), ("rank", C.c_int), ("ngpw_local", C.c_int), ("nray_local", C.c_int),
                ("plane0", C.c_int), ("nplane", C.c_int), ("gzero_local", C.c_int), ("elem_bytes", C.c_int),
                ("send_elems", C.c_long * MAXRANKS), ("recv_elems", C.c_long * MAXRANKS)]


def _bind(lib):
    if getattr(lib, "_slab_bound", False):
        return lib
    P = C.c_void_p
    IP = C.POINTER(C.c_int)
    from .engine import _System
    lib.amdk_slab_layout.argtypes = [C.POINTER(_System), C.c_int, IP, IP]
    lib.amdk_slab_create.argtypes = [P, C.c_int, C.c_int, C.POINTER(P)]
    lib.amdk_slab_info_get.argtypes = [P, C.POINTER(_SlabInfo)]
    lib.amdk_slab_local_g.argtypes = [P, IP]
    lib.amdk_slab_pairs_out.argtypes = [P, P, C.c_int, C.c_int, P, P]
    lib.amdk_slab_planes_vpsi.argtypes = [P, P, C.c_int, P, P]
    lib.amdk_slab_planes_density.argtypes = [P, P, C.c_int, C.c_int, P, C.c_int, P]
    lib.amdk_slab_pairs_in.argtypes = [P, P, P, C.c_int, C.c_int, P, P]
    lib.amdk_slab_gram.argtypes = [P, P, P, C.c_int, P, P]
    lib.amdk_slab_destroy.argtypes = [P]
    lib._slab_bound = True
    return lib


@dataclass
class SlabLayout:
    """Owner of every plane-wave G vector and the x-plane ranges (host only,
    no GPU): g_owner[ig] is the rank of G vector ig (0-based, the library's G
    order), plane0[r] .. plane0[r+1]-1 the x planes of rank r."""
    nranks: int
    g_owner: np.ndarray
    plane0: np.ndarray

    @staticmethod
    def of(system: System, nranks: int) -> "SlabLayout":
        from .engine import host_gvectors
        if not 1 <= nranks <= MAXRANKS:
            raise ValueError(f"nranks must be 1..{MAXRANKS}")
        lib = _bind(load_library())
        ngpw = host_gvectors(system)["ngpw"]
        s, keep = system_struct(system)
        g_owner = np.zeros(ngpw, np.int32)
        plane0 = np.zeros(nranks + 1, np.int32)
        _check(lib.amdk_slab_layout(C.byref(s), nranks, g_owner.ctypes.data_as(C.POINTER(C.c_int)),
                                    plane0.ctypes.data_as(C.POINTER(C.c_int))), "amdk_slab_layout")
        return SlabLayout(nranks, g_owner, plane0)

    def local_g(self, rank: int) -> np.ndarray:
        return np.flatnonzero(self.g_owner == rank)


def _ptr(t) -> int:
    return t.data_ptr()


class Slab:
    """One rank's share of the band-pair transforms of an Engine's system
    (the Engine's context supplies the grid, tables and precision).  The
    buffers are torch tensors on the Engine's device: C0/C2 complex128
    [nstate, ngpw_local], V/rho float64 [n3, n2, nplane], the exchange
    buffers real tensors of 2 x elements (float64 FP64, float32 mixed)."""

    def __init__(self, engine, nranks: int, rank: int):
        self.lib = _bind(load_library())
        self.engine = engine
        h = C.c_void_p()
        _check(self.lib.amdk_slab_create(engine.h, nranks, rank, C.byref(h)), "amdk_slab_create")
        self.h = h
        info = _SlabInfo()
        _check(self.lib.amdk_slab_info_get(self.h, C.byref(info)), "amdk_slab_info_get")
        self.nranks, self.rank = info.nranks, info.rank
        self.ngpw_local, self.nray_local = info.ngpw_local, info.nray_local
        self.plane0, self.nplane = info.plane0, info.nplane
        self.gzero_local = info.gzero_local
        self.elem_bytes = info.elem_bytes
        self.send_elems = [int(info.send_elems[r]) for r in range(nranks)]
        self.recv_elems = [int(info.recv_elems[r]) for r in range(nranks)]
        ig = np.zeros(self.ngpw_local, np.int32)
        _check(self.lib.amdk_slab_local_g(self.h, ig.ctypes.data_as(C.POINTER(C.c_int))), "amdk_slab_local_g")
        self.local_g = ig
        self.nstate = engine.nstate
        n1, n2, n3 = engine.nr
        self.grid = (n3, n2, self.nplane)

    # exchange buffers: counts in real scalars (two per complex element)
    def send_counts(self, npairs: int) -> List[int]:
        return [2 * npairs * e for e in self.send_elems]

    def recv_counts(self, npairs: int) -> List[int]:
        return [2 * npairs * e for e in self.recv_elems]

    def _dtype(self):
        import torch
        return torch.float64 if self.elem_bytes == 16 else torch.float32

    def new_send(self, npairs: int):
        import torch
        return torch.empty(sum(self.send_counts(npairs)), dtype=self._dtype(), device="cuda")

    @staticmethod
    def _stream():
        import torch
        return C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def pairs_out(self, c0, band0: int, npairs: int, send):
        _check(self.lib.amdk_slab_pairs_out(self.h, _ptr(c0), band0, npairs, _ptr(send), self._stream()),
               "amdk_slab_pairs_out")

    def planes_vpsi(self, recv, npairs: int, v):
        _check(self.lib.amdk_slab_planes_vpsi(self.h, _ptr(recv), npairs, _ptr(v), self._stream()),
               "amdk_slab_planes_vpsi")

    def planes_density(self, recv, band0: int, npairs: int, rho, accumulate: bool):
        _check(self.lib.amdk_slab_planes_density(self.h, _ptr(recv), band0, npairs, _ptr(rho), int(accumulate),
                                                 self._stream()), "amdk_slab_planes_density")

    def pairs_in(self, back, c0, band0: int, npairs: int, c2):
        _check(self.lib.amdk_slab_pairs_in(self.h, _ptr(back), _ptr(c0), band0, npairs, _ptr(c2), self._stream()),
               "amdk_slab_pairs_in")

    def gram(self, a, b, n: int, out):
        """out (n x n float64, column-major) = this rank's share of 2 Re a^H b
        over its G vectors (the G = 0 term once, on its owner)."""
        _check(self.lib.amdk_slab_gram(self.h, _ptr(a), _ptr(b), n, _ptr(out), self._stream()), "amdk_slab_gram")

    def close(self):
        if getattr(self, "h", None):
            self.lib.amdk_slab_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class TorchExchange:
    """The all-to-all of one rank per process through torch.distributed
    (all_to_all_single: NCCL between GPUs, gloo on the CPU)."""

    def __init__(self, group=None):
        self.group = group

    def __call__(self, sends: Sequence, send_counts: Sequence[Sequence[int]], recv_counts: Sequence[Sequence[int]]):
        import torch
        import torch.distributed as dist
        if len(sends) != 1:
            raise ValueError("TorchExchange moves the buffers of one rank per process")
        out = torch.empty(sum(recv_counts[0]), dtype=sends[0].dtype, device=sends[0].device)
        dist.all_to_all_single(out, sends[0], list(recv_counts[0]), list(send_counts[0]), group=self.group)
        return [out]

    def all_reduce(self, parts):
        """The sum over ranks of each rank's array (a band-space partial sum)."""
        import torch.distributed as dist
        out = parts[0].clone()
        dist.all_reduce(out, group=self.group)
        return [out]

    def gather_planes(self, parts, plane0):
        """Every rank's [nr3][nr2][nplane] slab assembled along x into the full
        grid (all_gather of slabs padded to the largest plane count)."""
        import torch
        import torch.distributed as dist
        x = parts[0]
        counts = np.diff(plane0)
        pad = torch.zeros(x.shape[:2] + (int(counts.max()),), dtype=x.dtype, device=x.device)
        pad[:, :, : x.shape[2]] = x
        outs = [torch.empty_like(pad) for _ in counts]
        dist.all_gather(outs, pad, group=self.group)
        return [torch.cat([o[:, :, : int(c)] for o, c in zip(outs, counts)], dim=2)]


class LocalExchange:
    """The all-to-all among ranks held by one process: receive buffer r is
    the concatenation over sources s of the block s addressed to r."""

    def __call__(self, sends: Sequence, send_counts: Sequence[Sequence[int]], recv_counts: Sequence[Sequence[int]]):
        import torch
        R = len(sends)
        offs = [np.concatenate([[0], np.cumsum(send_counts[s])]) for s in range(R)]
        outs = []
        for r in range(R):
            parts = [sends[s][int(offs[s][r]):int(offs[s][r + 1])] for s in range(R)]
            out = torch.cat(parts)
            if out.numel() != sum(recv_counts[r]):
                raise ValueError("send and receive counts disagree")
            outs.append(out)
        return outs

    def all_reduce(self, parts):
        """The sum over the ranks' arrays (in rank order), one copy per rank."""
        total = parts[0].clone()
        for p in parts[1:]:
            total += p
        return [total for _ in parts]

    def gather_planes(self, parts, plane0):
        """The ranks' slabs assembled along x into the full grid, one copy per rank."""
        import torch
        full = torch.cat(list(parts), dim=2)
        return [full for _ in parts]


def _pair_range(nstate: int, band0: int, npairs):
    if band0 % 2:
        raise ValueError("band0 must be even (bands are transformed in pairs)")
    total = (nstate + 1) // 2 - band0 // 2
    return total if npairs is None else npairs


def apply_local_h(slabs: Sequence, exchange, c0s: Sequence, vs: Sequence, c2s: Sequence, band0: int = 0,
                  npairs=None):
    """C2 = -f (G^2/2 C0 + FFT(V psi)) on every rank's G vectors for the band
    pairs [band0/2, band0/2 + npairs): the local part of H|psi> (vpsi)."""
    npairs = _pair_range(slabs[0].nstate, band0, npairs)
    sends = []
    for s, c0 in zip(slabs, c0s):
        buf = s.new_send(npairs)
        s.pairs_out(c0, band0, npairs, buf)
        sends.append(buf)
    sc = [s.send_counts(npairs) for s in slabs]
    rc = [s.recv_counts(npairs) for s in slabs]
    recvs = exchange(sends, sc, rc)
    for s, buf, v in zip(slabs, recvs, vs):
        s.planes_vpsi(buf, npairs, v)
    backs = exchange(recvs, rc, sc)
    for s, buf, c0, c2 in zip(slabs, backs, c0s, c2s):
        s.pairs_in(buf, c0, band0, npairs, c2)


def density(slabs: Sequence, exchange, c0s: Sequence, rhos: Sequence, band0: int = 0, npairs=None,
            accumulate: bool = False):
    """rho(r) = sum_b f_b/Omega |psi_b(r)|^2 over the band pairs on every
    rank's x planes (eval_density, density.f90:19-90)."""
    npairs = _pair_range(slabs[0].nstate, band0, npairs)
    sends = []
    for s, c0 in zip(slabs, c0s):
        buf = s.new_send(npairs)
        s.pairs_out(c0, band0, npairs, buf)
        sends.append(buf)
    recvs = exchange(sends, [s.send_counts(npairs) for s in slabs], [s.recv_counts(npairs) for s in slabs])
    for s, buf, rho in zip(slabs, recvs, rhos):
        s.planes_density(buf, band0, npairs, rho, accumulate)


def potential_slabs(engine, slabs: Sequence, exchange, rhos: Sequence):
    """V(r) on every rank's x planes from the ranks' density slabs: the slabs
    gathered into rho(r), eval_pot + cal_vpot_ex (potential.f90:4-46,
    xc.f90:4-434) on that full grid, each rank keeping its planes."""
    import torch
    fulls = exchange.gather_planes(rhos, plane_ranges(engine.nr[0], slabs[0].nranks))
    vs = []
    for s, full in zip(slabs, fulls):
        engine.set_density(full.cpu().numpy())
        engine.potential()
        v = engine.get("v_pot")
        vs.append(torch.from_numpy(np.ascontiguousarray(v[:, :, s.plane0:s.plane0 + s.nplane])).to(rhos[0].device))
    return vs


def plane_ranges(n1: int, nranks: int) -> np.ndarray:
    """plane0[0..nranks] of the decomposition: rank r holds x planes
    floor(r n1 / nranks) .. floor((r+1) n1 / nranks) - 1."""
    return np.array([(r * n1) // nranks for r in range(nranks + 1)])


def local_h_from_c0(engine, slabs: Sequence, exchange, c0s: Sequence, c2s: Sequence):
    """The local part of H|psi> of a slab-decomposed wavefunction from C0
    alone: rho(r) by the slab transforms, V(r) from the gathered density,
    then C2 = -f (G^2/2 C0 + FFT(V psi)) by the slab transforms (eval_density,
    eval_pot, cal_vpot_ex, vpsi of one CG iteration)."""
    import torch
    rhos = [torch.zeros(engine.nr[2], engine.nr[1], s.nplane, dtype=torch.float64, device=c.device)
            for s, c in zip(slabs, c0s)]
    density(slabs, exchange, c0s, rhos)
    vs = potential_slabs(engine, slabs, exchange, rhos)
    apply_local_h(slabs, exchange, c0s, vs, c2s)
    return rhos, vs


def gram(slabs: Sequence, exchange, a_s: Sequence, b_s: Sequence, n: int):
    """The band-space Gram matrix 2 Re A^H B - Re a(0) Re b(0)^T (n x n,
    column-major) of a slab-decomposed pair of band arrays: each rank's share
    over its G vectors, then an all-reduce (the overlap of ortho_gs,
    wfn_initialize.f90:481-482, and Lambda of OVLAP_D are this product)."""
    import torch
    parts = []
    for s, a, b in zip(slabs, a_s, b_s):
        out = torch.empty(n * n, dtype=torch.float64, device=a.device)
        s.gram(a, b, n, out)
        parts.append(out)
    return [x.reshape(n, n).T for x in exchange.all_reduce(parts)]
