"""ctypes binding of libamdk (include/amdk.h) and the driver loops.

The driver loops restate AMDKIIT's outer loops, which stay outside the
C-ABI in the reference design: wfn_opt (do_opt.f90:51-138) and the
velocity-Verlet BOMD step (molecular_dynamics.f90:92-130).  Every
numerical operation runs in libamdk on the GPU; there is no CPU fallback:
constructing an Engine fails if the CUDA library cannot be loaded or the
device cannot be initialised.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

from .inputs import System

HERE = os.path.dirname(os.path.abspath(__file__))
LIBPATH = os.path.join(HERE, "libamdk.so")
MAXSP = 4

FP64, MIXED = 0, 1


class _Species(C.Structure):
    _fields_ = [("type", C.c_int), ("z", C.c_int), ("zv", C.c_double), ("mesh", C.c_int),
                ("rr", C.POINTER(C.c_double)), ("vr", C.POINTER(C.c_double)), ("rps", C.POINTER(C.c_double)),
                ("lmax", C.c_int), ("l_local", C.c_int), ("skip", C.c_int), ("tkb", C.c_int),
                ("rab", C.POINTER(C.c_double)), ("vloc", C.POINTER(C.c_double)), ("nbeta", C.c_int),
                ("beta_l", C.POINTER(C.c_int)), ("beta", C.POINTER(C.c_double)), ("dij", C.POINTER(C.c_double)),
                ("upf_lmax", C.c_int)]


class _System(C.Structure):
    _fields_ = [("a_cell", C.c_double * 9), ("alat", C.c_double), ("symmetry", C.c_int), ("ecut", C.c_double),
                ("nsp", C.c_int), ("na", C.c_int * MAXSP), ("na_max", C.c_int), ("atco", C.POINTER(C.c_double)),
                ("xc", C.c_int), ("nstate", C.c_int), ("sp", _Species * MAXSP), ("multiplicity", C.c_int)]


class _Options(C.Structure):
    _fields_ = [("device", C.c_int), ("precision", C.c_int), ("pair_batch", C.c_int), ("reserved", C.c_int * 8)]


class _Info(C.Structure):
    _fields_ = [("nr", C.c_int * 3), ("ngpw", C.c_int), ("ngrho", C.c_int), ("ngrays", C.c_int), ("nhrays", C.c_int),
                ("nstate", C.c_int), ("nat", C.c_int), ("nghmax", C.c_int), ("omega", C.c_double)]


class Energies(C.Structure):
    _fields_ = [(k, C.c_double) for k in ("etotal", "eke", "estat", "eself", "esr", "eloc", "enl", "exc", "eh")]

    def asdict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class AmdkError(RuntimeError):
    pass


_LIB = None


def load_library(path: str = LIBPATH):
    """Load libamdk.so (building it first when the sources are newer)."""
    global _LIB
    if _LIB is not None:
        return _LIB
    from . import build as _build
    if _build.needs_build():
        _build.build()
    lib = C.CDLL(path)
    P = C.c_void_p
    lib.amdk_last_error.restype = C.c_char_p
    lib.amdk_create.argtypes = [C.POINTER(_System), C.POINTER(_Options), C.POINTER(P)]
    lib.amdk_destroy.argtypes = [P]
    lib.amdk_info_get.argtypes = [P, C.POINTER(_Info)]
    lib.amdk_get_gvectors.argtypes = [P, P, P, P, P, P]
    lib.amdk_host_gvectors.argtypes = [C.POINTER(_System), C.POINTER(_Info), P, P, P, P, P]
    lib.amdk_set_positions.argtypes = [P, C.POINTER(C.c_double)]
    lib.amdk_set_precision.argtypes = [P, C.c_int]
    lib.amdk_wfn_extrapolate.argtypes = [P]
    lib.amdk_wfn_set_predictor.argtypes = [P, C.c_int, C.c_void_p]
    lib.amdk_wfn_history_clear.argtypes = [P]
    lib.amdk_set_wfn.argtypes = [P, C.POINTER(C.c_double)]
    lib.amdk_set_density.argtypes = [P, C.POINTER(C.c_double)]
    lib.amdk_get_wfn.argtypes = [P, C.POINTER(C.c_double)]
    for f in ("amdk_ortho", "amdk_density", "amdk_potential", "amdk_apply_h"):
        getattr(lib, f).argtypes = [P]
    lib.amdk_energy.argtypes = [P, C.POINTER(Energies)]
    lib.amdk_gradient.argtypes = [P, C.POINTER(C.c_double)]
    lib.amdk_pcg.argtypes = [P, C.c_int]
    lib.amdk_scf_iteration.argtypes = [P, C.c_int, C.c_double, C.POINTER(Energies), C.POINTER(C.c_double),
                                       C.POINTER(C.c_int)]
    lib.amdk_ionic_forces.argtypes = [P, C.POINTER(C.c_double)]
    lib.amdk_backward.argtypes = [P, P, P]
    lib.amdk_get_array.argtypes = [P, C.c_char_p, P, C.c_size_t]
    lib.amdk_fft_sphere.argtypes = [P, C.c_int, P, P]
    lib.amdk_last_iteration_ms.argtypes = [P, C.POINTER(C.c_double)]
    lib.amdk_profile.argtypes = [P, C.c_int]
    lib.amdk_launch_count.argtypes = [P, C.POINTER(C.c_long)]
    lib.amdk_profile_get.argtypes = [P, C.c_int, C.POINTER(C.c_long), C.POINTER(C.c_double), C.POINTER(C.c_double)]
    lib.amdk_ensemble_create.argtypes = [C.POINTER(P), C.c_int, C.POINTER(P)]
    lib.amdk_ensemble_iteration.argtypes = [P, C.POINTER(C.c_int), C.c_double, C.POINTER(Energies),
                                            C.POINTER(C.c_double), C.POINTER(C.c_int)]
    lib.amdk_ensemble_last_ms.argtypes = [P, C.POINTER(C.c_double)]
    lib.amdk_ensemble_destroy.argtypes = [P]
    _LIB = lib
    return lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def system_struct(system: System):
    """Fill the amdk_system struct; returns (struct, keep-alive list)."""
    keep = []
    s = _System()
    a = np.asarray(system.a_cell, dtype=np.float64).flatten(order="F")
    for k in range(9):
        s.a_cell[k] = a[k]
    s.alat = system.alat
    s.symmetry = system.symmetry
    s.ecut = system.ecut
    s.nsp = len(system.species)
    for i, n in enumerate(system.na):
        s.na[i] = n
    s.na_max = system.na_max
    atco = system.atco()
    keep.append(atco)
    s.atco = _dp(atco)
    s.xc = system.xc
    s.nstate = system.nstate
    s.multiplicity = getattr(system, "multiplicity", 0)
    for i, sp in enumerate(system.species):
        o = s.sp[i]
        o.type, o.z, o.zv, o.mesh = sp.kind, sp.z, sp.zv, sp.mesh
        for name in ("rr", "vr", "rps", "rab", "vloc", "beta", "dij"):
            v = getattr(sp, name)
            if v is not None:
                v = np.ascontiguousarray(v, dtype=np.float64)
                keep.append(v)
                setattr(o, name, _dp(v))
        o.lmax, o.l_local, o.skip, o.tkb = sp.lmax, sp.l_local, sp.skip, int(sp.tkb)
        o.nbeta = sp.nbeta
        if sp.beta_l is not None and sp.nbeta:
            bl = np.ascontiguousarray(sp.beta_l, dtype=np.int32)
            keep.append(bl)
            o.beta_l = bl.ctypes.data_as(C.POINTER(C.c_int))
        o.upf_lmax = sp.upf_lmax
    return s, keep


def _check(rc, what=""):
    if rc != 0:
        msg = load_library().amdk_last_error().decode()
        raise AmdkError(f"{what} failed ({rc}): {msg}")


def subspace_eigenvalues(c0: np.ndarray, hc: np.ndarray) -> np.ndarray:
    """Eigenvalues (Ha, ascending) of H in the span of the bands c0, given
    hc = H|c0> band by band.  Both are (nstate, ngpw) on the G half sphere
    with G = 0 first, so <a|b> = 2 Re sum_G a*(G) b(G) - a(0) b(0) (real
    bands at the Gamma point).  The reference prints no eigenvalues; this
    forms the nstate x nstate subspace Hamiltonian and overlap and solves
    H x = e S x (S = 1 for orthonormal bands)."""
    import scipy.linalg

    def gram(a, b):
        return 2.0 * np.real(np.conj(a) @ b.T) - np.outer(a[:, 0].real, b[:, 0].real)

    h = gram(c0, hc)
    return scipy.linalg.eigh(0.5 * (h + h.T), gram(c0, c0), eigvals_only=True)


def host_gvectors(system: System) -> dict:
    """The G half-sphere and ray maps from the library's host setup (no GPU)."""
    lib = load_library()
    s, keep = system_struct(system)
    info = _Info()
    _check(lib.amdk_host_gvectors(C.byref(s), C.byref(info), None, None, None, None, None), "amdk_host_gvectors")
    ng = info.ngrho
    inyh = np.zeros((ng, 3), np.int32)
    hg = np.zeros(ng)
    gvec = np.zeros((ng, 3))
    mp = np.zeros(ng, np.int32)
    mm = np.zeros(ng, np.int32)
    _check(lib.amdk_host_gvectors(C.byref(s), C.byref(info), inyh.ctypes.data, hg.ctypes.data, gvec.ctypes.data,
                                  mp.ctypes.data, mm.ctypes.data), "amdk_host_gvectors")
    return dict(inyh=inyh, hg=hg, gvec=gvec, mapp=mp, mapm=mm, ngpw=info.ngpw, ngrho=ng, ngrays=info.ngrays,
                nhrays=info.nhrays, nr=tuple(info.nr), omega=info.omega)


# mixed-precision CG hands over to FP64 at this GEMAX: below it the FP32 pair
# transforms and the 28-bit Gram products limit the gradient.  It also hands
# over after MIXED_STALL iterations without a new GEMAX minimum, but only once
# GEMAX has come within MIXED_STALL_ZONE x MIXED_GCUT: higher up a plateau is
# the CG's own (the reference's fixed-step PCG plateaus for hundreds of
# iterations on bulk Si in FP64 too), not the FP32 noise floor
MIXED_GCUT = 1e-6
MIXED_STALL = 40
MIXED_STALL_ZONE = 10.0


class Engine:
    """One system resident on one GPU."""

    def __init__(self, system: System, precision: int = FP64, pair_batch: int = 0, device: int = 0,
                 wait_limit: int = 0, fp64_wait_limit: int = 0):
        """wait_limit / fp64_wait_limit != 0 (tests of the failure path
        only): the pipeline waits of the int8 / FP64 tensor-core kernels give
        up after max(limit, 0) polls (amdk_options.reserved[0] / [1])."""
        self.lib = load_library()
        self.system = system
        s, self._keep = system_struct(system)
        opt = _Options()
        opt.device, opt.precision, opt.pair_batch = device, precision, pair_batch
        opt.reserved[0] = wait_limit
        opt.reserved[1] = fp64_wait_limit
        h = C.c_void_p()
        _check(self.lib.amdk_create(C.byref(s), C.byref(opt), C.byref(h)), "amdk_create")
        self.h = h
        info = _Info()
        _check(self.lib.amdk_info_get(self.h, C.byref(info)), "amdk_info_get")
        self.info = info
        self.ngpw, self.ngrho, self.nstate = info.ngpw, info.ngrho, info.nstate
        self.nr = tuple(info.nr)
        self.precision = precision      # precision the engine was created with
        self.pair_precision = precision  # precision of the band-pair FFTs now

    def set_predictor(self, npoints: int = 2, coef=None):
        """Points (C0(t) included) and weights of the BOMD predictor; coef
        None selects the always-stable predictor weights (aspc_coefficients)."""
        w = None if coef is None else np.ascontiguousarray(coef, dtype=np.float64)
        if w is not None and w.shape != (npoints,):
            raise ValueError("coef must have npoints entries")
        _check(self.lib.amdk_wfn_set_predictor(self.h, int(npoints), None if w is None else w.ctypes.data),
               "amdk_wfn_set_predictor")

    def extrapolate(self):
        """BOMD predictor: C0 <- sum_j w_j C0(t-j dt) [C0(t-j dt)^T C0(t)] over
        the stored steps (stores C0(t)); orthonormalise afterwards."""
        _check(self.lib.amdk_wfn_extrapolate(self.h), "amdk_wfn_extrapolate")

    def clear_history(self):
        _check(self.lib.amdk_wfn_history_clear(self.h), "amdk_wfn_history_clear")

    def set_precision(self, precision: int):
        """Precision of the band-pair transforms from the next call on."""
        _check(self.lib.amdk_set_precision(self.h, precision), "amdk_set_precision")
        self.pair_precision = precision

    def close(self):
        if getattr(self, "h", None):
            self.lib.amdk_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # --------------------------------------------------------------- data
    def gvectors(self) -> dict:
        ng = self.ngrho
        inyh = np.zeros((ng, 3), np.int32)
        hg = np.zeros(ng)
        gvec = np.zeros((ng, 3))
        mp = np.zeros(ng, np.int32)
        mm = np.zeros(ng, np.int32)
        _check(self.lib.amdk_get_gvectors(self.h, inyh.ctypes.data, hg.ctypes.data, gvec.ctypes.data, mp.ctypes.data,
                                          mm.ctypes.data))
        return dict(inyh=inyh, hg=hg, gvec=gvec, mapp=mp, mapm=mm)

    def set_wfn(self, c0: np.ndarray):
        c = np.ascontiguousarray(c0, dtype=np.complex128)
        assert c.shape == (self.nstate, self.ngpw)
        _check(self.lib.amdk_set_wfn(self.h, c.ctypes.data_as(C.POINTER(C.c_double))), "amdk_set_wfn")

    def set_density(self, rho: np.ndarray):
        """rho(r) as (nr3, nr2, nr1) float64 in place of the density of C0
        (rhor2g applied): the gathered density of a slab-decomposed system."""
        r = np.ascontiguousarray(rho, dtype=np.float64)
        n1, n2, n3 = self.nr
        if r.size != n1 * n2 * n3:
            raise ValueError("set_density: rho must have nr3 * nr2 * nr1 values")
        _check(self.lib.amdk_set_density(self.h, _dp(r)), "amdk_set_density")

    def get_wfn(self, out: np.ndarray | None = None) -> np.ndarray:
        """C0 as (nstate, ngpw) complex128; with `out` (C-contiguous, that
        shape and dtype, e.g. a pinned host buffer) the copy lands there."""
        c = out
        if c is None:
            c = np.empty((self.nstate, self.ngpw), np.complex128)
        elif c.shape != (self.nstate, self.ngpw) or c.dtype != np.complex128 or not c.flags.c_contiguous:
            raise ValueError("get_wfn: out must be C-contiguous complex128 of shape (nstate, ngpw)")
        _check(self.lib.amdk_get_wfn(self.h, c.ctypes.data_as(C.POINTER(C.c_double))), "amdk_get_wfn")
        return c

    def set_positions(self, atco: np.ndarray):
        a = np.ascontiguousarray(atco, dtype=np.float64)
        _check(self.lib.amdk_set_positions(self.h, _dp(a)), "amdk_set_positions")

    def get(self, name: str) -> np.ndarray:
        n1, n2, n3 = self.nr
        nsp = len(self.system.species)
        nproj = sum(n * 0 for n in self.system.na)
        shapes = {
            "rho": ((n3, n2, n1), np.float64), "v_pot": ((n3, n2, n1), np.float64),
            "rho2": ((n3, n2, n1), np.float64), "v_pot2": ((n3, n2, n1), np.float64),
            "rho_g": ((self.ngrho,), np.complex128), "c2": ((self.nstate, self.ngpw), np.complex128),
            "c0": ((self.nstate, self.ngpw), np.complex128),
            "vps": ((nsp, self.ngrho), np.float64), "rhos": ((nsp, self.ngrho), np.float64),
            "twnl": ((nsp, self.info.nghmax, self.ngpw), np.float64),
            "eigrxvps": ((self.ngrho,), np.complex128), "eigrxrhos": ((self.ngrho,), np.complex128),
            "vpp": ((self.ngpw,), np.float64),
            "force": ((nsp, self.system.na_max, 3), np.float64),
            "overlap": ((self.nstate, self.nstate), np.float64),
        }
        del nproj
        shape, dt = shapes[name]
        a = np.zeros(shape, dt)
        _check(self.lib.amdk_get_array(self.h, name.encode(), a.ctypes.data, a.nbytes), f"amdk_get_array({name})")
        return a

    # ----------------------------------------------------------- routines
    def ortho(self):
        _check(self.lib.amdk_ortho(self.h), "amdk_ortho")

    def density(self):
        _check(self.lib.amdk_density(self.h), "amdk_density")

    def potential(self):
        _check(self.lib.amdk_potential(self.h), "amdk_potential")

    def energy(self) -> dict:
        e = Energies()
        _check(self.lib.amdk_energy(self.h, C.byref(e)), "amdk_energy")
        return e.asdict()

    def apply_h(self):
        _check(self.lib.amdk_apply_h(self.h), "amdk_apply_h")

    def eigenvalues(self) -> np.ndarray:
        """Eigenvalues (Ha) of the Hamiltonian in the occupied subspace at the
        current wavefunction.  Density, potential, projections and H|psi> run
        on the GPU; C2 = -f_i H|psi_i> with f_i = 2 (the pair unpack of
        wfn_initialize.f90:342-361 scales by f_i/2 and the pair transform
        doubles V psi), so H|psi_i> = -C2_i / 2.  The nstate x nstate
        matrix is formed and diagonalised on the host.  Open shell: f_i = 1,
        and each spin's block separately (spin 1 first).  Overwrites C2."""
        self.density()
        self.potential()
        self.energy()
        self.apply_h()
        c = self.get_wfn()
        mult = getattr(self.system, "multiplicity", 0)
        if mult > 0:
            hc = -self.get("c2")
            nu = (self.nstate - (mult - 1)) // 2
            return np.concatenate([subspace_eigenvalues(c[:nu], hc[:nu]), subspace_eigenvalues(c[nu:], hc[nu:])])
        return subspace_eigenvalues(c, -0.5 * self.get("c2"))

    def gradient(self) -> float:
        g = C.c_double()
        _check(self.lib.amdk_gradient(self.h, C.byref(g)), "amdk_gradient")
        return g.value

    def pcg(self, istep: int):
        _check(self.lib.amdk_pcg(self.h, istep), "amdk_pcg")

    def scf_iteration(self, istep: int, gcut: float):
        e = Energies()
        g = C.c_double()
        conv = C.c_int()
        _check(self.lib.amdk_scf_iteration(self.h, istep, gcut, C.byref(e), C.byref(g), C.byref(conv)),
               "amdk_scf_iteration")
        return e.asdict(), g.value, bool(conv.value)

    def last_iteration_ms(self) -> float:
        m = C.c_double()
        self.lib.amdk_last_iteration_ms(self.h, C.byref(m))
        return m.value

    KERNELS = {0: "z_vpsi", 1: "z_density", 2: "y_pass", 3: "x_fwd"}

    def launch_count(self) -> int:
        n = C.c_long()
        _check(self.lib.amdk_launch_count(self.h, C.byref(n)), "amdk_launch_count")
        return n.value

    def profile(self, enable: bool):
        _check(self.lib.amdk_profile(self.h, int(enable)), "amdk_profile")

    def profile_get(self, kind: int):
        n, ms, b = C.c_long(), C.c_double(), C.c_double()
        _check(self.lib.amdk_profile_get(self.h, kind, C.byref(n), C.byref(ms), C.byref(b)), "amdk_profile_get")
        return n.value, ms.value, b.value

    def ionic_forces(self) -> np.ndarray:
        s = self.system
        f = np.zeros((len(s.species), s.na_max, 3))
        _check(self.lib.amdk_ionic_forces(self.h, _dp(f)), "amdk_ionic_forces")
        return f

    def backward(self, want_psi: bool = False):
        """dE/dR (same layout as the forces), and f (H c) when want_psi."""
        s = self.system
        g = np.zeros((len(s.species), s.na_max, 3))
        p = np.zeros((self.nstate, self.ngpw), np.complex128) if want_psi else None
        _check(self.lib.amdk_backward(self.h, g.ctypes.data, p.ctypes.data if want_psi else None), "amdk_backward")
        return (g, p) if want_psi else g

    def fft_sphere(self, sign: int, coef: Optional[np.ndarray] = None, grid: Optional[np.ndarray] = None):
        n1, n2, n3 = self.nr
        if coef is None:
            coef = np.zeros(self.ngrho, np.complex128)
        if grid is None:
            grid = np.zeros((n3, n2, n1), np.complex128)
        coef = np.ascontiguousarray(coef, dtype=np.complex128)
        grid = np.ascontiguousarray(grid, dtype=np.complex128)
        _check(self.lib.amdk_fft_sphere(self.h, sign, coef.ctypes.data, grid.ctypes.data), "amdk_fft_sphere")
        return coef, grid

    # ------------------------------------------------------------ drivers
    def wfn_opt(self, max_step: int = 800, gcut: float = 1e-7, callback=None, refine: bool = True):
        """do_opt.f90:51-138: CG iterations until GEMAX < gcut.

        On a mixed-precision engine with refine=True the iterations run with
        FP64 band-pair transforms (and FP64 Gram products) from the first one
        with GEMAX < max(gcut, MIXED_GCUT), or once GEMAX, within
        MIXED_STALL_ZONE of that threshold, has not reached a new minimum for
        MIXED_STALL iterations, until GEMAX < gcut holds there: the returned energy, gradient and forces are those of the FP64
        path at a converged wavefunction (the CG history carries on; only the
        precision changes).  The mixed path's gradient carries FP32-level
        errors, so a tighter gcut than MIXED_GCUT is reached in FP64."""
        e, g = None, None
        refining = False
        best, since = float("inf"), 0
        switch = max(gcut, MIXED_GCUT)
        try:
            for i in range(1, max_step + 1):
                e, g, conv = self.scf_iteration(i, gcut)
                if callback:
                    callback(i, e, g)
                if refine and self.pair_precision == MIXED and not refining:
                    if g < best:
                        best, since = g, 0
                    else:
                        since += 1
                    if g < switch or (best < MIXED_STALL_ZONE * switch and since >= MIXED_STALL):
                        refining = True
                        self.set_precision(FP64)
                        continue
                if conv:
                    return i, e, g
            return max_step, e, g
        finally:
            if refining:
                self.set_precision(self.precision)


class Ensemble:
    """Several engines (independent systems on one GPU) iterated together
    through amdk_ensemble_iteration: each CG segment of all members is one
    CUDA graph launch once every member has run its first iteration."""

    def __init__(self, engines):
        self.lib = load_library()
        self.engines = list(engines)
        n = len(self.engines)
        arr = (C.c_void_p * n)(*[e.h.value for e in self.engines])
        h = C.c_void_p()
        _check(self.lib.amdk_ensemble_create(arr, n, C.byref(h)), "amdk_ensemble_create")
        self.h = h

    def iteration(self, isteps, gcut: float):
        n = len(self.engines)
        st = (C.c_int * n)(*[int(i) for i in isteps])
        en = (Energies * n)()
        gm = (C.c_double * n)()
        cv = (C.c_int * n)()
        _check(self.lib.amdk_ensemble_iteration(self.h, st, gcut, en, gm, cv), "amdk_ensemble_iteration")
        return [x.asdict() for x in en], np.array(gm[:]), np.array(cv[:], dtype=bool)

    def last_ms(self) -> float:
        m = C.c_double()
        self.lib.amdk_ensemble_last_ms(self.h, C.byref(m))
        return m.value

    def close(self):
        if getattr(self, "h", None):
            self.lib.amdk_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
