"""ctypes binding of the CPU restatement (liboracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline leg of bench.py.  The product (amdkiit_b200) never imports it.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
MAXSP = 4


class OrcSpecies(C.Structure):
    _fields_ = [("type", C.c_int), ("z", C.c_int), ("zv", C.c_double), ("mesh", C.c_int),
                ("rr", C.POINTER(C.c_double)), ("vr", C.POINTER(C.c_double)), ("rps", C.POINTER(C.c_double)),
                ("lmax", C.c_int), ("l_local", C.c_int), ("skip", C.c_int), ("tkb", C.c_int),
                ("rab", C.POINTER(C.c_double)), ("vloc", C.POINTER(C.c_double)), ("nbeta", C.c_int),
                ("beta_l", C.POINTER(C.c_int)), ("beta", C.POINTER(C.c_double)), ("dij", C.POINTER(C.c_double)),
                ("upf_lmax", C.c_int)]


class OrcInput(C.Structure):
    _fields_ = [("a_cell", C.c_double * 9), ("alat", C.c_double), ("symmetry", C.c_int), ("ecut", C.c_double),
                ("nsp", C.c_int), ("na", C.c_int * MAXSP), ("na_max", C.c_int), ("atco", C.POINTER(C.c_double)),
                ("xc", C.c_int), ("nstate", C.c_int), ("sp", OrcSpecies * MAXSP), ("multiplicity", C.c_int)]


def build():
    subprocess.check_call(["make", "-s", "-C", HERE])


def _lib():
    if not os.path.exists(LIB):
        build()
    lib = C.CDLL(LIB)
    P = C.c_void_p
    lib.orc_create.restype = P
    lib.orc_create.argtypes = [C.POINTER(OrcInput), C.c_int]
    lib.orc_destroy.argtypes = [P]
    lib.orc_get_int.restype = C.c_long
    lib.orc_get_int.argtypes = [P, C.c_char_p]
    lib.orc_get_dbl.restype = C.c_double
    lib.orc_get_dbl.argtypes = [P, C.c_char_p]
    lib.orc_get_ptr.restype = C.c_void_p
    lib.orc_get_ptr.argtypes = [P, C.c_char_p]
    for f in ("orc_eval_density", "orc_rhor2g", "orc_eval_pot", "orc_cal_vpot_ex", "orc_pp_energy",
              "orc_e_total", "orc_vpsi", "orc_fnonloc", "orc_forces", "orc_potfor", "orc_nlfor"):
        getattr(lib, f).argtypes = [P]
    lib.orc_e_sr.argtypes = [P, C.c_int]
    lib.orc_pcg.argtypes = [P, C.c_int]
    lib.orc_ortho.argtypes = [P]
    lib.orc_ortho.restype = C.c_int
    lib.orc_scf_iteration.argtypes = [P, C.c_int, C.c_double]
    lib.orc_scf_iteration.restype = C.c_int
    lib.orc_wfn_opt.argtypes = [P, C.c_int, C.c_double]
    lib.orc_wfn_opt.restype = C.c_int
    lib.orc_set_positions.argtypes = [P, C.POINTER(C.c_double)]
    lib.orc_set_wfn.argtypes = [P, C.POINTER(C.c_double)]
    lib.orc_fft.argtypes = [P, C.c_int, C.POINTER(C.c_double)]
    lib.orc_xc_point.argtypes = [C.c_int, C.c_double, C.c_double] + [C.POINTER(C.c_double)] * 3
    return lib


_L = None


def lib():
    global _L
    if _L is None:
        _L = _lib()
    return _L


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Oracle:
    """One reference system held by the CPU restatement."""

    def __init__(self, system, nthreads: int = 0):
        self.system = system
        self._keep = []
        inp = OrcInput()
        a = np.asfortranarray(system.a_cell)
        for k in range(9):
            inp.a_cell[k] = a.flatten(order="F")[k]
        inp.alat = system.alat
        inp.symmetry = system.symmetry
        inp.ecut = system.ecut
        inp.nsp = len(system.species)
        for i, n in enumerate(system.na):
            inp.na[i] = n
        inp.na_max = system.na_max
        atco = system.atco()
        self._keep.append(atco)
        inp.atco = _dp(atco)
        inp.xc = system.xc
        inp.nstate = system.nstate
        inp.multiplicity = getattr(system, "multiplicity", 0)
        for i, sp in enumerate(system.species):
            o = inp.sp[i]
            o.type = sp.kind
            o.z = sp.z
            o.zv = sp.zv
            o.mesh = sp.mesh
            for name in ("rr", "vr", "rps", "rab", "vloc", "beta", "dij"):
                v = getattr(sp, name)
                if v is not None:
                    v = np.ascontiguousarray(v, dtype=np.float64)
                    self._keep.append(v)
                    setattr(o, name, _dp(v))
            o.lmax, o.l_local, o.skip, o.tkb = sp.lmax, sp.l_local, sp.skip, int(sp.tkb)
            o.nbeta = sp.nbeta
            if sp.beta_l is not None and sp.nbeta:
                bl = np.ascontiguousarray(sp.beta_l, dtype=np.int32)
                self._keep.append(bl)
                o.beta_l = bl.ctypes.data_as(C.POINTER(C.c_int))
            o.upf_lmax = sp.upf_lmax
        self._inp = inp
        self.h = lib().orc_create(C.byref(inp), nthreads)

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().orc_destroy(self.h)
                self.h = None
        except Exception:
            pass

    # accessors ----------------------------------------------------------
    def i(self, k):
        return int(lib().orc_get_int(self.h, k.encode()))

    def d(self, k):
        return float(lib().orc_get_dbl(self.h, k.encode()))

    def arr(self, k, shape, dtype=np.float64):
        p = lib().orc_get_ptr(self.h, k.encode())
        n = int(np.prod(shape))
        ct = {np.float64: C.c_double, np.int32: C.c_int, np.complex128: C.c_double}[dtype]
        m = 2 if dtype == np.complex128 else 1
        buf = (ct * (n * m)).from_address(p)
        out = np.frombuffer(buf, dtype=dtype, count=n).reshape(shape).copy()
        return out

    @property
    def ngpw(self):
        return self.i("ngpw")

    @property
    def ngrho(self):
        return self.i("ngrho")

    @property
    def nstate(self):
        return self.i("nstate")

    def gvectors(self):
        ng = self.ngrho
        return dict(inyh=self.arr("inyh", (ng, 3), np.int32), hg=self.arr("hg", (ng,)),
                    hg_pert=self.arr("hg_pert", (ng,)), gvec=self.arr("gvec", (ng, 3)),
                    mapp=self.arr("mapp", (ng,), np.int32), mapm=self.arr("mapm", (ng,), np.int32),
                    msp=self.arr("msp", (self.i("nhrays"),), np.int32),
                    ngpw=self.ngpw, ngrho=ng, ngrays=self.i("ngrays"), nhrays=self.i("nhrays"),
                    nr=(self.i("nr1"), self.i("nr2"), self.i("nr3")))

    def c0(self):
        return self.arr("c0", (self.nstate, self.ngpw), np.complex128)

    def c2(self):
        return self.arr("c2", (self.nstate, self.ngpw), np.complex128)

    def set_wfn(self, c0):
        c = np.ascontiguousarray(c0, dtype=np.complex128)
        lib().orc_set_wfn(self.h, c.ctypes.data_as(C.POINTER(C.c_double)))

    def set_positions(self, atco):
        a = np.ascontiguousarray(atco, dtype=np.float64)
        lib().orc_set_positions(self.h, _dp(a))

    def real_grid(self, k):
        """A real-space array with the padding dropped: shape (nr3, nr2, nr1)."""
        l1, l2, l3 = self.i("nrl1"), self.i("nrl2"), self.i("nrl3")
        n1, n2, n3 = self.i("nr1"), self.i("nr2"), self.i("nr3")
        a = self.arr(k, (l3, l2, l1))
        return a[:n3, :n2, :n1].copy()

    def energies(self):
        return {k: self.d(k) for k in ("etotal", "eke", "estat", "eself", "esr", "eloc", "enl", "exc")}

    def force(self):
        s = self.system
        f = self.arr("force", (len(s.species), s.na_max, 3))
        return f

    # routines -------------------------------------------------------------
    def call(self, name, *args):
        return getattr(lib(), "orc_" + name)(self.h, *args)

    def ortho(self):
        return lib().orc_ortho(self.h)

    def scf_iteration(self, istep, gcut):
        return lib().orc_scf_iteration(self.h, istep, gcut)

    def wfn_opt(self, max_step, gcut):
        return lib().orc_wfn_opt(self.h, max_step, gcut)


def xc_point(xc, rho, sigma):
    e, v, vs = C.c_double(), C.c_double(), C.c_double()
    lib().orc_xc_point(xc, rho, sigma, C.byref(e), C.byref(v), C.byref(vs))
    return e.value, v.value, vs.value
