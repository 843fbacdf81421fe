"""Geometry optimisation by limited-memory BFGS on top of the GPU engine.

Restates the reference's driver `geom_opt_lbfgs` (do_opt.f90:197-266): at
every geometry a full wavefunction optimisation, the ionic forces of the
converged state, and one reverse-communication call of `LBFGS` (lbfgs.f),
the Liu-Nocedal limited-memory BFGS (Math. Prog. 45, 503 (1989)) with the
More-Thuente line search (ACM TOMS 20, 286 (1994)).  Settings of the
reference's call: M = 5 corrections, XTOL = 1e-16, FTOL = 1e-4, GTOL = 0.9,
MAXFEV = 20, STPMIN = 1e-20, STPMAX = 1e20, no user diagonal, and the
convergence test ||g|| <= EPS with EPS the geometry gradient cutoff
(lbfgs.f:397, absolute, not relative to ||x||).  Units: bohr, Hartree.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import Callable, List, Tuple

import numpy as np

P5, P66, XTRAPF = 0.5, 0.66, 4.0


def _cstep(stx, fx, dx, sty, fy, dy, stp, fp, dp, brackt, stpmin, stpmax):
    """One safeguarded step of the More-Thuente interval update (MCSTEP).

    (stx, fx, dx): best step so far, its value and derivative; (sty, fy, dy):
    the other end of the interval; (stp, fp, dp): the trial step.  Returns
    the updated interval, the next trial step, brackt, and info (0: bad
    input, 1-4: which case was taken)."""
    if (brackt and (stp <= min(stx, sty) or stp >= max(stx, sty))) or dx * (stp - stx) >= 0.0 or stpmax < stpmin:
        return stx, fx, dx, sty, fy, dy, stp, brackt, 0
    sgnd = dp * (dx / abs(dx))
    if fp > fx:
        # case 1: higher value; the minimum is bracketed.  Cubic or the mean
        # of the cubic and quadratic steps, whichever is closer to stx.
        info, bound = 1, True
        theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * np.sqrt((theta / s) ** 2 - (dx / s) * (dp / s))
        if stp < stx:
            gamma = -gamma
        p = (gamma - dx) + theta
        q = ((gamma - dx) + gamma) + dp
        r = p / q
        stpc = stx + r * (stp - stx)
        stpq = stx + ((dx / ((fx - fp) / (stp - stx) + dx)) / 2.0) * (stp - stx)
        stpf = stpc if abs(stpc - stx) < abs(stpq - stx) else stpc + (stpq - stpc) / 2.0
        brackt = True
    elif sgnd < 0.0:
        # case 2: lower value, derivatives of opposite sign; bracketed.
        info, bound = 2, False
        theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * np.sqrt((theta / s) ** 2 - (dx / s) * (dp / s))
        if stp > stx:
            gamma = -gamma
        p = (gamma - dp) + theta
        q = ((gamma - dp) + gamma) + dx
        r = p / q
        stpc = stp + r * (stx - stp)
        stpq = stp + (dp / (dp - dx)) * (stx - stp)
        stpf = stpc if abs(stpc - stp) > abs(stpq - stp) else stpq
        brackt = True
    elif abs(dp) < abs(dx):
        # case 3: lower value, same sign, derivative magnitude decreases.
        info, bound = 3, True
        theta = 3.0 * (fx - fp) / (stp - stx) + dx + dp
        s = max(abs(theta), abs(dx), abs(dp))
        gamma = s * np.sqrt(max(0.0, (theta / s) ** 2 - (dx / s) * (dp / s)))
        if stp > stx:
            gamma = -gamma
        p = (gamma - dp) + theta
        q = (gamma + (dx - dp)) + gamma
        r = p / q
        if r < 0.0 and gamma != 0.0:
            stpc = stp + r * (stx - stp)
        elif stp > stx:
            stpc = stpmax
        else:
            stpc = stpmin
        stpq = stp + (dp / (dp - dx)) * (stx - stp)
        if brackt:
            stpf = stpc if abs(stp - stpc) < abs(stp - stpq) else stpq
        else:
            stpf = stpc if abs(stp - stpc) > abs(stp - stpq) else stpq
    else:
        # case 4: lower value, same sign, derivative does not decrease.
        info, bound = 4, False
        if brackt:
            theta = 3.0 * (fp - fy) / (sty - stp) + dy + dp
            s = max(abs(theta), abs(dy), abs(dp))
            gamma = s * np.sqrt((theta / s) ** 2 - (dy / s) * (dp / s))
            if stp > sty:
                gamma = -gamma
            p = (gamma - dp) + theta
            q = ((gamma - dp) + gamma) + dy
            r = p / q
            stpf = stp + r * (sty - stp)
        elif stp > stx:
            stpf = stpmax
        else:
            stpf = stpmin
    # update the interval
    if fp > fx:
        sty, fy, dy = stp, fp, dp
    else:
        if sgnd < 0.0:
            sty, fy, dy = stx, fx, dx
        stx, fx, dx = stp, fp, dp
    stpf = min(stpmax, stpf)
    stpf = max(stpmin, stpf)
    stp = stpf
    if brackt and bound:
        if sty > stx:
            stp = min(stx + 0.66 * (sty - stx), stp)
        else:
            stp = max(stx + 0.66 * (sty - stx), stp)
    return stx, fx, dx, sty, fy, dy, stp, brackt, info


@dataclass
class LineSearchResult:
    x: np.ndarray
    f: float
    g: np.ndarray
    stp: float
    info: int
    nfev: int


def line_search(fun: Callable[[np.ndarray], Tuple[float, np.ndarray]], x: np.ndarray, f: float, g: np.ndarray,
                s: np.ndarray, stp: float, ftol: float = 1e-4, gtol: float = 0.9, xtol: float = 1e-16,
                stpmin: float = 1e-20, stpmax: float = 1e20, maxfev: int = 20) -> LineSearchResult:
    """MCSRCH: a step along s satisfying the sufficient-decrease and
    curvature conditions.  info 1 = converged, 2-6 = stopped (see lbfgs.f),
    0/-1 = bad input or not a descent direction."""
    dginit = float(g @ s)
    if stp <= 0.0 or dginit >= 0.0:
        return LineSearchResult(x, f, g, stp, 0 if stp <= 0.0 else -1, 0)
    brackt, stage1, infoc, nfev = False, True, 1, 0
    finit, dgtest = f, ftol * dginit
    width = stpmax - stpmin
    width1 = width / P5
    wa = x.copy()
    stx, fx, dgx = 0.0, finit, dginit
    sty, fy, dgy = 0.0, finit, dginit
    while True:
        if brackt:
            stmin, stmax = min(stx, sty), max(stx, sty)
        else:
            stmin, stmax = stx, stp + XTRAPF * (stp - stx)
        stp = min(max(stp, stpmin), stpmax)
        if (brackt and (stp <= stmin or stp >= stmax)) or nfev >= maxfev - 1 or infoc == 0 or \
                (brackt and stmax - stmin <= xtol * stmax):
            stp = stx
        xn = wa + stp * s
        f, g = fun(xn)
        nfev += 1
        dg = float(g @ s)
        ftest1 = finit + stp * dgtest
        info = 0
        if (brackt and (stp <= stmin or stp >= stmax)) or infoc == 0:
            info = 6
        if stp == stpmax and f <= ftest1 and dg <= dgtest:
            info = 5
        if stp == stpmin and (f > ftest1 or dg >= dgtest):
            info = 4
        if nfev >= maxfev:
            info = 3
        if brackt and stmax - stmin <= xtol * stmax:
            info = 2
        if f <= ftest1 and abs(dg) <= gtol * (-dginit):
            info = 1
        if info != 0:
            return LineSearchResult(xn, f, g, stp, info, nfev)
        if stage1 and f <= ftest1 and dg >= min(ftol, gtol) * dginit:
            stage1 = False
        if stage1 and fx >= f > ftest1:
            # modified function (More-Thuente's psi) while in stage 1
            fm, fxm, fym = f - stp * dgtest, fx - stx * dgtest, fy - sty * dgtest
            dgm, dgxm, dgym = dg - dgtest, dgx - dgtest, dgy - dgtest
            stx, fxm, dgxm, sty, fym, dgym, stp, brackt, infoc = _cstep(
                stx, fxm, dgxm, sty, fym, dgym, stp, fm, dgm, brackt, stmin, stmax)
            fx, fy = fxm + stx * dgtest, fym + sty * dgtest
            dgx, dgy = dgxm + dgtest, dgym + dgtest
        else:
            stx, fx, dgx, sty, fy, dgy, stp, brackt, infoc = _cstep(
                stx, fx, dgx, sty, fy, dgy, stp, f, dg, brackt, stmin, stmax)
        if brackt:
            if abs(sty - stx) >= P66 * width1:
                stp = stx + P5 * (sty - stx)
            width1 = width
            width = abs(sty - stx)


@dataclass
class LBFGSResult:
    x: np.ndarray
    f: float
    g: np.ndarray
    iterations: int
    evaluations: int
    converged: bool
    info: int
    history: List[Tuple[float, float]] = field(default_factory=list)  # (f, ||g||) per iteration


def lbfgs(fun: Callable[[np.ndarray], Tuple[float, np.ndarray]], x0: np.ndarray, eps: float, m: int = 5,
          max_iter: int = 100, max_eval: int = 10**9, xtol: float = 1e-16) -> LBFGSResult:
    """LBFGS (lbfgs.f): two-loop recursion with the scaling ys/yy of the
    last pair, first step 1/||g||, unit steps afterwards, stop when
    ||g|| <= eps (absolute, as the reference)."""
    x = np.asarray(x0, dtype=np.float64).copy()
    f, g = fun(x)
    nfev = 1
    hist = [(f, float(np.linalg.norm(g)))]
    if hist[0][1] <= eps:
        return LBFGSResult(x, f, g, 0, nfev, True, 0, hist)
    S: List[np.ndarray] = []
    Y: List[np.ndarray] = []
    it = 0
    while it < max_iter and nfev < max_eval:
        it += 1
        q = -g.copy()
        if S:
            rho = [1.0 / float(y @ s) for s, y in zip(S, Y)]
            alpha = [0.0] * len(S)
            for k in range(len(S) - 1, -1, -1):
                alpha[k] = rho[k] * float(S[k] @ q)
                q -= alpha[k] * Y[k]
            q *= float(Y[-1] @ S[-1]) / float(Y[-1] @ Y[-1])
            for k in range(len(S)):
                beta = rho[k] * float(Y[k] @ q)
                q += S[k] * (alpha[k] - beta)
        stp = 1.0 / float(np.linalg.norm(g)) if it == 1 else 1.0
        r = line_search(fun, x, f, g, q, stp, xtol=xtol, maxfev=min(20, max_eval - nfev))
        nfev += r.nfev
        if r.info != 1:
            return LBFGSResult(r.x, r.f, r.g, it, nfev, False, r.info, hist)
        S.append(r.stp * q)
        Y.append(r.g - g)
        if len(S) > m:
            S.pop(0)
            Y.pop(0)
        x, f, g = r.x, r.f, r.g
        gn = float(np.linalg.norm(g))
        hist.append((f, gn))
        if gn <= eps:
            return LBFGSResult(x, f, g, it, nfev, True, 1, hist)
    return LBFGSResult(x, f, g, it, nfev, False, 0, hist)


class GeometryOptimizer:
    """geom_opt_lbfgs: energy and forces of the converged wavefunction at each
    geometry (wfn_opt from the previous wavefunction after exp_igrxfactor +
    ortho_gs), minimised with LBFGS over all atomic coordinates."""

    def __init__(self, engine, gcut_wfn: float = 1e-6, gcut_geo: float = 1e-4, max_scf: int = 800,
                 max_step: int = 100):
        self.e = engine
        self.system = engine.system
        self.gcut_wfn = gcut_wfn
        self.gcut_geo = gcut_geo
        self.max_scf = max_scf
        self.max_step = max_step
        s = self.system
        self.mask = np.zeros((len(s.species), s.na_max), dtype=bool)
        for i in range(len(s.species)):
            self.mask[i, : s.na[i]] = True
        self.shape = (len(s.species), s.na_max, 3)
        self.evaluations = []  # (energy, max |F|, SCF iterations) per geometry

    def _x_to_atco(self, x):
        a = np.zeros(self.shape)
        a[self.mask] = x.reshape(-1, 3)
        return a

    def energy_gradient(self, x):
        self.e.set_positions(self._x_to_atco(x))
        self.e.ortho()
        n, en, gm = self.e.wfn_opt(self.max_scf, self.gcut_wfn)
        force = self.e.get("force") if n > 1 else self.e.ionic_forces()
        self.evaluations.append((en["etotal"], float(np.abs(force[self.mask]).max()), n))
        return en["etotal"], -force[self.mask].reshape(-1)

    def run(self):
        x0 = self.system.atco()[self.mask].reshape(-1)
        self.e.ortho()
        res = lbfgs(self.energy_gradient, x0, self.gcut_geo, max_iter=self.max_step)
        return res, self._x_to_atco(res.x)
