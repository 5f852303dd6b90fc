"""Quasi-Newton fixed-point solve of one density on the device pipeline.

Restates QuasiNewton (cmmdft/solver.py:701-1053) and its helpers
(:1054-1212): hybrid Picard steps for the first iterations and after a
failure, then limited-memory quasi-Newton steps on the grand potential --
L-BFGS two-loop, 'good' Broyden or Hager-Zhang CG-descent directions from
the histories of rho and dOmega/drho, projected onto rho >= 0, capped by a
trust radius and accepted through a backtracking, quadratic or fixed line
search.  Every C1 and Omega is one pass of the functional pipeline
(cmm_fmt_c1); the vector algebra over the histories (dot products, axpys of
whole fields) runs as torch reductions on the device.  The control flow,
constants and failure paths follow the reference step for step, its quirks
included: the projected-steepest-descent retry re-tests the first
direction's slope, and a Broyden direction from an empty history fails as
it does there (TypeError).
"""
import numpy as np
import scipy.optimize as opt
import torch

from . import _lib as L
from . import engine as E
from .units import kjmol

__all__ = ['QuasiNewtonSolve', 'SwitchToPicard']


class SwitchToPicard(Exception):
    """A quasi-Newton step gave up: take a hybrid Picard step (SwitchToPicardError)."""


def _dot(a, b):
    return float(torch.dot(a, b))


def _norm(a):
    return float(torch.linalg.vector_norm(a))


def _gamma_last_pair(dX, dG, default=1.0):
    """H0 scale s.y / y.y of the newest pair (_gamma_from_last_pair, :1087-1097)."""
    for i in range(len(dX) - 1, -1, -1):
        sy = _dot(dX[i], dG[i])
        if sy > 1e-12:
            yy = _dot(dG[i], dG[i])
            return sy / yy if yy > 0 else default
        return default
    return None


def _lbfgs(g, dX, dG, h0, eps=1e-12):
    """Two-loop recursion, -H g (lbfgs_direction, :1099-1127)."""
    q = g.clone()
    kept = []
    mk = len(dX)
    # s.y, |s| and |y| of every pair do not depend on q: one read-back for
    # all of them (the same reductions, so the same values)
    sc = torch.stack([v for s, y in zip(dX, dG) for v in (torch.dot(s, y), torch.linalg.vector_norm(s),
                                                          torch.linalg.vector_norm(y))]).cpu().tolist() if mk else []
    for i in range(mk - 1, -1, -1):
        s, y = dX[i], dG[i]
        sy, ns, ny = sc[3 * i:3 * i + 3]
        if sy <= eps * ns * ny:
            continue
        r = 1.0 / sy
        a = r * torch.dot(s, q)   # a device scalar: the same double products, no read-back
        q -= a * y
        kept.append((i, a, r))
    if (mk - len(kept)) / mk > 0.5:
        raise SwitchToPicard('Too many skipped pairs')
    z = h0 * q
    for i, a, r in reversed(kept):
        b = r * torch.dot(dG[i], z)
        z += dX[i] * (a - b)
    return -z


def _lbroyden(g, dX, dG, h0, eps=1e-12):
    """Inverse 'good' Broyden, -H g (lbroyden_direction, :1129-1144)."""
    p = -h0 * g
    for s, y in zip(dX, dG):
        ys = _dot(y, s)
        if abs(ys) <= eps * _norm(s) * _norm(y):
            continue
        p += (s - h0 * y) * (_dot(y, p) / ys)
    return p


def _cg_descent(g, g_prev, d_prev, eps=1e-12, beta_floor=-0.1):
    """Hager-Zhang direction; (direction, take_picard) (cgdescent_direction, :1146-1205)."""
    p_sd = -g
    if g_prev is None or d_prev is None:
        return p_sd, False
    y = g - g_prev
    s = d_prev
    ys = _dot(y, s)
    if abs(ys) <= eps:
        return p_sd, True
    beta = (_dot(y, g) - 2.0 * _dot(y, y) * _dot(s, g) / ys) / ys
    p = p_sd + max(beta, beta_floor) * s
    if _dot(p, g) >= 0.0:
        return p_sd, True
    return p, False


def _cone_project(x, d, lower):
    """Zero the components that would push x below its bound (cone_project_direction, :1054-1063)."""
    return torch.where((x <= lower + lower) & (d < 0), torch.zeros_like(d), d)


def _cap(p, radius):
    n = _norm(p)
    return p * (radius / max(n, 1e-16)) if n > radius else p


class QuasiNewtonSolve(object):
    """One density, one chemical potential: QuasiNewton.solve on the GPU.

    fn: a device Functional (engine.Functional); other arguments as the
    reference's QuasiNewton and Solver (threshold/criterion/a_tol/r_tol).
    """

    def __init__(self, fn, nsteps=500, m=10, method='bfgs', hybrid=True, delta=0.5, alpha_init=0.05, c1=1e-4,
                 c2=0.9, line_search='backtracking', n_line_search=10, trust_radius=1, threshold=1e-6,
                 criterion='riue', a_tol=1e-6, r_tol=1e-4, alpha_mix=0.1):
        self.fn, self.plan = fn, fn.plan
        self.nsteps, self.m = int(nsteps), int(m)
        self.method = method.lower()
        assert self.method in ('bfgs', 'broyden', 'cg'), self.method
        assert line_search in ('backtracking', 'quadratic', 'none'), line_search
        self.line_search = line_search
        self.hybrid, self.delta, self.alpha_init = hybrid, delta, alpha_init
        self.c1, self.c2, self.n_line_search = c1, c2, n_line_search
        self.trust_radius = trust_radius
        crit = criterion if isinstance(criterion, (list, tuple)) else [criterion]
        thr = threshold if isinstance(threshold, (list, tuple)) else [threshold] * len(crit)
        if not isinstance(criterion, (list, tuple)) and criterion.lower() == 'der':
            thr = [1]
        self.criteria = [c.lower() for c in crit]
        self.thresholds = [float(t) for t in thr]
        self.a_tol, self.r_tol = a_tol, r_tol
        self.alpha_mix = alpha_mix
        self.thresh = 1 * kjmol
        self.lower = 1e-12
        self.picard_first, self.qn_limit = 5, 20
        self.buf = E.Buffers(self.plan, 1, nwork=fn.nwork)
        self.npts = self.plan.npts
        self.dV = self.plan.dr
        self.V = fn.V.reshape(-1)

    # ---- functional -------------------------------------------------------
    def _pipeline(self, rho, want):
        buf = self.buf
        if want & 4:
            buf.part[:, L.STAT_N3MAX, :] = -np.inf
        spec = self.plan.rfft_yz(rho.reshape((1,) + self.plan.npoints))
        chat = self.plan.new_spec(1) if want & 1 else None
        self.fn.c1(buf, spec, chat, want=want)
        st = None
        if want & 6:   # the sums stay on the device; the caller reads them back with its own
            E.finalize(buf, (1 << L.NSTAT) - 1)
            st = buf.stats[0]
        C1 = self.plan.irfft_yz(chat).reshape(-1) + self.V if want & 1 else None
        return C1, st

    def _clip(self, rho):   # _clip_density (solver.py:146-148)
        return torch.where(rho < self.lower, torch.full_like(rho, 1e-30), rho)

    def C1(self, rho):
        return self._pipeline(rho, 1)[0]

    def omega(self, rho):   # _get_Omega (solver.py:103-119); stores omega0
        _, st = self._pipeline(rho, 2)
        fn, dV = self.fn, self.dV
        rr = self._clip(rho)
        # one read-back of the pipeline's sums and the three reductions here
        sums = torch.stack([rho.sum(), (rr * (torch.log(fn.lambda3 * rr) - 1.0)).sum(), (rho * self.V).sum()])
        vals = torch.cat([st, sums]).cpu().numpy()
        st, (s_n, s_id, s_ext) = vals[:L.NSTAT], vals[L.NSTAT:]
        N = float(s_n) * dV
        fid = float(s_id) * dV / fn.beta
        G = fid - self.mu * N
        G += st[L.STAT_PHI] * dV / fn.beta
        G += 0.5 * st[L.STAT_MFA] * dV
        G += float(s_ext) * dV
        self.omega0 = G
        return G

    def n3max(self, field):
        return float(self._pipeline(field, 4)[1][L.STAT_N3MAX])

    def new_rho(self, C1):  # get_new_rho
        fn = self.fn
        return fn.beta * torch.exp(-fn.beta * C1) * self.fugacity

    def domega(self, rho, C1):   # _get_dOmega
        return torch.log(self.fn.lambda3 * self._clip(rho)) / self.fn.beta + C1 - self.mu

    def alpha_max(self, rho, G):   # _get_alpha_max (solver.py:150-165), G any field
        a, b = self.n3max(rho), self.n3max(G)
        return min(abs((1 - a) / ((b - a) + 1e-16)), 1.0)

    # ---- hybrid Picard step (solver.py:403-457) -----------------------------
    def hybrid_step(self, rho, C1):
        prev = self.omega0
        G = self.new_rho(C1)
        amax = self.alpha_max(rho, G)
        if np.isclose(amax, 0):
            aopt, lo, hi = 0, 0, 0
        else:
            a1 = 0.45 * amax
            o1 = self.omega((1 - a1) * rho + a1 * G)
            a2 = 0.9 * amax if o1 <= prev else 0.225 * amax
            o2 = self.omega((1 - a2) * rho + a2 * G)
            c, b, a = np.polyfit([0, a1, a2], [prev, o1, o2], 2)
            al = np.linspace(-max(a1, a2) / 4, max(a1, a2), 10000)
            om = a + b * al + c * al ** 2
            aopt = al[np.where(om == np.min(om))[0][0]]
            lo, hi = np.min(om) / kjmol, np.max(om) / kjmol
        if aopt <= 0:
            if hi - lo > self.thresh:
                fun = lambda x: self.omega((1 - x[0]) * rho + x[0] * G)  # noqa: E731
                aopt = opt.minimize(fun, [self.alpha_mix * amax], bounds=opt.Bounds(0.01 * amax, 0.9 * amax),
                                    method='SLSQP', options={'ftol': 1e-8}).x[0]
            else:
                aopt = self.alpha_mix * amax
        if aopt <= 0 or np.isclose(aopt, 0):
            aopt = self.alpha_mix * amax
        cf = self.correction_factor
        rho_new = self._clip((1 - aopt * cf) * rho + aopt * cf * G)
        C1n = self.C1(rho_new)
        self.omega(rho_new)
        return rho_new, C1n

    # ---- quasi-Newton step --------------------------------------------------
    def _flush(self):
        self.X, self.G = [], []
        self.g_prev = self.d_prev = None
        self.omega_hist = []
        self.k_picard = self.k_qn = 0

    def _record(self, rho, C1):   # _update_histories (:820-836)
        keep = rho > self.lower
        zero = torch.zeros_like(rho)
        self.X = (self.X + [torch.where(keep, rho, zero)])[-(self.m + 1):]
        self.G = (self.G + [torch.where(keep, self.domega(rho, C1), zero)])[-(self.m + 1):]
        self.omega_hist = (self.omega_hist + [self.omega0])[-(self.m + 1):]

    def _direction(self, g):   # _find_direction (:843-872)
        dX = [self.X[i + 1] - self.X[i] for i in range(len(self.X) - 1)]
        dG = [self.G[i + 1] - self.G[i] for i in range(len(self.G) - 1)]
        if self.method == 'bfgs':
            if not dX:
                return -g
            return _lbfgs(g, dX, dG, _gamma_last_pair(dX, dG))
        if self.method == 'broyden':
            h0 = _gamma_last_pair(dX, dG)
            if h0 is None:   # the reference multiplies by None here
                raise TypeError("bad operand type for unary -: 'NoneType'")
            return _lbroyden(g, dX, dG, h0)
        d, picard = _cg_descent(g, self.g_prev, self.d_prev)
        return None if picard else d

    def _backtracking(self, rho, g, d):   # _line_search_feasible (:874-934)
        f0 = self.omega_hist[-1]
        a = self.alpha_max(rho, d)
        while a > 1e-8:
            trial = self._clip(rho + a * d)
            f = self.omega(trial)
            gtp = _dot(g, trial - rho)
            if f0 - f > 1e3 * kjmol:
                a *= 0.01
                continue
            if f <= f0 + self.c1 * gtp * a:
                C1n = self.C1(trial)
                if bool(torch.isinf(self.new_rho(C1n)).any()):
                    a *= 0.01
                    continue
                return trial, C1n, f
            ratio = (f - f0) / abs(self.c1 * gtp) if gtp != 0 else np.inf
            a *= 0.01 if ratio > 100 else (0.1 if ratio > 10 else 0.6)
        raise SwitchToPicard('Line search not converging')

    def _quadratic(self, rho, g, d):   # _quadratic_line_search (:936-971)
        f0 = self.omega_hist[-1]
        a1 = self.alpha_max(rho, d) * self.correction_factor
        trial = self._clip(rho + a1 * d)
        f = self.omega(trial)
        gtp = _dot(g, trial - rho)
        if f <= f0 + self.c1 * gtp * a1:
            C1n = self.C1(trial)
            if not bool(torch.isinf(self.new_rho(C1n)).any()):
                return trial, C1n, f
        slope = _dot(g, d)
        aopt = -slope * a1 ** 2 / (2 * (f - f0 - slope * a1))
        if aopt < 0 or aopt > a1:
            raise SwitchToPicard('Quadratic line search not converging')
        rho_new = self._clip(rho + aopt * d)
        C1n = self.C1(rho_new)
        if bool(torch.isinf(self.new_rho(C1n)).any()):
            raise SwitchToPicard('Grho_new contains Infs, skipping this step')
        return rho_new, C1n, self.omega(rho_new)

    def _fixed(self, rho, g, d):   # _no_line_search (:973-985)
        a = 0.5 * self.alpha_max(rho, d) * self.correction_factor
        trial = self._clip(rho + a * d)
        C1n = self.C1(trial)
        if bool(torch.isinf(self.new_rho(C1n)).any()):
            raise SwitchToPicard('Grho_new contains Infs, skipping this step')
        return trial, C1n, self.omega(trial)

    def qn_step(self, rho, C1):   # _update_rho_QN (:987-1026)
        g = self.G[-1]
        d = self._direction(g)
        if d is None:
            raise SwitchToPicard('No descent direction found')
        dp = _cone_project(rho, d, self.lower)
        slope = _dot(g, dp)
        small = 1e-12 * max(1.0, _norm(rho))
        if _norm(dp) < small or slope >= 0:
            dp = _cone_project(rho, -g, self.lower)
            if _norm(dp) < small or slope >= 0:   # the first direction's slope, as in the reference
                raise SwitchToPicard('Projected steepest descent failed')
        if self.trust_radius is not None:
            dp = _cap(dp, max(1e-2, 0.5 * _norm(rho)))
        self.g_prev, self.d_prev = g, dp
        search = {'backtracking': self._backtracking, 'quadratic': self._quadratic, 'none': self._fixed}
        rho_new, C1n, om = search[self.line_search](rho, g, dp)
        res = _norm(self.new_rho(C1) - rho)
        res_new = _norm(self.new_rho(C1n) - rho_new)
        if res_new * 0.8 > res:
            raise SwitchToPicard('Residual norm increased too much')
        return rho_new, C1n, om

    def update(self, rho, C1):   # QuasiNewton.update_rho (:1028-1053)
        self._record(rho, C1)
        prev = self.omega0
        if self.k_picard < self.picard_first:
            out = self.hybrid_step(rho, C1)
            self.k_picard += 1
            return out
        if self.k_qn < self.qn_limit:
            try:
                rho_new, C1n, om = self.qn_step(rho, C1)
                if om > prev * 0.8:
                    raise SwitchToPicard('Quasi-Newton increased the grand potential')
                self.k_qn += 1
                return rho_new, C1n
            except SwitchToPicard:
                out = self.hybrid_step(rho, C1)
                self._flush()
                return out
        out = self.hybrid_step(rho, C1)
        self._flush()
        return out

    # ---- Solver._solve / solve ------------------------------------------------
    def _converged(self, rho_new, C1n, rho, N):   # _check_convergence (:167-234)
        dV, n = self.dV, self.npts
        iue = float((rho_new - rho).abs().sum()) * dV
        riue = iue / N if N > 0 else np.nan
        ok = True
        for c, t in zip(self.criteria, self.thresholds):
            if c == 'riue':
                v = riue
            elif c == 'res':
                v = _norm(self.new_rho(C1n) - rho_new) / np.sqrt(N) / np.sqrt(n)
            else:
                beta = self.fn.beta
                w = rho_new.abs() * beta * self.domega(rho_new, C1n) / (self.a_tol + self.r_tol * rho_new.abs())
                v = _norm(w[~(rho_new.abs() <= 1e-8)]) / np.sqrt(n)
            ok = ok and (v < t)
        if iue == 0 and np.isnan(riue):
            ok = True
        return ok

    def _solve(self, rho):
        self._flush()
        C1 = self.C1(rho)
        self.omega(rho)
        N_new, rho_new = float(rho.sum()) * self.dV, rho
        for k in range(self.nsteps):
            self.steps = k + 1
            rho_new, C1n = self.update(rho, C1)
            if not bool(torch.isfinite(rho_new).all()):
                raise FloatingPointError
            N_new = float(rho_new.sum()) * self.dV
            if self._converged(rho_new, C1n, rho, N_new):
                return N_new, rho_new, True
            rho, C1 = rho_new, C1n
        return N_new, rho_new, False

    def solve(self, chempot, rho0):
        """(N, rho [N1, N2, N3] on the device, converged); retries with the
        correction factor halved on non-finite densities (solver.py:317-345)."""
        from .batch import NoSolutionError
        fn = self.fn
        self.mu = float(chempot)
        self.fugacity = np.exp(fn.beta * self.mu) / fn.beta / fn.wavelength ** 3
        rho = torch.as_tensor(rho0, dtype=torch.float64, device="cuda").reshape(-1).clone()
        self.correction_factor = 1.0
        while self.correction_factor >= 0.25:
            try:
                N, r, conv = self._solve(rho)
                return N, r.reshape(self.plan.npoints), conv
            except FloatingPointError:
                self.correction_factor /= 2
        raise NoSolutionError("no finite solution for chempot %r" % chempot)
