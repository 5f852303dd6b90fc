"""Batched fixed-point solves on one grid shape (one "shape group").

``BatchSolve`` runs B independent solves (e.g. the pressures of an isotherm
on one host) together: every field operation is one kernel launch over all
active instances, and the per-instance control flow of the reference's
solvers is evaluated on the host from per-instance scalars (one small
device-to-host read per decision point).  A batch of one is the plain
per-point solve.

Control flow restated from cmmdft/solver.py:
  Solver._solve / solve            :236-345 (loop, non-finite retry)
  _check_convergence               :167-234 (RES / RIUE)
  _get_Omega                       :103-119
  Picard.update_rho_static         :392-401
  Picard.update_rho_hybrid         :403-457 (+ _get_alpha_max :150-165)
  Anderson.update_rho              :546-579
  Anderson.update_rho_Anderson     :581-604 (+ damping :537-544)
The Anderson mixing coefficients are the reference's SLSQP iterate
(anderson_coefs='slsqp', default: Kraft's SLSQP restated in
cmm_anderson_slsqp on the Gram matrix of the residuals), or with
anderson_coefs='exact' the exact minimiser of ||sum a_i r_i|| subject to
a_i >= 0, sum a_i = 1 (support enumeration on the Gram matrix), which
converges in fewer steps but leaves the reference's trajectory.
"""
import ctypes
import itertools

import numpy as np
import scipy.optimize as opt
import torch

from . import _lib as L
from . import engine as E
from .units import angstrom, kjmol


class NoSolutionError(Exception):
    """All retries of a solve hit non-finite densities (solver.py:343-345)."""


def simplex_qp(M, idx):
    """argmin_a a^T M a  s.t. a >= 0, sum a = 1, over the entries ``idx``.

    Exact minimiser by enumerating supports: on each support S the
    equality-constrained minimum is a_S = M_SS^+ 1 / (1^T M_SS^+ 1); the
    feasible candidate with the lowest objective is the global minimum of
    this convex problem.
    """
    n = len(idx)
    Ms = M[np.ix_(idx, idx)]
    best, best_val = None, np.inf
    scale = max(np.max(np.abs(np.diag(Ms))), 1e-300)
    for k in range(1, n + 1):
        for S in itertools.combinations(range(n), k):
            A = Ms[np.ix_(S, S)] / scale
            one = np.ones(k)
            try:
                x = np.linalg.solve(A, one)
            except np.linalg.LinAlgError:
                x = np.linalg.lstsq(A, one, rcond=None)[0]
            s = x.sum()
            if not np.isfinite(s) or abs(s) < 1e-300:
                continue
            a = x / s
            if np.any(a < -1e-14):
                continue
            a = np.clip(a, 0.0, None)
            a /= a.sum()
            full = np.zeros(n)
            full[list(S)] = a
            val = full @ Ms @ full
            if val < best_val * (1 - 1e-13) or best is None:
                best, best_val = full, val
    if best is None:
        best = np.full(n, 1.0 / n)
    return best


_SUPPORTS = {}


def _supports(n):
    """All non-empty supports of n variables as a boolean matrix [2^n - 1, n]."""
    if n not in _SUPPORTS:
        rows = [[(k >> i) & 1 for i in range(n)] for k in range(1, 1 << n)]
        _SUPPORTS[n] = np.array(rows, dtype=bool)
    return _SUPPORTS[n]


def anderson_slsqp(gram):
    """SLSQP mixing coefficients of one instance (cmm_anderson_slsqp).

    gram [n, n] = <r_i, r_j>, oldest residual first.  Returns (alpha, mode,
    iterations) with SLSQP's exit mode (0 converged, 8, 9); alpha is its last
    iterate whatever the mode, as solver.py:589-591 takes ``.x``.
    """
    G = np.ascontiguousarray(gram, dtype=np.float64)
    n = G.shape[0]
    a = np.empty(n)
    mode, nit = ctypes.c_int(0), ctypes.c_int(0)
    dp = ctypes.POINTER(ctypes.c_double)
    L.check(L.lib().cmm_anderson_slsqp(G.ctypes.data_as(dp), n, a.ctypes.data_as(dp), ctypes.byref(mode),
                                       ctypes.byref(nit)), "cmm_anderson_slsqp")
    return a, mode.value, nit.value


def simplex_qp_batched(M):
    """simplex_qp for a stack of Gram matrices M [B, n, n].

    For every support S the equality-constrained minimiser solves the
    bordered system [M_SS 1; 1^T 0] [a; lam] = [0; 1] (well posed also for
    rank-deficient Gram matrices); variables outside S are pinned to 0 by
    identity rows.  All supports of all instances go through one stacked
    solve; a singular support falls back to a least-squares solve on its own.
    """
    B, n, _ = M.shape
    S = _supports(n)                                     # [K, n]
    K = len(S)
    diag = np.abs(np.diagonal(M, axis1=1, axis2=2))
    scale = np.maximum(diag.max(axis=1), 1e-300)
    Ms = M / scale[:, None, None]
    A = np.zeros((B, K, n + 1, n + 1))
    inS = S[:, :, None] & S[:, None, :]
    A[:, :, :n, :n] = np.where(inS[None], Ms[:, None], 0.0)
    idx = np.arange(n)
    A[:, :, idx, idx] = np.where(S[None], A[:, :, idx, idx], 1.0)
    A[:, :, :n, n] = S[None].astype(float)
    A[:, :, n, :n] = S[None].astype(float)
    rhs = np.zeros((B, K, n + 1, 1))
    rhs[:, :, n, 0] = 1.0
    try:
        x = np.linalg.solve(A, rhs)[..., 0]
    except np.linalg.LinAlgError:
        x = np.empty((B, K, n + 1))
        for k in range(K):
            try:
                x[:, k] = np.linalg.solve(A[:, k], rhs[:, k])[..., 0]
            except np.linalg.LinAlgError:
                for b in range(B):
                    x[b, k] = np.linalg.lstsq(A[b, k], rhs[b, k, :, 0], rcond=None)[0]
    a = np.where(S[None], x[..., :n], 0.0)
    with np.errstate(all='ignore'):
        ok = np.all(np.isfinite(a), axis=2) & np.all(a >= -1e-12, axis=2)
        a = np.clip(np.nan_to_num(a), 0.0, None)
        a /= np.maximum(a.sum(axis=2, keepdims=True), 1e-300)
        val = np.einsum('bki,bij,bkj->bk', a, Ms, a)
    val = np.where(ok, val, np.inf)
    # lowest objective (Ms is scaled to unit diagonal maximum, so values are
    # O(1)); ties within 1e-14 go to the support enumerated first
    vmin = val.min(axis=1, keepdims=True)
    pick = np.argmax(val <= vmin + 1e-14, axis=1)
    best = a[np.arange(B), pick]
    best[~np.isfinite(vmin[:, 0])] = 1.0 / n
    return best


def _grid_full(cf, hi, n):
    al = np.linspace(-hi / 4, hi, n, axis=1)
    om = cf[:, 2:3] + cf[:, 1:2] * al + cf[:, 0:1] * al ** 2
    j = np.argmin(om, axis=1)                 # first minimum, as np.where(om == min)[0][0]
    rows = np.arange(len(hi))
    return al[rows, j], om[rows, j], np.max(om, axis=1)


def parabola3(x1, x2, y0, y1, y2):
    """Coefficients [c2, c1, c0] (np.polyfit order) of the parabola through
    (0, y0), (x1, y1), (x2, y2), per row: the fit of np.polyfit([0, x1, x2],
    [y0, y1, y2], 2) (solver.py:425), in closed form for all rows at once."""
    with np.errstate(all='ignore'):
        d1 = (y1 - y0) / x1
        d2 = (y2 - y0) / x2
        c2 = (d2 - d1) / (x2 - x1)
        c1 = d1 - c2 * x1
    return np.stack([c2, c1, np.asarray(y0, dtype=float)], axis=1)


def grid_parabola(cf, hi, n=10000):
    """First grid point minimising om = c a^2 + b a + a0 on
    np.linspace(-hi/4, hi, n) per row, and the min/max of om on that grid
    (cmmdft/solver.py:426-432).  Exact against evaluating all n points: for a
    convex parabola om is evaluated with the reference's expression on the
    ends and on every grid point within reach of the vertex, where reach
    covers all points whose value can lie within 64 ulps of the vertex value
    (rounding ties near a flat vertex resolve as the full search does).
    Concave, linear or rounding-flat rows use the full grid."""
    cf = np.asarray(cf, dtype=float)
    hi = np.asarray(hi, dtype=float)
    R = len(hi)
    aopt, mn, mx = np.zeros(R), np.zeros(R), np.zeros(R)
    c, b, a0 = cf[:, 0], cf[:, 1], cf[:, 2]
    lo = -hi / 4
    step = (hi - lo) / (n - 1)
    eps = np.finfo(float).eps
    with np.errstate(all='ignore'):
        vert = -b / (2 * c)
        scale = np.maximum(np.abs(a0), np.abs(a0 + b * vert + c * vert * vert))
        W = np.ceil(np.sqrt(64 * eps * scale / c) / step) + 2
    fast = (c > 0) & np.isfinite(W) & (W < n // 4) & (step > 0) & np.isfinite(vert)
    slow = ~fast
    if slow.any():
        aopt[slow], mn[slow], mx[slow] = _grid_full(cf[slow], hi[slow], n)
    if fast.any():
        f = np.where(fast)[0]
        jv = np.clip(np.floor((vert[f] - lo[f]) / step[f]), 0, n - 1)
        Wm = int(np.max(W[f]))
        offs = np.arange(-Wm, Wm + 1)
        cand = np.concatenate([np.zeros((len(f), 1)), jv[:, None] + offs[None, :], np.full((len(f), 1), n - 1)],
                              axis=1)
        cand = np.sort(np.clip(cand, 0, n - 1).astype(np.int64), axis=1)
        # grid values as numpy.linspace forms them: j * step + lo, last point = hi
        al = cand * step[f, None] + lo[f, None]
        al = np.where(cand == n - 1, hi[f, None], al)
        om = a0[f, None] + b[f, None] * al + c[f, None] * al ** 2
        rows = np.arange(len(f))
        j = np.argmin(om, axis=1)             # first minimum (candidates sorted by index)
        aopt[f], mn[f], mx[f] = al[rows, j], om[rows, j], np.max(om, axis=1)
    return aopt, mn, mx


def workspace(fn, B, nring, group=0):
    """Device buffers of a batch of B instances with an nring-deep history,
    cached on the Functional so repeated solves of the same shape reuse them
    (one set per group of a grouped solve)."""
    cache = fn.__dict__.setdefault('_workspaces', {})
    key = (B, nring, group)
    if key in cache:
        return cache[key]
    plan = fn.plan
    n1, n2, n3 = plan.npoints
    dev, f64 = 'cuda', torch.float64
    ws = dict(
        ring=torch.zeros((nring, B, n1, n2, n3), dtype=f64, device=dev),
        rres=torch.zeros((nring, B, n1, n2, n3), dtype=f64, device=dev),
        trial=torch.empty((B, n1, n2, n3), dtype=f64, device=dev),
        rho0=torch.empty((B, n1, n2, n3), dtype=f64, device=dev),
        rhohat=plan.new_spec(B), that=plan.new_spec(B), chat=plan.new_spec(B), chat2=plan.new_spec(B),
        buf=E.Buffers(plan, B, nwork=fn.nwork),
        params=torch.zeros((B, 4), dtype=f64, device=dev),
        coef=torch.zeros((B, L.MAX_FIELDS), dtype=f64, device=dev),
        active=torch.zeros(B, dtype=torch.int32, device=dev),
    )
    ws['buf'].part[:, L.STAT_N3MAX, :] = -np.inf
    # pinned staging of uploads (8-deep rings) and the native driver's
    # read-backs, carved from two page-locked blocks
    nf = 8 * B * (L.MAX_FIELDS + 4) + B * (L.NSTAT + L.NLS + 1)
    pf = torch.zeros(nf, dtype=f64, pin_memory=True)
    pi = torch.zeros(8 * B, dtype=torch.int32, pin_memory=True)
    cuts = itertools.accumulate([0] + [B * L.MAX_FIELDS] * 8 + [B * 4] * 8 + [B * L.NSTAT, B * L.NLS, B])
    o = list(cuts)
    ws['pin'] = dict(active=[pi[i * B:(i + 1) * B] for i in range(8)],
                     coef=[pf[o[i]:o[i + 1]].view(B, L.MAX_FIELDS) for i in range(8)],
                     params=[pf[o[8 + i]:o[9 + i]].view(B, 4) for i in range(8)])
    ws['pin_read'] = dict(stats=pf[o[16]:o[17]].view(B, L.NSTAT), ls=pf[o[17]:o[18]].view(B, L.NLS),
                          alpha=pf[o[18]:o[19]])
    cache[key] = ws
    return ws


def ls_workspace(fn, ws, B, nring):
    """Buffers of the transform-free hybrid line search, added to ``ws`` on
    first use: per ring slot the yz-spectrum and the weighted densities of
    its density, the weighted densities and spectrum of a residual, and the
    line-search partial sums."""
    if 'wd_ring' in ws:
        return ws
    plan = fn.plan
    n1, n2, n3 = plan.npoints
    dev, f64 = 'cuda', torch.float64
    nslot = ws['buf'].nslot
    ws['wd_ring'] = torch.empty((nring, fn.nwd, B, n1, n2, n3), dtype=f64, device=dev)
    ws['spec_ring'] = torch.empty((nring, B, plan.nspec * 2), dtype=f64, device=dev)
    ws['wd_r'] = torch.empty((fn.nwd, B, n1, n2, n3), dtype=f64, device=dev)
    ws['rhat'] = plan.new_spec(B)
    ls_part = torch.zeros((B, L.NLS, nslot), dtype=f64, device=dev)
    ls_part[:, L.LS_N3MAX_G, :] = -np.inf
    ws['ls_part'] = ls_part
    ws['ls'] = torch.zeros((B, L.NLS), dtype=f64, device=dev)
    ws['ls_alpha'] = torch.zeros(B, dtype=f64, device=dev)
    return ws


class BatchSolve(object):
    """Solve B fixed points that share a Functional (grid, host, guest, T).

    method: 'static' (Picard), 'hybrid' (Picard line search), 'anderson'
    or 'hybridanderson' (the reference's Anderson default).
    """

    def __init__(self, fn, chempots, method='hybridanderson', nsteps=500, threshold=1e-6,
                 criterion='res', alpha_mix=0.1, m=5, damping=0.3, delta=0.2, damping_max=0.8,
                 damping_min=0.01, adaptive_damping=True, damping_factors=(1.5, 0.5), divergence_guard=False,
                 a_tol=1e-6, r_tol=1e-4, group=0, anderson_coefs='slsqp', track_history=False):
        self.fn = fn
        if anderson_coefs not in ('slsqp', 'exact'):
            raise ValueError("anderson_coefs must be 'slsqp' or 'exact'")
        self.anderson_coefs = anderson_coefs
        self.host_out = None
        self.plan = fn.plan
        self.mu = np.asarray(chempots, dtype=np.float64).ravel()
        self.B = B = len(self.mu)
        self.method = method.lower()
        assert self.method in ('static', 'hybrid', 'anderson', 'hybridanderson'), method
        self.nsteps = int(nsteps)
        crit = criterion if isinstance(criterion, (list, tuple)) else [criterion]
        thr = threshold if isinstance(threshold, (list, tuple)) else [threshold] * len(crit)
        self.criteria = [c.lower() for c in crit]
        for c in self.criteria:
            if c not in ('res', 'riue', 'der'):
                raise NotImplementedError("criterion %r" % c)
        self.thresholds = [float(t) for t in thr]
        self.tol = (float(a_tol), float(r_tol))   # DER tolerances (solver.py:25-26)
        # The history's derivative column (solver.py:218-220) is the DER sum
        # without the tolerance weighting: with no 'der' criterion to serve,
        # the kernels' DER sum is taken with a_tol = 1, r_tol = 0, which is
        # exactly that.  With a 'der' criterion the column stays NaN.
        self.der_history = bool(track_history) and 'der' not in self.criteria
        if self.der_history:
            self.tol = (1.0, 0.0)
        self.alpha_mix = float(alpha_mix)
        self.thresh = 1 * kjmol
        self.m = int(m)
        self.damping0 = float(damping)
        self.damping_max, self.damping_min = damping_max, damping_min
        self.adaptive = adaptive_damping
        self.dfac = damping_factors
        self.delta = delta
        # Opt-in: retire an instance as not converged once RES exceeds 1e6 x its
        # best value and has not decreased over the last 5 steps.  The
        # reference iterates such instances to nsteps (and reports them not
        # converged); with this guard the batch stops paying for them.
        self.divergence_guard = bool(divergence_guard)
        self.diverged = np.zeros(len(np.atleast_1d(chempots)), dtype=bool)
        beta = fn.beta
        # fugacity = exp(beta mu) / beta / Lambda^3 (solver.py:92)
        self.fug = np.exp(beta * self.mu) / beta / fn.wavelength ** 3
        n1, n2, n3 = self.plan.npoints
        self.npts = n1 * n2 * n3
        self.dr = self.plan.dr
        self.nring = max(self.m, 2) if 'anderson' in self.method else 2
        ws = workspace(fn, B, self.nring, group)
        if self.method != 'static':
            ls_workspace(fn, ws, B, self.nring)
        for k, v in ws.items():
            setattr(self, k, v)
        self._pin_i = 0
        self.mask_host = np.zeros(B, dtype=bool)
        # optional per-step record: (step, branch, omega, RES) per instance
        self.trace = None
        self.kernel_launches = 0
        self.omega_evals = 0
        # optional timing of the functional pipeline: list of
        # (start_event, end_event, want, n_active) appended per launch
        self.pipeline_events = None

    # ------------------------------------------------------------ helpers --
    def _pinned(self, kind):
        """Next pinned staging buffer of a small ring (host -> device uploads
        are asynchronous; every step drains the stream at its stats read long
        before a ring slot comes round again)."""
        ring = self.pin[kind]
        self._pin_i = (self._pin_i + 1) % len(ring)
        return ring[self._pin_i]

    def _set_active(self, mask):
        self.mask_host = np.asarray(mask, dtype=bool).copy()
        h = self._pinned('active')
        h.numpy()[:] = self.mask_host
        self.active.copy_(h, non_blocking=True)

    def _stats(self, mask_bits=(1 << L.NSTAT) - 1):
        E.finalize(self.buf, mask_bits, self.active)
        self.kernel_launches += 1
        return self.buf.stats.cpu().numpy()

    def _mix(self, coefs, fields, clip, ref, out, thr=0.0, spec_out=None):
        """out = sum_j coefs[:, j] * fields[j] (fields: [B, ...] tensors); spectrum
        into spec_out (default self.that)."""
        h = self._pinned('coef')
        c = h.numpy()
        c[:] = 0.0
        c[:, :len(fields)] = coefs
        self.coef.copy_(h, non_blocking=True)
        E.mix_step(self.fn, self.buf, self.coef, fields, [self.npts] * len(fields), clip, ref, out,
                   self.that if spec_out is None else spec_out, thr=thr, active=self.active)
        self.kernel_launches += 1

    def _c1(self, spec, chat, want, wd=None):
        ev = self.pipeline_events
        if ev is not None:
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record()
        self.fn.c1(self.buf, spec, chat, want=want, active=self.active, wd=wd)
        if ev is not None:
            e1.record()
            ev.append((e0, e1, want, int(self.mask_host.sum())))
        self.kernel_launches += 3 if (want & 1) else 2

    def _set_params(self, a=None, n3=None):
        """params[b] = (fugacity, Picard mixing a, mu, max n3 of the current density)."""
        h = self._pinned('params')
        p = h.numpy()
        p[:] = 0.0
        p[:, 0] = self.fug
        if a is not None:
            p[:, 1] = a
        p[:, 2] = self.mu
        if n3 is not None:
            p[:, 3] = n3
        self.params.copy_(h, non_blocking=True)

    def _residual(self, chat, rho, r_out, hist):
        E.residual_step(self.fn, self.buf, self.params, chat, rho, r_out, hist=hist, hstride=self.npts,
                        active=self.active, tol=self.tol)
        self.kernel_launches += 1

    def _omega(self, st, b):
        """Grand potential from the per-instance sums (solver.py:103-119)."""
        beta, dr = self.fn.beta, self.dr
        N = st[L.STAT_N] * dr
        Fid = (st[L.STAT_FID] * dr) / beta
        G = Fid - self.mu[b] * N
        G += (st[L.STAT_PHI] * dr) / beta
        G += 0.5 * (st[L.STAT_MFA] * dr)
        G += st[L.STAT_FEXT] * dr
        if self.fn.wda is not None:
            G += st[L.STAT_WDA] * dr
        return G

    def _omega_rows(self, st, idx):
        """_omega for the instances idx (rows st[idx]), elementwise in the same order."""
        beta, dr = self.fn.beta, self.dr
        s = st[idx]
        N = s[:, L.STAT_N] * dr
        G = (s[:, L.STAT_FID] * dr) / beta - self.mu[idx] * N
        G += (s[:, L.STAT_PHI] * dr) / beta
        G += 0.5 * (s[:, L.STAT_MFA] * dr)
        G += s[:, L.STAT_FEXT] * dr
        if self.fn.wda is not None:
            G += s[:, L.STAT_WDA] * dr
        return G

    def _omega_parts(self, st):
        beta, dr = self.fn.beta, self.dr
        out = dict(N=st[L.STAT_N] * dr, Fid=(st[L.STAT_FID] * dr) / beta,
                   HardSphere=(st[L.STAT_PHI] * dr) / beta, MFA=0.5 * (st[L.STAT_MFA] * dr),
                   ExtPot=st[L.STAT_FEXT] * dr)
        if self.fn.wda is not None:
            out['WDA-V'] = st[L.STAT_WDA] * dr
        return out

    def _eval_density(self, mask, coefs, fields, clip, out, want, ref):
        """Mix a density into `out`, forward it, run the functional pipeline
        (want bits: 1 C1 spectrum into chat2, 2 free-energy sums, 4 max n3)."""
        self._set_active(mask)
        self._mix(coefs, fields, clip, ref, out)
        self._c1(self.that, self.chat2 if (want & 1) else None, want)
        return self._stats()

    # ------------------------------------------------------------- solve ---
    def initial_density(self, rho0):
        self.rho0.copy_(rho0)

    def solve(self, rho0, cf=None, host_out=None):
        """Run all instances from rho0 [B, N1, N2, N3]; returns (N, rho, converged).

        host_out: optional pinned CPU tensor [B, N1, N2, N3].  Each instance's
        final density is copied into it on a side stream as soon as that
        instance is finished, overlapping the copy with the iterations of
        the instances still running; all copies have landed when solve
        returns."""
        self.host_out = host_out
        if host_out is not None:
            if not host_out.is_pinned() or tuple(host_out.shape) != tuple(rho0.shape):
                raise ValueError("host_out must be a pinned tensor of the shape of rho0")
            self._copy_stream = torch.cuda.Stream()
        self.initial_density(rho0)
        B = self.B
        self.cf = np.ones(B) if cf is None else np.asarray(cf, dtype=float).copy()
        self._set_params()
        self.result = torch.empty_like(self.rho0)
        self.N_out = np.full(B, np.nan)
        self.conv = np.zeros(B, dtype=bool)
        self.steps = np.zeros(B, dtype=int)
        self.failed = np.zeros(B, dtype=bool)
        self.history = [[] for _ in range(B)]
        if self.trace is not None:
            self.trace = [[] for _ in range(B)]
        todo = np.ones(B, dtype=bool)
        while todo.any():
            retry = self._solve_once(todo)
            # non-finite -> halve the correction factor and restart (solver.py:335-345)
            for b in np.where(retry)[0]:
                self.cf[b] /= 2
                if self.cf[b] < 0.25:
                    self.failed[b] = True
                    retry[b] = False
            todo = retry
        if host_out is not None:
            self._copy_stream.synchronize()
        if self.failed.any():
            raise NoSolutionError("instances %s hit non-finite densities on every retry"
                                  % list(np.where(self.failed)[0]))
        return self.N_out, self.result, self.conv

    def _init_state(self, todo):
        """rho0 -> ring slot 0, its spectrum, C1, Omega and (for Anderson) r_0.
        The hybrid/Anderson loop also keeps the spectrum and weighted densities
        of ring slot 0 for the line search."""
        if self.method == 'static':
            st = self._eval_density(todo, np.ones((self.B, 1)), [self.rho0], L.CLIP_NONE, self.ring[0],
                                    1 | 2 | 4, self.rho0)
            self.rhohat.copy_(self.that)
        else:
            self._set_active(todo)
            self._mix(np.ones((self.B, 1)), [self.rho0], L.CLIP_NONE, self.rho0, self.ring[0],
                      spec_out=self.spec_ring[0])
            self._c1(self.spec_ring[0], self.chat2, 1 | 2 | 4 | 8, wd=self.wd_ring[0])
            st = self._stats()
        self.chat.copy_(self.chat2)
        self.omega0 = np.array([self._omega(st[b], b) for b in range(self.B)])
        self.n3max = st[:, L.STAT_N3MAX].copy()
        self.Ncur = st[:, L.STAT_N] * self.dr
        self.last_stats = st.copy()
        return st

    def _solve_once(self, todo):
        method = self.method
        self._init_state(todo)
        live = todo.copy()
        retry = np.zeros(self.B, dtype=bool)
        if method == 'static':
            return self._loop_static(live, retry)
        return self._loop_general(live, retry)

    # ---------------------------------------------------- static Picard ---
    def _loop_static(self, live, retry):
        B = self.B
        cur = np.zeros(B, dtype=int)  # ring slot of the current density
        thr = 1e-10 / angstrom ** 3
        prev = None  # stats of the previous launch
        step = 0
        self._set_active(live)
        pending = np.zeros(B, dtype=bool)  # instances whose step `step` awaits its RES check
        while live.any():
            step += 1
            self._set_params(self.alpha_mix * self.cf)
            # slot choice: ring slot (cur+1)%2 per instance -> launch per parity group
            for par in (0, 1):
                grp = live & (cur == par)
                if not grp.any():
                    continue
                self._set_active(grp)
                E.picard_static_step(self.fn, self.buf, self.params, thr, self.chat, self.ring[par],
                                     self.ring[1 - par], self.rhohat, active=self.active, tol=self.tol)
                self.kernel_launches += 1
            self._set_active(live)
            st = self._stats()
            # RES of the density produced by the previous step
            for b in np.where(live)[0]:
                if step > 1:
                    N = prev[b, L.STAT_N] * self.dr
                    res = np.sqrt(st[b, L.STAT_RES2]) / np.sqrt(N) / np.sqrt(self.npts)
                    iue = prev[b, L.STAT_IUE] * self.dr
                    der = np.sqrt(st[b, L.STAT_DER]) / np.sqrt(self.npts)
                    if self._converged(b, N, res, iue, der):
                        self._finish(b, self.ring[cur[b], b], N, step - 1, True)
                        live[b] = False
                        continue
                    if step - 1 >= self.nsteps or self._diverging(b):
                        self.diverged[b] = step - 1 < self.nsteps
                        self._finish(b, self.ring[cur[b], b], N, step - 1, False)
                        live[b] = False
                        continue
                if st[b, L.STAT_NONFIN] > 0:
                    retry[b] = True
                    live[b] = False
                    continue
                cur[b] = 1 - cur[b]
            if not live.any():
                break
            self._set_active(live)
            self._c1(self.rhohat, self.chat, 1)
            prev = st
        return retry

    def _diverging(self, b):
        if not self.divergence_guard:
            return False
        r = np.array([h[1] for h in self.history[b]])
        if len(r) < 8 or not np.isfinite(r[-1]):
            return len(r) >= 8
        best = np.nanmin(r)
        return bool(r[-1] > 1e6 * best and np.all(np.diff(r[-6:]) >= 0))

    def _diverging_rows(self, idx, k):
        """_diverging for the instances idx at step k from the RES history array."""
        if not self.divergence_guard or k < 8:
            return np.zeros(len(idx), dtype=bool)
        r = self.res_hist[idx, 1:k + 1]
        last = r[:, -1]
        with np.errstate(invalid='ignore'):
            best = np.nanmin(r, axis=1)
            rising = np.all(np.diff(r[:, -6:], axis=1) >= 0, axis=1)
        return ~np.isfinite(last) | ((last > 1e6 * best) & rising)

    def _converged(self, b, N, res, iue, der=np.nan):
        ok = True
        riue = iue / N if N > 0 else np.nan
        for c, t in zip(self.criteria, self.thresholds):
            v = res if c == 'res' else (riue if c == 'riue' else der)
            ok = ok and (v < t)
        self.history[b].append((N, res, riue, float(self.omega0[b]), der if self.der_history else np.nan))
        if iue == 0 and np.isnan(riue):
            ok = True
        return bool(ok)

    def _finish(self, b, rho_b, N, steps, conv):
        self.result[b].copy_(rho_b)
        if self.host_out is not None:
            ev = torch.cuda.Event()
            ev.record()
            cs = self._copy_stream
            cs.wait_event(ev)
            with torch.cuda.stream(cs):
                self.host_out[b].copy_(self.result[b], non_blocking=True)
        self.N_out[b] = N
        self.conv[b] = conv
        self.steps[b] = steps

    # -------------------------------------------- hybrid / Anderson loop ---
    def _loop_general(self, live, retry):
        B, m = self.B, self.nring
        anderson = 'anderson' in self.method
        pure = self.method == 'anderson'
        # ring bookkeeping: density j and residual j live in slot j % m
        self.gram = np.zeros((B, m, m))
        self.rnorm2 = np.zeros((B, m))
        self.And_true = np.zeros(B, dtype=bool)
        self.it_eps0 = np.full(B, np.nan)
        self.damping = np.full(B, self.damping0)
        self.res_hist = np.full((B, self.nsteps + 2), np.nan)
        self.ls_host = np.zeros((B, L.NLS))
        self.alpha_host = np.zeros(B)
        self.ls_slot = np.full(B, -1)
        # r_0 for the initial density, and the first line search ahead
        self._set_active(live)
        self._residual(self.chat, self.ring[0], self.rres[0], [])
        E.finalize(self.buf, (1 << L.NSTAT) - 1, self.active)
        self.kernel_launches += 1
        self._launch_ls(live, 0, self.buf.stats[:, L.STAT_N3MAX])
        st, ls, al = self._read(ls=True)
        self._keep_ls(live, 0, ls, al)
        self.rnorm2[:, 0] = st[:, L.STAT_RES2]
        self.gram[:, 0, 0] = st[:, L.STAT_RES2]
        self.gnonfin = st[:, L.STAT_GNONFIN].copy()
        k = 0
        while live.any():
            k += 1  # curr_step
            s_prev = (k - 1) % m
            s_new = k % m
            # --- Anderson.update_rho bookkeeping (solver.py:546-561)
            res_norm = np.sqrt(self.rnorm2[:, s_prev])
            it_eps = res_norm / self.Ncur
            if k < 3:
                self.it_eps0 = np.where(live, it_eps, self.it_eps0)
            if anderson:
                cond = pure | ((it_eps <= self.it_eps0 * self.delta) & (k > 4)) | self.And_true
            else:
                cond = np.zeros(B, dtype=bool)
            cond &= live
            hyb = live & ~cond
            prev_omega = self.omega0.copy()
            if cond.any():
                ok = self._anderson_candidate(cond, k, s_prev, s_new)
                self.And_true |= cond
                hyb |= cond & ~ok
                if self.trace is not None:
                    for b in np.where(cond)[0]:
                        self.trace[b].append((k, 'A' if ok[b] else 'A-rejected', float(self.omega0[b])))
            if hyb.any():
                self._hybrid_step(hyb, k, s_prev, s_new)
                if self.trace is not None:
                    for b in np.where(hyb)[0]:
                        self.trace[b].append((k, 'H', float(self.omega0[b])))
            # --- after the update: non-finite check, N, convergence (solver.py:286-305)
            idx = np.where(live)[0]
            self.steps[idx] = k
            st = self.last_stats[idx]
            bad = st[:, L.STAT_NONFIN] > 0
            retry[idx[bad]] = True
            live[idx[bad]] = False
            idx, st = idx[~bad], st[~bad]
            if idx.size == 0:
                continue
            with np.errstate(invalid='ignore', divide='ignore'):
                N = st[:, L.STAT_N] * self.dr
                res = np.sqrt(self.rnorm2[idx, s_new]) / np.sqrt(N) / np.sqrt(self.npts)
                iue = st[:, L.STAT_IUE] * self.dr
                der = np.sqrt(st[:, L.STAT_DER]) / np.sqrt(self.npts)
            self.Ncur[idx] = N
            conv = self._converged_rows(idx, N, res, iue, der)
            self.res_hist[idx, k] = res
            done = conv | (k >= self.nsteps) | self._diverging_rows(idx, k)
            for j in np.where(done)[0]:
                b = idx[j]
                if not conv[j]:
                    self.diverged[b] = k < self.nsteps
                self._finish(b, self.ring[s_new, b], N[j], k, bool(conv[j]))
                live[b] = False
        return retry

    def _converged_rows(self, idx, N, res, iue, der):
        """_converged for the instances idx (arrays), with their history entries."""
        with np.errstate(invalid='ignore', divide='ignore'):
            riue = np.where(N > 0, iue / N, np.nan)
        ok = np.ones(len(idx), dtype=bool)
        for c, t in zip(self.criteria, self.thresholds):
            v = res if c == 'res' else (riue if c == 'riue' else der)
            ok &= (v < t)
        for j, b in enumerate(idx):
            self.history[b].append((N[j], res[j], riue[j], float(self.omega0[b]),
                                    der[j] if self.der_history else np.nan))
        ok |= (iue == 0) & np.isnan(riue)
        return ok

    def _valid_hist(self, k_new, s_new):
        """Slots of residuals r_{k_new-m+1} .. r_{k_new-1} (excluding s_new)."""
        m = self.nring
        return [j % m for j in range(max(0, k_new - m + 1), k_new)]

    def _post_update(self, mask, k, s_new, st_mix, ahead=None):
        """C1, Omega and residual of the density just written to ring slot s_new
        (its spectrum in spec_ring[s_new]); its weighted densities are kept.
        ahead: instances whose next step is likely a hybrid one; their line
        search for this density is launched before the single read-back."""
        self._c1(self.spec_ring[s_new], self.chat2, 1 | 2 | 4 | 8, wd=self.wd_ring[s_new])
        hist_slots = self._valid_hist(k, s_new)
        self._residual(self.chat2, self.ring[s_new], self.rres[s_new], [self.rres[j] for j in hist_slots])
        E.finalize(self.buf, (1 << L.NSTAT) - 1, self.active)
        self.kernel_launches += 1
        if ahead is not None and ahead.any():
            self._launch_ls(ahead, s_new, self.buf.stats[:, L.STAT_N3MAX])
            st, ls, al = self._read(ls=True)
            self._keep_ls(ahead, s_new, ls, al)
        else:
            st = self._read()
        return st, hist_slots

    def _commit_residual(self, mask, st, k, s_new, hist_slots):
        idx = np.where(mask)[0]
        if idx.size == 0:
            return
        self.rnorm2[idx, s_new] = st[idx, L.STAT_RES2]
        self.gram[idx, s_new, s_new] = st[idx, L.STAT_RES2]
        for h, j in enumerate(hist_slots):
            g = st[idx, L.STAT_GRAM0 + h]
            self.gram[idx, s_new, j] = g
            self.gram[idx, j, s_new] = g
        self.n3max[idx] = st[idx, L.STAT_N3MAX]
        self.last_stats[idx] = st[idx]

    def _anderson_candidate(self, mask, k, s_prev, s_new):
        """Anderson.update_rho_Anderson + the acceptance tests; returns accepted mask."""
        B, m = self.B, self.nring
        mk = min(k, self.m)
        slots = [j % m for j in range(k - mk, k)]  # oldest .. newest
        coefs = np.zeros((B, 2 * mk))
        idx = np.where(mask)[0]
        grams = self.gram[idx][:, slots][:, :, slots]
        if self.anderson_coefs == 'exact':
            alphas = simplex_qp_batched(grams)
        else:   # update_rho_Anderson's SLSQP (solver.py:585-591)
            alphas = np.stack([anderson_slsqp(G)[0] for G in grams]) if len(idx) else np.zeros((0, mk))
        if self.adaptive:  # _get_damping_coefficient (solver.py:537-544)
            r = np.sqrt(self.rnorm2[idx, s_prev])
            p = np.sqrt(self.rnorm2[idx, (k - 2) % m]) if k >= 2 else np.zeros(len(idx))
            dm = self.damping[idx]
            self.damping[idx] = np.where(r < p, np.minimum(dm * self.dfac[0], self.damping_max),
                                         np.maximum(dm * self.dfac[1], self.damping_min))
        d = self.cf[idx] * self.damping[idx]
        coefs[idx, :mk] = alphas
        coefs[idx, mk:] = d[:, None] * alphas
        fields = [self.ring[j] for j in slots] + [self.rres[j] for j in slots]
        self._set_active(mask)
        self.ls_slot[mask & (self.ls_slot == s_new)] = -1  # slot s_new gets a new density
        self._mix(coefs, fields, L.CLIP_DENSITY, self.ring[s_prev], self.ring[s_new], spec_out=self.spec_ring[s_new])
        st, hist_slots = self._post_update(mask, k, s_new, None)
        ok = np.zeros(B, dtype=bool)
        cand = idx[~(st[idx, L.STAT_GNONFIN] > 0)]
        if cand.size:
            om = self._omega_rows(st, cand)
            prev = self.omega0[cand].copy()
            self.omega0[cand] = om  # _get_Omega stores omega0 even when rejected
            self.omega_evals += len(cand)
            ok[cand[~(om > prev * 0.8)]] = True
        self._commit_residual(ok, st, k, s_new, hist_slots)
        return ok

    def _trial_omega(self, mask, alpha, s_prev):
        """Omega((1-a) rho + a G) = Omega(rho + a r) for every instance in mask."""
        coefs = np.zeros((self.B, 2))
        coefs[:, 0] = 1.0
        coefs[:, 1] = alpha
        st = self._eval_density(mask, coefs, [self.ring[s_prev], self.rres[s_prev]], L.CLIP_NONE,
                                self.trial, 2, self.ring[s_prev])
        self.omega_evals += int(mask.sum())
        return np.array([self._omega(st[b], b) if mask[b] else np.nan for b in range(self.B)])

    def _ls_omega(self, ls_b, b, i, alpha):
        """Omega(rho + alpha r) of instance b from the line-search sums ls_b
        (alpha = the i-th trial alpha) and the sums of rho itself, in the
        order of _omega (solver.py:103-119)."""
        beta, dr = self.fn.beta, self.dr
        st = self.last_stats[b]
        N = (st[L.STAT_N] + alpha * ls_b[L.LS_SUM_R]) * dr
        G = (ls_b[L.LS_FID + i] * dr) / beta - self.mu[b] * N
        G += (ls_b[L.LS_PHI + i] * dr) / beta
        G += 0.5 * ((st[L.STAT_MFA] + 2 * alpha * ls_b[L.LS_MFA_XR] + alpha * alpha * ls_b[L.LS_MFA_RR]) * dr)
        G += (st[L.STAT_FEXT] + alpha * ls_b[L.LS_SUM_RV]) * dr
        if self.fn.wda is not None:
            G += ls_b[L.LS_WDA + i] * dr
        return G

    def _ls_omega_rows(self, ls, idx, i, alpha):
        """_ls_omega for the instances idx; i (scalar or per-row) selects the trial alpha."""
        beta, dr = self.fn.beta, self.dr
        st = self.last_stats[idx]
        lb = ls[idx]
        rows = np.arange(len(idx))
        i = np.broadcast_to(np.asarray(i), rows.shape)
        N = (st[:, L.STAT_N] + alpha * lb[:, L.LS_SUM_R]) * dr
        G = (lb[rows, L.LS_FID + i] * dr) / beta - self.mu[idx] * N
        G += (lb[rows, L.LS_PHI + i] * dr) / beta
        G += 0.5 * ((st[:, L.STAT_MFA] + 2 * alpha * lb[:, L.LS_MFA_XR] + alpha * alpha * lb[:, L.LS_MFA_RR]) * dr)
        G += (st[:, L.STAT_FEXT] + alpha * lb[:, L.LS_SUM_RV]) * dr
        if self.fn.wda is not None:
            G += lb[rows, L.LS_WDA + i] * dr
        return G

    LS_COEFS = (0.45, 0.9, 0.225)   # trial alphas / alpha_max (solver.py:414-423)

    def _launch_ls(self, mask, s, n3a):
        """Line-search passes for the densities in ring slot s of the instances
        in mask; n3a: device vector of their max n3."""
        self._set_active(mask)
        fn = self.fn
        fn.ls_prepare(self.buf, self.rres[s], self.spec_ring[s], self.wd_ring[s], self.rhat, self.wd_r,
                      self.ls_part, active=self.active)
        fn.ls_omega(self.buf, n3a, self.LS_COEFS, self.ring[s], self.rres[s], self.wd_ring[s], self.wd_r,
                    self.ls_part, self.ls_alpha, active=self.active)
        fn.ls_finalize(self.buf, self.ls_part, self.ls, active=self.active)
        self.kernel_launches += 6

    def _read(self, stats=True, ls=False):
        """Copy the finalized stats and/or the line-search sums to pinned host
        memory and synchronise once."""
        pin = self.pin_read
        if stats:
            pin['stats'].copy_(self.buf.stats, non_blocking=True)
        if ls:
            pin['ls'].copy_(self.ls, non_blocking=True)
            pin['alpha'].copy_(self.ls_alpha, non_blocking=True)
        torch.cuda.current_stream().synchronize()
        if ls:
            return pin['stats'].numpy().copy(), pin['ls'].numpy().copy(), pin['alpha'].numpy().copy()
        return pin['stats'].numpy().copy()

    def _keep_ls(self, mask, s, ls, alpha):
        self.ls_host[mask] = ls[mask]
        self.alpha_host[mask] = alpha[mask]
        self.ls_slot[mask] = s

    def _hybrid_step(self, mask, k, s_prev, s_new):
        """Picard.update_rho_hybrid for the instances in mask (solver.py:403-457).

        alpha_max (from max n3 of G = rho + r) and Omega at the trial alphas
        0.45, 0.9 and 0.225 alpha_max come from one pass over the stored
        weighted densities of rho and r (cmm_ls_*): the trial densities are
        never transformed, and both candidates for the second trial point are
        evaluated before the host chooses between them."""
        B = self.B
        prev = self.omega0.copy()
        fresh = mask & (self.ls_slot != s_prev)  # not computed ahead with the last evaluation
        if fresh.any():
            self._set_params(n3=self.n3max)
            self._launch_ls(fresh, s_prev, self.params[:, 3])
            _, ls_new, al_new = self._read(stats=False, ls=True)
            self._keep_ls(fresh, s_prev, ls_new, al_new)
        ls = self.ls_host
        amax = np.where(mask, self.alpha_host, 0.0)
        aopt = np.zeros(B)
        mn = np.zeros(B)
        mx = np.zeros(B)
        need = mask & ~np.isclose(amax, 0)
        if need.any():
            idx = np.where(need)[0]
            a1 = 0.45 * amax[idx]
            o1 = self._ls_omega_rows(ls, idx, 0, a1)
            first = o1 <= prev[idx]
            a2 = np.where(first, 0.9 * amax[idx], 0.225 * amax[idx])
            o2 = self._ls_omega_rows(ls, idx, np.where(first, 1, 2), a2)
            self.omega_evals += 2 * len(idx)
            cf = parabola3(a1, a2, prev[idx], o1, o2)
            hi = np.maximum(a1, a2)
            aopt[idx], mn[idx], mx[idx] = grid_parabola(cf, hi)
            mn[idx] /= kjmol
            mx[idx] /= kjmol
            self.omega0[idx] = o2
        midx = np.where(mask)[0]
        neg = aopt[midx] <= 0
        spread = (mx[midx] - mn[midx]) > self.thresh
        aopt[midx[neg & ~spread]] = self.alpha_mix * amax[midx[neg & ~spread]]
        for b in midx[neg & spread]:  # SLSQP on full evaluations of the trial density (rare)
            one = np.zeros(B, dtype=bool)
            one[b] = True

            def fun(alpha, b=b, one=one):
                al = np.zeros(B)
                al[b] = float(np.asarray(alpha).ravel()[0])
                o = self._trial_omega(one, al, s_prev)[b]
                self.omega0[b] = o
                return o
            bnd = opt.Bounds(0.01 * amax[b], 0.9 * amax[b])
            aopt[b] = float(opt.minimize(fun, [self.alpha_mix * amax[b]], bounds=bnd, method='SLSQP',
                                         options={'ftol': 1e-8}).x[0])
        small = (aopt[midx] <= 0) | np.isclose(aopt[midx], 0)
        aopt[midx[small]] = self.alpha_mix * amax[midx[small]]
        coefs = np.zeros((B, 2))
        coefs[:, 0] = 1.0
        coefs[:, 1] = aopt * self.cf
        self._set_active(mask)
        self.ls_slot[mask & (self.ls_slot == s_new)] = -1  # slot s_new gets a new density
        self._mix(coefs, [self.ring[s_prev], self.rres[s_prev]], L.CLIP_DENSITY, self.ring[s_prev],
                  self.ring[s_new], spec_out=self.spec_ring[s_new])
        # the next step is a hybrid one for every instance while k + 1 <= 4
        # (Anderson needs curr_step > 4, solver.py:561): its line search ahead
        ahead = mask & ~self.And_true if k + 1 <= 4 else None
        st, hist_slots = self._post_update(mask, k, s_new, None, ahead=ahead)
        self.omega0[midx] = self._omega_rows(st, midx)
        self.omega_evals += len(midx)
        self._commit_residual(mask, st, k, s_new, hist_slots)

    def n3max_of_current(self, b):
        return self.n3max[b]


_STREAMS = {}


def _group_streams(n):
    """n CUDA streams of the current device, the same ones on every call: the
    caching allocator keeps freed blocks per stream, so the workspaces of one
    solve serve the next instead of new device allocations."""
    dev = torch.cuda.current_device()
    pool = _STREAMS.setdefault(dev, [])
    while len(pool) < n:
        pool.append(torch.cuda.Stream(device=dev))
    return pool[:n]


class GroupedSolve(object):
    """A batch of instances solved as G independent groups, each a BatchSolve
    on its own CUDA stream driven by its own host thread.

    The batched loop alternates device work and host decisions (line-search
    fits, Anderson coefficients, convergence tests) that read per-instance
    sums back from the device.  With one group the device idles while the
    host decides; with two or more, one group's kernels run while another
    group's host logic executes (CUDA synchronisation and the ctypes launches
    release the interpreter lock).  Instances are independent, so the
    results equal those of a single BatchSolve over all of them.
    Interface of BatchSolve.solve; per-instance arrays are concatenated.
    """

    def __init__(self, fn, chempots, groups=2, native=True, **kwargs):
        self.mu = np.asarray(chempots, dtype=np.float64).ravel()
        B = len(self.mu)
        G = max(1, min(int(groups), B))
        self.parts = [p for p in np.array_split(np.arange(B), G) if len(p)]
        cls = NativeBatchSolve if native else BatchSolve
        self.solvers = [cls(fn, self.mu[p], group=i, **kwargs) for i, p in enumerate(self.parts)]
        self.B = B
        self.pipeline_events = None

    def solve(self, rho0, host_out=None):
        import threading
        if len(self.parts) == 1:  # one group: the caller's thread and stream
            s = self.solvers[0]
            s.pipeline_events = self.pipeline_events
            self.N_out, self.result, self.conv = s.solve(rho0, host_out=host_out)
            return self.N_out, self.result, self.conv
        cur = torch.cuda.current_stream()
        streams = _group_streams(len(self.parts))
        out = [None] * len(self.parts)
        errors = []

        def run(i):
            p, s, st = self.parts[i], self.solvers[i], streams[i]
            try:
                st.wait_stream(cur)  # rho0 and the functional are ready
                with torch.cuda.stream(st):
                    s.pipeline_events = self.pipeline_events
                    ho = None if host_out is None else host_out[p[0]:p[-1] + 1]
                    out[i] = s.solve(rho0[p[0]:p[-1] + 1], host_out=ho)
            except BaseException as e:  # re-raised on the calling thread
                errors.append(e)

        threads = [threading.Thread(target=run, args=(i,)) for i in range(len(self.parts))]
        for t in threads:
            t.start()
        for t in threads:
            t.join()
        for st in streams:
            cur.wait_stream(st)
        if errors:
            raise errors[0]
        self.result = torch.cat([o[1] for o in out], dim=0)
        self.N_out = np.concatenate([o[0] for o in out])
        self.conv = np.concatenate([o[2] for o in out])
        return self.N_out, self.result, self.conv

    def _cat(self, name):
        return np.concatenate([getattr(s, name) for s in self.solvers])

    @property
    def steps(self):
        return self._cat('steps')

    @property
    def diverged(self):
        return self._cat('diverged')

    @property
    def omega0(self):
        return self._cat('omega0')

    @property
    def kernel_launches(self):
        return sum(s.kernel_launches for s in self.solvers)

    @property
    def omega_evals(self):
        return sum(s.omega_evals for s in self.solvers)


class NativeBatchSolve(BatchSolve):
    """BatchSolve whose hybrid / Anderson loop runs in the library
    (cmm_solve_batched): the same kernels on the same buffers, with the
    per-instance decisions evaluated in C++ between read-backs instead of in
    the interpreter.  The rare SLSQP fallback of the line search is called
    back into Python (scipy, on full evaluations of the trial density).
    Static Picard runs with its decisions on the device and the step
    replayed as a CUDA graph (``device_loop``; False: host decisions after
    every step).  Same results as BatchSolve."""

    device_loop = True

    def solve(self, rho0, cf=None, host_out=None):
        if host_out is not None and (not host_out.is_pinned() or tuple(host_out.shape) != tuple(rho0.shape)):
            raise ValueError("host_out must be a pinned tensor of the shape of rho0")
        import ctypes
        B, fn = self.B, self.fn
        self.initial_density(rho0)
        self.cf = np.ones(B) if cf is None else np.asarray(cf, dtype=float).copy()
        self.result = torch.empty_like(self.rho0)
        self.history = [[] for _ in range(B)]
        self.fallbacks = 0
        method = {'hybrid': L.SOLVE_HYBRID, 'anderson': L.SOLVE_ANDERSON,
                  'hybridanderson': L.SOLVE_HYBRIDANDERSON, 'static': L.SOLVE_STATIC}[self.method]
        crit = {'res': L.CRIT_RES, 'riue': L.CRIT_RIUE, 'der': L.CRIT_DER}
        nc = len(self.criteria)
        opts = L.SolveOpts(method=method, nsteps=self.nsteps, m=self.m, ncrit=nc,
                           alpha_mix=self.alpha_mix, damping=self.damping0, delta=self.delta,
                           damping_max=self.damping_max, damping_min=self.damping_min,
                           damping_up=self.dfac[0], damping_down=self.dfac[1],
                           adaptive_damping=int(bool(self.adaptive)), divergence_guard=int(self.divergence_guard),
                           a_tol=self.tol[0], r_tol=self.tol[1], ls_thresh=self.thresh, kjmol=kjmol,
                           coefs=L.COEF_EXACT if self.anderson_coefs == 'exact' else L.COEF_SLSQP,
                           picard_thr=1e-10 / angstrom ** 3, device_loop=int(bool(self.device_loop)))
        for i, (c, t) in enumerate(zip(self.criteria, self.thresholds)):
            opts.crit[i] = crit[c]
            opts.thr[i] = t
        wda = ctypes.addressof(fn.wda) if fn.wda is not None else None
        desc = L.FunctionalDesc(fn.plan.handle.value, fn.R, fn.beta, fn.lambda3, fn.version, wda,
                                fn.kst.data_ptr(), fn.wtab.data_ptr() if fn.wtab is not None else None,
                                fn.V.data_ptr())
        ws_d = self.__dict__
        stage = self.pin_read.get('stage')
        nstage = int(L.lib().cmm_solve_stage_bytes(B))
        if stage is None or stage.numel() < nstage:
            stage = torch.empty(nstage, dtype=torch.uint8, pin_memory=True)
            self.pin_read['stage'] = stage
        names = ("ring", "rres", "trial", "rho0", "spec_ring", "wd_ring", "wd_r", "rhat", "chat", "chat2", "that",
                 "params", "coef", "active", "ls_part", "ls", "ls_alpha")
        ws = L.SolveWs(**{n: ws_d[n].data_ptr() for n in names if n in ws_d})   # static: no line-search buffers
        ws.result = self.result.data_ptr()
        ws.work, ws.part, ws.stats = self.buf.work.data_ptr(), self.buf.part.data_ptr(), self.buf.stats.data_ptr()
        ws.nslot = self.buf.nslot
        ws.h_stats = self.pin_read['stats'].data_ptr()
        ws.h_ls = self.pin_read['ls'].data_ptr()
        ws.h_alpha = self.pin_read['alpha'].data_ptr()
        ws.h_stage = stage.data_ptr()
        ws.h_result = host_out.data_ptr() if host_out is not None else None
        N = np.full(B, np.nan)
        om = np.full(B, np.nan)
        conv, steps, div, failed = (np.zeros(B, dtype=np.int32) for _ in range(4))
        hist = np.full((B, self.nsteps + 2, 5), np.nan)
        cf_out = np.ones(B)
        arr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
        out = L.SolveOut(N=arr(N), omega=arr(om), converged=arr(conv), steps=arr(steps), diverged=arr(div),
                         failed=arr(failed), history=arr(hist), cf=arr(cf_out))
        if self.pipeline_events is not None:  # CUDA-event times of the full pipeline launches
            plog = np.zeros((4096, 3))
            out.pipe_log, out.pipe_cap = arr(plog), len(plog)
        cb = L.FALLBACK_FN(self._native_fallback)
        mu = np.ascontiguousarray(self.mu, dtype=np.float64)
        fug = np.ascontiguousarray(self.fug, dtype=np.float64)
        cf0 = np.ascontiguousarray(self.cf, dtype=np.float64)
        self._fallback_error = None
        rc = L.lib().cmm_solve_batched(ctypes.byref(desc), ctypes.byref(opts), B, arr(mu), arr(fug), arr(cf0),
                                       ctypes.byref(ws), ctypes.byref(out), cb, None, E._stream())
        if self._fallback_error is not None:
            raise self._fallback_error
        L.check(rc, "cmm_solve_batched")
        self.N_out, self.conv = N, conv.astype(bool)
        self.steps, self.diverged, self.failed = steps.astype(int), div.astype(bool), failed.astype(bool)
        self.omega0 = om
        self.cf = cf_out
        if not self.der_history:
            hist[:, :, 4] = np.nan
        self.kernel_launches += int(out.launches)
        self.omega_evals += int(out.omega_evals)
        if self.pipeline_events is not None:
            for want, nact, ms in plog[:out.pipe_n]:
                self.pipeline_events.append((float(ms), None, int(want), int(nact)))
        steps_max = int(self.steps.max()) if B else 0
        h = hist[:, 1:steps_max + 1]
        keep = ~np.isnan(h[:, :, 0])
        self.history = [list(map(tuple, h[b][keep[b]])) for b in range(B)]
        if self.failed.any():
            raise NoSolutionError("instances %s hit non-finite densities on every retry"
                                  % list(np.where(self.failed)[0]))
        return self.N_out, self.result, self.conv

    def _native_fallback(self, ctx, b, s_prev, amax, alpha_p, omega_p):
        """SLSQP over Omega((1-a) rho + a G) on full evaluations (solver.py:437-447)."""
        try:
            B = self.B
            one = np.zeros(B, dtype=bool)
            one[b] = True
            last = [np.nan]

            def fun(alpha):
                al = np.zeros(B)
                al[b] = float(np.asarray(alpha).ravel()[0])
                o = self._trial_omega(one, al, s_prev)[b]
                last[0] = o
                return o
            bnd = opt.Bounds(0.01 * amax, 0.9 * amax)
            res = opt.minimize(fun, [self.alpha_mix * amax], bounds=bnd, method='SLSQP', options={'ftol': 1e-8})
            alpha_p[0] = float(res.x[0])
            omega_p[0] = float(last[0])
            self.fallbacks += 1
            return 0
        except BaseException as e:  # reported after the native call returns
            self._fallback_error = e
            return 1
