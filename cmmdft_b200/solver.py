"""Fixed-point solvers with the reference's interface (cmmdft/solver.py:18-604).

Solver / Picard / Anderson / QuasiNewton / Fire keep the reference's
constructor arguments and ``solve(chempot, rho, log_level) -> (N, rho,
converged)``.  Each call runs a batch of one through the native batched
driver (``quasinewton.QuasiNewtonSolve`` for QuasiNewton, ``fire.FireSolve``
for Fire; all field work on the GPU); the
batched isotherm entry point is ``isotherm.solve_isotherm`` /
``Program.solve_isotherm``.
"""
import numpy as np

from . import batch as BT
from .batch import NoSolutionError

__all__ = ['Solver', 'Picard', 'Anderson', 'QuasiNewton', 'Fire', 'NoSolutionError']


class Solver(object):
    name = 'SOLVER'

    def __init__(self, program, nsteps=500, threshold=1e-6, criterion='RIUE', a_tol=1e-6, r_tol=1e-4,
                 min_iter=1, track_history=False):
        self.grid = program.grid
        self.fener = program.fener
        self.nsteps = nsteps
        if isinstance(criterion, list):
            for c in criterion:
                assert c.lower() in ['riue', 'res', 'der'], \
                    'Criterion must be either RIUE (relative integrated unsigned error), RES (Residual error) or DER (Derivative error)'
            self.criterion = [c.lower() for c in criterion]
            if isinstance(threshold, list):
                assert len(criterion) == len(threshold), \
                    'If multiple criterions are given, the same amount of thresholds should be given'
                self.threshold = threshold
            else:
                self.threshold = [threshold] * len(criterion)
        else:
            assert criterion.lower() in ['riue', 'res', 'der'], \
                'Criterion must be either RIUE (relative integrated unsigned error), RES (Residual error) or DER (Derivative error)'
            if criterion.lower() == 'der':
                threshold = 1
            self.criterion = [criterion.lower()]
            self.threshold = [threshold]
        self.a_tol, self.r_tol, self.min_iter = a_tol, r_tol, min_iter
        self.curr_step = 0
        self.correction_factor = 1
        self.track_history = track_history
        self.history_header = ("Loading [au], Grand potential [Eh], Norm of residuals, RIUE, "
                               "Norm of derivative, Time per step [s], Cumulative time [s]")
        self.history = np.zeros((nsteps + 1, 7))
        self.omega0 = None
        self._last = None

    def _method(self):
        raise NotImplementedError

    def _options(self):
        return {}

    def solve(self, chempot, rho, log_level=2):
        """Converge one density (B = 1) on the GPU; returns (N, rho, converged)."""
        import torch
        fn = self.fener.device()
        s = BT.NativeBatchSolve(fn, [chempot], method=self._method(), nsteps=self.nsteps, threshold=self.threshold,
                                criterion=self.criterion, a_tol=self.a_tol, r_tol=self.r_tol,
                                track_history=self.track_history, **self._options())
        r0 = rho if hasattr(rho, 'detach') else torch.as_tensor(np.ascontiguousarray(rho, dtype=np.float64))
        r0 = r0.to('cuda', dtype=torch.float64).reshape((1,) + tuple(self.grid.npoints))
        N, rr, conv = s.solve(r0)
        self._last = s
        self.curr_step = int(s.steps[0])
        self.omega0 = float(s.omega0[0]) if hasattr(s, 'omega0') else None
        if self.track_history:
            self.history = self._history(s.history[0], float(r0.sum().item()) * self.grid.dr)
        return float(N[0]), rr[0].cpu().numpy(), bool(conv[0])


    def _history(self, rows, N0):
        """The reference's history array (solver.py:270-279, 208-222) from the
        driver's per-step rows (N, RES, RIUE, Omega, DER): columns loading,
        grand potential, residual norm (RES, or |G - rho| / N / sqrt(Npts)
        when RES is not a criterion), RIUE, derivative norm (NaN when 'der'
        is a criterion, whose tolerance-weighted sum the kernels then
        compute), time per step and cumulative time (not timed: NaN).  Row 0
        holds the loading of the initial density.  Omega is the grand
        potential of the step's new density for the hybrid and Anderson
        methods, the initial one for static Picard (the reference's omega0
        without energy tracking)."""
        h = np.array(rows, dtype=float).reshape(-1, 5)
        out = np.full((len(h) + 1, 7), np.nan)
        out[0, 0] = N0
        if len(h):
            N, res, riue, om, der = h.T
            out[1:, 0] = N
            out[1:, 1] = om
            with np.errstate(invalid='ignore', divide='ignore'):
                out[1:, 2] = res if 'res' in self.criterion else res / np.sqrt(N)
            out[1:, 3] = riue
            out[1:, 4] = der
        return out


class Picard(Solver):
    name = 'PICARD'

    def __init__(self, program, nsteps=500, alpha_mix=0.1, method='hybrid', **kwargs):
        Solver.__init__(self, program, nsteps, **kwargs)
        self.alpha_mix = alpha_mix
        assert method in ('hybrid', 'static'), method
        self.method = method

    def _method(self):
        return self.method

    def _options(self):
        return dict(alpha_mix=self.alpha_mix)


class Anderson(Picard):
    """Anderson and hybrid-Anderson mixing (https://doi.org/10.1063/5.0067172)."""
    name = 'ANDERSON'

    def __init__(self, program, nsteps=500, method='hybridanderson', m=5, damping=0.3, delta=0.2,
                 damping_max=0.8, damping_min=0.01, adaptive_damping=True, damping_factors=(1.5, 0.5), **kwargs):
        Solver.__init__(self, program, nsteps, **{k: v for k, v in kwargs.items() if k != 'alpha_mix'})
        self.alpha_mix = kwargs.get('alpha_mix', 0.1)
        assert method in ('hybridanderson', 'anderson'), method
        self.Anderson_method = method
        self.m, self.damping, self.delta = m, damping, delta
        self.damping_max, self.damping_min = damping_max, damping_min
        self.adaptive_damping, self.damping_factors = adaptive_damping, damping_factors

    def _method(self):
        return self.Anderson_method

    def _options(self):
        return dict(alpha_mix=self.alpha_mix, m=self.m, damping=self.damping, delta=self.delta,
                    damping_max=self.damping_max, damping_min=self.damping_min,
                    adaptive_damping=self.adaptive_damping, damping_factors=self.damping_factors)


class QuasiNewton(Picard):
    """Limited-memory quasi-Newton steps on Omega between hybrid Picard steps
    (cmmdft/solver.py:701-1053), through ``quasinewton.QuasiNewtonSolve``."""
    name = 'QUASI_NEWTON'

    def __init__(self, program, nsteps=500, m=10, method='bfgs', hybrid=True, delta=0.5, alpha_init=0.05, c1=1e-4,
                 c2=0.9, line_search='backtracking', n_line_search=10, trust_radius=1, verbose=True, **kwargs):
        alpha_mix = kwargs.pop('alpha_mix', 0.1)
        Solver.__init__(self, program, nsteps, **kwargs)
        self.alpha_mix = alpha_mix
        assert method.lower() in ('bfgs', 'broyden', 'cg'), \
            "Method %s not recognized. Choose from 'bfgs', 'broyden' or 'cg'." % method
        assert line_search in ('backtracking', 'quadratic', 'none'), \
            "Line search method %s not recognized." % line_search
        self.m, self.QN_method, self.hybrid, self.delta = m, method.lower(), hybrid, delta
        self.alpha_init, self.c1, self.c2 = alpha_init, c1, c2
        self.line_search, self.n_line_search, self.trust_radius = line_search, n_line_search, trust_radius
        self.verbose = verbose

    def solve(self, chempot, rho, log_level=2):
        from .quasinewton import QuasiNewtonSolve
        s = QuasiNewtonSolve(self.fener.device(), nsteps=self.nsteps, m=self.m, method=self.QN_method,
                             hybrid=self.hybrid, delta=self.delta, alpha_init=self.alpha_init, c1=self.c1,
                             c2=self.c2, line_search=self.line_search, n_line_search=self.n_line_search,
                             trust_radius=self.trust_radius, threshold=self.threshold, criterion=self.criterion,
                             a_tol=self.a_tol, r_tol=self.r_tol, alpha_mix=self.alpha_mix)
        N, r, conv = s.solve(chempot, rho)
        self._last = s
        self.curr_step = int(s.steps)
        self.omega0 = float(s.omega0)
        return float(N), r.cpu().numpy(), bool(conv)


class Fire(Solver):
    """FIRE / ABC-FIRE relaxation of the log-density (cmmdft/solver.py:606-698),
    through ``fire.FireSolve``.  As in the reference the update acts on the
    points of ``self.mask``, which the caller sets (a boolean field of the
    grid's shape selecting points with rho > 0) before solving; without it
    solve raises AttributeError, as the reference's update does."""
    name = 'FIRE'

    def __init__(self, program, nsteps=500, method='abc-fire', alpha=0.2, dt=0.02, **kwargs):
        Solver.__init__(self, program, nsteps, **kwargs)
        self.method = method
        self.alpha0 = self.alpha = alpha
        self.dt0 = self.dt = dt
        self._solver = None

    def solve(self, chempot, rho, log_level=2):
        from .fire import FireSolve
        mask = self.mask   # AttributeError when unset, as Fire.update_rho raises
        if self._solver is None or self._solver.fn is not self.fener.device():
            self._solver = FireSolve(self.fener.device(), mask, nsteps=self.nsteps, method=self.method,
                                     alpha=self.alpha0, dt=self.dt0, threshold=self.threshold,
                                     criterion=self.criterion, a_tol=self.a_tol, r_tol=self.r_tol)
        else:
            self._solver.set_mask(mask)
        s = self._solver
        N, r, conv = s.solve(chempot, rho)
        self.curr_step = int(s.steps)
        self.omega0 = float(s.omega0)
        self.dt, self.alpha, self.Npos, self.Nneg = s.dt, s.alpha, s.Npos, s.Nneg
        return float(N), r.cpu().numpy(), bool(conv)
