"""Bulk equations of state (host-side scalars).

Restates cmmdft/eos.py: the EquationOfState interface (:22-223), SumOfEOS
(:226-265), the modified Benedict-Webb-Rubin LJ equation of Johnson, Zollweg
and Gubbins (Mol. Phys. 78, 591 (1993), regression parameters of their
Table 10; cmmdft/eos.py:295-469), Carnahan-Starling (:471-520) and the
mean-field EOS (:523-546).  These are scalar/1-D numpy evaluations that set
up mu(P) and bulk densities; the grid solve never calls them per point.
"""
import numpy as np

from .units import angstrom, boltzmann, planck

__all__ = ['EquationOfState', 'SumOfEOS', 'ModifiedBenedictWebbRubinEOS', 'CarnahanStarlingEOS', 'MFAEOS']


_scalar_powers = [False]


def _ipow(x, k):
    """x ** k for an integer k.  While brentq lanes are evaluated, each
    element is raised as a Python float (C pow), which rounds differently
    from numpy's array power in the last bit: the lanes then reproduce the
    scalar evaluations scipy's brentq makes one root at a time."""
    if _scalar_powers[0] and isinstance(x, np.ndarray):
        return np.array([v ** k for v in x.tolist()])
    return x ** k


def brentq_lanes(f, a, b, xtol=2e-12, rtol=4 * np.finfo(float).eps, maxiter=100):
    """Brent's root finder (R. P. Brent, Algorithms for Minimization without
    Derivatives, 1973, ch. 4) run on many brackets at once.

    Every lane takes the steps scipy.optimize.brentq (default tolerances)
    takes on its own bracket: the same bracket bookkeeping, inverse
    quadratic / secant trial step, acceptance test, bisection fallback and
    minimum step of (xtol + rtol |x|) / 2.  ``f(x, idx)`` evaluates the
    function of lanes ``idx`` at ``x`` (vectorised).  Returns the roots.
    """
    _scalar_powers[0] = True
    try:
        return _brent_loop(f, a, b, xtol, rtol, maxiter)
    finally:
        _scalar_powers[0] = False


def _brent_loop(f, a, b, xtol, rtol, maxiter):
    xpre = np.array(a, dtype=float)
    xcur = np.array(b, dtype=float)
    n = xpre.size
    fpre = f(xpre, np.arange(n))
    fcur = f(xcur, np.arange(n))
    root = np.full(n, np.nan)
    done = np.zeros(n, dtype=bool)
    if np.any((fpre * fcur) > 0):
        raise ValueError("f(a) and f(b) must have different signs")
    z = fpre == 0
    root[z], done[z] = xpre[z], True
    z = (fcur == 0) & ~done
    root[z], done[z] = xcur[z], True
    xblk = np.zeros(n)
    fblk = np.zeros(n)
    spre = np.zeros(n)
    scur = np.zeros(n)
    for _ in range(maxiter):
        live = np.nonzero(~done)[0]
        if live.size == 0:
            break
        xp, xc, xb = xpre[live], xcur[live], xblk[live]
        fp, fc, fb = fpre[live], fcur[live], fblk[live]
        sp, sc = spre[live], scur[live]
        # a sign change between pre and cur: the bracket is [pre, cur]
        m = (fp * fc) < 0
        xb = np.where(m, xp, xb)
        fb = np.where(m, fp, fb)
        sp = np.where(m, xc - xp, sp)
        sc = np.where(m, xc - xp, sc)
        # keep the best estimate in cur
        sw = np.abs(fb) < np.abs(fc)
        xp = np.where(sw, xc, xp)
        xc, xb = np.where(sw, xb, xc), np.where(sw, xp, xb)
        fp = np.where(sw, fc, fp)
        fc, fb = np.where(sw, fb, fc), np.where(sw, fp, fb)
        delta = (xtol + rtol * np.abs(xc)) / 2
        sbis = (xb - xc) / 2
        fin = (fc == 0) | (np.abs(sbis) < delta)
        root[live[fin]] = xc[fin]
        done[live[fin]] = True
        # trial step: secant when pre and blk coincide, else inverse quadratic
        tryit = ~fin & (np.abs(sp) > delta) & (np.abs(fc) < np.abs(fp))
        with np.errstate(divide='ignore', invalid='ignore'):
            stry_s = -fc * (xc - xp) / (fc - fp)
            dpre = (fp - fc) / (xp - xc)
            dblk = (fb - fc) / (xb - xc)
            stry_q = -fc * (fb * dblk - fp * dpre) / (dblk * dpre * (fb - fp))
        stry = np.where(xp == xb, stry_s, stry_q)
        good = tryit & (2 * np.abs(stry) < np.minimum(np.abs(sp), 3 * np.abs(sbis) - delta))
        sp_new = np.where(good, sc, sbis)
        sc_new = np.where(good, stry, sbis)
        step = np.where(np.abs(sc_new) > delta, sc_new, np.where(sbis > 0, delta, -delta))
        act = ~fin
        li = live[act]
        xpre[li], fpre[li] = xc[act], fc[act]
        xblk[li], fblk[li] = xb[act], fb[act]
        spre[li], scur[li] = sp_new[act], sc_new[act]
        xcur[li] = xc[act] + step[act]
        if li.size:
            fcur[li] = f(xcur[li], li)
    live = ~done
    root[live] = xcur[live]   # maxiter reached: the last iterate, as brentq returns it
    return root


class EquationOfState(object):
    def __init__(self, mass):
        self.mass = mass
        self.temperature = None

    def set_temperature(self, temperature):
        self.temperature = temperature
        self.wvl = planck / np.sqrt(2 * np.pi * self.mass * boltzmann * temperature)

    def excess_free_energy_particle(self, rho):
        raise NotImplementedError

    def derivative_excess_free_energy_particle(self, rho):
        raise NotImplementedError

    def excess_free_energy_volume(self, rho):
        return rho * self.excess_free_energy_particle(rho)

    def derivative_excess_free_energy_volume(self, rho):
        v = rho * self.derivative_excess_free_energy_particle(rho)
        v += self.excess_free_energy_particle(rho)
        return v

    def compute_chempot(self, rho):
        kT = boltzmann * self.temperature
        return kT * np.log(self.wvl ** 3 * rho) + self.derivative_excess_free_energy_volume(rho)

    def compute_pressure(self, rho):
        kT = boltzmann * self.temperature
        return kT * rho + rho ** 2 * self.derivative_excess_free_energy_particle(rho)

    def get_rough_density_grid(self, npoints):
        return np.logspace(-10, 0, npoints) / angstrom ** 3

    def _brackets(self, values, grid_values, grid):
        """Intervals [grid[j-1], grid[j]] with grid_values[j-1] <= v <= grid_values[j],
        in increasing j (the scan of eos.py:101-108 / 137-144, vectorised)."""
        out = []
        lo, hi = grid_values[:-1], grid_values[1:]
        for v in values:
            js = np.nonzero((lo <= v) & (v <= hi))[0] + 1
            out.append([(grid[j - 1], grid[j]) for j in js])
        return out

    def _solve_all(self, targets, func, grid, ncol):
        """Every root of func(rho) = target in each bracketing interval of the
        rough grid, sorted per target (the scan and brentq loop of
        eos.py:85-157); the brackets of all targets are solved together by
        brentq_lanes."""
        targets = np.asarray(targets, dtype=float).ravel()
        brackets = self._brackets(targets, func(grid), grid)
        owner = np.array([i for i, iv in enumerate(brackets) for _ in iv], dtype=int)
        out = np.zeros([len(targets), ncol]) * np.nan
        if owner.size == 0:
            return out
        lo = np.array([a for iv in brackets for a, _ in iv])
        hi = np.array([b for iv in brackets for _, b in iv])
        tg = targets[owner]
        roots = brentq_lanes(lambda r, idx: func(r) - tg[idx], lo, hi)
        for i in range(len(targets)):
            sols = sorted(roots[owner == i])
            if len(sols) > 3:
                raise ValueError('more than 3 density branches')
            out[i, :len(sols)] = sols
        return out

    def solve_densities_from_chempots(self, chempots, n_rough_gridpoints=1000):
        """All roots rho of mu(rho) = mu per chempot (<= 2 branches kept), eos.py:85-119."""
        kT = boltzmann * self.temperature
        func = lambda r: kT * np.log(self.wvl ** 3 * r) + self.excess_free_energy_particle(r) + \
            r * self.derivative_excess_free_energy_particle(r)
        return self._solve_all(chempots, func, self.get_rough_density_grid(n_rough_gridpoints), 2)

    def solve_densities_from_pressures(self, pressures, n_rough_gridpoints=10000):
        """All roots rho of p(rho) = p, eos.py:121-157."""
        kT = boltzmann * self.temperature
        func = lambda r: kT * r + _ipow(r, 2) * self.derivative_excess_free_energy_particle(r)
        return self._solve_all(pressures, func, self.get_rough_density_grid(n_rough_gridpoints), 3)

    def calculate_pressure(self, temp, chempot):
        """Pressure of the lowest-density branch at a chemical potential (eos.py:201-207)."""
        self.set_temperature(temp)
        rho = self.solve_densities_from_chempots([chempot])[0][0]
        return self.compute_pressure(rho)

    def calculate_mu(self, temp, pressure):
        """Chemical potential of the lowest-density branch at (T, P), eos.py:209-215.
        ``pressure`` may be an array: one chemical potential per pressure."""
        self.set_temperature(temp)
        rho = self.solve_densities_from_pressures(np.atleast_1d(pressure))[:, 0]
        mu = self.compute_chempot(rho)
        return mu if np.ndim(pressure) else float(mu[0])

    def bulk_density(self, temp, chempot):
        """Lowest density branch at (T, mu) (Calculator.return_loading, calculator.py:129-131).
        ``chempot`` may be an array: one density per chemical potential."""
        self.set_temperature(temp)
        rho = np.nanmin(self.solve_densities_from_chempots(np.atleast_1d(chempot)), axis=1)
        return rho if np.ndim(chempot) else float(rho[0])


class SumOfEOS(EquationOfState):
    def __init__(self, mass, list_eos, factors=None):
        EquationOfState.__init__(self, mass)
        self.list_eos = list(list_eos)
        self.factors = [1.0] * len(self.list_eos) if factors is None else list(factors)

    def set_temperature(self, temperature):
        for e in self.list_eos:
            e.set_temperature(temperature)
        EquationOfState.set_temperature(self, temperature)

    def _sum(self, name, rho):
        r = rho * 0.0
        for e, f in zip(self.list_eos, self.factors):
            r += f * getattr(e, name)(rho)
        return r

    def excess_free_energy_particle(self, rho):
        return self._sum('excess_free_energy_particle', rho)

    def excess_free_energy_volume(self, rho):
        return self._sum('excess_free_energy_volume', rho)

    def derivative_excess_free_energy_particle(self, rho):
        return self._sum('derivative_excess_free_energy_particle', rho)

    def derivative_excess_free_energy_volume(self, rho):
        return self._sum('derivative_excess_free_energy_volume', rho)


# Johnson-Zollweg-Gubbins (1993) Table 10 regression parameters x1..x32.
_MBWR_X = (0.8623085097507421, 2.976218765822098, -8.402230115796038, 0.1054136629203555,
           -0.8564583828174598, 1.582759470107601, 0.7639421948305453, 1.753173414312048,
           2.798291772190376e+3, -4.8394220260857657e-2, 0.9963265197721935, -3.698000291272493e+1,
           2.084012299434647e+1, 8.305402124717285e+1, -9.574799715203068e+2, -1.477746229234994e+2,
           6.398607852471505e+1, 1.603993673294834e+1, 6.805916615864377e+1, -2.791293578795945e+3,
           -6.245128304568454, -8.116836104958410e+3, 1.488735559561229e+1, -1.059346754655084e+4,
           -1.131607632802822e+2, -8.867771540418822e+3, -3.986982844450543e+1, -4.689270299917261e+3,
           2.593535277438717e+2, -2.694523589434903e+3, -7.218487631550215e+2, 1.721802063863269e+2)


class ModifiedBenedictWebbRubinEOS(EquationOfState):
    name = 'MBWR'
    gamma = 3.0

    def __init__(self, mass, sigma, epsilon):
        EquationOfState.__init__(self, mass)
        self.sigma, self.epsilon = sigma, epsilon

    def set_temperature(self, temperature):
        EquationOfState.set_temperature(self, temperature)
        x = (None,) + _MBWR_X
        T = boltzmann * temperature / self.epsilon
        self.a = [x[1] * T + x[2] * np.sqrt(T) + x[3] + x[4] / T + x[5] / T ** 2,
                  x[6] * T + x[7] + x[8] / T + x[9] / T ** 2,
                  x[10] * T + x[11] + x[12] / T,
                  x[13],
                  x[14] / T + x[15] / T ** 2,
                  x[16] / T,
                  x[17] / T + x[18] / T ** 2,
                  x[19] / T ** 2]
        self.b = [x[20] / T ** 2 + x[21] / T ** 3,
                  x[22] / T ** 2 + x[23] / T ** 4,
                  x[24] / T ** 2 + x[25] / T ** 3,
                  x[26] / T ** 2 + x[27] / T ** 4,
                  x[28] / T ** 2 + x[29] / T ** 3,
                  x[30] / T ** 2 + x[31] / T ** 3 + x[32] / T ** 4]

    def _G(self, rho):
        rr = rho * self.sigma ** 3
        F = np.exp(-self.gamma * _ipow(rr, 2))
        ig = 1.0 / (2 * self.gamma)
        G = [ig * (1 - F)]
        for n in range(2, 7):
            G.append(-ig * (F * _ipow(rr, 2 * (n - 1)) - 2 * (n - 1) * G[-1]))
        return G

    def excess_free_energy_particle(self, rho):
        A = 0.0
        rr = rho * self.sigma ** 3
        for i, ai in enumerate(self.a):
            A += ai / (i + 1) * _ipow(rr, i + 1)
        for bi, Gi in zip(self.b, self._G(rho)):
            A += bi * Gi
        return A * self.epsilon

    def derivative_excess_free_energy_particle(self, rho):
        dA = 0.0
        rr = rho * self.sigma ** 3
        for i, ai in enumerate(self.a):
            dA += ai * _ipow(rr, i) * self.sigma ** 3
        F = np.exp(-self.gamma * _ipow(rr, 2))
        for t, bi in enumerate(self.b):
            dA += bi * self.sigma ** 3 * _ipow(rr, 2 * t + 1) * F
        return dA * self.epsilon

    def get_rough_density_grid(self, npoints):
        return np.logspace(-10, 0, npoints) * 1.5 / self.sigma ** 3


class CarnahanStarlingEOS(EquationOfState):
    name = 'CS'

    def __init__(self, mass, Rhs):
        EquationOfState.__init__(self, mass)
        self.R = float(Rhs)
        self.eta = 4 * np.pi * self.R ** 3 / 3

    def excess_free_energy_particle(self, rho):
        kT = boltzmann * self.temperature
        return kT * (4 * self.eta * rho - 3 * _ipow(self.eta * rho, 2)) / _ipow(1 - self.eta * rho, 2)

    def derivative_excess_free_energy_particle(self, rho):
        kT = boltzmann * self.temperature
        return 2 * kT * self.eta * (2 - self.eta * rho) / _ipow(1 - self.eta * rho, 3)


class MFAEOS(EquationOfState):
    name = 'MFA'

    def __init__(self, mass, sigma=None, epsilon=None, a=None):
        EquationOfState.__init__(self, mass)
        self.a = a if a is not None else -16 / 9 * np.pi * epsilon * sigma ** 3

    def excess_free_energy_particle(self, rho):
        return self.a * rho

    def derivative_excess_free_energy_particle(self, rho):
        return self.a + 0 * rho
