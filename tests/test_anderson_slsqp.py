"""Anderson mixing coefficients: cmm_anderson_slsqp against scipy's SLSQP.

The reference takes its Anderson coefficients from
``scipy.optimize.minimize(sum_res, full(mk, 1/mk), method='SLSQP', tol=1e-10,
bounds=Bounds(0, 1), constraints=LinearConstraint(ones(mk), 1, 1)).x``
(cmmdft/solver.py:585-591).  cmm_anderson_slsqp restates that method on the
host from the Gram matrix of the residuals.  These tests run on the CPU: the
routine is host code in the library, and scipy is the reference's own
dependency.
"""
import numpy as np
import pytest
import scipy.optimize as opt

from cmmdft_b200.batch import anderson_slsqp
from oracle import cmm_oracle as O
from tests._common import oracle_case, scalar_rel, relerr


def scipy_coefficients(R):
    """solver.py:585-591 verbatim in behaviour: the objective on the residual vectors."""
    mk = len(R)

    def sum_res(a):
        return np.linalg.norm(np.einsum('i,ij->j', a, R))
    res = opt.minimize(sum_res, np.full(mk, 1 / mk), method='SLSQP', tol=1e-10, bounds=opt.Bounds(0, 1),
                       constraints=opt.LinearConstraint(np.ones(mk), 1, 1))
    return res.x, res.status, res.nit


def residual_history(rng, mk, npts=300):
    """Residuals that share a dominant direction, as a fixed-point history does."""
    scale = 10.0 ** rng.uniform(-10, 0)
    base = rng.normal(size=npts)
    return np.array([rng.uniform(0.2, 3) * base + rng.uniform(0.01, 1) * rng.normal(size=npts)
                     for _ in range(mk)]) * scale


# Measured over 1000 such problems: exit mode and iteration count always equal,
# coefficients equal to the last bit in most cases and within 5e-7 otherwise
# (rounding of the QP subproblem, amplified by the finite-difference gradient).
COEF_TOL = 2e-6


@pytest.mark.parametrize("seed", [0, 1, 2, 3])
def test_matches_scipy_on_residual_histories(seed):
    rng = np.random.default_rng(seed)
    for _ in range(100):
        R = residual_history(rng, int(rng.integers(1, 7)))
        x_ref, mode_ref, nit_ref = scipy_coefficients(R)
        x, mode, nit = anderson_slsqp(R @ R.T)
        assert mode == mode_ref and nit == nit_ref
        assert np.max(np.abs(x - x_ref)) < COEF_TOL


def test_edge_cases():
    rng = np.random.default_rng(7)
    base = rng.normal(size=200)
    cases = {
        "single residual": base[None] * 1e-3,
        "identical residuals": np.array([base, base, base]) * 1e-4,
        "newest much smaller (vertex optimum)": np.array([3 * base, 2 * base, 1e-3 * base + 1e-6 * rng.normal(size=200)]),
        "orthogonal residuals": np.eye(4, 200) * np.array([[1.0], [2.0], [0.5], [4.0]]),
        "tiny residuals (first-step exit)": np.array([base, 0.9 * base + 0.01 * rng.normal(size=200)]) * 1e-12,
        "zero residuals": np.zeros((3, 200)),
    }
    for name, R in cases.items():
        x_ref, mode_ref, nit_ref = scipy_coefficients(R)
        x, mode, nit = anderson_slsqp(R @ R.T)
        assert (mode, nit) == (mode_ref, nit_ref), name
        assert np.max(np.abs(x - x_ref)) < COEF_TOL, name


def test_rejects_unsupported_size():
    with pytest.raises(Exception):
        anderson_slsqp(np.eye(9))


def test_oracle_trajectory_with_native_coefficients(golden32):
    """The oracle's hybrid Anderson at the reference's loose tolerance (RES <
    1e-8, where the trajectory depends on every SLSQP iterate) takes the same
    steps and reaches the same loading when its SLSQP call is replaced by
    cmm_anderson_slsqp on the Gram matrix."""
    grid, fe = oracle_case(32)
    mu = float(golden32["mu"])
    runs = []
    for native in (False, True):
        s = O.Anderson(fe, nsteps=200, m=5, criterion="res", threshold=1e-8)
        if native:
            s.anderson_coefficients = lambda R: anderson_slsqp(R @ R.T)[0]
        N, rho, conv = s.solve(mu, golden32["rho_a"].copy())
        assert conv
        runs.append((s.curr_step, N, rho))
    assert runs[0][0] == runs[1][0]
    assert scalar_rel(runs[0][1], runs[1][1]) < 1e-10
    assert relerr(runs[0][2], runs[1][2]) < 1e-9
