"""QuasiNewton (cmmdft/solver.py:701-1212) on the device pipeline against the
reference's own runs (tests/golden/qn32.npz, written by make_golden.py --qn):
the 32^3 case at 1 bar, RES < 1e-8 from Ninit = rho_bulk, for the L-BFGS,
Broyden and CG-descent directions with the backtracking line search and
L-BFGS with the quadratic and fixed-step searches.  At this tolerance the
result depends on the whole trajectory: the same number of steps and N
within 1e-10 are required (1e-8 for the quadratic search, see below)."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from cmmdft_b200 import workload as W
from cmmdft_b200.hosts import cubic_host_276, methane_guest_params
from cmmdft_b200.quasinewton import QuasiNewtonSolve
from tests._common import scalar_rel

CASES = [('bfgs', 'backtracking'), ('broyden', 'backtracking'), ('cg', 'backtracking'), ('bfgs', 'quadratic'),
         ('bfgs', 'none')]


@pytest.fixture(scope="module")
def qn32():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    path = os.path.join(os.path.dirname(__file__), "golden", "qn32.npz")
    return dict(np.load(path))


@pytest.fixture(scope="module")
def fn32q(qn32):
    return W.build_functional(cubic_host_276(0), (32, 32, 32), 300.0, methane_guest_params())


@pytest.mark.parametrize("method,search", CASES)
def test_quasinewton_matches_reference(qn32, fn32q, method, search):
    mu = float(qn32["mu"])
    rho0 = W.initial_density(fn32q, [mu], ninit=[float(qn32["rho_bulk"])])[0]
    s = QuasiNewtonSolve(fn32q, nsteps=300, method=method, line_search=search, threshold=1e-8, criterion='res')
    N, rho, conv = s.solve(mu, rho0)
    tag = '%s_%s' % (method, search)
    assert conv and bool(qn32[tag + '_conv'])
    assert s.steps == int(qn32[tag + '_steps']), (s.steps, int(qn32[tag + '_steps']))
    # the quadratic search's step -s a1^2 / (2 (f - f0 - s a1)) divides by a
    # difference of nearly equal grand potentials: last-bit differences of
    # Omega move its N by ~7e-10 at this tolerance (1e-8 allowed there)
    tol = 1e-8 if search == 'quadratic' else 1e-10
    assert scalar_rel(N, float(qn32[tag + '_N'])) < tol, (N, float(qn32[tag + '_N']))
    assert scalar_rel(s.omega0, float(qn32[tag + '_omega'])) < tol
