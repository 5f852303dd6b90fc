"""Public batched entry point: a whole isotherm (or any set of chemical
potentials) on one host in one batched solve.

The reference solves an isotherm as a Python loop of Program.solve calls, one
per pressure (examples/methane_ZIF8.ipynb cells 7-11, cmmdft/program.py:
331-404).  ``solve_isotherm`` takes host arrays on the CPU, builds the
external potential and MFA kernel on the GPU, solves every point of the
isotherm as one batch, and returns loadings (and densities) on the CPU.
"""
import numpy as np
import torch

from . import batch as BT
from . import workload as W
from .units import angstrom, kjmol

__all__ = ['solve_isotherm', 'excess_loading']


def solve_isotherm(host, pressures, temperature, guest, npoints, method='hybridanderson', threshold=1e-8,
                   criterion='res', nsteps=500, start='bulk', version='WBII', tailcorrections=False,
                   return_density=True, fn=None, m=5, alpha_mix=0.1, divergence_guard=True, groups=1, native=True,
                   anderson_coefs='slsqp'):
    """Solve the adsorption isotherm of a spherical LJ guest in ``host``.

    pressures: array in atomic units (e.g. ``np.logspace(-3, 2, 24) * bar``).
    start: 'bulk' -> rho0 = rho_bulk exp(-max(V,0)/kT) (Ninit=rho_bulk, the
    reference notebook's choice); 'ideal' -> exp(beta (mu - V)) / Lambda^3.
    groups: independent instance groups solved on concurrent streams (host
    decisions of one group overlap the device work of another).
    native: run the batched loop in the library (cmm_solve_batched); False
    runs the Python driver (the same kernels and decisions).
    anderson_coefs: 'slsqp' takes the reference's SLSQP coefficients (same
    trajectory and result as the reference at any tolerance); 'exact' the
    exact simplex minimiser (fewer steps, a different point within the
    tolerance).
    Returns a dict with mu, rho_bulk, N (absolute loading per cell),
    converged, steps, omega and (optionally) the densities [B, N1, N2, N3].
    """
    if fn is None:
        fn = W.build_functional(host, npoints, temperature, guest, version=version,
                                tailcorrections=tailcorrections)
    mus, bulks = W.isotherm_inputs(pressures, temperature, guest)
    rho0 = W.initial_density(fn, mus, ninit=bulks if start == 'bulk' else None)
    s = BT.GroupedSolve(fn, mus, groups=groups, native=native, method=method, nsteps=nsteps, threshold=threshold,
                        criterion=criterion, m=m, alpha_mix=alpha_mix, divergence_guard=divergence_guard,
                        anderson_coefs=anderson_coefs)
    # densities land in pinned host memory while the rest of the batch iterates
    host = torch.empty(tuple(rho0.shape), dtype=torch.float64, pin_memory=True) if return_density else None
    N, rho, conv = s.solve(rho0, host_out=host)
    out = dict(mu=mus, rho_bulk=bulks, N=np.array(N), converged=np.array(conv), steps=s.steps.copy(),
               diverged=s.diverged.copy(),
               solver=s, functional=fn)
    if return_density:
        out['rho'] = host.numpy()
    return out


def excess_loading(N, rho_bulk, he_fraction, cell_volume):
    """N_ex = N - rho_bulk * He_frac * V_cell (Calculator.return_loading, calculator.py:114-138)."""
    return np.asarray(N) - np.asarray(rho_bulk) * he_fraction * cell_volume
