"""Program orchestration with the reference's interface (cmmdft/program.py:21-405).

Keeps the work-directory layout and the ``rho_{mu}kJmol_{T}K.npy`` density
cache of the reference, so existing work directories are reused, and adds
``solve_isotherm`` for batched solves of many chemical potentials.
"""
import os
from pathlib import Path

import numpy as np

from .functionals import FreeEnergy
from .solver import Solver, NoSolutionError
from .system import System, Grid
from .tools import get_file_suffix
from .units import angstrom, boltzmann

__all__ = ['Program']

# Solver.lower_density (cmmdft/solver.py:83): the clip of the solvers' tracking lines
LOWER_DENSITY = 1e-12


class Program(object):
    def __init__(self, prefix='', hostname='', guestname='', ff_suffix='', funct_suffix='', grid_suffix='',
                 suffix='', overwrite=False):
        self.name_dict = {'prefix': prefix, 'hostname': hostname, 'guestname': guestname,
                          'ff_suffix': ff_suffix, 'funct_suffix': funct_suffix,
                          'grid_suffix': grid_suffix, 'suffix': suffix}
        workdir = Path(prefix) / hostname / guestname / ff_suffix / funct_suffix / grid_suffix / suffix
        workdir.mkdir(parents=True, exist_ok=True)
        self.workdir = workdir
        self.overwrite = overwrite
        self.rho_fn = None
        self.system = None
        self.grid = None
        self.fener = None
        self.solver = None

    def set_system(self, host, guest):
        self.system = System(host, guest)

    def set_grid(self, npoints=None, spacing=0.5 * angstrom):
        assert self.system is not None, "Host and guest must first be set using 'set_system'"
        self.grid = Grid(self.system.host.cell, npoints=npoints, spacing=spacing)

    def init_free_energy(self, temperature):
        assert self.grid is not None, "Grid must first be set using 'set_grid'"
        self.fener = FreeEnergy(self.grid, self.system, temperature, workdir=self.workdir,
                                overwrite=self.overwrite, name_dict=self.name_dict)

    def set_temperature(self, temperature):
        self.fener.set_temperature(temperature)

    def set_solver(self, solver):
        assert isinstance(solver, Solver), "solver is not an instance of Solver, aborting!"
        self.solver = solver

    def _extpot(self):
        for n in self.fener.part_names:
            if 'ExtPot' in n:
                return self.fener.part_dict[n].potential
        return None

    def _set_initial_density(self, Ninit=None, chempot=None, rewrite=False, temperature=None, silent=False):
        """Initial guess (cmmdft/program.py:219-305)."""
        if self.rho_fn is not None and os.path.isfile(self.rho_fn) and not self.overwrite and not rewrite:
            self.rho0 = np.load(self.rho_fn)
            return
        V = self._extpot()
        if Ninit is not None:
            if isinstance(Ninit, (str, Path)):
                if not Path(Ninit).is_file():
                    raise FileNotFoundError('File %s for setting initial density not found' % Ninit)
                self.rho0 = np.load(Ninit)
            elif isinstance(Ninit, float):
                if V is not None:
                    self.rho0 = Ninit * np.exp(-np.maximum(V, 0) / boltzmann / temperature)
                else:
                    self.rho0 = np.full(self.grid.npoints, Ninit)
            elif isinstance(Ninit, np.ndarray):
                assert Ninit.shape == tuple(self.grid.npoints), 'Ninit must have the same shape as the grid'
                self.rho0 = Ninit
            return
        if V is None:
            V = np.zeros(self.grid.npoints)
        self.rho0 = np.exp(self.fener.beta * (chempot - V)) / self.fener.wavelength ** 3

    def cascade_solver(self, solvers, chempot, **kwargs):
        """Try solvers in turn until one converges (cmmdft/program.py:315-328)."""
        for solver in solvers:
            self.set_solver(solver)
            try:
                N, rho, converged = self.solve(chempot, **kwargs)
                if converged:
                    return N, rho, converged
            except NoSolutionError:
                continue
        return None

    def solve(self, chempot, Ninit=None, rewrite=False, energy_tracking=True, silent=False,
              continue_solving=False):
        """Equilibrium density at one chemical potential (cmmdft/program.py:331-404)."""
        self.file_suffix = get_file_suffix(chempot, self.fener.temperature)
        if energy_tracking:   # convergence_*.txt (program.py:372-374, functionals.py:121-174)
            self.fener.init_tracking(os.path.join(self.workdir, 'convergence_%s.txt' % self.file_suffix))
        self.rho_fn = os.path.join(self.workdir, 'rho_%s.npy' % self.file_suffix)
        if os.path.isfile(self.rho_fn) and not self.overwrite and not rewrite and not continue_solving:
            rho = np.load(self.rho_fn)
            return self.grid.integrate(rho), rho, True
        self._set_initial_density(Ninit=Ninit, chempot=chempot, rewrite=rewrite,
                                  temperature=self.fener.temperature, silent=silent)
        # the start density's line, as the solver writes it (solver.py:103-127;
        # the reference's solvers add one line per step)
        if energy_tracking:
            self.fener.track(chempot, self.rho0, step=0, lower_density=LOWER_DENSITY)
        N, rho, converged = self.solver.solve(chempot, self.rho0.copy(), 2)
        if energy_tracking:   # the final density's line
            self.fener.track(chempot, rho, step=self.solver.curr_step, lower_density=LOWER_DENSITY)
        if self.solver.track_history:
            fn = self.workdir / ('solving_history_%s.csv' % self.file_suffix)
            np.savetxt(fn, self.solver.history[:self.solver.curr_step + 1], delimiter=',',
                       header=self.solver.history_header)
        np.save(self.rho_fn, rho)
        return N, rho, converged

    def solve_isotherm(self, chempots, Ninit=None, method='hybridanderson', threshold=1e-8, criterion='res',
                       nsteps=500, save=True, **options):
        """Batched solve of many chemical potentials in one launch sequence.

        Ninit: None (ideal-gas start) or an array of bulk densities (Ninit=float start per point).
        Returns (N[B], rho[B, N1, N2, N3], converged[B]); densities are cached as rho_*.npy.
        """
        from . import batch as BT
        from . import workload as W
        fn = self.fener.device()
        mus = np.asarray(chempots, dtype=float)
        rho0 = W.initial_density(fn, mus, ninit=None if Ninit is None else np.asarray(Ninit, dtype=float))
        s = BT.NativeBatchSolve(fn, mus, method=method, nsteps=nsteps, threshold=threshold, criterion=criterion,
                                **options)
        N, rho, conv = s.solve(rho0)
        rho = rho.cpu().numpy()
        if save:
            for i, mu in enumerate(mus):
                np.save(os.path.join(self.workdir, 'rho_%s.npy' % get_file_suffix(mu, self.fener.temperature)), rho[i])
        return np.asarray(N), rho, np.asarray(conv)
