"""Observables of converged densities (cmmdft/calculator.py:20-183, 343-492).

loading / return_loading (absolute and excess uptake), the helium void
fraction, the Henry coefficient and the grand potential with its parts,
read from the reference's ``rho_{mu}kJmol_{T}K.npy`` files.  Field work
(potentials, functional values) runs on the GPU.
"""
import numpy as np

from . import engine as E
from .eos import EquationOfState
from .hosts import HELIUM
from .tools import get_file_suffix
from .units import angstrom, avogadro, boltzmann

__all__ = ['Calculator']


class Calculator(object):
    def __init__(self, program, label=None):
        self.program = program
        self.workdir = program.workdir
        self.grid = program.grid
        self.fener = program.fener
        self.host = program.system.host
        self.guest = program.system.guest
        self.label = label

    def _rho(self, temp, chempot):
        fn = self.workdir / ('rho_%s.npy' % get_file_suffix(chempot, temp))
        assert fn.is_file(), 'No file found at %s' % fn
        return np.load(fn)

    def loading(self, temp, chempot, mask=None):
        """N = integral rho (calculator.py:60-88)."""
        rho = self._rho(temp, chempot)
        if mask is not None:
            rho = np.where(mask, rho, 0.0)
        return float(self.grid.integrate(rho))

    def get_helium_fraction(self, temperature):
        """He void fraction: integral clip(exp(-V_He / kT), 0, 1) / V_cell (intent of
        calculator.py:152-167, whose call of read_pars_file is broken in the reference)."""
        h = self.host
        sig = np.array([h.ff[t][0] for t in h.ffatypes])
        eps = np.array([h.ff[t][1] for t in h.ffatypes])
        V = E.external_potential(self.grid.plan, h.recentred_pos(), h.ffatype_ids, sig, eps,
                                 HELIUM['sigma'] * angstrom, HELIUM['epsilon_K'] * boltzmann, 12 * angstrom,
                                 float('inf'))
        import torch
        e = torch.clamp(torch.exp(-V / boltzmann / temperature), 0, 1)
        return float(e.sum().item()) * self.grid.dr / self.host.cell.volume

    def return_loading(self, temp, chempots, excess=False, eos=None, He_frac=None):
        """Absolute or excess loadings for a list of chemical potentials (calculator.py:114-138)."""
        out = np.zeros(len(chempots))
        for i, mu in enumerate(chempots):
            try:
                out[i] = self.loading(temp, mu)
            except AssertionError:
                out[i] = np.nan
        if excess:
            assert eos is not None, 'Must provide an equation of state object when calculating excess uptake'
            if He_frac is None:
                He_frac = self.get_helium_fraction(temp)
            eos.set_temperature(temp)
            dens = np.nanmin(eos.solve_densities_from_chempots(chempots), axis=1)
            out -= dens * He_frac * self.host.cell.volume
        return out

    def get_Henry_Coefficient(self, temperature):
        """Henry coefficient from the external potential (calculator.py:169-183)."""
        V = self.fener.part_dict['ExtPot'].potential
        integ = self.grid.integrate(np.exp(-V / temperature / boltzmann))
        return 1 / avogadro / boltzmann / temperature / self.host.cell.volume * integ

    def free_energy_contrib(self, temp, chempot, partname, over_loading=False, local=False, fn=None, rho=None):
        """One free-energy contribution (calculator.py:343-406)."""
        if rho is None:
            rho = np.load(fn) if fn is not None else self._rho(temp, chempot)
        N = self.grid.integrate(rho) if over_loading else 1.0
        if partname.lower() in ('fid', 'fideal'):
            rr = np.clip(rho, 1e-20, None)
            v = boltzmann * temp * rr * (np.log(rr * self.fener.wavelength ** 3) - 1)
            return (v if local else self.grid.integrate(v)) / N
        assert partname in self.fener.part_names, '%s not found in %s' % (partname, self.fener.part_names)
        return self.fener.part_dict[partname].value(self.grid.fft(rho), local) / N

    def free_energy(self, temp, chempot, local=False):
        v = self.free_energy_contrib(temp, chempot, 'fid', local=local)
        for p in self.fener.parts:
            v += self.free_energy_contrib(temp, chempot, p.name, local=local)
        return v

    def grand_potential(self, temp, chempot, local=False):
        """Omega = F - mu N (calculator.py:463-492)."""
        v = self.free_energy(temp, chempot, local=local)
        if local:
            return v - chempot * self._rho(temp, chempot)
        return v - chempot * self.loading(temp, chempot)
