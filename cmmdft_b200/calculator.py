"""Observables of converged densities (cmmdft/calculator.py:20-340, 343-492).

loading / return_loading (absolute and excess uptake), the helium void
fraction, the Henry coefficient and the grand potential with its parts,
read from the reference's ``rho_{mu}kJmol_{T}K.npy`` files.  Field work
(potentials, functional values) runs on the GPU.
"""
import re
from pathlib import Path

import numpy as np

from . import engine as E
from .eos import EquationOfState
from .hosts import HELIUM
from .tools import get_file_suffix, convert_units, Document
from .units import angstrom, avogadro, bar, boltzmann, kjmol

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

    def get_chemical_potential(self, temperature):
        """Chemical potentials of the densities saved at ``temperature``, in
        ascending order, from the rho_*.npy names (calculator.py:140-150)."""
        tag = f'{temperature:#7.5f}K.npy'
        mus = []
        for f in self.workdir.iterdir():
            if f.name.startswith('rho') and f.name.endswith(tag):
                m = re.match(r'rho_([-+]?\d*\.?\d+(?:[eE][-+]?\d+)?)kJmol', f.name)
                if m:
                    mus.append(float(m.group(1)))
        return np.sort(np.array(mus)) * kjmol

    def save_loadings(self, temperature, chempots=None, pressure=False, excess=False, eos=None, fn=None):
        """Loadings vs chemical potential (or pressure) as CSV (calculator.py:186-228)."""
        if chempots is None:
            chempots = self.get_chemical_potential(temperature)
        data = np.zeros((2, len(chempots)))
        if pressure:
            header = 'pressures [au], loadings [molecules/uc]'
            data[0] = np.array([eos.calculate_pressure(temperature, mu) for mu in chempots])
        else:
            header = 'chempot [au], loadings [molecules/uc]'
            data[0] = chempots
        data[1] = self.return_loading(temperature, chempots, excess=excess, eos=eos)
        if fn is None:
            fn = self.workdir / f'{"excess_" if excess else ""}loads_{temperature:#3.0f}K{"_vs_P" if pressure else ""}.csv'
        np.savetxt(Path(fn), data.T, delimiter=',', header=header, comments='')
        return Path(fn)

    def save_loadings_AIF(self, temp, chempots=None, pressures=None, eos=None, input_fn=None, user=None,
                          excess=False, loading_unit='au/uc', fn=None, He_frac=None):
        """Loadings as an Adsorption Information File (calculator.py:230-340):
        the same data block, metadata keys and loop (pressure, fugacity,
        chemical potential, absolute amount) as the reference writes, with
        this package as the simulation code.  As in the reference, the loop
        carries the absolute uptake; ``excess`` sets the isotherm type."""
        import datetime
        import getpass
        from . import __version__
        from .system import NanoporousHost
        d = Document()
        d.add_new_block('CmmDFT2aif')
        blk = d.sole_block()
        blk.set_pair('_audit_aif_version', '6acf6ef')
        blk.set_pair('_exptl_operator', getpass.getuser() if user is None else user)
        blk.set_pair('_adsnt_material_id', self.host.name)
        blk.set_pair('_exptl_adsorptive', self.guest.name)
        blk.set_pair('_exptl_temperature', f'{temp:0.3f}K')
        blk.set_pair('_exptl_method', 'simulation')
        blk.set_pair('_exptl_isotherm_type', 'excess' if excess else 'absolute')
        blk.set_pair('_simltn_date', datetime.datetime.now().strftime('%Y-%m-%d'))
        blk.set_pair('_simltn_code', f'cmmdft_b200-{__version__}')
        blk.set_pair('_simltn_sampling', 'cDFT')
        files = [str(input_fn)] if input_fn is not None else []
        for obj in (self.host, self.guest):
            for attr in ('chk', 'par'):
                if getattr(obj, attr, None) is not None:
                    files.append(str(getattr(obj, attr)))
        blk.set_pair('_simltn_input_files', files)
        ff = self.program.name_dict.get('ff_suffix', '')
        if isinstance(self.host, NanoporousHost):
            ffs = ff.split('_')
            blk.set_pair('_simltn_forcefield_adsorptive', ffs[0])
            blk.set_pair('_simltn_forcefield_adsorbent', ffs[1] if len(ffs) > 1 else '')
        else:
            blk.set_pair('_simltn_forcefield_adsorbent', ff)
        for k, v in (('temperature', 'K'), ('energy', 'kJ/mol'), ('loading', loading_unit), ('pressure', 'bar'),
                     ('mass', 'amu')):
            blk.set_pair('_units_' + k, v)
        if pressures is None:
            assert eos is not None and chempots is not None, \
                'Must provide chemical potentials and an equation of state to compute pressures'
            pressures = np.array([eos.calculate_pressure(temp, mu) for mu in chempots])
        if chempots is None:
            assert eos is not None, 'Must provide an equation of state to compute chemical potentials'
            chempots = np.array([eos.calculate_mu(temp, p) for p in pressures])
        chempots = np.asarray(chempots, dtype=float)
        pressures = np.asarray(pressures, dtype=float)
        fug = np.exp(self.fener.beta * chempots) / self.fener.beta / self.fener.wavelength ** 3
        uptake = self.return_loading(temp, chempots, excess=False)
        if loading_unit not in ('au/uc', 'mol/mol'):
            masses = getattr(self.host, 'masses', None)
            assert masses is not None, 'loading units other than au/uc need the host atoms\' masses'
            uptake = uptake * convert_units(self.guest.mass, float(np.sum(masses)),
                                            self.host.cell.volume).conversion_factor('au/uc', loading_unit)
        loop = blk.init_loop('_adsorp_', ['pressure', 'fugacity', 'chemicalpotential', 'amount_absolute'])
        loop.set_all_values([['%.5E' % x for x in pressures / bar], ['%.5E' % x for x in fug / bar],
                             ['%.5E' % x for x in chempots / kjmol], ['%.5E' % x for x in uptake]])
        if fn is None:
            fn = self.workdir / f'adsorption_{temp:0.2f}K.aif'
        d.write_file(str(fn))
        return Path(fn)

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
        if partname in ('WDA-V', 'LDA'):   # evaluated inside the fused pipeline only
            if local:
                raise NotImplementedError("local values of the %s part are not exposed" % partname)
            from .functionals import _fused_part_values
            return _fused_part_values(self.fener, rho)[self.fener.part_names.index(partname)] / N
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
