"""Observables of converged densities (cmmdft/calculator.py:20-899).

loading / return_loading (absolute and excess uptake), the helium void
fraction, the Henry coefficient and the grand potential with its parts, the
loading exports, and the projections onto a collective variable with the
free-energy path built from them, read from the reference's
``rho_{mu}kJmol_{T}K.npy`` files.  Field work (potentials, functional values,
the projections' binned sums) runs on the GPU.
"""
import bisect
import re
from pathlib import Path

import numpy as np

from . import engine as E
from .eos import EquationOfState
from .hosts import HELIUM
from .tools import get_file_suffix, convert_units, Document
from .units import angstrom, avogadro, bar, boltzmann, kjmol

__all__ = ['Calculator', 'make_supercell']


def make_supercell(data, repetitions=(3, 3, 3), grid_spacings=None, periodic=True):
    """Tile a field over repetitions of the cell (cmmdft/tools.py:345-366);
    with periodic=False ``data`` holds points [N1, N2, N3, 3] and each copy
    is shifted by index x spacing x N per axis."""
    data = np.asarray(data)
    reps = [int(r) for r in repetitions]
    assert len(reps) == 3, 'The repetitions parameter must be a list of 3 integers'
    nop = data.shape[:3]
    if periodic:
        return np.tile(data, reps)
    assert grid_spacings is not None, 'If periodic, grid_spacings must be provided'
    out = np.zeros((nop[0] * reps[0], nop[1] * reps[1], nop[2] * reps[2], 3))
    step = np.array(grid_spacings) * nop
    for i in range(reps[0]):
        for j in range(reps[1]):
            for k in range(reps[2]):
                out[i * nop[0]:(i + 1) * nop[0], j * nop[1]:(j + 1) * nop[1], k * nop[2]:(k + 1) * nop[2]] = \
                    data + np.array([i, j, k]) * step
    return out


def _binned_sums(cvs, cvs_mat, weights, mask, counts=False):
    """Per bin e of the sorted edges ``cvs``: the sum of weights * mask over
    the points with cvs[e] < cv < cvs[e+1] (strict, as the reference's
    masks), on the GPU (and the sum of mask there when ``counts``)."""
    import torch
    dev = 'cuda'
    E.require_cuda()
    edges = torch.as_tensor(np.ascontiguousarray(cvs, dtype=np.float64), device=dev)
    cv = torch.as_tensor(np.ascontiguousarray(cvs_mat, dtype=np.float64).reshape(-1), device=dev)
    w = torch.as_tensor(np.ascontiguousarray(weights, dtype=np.float64).reshape(-1), device=dev)
    m = torch.as_tensor(np.ascontiguousarray(mask, dtype=np.float64).reshape(-1), device=dev)
    nb = len(cvs) - 1
    i = torch.searchsorted(edges, cv, right=False)          # first edge >= cv
    e = i - 1
    ok = (e >= 0) & (e < nb)
    ok &= cv < edges[torch.clamp(i, max=nb)]                # strictly below the upper edge
    e = torch.where(ok, e, torch.full_like(e, nb))          # out of every bin -> a discard slot
    tot = torch.zeros(nb + 1, dtype=torch.float64, device=dev).index_add_(0, e, w * m)
    if not counts:
        return tot[:nb].cpu().numpy()
    cnt = torch.zeros(nb + 1, dtype=torch.float64, device=dev).index_add_(0, e, m)
    return tot[:nb].cpu().numpy(), cnt[:nb].cpu().numpy()


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
        # the ideal part is always the integral, as in the reference (calculator.py:426-430)
        v = self.free_energy_contrib(temp, chempot, 'fid')
        for p in self.fener.parts:
            v += self.free_energy_contrib(temp, chempot, p.name, local=local)
        return v

    def grand_potential(self, temp, chempot, local=False):
        """Omega = F - mu N (calculator.py:463-492)."""
        v = self.free_energy(temp, chempot, local=local)
        if local:
            return v - chempot * self._rho(temp, chempot)
        return v - chempot * self.loading(temp, chempot)

    def excess_free_energy(self, temp, chempot, local=False, fn=None):
        """Free energy without the ideal part (calculator.py:433-461)."""
        rho = np.load(fn) if fn is not None else None
        v = 0.0
        for p in self.fener.parts:
            v = v + self.free_energy_contrib(temp, chempot, p.name, local=local, rho=rho)
        return v

    def save_loading_and_grand_potential(self, temp, chempot):
        """Add (or update) the row of ``chempot`` in
        loading_grand_potential_<T>K.csv, rows in ascending chemical
        potential (calculator.py:738-784; chemical potentials in au)."""
        n = self.loading(temp, chempot)
        omega = float(np.real(self.grand_potential(temp, chempot)))
        key = f'{chempot:#0.8f}'
        fn = self.workdir / f'loading_grand_potential_{temp:7.5f}K.csv'
        if fn.is_file():
            data = np.atleast_2d(np.loadtxt(fn, delimiter=',', skiprows=1)).T
            keys = [f'{k:#0.8f}' for k in data[0]]
            if key in keys:
                i = keys.index(key)
                data[1][i] = n
                data[2][i] = omega
            else:
                mus = np.sort(np.array(data[0]))
                col = np.array([[chempot], [n], [omega]])
                if chempot > mus[-1]:
                    data = np.hstack((data, col))
                else:
                    i = bisect.bisect_left(mus, chempot)
                    data = np.hstack((data[:, :i], col, data[:, i:]))
        else:
            data = np.array([[chempot], [n], [omega]])
        np.savetxt(fn, data.T, delimiter=',', header='chempot [kJ/mol], loading [molecules/uc], grand potential [au]',
                   comments='')
        return fn

    # ---- collective variables and projections (calculator.py:494-736) ----
    def collective_variable(self, diffusion_path=None, ring_indices=None, dist_from_axis=None, supercell=False,
                            step_dist=0.5 * angstrom, cvs_limits=None):
        """(cvs, cvs_mat, dist_mask): bin edges of the coordinate along a
        diffusion axis at ``step_dist`` through 0, the coordinate of every
        grid point (of the 3 x 3 x 3 supercell's points with ``supercell``),
        and the points within ``dist_from_axis`` of the axis (calculator.py:
        494-568).  The axis is diffusion_path (2 x 3: a point on it and a
        second point) or the normal through the centre of the host atoms
        ``ring_indices``."""
        assert diffusion_path is not None or ring_indices is not None, \
            "Must provide a diffusion path (diffusion_path) or indices of the atom which form the ring through " \
            "which the diffusion takes place (ring_indices)"
        if ring_indices is not None and diffusion_path is None:
            diffusion_path = np.empty((2, 3))
            pos = self.host.pos[ring_indices]
            center = np.mean(pos, axis=0)
            u, sv, vh = np.linalg.svd(pos - center)
            diffusion_path[0] = center
            diffusion_path[1] = (vh[-1, :] + center) / np.linalg.norm(vh[-1, :] + center)
        diffusion_path = np.asarray(diffusion_path, dtype=np.float64)
        points = self.grid.points[:, :, :, :-1]
        unit = (diffusion_path[1] - diffusion_path[0]) / np.linalg.norm(diffusion_path[1] - diffusion_path[0])
        cvs_mat = (points - diffusion_path[0]) @ unit
        if supercell:
            points = make_supercell(points, grid_spacings=self.grid.spacings, repetitions=[3, 3, 3], periodic=False)
            cvs_mat = (points - diffusion_path[0]) @ unit
        cvs_pos = np.arange(0, np.max(cvs_mat) + step_dist, step_dist)
        cvs_neg = np.arange(0, np.min(cvs_mat) - step_dist, -step_dist)[::-1]
        cvs = np.concatenate((cvs_neg, cvs_pos[1:]))
        if cvs_limits is not None:
            assert len(cvs_limits) == 2, 'cvs_limits must be a tuple of two numbers constraining the cvs values ' \
                                         'for which the free energy is calculated'
            lo, hi = np.min(np.array(cvs_limits)), np.max(np.array(cvs_limits))
            cvs = cvs[bisect.bisect_left(cvs, lo):bisect.bisect_left(cvs, hi)]
        dist_mask = np.ones_like(cvs_mat)
        if dist_from_axis is not None:
            dist_mask = np.linalg.norm(np.cross(points - diffusion_path[0], unit), axis=-1) < dist_from_axis
        return cvs, cvs_mat, dist_mask

    def project_density(self, temp, chempot, cvs, cvs_mat, dist_mask, rewrite=False, supercell=True):
        """(q, n): the loading in each collective-variable bin, at the bin
        centres, written to projected_density_<suffix>.csv and read back from
        there unless ``rewrite`` (calculator.py:570-637)."""
        suff = get_file_suffix(chempot, temp)
        fn = self.workdir / f'projected_density_{suff}.csv'
        if fn.is_file() and not rewrite:
            data = np.loadtxt(fn, delimiter=',', skiprows=1).T
            return data[0], data[1]
        rho = self._rho(temp, chempot).real
        if supercell:
            rho = make_supercell(rho, repetitions=[3, 3, 3], periodic=True)
        n_list = _binned_sums(cvs, cvs_mat, rho, dist_mask) * self.grid.dr
        q_list = (cvs[1:] + cvs[:-1]) / 2
        np.savetxt(fn, np.array((q_list, n_list)).T, delimiter=',', header='cv, density')
        return q_list, n_list

    def project_contributions(self, temp, chempot, contrib_names, cvs, cvs_mat, dist_mask, supercell=True, fn=None,
                              rewrite=False):
        """Per collective-variable bin: the loading and, for each name, the
        integral of that local free-energy contribution, or for
        'pure_extpot' the mean external potential over the bin's points
        where rho is not ~0; written to projected_contributions_<suffix>.csv
        (calculator.py:639-736).  Names are lower-cased first, as the
        reference does, so besides 'fid' and 'pure_extpot' only lower-case
        part names are found."""
        if not isinstance(contrib_names, list):
            contrib_names = [contrib_names]
        contrib_names = [name.lower() for name in contrib_names]
        header = 'cv, density'
        q_list = (cvs[1:] + cvs[:-1]) / 2
        qq, density = self.project_density(temp, chempot, cvs, cvs_mat, dist_mask, rewrite=rewrite,
                                           supercell=supercell)
        out = np.empty((2 + len(contrib_names), len(q_list)))
        out[0] = q_list
        out[1] = density
        rho = self._rho(temp, chempot).real
        rho_mask = None
        if 'pure_extpot' in contrib_names:
            if 'ExtPot' not in self.fener.part_names:
                raise IOError('No external potential present in the functional')
            rs = make_supercell(rho, repetitions=[3, 3, 3], periodic=True) if supercell else rho
            rho_mask = np.isclose(rs, 0, atol=1e-7)
        for ee, name in enumerate(contrib_names):
            header += f', {name}'
            if 'pure_extpot' in name:
                data = self.fener.part_dict['ExtPot'].potential
            else:
                data = self.free_energy_contrib(temp, chempot, name, local=True, rho=rho)
            if supercell:
                data = make_supercell(data, repetitions=[3, 3, 3], periodic=True)
            if 'pure_extpot' in name:
                m = np.asarray(dist_mask, dtype=np.float64) * (~rho_mask)
                tot, cnt = _binned_sums(cvs, cvs_mat, data, m, counts=True)
                with np.errstate(invalid='ignore', divide='ignore'):
                    out[ee + 2] = tot / cnt        # NaN in an empty bin, as the reference's 0/0
            else:
                out[ee + 2] = _binned_sums(cvs, cvs_mat, data, dist_mask) * self.grid.dr
        if fn is None:
            fn = self.workdir / f'projected_contributions_{get_file_suffix(chempot, temp)}.csv'
        np.savetxt(fn, out.T, delimiter=',', header=header)
        return out

    def free_energy_path(self, temp, chempot, chempots=None, fn=None, max_n_chems=0, dens_omega_fn=None,
                         fn_suffix=''):
        """Free-energy profile along the collective variable at ``chempot``
        from the projected densities and grand potentials of the chemical
        potentials up to it (calculator.py:786-899):
          Omega(q) = -(logsumexp(-beta Omega_mu, b=n_mu(q)) + ln beta) / beta,
          F(q) = Omega(q) + mu_last-row * chempot,
        written to free_energy_profile_<mu>kjmol_<T>K.csv.  project_density
        and save_loading_and_grand_potential must have run for those
        chemical potentials.  (Without ``chempots`` the saved densities'
        chemical potentials are used; the reference's own lookup of them
        fails.)"""
        from scipy.special import logsumexp
        beta = 1 / temp / boltzmann
        if chempots is None:
            chems = np.array(self.get_chemical_potential(temp))
            chems = chems[chems <= chempot + 1e-12 * abs(chempot)]
        else:
            ic = np.sort(np.array(chempots, dtype=float))
            chems = ic[:bisect.bisect_left(ic, chempot) + 1]
        assert chems.shape[0] > 0, 'No chemical potentials lower than %s kJ/mol found' % (chempot / kjmol)
        assert np.isclose(chems[-1], chempot), 'The last chemical potential in the list must be equal to the input ' \
                                               'chemical potential'
        assert (chems <= chempot).all(), 'All chemical potentials in the list must be lower than the input ' \
                                         'chemical potential'
        if len(chems) > max_n_chems and max_n_chems != 0:
            idx = np.rint(np.linspace(0, len(chems) - 1, int(max_n_chems))).astype(int)
            it_chems = np.append(chems[idx], chempot)
        else:
            it_chems = chems
        n_proj = []
        for mu in it_chems:
            pfn = self.workdir / f'projected_density_{get_file_suffix(mu, temp)}{fn_suffix}.csv'
            q_list, n = np.loadtxt(pfn, delimiter=',', skiprows=1).T
            n_proj.append(n)
        n_proj = np.array(n_proj)
        dfn = self.workdir / f'loading_grand_potential_{temp:#7.5f}K.csv' if dens_omega_fn is None \
            else Path(dens_omega_fn)
        assert dfn.is_file(), 'No loading and grand potential found for %sK, please run the ' \
                              'save_loading_and_grand_potential function first' % temp
        rows = np.atleast_2d(np.loadtxt(dfn, delimiter=',', skiprows=1))
        keys = [f'{k / kjmol:#0.8f}' for k in rows[:, 0]]
        dens_omega = np.zeros((len(it_chems), 2))
        for i, mu in enumerate(it_chems):
            k = f'{mu / kjmol:#0.8f}'
            assert k in keys, 'No loading and grand potential found for %sK and %s kJ/mol' % (temp, mu / kjmol)
            dens_omega[i] = rows[keys.index(k), 1:]
        gp = -beta * dens_omega[:, 1]
        q_len = q_list.shape[0]
        omega = np.empty(q_len)
        free = np.empty(q_len)
        for e in range(q_len):
            omega[e] = -(logsumexp(gp, b=n_proj[:, e], axis=0) + np.log(beta)) / beta
            free[e] = omega[e] + dens_omega[-1, 0] * chempot
        data = np.array([q_list, n_proj[-1], omega, free])
        fn = self.workdir / (f'free_energy_profile_{chempot / kjmol:#0.8f}kjmol_{temp:#0.3f}K.csv' if fn is None else fn)
        np.savetxt(fn, data.T, delimiter=',', header='cv,density,grand canonical potential,free energy')
        return data
