"""System description and the grid, mirroring cmmdft/system.py.

Same class names and arguments as the reference (System, NanoporousHost,
EmptyHost, SphericalLJGuest, Grid).  Differences that follow from the GPU
design:
  * Grid.fft returns a ``Spectrum`` (the density's yz-spectrum on the GPU);
    ``np.asarray(spectrum)`` gives the reference's full complex spectrum
    with its phase convention (cmmdft/system.py:310-311) for inspection.
  * NanoporousHost reads yaff text checkpoints (.chk) and LJ:PARS files
    itself (yaff is not a dependency), or takes arrays directly.
"""
import math
import os

import numpy as np

from . import _lib as L
from .units import angstrom, boltzmann, planck, parse_unit
from .workload import hardsphere_radius

__all__ = ['Cell', 'System', 'Host', 'NanoporousHost', 'EmptyHost', 'Guest', 'SphericalLJGuest',
           'NonSphericalGuest', 'DualModelGuest', 'Grid', 'Spectrum', 'read_chk', 'read_pars_file']


class Cell(object):
    """Periodic cell with cell vectors as rows (yaff's Cell interface)."""

    def __init__(self, rvecs):
        self.rvecs = np.asarray(rvecs, dtype=np.float64).reshape(3, 3)
        self.nvec = 3

    @property
    def volume(self):
        return float(abs(np.linalg.det(self.rvecs)))

    @property
    def parameters(self):
        lengths = np.linalg.norm(self.rvecs, axis=1)
        ang = []
        for i in range(3):
            a, b = self.rvecs[(i + 1) % 3], self.rvecs[(i + 2) % 3]
            ang.append(math.acos(max(-1.0, min(1.0, float(a @ b / (np.linalg.norm(a) * np.linalg.norm(b)))))))
        return lengths, np.array(ang)


def read_chk(fn):
    """Minimal reader of yaff text checkpoints: returns a dict of arrays.

    The format is a sequence of ``name kind=<type> <shape>`` headers followed
    by whitespace-separated values (InputFiles/Host/*/struct.chk).
    """
    out = {}
    with open(fn) as f:
        tokens = f.read().split('\n')
    i = 0
    while i < len(tokens):
        line = tokens[i].strip()
        i += 1
        if not line or 'kind=' not in line:
            continue
        head = line.split()
        name = head[0]
        kind = [h for h in head if h.startswith('kind=')][0][5:]
        shape_tok = head[-1] if len(head) > 2 else ''
        shape = tuple(int(x) for x in shape_tok.split(',')) if shape_tok and kind.endswith('ar') else ()
        n = int(np.prod(shape)) if shape else 1
        vals = []
        while len(vals) < n and i < len(tokens):
            if 'kind=' in tokens[i]:
                break
            vals.extend(tokens[i].split())
            i += 1
        if kind in ('fltar', 'intar'):
            arr = np.array([float(v) for v in vals[:n]])
            out[name] = arr.reshape(shape).astype(int if kind == 'intar' else float)
        elif kind == 'strar':
            out[name] = vals[:n]
        elif kind == 'flt':
            out[name] = float(head[2]) if len(head) > 2 else float(vals[0])
        elif kind == 'int':
            out[name] = int(head[2]) if len(head) > 2 else int(vals[0])
        else:
            out[name] = vals
    return out


def read_pars_file(pars_file):
    """LJ sigma/epsilon per atom type from a yaff ``LJ:PARS`` file
    (cmmdft/extpot_calculator.py:705-716)."""
    units = {}
    ff = {}
    with open(pars_file) as f:
        for line in f:
            line = line.split('#')[0].strip()
            if not line.startswith('LJ:'):
                continue
            key, _, rest = line.partition(' ')
            key = key[3:]
            rest = rest.split()
            if key == 'UNIT':
                units[rest[0]] = parse_unit(rest[1])
            elif key == 'PARS':
                ff[rest[0]] = (float(rest[1]) * units.get('SIGMA', 1.0), float(rest[2]) * units.get('EPSILON', 1.0))
    return ff


class System(object):
    def __init__(self, host, guest):
        self.host = host
        self.guest = guest

    def copy(self):
        return System(self.host.copy(), self.guest.copy())


class Host(object):
    def __init__(self, name, cell):
        self.name = name
        self.cell = cell

    def copy(self):
        return type(self)(self.name, self.cell)


class NanoporousHost(Host):
    """Host framework; positions are recentred to their mean (cmmdft/system.py:54-73).

    Either ``chk`` (yaff text checkpoint) and ``par`` (LJ:PARS file) or the
    arrays ``pos`` (bohr), ``ffatypes``, ``ffatype_ids``, ``rvecs`` and
    ``ff`` ({type: (sigma, epsilon)}) must be given.
    """

    def __init__(self, name, chk=None, par=None, pos=None, ffatypes=None, ffatype_ids=None, rvecs=None, ff=None,
                 masses=None):
        self.chk, self.par = chk, par
        if chk is not None:
            d = read_chk(chk)
            pos = d['pos']
            ffatypes = list(d['ffatypes'])
            ffatype_ids = d['ffatype_ids']
            rvecs = d['rvecs']
            masses = d.get('masses', masses)
        # atomic masses (atomic units), used for loading-unit conversions only
        self.masses = None if masses is None else np.asarray(masses, dtype=np.float64)
        if ff is None and par is not None:
            ff = read_pars_file(par)
        self.pos = np.asarray(pos, dtype=np.float64).copy()
        self.pos -= self.pos.sum(axis=0) / len(self.pos)
        self.ffatypes = list(ffatypes)
        self.ffatype_ids = np.asarray(ffatype_ids, dtype=np.int32)
        self.rvecs = np.asarray(rvecs, dtype=np.float64).reshape(3, 3)
        self.ff = dict(ff) if ff is not None else None
        Host.__init__(self, name, Cell(self.rvecs))

    @classmethod
    def from_synthetic(cls, name, synth):
        """Wrap a hosts.SyntheticHost."""
        return cls(name, pos=synth.pos, ffatypes=synth.ffatypes, ffatype_ids=synth.ffatype_ids,
                   rvecs=synth.rvecs, ff=synth.ff, masses=getattr(synth, 'masses', None))

    @property
    def natom(self):
        return len(self.pos)

    @property
    def volume(self):
        return self.cell.volume

    def recentred_pos(self):
        return self.pos

    def copy(self):
        h = NanoporousHost.__new__(NanoporousHost)
        h.__dict__.update(self.__dict__)
        return h


class EmptyHost(Host):
    """Empty periodic cell (cmmdft/system.py:76-96)."""

    def __init__(self, name, cell=None, volume=None):
        if cell is None:
            assert volume is not None, 'Either cell or volume keyword argument must be defined'
            cell = Cell(np.diag([1., 1., 1.]) * volume ** (1. / 3.))
        elif not isinstance(cell, Cell):
            cell = Cell(cell)
        Host.__init__(self, name, cell)


class Guest(object):
    def __init__(self, name, mass):
        self.name = name
        self.mass = mass
        self.preset_Rhs = None
        self.preset_Rhs_zero = None
        self.Rhs = None
        self.Rhs_zero = None

    def copy(self):
        return type(self)(self.name, self.mass)

    def wavelength(self, temperature):
        """Thermal de Broglie wavelength (cmmdft/system.py:115-117)."""
        kT = boltzmann * temperature
        return planck / np.sqrt(2 * np.pi * self.mass * kT)

    def set_fixed_rhs(self, Rhs, Rhs_zero):
        self.preset_Rhs = Rhs
        self.preset_Rhs_zero = Rhs_zero

    def compute_hardsphere_radius(self, temperature, **kwargs):
        if self.preset_Rhs_zero is not None:
            self.Rhs, self.Rhs_zero = self.preset_Rhs, self.preset_Rhs_zero
        else:
            self.Rhs, self.Rhs_zero = self._calculate_hardsphere_radius(temperature, **kwargs)

    def _calculate_hardsphere_radius(self, temperature, **kwargs):
        raise NotImplementedError


class SphericalLJGuest(Guest):
    """Spherical LJ guest with the Barker-Henderson radius fit (cmmdft/system.py:137-158)."""

    def __init__(self, name, mass, sigma, epsilon):
        Guest.__init__(self, name, mass)
        self.sigma = sigma
        self.epsilon = epsilon
        self.natom = 1

    def copy(self):
        return type(self)(self.name, self.mass, self.sigma, self.epsilon)

    def _calculate_hardsphere_radius(self, temperature, **kwargs):
        return hardsphere_radius(self.sigma, self.epsilon, temperature), self.sigma


class _Molecule(object):
    """The guest's atoms as the reference reads them from a yaff checkpoint
    (positions in bohr, masses in atomic units, atom types)."""

    def __init__(self, pos, masses, ffatypes, ffatype_ids):
        self.pos = np.asarray(pos, dtype=np.float64).reshape(-1, 3).copy()
        self.masses = None if masses is None else np.asarray(masses, dtype=np.float64).reshape(-1)
        self.ffatypes = list(ffatypes)
        self.ffatype_ids = np.asarray(ffatype_ids, dtype=np.int32).reshape(-1)

    @property
    def natom(self):
        return len(self.pos)


class NonSphericalGuest(Guest):
    """Rigid multi-site guest (cmmdft/system.py:162-212).

    Either ``chk`` (yaff text checkpoint with masses) and ``par`` (LJ:PARS
    file of the guest's atom types) or the arrays ``pos`` (bohr),
    ``masses``, ``ffatypes``, ``ffatype_ids`` and ``ff``
    ({type: (sigma, epsilon)}) must be given.  The external potential of
    such a guest is the orientation average of the LJ potentials of its
    sites (ExternalPotential.generate_potential with a temperature).
    """

    def __init__(self, name, chk=None, par=None, pos=None, masses=None, ffatypes=None, ffatype_ids=None, ff=None):
        self.chk, self.par = chk, par
        if chk is not None:
            d = read_chk(chk)
            pos, ffatypes, ffatype_ids = d['pos'], list(d['ffatypes']), d['ffatype_ids']
            m = d.get('masses')
            masses = m if isinstance(m, np.ndarray) and m.size else None
        if ff is None and par is not None:
            ff = read_pars_file(par)
        self.mol = _Molecule(pos, masses, ffatypes, ffatype_ids)
        self.natom = self.mol.natom
        self.ff = dict(ff) if ff is not None else None
        if self.mol.masses is None:
            raise ValueError('Masses not defined in guest chk file, cannot compute total mass for NonSphericalGuest')
        Guest.__init__(self, name, self.mol.masses.sum())

    def _arrays(self):
        return dict(chk=self.chk, par=self.par, pos=self.mol.pos, masses=self.mol.masses,
                    ffatypes=self.mol.ffatypes, ffatype_ids=self.mol.ffatype_ids, ff=self.ff)

    def copy(self):
        return type(self)(self.name, **self._arrays())

    def site_parameters(self):
        """(sigma, epsilon) per guest atom from the guest's LJ table."""
        if self.ff is None:
            raise ValueError("guest %s has no LJ parameters (par file or ff)" % self.name)
        ids = self.mol.ffatype_ids
        sig = np.array([self.ff[self.mol.ffatypes[t]][0] for t in ids])
        eps = np.array([self.ff[self.mol.ffatypes[t]][1] for t in ids])
        return sig, eps

    def _calculate_hardsphere_radius(self, temperature, **kwargs):
        raise NotImplementedError('Using generic NonSphericalGuest class, cannot compute hardsphere radius, '
                                  'use DualModelGuest class')


class DualModelGuest(SphericalLJGuest, NonSphericalGuest):
    """Guest with a spherical LJ model (hard-sphere radius, attraction) and a
    multi-site model (external potential), cmmdft/system.py:214-228."""

    def __init__(self, name, mass, sigma, epsilon, chk=None, par=None, **arrays):
        SphericalLJGuest.__init__(self, name, mass, sigma, epsilon)
        NonSphericalGuest.__init__(self, name, chk, par, **arrays)

    def copy(self):
        a = self._arrays()
        chk, par = a.pop('chk'), a.pop('par')
        return type(self)(self.name, self.mass, self.sigma, self.epsilon, chk, par, **a)

    def _calculate_hardsphere_radius(self, temperature, **kwargs):
        return SphericalLJGuest._calculate_hardsphere_radius(self, temperature, **kwargs)


class Spectrum(object):
    """Spectra of real fields on the GPU (yz-spectrum layout of the C ABI).

    ``np.asarray(spec)`` materialises the reference convention
    ``fftn(rho) * exp(i pi scalprod) / Npts`` (cmmdft/system.py:310-311).
    """

    def __init__(self, grid, data, rho=None):
        self.grid = grid
        self.data = data      # torch [B, 2*nspec] yz-spectrum
        self.rho = rho        # torch [B, N1, N2, N3] real field (kept for value())

    def __array__(self, dtype=None, copy=None):
        import torch
        g = self.grid
        rho = self.rho if self.rho is not None else g.plan.irfft_yz(self.data) / float(np.prod(g.npoints))
        full = g.plan.spec_to_full(g.plan.rfft(rho.contiguous()))
        out = full * np.exp(1j * np.pi * g.scalprod)[None] / np.prod(g.npoints)
        out = out[0] if out.shape[0] == 1 else out
        return out.astype(dtype) if dtype is not None else out


class Grid(object):
    """Periodic centred grid (cmmdft/system.py:231-332)."""

    def __init__(self, cell, npoints=None, spacing=0.25 * angstrom, silent=False):
        if not isinstance(cell, Cell):
            cell = Cell(cell.rvecs if hasattr(cell, 'rvecs') else cell)
        self.cell = cell
        if npoints is None:
            lengths, angles = cell.parameters
            self.npoints = [int(np.ceil(l / spacing)) for l in lengths]
        elif isinstance(npoints, (int, np.integer)):
            self.npoints = [int(npoints)] * 3
        else:
            self.npoints = [int(n) for n in npoints]
        self.suffix = '_'.join("%d" % n for n in self.npoints)
        self.spacings = [np.linalg.norm(cell.rvecs[:, a]) / self.npoints[a] for a in range(3)]
        self.dr = cell.volume / np.prod(self.npoints)
        self.dk = 1.0 / self.dr
        self._plan = None
        self._points = None
        self._kpoints = None

    # ---- lazily built numpy tables (compatibility; the solve does not use them)
    @property
    def points(self):
        if self._points is None:
            n = self.npoints
            pts = np.zeros(n + [4])
            g = [np.linspace(-0.5, 0.5, num=n[a], endpoint=False) for a in range(3)]
            gp = np.asarray(np.meshgrid(g[0], g[1], g[2], indexing='ij'))
            pts[..., :3] = np.einsum('ab,aijk->ijkb', self.cell.rvecs, gp)
            pts[..., 3] = np.sqrt(pts[..., 0] ** 2 + pts[..., 1] ** 2 + pts[..., 2] ** 2)
            self._points = pts
        return self._points

    @property
    def kpoints(self):
        if self._kpoints is None:
            n = self.npoints
            kp = np.zeros(n + [4])
            kg = [np.fft.fftfreq(n[a], d=self.spacings[a]) for a in range(3)]
            m = np.meshgrid(kg[0], kg[1], kg[2], indexing='ij')
            for a in range(3):
                kp[..., a] = 2 * np.pi * m[a]
            kp[..., 3] = np.sqrt(kp[..., 0] ** 2 + kp[..., 1] ** 2 + kp[..., 2] ** 2)
            self._kpoints = kp
        return self._kpoints

    @property
    def scalprod(self):
        k, n, d = self.kpoints, self.npoints, self.spacings
        return k[..., 0] * d[0] * n[0] + k[..., 1] * d[1] * n[1] + k[..., 2] * d[2] * n[2]

    @property
    def sigma_lanczos(self):
        k = self.kpoints
        kc = 2 * np.pi / np.array(self.spacings)
        return np.sinc(k[..., 0] / kc[0]) * np.sinc(k[..., 1] / kc[1]) * np.sinc(k[..., 2] / kc[2])

    # ---- GPU plan
    @property
    def plan(self):
        if self._plan is None:
            from . import engine as E
            self._plan = E.GridPlan(self.npoints, self.cell.rvecs)
        return self._plan

    def supercell(self, supercell):
        supercell = np.asarray(supercell)
        return Grid(Cell(self.cell.rvecs * supercell), npoints=list(np.asarray(self.npoints) * supercell))

    def copy(self):
        g = Grid(self.cell, npoints=self.npoints)
        g._plan = self._plan
        return g

    def integrate(self, data):
        """sum(data) * dr (cmmdft/system.py:307-308); numpy or torch input."""
        if hasattr(data, 'detach'):
            return float(data.sum().item()) * self.dr
        return np.sum(data) * self.dr

    def _to_device(self, rdata):
        import torch
        t = rdata if hasattr(rdata, 'detach') else torch.as_tensor(np.ascontiguousarray(rdata, dtype=np.float64))
        t = t.to('cuda', dtype=torch.float64)
        return t.reshape((-1,) + tuple(self.npoints)).contiguous()

    def fft(self, rdata):
        """Spectrum of a real field (GPU)."""
        if isinstance(rdata, Spectrum):
            return rdata
        rho = self._to_device(rdata)
        return Spectrum(self, self.plan.rfft_yz(rho), rho)

    def ifft(self, fdata):
        """Real field of a spectrum (numpy); accepts a Spectrum or a reference-convention array."""
        if isinstance(fdata, Spectrum):
            if fdata.rho is not None:
                r = fdata.rho
            else:
                r = self.plan.irfft_yz(fdata.data) / float(np.prod(self.npoints))
            r = r.cpu().numpy()
            return r[0] if r.shape[0] == 1 else r
        raise TypeError("Grid.ifft takes the Spectrum returned by Grid.fft")

    def as_spectrum(self, krho):
        if isinstance(krho, Spectrum):
            return krho
        raise TypeError("functional parts take the Spectrum returned by Grid.fft")
