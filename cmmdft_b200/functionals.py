"""Free-energy functional parts, mirroring cmmdft/functionals.py.

FreeEnergy keeps the reference's part list and add_* methods; the parts
expose derive(krho) / value(krho) like the reference (functionals.py:365-373)
with krho the Spectrum returned by Grid.fft.  Every evaluation runs on the
GPU through the C ABI; the solver uses the fused pipeline of all parts at once
(``FreeEnergy.device()``).

Built: HardSphere (FMT, MFMT, WBII with the antisymmetric 'a' and tensor
't' options, 'atWBII' being the default), MFA (with or without supercell
tail corrections), ExtPot (spherical LJ guests, and multi-site guests by the
orientational average, directly or tricubically interpolated), the WDA
correlation part of add_correlation_wda_lj and the LDA part (LDAFunctional,
add_lda).
"""
import os
from pathlib import Path

import numpy as np

from . import _lib as L
from . import engine as E
from .system import Spectrum
from .units import angstrom, kjmol, boltzmann
from .workload import hs_version_code

__all__ = ['FreeEnergy', 'Functional', 'HardSphereFunctional', 'MFAFunctional', 'ExternalPotential',
           'WDAVFunctional', 'LDAFunctional', 'eos_struct']


def _torch():
    import torch
    return torch


def format_temperature(temperature):
    """'<T>K' as the reference names temperature-dependent files (f'{T:#3.2f}K')."""
    return '%#3.2fK' % temperature


class Functional(object):
    name = None

    def copy(self, **kwargs):
        raise NotImplementedError

    def set_temperature(self, temperature, **kwargs):
        pass


class FreeEnergy(object):
    """Container of functional parts (cmmdft/functionals.py:25-174)."""

    def __init__(self, grid, system, temperature, workdir='.', name_dict={}, overwrite=False):
        self.grid = grid
        self.system = system
        self.temperature = None
        self.beta = None
        self.wavelength = None
        self.parts = []
        self.part_names = []
        self.part_dict = {}
        self.workdir = Path(workdir)
        self.name_dict = name_dict
        self.overwrite = overwrite
        self.fn_tracking = None
        self._device = None
        self.set_temperature(temperature)

    def set_temperature(self, temperature, **kwargs):
        self.temperature = temperature
        self.beta = 1.0 / (boltzmann * temperature)
        self.wavelength = self.system.guest.wavelength(temperature)
        self.system.guest.compute_hardsphere_radius(temperature, **kwargs)
        for p in self.parts:
            p.set_temperature(temperature, Rhs=self.system.guest.Rhs, **kwargs)
        self._device = None

    def add_part(self, part):
        self.parts.append(part)
        self.part_names.append(part.name)
        self.part_dict[part.name] = part
        self._device = None

    def remove_part(self, part_name):
        i = self.part_names.index(part_name)
        self.parts.pop(i)
        self.part_names.pop(i)
        self.part_dict.pop(part_name, None)
        self._device = None

    def add_hard_sphere(self, version='atWBII'):
        hs = HardSphereFunctional(self.grid, self.system.guest.Rhs, version=version)
        hs.set_temperature(self.temperature, Rhs=self.system.guest.Rhs)
        self.add_part(hs)

    def add_mean_field(self, tailcorrections=False, repetitions=[2, 2, 2], cutoff=12 * angstrom, **kwargs):
        g = self.system.guest
        mfa = MFAFunctional(self.grid, tailcorrections=tailcorrections, repetitions=repetitions)
        mfa.generate_potential_lj(g.sigma, g.epsilon, cutoff=cutoff, **kwargs)
        self.add_part(mfa)

    def add_external_potential(self, temperature=None, cutoff=12 * angstrom, limit_potential=1e4 * kjmol,
                               degree=9, interpolate=False, rewrite=False, load_fn=None, save_fn=None, **kwargs):
        """External potential part (cmmdft/functionals.py:176-254).

        With the Program's names set, the potential is kept where the
        reference keeps it, prefix/host/guest/ff_suffix/grid_suffix/suffix/
        (epot.npy, or eff_epot_<T>K.npy for a multi-site guest, with a
        workdir/ExtPots link to it) and loaded from there unless
        ``rewrite`` or the FreeEnergy's ``overwrite`` is set.  Capping:
        non-finite or above ``limit_potential`` -> ``limit_potential``.
        """
        from .system import NonSphericalGuest
        fn = None
        if load_fn is not None:
            assert str(load_fn).endswith('.npy'), 'fn must be a filename of an external potential'
            assert os.path.isfile(load_fn), 'fn must be a filename of an external potential, %s' % load_fn
            ep = ExternalPotential(self.grid, self.system, Path(load_fn).parent, limit_potential=limit_potential,
                                   **kwargs)
            ep.load_potential(load_fn)
        else:
            epot_dr = None
            if save_fn is not None:
                fn = Path(save_fn)
                epot_dr = fn.parent
            elif self.name_dict:
                nd = self.name_dict
                epot_dr = Path(nd.get('prefix', '')) / nd.get('hostname', '') / nd.get('guestname', '') / \
                    nd.get('ff_suffix', '') / nd.get('grid_suffix', '') / nd.get('suffix', '')
                epot_dr.mkdir(parents=True, exist_ok=True)
                g = self.system.guest
                if isinstance(g, NonSphericalGuest) and g.mol.natom != 1:
                    assert temperature is not None, 'Temperature must be provided for non-spherical particles'
                    fn = epot_dr / ('eff_epot_%s.npy' % format_temperature(temperature))
                else:
                    fn = epot_dr / 'epot.npy'
                link = self.workdir / 'ExtPots'
                if not link.is_symlink() and not link.exists():
                    link.symlink_to(epot_dr.absolute())
            ep = ExternalPotential(self.grid, self.system, epot_dr, limit_potential=limit_potential, degree=degree,
                                   interpolate=interpolate, cutoff=cutoff)
            if fn is None or not os.path.isfile(fn) or self.overwrite or rewrite:
                ep.generate_potential(temperature, rewrite=rewrite)
                if fn is not None:
                    ep.dump_potential(fn)
            else:
                ep.load_potential(fn)
        ep.cap()
        self.add_part(ep)

    def add_correlation_wda_lj(self, **kwargs):
        """WDA correlation part with SumOfEOS([MBWR, CS, MFA], factors=[1, -1, -1])
        (cmmdft/functionals.py:339-362); a = 0.5 integral U of the MFA part if present."""
        from .eos import ModifiedBenedictWebbRubinEOS, CarnahanStarlingEOS, MFAEOS, SumOfEOS
        g = self.system.guest
        a = self.part_dict['MFA'].compute_vdw_a() if 'MFA' in self.part_names else None
        mbwr = ModifiedBenedictWebbRubinEOS(g.mass, g.sigma, g.epsilon)
        cs = CarnahanStarlingEOS(g.mass, g.Rhs)
        mfa = MFAEOS(g.mass, g.sigma, g.epsilon, a=a)
        eos = SumOfEOS(g.mass, [mbwr, cs, mfa], factors=[1, -1, -1])
        wda = WDAVFunctional(self.grid, g.Rhs, eos)
        wda.set_temperature(self.temperature, Rhs=g.Rhs)
        self.add_part(wda)

    def add_lda(self, eos):
        """LDA part of an EOS (cmmdft/functionals.py:256-268; the reference
        passes its temperature as an extra constructor argument there, which
        its LDAFunctional does not take -- the part itself follows
        functionals.py:1085-1114)."""
        eos.set_temperature(self.temperature)
        lda = LDAFunctional(self.grid, eos)
        lda.set_temperature(self.temperature)
        self.add_part(lda)

    def add_wdav(self, eos, **kwargs):
        raise NotImplementedError("the WDA part is not built in this package")

    # ---- device functional used by the solvers
    def device(self):
        """engine.Functional combining the parts (HardSphere [+ MFA] [+ ExtPot])."""
        if self._device is not None:
            return self._device
        names = self.part_names
        for n in names:
            if n not in ('HardSphere', 'MFA', 'ExtPot', 'WDA-V', 'LDA'):
                raise NotImplementedError("part %r has no GPU path" % n)
        if 'WDA-V' in names and 'LDA' in names:
            raise NotImplementedError("the fused pipeline holds one EOS part: WDA-V or LDA")
        if 'HardSphere' not in names:
            raise NotImplementedError("the fused solve needs a HardSphere part")
        hs = self.part_dict['HardSphere']
        plan = self.grid.plan
        torch = _torch()
        V = self.part_dict['ExtPot'].potential_device() if 'ExtPot' in names else \
            torch.zeros(plan.npoints, dtype=torch.float64, device='cuda')
        kst = self.part_dict['MFA'].kst if 'MFA' in names else None
        a = self.part_dict['MFA'].vdw_a if 'MFA' in names else None
        wda = self.part_dict['WDA-V'].eos_struct() if 'WDA-V' in names else \
            (self.part_dict['LDA'].eos_struct() if 'LDA' in names else None)
        self._device = E.Functional(plan, hs.R, self.beta, self.wavelength, V, hs_version_code(hs.version), kst, a,
                                    wda=wda)
        return self._device

    def _part_values(self, rho_np, krho=None):
        """Values of the parts at rho: the fused pipeline when it holds every
        part (the WDA and LDA parts have no standalone value), else part by
        part."""
        if 'HardSphere' in self.part_names:
            return _fused_part_values(self, rho_np)
        if krho is None:
            krho = self.grid.fft(rho_np)
        return [p.value(krho) for p in self.parts]

    def init_tracking(self, fn, rewrite=False):
        self.fn_tracking = fn
        if not os.path.isfile(fn) or self.overwrite or rewrite:
            with open(fn, 'w') as f:
                print("#phase\tstep\t     loading\t         -\u00b5N\t        IdGas\t" +
                      "\t".join("%13s" % p.name for p in self.parts) + "\t        Total", file=f)

    def track(self, chempot, rho, krho=None, iphase=0, write=True, print_out=False, fn=None, unit=1, step=0,
              lower_density=None):
        """Grand potential of rho with its parts (cmmdft/functionals.py:121-174),
        appended as one line (phase, step, loading, -mu N, ideal part, each
        part, total) to the tracking file when one is set.

        The ideal part regularises rho as FreeEnergy.track does (values <= 0,
        or within 1e-8 of 0, -> 1e-30); with ``lower_density`` it clips as
        the solvers' own tracking lines do instead (Solver._get_Omega and
        _clip_density, cmmdft/solver.py:103-148: rho < lower_density ->
        1e-30)."""
        g = self.grid
        rho_np = rho if not hasattr(rho, 'detach') else rho.detach().cpu().numpy()
        N = g.integrate(rho_np)
        if lower_density is None:
            rr = np.where(rho_np <= 0 + np.isclose(rho_np, 0), 1e-30, rho_np)
        else:
            rr = np.where(rho_np < lower_density, 1e-30, rho_np)
        Fid = g.integrate(rr * (np.log(self.wavelength ** 3 * rr) - 1.0)) / self.beta
        G = Fid - chempot * N
        vals = self._part_values(rho_np, krho)
        G += sum(vals)
        if write and (fn or self.fn_tracking):
            with open(fn or self.fn_tracking, 'a') as f:
                print("%6i\t%4i\t%.6e\t%.6e\t% .6e\t" % (iphase, step, N, -chempot * N / unit, Fid / unit) +
                      "\t".join("% .6e" % (v / unit) for v in vals) + "\t% .6e" % (G / unit), file=f)
        return G


def _fused_part_values(fe, rho_np):
    """Free-energy value of every part of ``fe`` at the density rho (numpy),
    in part order, from one evaluation of the fused pipeline: PHI, the MFA
    Parseval sum and the EOS part's sum from its reductions, the external
    part as integral rho V."""
    torch = _torch()
    fn = fe.device()
    plan = fn.plan
    rho_t = torch.as_tensor(np.ascontiguousarray(rho_np, dtype=np.float64), device='cuda').reshape(
        (1,) + tuple(plan.npoints))
    buf = E.Buffers(plan, 1, nwork=fn.nwork)
    buf.part[:, L.STAT_N3MAX, :] = -np.inf
    fn.c1(buf, plan.rfft_yz(rho_t), None, want=2)
    st = _stats_of(plan, buf)
    dr = plan.dr
    by = {'HardSphere': st[L.STAT_PHI] * dr / fn.beta, 'MFA': 0.5 * st[L.STAT_MFA] * dr,
          'WDA-V': st[L.STAT_WDA] * dr, 'LDA': st[L.STAT_WDA] * dr,
          'ExtPot': float((rho_t[0] * fn.V).sum().item()) * dr}
    return [float(by[p.name]) for p in fe.parts]


def _stats_of(plan, buf):
    E.finalize(buf, (1 << L.NSTAT) - 1)
    return buf.stats.cpu().numpy()[0]


class HardSphereFunctional(Functional):
    """Hard-sphere FMT part (cmmdft/functionals.py:375-618)."""
    name = 'HardSphere'

    def __init__(self, grid, Rhs, version='atWBII'):
        self.grid = grid
        self.R = Rhs
        self.version = version
        self.code = hs_version_code(version)
        self.temperature = None
        self.beta = None

    def copy(self, grid=None):
        return type(self)(grid or self.grid.copy(), self.R, self.version)

    def set_temperature(self, temperature, Rhs=None, **kwargs):
        self.temperature = temperature
        self.beta = 1 / (boltzmann * temperature)
        if Rhs is not None:
            self.R = Rhs

    def _functional(self):
        torch = _torch()
        plan = self.grid.plan
        return E.Functional(plan, self.R, self.beta, 1.0, torch.zeros(plan.npoints, dtype=torch.float64,
                                                                       device='cuda'), self.code)

    def _run(self, krho, want):
        krho = self.grid.as_spectrum(krho)
        fn = self._functional()
        buf = E.Buffers(fn.plan, 1, nwork=fn.nwork)
        buf.part[:, L.STAT_N3MAX, :] = -np.inf
        chat = fn.plan.new_spec(1) if want & 1 else None
        fn.c1(buf, krho.data, chat, want=want)
        return fn, buf, chat

    def derive(self, krho):
        """dF_HS/drho (Hartree) as a numpy field."""
        fn, buf, chat = self._run(krho, 1)
        return fn.plan.irfft_yz(chat)[0].cpu().numpy()

    def value(self, krho, local=False):
        if local:
            raise NotImplementedError("local hard-sphere free-energy density is not exposed")
        fn, buf, chat = self._run(krho, 2)
        st = _stats_of(fn.plan, buf)
        return (st[L.STAT_PHI] * self.grid.dr) / self.beta

    def get_n3(self, krho):
        raise NotImplementedError("the n3 field is not exposed; max n3 is a solver reduction")


class MFAFunctional(Functional):
    """Mean-field attraction part (cmmdft/functionals.py:770-939)."""
    name = 'MFA'

    def __init__(self, grid, tailcorrections=False, repetitions=[2, 2, 2]):
        self.grid = grid
        self.tailcorrections = tailcorrections
        self.repetitions = list(repetitions)
        if tailcorrections and len(set(self.repetitions)) != 1:
            raise NotImplementedError("tail corrections need equal repetitions per axis")
        self.kst = None
        self.vdw_a = None
        self.params = None

    def copy(self, grid=None):
        m = type(self)(grid or self.grid.copy(), self.tailcorrections, self.repetitions)
        m.kst, m.vdw_a, m.params = self.kst, self.vdw_a, self.params
        return m

    def generate_potential_lj(self, sigma, epsilon, rmin=None, limit_potential=0, cutoff=None, **kwargs):
        rep = self.repetitions[0] if self.tailcorrections else 1
        self.kst, self.vdw_a = E.mfa_kernel_spectrum(self.grid.plan, sigma, epsilon, cutoff, rmin=rmin,
                                                     limit=limit_potential, rep=rep)
        self.params = dict(sigma=sigma, epsilon=epsilon, rmin=rmin, limit=limit_potential, cutoff=cutoff)

    def compute_vdw_a(self):
        self.a = self.vdw_a
        return self.a

    def derive(self, krho):
        krho = self.grid.as_spectrum(krho)
        torch = _torch()
        plan = self.grid.plan
        fn = E.Functional(plan, 1.0, 1.0, 1.0, torch.zeros(plan.npoints, dtype=torch.float64, device='cuda'),
                          L.NOHS, self.kst)
        buf = E.Buffers(plan, 1)
        chat = plan.new_spec(1)
        fn.c1(buf, krho.data, chat, want=1)
        return plan.irfft_yz(chat)[0].cpu().numpy()

    def value(self, krho, local=False):
        rho = self.grid.ifft(krho)
        d = self.derive(krho)
        if local:
            return 0.5 * rho * d
        return 0.5 * self.grid.integrate(rho * d)


class WDAVFunctional(Functional):
    """Weighted-density approximation of an EOS excess free energy
    (cmmdft/functionals.py:1116-1184).  Evaluated inside the fused functional
    pipeline (FreeEnergy.device()); the EOS must be the SumOfEOS of
    add_correlation_wda_lj (MBWR, Carnahan-Starling and mean-field terms)."""
    name = 'WDA-V'

    def __init__(self, grid, Rhs, eos):
        self.grid = grid
        self.R = Rhs
        self.eos = eos
        self.temperature = None

    def copy(self, grid=None):
        return type(self)(grid or self.grid.copy(), self.R, self.eos)

    def set_temperature(self, temperature, Rhs=None, **kwargs):
        self.temperature = temperature
        if Rhs is not None:
            self.R = Rhs
        self.D = 2 * self.R
        self.eos.set_temperature(temperature)

    def eos_struct(self):
        return eos_struct(self.eos, self.D)

    def derive(self, krho):
        raise NotImplementedError("the WDA part is evaluated inside FreeEnergy.device()'s fused pipeline")

    def value(self, krho, local=False):
        raise NotImplementedError("the WDA part is evaluated inside FreeEnergy.device()'s fused pipeline")


def eos_struct(eos, D):
    """cmm_wda_eos of an EOS the GPU evaluates: MBWR, Carnahan-Starling, the
    mean-field EOS, or a SumOfEOS with at most one of each (cmmdft/eos.py);
    D is the weight diameter of a WDA part, or -1 for the LDA part."""
    from .eos import ModifiedBenedictWebbRubinEOS, CarnahanStarlingEOS, MFAEOS, SumOfEOS
    if isinstance(eos, SumOfEOS):
        comps = list(zip(eos.list_eos, eos.factors))
    else:
        comps = [(eos, 1.0)]
    w = L.WdaEos()
    w.D = D
    w.gamma = 3.0
    seen = set()
    for e, f in comps:
        kind = type(e)
        if kind in seen or kind not in (ModifiedBenedictWebbRubinEOS, CarnahanStarlingEOS, MFAEOS):
            raise NotImplementedError("the GPU EOS parts evaluate MBWR, CS and MFA terms, one of each")
        seen.add(kind)
        if kind is ModifiedBenedictWebbRubinEOS:
            w.sigma3, w.epsilon, w.gamma = e.sigma ** 3, e.epsilon, e.gamma
            for i in range(8):
                w.a[i] = e.a[i]
            for i in range(6):
                w.b[i] = e.b[i]
            w.factors[0] = f
        elif kind is CarnahanStarlingEOS:
            w.eta, w.kT = e.eta, boltzmann * e.temperature
            w.factors[1] = f
        else:
            w.a_mfa = e.a
            w.factors[2] = f
    return w


class LDAFunctional(Functional):
    """Local density approximation of an EOS excess free energy
    (cmmdft/functionals.py:1085-1114): dF/drho = f'_EOS(rho), F = integral
    f_EOS(rho).  Evaluated inside the fused functional pipeline
    (FreeEnergy.device()) as the WDA machinery with weight 1; the EOS must be
    one the GPU evaluates (see ``eos_struct``).  A FreeEnergy holds at most
    one of the LDA and WDA parts."""
    name = 'LDA'

    def __init__(self, grid, eos):
        self.grid = grid
        self.eos = eos
        self.temperature = None

    def copy(self, grid=None):
        return type(self)(grid or self.grid.copy(), self.eos)

    def set_temperature(self, temperature, **kwargs):
        self.temperature = temperature
        self.eos.set_temperature(temperature)

    def eos_struct(self):
        return eos_struct(self.eos, -1.0)

    def derive(self, krho):
        raise NotImplementedError("the LDA part is evaluated inside FreeEnergy.device()'s fused pipeline")

    def value(self, krho, local=False):
        raise NotImplementedError("the LDA part is evaluated inside FreeEnergy.device()'s fused pipeline")


class ExternalPotential(Functional):
    """External potential part (cmmdft/functionals.py:941-1083).

    Spherical LJ guests: the LJ potential of the host atoms
    (extpot_calculator.py:186-222).  Multi-site guests (NonSphericalGuest,
    DualModelGuest): the orientation average of their sites' LJ potentials at
    the temperature (extpot_calculator.py:569-655), regenerated by
    set_temperature.  Both on the GPU.
    """
    name = 'ExtPot'

    def __init__(self, grid, system, epot_dr=None, limit_potential=1e4 * kjmol, degree=9, interpolate=False,
                 cutoff=12 * angstrom):
        self.grid = grid
        self.system = system
        self.host = system.host
        self.guest = system.guest
        self.epot_dr = epot_dr
        self.limit_potential = limit_potential
        self.degree = degree
        self.interpolate = interpolate
        self.cutoff = cutoff
        self._V = None

    def copy(self, grid=None):
        e = type(self)(grid or self.grid.copy(), self.system, self.epot_dr, self.limit_potential, self.degree,
                       self.interpolate, self.cutoff)
        e._V = self._V
        return e

    def set_temperature(self, temperature, **kwargs):
        """A multi-site guest's potential depends on the temperature: it is
        generated for a new one unless its file exists (functionals.py:
        1019-1025; the reference then keeps the potential it has, and leaves
        a regenerated one uncapped -- here it is capped like every other)."""
        from .system import NonSphericalGuest
        if not isinstance(self.guest, NonSphericalGuest):
            return
        fn = None
        if self.epot_dr is not None:
            fn = Path(self.epot_dr) / ('eff_epot_%s.npy' % format_temperature(temperature))
            if fn.exists():
                return
        self.generate_potential(temperature)
        if fn is not None:
            self.dump_potential(fn)
        self.cap()

    def _host_arrays(self):
        h = self.host
        if not hasattr(h, 'ff') or h.ff is None:
            raise NotImplementedError("generate_potential needs a host with LJ parameters")
        sig = np.array([h.ff[t][0] for t in h.ffatypes])
        eps = np.array([h.ff[t][1] for t in h.ffatypes])
        return h.recentred_pos(), h.ffatype_ids, sig, eps

    # fine grid of the interpolated path and the interpolator's spacing
    # (cmmdft/functionals.py:1039, 1047: both 0.15 angstrom)
    INTERP_SPACING = 0.15 * angstrom
    DERIV_VMAX = 1e+6 * kjmol            # clip of get_external_potential_derivatives

    def _interpolated(self, pos, ids, sig, eps, rot, w, beta):
        """interpolate=True (functionals.py:1032-1055): for every guest atom
        type the eight LJ channels on a grid of spacing 0.15 A over the cell,
        then the orientational average with tricubic interpolation, the
        interpolator at the solve grid's first point with spacing 0.15 A on
        every axis (as the reference sets it, not the fine grid's own
        spacing)."""
        torch = _torch()
        g = self.guest
        h = self.host
        rv = h.cell.rvecs
        lengths = np.linalg.norm(rv, axis=1)
        fine_n = [int(np.ceil(l / self.INTERP_SPACING)) for l in lengths]
        fine_sp = [np.linalg.norm(rv[:, a]) / fine_n[a] for a in range(3)]
        if g.ff is None:
            raise ValueError("guest %s has no LJ parameters (par file or ff)" % g.name)
        types = list(g.mol.ffatypes)
        tables = torch.empty((len(types), 8) + tuple(fine_n), dtype=torch.float64, device='cuda')
        for k, t in enumerate(types):
            sg, eg = g.ff[t]
            E.external_potential_derivatives(rv, fine_n, fine_sp, pos, ids, sig, eps, sg, eg, self.cutoff,
                                             self.DERIV_VMAX, out=tables[k])
        origin = self.grid.points[0, 0, 0, :3]
        spacing = np.array([1.0, 1.0, 1.0]) * self.INTERP_SPACING
        V = E.effective_potential_interpolated(self.grid.plan, tables, g.mol.ffatype_ids, origin, spacing,
                                               g.mol.pos, g.mol.masses, rot, w, beta, self.limit_potential)
        del tables
        return V

    def generate_potential(self, temperature=None, rewrite=False):
        """The potential on the grid, uncapped above limit_potential for
        multi-site guests and capped for spherical ones (cap() caps both)."""
        from .system import NonSphericalGuest
        from .rotations import combined_rotations
        pos, ids, sig, eps = self._host_arrays()
        g = self.guest
        if isinstance(g, NonSphericalGuest):
            if temperature is None:
                raise ValueError('Temperature must be provided for non-spherical particles')
            beta = 1 / temperature / boltzmann
            rot, w = combined_rotations(self.degree)
            if self.interpolate:
                self._V = self._interpolated(pos, ids, sig, eps, rot, w, beta)
            else:
                ssig, seps = g.site_parameters()
                self._V = E.effective_potential(self.grid.plan, pos, ids, sig, eps, g.mol.pos, g.mol.masses, ssig,
                                                seps, rot, w, self.cutoff, beta, self.limit_potential)
        else:
            self._V = E.external_potential(self.grid.plan, pos, ids, sig, eps, g.sigma, g.epsilon, self.cutoff,
                                           self.limit_potential)

    def cap(self):
        torch = _torch()
        V = self._V
        V = torch.where(torch.isfinite(V), V, torch.full_like(V, self.limit_potential))
        self._V = torch.clamp(V, max=self.limit_potential)

    def load_potential(self, fn):
        torch = _torch()
        pot = np.load(fn)
        shape = tuple(self.grid.npoints)
        if pot.shape == tuple(n + 1 for n in shape):
            pot = pot[:-1, :-1, :-1]
        elif pot.shape != shape:
            raise ValueError('Grid shape %s does not match potential shape %s' % (shape, pot.shape))
        self._V = torch.as_tensor(np.ascontiguousarray(pot, dtype=np.float64), device='cuda')

    def dump_potential(self, fn):
        np.save(fn, self.potential)

    def potential_device(self):
        return self._V

    @property
    def potential(self):
        return self._V.cpu().numpy()

    def derive(self, krho):
        return self.potential

    def value(self, krho, local=False):
        rho = self.grid.ifft(krho)
        if local:
            return rho * self.potential
        return self.grid.integrate(rho * self.potential)
