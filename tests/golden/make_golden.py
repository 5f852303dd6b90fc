"""Generate golden fixtures by running the UNMODIFIED reference package.

Run in the build container only (the reference tree is not present on GPU
machines):

    python tests/golden/make_golden.py --reference <reference tree> [--skip64]
    python tests/golden/make_golden.py --reference <reference tree> --iso64 [--procs 8]
    python tests/golden/make_golden.py --reference <reference tree> --qn
    python tests/golden/make_golden.py --reference <reference tree> --dropin
    python tests/golden/make_golden.py --reference <reference tree> --uneven
    python tests/golden/make_golden.py --reference <reference tree> --lda
    python tests/golden/make_golden.py --reference <reference tree> --rot
    python tests/golden/make_golden.py --reference <reference tree> --rotinterp
    python tests/golden/make_golden.py --reference <reference tree> --proj
    python tests/golden/make_golden.py --reference <reference tree> --fire

``--reference`` (or the environment variable CMM_REFERENCE_ROOT) names the
root of the reference's source tree, the directory that holds ``cmmdft/``.

The reference is imported from its own source tree through the import shims
in ``tests/golden/refshim`` (molmod units/constants backed by
``cmmdft_b200.units``, a minimal yaff ``System``/``Cell``, a matplotlib stub)
plus the ``np.complex_`` alias that numpy 2 removed.  Hosts are built by
setting attributes (the shim cannot read yaff checkpoints); the external
potential is computed by the reference's own ``get_external_potential`` and
handed to ``FreeEnergy.add_external_potential(load_fn=...)`` so its capping
code runs too.

Outputs (small ``.npz`` files) land next to this script:
  c0_32.npz   32^3 cubic host: V, two C1 evaluations, Omega parts,
              static-Picard trajectory and converged density,
              tight hybrid-Anderson solution, tail-corrected MFA.
  c1_64.npz   64^3 cubic host: V summary and tight hybrid-Anderson solutions
              at three pressures (scalars + one density field).
  qn32.npz    the 32^3 case at 1 bar solved by the reference's QuasiNewton
              (RES < 1e-8, Ninit = rho_bulk) for five direction / line-search
              variants: N, Omega, steps (``--qn`` only).
  iso64_res8.npz  the 24-pressure 64^3 isotherm (1e-3..100 bar) solved as
              the reference's example does it: hybrid Anderson m=5 to
              RES < 1e-8 from Ninit = rho_bulk; N, Omega, steps and the
              convergence flag per pressure, the helium void fraction and
              the excess uptake from the reference's own
              Calculator.return_loading(excess=True) (``--iso64`` only; one
              process per pressure).
  dropin32.npz    the 32^3 case driven through the reference's public API:
              Program -> FreeEnergy.add_* -> Program.cascade_solver (static
              Picard for 3 steps, then hybrid Anderson to RES < 1e-13 and
              RIUE < 1e-12, continue_solving=True); Program.solve with
              Ninit = rho_bulk (float) under hybrid Anderson to RES < 1e-8
              with track_history=True (the history's N, Omega, RES, RIUE and
              DER columns); and Calculator.return_loading (absolute and
              excess), free_energy_contrib per part and grand_potential of
              both solutions (``--dropin`` only).
  uneven5.npz     host 5 of the uneven batch (uneven_hosts(8, 2)) on its
              0.25 A grid, 119 x 157 x 125 (157 prime: Rader stages on the
              GPU), at 0.1, 1 and 10 bar: N, Omega, steps (``--uneven``).
  lda32.npz       the 32^3 case with an LDA part (SumOfEOS of MBWR, CS and
              the mean-field EOS): part values, the LDA derivative, C1 and
              Omega of the two profiles, three static Picard steps and their
              rounding floor (the same steps from a start one ulp above)
              (``--lda``).
  rot20.npz       the orientation-averaged external potential of rigid CO2
              (the reference's InputFiles/Guest/CO2 struct_AA.chk and
              pars_vdw_AA_trappe.txt) in the 32^3 case's host on a 20^3
              grid at 300 K, from the reference's own
              generate_effective_potential and get_external_potential_dict
              (their file readers answered from memory), at Lebedev degrees 9
              and 11; with the reference's rotation matrices and weights and
              the guest's arrays (``--rot``).
  rotinterp12.npz the same guest and host through the reference's
              ExternalPotential.generate_potential(interpolate=True) on a
              12^3 grid at Lebedev degree 9 (derivative grids at 0.15 A,
              tricubic interpolation), with the channel values of
              get_external_potential_derivatives at 3000 seeded points of
              each type's derivative grid (``--rotinterp``).
  proj32.npz      the reference's Calculator post-processing of three
              converged 32^3 densities (0.1, 1 and 10 bar, Program.solve,
              hybrid Anderson to RES < 1e-8): collective_variable along a
              tilted axis (3 x 3 x 3 supercell, 3 A from the axis) and from
              ring atoms, project_density, save_loading_and_grand_potential,
              free_energy_path and project_contributions('fid',
              'pure_extpot'); with the densities themselves (``--proj``).
  fire32.npz      the reference's Fire solver ('abc-fire' and 'fire') on
              the 32^3 case at 1 bar from Ninit = rho_bulk, RES < 1e-6, the
              mask (which the reference reads but never sets) = rho0 > 0:
              steps, N, density and the final dt, alpha, N_pos, N_neg; a
              second 'abc-fire' solve with the same solver object (its
              counters carry over); and the first solves' rounding floors
              (the same solves with the density moved one ulp up before
              every update) (``--fire``).
  iso64_rho.npz   the converged densities of that isotherm at the pressure
              indices ISO_RHO_IDX, and the reference run against itself: the
              same points re-solved from a start perturbed by one ulp, with
              the relative differences of rho, N and Omega that this causes
              (the trajectory's own rounding floor).
"""

import argparse
import contextlib
import io
import os
import sys
import tempfile
import time
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# Converged-solution fixtures are taken well below the reference's default
# tolerance: RES normalises by sqrt(N), so RES < 1e-11 pins rho only to ~1e-8;
# RES < 1e-13 (its noise floor is ~8e-14 at 32^3) plus RIUE < 1e-12 keeps
# low-loading points equally tight.
TIGHT_CRIT = ['res', 'riue']
TIGHT_THR = [1e-13, 1e-12]
REPO = os.path.dirname(os.path.dirname(HERE))


def import_reference(ref_root):
    sys.path.insert(0, REPO)
    sys.path.insert(0, os.path.join(HERE, 'refshim'))
    sys.path.insert(0, ref_root)
    if not hasattr(np, 'complex_'):
        np.complex_ = np.complex128
    import cmmdft  # noqa: F401
    from cmmdft import system, functionals, solver, extpot_calculator, eos
    from cmmdft.log import log as reflog
    reflog.set_level(0)
    return system, functionals, solver, extpot_calculator, eos


def build(ref, npts, host, T, P_bar, tmp, tail=False, wda=False):
    system, functionals, solver, extpot, eos = ref
    import yaff
    from cmmdft_b200.units import bar, angstrom
    from cmmdft_b200.hosts import methane_guest_params
    sig, eps, mass = methane_guest_params()
    mol = yaff.System(pos=host.pos.copy(), ffatypes=host.ffatypes,
                      ffatype_ids=host.ffatype_ids, rvecs=host.rvecs)
    mol.pos -= mol.pos.sum(axis=0) / len(mol.pos)  # as system.py:70
    h = system.NanoporousHost.__new__(system.NanoporousHost)
    system.Host.__init__(h, 'synthetic', mol.cell)
    h.mol, h.chk, h.par = mol, None, None
    guest = system.SphericalLJGuest('CH4', mass, sig, eps)
    syst = system.System(h, guest)
    grid = system.Grid(mol.cell, npoints=npts)
    pts = grid.points[..., :3].reshape(-1, 3)
    t0 = time.time()
    V = extpot.get_external_potential(pts, host.ff, sig, eps, mol, cutoff=12 * angstrom)
    t_ext = time.time() - t0
    fn = os.path.join(tmp, 'epot_%s.npy' % '_'.join(str(n) for n in np.atleast_1d(npts)))
    np.save(fn, V.reshape(grid.npoints))
    fe = functionals.FreeEnergy(grid, syst, T, workdir=tmp, name_dict={}, overwrite=True)
    fe.add_hard_sphere(version='WBII')
    fe.add_mean_field(tailcorrections=tail, cutoff=12 * angstrom, rewrite=True)
    fe.add_external_potential(load_fn=fn)
    if wda:
        fe.add_correlation_wda_lj()
    fe.set_temperature(T)  # user flow after adding parts (methane_ZIF8.ipynb)
    mb = eos.ModifiedBenedictWebbRubinEOS(mass, sig, eps)
    mu = mb.calculate_mu(T, P_bar * bar)
    prog = types.SimpleNamespace(grid=grid, fener=fe)
    return dict(grid=grid, fe=fe, mu=mu, prog=prog, V_raw=V, t_ext=t_ext, mbwr=mb,
                guest=guest, mol=mol, host=h)


def omega_parts(ref, b, rho, mu):
    solver = ref[2]
    s = solver.Picard(b['prog'], nsteps=1, method='static')
    s._initiate_solving(mu)
    krho = b['grid'].fft(rho)
    parts = [p.value(krho) for p in b['fe'].parts]
    om = s._get_Omega(rho, krho)
    derivs = [p.derive(krho) for p in b['fe'].parts]
    C1 = s._get_C1(rho, krho)
    return parts, om, derivs, C1


def quiet(fn, *a, **k):
    buf = io.StringIO()
    with contextlib.redirect_stdout(buf):
        return fn(*a, **k)


ISO_PRESSURES = np.logspace(-3, 2, 24)


# pressure indices whose converged densities are kept: 1e-3, 1.1 and 8.2 bar
ISO_RHO_IDX = (0, 14, 18)


def _iso64_point(task):
    ref_root, i, perturb = task
    ref = import_reference(ref_root)
    solver = ref[2]
    from cmmdft_b200.hosts import cubic_host_276
    from cmmdft_b200.units import bar, boltzmann
    T = 300.0
    P = ISO_PRESSURES[i]
    b = quiet(build, ref, 64, cubic_host_276(seed=0), T, P, tempfile.mkdtemp(prefix='cmm_iso64_'))
    mb, V = b['mbwr'], b['fe'].part_dict['ExtPot'].potential
    mb.set_temperature(T)
    bulk = np.nanmin(mb.solve_densities_from_chempots([b['mu']]), axis=1)[0]
    rho0 = bulk * np.exp(-np.maximum(V, 0) / boltzmann / T)
    if perturb:
        # one ulp up at every point: the reference's sensitivity to rounding
        rho0 = np.nextafter(rho0, np.inf)
    s = solver.Anderson(b['prog'], nsteps=500, m=5, criterion='res', threshold=1e-8)
    t0 = time.time()
    try:
        N, rho, conv = quiet(s.solve, b['mu'], rho0, 3)
    except Exception as e:  # noqa: BLE001 - recorded, not raised
        print('P=%g bar: %s' % (P, e), flush=True)
        return i, b['mu'], bulk, np.nan, np.nan, s.curr_step, False, None
    print('iso64 P=%.4g bar%s: N=%.12e steps=%d conv=%s (%.0f s)'
          % (P, ' (perturbed start)' if perturb else '', N, s.curr_step, conv, time.time() - t0), flush=True)
    return i, b['mu'], bulk, N, s.omega0, s.curr_step, bool(conv), (rho if conv else None)


def lda32(args):
    """The LDA part (LDAFunctional, cmmdft/functionals.py:1085-1114) on the
    32^3 case: WBII + MFA + ExtPot + LDA of SumOfEOS([MBWR, CS, MFA],
    [1, -1, -1]).  The reference's own FreeEnergy.add_lda passes an extra
    argument to LDAFunctional (functionals.py:267) and its set_temperature
    forwards Rhs to an EOS that does not take it, so the part is built
    directly, added with add_part and given its temperature alone."""
    ref = import_reference(args.reference)
    system, functionals, solver, extpot, eos = ref
    from cmmdft_b200.hosts import cubic_host_276, methane_guest_params
    from cmmdft_b200.units import angstrom
    sig, eps, mass = methane_guest_params()
    T = 300.0
    b = quiet(build, ref, 32, cubic_host_276(seed=0), T, 1.0, tempfile.mkdtemp(prefix='cmm_lda_'))
    fe, grid, mu = b['fe'], b['grid'], b['mu']
    Rhs = b['guest'].Rhs
    a = fe.part_dict['MFA'].compute_vdw_a()
    S = eos.SumOfEOS(mass, [eos.ModifiedBenedictWebbRubinEOS(mass, sig, eps), eos.CarnahanStarlingEOS(mass, Rhs),
                            eos.MFAEOS(mass, sig, eps, a=a)], factors=[1, -1, -1])
    lda = functionals.LDAFunctional(grid, S)
    lda.set_temperature(T)
    fe.add_part(lda)
    out = dict(mu=mu, T=T)
    V = fe.part_dict['ExtPot'].potential
    rho_a = np.exp(fe.beta * (mu - V)) / fe.wavelength ** 3
    from cmmdft_b200.units import angstrom as A
    rho_b = 0.02 / A ** 3 * np.clip(np.exp(-fe.beta * V), 0, 1)
    for tag, rho in (('a', rho_a), ('b', rho_b)):
        parts, om, derivs, C1 = quiet(omega_parts, ref, b, rho, mu)
        out['values_' + tag] = np.array(parts)
        out['omega_' + tag] = om
        out['dLDA_' + tag] = derivs[3]
        out['C1_' + tag] = C1
    s = solver.Picard(b['prog'], nsteps=3, alpha_mix=0.1, method='static', criterion='res', threshold=1e-8)
    N, rho, conv = quiet(s.solve, mu, rho_a.copy(), 3)
    out.update(picard3_rho=rho, picard3_N=N)
    # the reference against itself from a start one ulp above: the rounding
    # floor of the three-step trajectory
    s2 = solver.Picard(b['prog'], nsteps=3, alpha_mix=0.1, method='static', criterion='res', threshold=1e-8)
    N2, rho2, _ = quiet(s2.solve, mu, np.nextafter(rho_a, np.inf), 3)
    out['picard3_floor'] = np.max(np.abs(rho2 - rho)) / np.max(np.abs(rho))
    out['picard3_N_floor'] = abs(N2 - N) / abs(N)
    np.savez_compressed(os.path.join(HERE, 'lda32.npz'), **out)
    print('wrote lda32.npz', {k: v for k, v in out.items() if np.ndim(v) == 0})


UNEVEN_HOST = 5                       # uneven_hosts(8, 2)[5]: 119 x 157 x 125 (prime 157), 2026 atoms
UNEVEN_PRESSURES = (0.1, 1.0, 10.0)   # bar


def _uneven_point(task):
    ref_root, P_bar = task
    ref = import_reference(ref_root)
    solver = ref[2]
    from cmmdft_b200.hosts import uneven_hosts
    from cmmdft_b200.units import boltzmann, angstrom
    T = 300.0
    host = uneven_hosts(8, 2)[UNEVEN_HOST]
    npts = [int(np.ceil(np.linalg.norm(host.rvecs[:, a]) / (0.25 * angstrom))) for a in range(3)]
    b = quiet(build, ref, npts, host, T, P_bar, tempfile.mkdtemp(prefix='cmm_uneven_'))
    mb, V = b['mbwr'], b['fe'].part_dict['ExtPot'].potential
    mb.set_temperature(T)
    bulk = np.nanmin(mb.solve_densities_from_chempots([b['mu']]), axis=1)[0]
    rho0 = bulk * np.exp(-np.maximum(V, 0) / boltzmann / T)
    s = solver.Anderson(b['prog'], nsteps=500, m=5, criterion='res', threshold=1e-8)
    t0 = time.time()
    N, rho, conv = quiet(s.solve, b['mu'], rho0, 3)
    print('uneven host %d %s P=%g bar: N=%.12e steps=%d conv=%s (%.0f s)'
          % (UNEVEN_HOST, npts, P_bar, N, s.curr_step, conv, time.time() - t0), flush=True)
    return P_bar, b['mu'], bulk, N, s.omega0, s.curr_step, bool(conv), npts


def uneven(args):
    """One host of the uneven batch at its spacing-derived grid (a Rader
    prime on y), hybrid Anderson m=5 to RES < 1e-8 from Ninit = rho_bulk."""
    import multiprocessing as mp
    with mp.get_context('spawn').Pool(len(UNEVEN_PRESSURES)) as pool:
        res = pool.map(_uneven_point, [(args.reference, p) for p in UNEVEN_PRESSURES])
    cols = list(zip(*res))
    out = dict(host=UNEVEN_HOST, npoints=np.array(cols[7][0]), pressures=np.array(cols[0]), mu=np.array(cols[1]),
               rho_bulk=np.array(cols[2]), N=np.array(cols[3]), omega=np.array(cols[4]), steps=np.array(cols[5]),
               converged=np.array(cols[6]))
    np.savez_compressed(os.path.join(HERE, 'uneven5.npz'), **out)
    print('wrote uneven5.npz')


QN_CASES = [('bfgs', 'backtracking'), ('broyden', 'backtracking'), ('cg', 'backtracking'), ('bfgs', 'quadratic'),
            ('bfgs', 'none')]


def dropin32(args):
    """The reference's own Program / Solver / Calculator flow on the 32^3 case."""
    from pathlib import Path
    ref = import_reference(args.reference)
    system, functionals, solver, extpot, eos = ref
    from cmmdft import program as rprogram, calculator as rcalculator
    import yaff
    from cmmdft_b200.hosts import cubic_host_276, methane_guest_params, HELIUM
    from cmmdft_b200.units import angstrom, boltzmann, bar
    T = 300.0
    host = cubic_host_276(seed=0)
    sig, eps, mass = methane_guest_params()
    mol = yaff.System(pos=host.pos.copy(), ffatypes=host.ffatypes, ffatype_ids=host.ffatype_ids, rvecs=host.rvecs,
                      masses=host.masses)
    mol.pos -= mol.pos.sum(axis=0) / len(mol.pos)  # as system.py:70
    h = system.NanoporousHost.__new__(system.NanoporousHost)
    system.Host.__init__(h, 'synthetic', mol.cell)
    h.mol, h.chk, h.par = mol, None, None
    guest = system.SphericalLJGuest('CH4', mass, sig, eps)
    tmp = tempfile.mkdtemp(prefix='cmm_dropin_')
    grid0 = system.Grid(mol.cell, npoints=32)
    V = extpot.get_external_potential(grid0.points[..., :3].reshape(-1, 3), host.ff, sig, eps, mol,
                                      cutoff=12 * angstrom)
    vfn = os.path.join(tmp, 'epot_32.npy')
    np.save(vfn, V.reshape(grid0.npoints))
    Vhe = extpot.get_external_potential(grid0.points[..., :3].reshape(-1, 3), host.ff,
                                        HELIUM['sigma'] * angstrom, HELIUM['epsilon_K'] * boltzmann, mol,
                                        cutoff=12 * angstrom)
    he = grid0.integrate(np.clip(np.exp(-Vhe / boltzmann / T), 0, 1)).real / grid0.cell.volume

    def program(suffix):
        prog = rprogram.Program(prefix=tmp, hostname='synthetic', guestname='CH4', ff_suffix='trappe_uff',
                                suffix=suffix)
        prog.set_system(h, guest)
        prog.set_grid(npoints=32)
        prog.init_free_energy(T)
        prog.fener.add_hard_sphere(version='WBII')
        prog.fener.add_mean_field(cutoff=12 * angstrom, rewrite=True)
        prog.fener.add_external_potential(load_fn=vfn)
        prog.fener.set_temperature(T)
        return prog

    mb = eos.ModifiedBenedictWebbRubinEOS(mass, sig, eps)
    mu = mb.calculate_mu(T, 1.0 * bar)
    mb.set_temperature(T)
    bulk = float(np.nanmin(mb.solve_densities_from_chempots([mu]), axis=1)[0])
    out = dict(T=T, mu=mu, rho_bulk=bulk, he_frac=he)
    # A: cascade, static Picard (3 steps, not converged) then tight hybrid Anderson
    pa = program('cascade')
    sv = [solver.Picard(pa, nsteps=3, alpha_mix=0.1, method='static', criterion='res', threshold=1e-8),
          solver.Anderson(pa, nsteps=500, m=5, criterion=TIGHT_CRIT, threshold=TIGHT_THR)]
    quiet(pa.cascade_solver, sv, mu, continue_solving=True)
    rho = np.load(pa.rho_fn)
    out.update(cascade_rho=rho, cascade_N=pa.grid.integrate(rho).real, cascade_steps=np.array([s.curr_step for s in sv]),
               cascade_omega=sv[1].omega0)
    # B: Program.solve from Ninit = rho_bulk (float), RES < 1e-8, history tracked
    pb = program('ninit')
    sb = solver.Anderson(pb, nsteps=500, m=5, criterion='res', threshold=1e-8, track_history=True)
    pb.set_solver(sb)
    N, rho, conv = quiet(pb.solve, mu, Ninit=bulk)
    out.update(ninit_rho=rho, ninit_N=N, ninit_conv=conv, ninit_steps=sb.curr_step, ninit_omega=sb.omega0,
               ninit_history=sb.history[:sb.curr_step + 1, :5].copy())
    # energy tracking (Program.solve's default): the start and final lines
    conv_fn = os.path.join(pb.workdir, 'convergence_%s.txt' % pb.file_suffix)
    with open(conv_fn) as f:
        lines = [l.split() for l in f if l.strip() and not l.startswith('#')]
    out['ninit_track_first'] = np.array([float(x) for x in lines[0]])
    out['ninit_track_last'] = np.array([float(x) for x in lines[-1]])
    # The reference against itself: both flows again from a start one ulp
    # above the nominal one (the ideal-gas start of A given as an array),
    # recording the relative change of each observable (the rounding floor
    # of a comparison along separate trajectories).
    pa2, pb2 = program('cascade_ulp'), program('ninit_ulp')
    sv2 = [solver.Picard(pa2, nsteps=3, alpha_mix=0.1, method='static', criterion='res', threshold=1e-8),
           solver.Anderson(pa2, nsteps=500, m=5, criterion=TIGHT_CRIT, threshold=TIGHT_THR)]
    V32 = pa2.fener.part_dict['ExtPot'].potential
    rho_ig = np.exp(pa2.fener.beta * (mu - V32)) / pa2.fener.wavelength ** 3
    quiet(pa2.cascade_solver, sv2, mu, continue_solving=True, Ninit=np.nextafter(rho_ig, np.inf))
    sb2 = solver.Anderson(pb2, nsteps=500, m=5, criterion='res', threshold=1e-8)
    pb2.set_solver(sb2)
    V0 = pb2.fener.part_dict['ExtPot'].potential
    quiet(pb2.solve, mu, Ninit=np.nextafter(bulk * np.exp(-np.maximum(V0, 0) / boltzmann / T), np.inf))
    out['cascade_ulp_steps'] = np.array([x.curr_step for x in sv2])
    out['ninit_ulp_steps'] = sb2.curr_step
    # Calculator observables of both solutions (and of the perturbed runs)
    for tag, prog in (('cascade', pa), ('ninit', pb), ('cascade_ulp', pa2), ('ninit_ulp', pb2)):
        # Calculator.__init__ (calculator.py:27-35) copies the FreeEnergy, whose
        # host copy re-reads a yaff checkpoint that the synthetic host does not
        # have: set the same attributes around the program's own objects.
        calc = rcalculator.Calculator.__new__(rcalculator.Calculator)
        calc.program, calc.name_dict, calc.workdir = prog, prog.name_dict, prog.workdir
        calc.grid, calc.fener = prog.grid, prog.fener
        calc.host, calc.guest, calc.label = prog.system.host, prog.system.guest, None
        out[tag + '_loading'] = calc.return_loading(T, [mu])[0]
        out[tag + '_excess'] = calc.return_loading(T, [mu], excess=True, eos=mb, He_frac=he)[0]
        out[tag + '_grand_potential'] = quiet(calc.grand_potential, T, mu)
        for part in ('fid', 'HardSphere', 'MFA', 'ExtPot'):
            out['%s_F_%s' % (tag, part)] = quiet(calc.free_energy_contrib, T, mu, part)
        if tag.endswith('_ulp'):
            rho = np.load(prog.rho_fn)
            out[tag + '_rho'] = rho
        if tag == 'ninit':   # the loading exports (calculator.py:186-340)
            f1 = calc.save_loadings(T, [mu], fn=os.path.join(tmp, 'loads.csv'))
            calc.save_loadings(T, [mu], pressure=True, eos=mb, fn=os.path.join(tmp, 'loads_P.csv'))
            calc.save_loadings_AIF(T, chempots=np.array([mu]), eos=mb, user='tester', loading_unit='mol/kg',
                                   fn=os.path.join(tmp, 'ads.aif'))
            for key, name in (('csv', 'loads.csv'), ('csv_P', 'loads_P.csv'), ('aif', 'ads.aif')):
                with open(os.path.join(tmp, name)) as f:
                    out['ninit_' + key] = np.array(f.read())
            del f1
    for tag in ('cascade', 'ninit'):
        base, pert = tag, tag + '_ulp'
        fl = dict(rho=float(np.max(np.abs(out[pert + '_rho'] - out[base + '_rho'])) / np.max(np.abs(out[base + '_rho']))))
        for q in ('loading', 'excess', 'grand_potential', 'F_fid', 'F_HardSphere', 'F_MFA', 'F_ExtPot'):
            fl[q] = abs(out['%s_%s' % (pert, q)] - out['%s_%s' % (base, q)]) / abs(out['%s_%s' % (base, q)])
        out[tag + '_floor_names'] = np.array(list(fl))
        out[tag + '_floor'] = np.array(list(fl.values()))
        print('%s floor (1-ulp start):' % tag, {k: '%.2e' % v for k, v in fl.items()}, flush=True)
        del out[pert + '_rho']
    for k, v in out.items():
        if np.ndim(v) == 0:
            print('dropin %s = %r' % (k, v), flush=True)
    np.savez_compressed(os.path.join(HERE, 'dropin32.npz'), **out)
    print('wrote dropin32.npz')


def qn32(args):
    """The reference's QuasiNewton on the 32^3 case at 1 bar, RES < 1e-8, from
    Ninit = rho_bulk, for every direction / line-search variant in QN_CASES."""
    ref = import_reference(args.reference)
    solver = ref[2]
    from cmmdft_b200.hosts import cubic_host_276
    from cmmdft_b200.units import boltzmann
    b = quiet(build, ref, 32, cubic_host_276(seed=0), 300.0, 1.0, tempfile.mkdtemp(prefix='cmm_qn_'))
    V = b['fe'].part_dict['ExtPot'].potential
    mb = b['mbwr']
    mb.set_temperature(300.0)
    bulk = np.nanmin(mb.solve_densities_from_chempots([b['mu']]), axis=1)[0]
    rho0 = bulk * np.exp(-np.maximum(V, 0) / boltzmann / 300.0)
    out = dict(mu=b['mu'], rho_bulk=bulk, threshold=1e-8)
    for meth, ls in QN_CASES:
        s = solver.QuasiNewton(b['prog'], nsteps=300, method=meth, line_search=ls, criterion='res',
                               threshold=1e-8, verbose=False)
        N, rho, conv = quiet(s.solve, b['mu'], rho0.copy(), 3)
        tag = '%s_%s' % (meth, ls)
        out[tag + '_N'], out[tag + '_steps'], out[tag + '_conv'] = N, s.curr_step, conv
        out[tag + '_omega'] = s.omega0
        print('qn %s: N=%.12e steps=%d conv=%s' % (tag, N, s.curr_step, conv), flush=True)
    np.savez_compressed(os.path.join(HERE, 'qn32.npz'), **out)
    print('wrote qn32.npz')


def _excess_uptake(ref_root, mus, rhos, T=300.0):
    """He void fraction and the excess uptake of the densities ``rhos`` (None
    where a point did not converge) through the reference's own
    Calculator.return_loading(excess=True) (cmmdft/calculator.py:114-138).
    The fraction is computed as get_helium_fraction intends
    (calculator.py:152-167; its own call of read_pars_file is broken): the
    reference's get_external_potential for helium, clip(exp(-V/kT), 0, 1),
    Grid.integrate, divided by the cell volume."""
    from pathlib import Path
    ref = import_reference(ref_root)
    extpot = ref[3]
    from cmmdft import calculator, tools
    from cmmdft_b200.hosts import cubic_host_276, HELIUM
    from cmmdft_b200.units import angstrom, boltzmann
    host = cubic_host_276(seed=0)
    tmp = tempfile.mkdtemp(prefix='cmm_iso64_nex_')
    b = quiet(build, ref, 64, host, T, 1.0, tmp)
    grid = b['grid']
    Vhe = extpot.get_external_potential(grid.points[..., :3].reshape(-1, 3), host.ff,
                                        HELIUM['sigma'] * angstrom, HELIUM['epsilon_K'] * boltzmann,
                                        b['mol'], cutoff=12 * angstrom)
    he = grid.integrate(np.clip(np.exp(-Vhe / boltzmann / T), 0, 1)).real / grid.cell.volume
    for mu, rho in zip(mus, rhos):
        if rho is not None:
            np.save(os.path.join(tmp, 'rho_%s.npy' % tools.get_file_suffix(mu, T)), rho)
    calc = calculator.Calculator.__new__(calculator.Calculator)
    calc.workdir, calc.grid, calc.host = Path(tmp), grid, b['host']
    Nex = calc.return_loading(T, list(mus), excess=True, eos=b['mbwr'], He_frac=he)
    return float(he), np.asarray(Nex)


def iso64(args):
    import multiprocessing as mp
    n = len(ISO_PRESSURES)
    tasks = [(args.reference, i, False) for i in range(n)] + [(args.reference, i, True) for i in ISO_RHO_IDX]
    with mp.get_context('spawn').Pool(args.procs) as pool:
        allres = pool.map(_iso64_point, tasks)
    res, pert = sorted(allres[:n], key=lambda r: r[0]), allres[n:]
    cols = list(zip(*res))
    he, Nex = _excess_uptake(args.reference, cols[1], cols[7])
    out = dict(pressures=ISO_PRESSURES, mu=np.array(cols[1]), rho_bulk=np.array(cols[2]), N=np.array(cols[3]),
               omega=np.array(cols[4]), steps=np.array(cols[5]), converged=np.array(cols[6]),
               threshold=1e-8, criterion='res', m=5, he_frac=he, N_ex=Nex)
    np.savez_compressed(os.path.join(HERE, 'iso64_res8.npz'), **out)
    print('wrote iso64_res8.npz')
    rout = dict(idx=np.array(ISO_RHO_IDX))
    fl = []
    for j, i in enumerate(ISO_RHO_IDX):
        rho = res[i][7]
        rout['rho_%d' % i] = rho
        p = pert[j]
        d_rho = float(np.max(np.abs(p[7] - rho)) / np.max(np.abs(rho)))
        d_N = abs(p[3] - res[i][3]) / abs(res[i][3])
        d_om = abs(p[4] - res[i][4]) / abs(res[i][4])
        fl.append((d_rho, d_N, d_om, p[5]))
        print('floor P=%.4g bar: rho %.3e  N %.3e  Omega %.3e  steps %d vs %d'
              % (ISO_PRESSURES[i], d_rho, d_N, d_om, p[5], res[i][5]), flush=True)
    rout['floor'] = np.array(fl)   # per index: rel. diff of rho, N, Omega; steps of the perturbed run
    np.savez_compressed(os.path.join(HERE, 'iso64_rho.npz'), **rout)
    print('wrote iso64_rho.npz')


def rot20(args):
    """Effective potential of rigid CO2 from the reference's own code."""
    ref = import_reference(args.reference)
    system, extpot = ref[0], ref[3]
    import yaff
    from cmmdft_b200.system import read_chk, read_pars_file
    from cmmdft_b200.hosts import cubic_host_276
    from cmmdft_b200.units import angstrom, boltzmann
    gdir = os.path.join(args.reference, 'InputFiles', 'Guest', 'CO2')
    g = read_chk(os.path.join(gdir, 'struct_AA.chk'))
    gff = read_pars_file(os.path.join(gdir, 'pars_vdw_AA_trappe.txt'))
    host = cubic_host_276(0)
    files = {
        'host.chk': lambda: yaff.System(pos=host.pos.copy(), ffatypes=host.ffatypes,
                                        ffatype_ids=host.ffatype_ids, rvecs=host.rvecs),
        'guest.chk': lambda: yaff.System(pos=g['pos'].copy(), ffatypes=list(g['ffatypes']),
                                         ffatype_ids=g['ffatype_ids'], masses=g['masses'].copy()),
    }
    pars = {'host.par': dict(host.ff), 'guest.par': dict(gff)}

    class _System(object):          # System.from_file of the shim cannot read checkpoints
        from_file = staticmethod(lambda fn: files[fn]())
    extpot.System = _System
    extpot.read_pars_file = lambda fn: pars[fn]
    epot_dict = extpot.get_external_potential_dict('host.par', 'guest.par', 'host.chk', cutoff=12 * angstrom)
    n, T = 20, 300.0
    grid = system.Grid(files['host.chk']().cell, npoints=n)
    out = dict(T=T, n=n, guest_pos=g['pos'], guest_masses=g['masses'], guest_ffatypes=np.array(g['ffatypes']),
               guest_ffatype_ids=g['ffatype_ids'],
               guest_sigma=np.array([gff[t][0] for t in g['ffatypes']]),
               guest_epsilon=np.array([gff[t][1] for t in g['ffatypes']]))
    # the reference reads its Lebedev tables relative to the working directory
    cwd = os.getcwd()
    tmp = tempfile.mkdtemp(prefix='cmm_rot_')
    os.symlink(os.path.abspath(args.reference), os.path.join(tmp, 'CmmDFT'))
    os.chdir(tmp)
    try:
        for deg in (9, 11):
            t0 = time.time()
            V = extpot.generate_effective_potential('guest.chk', grid.points[..., :3], 1 / T / boltzmann, epot_dict,
                                                    degree=deg)
            print('degree %d: %.1f s, V in [%.4g, %.4g]' % (deg, time.time() - t0, np.nanmin(V), np.nanmax(V)))
            R1, w1 = extpot.generate_rotation_matrix(deg, 3)
            R2, w2 = extpot.generate_rotation_matrix(deg, 2)
            out['V%d' % deg] = V
            out['rot%d' % deg] = np.einsum('aij,bjk->abij', R1, R2).reshape(-1, 3, 3)
            out['w%d' % deg] = np.repeat(w1 * w2, len(R2))
    finally:
        os.chdir(cwd)
    np.savez_compressed(os.path.join(HERE, 'rot20.npz'), **out)


def rotinterp12(args):
    """Tricubic-interpolated effective potential of rigid CO2 from the
    reference's own ExternalPotential.generate_potential(interpolate=True)."""
    ref = import_reference(args.reference)
    system, functionals, extpot = ref[0], ref[1], ref[3]
    import yaff
    from cmmdft_b200.system import read_chk, read_pars_file
    from cmmdft_b200.hosts import cubic_host_276
    from cmmdft_b200.units import angstrom, kjmol
    gdir = os.path.join(args.reference, 'InputFiles', 'Guest', 'CO2')
    g = read_chk(os.path.join(gdir, 'struct_AA.chk'))
    gff = read_pars_file(os.path.join(gdir, 'pars_vdw_AA_trappe.txt'))
    host = cubic_host_276(0)
    guest_mol = lambda: yaff.System(pos=g['pos'].copy(), ffatypes=list(g['ffatypes']),
                                    ffatype_ids=g['ffatype_ids'], masses=g['masses'].copy())
    pars = {'host.par': dict(host.ff), 'guest.par': dict(gff)}

    class _System(object):          # System.from_file of the shim cannot read checkpoints
        from_file = staticmethod(lambda fn: guest_mol())
    extpot.System = _System
    extpot.read_pars_file = functionals.read_pars_file = lambda fn: pars[fn]
    mol = yaff.System(pos=host.pos.copy(), ffatypes=host.ffatypes, ffatype_ids=host.ffatype_ids, rvecs=host.rvecs)
    mol.pos -= mol.pos.sum(axis=0) / len(mol.pos)  # as system.py:70
    h = system.NanoporousHost.__new__(system.NanoporousHost)
    system.Host.__init__(h, 'synthetic', mol.cell)
    h.mol, h.chk, h.par = mol, 'host.chk', 'host.par'
    gu = system.NonSphericalGuest.__new__(system.NonSphericalGuest)
    system.Guest.__init__(gu, 'CO2', g['masses'].sum())
    gu.mol, gu.natom, gu.chk, gu.par = guest_mol(), 3, 'guest.chk', 'guest.par'
    syst = system.System(h, gu)
    n, T, deg = 12, 300.0, 9
    grid = system.Grid(mol.cell, npoints=n)
    tmp = tempfile.mkdtemp(prefix='cmm_rotinterp_')
    ep = functionals.ExternalPotential(grid, syst, tmp, limit_potential=1e4 * kjmol, degree=deg, interpolate=True,
                                       cutoff=12 * angstrom)
    cwd = os.getcwd()
    os.symlink(os.path.abspath(args.reference), os.path.join(tmp, 'CmmDFT'))
    os.chdir(tmp)
    try:
        t0 = time.time()
        quiet(ep.generate_potential, T)
        print('interpolated potential: %.1f s' % (time.time() - t0))
    finally:
        os.chdir(cwd)
    fine = system.Grid(mol.cell, spacing=0.15 * angstrom)
    out = dict(T=T, n=n, degree=deg, V=ep.potential, fine_npoints=np.array(fine.npoints),
               fine_spacings=np.array(fine.spacings), origin=grid.points[0, 0, 0, :3],
               interp_spacing=np.array([0.15, 0.15, 0.15]) * angstrom,
               guest_pos=g['pos'], guest_masses=g['masses'], guest_ffatypes=np.array(g['ffatypes']),
               guest_ffatype_ids=g['ffatype_ids'],
               guest_sigma=np.array([gff[t][0] for t in g['ffatypes']]),
               guest_epsilon=np.array([gff[t][1] for t in g['ffatypes']]))
    rng = np.random.default_rng(17)
    idx = np.stack([rng.integers(0, m, 3000) for m in fine.npoints], axis=1)
    out['deriv_idx'] = idx
    pts = fine.points[idx[:, 0], idx[:, 1], idx[:, 2], :3]
    for t in g['ffatypes']:
        sg, eg = gff[t]
        out['deriv_' + t] = extpot.get_external_potential_derivatives(pts, host.ff, sg, eg, mol, fine.spacings,
                                                                      cutoff=12 * angstrom)
    np.savez_compressed(os.path.join(HERE, 'rotinterp12.npz'), **out)


PROJ_PRESSURES = (0.1, 1.0, 10.0)   # bar


def proj32(args):
    """The reference's projections and free-energy path on three 32^3 densities."""
    ref = import_reference(args.reference)
    system, functionals, solver, extpot, eos = ref
    from cmmdft import program as rprogram, calculator as rcalculator
    import yaff
    from cmmdft_b200.hosts import cubic_host_276, methane_guest_params
    from cmmdft_b200.units import angstrom, bar
    T = 300.0
    host = cubic_host_276(seed=0)
    sig, eps, mass = methane_guest_params()
    mol = yaff.System(pos=host.pos.copy(), ffatypes=host.ffatypes, ffatype_ids=host.ffatype_ids, rvecs=host.rvecs,
                      masses=host.masses)
    mol.pos -= mol.pos.sum(axis=0) / len(mol.pos)  # as system.py:70
    h = system.NanoporousHost.__new__(system.NanoporousHost)
    system.Host.__init__(h, 'synthetic', mol.cell)
    h.mol, h.chk, h.par = mol, None, None
    guest = system.SphericalLJGuest('CH4', mass, sig, eps)
    tmp = tempfile.mkdtemp(prefix='cmm_proj_')
    grid0 = system.Grid(mol.cell, npoints=32)
    V = extpot.get_external_potential(grid0.points[..., :3].reshape(-1, 3), host.ff, sig, eps, mol,
                                      cutoff=12 * angstrom)
    vfn = os.path.join(tmp, 'epot_32.npy')
    np.save(vfn, V.reshape(grid0.npoints))
    prog = rprogram.Program(prefix=tmp, hostname='synthetic', guestname='CH4', ff_suffix='trappe_uff', suffix='proj')
    prog.set_system(h, guest)
    prog.set_grid(npoints=32)
    prog.init_free_energy(T)
    prog.fener.add_hard_sphere(version='WBII')
    prog.fener.add_mean_field(cutoff=12 * angstrom, rewrite=True)
    prog.fener.add_external_potential(load_fn=vfn)
    prog.fener.set_temperature(T)
    mb = eos.ModifiedBenedictWebbRubinEOS(mass, sig, eps)
    mb.set_temperature(T)
    mus = [mb.calculate_mu(T, p * bar) for p in PROJ_PRESSURES]
    out = dict(T=T, mus=np.array(mus))
    for i, mu in enumerate(mus):
        bulk = float(np.nanmin(mb.solve_densities_from_chempots([mu]), axis=1)[0])
        prog.set_solver(solver.Anderson(prog, nsteps=500, m=5, criterion='res', threshold=1e-8))
        N, rho, conv = quiet(prog.solve, mu, Ninit=bulk, energy_tracking=False)
        assert conv
        out['rho%d' % i] = rho
    calc = rcalculator.Calculator.__new__(rcalculator.Calculator)
    calc.program, calc.name_dict, calc.workdir = prog, prog.name_dict, prog.workdir
    calc.grid, calc.fener = prog.grid, prog.fener
    calc.host, calc.guest, calc.label = prog.system.host, prog.system.guest, None
    path = np.array([[1.0, -0.5, 0.0], [1.6, -0.1, 1.0]])
    cvs, cvs_mat, dist_mask = quiet(calc.collective_variable, diffusion_path=path, dist_from_axis=3 * angstrom,
                                    supercell=True, step_dist=0.5 * angstrom)
    out.update(path=path, cvs=cvs, cvs_mat_sum=np.sum(cvs_mat), cvs_mat_sample=cvs_mat.reshape(-1)[::997],
               dist_mask_count=int(np.sum(dist_mask)), cvs_mat_shape=np.array(cvs_mat.shape))
    for i, mu in enumerate(mus):
        q, n = quiet(calc.project_density, T, mu, cvs, cvs_mat, dist_mask, rewrite=True)
        out['proj_q'], out['proj_n%d' % i] = q, n
        quiet(calc.save_loading_and_grand_potential, T, mu)
    with open(os.path.join(prog.workdir, 'loading_grand_potential_%7.5fK.csv' % T)) as f:
        out['lgp_csv'] = np.array(f.read())
    quiet(calc.free_energy_path, T, mus[-1], chempots=mus)
    fe_fn = prog.workdir / ('free_energy_profile_%#0.8fkjmol_%#0.3fK.csv' % (mus[-1] / kjmol_unit(), T))
    out['fe_path'] = np.loadtxt(fe_fn, delimiter=',', skiprows=1)
    quiet(calc.project_contributions, T, mus[1], ['fid', 'pure_extpot'], cvs, cvs_mat, dist_mask)
    from cmmdft_b200.tools import get_file_suffix
    pc_fn = prog.workdir / ('projected_contributions_%s.csv' % get_file_suffix(mus[1], T))
    out['proj_contrib'] = np.loadtxt(pc_fn, delimiter=',', skiprows=1)
    ring = list(range(6))
    cvs_r, cvs_mat_r, mask_r = quiet(calc.collective_variable, ring_indices=ring, step_dist=0.5 * angstrom)
    out.update(ring=np.array(ring), ring_cvs=cvs_r, ring_cvs_mat=cvs_mat_r)
    np.savez_compressed(os.path.join(HERE, 'proj32.npz'), **out)
    print('wrote proj32.npz', {k: v for k, v in out.items() if np.ndim(v) == 0})


def kjmol_unit():
    from cmmdft_b200.units import kjmol
    return kjmol


def fire32(args):
    """The reference's Fire solver on the 32^3 case."""
    ref = import_reference(args.reference)
    solver = ref[2]
    from cmmdft_b200.hosts import cubic_host_276
    from cmmdft_b200.units import boltzmann
    T = 300.0
    b = quiet(build, ref, 32, cubic_host_276(0), T, 1.0, tempfile.mkdtemp(prefix='cmm_fire_'))
    fe, mu = b['fe'], b['mu']
    V = fe.part_dict['ExtPot'].potential
    mb = b['mbwr']
    mb.set_temperature(T)
    bulk = float(np.nanmin(mb.solve_densities_from_chempots([mu]), axis=1)[0])
    rho0 = bulk * np.exp(-np.maximum(V, 0) / boltzmann / T)
    out = dict(T=T, mu=mu, rho_bulk=bulk)
    for meth, tag in (('abc-fire', 'abc'), ('fire', 'plain')):
        f = solver.Fire(b['prog'], nsteps=400, method=meth, criterion='res', threshold=1e-6)
        f.mask = rho0 > 0
        runs = 2 if tag == 'abc' else 1
        for r in range(runs):
            N, rho, conv = quiet(f.solve, mu, rho0.copy(), 3)
            key = '%s%d' % (tag, r)
            out.update({key + '_steps': f.curr_step, key + '_N': N, key + '_conv': conv, key + '_rho': rho,
                        key + '_dt': f.dt, key + '_alpha': f.alpha, key + '_Npos': f.Npos, key + '_Nneg': f.Nneg})
            print(key, f.curr_step, N, conv, f.dt, f.alpha, f.Npos, f.Nneg, flush=True)
        # the reference against itself with its density moved one ulp up
        # before every update: the rounding floor of the first solve's
        # trajectory under a per-step perturbation of rounding size
        class _FireUlp(solver.Fire):
            def update_rho(self, rho, krho, C1):
                return solver.Fire.update_rho(self, np.nextafter(rho, np.inf), krho, C1)
        f2 = _FireUlp(b['prog'], nsteps=400, method=meth, criterion='res', threshold=1e-6)
        f2.mask = rho0 > 0
        N2, rho2, _ = quiet(f2.solve, mu, rho0.copy(), 3)
        key = tag + '0'
        out[key + '_rho_floor'] = np.max(np.abs(rho2 - out[key + '_rho'])) / np.max(np.abs(out[key + '_rho']))
        out[key + '_N_floor'] = abs(N2 - out[key + '_N']) / abs(out[key + '_N'])
        print(key, 'floor rho %.2e N %.2e' % (out[key + '_rho_floor'], out[key + '_N_floor']), flush=True)
    np.savez_compressed(os.path.join(HERE, 'fire32.npz'), **out)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--reference', default=os.environ.get('CMM_REFERENCE_ROOT'),
                    help="root of the reference's source tree (the directory holding cmmdft/); "
                         "default: $CMM_REFERENCE_ROOT")
    ap.add_argument('--skip64', action='store_true')
    ap.add_argument('--iso64', action='store_true')
    ap.add_argument('--qn', action='store_true')
    ap.add_argument('--dropin', action='store_true')
    ap.add_argument('--uneven', action='store_true')
    ap.add_argument('--lda', action='store_true')
    ap.add_argument('--rot', action='store_true')
    ap.add_argument('--rotinterp', action='store_true')
    ap.add_argument('--proj', action='store_true')
    ap.add_argument('--fire', action='store_true')
    ap.add_argument('--procs', type=int, default=8)
    args = ap.parse_args()
    if not args.reference:
        ap.error('--reference (or CMM_REFERENCE_ROOT) is required')
    if args.iso64:
        return iso64(args)
    if args.qn:
        return qn32(args)
    if args.dropin:
        return dropin32(args)
    if args.uneven:
        return uneven(args)
    if args.lda:
        return lda32(args)
    if args.rot:
        return rot20(args)
    if args.rotinterp:
        return rotinterp12(args)
    if args.proj:
        return proj32(args)
    if args.fire:
        return fire32(args)
    ref = import_reference(args.reference)
    solver = ref[2]
    from cmmdft_b200.hosts import cubic_host_276, HELIUM
    from cmmdft_b200.units import angstrom, boltzmann, bar
    extpot = ref[3]
    T = 300.0
    host = cubic_host_276(seed=0)
    tmp = tempfile.mkdtemp(prefix='cmm_golden_')
    out = {}
    b = quiet(build, ref, 32, host, T, 1.0, tmp)
    fe, grid, mu = b['fe'], b['grid'], b['mu']
    out.update(host_pos=host.pos, host_ids=host.ffatype_ids, host_rvecs=host.rvecs,
               T=T, mu=mu, Rhs=b['guest'].Rhs, wavelength=fe.wavelength, beta=fe.beta,
               V=fe.part_dict['ExtPot'].potential, V_raw=b['V_raw'].reshape(grid.npoints),
               mfa_potential=fe.part_dict['MFA'].potential)
    # bulk density on the lowest branch at mu (calculator.py:129-131)
    mb = b['mbwr']
    mb.set_temperature(T)
    out['rho_bulk'] = np.nanmin(mb.solve_densities_from_chempots([mu]), axis=1)[0]
    # helium void fraction through the reference's own potential routine
    Vhe = extpot.get_external_potential(grid.points[..., :3].reshape(-1, 3), host.ff,
                                        HELIUM['sigma'] * angstrom, HELIUM['epsilon_K'] * boltzmann,
                                        b['mol'], cutoff=12 * angstrom)
    out['he_frac'] = grid.integrate(np.clip(np.exp(-Vhe / boltzmann / T), 0, 1)).real / grid.cell.volume
    # two C1 evaluations: ideal-gas start and a dense liquid-like profile
    rho_a = np.exp(fe.beta * (mu - out['V'])) / fe.wavelength ** 3
    rho_b = 0.02 / angstrom ** 3 * np.clip(np.exp(-fe.beta * out['V']), 0, 1)
    for tag, rho in (('a', rho_a), ('b', rho_b)):
        parts, om, derivs, C1 = quiet(omega_parts, ref, b, rho, mu)
        out['rho_' + tag] = rho
        out['values_' + tag] = np.array(parts)
        out['omega_' + tag] = om
        out['dHS_' + tag] = derivs[0]
        out['dMFA_' + tag] = derivs[1]
        out['C1_' + tag] = C1
        out['n3_' + tag] = fe.part_dict['HardSphere'].get_n3(grid.fft(rho))
    # static Picard trajectory (solver.py:392-401), criterion RES
    for nst, key in ((3, 'picard3'), (500, 'picard')):
        s = solver.Picard(b['prog'], nsteps=nst, alpha_mix=0.1, method='static',
                          criterion='res', threshold=1e-8)
        N, rho, conv = quiet(s.solve, mu, rho_a.copy(), 3)
        out[key + '_rho'] = rho
        out[key + '_N'] = N
        out[key + '_steps'] = s.curr_step
        out[key + '_conv'] = conv
    # static Picard under the DER criterion (solver.py:200-205); a list criterion
    # keeps its threshold (a plain 'der' forces 1, solver.py:72-73)
    s = solver.Picard(b['prog'], nsteps=500, alpha_mix=0.1, method='static', criterion=['der'],
                      threshold=[1e-3])
    N, rho, conv = quiet(s.solve, mu, rho_a.copy(), 3)
    out.update(der_rho=rho, der_N=N, der_steps=s.curr_step, der_conv=conv, der_value=s.DER)
    s = solver.Picard(b['prog'], nsteps=1, method='static')
    s._initiate_solving(mu)
    out['picard_omega'] = s._get_Omega(out['picard_rho'], grid.fft(out['picard_rho']))
    # tight hybrid-Anderson (reference default method) at 1 bar
    s = solver.Anderson(b['prog'], nsteps=500, m=5, criterion=TIGHT_CRIT, threshold=TIGHT_THR)
    t0 = time.time()
    N, rho, conv = quiet(s.solve, mu, rho_a.copy(), 3)
    out['and_time'] = time.time() - t0
    out.update(and_rho=rho, and_N=N, and_steps=s.curr_step, and_conv=conv)
    s2 = solver.Picard(b['prog'], nsteps=1, method='static')
    s2._initiate_solving(mu)
    out['and_omega'] = s2._get_Omega(rho, grid.fft(rho))
    # tail-corrected MFA on the 2x2x2 supercell (functionals.py:794-796, 918-923)
    bt = quiet(build, ref, 32, host, T, 1.0, tempfile.mkdtemp(prefix='cmm_golden_t_'), tail=True)
    k = grid.fft(rho_b)
    out['dMFA_tail_b'] = bt['fe'].part_dict['MFA'].derive(k)
    out['vMFA_tail_b'] = bt['fe'].part_dict['MFA'].value(k)
    # WDA correlation part on top (add_correlation_wda_lj, functionals.py:339-362)
    bw = quiet(build, ref, 32, host, T, 1.0, tempfile.mkdtemp(prefix='cmm_golden_w_'), wda=True)
    for tag, rho in (('a', rho_a), ('b', rho_b)):
        parts, om, derivs, C1 = quiet(omega_parts, ref, bw, rho, mu)
        out['wda_values_' + tag] = np.array(parts)
        out['wda_omega_' + tag] = om
        out['wda_dWDA_' + tag] = derivs[3]
        out['wda_C1_' + tag] = C1
    # tensor FMT variants (functionals.py:457-487, 534-552, 620-717): the
    # hard-sphere part alone, as HardSphereFunctional(grid, R, version)
    functionals = ref[1]
    for ver, tags in (('atWBII', 'ab'), ('tWBII', 'ab'), ('atFMT', 'b'), ('tMFMT', 'b')):
        hs = functionals.HardSphereFunctional(grid, b['guest'].Rhs, version=ver)
        hs.set_temperature(T, b['guest'].Rhs)
        for tag in tags:
            k = grid.fft(rho_a if tag == 'a' else rho_b)
            out['hs_%s_d_%s' % (ver, tag)] = quiet(hs.derive, k)
            out['hs_%s_v_%s' % (ver, tag)] = quiet(hs.value, k)
    np.savez_compressed(os.path.join(HERE, 'c0_32.npz'), **out)
    print('wrote c0_32.npz', 'picard steps', out['picard_steps'], 'anderson steps', out['and_steps'])

    if args.skip64:
        return
    out = {}
    pressures = np.array([1e-3, 1.0, 10.0, 100.0])
    b = quiet(build, ref, 64, host, T, 1.0, tempfile.mkdtemp(prefix='cmm_golden64_'))
    fe, grid = b['fe'], b['grid']
    mb = b['mbwr']
    V = fe.part_dict['ExtPot'].potential
    Vhe = extpot.get_external_potential(grid.points[..., :3].reshape(-1, 3), host.ff,
                                        HELIUM['sigma'] * angstrom, HELIUM['epsilon_K'] * boltzmann,
                                        b['mol'], cutoff=12 * angstrom)
    he_frac = grid.integrate(np.clip(np.exp(-Vhe / boltzmann / T), 0, 1)).real / grid.cell.volume
    out.update(T=T, pressures=pressures, V_sum=V.sum(), V_min=V.min(),
               V_slice=V[:, :, 32].copy(), t_ext=b['t_ext'])
    mus, Ns, Oms, steps, bulks = [], [], [], [], []
    for P in pressures:
        mu = mb.calculate_mu(T, P * bar)
        mb.set_temperature(T)
        bulks.append(np.nanmin(mb.solve_densities_from_chempots([mu]), axis=1)[0])
        # Ninit = rho_bulk start of the reference's example notebook
        # (program.py:278-287); the ideal-gas default start overflows G at
        # 100 bar and the reference's hybrid step then fails in np.polyfit.
        rho0 = bulks[-1] * np.exp(-np.maximum(V, 0) / boltzmann / T)
        s = solver.Anderson(b['prog'], nsteps=500, m=5, criterion=TIGHT_CRIT, threshold=TIGHT_THR)
        N, rho, conv = quiet(s.solve, mu, rho0, 3)
        s2 = solver.Picard(b['prog'], nsteps=1, method='static')
        s2._initiate_solving(mu)
        Oms.append(s2._get_Omega(rho, grid.fft(rho)))
        mus.append(mu)
        Ns.append(N)
        steps.append(s.curr_step)
        if P == 1.0:
            out['rho_1bar'] = rho
        print('64^3 P=%g bar: N=%.12e steps=%d conv=%s' % (P, N, s.curr_step, conv), flush=True)
    out.update(mu=np.array(mus), N=np.array(Ns), omega=np.array(Oms), steps=np.array(steps),
               rho_bulk=np.array(bulks), he_frac=he_frac)
    np.savez_compressed(os.path.join(HERE, 'c1_64.npz'), **out)
    print('wrote c1_64.npz')


if __name__ == '__main__':
    main()
