"""The reference's public API end to end on the GPU path.

The 32^3 case (276-atom cubic host, methane, 300 K, 1 bar) driven the way a
user of the reference drives it: Program -> set_system / set_grid /
init_free_energy -> FreeEnergy.add_hard_sphere / add_mean_field /
add_external_potential -> a Solver -> Program.solve / cascade_solver ->
Calculator.  ``tests/golden/dropin32.npz`` holds the same calls made on the
unmodified reference (tests/golden/make_golden.py --dropin); c0_32.npz the
part derivatives and values.

Tolerances: converged loading, grand potential and Calculator observables
1e-10 relative; densities 1e-10 relative to max rho where both sides follow
the same trajectory to the same convergence test; part derivatives at the
reference's 1-ulp noise floor (tests/test_gpu_parity.py); helium fraction
1e-12.
"""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

import cmmdft_b200 as cd
from cmmdft_b200.hosts import cubic_host_276, methane_guest_params
from cmmdft_b200.units import angstrom, bar
from tests._common import relerr, scalar_rel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TIGHT_CRIT = ['res', 'riue']
TIGHT_THR = [1e-13, 1e-12]
T = 300.0


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


@pytest.fixture(scope="module")
def dropin():
    return dict(np.load(os.path.join(ROOT, "tests", "golden", "dropin32.npz")))


def make_program(prefix, suffix='', version='WBII'):
    """Program of the 32^3 case through the public API only."""
    h = cubic_host_276(0)
    host = cd.NanoporousHost('synthetic', pos=h.pos, ffatypes=h.ffatypes, ffatype_ids=h.ffatype_ids,
                             rvecs=h.rvecs, ff=h.ff, masses=h.masses)
    sig, eps, mass = methane_guest_params()
    guest = cd.SphericalLJGuest('CH4', mass, sig, eps)
    prog = cd.Program(prefix=str(prefix), hostname='synthetic', guestname='CH4', ff_suffix='trappe_uff',
                      suffix=suffix)
    prog.set_system(host, guest)
    prog.set_grid(npoints=32)
    prog.init_free_energy(T)
    prog.fener.add_hard_sphere(version=version)
    prog.fener.add_mean_field(cutoff=12 * angstrom)
    prog.fener.add_external_potential(cutoff=12 * angstrom)
    prog.fener.set_temperature(T)
    return prog


def mbwr():
    sig, eps, mass = methane_guest_params()
    return cd.ModifiedBenedictWebbRubinEOS(mass, sig, eps)


def test_parts_through_grid_fft(cuda, golden32, tmp_path):
    """part.derive(grid.fft(rho)) and part.value(...) against the reference's
    parts (functionals.py:574-618, 912-939, 1073-1083) on the ideal-gas
    profile; Grid.fft's numpy view against the reference convention."""
    prog = make_program(tmp_path)
    fe, grid = prog.fener, prog.grid
    assert relerr(fe.part_dict['ExtPot'].potential, golden32["V"]) < 1e-13
    rho = golden32["rho_a"]
    k = grid.fft(rho)
    beta = fe.beta
    dhs = fe.part_dict['HardSphere'].derive(k)
    dmfa = fe.part_dict['MFA'].derive(k)
    assert beta * np.max(np.abs(dhs - golden32["dHS_a"])) < 2e-9
    assert relerr(dmfa, golden32["dMFA_a"]) < 1e-12
    assert np.array_equal(fe.part_dict['ExtPot'].derive(k), fe.part_dict['ExtPot'].potential)
    vals = [p.value(k) for p in fe.parts]
    for v, ref in zip(vals, golden32["values_a"]):
        assert scalar_rel(v, ref) < 1e-11
    # Spectrum -> reference phase convention fftn(rho) exp(i pi scalprod) / Npts
    full = np.asarray(k)
    ref = np.fft.fftn(rho) * np.exp(1j * np.pi * grid.scalprod) / rho.size
    assert relerr(full, ref, np.abs(ref).max()) < 1e-13
    assert relerr(grid.ifft(k), rho) < 1e-15


def test_program_cascade_and_calculator(cuda, dropin, tmp_path):
    """Program.cascade_solver([static Picard x 3, tight hybrid Anderson],
    continue_solving=True) from the ideal-gas start (program.py:315-328),
    then Calculator.return_loading / free_energy_contrib / grand_potential
    (calculator.py:60-138, 343-492) on the cached density."""
    prog = make_program(tmp_path, 'cascade')
    mu = float(dropin["mu"])
    sv = [cd.Picard(prog, nsteps=3, alpha_mix=0.1, method='static', criterion='res', threshold=1e-8),
          cd.Anderson(prog, nsteps=500, m=5, criterion=TIGHT_CRIT, threshold=TIGHT_THR)]
    prog.cascade_solver(sv, mu, continue_solving=True)
    assert [s.curr_step for s in sv][0] == dropin["cascade_steps"][0]
    rho = np.load(prog.rho_fn)
    N = prog.grid.integrate(rho)
    errs = dict(rho=relerr(rho, dropin["cascade_rho"]), N=scalar_rel(N, dropin["cascade_N"]),
                omega=scalar_rel(sv[1].omega0, dropin["cascade_omega"]))
    calc = cd.Calculator(prog)
    errs['loading'] = scalar_rel(calc.return_loading(T, [mu])[0], dropin["cascade_loading"])
    errs['excess'] = scalar_rel(calc.return_loading(T, [mu], excess=True, eos=mbwr())[0], dropin["cascade_excess"])
    errs['grand_potential'] = scalar_rel(calc.grand_potential(T, mu), dropin["cascade_grand_potential"])
    for part in ('fid', 'HardSphere', 'MFA', 'ExtPot'):
        errs['F_' + part] = scalar_rel(calc.free_energy_contrib(T, mu, part), dropin["cascade_F_" + part])
    # (the Anderson stage's step count is not compared: the reference itself
    # takes 48 or 55 steps from starts one ulp apart at this tolerance)
    floor = dict(zip([str(x) for x in dropin["cascade_floor_names"]], dropin["cascade_floor"]))
    print("cascade (Anderson steps %d, reference %d) + Calculator relative errors:"
          % (sv[1].curr_step, dropin["cascade_steps"][1]), {k: "%.2e" % v for k, v in errs.items()},
          "| the reference against itself from a 1-ulp start:", {k: "%.2e" % v for k, v in floor.items()})
    # Both sides stop at RES < 1e-13 and RIUE < 1e-12 along their own
    # trajectories.  N, N_ex and the grand potentials meet 1e-10 outright; the
    # density and the free-energy parts are held to 1e-10 or five times the
    # reference's own spread under a 1-ulp change of its start (5e-11 for
    # rho, 3e-11 to 4e-11 for the parts), whichever is larger.
    for k in ('N', 'omega', 'loading', 'excess', 'grand_potential'):
        assert errs[k] < 1e-10, (k, errs[k])
    for k in ('rho', 'F_fid', 'F_HardSphere', 'F_MFA', 'F_ExtPot'):
        assert errs[k] < max(1e-10, 5 * floor[k]), (k, errs[k], floor[k])


def test_program_solve_ninit_float_history_and_cache(cuda, dropin, tmp_path):
    """Program.solve(mu, Ninit=rho_bulk) (the float branch of
    program.py:278-287) under hybrid Anderson to RES < 1e-8 with
    track_history: same steps, density, N and Omega as the reference, the
    history's N / Omega / RES / RIUE / DER columns per step
    (solver.py:208-222), rho_*.npy and solving_history_*.csv written, and a
    second solve served from the cache (program.py:381-386)."""
    prog = make_program(tmp_path, 'ninit')
    mu = float(dropin["mu"])
    s = cd.Anderson(prog, nsteps=500, m=5, criterion='res', threshold=1e-8, track_history=True)
    prog.set_solver(s)
    N, rho, conv = prog.solve(mu, Ninit=float(dropin["rho_bulk"]))
    assert conv and s.curr_step == int(dropin["ninit_steps"])
    errs = dict(rho=relerr(rho, dropin["ninit_rho"]), N=scalar_rel(N, dropin["ninit_N"]),
                omega=scalar_rel(s.omega0, dropin["ninit_omega"]))
    h, hr = s.history[:s.curr_step + 1, :5], dropin["ninit_history"]
    assert h.shape == hr.shape
    for c, name in enumerate(('N', 'Omega', 'RES', 'RIUE', 'DER')):
        rows = np.isfinite(hr[1:, c])
        assert np.array_equal(np.isfinite(h[1:, c]), rows), name
        errs['history_' + name] = float(np.max(np.abs(h[1:, c][rows] - hr[1:, c][rows]) / np.abs(hr[1:, c][rows])))
    print("Ninit=float relative errors:", {k: "%.2e" % v for k, v in errs.items()})
    assert errs['rho'] < 1e-10 and errs['N'] < 1e-10 and errs['omega'] < 1e-10
    assert errs['history_N'] < 1e-10 and errs['history_Omega'] < 1e-10
    # RES, RIUE, DER are differences of nearly equal fields: relative 1e-6 of their own size
    for name in ('RES', 'RIUE', 'DER'):
        assert errs['history_' + name] < 1e-6, name
    assert os.path.isfile(prog.rho_fn)
    csv = prog.workdir / ('solving_history_%s.csv' % prog.file_suffix)
    assert csv.is_file() and np.loadtxt(csv, delimiter=',').shape[0] == s.curr_step + 1

    # energy tracking (convergence_*.txt): the start and final lines against
    # the reference's first and last (its columns: phase, step, N, -mu N,
    # ideal part, each part, total; written with 7 significant digits)
    conv_fn = prog.workdir / ('convergence_%s.txt' % prog.file_suffix)
    rows = [l.split() for l in open(conv_fn) if l.strip() and not l.startswith('#')]
    for got, ref in ((rows[0], dropin["ninit_track_first"]), (rows[-1], dropin["ninit_track_last"])):
        got = np.array([float(x) for x in got])
        assert got.shape == ref.shape and np.allclose(got, ref, rtol=2e-6, atol=0), (got, ref)
    # the loading exports (calculator.py:186-340) against the reference's files
    calc = cd.Calculator(prog)
    eos = mbwr()
    tmp = tmp_path / 'exports'
    tmp.mkdir()
    calc.save_loadings(T, [mu], fn=tmp / 'loads.csv')
    calc.save_loadings(T, [mu], pressure=True, eos=eos, fn=tmp / 'loads_P.csv')
    calc.save_loadings_AIF(T, chempots=np.array([mu]), eos=eos, user='tester', loading_unit='mol/kg',
                           fn=tmp / 'ads.aif')
    for name, key in (('loads.csv', 'ninit_csv'), ('loads_P.csv', 'ninit_csv_P')):
        got = np.loadtxt(tmp / name, delimiter=',', skiprows=1)
        ref = np.loadtxt(str(dropin[key]).splitlines()[1:], delimiter=',')
        assert open(tmp / name).readline().strip() == str(dropin[key]).splitlines()[0]
        assert np.allclose(got, ref, rtol=1e-10, atol=0), (name, got, ref)
    skip = ('_simltn_date', '_simltn_code')
    got = [l for l in open(tmp / 'ads.aif').read().splitlines() if not l.startswith(skip)]
    ref = [l for l in str(dropin["ninit_aif"]).splitlines() if not l.startswith(skip)]
    assert got == ref, (got, ref)

    class Refuse(cd.Solver):
        def solve(self, *a, **k):
            raise AssertionError("the cached density must be used")
    prog.set_solver(Refuse(prog))
    N2, rho2, conv2 = prog.solve(mu)
    assert conv2 and np.array_equal(rho2, rho) and N2 == prog.grid.integrate(rho)


def test_initial_density_branches(cuda, golden32, tmp_path):
    """_set_initial_density (program.py:219-305): ideal gas, float, array and
    file branches, and the missing-file error."""
    prog = make_program(tmp_path)
    mu = float(golden32["mu"])
    V = golden32["V"]
    prog._set_initial_density(chempot=mu, temperature=T)
    assert relerr(prog.rho0, golden32["rho_a"]) < 1e-14
    n0 = 3.5e-6
    prog._set_initial_density(Ninit=n0, chempot=mu, temperature=T)
    assert relerr(prog.rho0, n0 * np.exp(-np.maximum(V, 0) / cd.boltzmann / T)) < 1e-14
    arr = np.full((32, 32, 32), 1e-7)
    prog._set_initial_density(Ninit=arr, chempot=mu, temperature=T)
    assert prog.rho0 is arr
    fn = tmp_path / 'guess.npy'
    np.save(fn, arr)
    prog._set_initial_density(Ninit=str(fn), chempot=mu, temperature=T)
    assert np.array_equal(prog.rho0, arr)
    with pytest.raises(FileNotFoundError):
        prog._set_initial_density(Ninit=str(tmp_path / 'missing.npy'), chempot=mu, temperature=T)
    with pytest.raises(AssertionError):
        prog._set_initial_density(Ninit=np.zeros((8, 8, 8)), chempot=mu, temperature=T)


def test_helium_fraction(cuda, golden32, golden64, tmp_path):
    """Calculator.get_helium_fraction on the GPU against the reference's
    helium void fraction at 32^3 and 64^3."""
    prog = make_program(tmp_path)
    he32 = cd.Calculator(prog).get_helium_fraction(T)
    h = cubic_host_276(0)
    host = cd.NanoporousHost('synthetic', pos=h.pos, ffatypes=h.ffatypes, ffatype_ids=h.ffatype_ids,
                             rvecs=h.rvecs, ff=h.ff)
    sig, eps, mass = methane_guest_params()
    p64 = cd.Program(prefix=str(tmp_path), hostname='s64')
    p64.set_system(host, cd.SphericalLJGuest('CH4', mass, sig, eps))
    p64.set_grid(npoints=64)
    p64.init_free_energy(T)
    he64 = cd.Calculator(p64).get_helium_fraction(T)
    e32 = scalar_rel(he32, golden32["he_frac"])
    e64 = scalar_rel(he64, golden64["he_frac"])
    print("helium fraction relative errors: 32^3 %.2e, 64^3 %.2e" % (e32, e64))
    assert e32 < 1e-12 and e64 < 1e-12


@pytest.mark.parametrize("method", ["static", "hybridanderson"])
@pytest.mark.parametrize("native", [True, False])
def test_nonfinite_member_retries_then_fails(cuda, tmp_path, native, method):
    """The reference's failure handling (solver.py:317-345) per batch member:
    a member seeded with NaN takes correction factors 1, 1/2 and 1/4 and then
    raises NoSolutionError; the other members converge exactly as they do
    without it.  (Static Picard is the reference's own path to this error: a
    non-finite density after the update raises FloatingPointError.  Its
    hybrid line search instead stops in np.polyfit on a NaN seed; the batch
    treats every method the same way.)"""
    from cmmdft_b200 import batch as BT, workload as W
    fn = W.build_functional(cubic_host_276(0), (32, 32, 32), T, methane_guest_params())
    mus, bulks = W.isotherm_inputs(np.array([0.1, 1.0, 10.0]) * bar, T, methane_guest_params())
    r0 = W.initial_density(fn, mus, ninit=bulks)
    cls = BT.NativeBatchSolve if native else BT.BatchSolve
    kw = dict(method=method, nsteps=200 if method != 'static' else 2000, threshold=1e-8, criterion='res')
    ref = cls(fn, mus[[0, 2]], **kw)
    Nref, rref, cref = ref.solve(r0[[0, 2]].contiguous())
    bad = r0.clone()
    bad[1, 3, 4, 5] = float('nan')
    s = cls(fn, mus, **kw)
    with pytest.raises(cd.NoSolutionError):
        s.solve(bad)
    assert list(s.failed) == [False, True, False]
    assert list(s.cf) == [1.0, 0.125, 1.0]
    assert list(s.conv[[0, 2]]) == list(cref) == [True, True]
    assert s.N_out[0] == Nref[0] and s.N_out[2] == Nref[1]
    assert torch.equal(s.result[0], rref[0]) and torch.equal(s.result[2], rref[1])
    # the drop-in Solver raises the same error for a single density
    prog = make_program(tmp_path)
    a = cd.Picard(prog, nsteps=50, alpha_mix=0.1, method='static', criterion='res', threshold=1e-8)
    with pytest.raises(cd.NoSolutionError):
        a.solve(float(mus[1]), bad[1].cpu().numpy())


def test_projections_and_free_energy_path(cuda, tmp_path):
    """Calculator post-processing (calculator.py:494-899) on the reference's
    own three converged 32^3 densities (tests/golden/proj32.npz, placed as
    the rho_*.npy files of the Program): collective variables along a tilted
    axis on the 3 x 3 x 3 supercell and from ring atoms (exact), projected
    densities and contributions (1e-12 of their largest value), the loading
    and grand-potential table (1e-12 / 1e-10) and the free-energy path
    (1e-10 relative to the largest Omega)."""
    from cmmdft_b200.tools import get_file_suffix
    ref = dict(np.load(os.path.join(ROOT, "tests", "golden", "proj32.npz")))
    prog = make_program(tmp_path, 'proj')
    mus = ref["mus"]
    for i, mu in enumerate(mus):
        np.save(prog.workdir / ('rho_%s.npy' % get_file_suffix(mu, T)), ref["rho%d" % i])
    calc = cd.Calculator(prog)
    cvs, cvs_mat, mask = calc.collective_variable(diffusion_path=ref["path"], dist_from_axis=3 * angstrom,
                                                  supercell=True, step_dist=0.5 * angstrom)
    assert np.array_equal(cvs, ref["cvs"]) and tuple(cvs_mat.shape) == tuple(ref["cvs_mat_shape"])
    assert np.array_equal(cvs_mat.reshape(-1)[::997], ref["cvs_mat_sample"])
    assert int(np.sum(mask)) == int(ref["dist_mask_count"])
    errs = {}
    for i, mu in enumerate(mus):
        q, n = calc.project_density(T, mu, cvs, cvs_mat, mask, rewrite=True)
        assert np.array_equal(q, ref["proj_q"])
        errs['n%d' % i] = float(np.max(np.abs(n - ref["proj_n%d" % i])) / np.max(np.abs(ref["proj_n%d" % i])))
        calc.save_loading_and_grand_potential(T, mu)
    got = np.loadtxt(prog.workdir / ('loading_grand_potential_%7.5fK.csv' % T), delimiter=',', skiprows=1)
    exp = np.array([[float(x) for x in l.split(',')] for l in str(ref["lgp_csv"]).strip().splitlines()[1:]])
    assert got.shape == exp.shape and np.array_equal(got[:, 0], exp[:, 0])
    errs['loading'] = float(np.max(np.abs(got[:, 1] - exp[:, 1]) / np.abs(exp[:, 1])))
    errs['omega'] = float(np.max(np.abs(got[:, 2] - exp[:, 2]) / np.abs(exp[:, 2])))
    fe = calc.free_energy_path(T, mus[-1], chempots=list(mus))
    rf = ref["fe_path"].T
    assert np.array_equal(fe[0], rf[0])
    for c, name in ((1, 'fe_density'), (2, 'fe_omega'), (3, 'fe_free')):
        fin = np.isfinite(rf[c])
        assert np.array_equal(np.isfinite(fe[c]), fin), name
        errs[name] = float(np.max(np.abs(fe[c][fin] - rf[c][fin])) / np.max(np.abs(rf[c][fin])))
    pc = calc.project_contributions(T, mus[1], ['fid', 'pure_extpot'], cvs, cvs_mat, mask)
    rc = ref["proj_contrib"].T
    for c, name in ((2, 'fid'), (3, 'pure_extpot')):
        fin = np.isfinite(rc[c])
        assert np.array_equal(np.isfinite(pc[c]), fin), name
        errs[name] = float(np.max(np.abs(pc[c][fin] - rc[c][fin])) / np.max(np.abs(rc[c][fin])))
    cr, cmr, _ = calc.collective_variable(ring_indices=list(ref["ring"]), step_dist=0.5 * angstrom)
    errs['ring_cvs'] = float(np.max(np.abs(cr - ref["ring_cvs"])))
    errs['ring_cvs_mat'] = float(np.max(np.abs(cmr - ref["ring_cvs_mat"])))
    print("projections:", {k: "%.1e" % v for k, v in errs.items()})
    assert max(errs[k] for k in errs if k.startswith('n')) < 1e-12
    assert errs['loading'] < 1e-12 and errs['omega'] < 1e-10
    assert errs['fe_density'] < 1e-12 and errs['fe_omega'] < 1e-10 and errs['fe_free'] < 1e-10
    assert errs['fid'] < 1e-12 and errs['pure_extpot'] < 1e-12
    assert errs['ring_cvs'] < 1e-12 and errs['ring_cvs_mat'] < 1e-12


def test_fire_against_reference(cuda, tmp_path):
    """Fire (solver.py:606-698) through the drop-in API against the
    reference's own runs (tests/golden/fire32.npz): 'abc-fire' twice with
    one solver object (its N_pos / N_neg counters carry over) and 'fire',
    from Ninit = rho_bulk to RES < 1e-6 with mask = rho0 > 0: the same step
    counts and FIRE state, N and rho within max(1e-10, 3 x the reference's
    own floor under a one-ulp perturbation per step) of the reference's; an
    unset mask raises AttributeError as in the reference."""
    from cmmdft_b200.units import boltzmann
    ref = dict(np.load(os.path.join(ROOT, "tests", "golden", "fire32.npz")))
    prog = make_program(tmp_path)
    V = prog.fener.part_dict['ExtPot'].potential
    mu, bulk = float(ref["mu"]), float(ref["rho_bulk"])
    rho0 = bulk * np.exp(-np.maximum(V, 0) / boltzmann / T)
    errs = {}
    for meth, tag, runs in (('abc-fire', 'abc', 2), ('fire', 'plain', 1)):
        f = cd.Fire(prog, nsteps=400, method=meth, criterion='res', threshold=1e-6)
        if tag == 'abc':
            with pytest.raises(AttributeError):
                f.solve(mu, rho0.copy())
        f.mask = rho0 > 0
        for r in range(runs):
            key = '%s%d' % (tag, r)
            N, rho, conv = f.solve(mu, rho0.copy())
            assert conv == bool(ref[key + "_conv"]) and f.curr_step == int(ref[key + "_steps"]), key
            assert (f.Npos, f.Nneg) == (int(ref[key + "_Npos"]), int(ref[key + "_Nneg"])), key
            errs[key] = dict(N=scalar_rel(N, ref[key + "_N"]), rho=relerr(rho, ref[key + "_rho"]),
                             dt=scalar_rel(f.dt, ref[key + "_dt"]), alpha=scalar_rel(f.alpha, ref[key + "_alpha"]))
    print("Fire vs reference:", {k: {q: "%.1e" % v for q, v in d.items()} for k, d in errs.items()})
    for key, d in errs.items():
        # the target 1e-10, or 3x the reference's own floor on the first
        # solve's trajectory (the same solve with its density moved one ulp
        # before every update); the second solve continues from the first's
        # counters and is held to the first's floor
        k0 = key[:-1] + '0'
        fl = ref.get(k0 + "_rho_floor", 0.0), ref.get(k0 + "_N_floor", 0.0)
        assert d['rho'] < max(1e-10, 3 * float(fl[0])) and d['N'] < max(1e-10, 3 * float(fl[1])), key
        assert d['dt'] < 1e-14 and d['alpha'] < 1e-12, key
