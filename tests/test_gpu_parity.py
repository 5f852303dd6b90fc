"""GPU parity: the CUDA path (through the C ABI) against the oracle and the
reference's golden fixtures.

Tolerances (stated per check):
  * FFTs against scipy.fft: 1e-13 relative to max |X|.
  * External potential: 1e-13 relative to the cap (max |V|).
  * Functional derivatives: beta * max |dC1| below the reference's own noise
    floor under 1-ulp input perturbations (5e-10 on the ideal-gas profile,
    1e-7 on the sharp dense profile; see tests/test_oracle_golden.py), and
    the MFA derivative to 1e-12 relative.
  * Free-energy parts: 1e-11 relative.
  * Converged densities: 1e-9 relative to max rho at RES < 1e-11; the
    loading N and grand potential to 1e-9 relative.
  * The 24-pressure 64^3 isotherm at the reference's tolerance (RES < 1e-8):
    the same number of steps per pressure, N and Omega to 1e-10 relative.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from cmmdft_b200 import _lib as L, engine as E, batch as BT, workload as W
from cmmdft_b200.hosts import cubic_host_276, methane_guest_params
from cmmdft_b200.units import angstrom, kjmol, bar
from tests._common import relerr, scalar_rel, oracle_case


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


@pytest.fixture(scope="module")
def fn32(cuda):
    return W.build_functional(cubic_host_276(0), (32, 32, 32), 300.0, methane_guest_params())


# shapes: specialised 32/64 kernels; small-radix mixes; odd radices 7, 11, 13;
# prime factors > 16 on each axis (direct-DFT stages for 17..59 and for
# primes whose p - 1 has a factor > 16, Rader stages for 97, 127, 157) with
# even and odd N3 (full-length z); a 160^3 fused plane and a 256^3 plane
# beyond shared memory (staged passes)
FFT_SHAPES = [(32, 32, 32), (64, 64, 64), (64, 32, 32), (32, 64, 64), (24, 20, 18), (30, 28, 14), (16, 12, 10),
              (7, 9, 22), (34, 51, 53), (53, 58, 62), (48, 64, 45), (37, 19, 23), (17, 29, 34), (160, 160, 160),
              (256, 256, 256), (91, 26, 22), (143, 14, 126), (97, 20, 18), (20, 127, 22), (18, 20, 157),
              (59, 23, 17), (118, 59, 20)]


@pytest.mark.parametrize("staged", [0, 1])
@pytest.mark.parametrize("shape", FFT_SHAPES)
def test_rfft3d_matches_scipy(cuda, shape, staged):
    if staged and shape not in ((32, 32, 32), (64, 64, 64), (24, 20, 18)):
        pytest.skip("forced staging is exercised on the fused shapes")
    rng = np.random.default_rng(1)
    B = 1 if np.prod(shape) > 3e6 else 2
    x = rng.standard_normal((B,) + shape)
    rv = np.diag([10.0, 11.0, 12.0])
    plan = E.GridPlan(shape, rv)
    plan.set_staging(staged)
    xt = torch.as_tensor(x, device="cuda")
    spec = plan.rfft(xt)
    full = plan.spec_to_full(spec)
    ref = np.fft.fftn(x, axes=(1, 2, 3))
    # direct-DFT stages of a prime p accumulate p terms: ~p eps relative
    tol = 1e-13 if max(shape) < 100 else 4e-13
    assert relerr(full.real, ref.real, np.abs(ref).max()) < tol
    assert relerr(full.imag, ref.imag, np.abs(ref).max()) < tol
    back = plan.irfft(spec).cpu().numpy() / np.prod(shape)
    assert relerr(back, x) < tol
    # yz transforms (the solver's exchange format) round trip
    yz = plan.rfft_yz(xt)
    back = plan.irfft_yz(yz).cpu().numpy() / (shape[1] * shape[2])
    assert relerr(back, x) < tol


def test_external_potential(golden32, fn32):
    V = fn32.V.cpu().numpy()
    assert relerr(V, golden32["V"]) < 1e-13


def _c1(fn, rho_np):
    plan = fn.plan
    buf = E.Buffers(plan, 1, nwork=fn.nwork)
    buf.part[:, L.STAT_N3MAX, :] = -np.inf
    rho = torch.as_tensor(rho_np[None], device="cuda")
    spec = plan.rfft_yz(rho)
    chat = plan.new_spec(1)
    fn.c1(buf, spec, chat, want=7)
    E.finalize(buf, (1 << L.NSTAT) - 1)
    st = buf.stats.cpu().numpy()[0]
    C1 = plan.irfft_yz(chat).cpu().numpy()[0]
    dr = plan.dr
    return C1, st, (st[L.STAT_PHI] * dr) / fn.beta, 0.5 * st[L.STAT_MFA] * dr


@pytest.mark.parametrize("tag", ["a", "b"])
def test_functional_derivative(golden32, fn32, tag):
    rho = golden32["rho_" + tag]
    C1, st, Fhs, Fmfa = _c1(fn32, rho)
    ref = golden32["dHS_" + tag] + golden32["dMFA_" + tag]
    # same closed forms, different rounding: the GPU sits at the reference's
    # own noise floor (max at the n3 ~ 1e-8..1e-6 cancellation points)
    floor = {"a": 2e-9, "b": 1e-7}[tag]
    dC = fn32.beta * np.abs(C1 - ref)
    assert dC.max() < floor
    assert (dC * rho).max() / rho.max() < 1e-9
    vals = golden32["values_" + tag]
    assert scalar_rel(Fhs, vals[0]) < 1e-11
    assert scalar_rel(Fmfa, vals[1]) < 1e-11
    assert scalar_rel(st[L.STAT_N3MAX], golden32["n3_" + tag].max()) < 1e-12


def _hs_only(plan, ver, R, T=300.0):
    """Device functional of the hard-sphere part alone (no MFA kernel, V = 0)."""
    from cmmdft_b200.units import boltzmann
    return E.Functional(plan, R, 1.0 / (boltzmann * T), 1.0, torch.zeros(plan.npoints, dtype=torch.float64,
                                                                          device="cuda"), W.hs_version_code(ver))


TENSOR_CASES = [("atWBII", "a"), ("atWBII", "b"), ("tWBII", "a"), ("tWBII", "b"), ("atFMT", "b"), ("tMFMT", "b")]


@pytest.mark.parametrize("staged", [0, 1])
@pytest.mark.parametrize("ver,tag", TENSOR_CASES)
def test_tensor_hard_sphere(golden32, cuda, ver, tag, staged):
    """Tensor FMT variants against the reference's HardSphereFunctional."""
    plan = E.GridPlan((32, 32, 32), cubic_host_276(0).rvecs)
    plan.set_staging(staged)
    fn = _hs_only(plan, ver, float(golden32["Rhs"]))
    C1, st, Fhs, _ = _c1(fn, golden32["rho_" + tag])
    floor = {"a": 2e-9, "b": 1e-7}[tag]   # the WBII noise floor of the plain case
    assert fn.beta * np.max(np.abs(C1 - golden32["hs_%s_d_%s" % (ver, tag)])) < floor
    assert scalar_rel(Fhs, golden32["hs_%s_v_%s" % (ver, tag)]) < 1e-11


@pytest.mark.parametrize("ver", ["WBII", "aWBII", "atWBII"])
def test_tensor_64_against_oracle(cuda, ver):
    """The 64^3 kernels (compile-time transform lengths) against the oracle."""
    from oracle import cmm_oracle as O
    host = cubic_host_276(0)
    sig, eps, mass = methane_guest_params()
    fn = W.build_functional(host, (64, 64, 64), 300.0, (sig, eps, mass))
    R = fn.R
    V = fn.V.cpu().numpy()
    rho = 0.02 / angstrom ** 3 * np.clip(np.exp(-fn.beta * V), 0, 1)   # dense, sharp profile
    hs = _hs_only(fn.plan, ver, R)
    C1, st, Fhs, _ = _c1(hs, rho)
    og = O.OGrid(host.rvecs, npoints=64)
    ohs = O.HardSphere(og, R, 300.0, version=ver)
    k = og.fft(rho)
    ref = ohs.derive(k)
    dC = hs.beta * np.abs(C1 - ref)
    assert dC.max() < 1e-7
    assert (dC * rho).max() / rho.max() < 1e-9
    assert scalar_rel(Fhs, ohs.value(k)) < 1e-11


@pytest.mark.parametrize("wda", [False, True])
@pytest.mark.parametrize("n", [32, 64])
def test_staged_plane_pass_matches_fused(golden32, cuda, n, wda):
    """The staged form (y pass + z rows) against the fused plane kernel."""
    host = cubic_host_276(0)
    fn = W.build_functional(host, (n, n, n), 300.0, methane_guest_params(), wda=wda)
    V = fn.V.cpu().numpy()
    rho = 0.02 / angstrom ** 3 * np.clip(np.exp(-fn.beta * V), 0, 1)
    fn.plan.set_staging(0)
    C1a, sta, Fa, Ma = _c1(fn, rho)
    fn.plan.set_staging(1)
    C1b, stb, Fb, Mb = _c1(fn, rho)
    fn.plan.set_staging(0)
    assert np.max(np.abs(C1a - C1b)) <= 1e-12 * np.max(np.abs(C1a))
    assert scalar_rel(Fb, Fa) < 1e-12 and scalar_rel(Mb, Ma) < 1e-12
    assert scalar_rel(stb[L.STAT_N3MAX], sta[L.STAT_N3MAX]) < 1e-14
    if wda:
        assert scalar_rel(stb[L.STAT_WDA], sta[L.STAT_WDA]) < 1e-12


@pytest.mark.parametrize("tag", ["a", "b"])
def test_wda_part(golden32, cuda, tag):
    fn = W.build_functional(cubic_host_276(0), (32, 32, 32), 300.0, methane_guest_params(), wda=True)
    rho = golden32["rho_" + tag]
    C1, st, Fhs, Fmfa = _c1(fn, rho)
    ref = golden32["wda_C1_" + tag] - golden32["V"]
    floor = {"a": 2e-9, "b": 1e-7}[tag]   # the hard-sphere noise floor, as above
    assert fn.beta * np.max(np.abs(C1 - ref)) < floor
    Fwda = st[L.STAT_WDA] * fn.plan.dr
    assert scalar_rel(Fwda, golden32["wda_values_" + tag][3]) < 1e-11


def test_mfa_tailcorrections(golden32, cuda):
    fn = W.build_functional(cubic_host_276(0), (32, 32, 32), 300.0, methane_guest_params(),
                            tailcorrections=True)
    rho = golden32["rho_b"]
    C1, st, Fhs, Fmfa = _c1(fn, rho)
    assert scalar_rel(Fmfa, golden32["vMFA_tail_b"]) < 1e-11


TIGHT_CRIT = ['res', 'riue']
TIGHT_THR = [1e-13, 1e-12]


def _solve(fn, mu, rho0, method, thr, nsteps=500, crit='res', native=False):
    cls = BT.NativeBatchSolve if native else BT.BatchSolve
    s = cls(fn, np.atleast_1d(mu), method=method, nsteps=nsteps, threshold=thr, criterion=crit)
    r0 = torch.as_tensor(np.asarray(rho0)[None] if np.ndim(rho0) == 3 else rho0, device="cuda")
    N, rho, conv = s.solve(r0)
    return s, N, rho.cpu().numpy(), conv


@pytest.mark.parametrize("native", [False, True])
def test_static_picard_matches_reference(golden32, fn32, native):
    mu = float(golden32["mu"])
    s, N, rho, conv = _solve(fn32, mu, golden32["rho_a"], 'static', 1e-8, native=native)
    assert conv[0]
    assert s.steps[0] == int(golden32["picard_steps"])
    assert relerr(rho[0], golden32["picard_rho"]) < 1e-10
    assert scalar_rel(N[0], golden32["picard_N"]) < 1e-10


@pytest.mark.parametrize("native", [False, True])
def test_static_picard_der_criterion(golden32, fn32, native):
    mu = float(golden32["mu"])
    s, N, rho, conv = _solve(fn32, mu, golden32["rho_a"], 'static', [1e-3], crit=['der'], native=native)
    assert conv[0]
    assert s.steps[0] == int(golden32["der_steps"])
    assert relerr(rho[0], golden32["der_rho"]) < 1e-10
    assert scalar_rel(N[0], golden32["der_N"]) < 1e-10


@pytest.mark.parametrize("staged", [0, 1])
def test_static_picard_three_steps(golden32, fn32, staged):
    mu = float(golden32["mu"])
    fn32.plan.set_staging(staged)
    try:
        s, N, rho, conv = _solve(fn32, mu, golden32["rho_a"], 'static', 1e-30, nsteps=3)
    finally:
        fn32.plan.set_staging(0)
    assert not conv[0]
    assert relerr(rho[0], golden32["picard3_rho"]) < 1e-10


def test_staged_hybrid_anderson_matches_reference(golden32, fn32):
    """Residual, mix and Picard passes in their staged form."""
    mu = float(golden32["mu"])
    fn32.plan.set_staging(1)
    try:
        s, N, rho, conv = _solve(fn32, mu, golden32["rho_a"], 'hybridanderson', TIGHT_THR, nsteps=500,
                                 crit=TIGHT_CRIT)
    finally:
        fn32.plan.set_staging(0)
    assert conv[0]
    assert relerr(rho[0], golden32["and_rho"]) < 1e-9
    assert scalar_rel(N[0], golden32["and_N"]) < 1e-10


@pytest.mark.parametrize("ver", ["WBII", "atWBII"])
def test_uneven_grid_against_oracle(cuda, ver):
    """A grid with prime factors > 16 and odd N3 (51 x 58 x 45, all staged):
    external potential, C1 and three static Picard steps against the oracle."""
    from oracle import cmm_oracle as O
    host = cubic_host_276(0)
    sig, eps, mass = methane_guest_params()
    shape = (51, 58, 45)
    fn = W.build_functional(host, shape, 300.0, (sig, eps, mass), version=ver)
    og = O.OGrid(host.rvecs, npoints=list(shape))
    Vo = O.external_potential(og.points[..., :3].reshape(-1, 3), host.ff, sig, eps, host.recentred_pos(),
                              host.ffatypes, host.ffatype_ids, host.rvecs).reshape(shape)
    Vo = O.cap_potential(Vo, 1e4 * kjmol)
    V = fn.V.cpu().numpy()
    assert relerr(V, Vo) < 1e-13
    fe = O.build_functional(og, sig, eps, mass, 300.0, Vo, hs_version=ver)
    mu = W.isotherm_inputs(np.array([1.0]) * bar, 300.0, (sig, eps, mass))[0][0]
    rho0 = O.initial_density(fe, mu)
    s = O.Picard(fe, nsteps=1, method='static')
    s._initiate_solving(mu)
    C1o = s._get_C1(rho0) - Vo
    C1, st, Fhs, Fmfa = _c1(fn, rho0)
    dC = fn.beta * np.abs(C1 - C1o)
    assert dC.max() < 2e-9
    s3 = O.Picard(fe, nsteps=3, alpha_mix=0.1, method='static', criterion='res', threshold=1e-30)
    N3o, rho3o, _ = s3.solve(mu, rho0.copy())
    sg, N, rho, conv = _solve(fn, mu, rho0, 'static', 1e-30, nsteps=3)
    assert relerr(rho[0], rho3o) < 1e-10
    assert scalar_rel(N[0], N3o) < 1e-10


def test_solve_batch_uneven_hosts(cuda):
    """Three hosts of uneven cells and grids (53x53x62, 50x58x60 and
    52x49x53: prime factors and odd N3) solved concurrently by solve_batch
    equal their one-host solves exactly; the 52x49x53 host's 1 bar point
    against the oracle at the reference's tolerance (RES < 1e-8): the same
    number of steps and N within 1e-10."""
    from oracle import cmm_oracle as O
    from cmmdft_b200 import isotherm as ISO
    from cmmdft_b200.hosts import uneven_hosts
    hosts = uneven_hosts(nhost=3, seed=2, edge_range=(12.0, 16.0))
    guest = methane_guest_params()
    P = np.array([0.1, 1.0, 10.0]) * bar
    res = ISO.solve_batch(hosts, P, 300.0, guest, max_concurrent=3)
    for h, r in zip(hosts, res):
        one = ISO.solve_isotherm(h, P, 300.0, guest, ISO.grid_points(h), return_density=False)
        assert r['npoints'] == ISO.grid_points(h)
        assert np.array_equal(r['N'], one['N']) and np.array_equal(r['steps'], one['steps'])
    h = hosts[2]
    sig, eps, mass = guest
    shape = ISO.grid_points(h)
    og = O.OGrid(h.rvecs, npoints=list(shape))
    V = O.external_potential(og.points[..., :3].reshape(-1, 3), h.ff, sig, eps, h.recentred_pos(), h.ffatypes,
                             h.ffatype_ids, h.rvecs).reshape(shape)
    V = O.cap_potential(V, 1e4 * kjmol)
    fe = O.build_functional(og, sig, eps, mass, 300.0, V)
    mb = O.MBWR(mass, sig, eps)
    mu = O.eos_calculate_mu(mb, 300.0, P[1])
    mb.set_temperature(300.0)
    rb = np.nanmin(O.eos_densities_from_chempots(mb, [mu]), axis=1)[0]
    s = O.Anderson(fe, nsteps=500, m=5, criterion='res', threshold=1e-8)
    N, rho, conv = s.solve(mu, rb * np.exp(-np.maximum(V, 0) * fe.beta))
    assert conv and res[2]['converged'][1]
    assert res[2]['steps'][1] == s.curr_step
    assert scalar_rel(res[2]['N'][1], N) < 1e-10


def test_hybrid_anderson_matches_reference(golden32, fn32):
    mu = float(golden32["mu"])
    s, N, rho, conv = _solve(fn32, mu, golden32["rho_a"], 'hybridanderson', TIGHT_THR, nsteps=500,
                             crit=TIGHT_CRIT)
    assert conv[0]
    # both sides converged to RES < 1e-13 and RIUE < 1e-12
    assert relerr(rho[0], golden32["and_rho"]) < 1e-9
    assert scalar_rel(N[0], golden32["and_N"]) < 1e-10
    om = s.omega0[0]
    assert scalar_rel(om, golden32["and_omega"]) < 1e-10


def test_isotherm_64_matches_reference(golden64, cuda):
    host = cubic_host_276(0)
    guest = methane_guest_params()
    fn = W.build_functional(host, (64, 64, 64), 300.0, guest)
    P = golden64["pressures"]
    ok = golden64["steps"] < 500  # points the reference itself converged
    mus, bulks = W.isotherm_inputs(P * bar, 300.0, guest)
    assert np.array_equal(mus, golden64["mu"])
    r0 = W.initial_density(fn, mus, ninit=bulks)
    s = BT.BatchSolve(fn, mus, method='hybridanderson', nsteps=500, threshold=TIGHT_THR,
                      criterion=TIGHT_CRIT)
    host = torch.empty(tuple(r0.shape), dtype=torch.float64, pin_memory=True)
    N, rho, conv = s.solve(r0, host_out=host)
    assert torch.equal(host, rho.cpu())   # copied per instance while the batch ran
    assert conv[ok].all()
    for i in np.where(ok)[0]:
        assert scalar_rel(N[i], golden64["N"][i]) < 1e-10
        assert scalar_rel(s.omega0[i], golden64["omega"][i]) < 1e-10
    i1 = int(np.where(P == 1.0)[0][0])
    assert relerr(rho[i1].cpu().numpy(), golden64["rho_1bar"]) < 1e-9


@pytest.mark.parametrize("case", ["wbii64", "atwbii_wda32"])
def test_line_search_matches_pipeline(cuda, case):
    """Omega(rho + alpha r) and alpha_max of the hybrid step from the stored
    weighted densities (cmm_ls_*) against full evaluations of the trial
    densities through the functional pipeline."""
    host = cubic_host_276(0)
    guest = methane_guest_params()
    if case == "wbii64":
        fn = W.build_functional(host, (64, 64, 64), 300.0, guest)
    else:
        fn = W.build_functional(host, (32, 32, 32), 300.0, guest, version='atWBII', wda=True)
    P = np.array([1e-3, 1.0, 10.0]) * bar
    mus, bulks = W.isotherm_inputs(P, 300.0, guest)
    r0 = W.initial_density(fn, mus, ninit=bulks)
    s = BT.BatchSolve(fn, mus, method='hybridanderson', nsteps=10, threshold=1e-8, criterion='res')
    s.initial_density(r0)
    s.cf = np.ones(3)
    s._set_params()
    live = np.ones(3, dtype=bool)
    s._init_state(live)
    s._set_active(live)
    s._residual(s.chat, s.ring[0], s.rres[0], [])
    s._stats()
    # line search sums
    s._set_active(live)
    s._set_params(n3=s.n3max)
    fn.ls_prepare(s.buf, s.rres[0], s.spec_ring[0], s.wd_ring[0], s.rhat, s.wd_r, s.ls_part, active=s.active)
    coefs = (0.45, 0.9, 0.225)
    fn.ls_omega(s.buf, s.params[:, 3], coefs, s.ring[0], s.rres[0], s.wd_ring[0], s.wd_r, s.ls_part, s.ls_alpha,
                active=s.active)
    fn.ls_finalize(s.buf, s.ls_part, s.ls, active=s.active)
    ls = s.ls.cpu().numpy()
    amax = s.ls_alpha.cpu().numpy()
    # alpha_max from a pipeline evaluation of G = rho + r (solver.py:150-165)
    stn = s._eval_density(live, np.ones((3, 2)), [s.ring[0], s.rres[0]], L.CLIP_NONE, s.trial, 4, s.ring[0])
    for b in range(3):
        a, g = s.n3max[b], stn[b, L.STAT_N3MAX]
        ref = np.min([abs((1 - a) / ((g - a) + 1e-16)), 1])
        assert scalar_rel(amax[b], ref) < 1e-12
        assert scalar_rel(ls[b, L.LS_N3MAX_G], g) < 1e-12
    for i, c in enumerate(coefs):
        om_pipe = s._trial_omega(live, c * amax, 0)
        for b in range(3):
            om_ls = s._ls_omega(ls[b], b, i, c * amax[b])
            assert scalar_rel(om_ls, om_pipe[b]) < 1e-12, (case, i, b, om_ls, om_pipe[b])


@pytest.mark.parametrize("native", [False, True])
@pytest.mark.parametrize("groups", [2, 3])
def test_grouped_solve_equals_single_batch(cuda, groups, native):
    """Instances are independent: groups on concurrent streams reproduce the
    single batched solve exactly."""
    host = cubic_host_276(0)
    guest = methane_guest_params()
    fn = W.build_functional(host, (32, 32, 32), 300.0, guest)
    P = np.logspace(-3, 1.3, 7) * bar
    mus, bulks = W.isotherm_inputs(P, 300.0, guest)
    r0 = W.initial_density(fn, mus, ninit=bulks)
    kw = dict(method='hybridanderson', nsteps=200, threshold=1e-10, criterion='res')
    s1 = (BT.NativeBatchSolve if native else BT.BatchSolve)(fn, mus, **kw)
    N1, rho1, c1 = s1.solve(r0)
    sg = BT.GroupedSolve(fn, mus, groups=groups, native=native, **kw)
    host_out = torch.empty(tuple(r0.shape), dtype=torch.float64, pin_memory=True)
    N2, rho2, c2 = sg.solve(r0, host_out=host_out)
    assert np.array_equal(c1, c2) and np.array_equal(s1.steps, sg.steps)
    assert np.array_equal(N1, N2)
    assert torch.equal(rho1, rho2)
    assert torch.equal(host_out, rho2.cpu())


@pytest.mark.parametrize("method,case", [("hybridanderson", "wbii"), ("hybrid", "wbii"), ("anderson", "wbii"), ("static", "wbii"),
                                         ("hybridanderson", "atwbii_wda")])
def test_native_driver_equals_python_driver(cuda, method, case):
    """cmm_solve_batched (C++ loop) against BatchSolve (Python loop): the same
    kernels and decisions, so the same steps and densities."""
    host = cubic_host_276(0)
    guest = methane_guest_params()
    kw = {} if case == "wbii" else dict(version='atWBII', wda=True)
    fn = W.build_functional(host, (32, 32, 32), 300.0, guest, **kw)
    P = np.logspace(-3, 1.5, 6) * bar
    mus, bulks = W.isotherm_inputs(P, 300.0, guest)
    r0 = W.initial_density(fn, mus, ninit=bulks)
    opts = dict(method=method, nsteps=120, threshold=1e-10, criterion='res', divergence_guard=True)
    sp = BT.BatchSolve(fn, mus, **opts)
    Np, rp, cp = sp.solve(r0)
    sn = BT.NativeBatchSolve(fn, mus, **opts)
    host_out = torch.empty(tuple(r0.shape), dtype=torch.float64, pin_memory=True)
    Nn, rn, cn = sn.solve(r0, host_out=host_out)
    assert np.array_equal(cp, cn)
    assert np.array_equal(sp.steps, sn.steps), (sp.steps, sn.steps)
    ok = np.isfinite(Np)
    assert np.all(np.abs(Nn[ok] - Np[ok]) <= 1e-12 * np.abs(Np[ok]))
    assert relerr(rn.cpu().numpy(), rp.cpu().numpy()) < 1e-10
    assert torch.equal(host_out, rn.cpu())
    assert np.allclose(sn.omega0[ok], sp.omega0[ok], rtol=1e-12, atol=0)


@pytest.fixture(scope="module")
def iso64():
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "iso64_res8.npz")
    if not os.path.exists(path):
        pytest.skip("isotherm fixture not generated")
    return dict(np.load(path))


@pytest.fixture(scope="module")
def iso64_rho():
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "iso64_rho.npz")
    if not os.path.exists(path):
        pytest.skip("isotherm density fixture not generated")
    return dict(np.load(path))


@pytest.mark.parametrize("native", [True, False])
def test_isotherm64_at_reference_tolerance(cuda, iso64, iso64_rho, native):
    """The 24-pressure 64^3 isotherm as the reference's example solves it
    (hybrid Anderson m=5, RES < 1e-8, Ninit = rho_bulk).  At this tolerance
    the result depends on the whole trajectory, SLSQP coefficients included:
    every pressure the reference converges takes the same number of steps and
    reaches density, N_abs, N_ex and Omega within 1e-10 relative (density:
    max |diff| / max rho at the stored pressures; N_ex from the GPU helium
    fraction against the reference's Calculator.return_loading(excess=True));
    the three it does not converge (it diverges there) are retired as not
    converged by the divergence guard."""
    guest = methane_guest_params()
    fn = W.build_functional(cubic_host_276(0), (64, 64, 64), 300.0, guest)
    mus, bulks = W.isotherm_inputs(iso64["pressures"] * bar, 300.0, guest)
    assert np.array_equal(mus, iso64["mu"])
    r0 = W.initial_density(fn, mus, ninit=bulks)
    cls = BT.NativeBatchSolve if native else BT.BatchSolve
    s = cls(fn, mus, method='hybridanderson', nsteps=500, threshold=1e-8, criterion='res', divergence_guard=True)
    N, rho, conv = s.solve(r0)
    ok = iso64["converged"].astype(bool)
    assert np.array_equal(np.asarray(conv, dtype=bool), ok)
    assert np.array_equal(s.steps[ok], iso64["steps"][ok]), (s.steps, iso64["steps"])
    from cmmdft_b200.adjoint import helium_fraction
    he = helium_fraction(fn.plan, cubic_host_276(0), 300.0)
    vol = cubic_host_276(0).volume
    Nex = np.asarray(N) - bulks * he * vol
    err = dict(rho=0.0, N_abs=0.0, N_ex=0.0, Omega=0.0)
    for i in np.where(ok)[0]:
        err['N_abs'] = max(err['N_abs'], scalar_rel(N[i], iso64["N"][i]))
        err['N_ex'] = max(err['N_ex'], scalar_rel(Nex[i], iso64["N_ex"][i]))
        err['Omega'] = max(err['Omega'], scalar_rel(s.omega0[i], iso64["omega"][i]))
    # The reference against itself: re-solved from a start one ulp away, its
    # own densities move by floor[j, 0] (3e-11 at 1.1 bar, 3e-10 at 8.2 bar);
    # a density is held to 1e-10 or to three times that floor.
    rho_err, rho_tol = [], []
    for j, i in enumerate(iso64_rho["idx"]):
        rho_err.append(relerr(rho[i].cpu().numpy(), iso64_rho["rho_%d" % i]))
        rho_tol.append(max(1e-10, 3 * iso64_rho["floor"][j, 0]))
    err['rho'] = max(rho_err)
    print("iso64 max relative errors vs the reference:", {k: "%.2e" % v for k, v in err.items()},
          "helium fraction %.2e" % scalar_rel(he, iso64["he_frac"]),
          "| rho per stored pressure %s, reference's own 1-ulp floor %s"
          % (["%.2e" % e for e in rho_err], ["%.2e" % f for f in iso64_rho["floor"][:, 0]]))
    assert scalar_rel(he, iso64["he_frac"]) < 1e-12
    for k in ('N_abs', 'N_ex', 'Omega'):
        assert err[k] < 1e-10, (k, err[k])
    for e, t in zip(rho_err, rho_tol):
        assert e < t, (rho_err, rho_tol)


def test_native_driver_matches_reference(golden32, fn32):
    mu = float(golden32["mu"])
    s = BT.NativeBatchSolve(fn32, np.atleast_1d(mu), method='hybridanderson', nsteps=500, threshold=TIGHT_THR,
                            criterion=TIGHT_CRIT)
    N, rho, conv = s.solve(torch.as_tensor(golden32["rho_a"][None], device="cuda"))
    assert conv[0]
    assert relerr(rho[0].cpu().numpy(), golden32["and_rho"]) < 1e-9
    assert scalar_rel(N[0], golden32["and_N"]) < 1e-10
    assert scalar_rel(s.omega0[0], golden32["and_omega"]) < 1e-10


@pytest.mark.parametrize("host_name,npts", [("cubic_host_779", (96, 96, 96)), ("cubic_host_64", (64, 64, 64)),
                                            ("uneven_host_1", None)])
def test_extpot_cell_list_matches_all_atom(cuda, host_name, npts):
    """The cell-list external potential (tiles of grid points with the atoms
    within the cutoff staged in shared memory) against the all-atom form on
    the same grid: the same pairs summed in another order, 1e-13 relative to
    the cap."""
    from cmmdft_b200 import hosts as H
    if host_name == "uneven_host_1":
        host = H.uneven_hosts(nhost=2)[1]
        npts = tuple(int(np.ceil(np.linalg.norm(host.rvecs[a]) / (0.25 * angstrom))) for a in range(3))
    else:
        host = getattr(H, host_name)()
    guest = methane_guest_params()
    plan = E.GridPlan(npts, host.rvecs)
    sig, eps = W.host_type_arrays(host)
    cap = 1e4 * kjmol
    lib = L.lib()
    out = {}
    try:
        for mode in (1, 2):
            assert lib.cmm_extpot_set_mode(mode) == 0
            out[mode] = E.external_potential(plan, host.recentred_pos(), host.ffatype_ids, sig, eps, guest[0],
                                             guest[1], 12 * angstrom, cap).cpu().numpy()
    finally:
        lib.cmm_extpot_set_mode(0)
    err = relerr(out[1], out[2], cap)
    print("%s %s: cell list vs all atoms %.2e of the cap" % (host_name, npts, err))
    assert err < 1e-13


def test_extpot_256_against_oracle(cuda):
    """The 256^3 grid of the 64 A host (14,680 atoms, cell-list form by size)
    against the oracle's get_external_potential restatement at 4096 seeded
    grid points: 1e-12 relative to the cap."""
    from cmmdft_b200.hosts import cubic_host_64
    from oracle import cmm_oracle as O
    host = cubic_host_64()
    guest = methane_guest_params()
    n = 256
    plan = E.GridPlan((n, n, n), host.rvecs)
    sig, eps = W.host_type_arrays(host)
    cap = 1e4 * kjmol
    V = E.external_potential(plan, host.recentred_pos(), host.ffatype_ids, sig, eps, guest[0], guest[1],
                             12 * angstrom, cap).cpu().numpy()
    rng = np.random.default_rng(11)
    idx = rng.integers(0, n, size=(4096, 3))
    g = np.linspace(-0.5, 0.5, n, endpoint=False)
    frac = g[idx]
    pts = np.einsum('ab,ia->ib', host.rvecs, frac)       # Grid.points
    Vo = O.external_potential(pts, host.ff, guest[0], guest[1], host.recentred_pos(), host.ffatypes,
                              host.ffatype_ids, host.rvecs)
    Vo = O.cap_potential(Vo, cap)
    err = relerr(V[idx[:, 0], idx[:, 1], idx[:, 2]], Vo, cap)
    print("256^3 extpot vs oracle at 4096 points: %.2e of the cap" % err)
    assert err < 1e-12


def test_uneven_host_at_spacing_grid_against_reference(cuda):
    """Host 5 of the uneven batch (uneven_hosts(8, 2): 29.7 x 39.1 x 31.1 A,
    2026 atoms) on its 0.25 A grid, 119 x 157 x 125 -- 157 prime (Rader
    stages on y), 119 = 7 x 17 -- at 0.1, 1 and 10 bar against the unmodified
    reference (tests/golden/uneven5.npz, hybrid Anderson m=5, RES < 1e-8,
    Ninit = rho_bulk): the same steps, N and Omega within 1e-10."""
    import os
    from cmmdft_b200 import isotherm as ISO
    from cmmdft_b200.hosts import uneven_hosts
    ref = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "uneven5.npz")))
    host = uneven_hosts(8, 2)[int(ref["host"])]
    guest = methane_guest_params()
    shape = ISO.grid_points(host)
    assert list(shape) == list(ref["npoints"])
    mus, bulks = W.isotherm_inputs(ref["pressures"] * bar, 300.0, guest)
    assert np.array_equal(mus, ref["mu"])
    fn = W.build_functional(host, shape, 300.0, guest)
    s = BT.NativeBatchSolve(fn, mus, method='hybridanderson', nsteps=500, threshold=1e-8, criterion='res')
    N, rho, conv = s.solve(W.initial_density(fn, mus, ninit=bulks))
    eN = max(scalar_rel(N[i], ref["N"][i]) for i in range(len(mus)))
    eO = max(scalar_rel(s.omega0[i], ref["omega"][i]) for i in range(len(mus)))
    print("uneven host 5 %s: steps %s (reference %s), N %.2e, Omega %.2e" % (shape, list(s.steps), list(ref["steps"]),
                                                                              eN, eO))
    assert np.all(conv) and np.array_equal(s.steps, ref["steps"])
    assert eN < 1e-10 and eO < 1e-10


@pytest.mark.parametrize("shape,wda,host_kind", [((32, 32, 32), False, "c"), ((64, 64, 64), False, "c"),
                                                 ((64, 64, 64), True, "c"), ((40, 36, 30), False, "o"),
                                                 ((28, 42, 26), True, "o")])
def test_split_plane_pass_is_bit_identical(cuda, shape, wda, host_kind):
    """The fused plane pass with the plane split over a 2-CTA cluster
    (staging mode 0, the default) gives bit for bit the one-CTA pass's
    (mode 2) C1 spectrum,
    reductions and stored weighted densities: compile-time 32/64 lengths,
    run-time lengths and a radix-7 axis, with and without the WDA field."""
    from cmmdft_b200.hosts import random_sequential_host
    host = cubic_host_276(0) if host_kind == "c" else random_sequential_host((14.0, 15.0, 13.0), 150, 3)
    sig, eps, mass = methane_guest_params()
    fn = W.build_functional(host, shape, 300.0, (sig, eps, mass), wda=wda)
    plan = fn.plan
    V = fn.V.cpu().numpy()
    B = 3
    rho = np.stack([s * 0.02 / angstrom ** 3 * np.clip(np.exp(-fn.beta * V), 0, 1) for s in (0.2, 0.6, 1.0)])
    rt = torch.as_tensor(rho, device="cuda")
    nwd = fn.nwd() if callable(fn.nwd) else fn.nwd
    outs = []
    for mode in (0, 2):
        plan.set_staging(mode)
        buf = E.Buffers(plan, B, nwork=fn.nwork)
        buf.part[:, L.STAT_N3MAX, :] = -np.inf
        chat = plan.new_spec(B)
        wd = torch.zeros((nwd, B) + tuple(plan.npoints), dtype=torch.float64, device="cuda")
        fn.c1(buf, plan.rfft_yz(rt), chat, want=15, wd=wd)
        torch.cuda.synchronize()
        outs.append((chat.cpu().numpy(), buf.part.cpu().numpy(), wd.cpu().numpy()))
    plan.set_staging(0)
    (c0, p0, w0), (c2, p2, w2) = outs
    assert np.array_equal(c0, c2)
    assert np.array_equal(p0, p2)
    assert np.array_equal(w0, w2)


@pytest.mark.parametrize("guard", [False, True])
def test_static_device_loop_matches_host_loop(cuda, guard):
    """Static Picard with the decisions in k_static_decide and the step
    replayed as a CUDA graph (the native driver's default) against the host
    decisions after every step: the same densities, loadings, step counts,
    divergence flags and per-step history, bit for bit, for four pressures
    (0.01 to 10 bar) with and without the divergence guard."""
    import time
    guest = methane_guest_params()
    fn = W.build_functional(cubic_host_276(0), (32, 32, 32), 300.0, guest)
    mus, bulks = W.isotherm_inputs(np.array([0.01, 0.3, 1.0, 10.0]) * bar, 300.0, guest)
    r0 = W.initial_density(fn, mus, ninit=bulks)
    outs, times = [], []
    for dl in (False, True):
        s = BT.NativeBatchSolve(fn, mus, method='static', nsteps=700, threshold=1e-8, criterion='res',
                                divergence_guard=guard, track_history=True)
        s.device_loop = dl
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        N, rho, conv = s.solve(r0.clone())
        torch.cuda.synchronize()
        times.append(time.perf_counter() - t0)
        outs.append((np.asarray(N), rho.cpu().numpy(), np.asarray(conv), np.asarray(s.steps),
                     np.asarray(s.diverged), [np.asarray(h) for h in s.history]))
    (Nh, rh, ch, sh, dh, hh), (Nd, rd, cd_, sd, dd, hd) = outs
    print("static Picard, 4 pressures at 32^3: steps %s, host loop %.3f s, device loop %.3f s"
          % (list(sd), times[0], times[1]))
    assert np.array_equal(Nh, Nd) and np.array_equal(rh, rd)
    assert np.array_equal(ch, cd_) and np.array_equal(sh, sd) and np.array_equal(dh, dd)
    for a, b in zip(hh, hd):
        assert a.shape == b.shape and np.array_equal(np.isnan(a), np.isnan(b)) and np.array_equal(a[~np.isnan(a)], b[~np.isnan(b)])
