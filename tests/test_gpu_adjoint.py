"""Implicit-adjoint gradients on the GPU.

Checks, with the tolerance stated per test:
  * the Hessian-vector product A v of cmm_fmt_hvp against central
    differences of C1 along v;
  * its transpose (conjugate MFA spectrum) through u . (A v) = v . (A^T u);
  * cmm_extpot_lj_grad against central differences of the external potential;
  * dN/dtheta, dOmega/dtheta and dN_ex/dtheta against central differences of
    re-converged solves (relative step 1e-5, as the differentiation workload
    specifies), at 32^3 and on the 96^3 excess isotherm through the
    torch.autograd.Function;
  * one gradient against central differences of the oracle (the reference's
    numpy path) re-converged on the CPU.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from cmmdft_b200 import _lib as L, engine as E, workload as W, adjoint as A
from cmmdft_b200.hosts import cubic_host_276, cubic_host_779, methane_guest_params
from cmmdft_b200.units import angstrom, kjmol, bar
from tests._common import oracle_case


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


def _c1_fields(fn, rho):
    plan = fn.plan
    B = rho.shape[0]
    buf = E.Buffers(plan, B, nwork=fn.nwork)
    chat = plan.new_spec(B)
    fn.c1(buf, plan.rfft_yz(rho), chat, want=1)
    return plan.irfft_yz(chat)


def _wd(fn, rho):
    plan = fn.plan
    B = rho.shape[0]
    buf = E.Buffers(plan, B, nwork=fn.nwork)
    wd = torch.empty((fn.nwd, B) + plan.npoints, dtype=torch.float64, device="cuda")
    fn.c1(buf, plan.rfft_yz(rho), None, want=8, wd=wd)
    return wd


def _smooth_fields(npts, B, seed):
    """A dense, smooth density (packing fraction 0.12-0.28) and a smooth
    direction: a few low Fourier modes with seeded amplitudes."""
    rng = np.random.default_rng(seed)
    x = [np.arange(n) / n for n in npts]
    X, Y, Z = np.meshgrid(*x, indexing='ij')

    def field():
        f = np.zeros(npts)
        for _ in range(6):
            k = rng.integers(0, 3, 3)
            ph = rng.uniform(0, 2 * np.pi)
            f += rng.uniform(-1, 1) * np.cos(2 * np.pi * (k[0] * X + k[1] * Y + k[2] * Z) + ph)
        return f / np.abs(f).max()
    R = 1.7 * angstrom                                  # about the methane hard-sphere radius
    rho0 = 0.2 / (4.0 / 3.0 * np.pi * R ** 3)           # packing fraction 0.2
    rho = np.stack([rho0 * (1 + 0.4 * field()) for _ in range(B)])
    v = np.stack([rho[b] * field() for b in range(B)])
    return torch.as_tensor(rho, device="cuda"), torch.as_tensor(v, device="cuda")


@pytest.mark.parametrize("version", ["WBII", "atWBII", "tWBII", "MFMT", "FMT", "WBII+WDA", "atWBII+WDA"])
def test_hvp_matches_directional_difference(cuda, version):
    """On a smooth dense profile A v against the central difference of C1
    along v (truncation ~eps^2 = 1e-8, rounding ~1e-16 / eps).  The physical
    profiles are not used here: where the packing fraction is tiny the WBII
    and MFMT expressions cancel catastrophically, and central differences of
    C1 there change by tens of percent between eps = 1e-3 and 1e-4."""
    ver, wda = version.replace('+WDA', ''), version.endswith('+WDA')
    fn = W.build_functional(cubic_host_276(0), (32, 32, 32), 300.0, methane_guest_params(), version=ver, wda=wda)
    rho, v = _smooth_fields((32, 32, 32), 2, 5)
    Av = A.hvp(fn, _wd(fn, rho), v)
    eps = 1e-4
    fd = (_c1_fields(fn, rho + eps * v) - _c1_fields(fn, rho - eps * v)) / (2 * eps)
    err = (Av - fd).abs().max().item() / fd.abs().max().item()
    assert err < 1e-6, err


@pytest.mark.parametrize("kind", ["smooth", "noise"])
def test_hvp_transpose(cuda, golden32, kind):
    """u . (A v) = v . (A^T u) for the hard-sphere part (transposed pointwise
    Jacobian at clipped n3) to 1e-7 relative -- the rounding of the WBII
    second derivatives where the packing fraction is tiny leaves ~1e-8 -- and
    for the MFA part (conjugate kernel spectrum) to 1e-12."""
    fn = W.build_functional(cubic_host_276(0), (32, 32, 32), 300.0, methane_guest_params())
    rho = torch.as_tensor(golden32["rho_b"][None], device="cuda")
    wd = _wd(fn, rho)
    if kind == "smooth":
        _, u = _smooth_fields((32, 32, 32), 1, 7)
        _, v = _smooth_fields((32, 32, 32), 1, 8)
    else:
        rng = np.random.default_rng(4)
        u = torch.as_tensor(rng.standard_normal(rho.shape), device="cuda")
        v = torch.as_tensor(rng.standard_normal(rho.shape), device="cuda")
    kst = fn.kst
    fn.kst = torch.zeros_like(kst)          # hard-sphere part alone
    hs = (float((u * A.hvp(fn, wd, v)).sum()), float((v * A.hvp(fn, wd, u, transpose=True)).sum()))
    fn.kst = kst
    fm = E.Functional(fn.plan, fn.R, fn.beta, fn.wavelength, fn.V, L.NOHS, kst)
    mf = (float((u * A.hvp(fm, wd, v)).sum()), float((v * A.hvp(fm, wd, u, transpose=True)).sum()))
    rel = lambda p: abs(p[0] - p[1]) / max(abs(p[0]), 1e-300)  # noqa: E731
    assert rel(hs) < 1e-7 and rel(mf) < 1e-12, dict(hs=hs, mfa=mf, rel_hs=rel(hs), rel_mfa=rel(mf))


def test_extpot_grad_matches_difference(cuda):
    host = cubic_host_276(0)
    guest = methane_guest_params()
    plan = E.GridPlan((32, 32, 32), host.rvecs)
    vcap = 1e4 * kjmol
    theta = A.pack_params(host, guest)

    def V(th):
        h, g = A.unpack_params(th, host, guest)
        hs, he = W.host_type_arrays(h)
        return E.external_potential(plan, h.recentred_pos(), h.ffatype_ids, hs, he, g[0], g[1], 12 * angstrom,
                                    vcap).reshape(-1)

    D = A._dv_fields(plan, host, guest[0], guest[1], 12 * angstrom, vcap)
    keep = V(theta) < 0.9 * vcap   # away from the cap, where the derivative jumps
    for k in range(len(theta)):
        h = 1e-5 * theta[k]
        tp, tm = theta.copy(), theta.copy()
        tp[k] += h
        tm[k] -= h
        fd = (V(tp) - V(tm)) / (2 * h)
        err = (D[k][keep] - fd[keep]).abs().max().item() / fd[keep].abs().max().item()
        assert err < 1e-6, (k, err)


TIGHT = dict(threshold=1e-12, criterion='riue')


@pytest.mark.parametrize("wda", [False, True])
def test_adjoint_gradients_match_resolved_differences(cuda, wda):
    """N, Omega and N_ex gradients (all 10 parameters, 3 pressures) against
    central differences of re-converged solves, each d/d ln theta within 1e-6
    of the largest of that pressure's and quantity's entries (1e-5 for Omega:
    d Omega / d theta deviates for every parameter, by ~4e-8 of that scale at
    1 bar, ~4e-7 at 3 bar and 4e-6 to 9e-6 at 10 bar, the same for central
    differences with relative steps from 3e-4 down to 1e-5, so it is no
    difference error; it is 0.2-0.5% of the adjoint correction from Omega's
    non-stationarity, cause not found).  With the WDA part the same bounds
    hold.  Step
    1e-4 for the solves: stopped at RIUE < 1e-12 they sit ~1e-11 from the
    fixed point, which a 1e-5 step would turn into ~1e-6 of noise;
    truncation at 1e-4 is ~1e-8."""
    host = cubic_host_276(0)
    guest = methane_guest_params()
    # (with the WDA part the 10 bar point does not reach RIUE < 1e-12 at every
    # perturbed parameter set: 0.3, 1 and 3 bar there)
    P = (np.array([0.3, 1.0, 3.0]) if wda else np.array([1.0, 3.0, 10.0])) * bar
    model = A.IsothermModel(host, guest, 300.0, (32, 32, 32), P, quantity='excess', wda=wda, **TIGHT)
    theta = model.theta0
    sol = model.solve(theta)
    assert np.all(sol['converged'])
    g = A.adjoint_gradients(sol['fn'], sol['host'], sol['guest'], 300.0, P, sol['mu'], sol['rho'])
    assert max(g['residual'][0].max(), g['residual'][1].max()) < 1e-10

    def values(th):
        s = model.solve(th)
        assert np.all(s['converged'])
        gg = A.adjoint_gradients(s['fn'], s['host'], s['guest'], 300.0, P, s['mu'], s['rho'])
        return gg['N'], gg['Omega'], gg['Nex']

    # N and Omega with a relative step of 1e-4; N_ex - N (EOS bulk density
    # and helium fraction, no solve) with 1e-5, since the helium fraction's
    # clip at V_He = 0 is a kink whose difference error grows with the step
    fd = {key: np.zeros_like(g[key]) for key in ('dN', 'dOmega', 'dNex')}
    for k in range(len(theta)):
        for rel in (1e-4, 1e-5):
            h = rel * theta[k]
            tp, tm = theta.copy(), theta.copy()
            tp[k] += h
            tm[k] -= h
            vp, vm = values(tp), values(tm)
            if rel == 1e-4:
                fd['dN'][:, k] = (vp[0] - vm[0]) / (2 * h)
                fd['dOmega'][:, k] = (vp[1] - vm[1]) / (2 * h)
            else:
                fd['dNex'][:, k] = (vp[2] - vp[0] - vm[2] + vm[0]) / (2 * h)
    fd['dNex'] += fd['dN']
    worst = {}
    for key in fd:
        a, f = g[key] * theta[None, :], fd[key] * theta[None, :]
        scale = np.abs(f).max(axis=1, keepdims=True)
        err = np.abs(a - f) / scale
        worst[key] = (float(err.max()), g['names'][int(np.argmax(err.max(axis=0)))])
    tol = dict(dN=1e-6, dNex=1e-6, dOmega=1e-5)
    print("adjoint vs re-converged central differences%s, worst relative errors:" % (" (WDA)" if wda else ""), worst)
    assert all(w[0] < tol[k] for k, w in worst.items()), worst


def test_excess_isotherm_loss_gradient_96(cuda):
    """The differentiation workload: squared error of a 16-point excess
    isotherm (0.01..10 bar) at 96^3 (a = 24 angstrom, 779 atoms) against a
    target from +-10% perturbed parameters (seed 3); the autograd gradient
    against central differences (relative step 1e-5) of the re-converged loss."""
    host = cubic_host_779(0)
    guest = methane_guest_params()
    P = np.logspace(-2, 1, 16) * bar
    model = A.IsothermModel(host, guest, 300.0, (96, 96, 96), P, quantity='excess', **TIGHT)
    theta0 = model.theta0
    rng = np.random.default_rng(3)
    target_theta = theta0 * (1 + rng.uniform(-0.1, 0.1, theta0.shape))
    with torch.no_grad():
        target = model(torch.as_tensor(target_theta)).clone()
    theta = torch.tensor(theta0.copy(), requires_grad=True)
    loss = ((model(theta) - target) ** 2).sum()
    loss.backward()
    grad = theta.grad.numpy()

    def lossval(th):
        with torch.no_grad():
            return float(((model(torch.as_tensor(th)) - target) ** 2).sum())

    scale = np.abs(grad * theta0).max()
    for k in range(len(theta0)):   # guest eps, sigma and every host type's eps and sigma
        h = 1e-5 * theta0[k]
        tp, tm = theta0.copy(), theta0.copy()
        tp[k] += h
        tm[k] -= h
        fd = (lossval(tp) - lossval(tm)) / (2 * h)
        assert abs(grad[k] - fd) * theta0[k] <= 1e-6 * scale, (k, grad[k], fd)


def test_gradient_against_oracle_differences(cuda):
    """dN/d(guest epsilon), dN/d(epsilon_C) and dN/d(sigma_C) at 32^3 and
    1 bar against central differences of the oracle (the reference's numpy
    path) re-converged on the CPU: the host parameters within 1e-6, the
    guest epsilon (which also moves the hard-sphere radius and the EOS)
    within 1e-5."""
    from oracle import cmm_oracle as O
    host = cubic_host_276(0)
    guest = methane_guest_params()
    P = np.array([1.0]) * bar
    model = A.IsothermModel(host, guest, 300.0, (32, 32, 32), P, quantity='absolute', **TIGHT)
    sol = model.solve(model.theta0)
    g = A.adjoint_gradients(sol['fn'], sol['host'], sol['guest'], 300.0, P, sol['mu'], sol['rho'], excess=False)
    sig, eps, mass = guest

    def oracle_N(e, h=None):
        grid, fe = oracle_case(32, guest=(sig, e, mass), host=h)
        mb = O.MBWR(mass, sig, e)
        mu = O.eos_calculate_mu(mb, 300.0, P[0])
        mb.set_temperature(300.0)
        rb = np.nanmin(O.eos_densities_from_chempots(mb, [mu]), axis=1)[0]
        V = fe.part_dict["ExtPot"].potential
        rho0 = rb * np.exp(-np.maximum(V, 0) * fe.beta)
        s = O.Anderson(fe, nsteps=500, m=5, criterion=TIGHT['criterion'], threshold=TIGHT['threshold'])
        N, rho, conv = s.solve(mu, rho0)
        assert conv
        return N

    h = 1e-4 * eps
    fd = (oracle_N(eps + h) - oracle_N(eps - h)) / (2 * h)
    errs = {'guest_epsilon': abs(g['dN'][0, 0] - fd) / abs(fd)}
    theta = model.theta0
    for k in (2, 6):   # epsilon and sigma of the first host atom type
        hk = 1e-4 * theta[k]
        tp, tm = theta.copy(), theta.copy()
        tp[k] += hk
        tm[k] -= hk
        fdk = (oracle_N(eps, A.unpack_params(tp, host, guest)[0]) -
               oracle_N(eps, A.unpack_params(tm, host, guest)[0])) / (2 * hk)
        errs[g['names'][k]] = abs(g['dN'][0, k] - fdk) / abs(fdk)
    print("dN/dtheta vs oracle central differences, relative errors:", {k: "%.2e" % v for k, v in errs.items()})
    assert errs['guest_epsilon'] <= 1e-5
    assert errs[g['names'][2]] <= 1e-6 and errs[g['names'][6]] <= 1e-6
