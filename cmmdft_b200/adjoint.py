"""Gradients of converged loadings and grand potentials with respect to the
Lennard-Jones parameters, by implicit adjoint at the fixed point.

The reference has no derivatives: a user differentiates its isotherms by
re-running whole solves.  Here, at a converged density rho* of
E(rho, theta) = ln(Lambda^3 rho) + beta (C1(rho; theta) - mu(theta)) = 0
(the fixed point of Solver.get_new_rho, cmmdft/solver.py:128-144), any
scalar Q(rho*, theta) has

    dQ/dtheta = dQ/dtheta|_rho - lambda^T dE/dtheta,   J^T lambda = dQ/drho,

J = dE/drho = diag(1/rho) + beta A, A = dC1/drho the Hessian of the excess
free energy.  A v is one pass of the functional pipeline with the pointwise
step replaced by its directional derivative (cmm_fmt_hvp).  A is not
symmetric: the MFA kernel spectrum carries the reference's exp(i pi
scalprod) phase (a translated kernel; A^T uses the conjugate spectrum), and
where n3 is clipped the reference's dPhi/dn3 is taken at the clipped value
(cmm_fmt_hvp's transpose mode handles those points).  The adjoint system
is solved in the scaled form (I + beta S A^T S) y = S rhs, S = diag(sqrt(rho)),
lambda = S y, by a batched BiCGSTAB whose vector steps and scalars stay on the
device (cmm_bicg_*).

Outputs per instance and parameter theta = (guest epsilon, guest sigma,
epsilon and sigma of every host atom type):
  * N = integral rho: right-hand side dV 1;
  * Omega (Solver._get_Omega, :103-119): the reference's MFA derivative is
    K rho while its value is 1/2 rho^T K rho, so Omega is not stationary at
    the fixed point (dOmega/drho = dV (K^T - K) rho / 2 there, plus the
    terms of its clipped ideal part); the right-hand side is formed term by
    term;
  * the excess uptake N - rho_bulk He V_cell (Calculator.return_loading,
    cmmdft/calculator.py:114-138) adds the EOS bulk density and the helium
    void fraction.
Explicit derivatives: dV/dtheta analytically on the device
(cmm_extpot_lj_grad).  The guest parameters also enter the hard-sphere part
through R_hs(sigma, epsilon) and the MFA kernel: the hard-sphere C1 and F_HS
are differentiated in R by fourth-order central differences (relative step
``fd_rel`` = 1e-3, truncation ~1e-12; a smaller step would amplify the
rounding noise C1 carries where the packing fraction is tiny) and chained
with dR/dtheta; the MFA kernel is linear in epsilon (exact) and is differenced
in sigma with a relative step of 1e-7 (its cut at r = sigma makes it jump
when a grid point crosses; a step that small almost never meets one, and
the convolution carries no cancellation noise).  mu(P) and rho_bulk(P)
come from root solves of the EOS whose tolerance makes them step-like at
the 1e-9 level, so they are differentiated implicitly: with rho* the root
of p(rho; theta) = P, d rho*/d theta = -p_theta / p_rho and
d mu/d theta = mu_theta + mu_rho d rho*/d theta, the partials taken by
central differences of the closed-form p and mu.  The iterative DFT solve
itself is never differentiated by finite differences.
"""
import numpy as np
import torch

from . import _lib as L
from . import engine as E
from . import workload as W
from .hosts import HELIUM, SyntheticHost
from .units import angstrom, kjmol, boltzmann

check, ptr = L.check, L.ptr

__all__ = ['param_names', 'pack_params', 'unpack_params', 'hvp', 'adjoint_gradients', 'IsothermModel',
           'IsothermFunction']


def param_names(host):
    return (['guest_epsilon', 'guest_sigma'] + ['epsilon_%s' % t for t in host.ffatypes] +
            ['sigma_%s' % t for t in host.ffatypes])


def pack_params(host, guest):
    """theta = (guest eps, guest sigma, eps_t..., sigma_t...) in atomic units."""
    sig, eps, _ = guest
    hs, he = W.host_type_arrays(host)
    return np.concatenate([[eps, sig], he, hs]).astype(np.float64)


def unpack_params(theta, host, guest):
    """Host (same atoms, new type parameters) and guest of a parameter vector."""
    theta = np.asarray(theta, dtype=np.float64)
    nt = len(host.ffatypes)
    ff = {t: (float(theta[2 + nt + i]), float(theta[2 + i])) for i, t in enumerate(host.ffatypes)}
    h = SyntheticHost(host.pos, host.ffatypes, host.ffatype_ids, host.rvecs, ff)
    return h, (float(theta[1]), float(theta[0]), guest[2])


def _stream():
    return E._stream()


def _conj_spectrum(kst):
    k = kst.clone()
    k[1::2] = -k[1::2]
    return k


def _dv_fields(plan, host, gsig, geps, cutoff, vcap):
    """dV/dtheta rows [2 + 2 ntype, npts] of the capped LJ potential."""
    dev = "cuda"
    hs, he = W.host_type_arrays(host)
    pos = torch.as_tensor(np.ascontiguousarray(host.recentred_pos()), device=dev)
    typ = torch.as_tensor(np.ascontiguousarray(host.ffatype_ids, dtype=np.int32), device=dev)
    sig = torch.as_tensor(hs, device=dev)
    eps = torch.as_tensor(he, device=dev)
    out = torch.empty((2 + 2 * len(hs), plan.npts), dtype=torch.float64, device=dev)
    check(L.lib().cmm_extpot_lj_grad(plan.handle, ptr(pos), ptr(typ), int(len(pos)), ptr(sig), ptr(eps),
                                     int(len(hs)), float(gsig), float(geps), float(cutoff), float(vcap),
                                     ptr(out), _stream()), "cmm_extpot_lj_grad")
    return out


def _contract(Wm, D, nchunk=148):
    """[nw, K] = W @ D^T over the points (device partial sums, host sum)."""
    Wm = Wm.contiguous()
    D = D.contiguous()
    nw, n = Wm.shape
    K = D.shape[0]
    part = torch.empty((nw, K, nchunk), dtype=torch.float64, device="cuda")
    check(L.lib().cmm_contract(ptr(Wm), n, nw, ptr(D), n, K, n, ptr(part), nchunk, _stream()), "cmm_contract")
    return part.cpu().numpy().sum(axis=2)


def _pair_dots(A, Bm):
    """sum_r A[b, r] B[b, r] for every b (the diagonal of a contraction)."""
    return np.diag(_contract(A, Bm))


def hvp(fn, wd_rho, v, transpose=False, work=None):
    """A v (or A^T v) for real fields v [B, N1, N2, N3] at the density whose
    weighted densities are wd_rho [nwd, B, N1, N2, N3]."""
    plan = fn.plan
    B = v.shape[0]
    vhat = plan.rfft_yz(v.reshape((B,) + plan.npoints))
    out = plan.new_spec(B)
    if work is None:
        work = torch.empty((fn.nwork, B, plan.nspec * 2), dtype=torch.float64, device="cuda")
    kst = _conj_spectrum(fn.kst) if transpose else fn.kst
    check(L.lib().cmm_fmt_hvp(plan.handle, B, None, fn.R, fn.beta, fn.version, _wda_ptr(fn), int(transpose), ptr(kst),
                              ptr(fn.wtab), ptr(wd_rho), ptr(vhat), ptr(out), ptr(work), _stream()), "cmm_fmt_hvp")
    return plan.irfft_yz(out)


def _wda_ptr(fn):
    import ctypes
    return ctypes.cast(ctypes.pointer(fn.wda), ctypes.c_void_p) if fn.wda is not None else None


class _BiCGStab(object):
    """Batched BiCGSTAB on (I + beta S A^T S) y = S rhs over B instances."""

    def __init__(self, fn, rho, wd_rho, nblk=None):
        self.fn, self.plan = fn, fn.plan
        self.B = rho.shape[0]
        self.npts = self.plan.npts
        self.rho = rho.reshape(self.B, self.npts).contiguous()
        self.wd = wd_rho
        self.kst_t = _conj_spectrum(fn.kst)
        self.work = torch.empty((fn.nwork, self.B, self.plan.nspec * 2), dtype=torch.float64, device="cuda")
        self.nblk = nblk or int(max(1, min(148, (self.npts + 1023) // 1024)))
        self.part = torch.zeros((self.B, 2, self.nblk), dtype=torch.float64, device="cuda")
        self.lib = L.lib()

    def _vec(self, op, out, x=None, y=None, a=None, out2=None, rhat=None, c=0.0):
        check(self.lib.cmm_bicg_vec(op, self.npts, self.B, None, ptr(self.rho), ptr(self.sc), float(c), ptr(x),
                                    ptr(y), ptr(a), ptr(out), ptr(out2), ptr(rhat), ptr(self.part), self.nblk,
                                    _stream()), "cmm_bicg_vec")

    def _scal(self, stage):
        check(self.lib.cmm_bicg_scalars(self.B, None, ptr(self.part), self.nblk, ptr(self.sc), stage, _stream()),
              "cmm_bicg_scalars")

    def _matvec(self, src, dst, a):
        self._vec(0, self.u, x=src)
        vhat = self.plan.rfft_yz(self.u.view((self.B,) + self.plan.npoints))
        out = self.plan.new_spec(self.B)
        fn = self.fn
        check(self.lib.cmm_fmt_hvp(self.plan.handle, self.B, None, fn.R, fn.beta, fn.version, _wda_ptr(fn), 1,
                                   ptr(self.kst_t), ptr(fn.wtab), ptr(self.wd), ptr(vhat), ptr(out), ptr(self.work),
                                   _stream()),
              "cmm_fmt_hvp")
        Au = self.plan.irfft_yz(out).view(self.B, self.npts)
        self._vec(1, dst, x=src, y=Au, a=a, c=fn.beta)

    def solve(self, rhs, tol=1e-11, maxiter=300, check_every=5):
        B, n = self.B, self.npts
        z = lambda: torch.zeros((B, n), dtype=torch.float64, device="cuda")  # noqa: E731
        self.sc = torch.zeros((B, L.BICG_NS), dtype=torch.float64, device="cuda")
        self.sc[:, L.BICG_RHO] = 1.0
        self.sc[:, L.BICG_FIRST] = 1.0
        x, p, v, s, t, self.u = z(), z(), z(), z(), z(), z()
        r = z()
        self._vec(0, r, x=rhs.reshape(B, n).contiguous())
        rhat = r.clone()
        self._vec(4, x, x=p, y=r, a=t, out2=r, rhat=rhat)   # alpha = omega = 0: the dots of r alone
        self._scal(0)
        rr0 = self.sc[:, L.BICG_RR].cpu().numpy().copy()
        rr0[rr0 == 0] = 1.0
        it, rel = 0, np.ones(B)
        for it in range(1, maxiter + 1):
            self._vec(2, p, x=r, y=v)
            self._matvec(p, v, rhat)
            self._scal(1)
            self._vec(3, s, x=r, y=v)
            self._matvec(s, t, s)
            self._scal(2)
            self._vec(4, x, x=p, y=s, a=t, out2=r, rhat=rhat)
            self._scal(0)
            if it % check_every == 0 or it == maxiter:
                rel = np.sqrt(np.abs(self.sc[:, L.BICG_RR].cpu().numpy()) / rr0)
                if np.all(rel < tol):
                    break
        lam = z()
        self._vec(0, lam, x=x)
        self.iterations, self.residual = it, rel
        return lam


def eos_inputs(pressures, temperature, guest, newton=3):
    """(mu, rho_bulk) per pressure with the EOS root polished by Newton steps
    on p(rho) = P.  The reference's bracketing solve (eos.py:121-157, 209-215;
    cmmdft_b200.eos keeps it bit for bit) stops within an absolute tolerance,
    which leaves mu(theta) step-like at ~1e-11 relative; the differentiable
    model needs it smooth."""
    from .eos import ModifiedBenedictWebbRubinEOS
    sig, eps, mass = guest
    P = np.atleast_1d(np.asarray(pressures, dtype=float))
    mb = ModifiedBenedictWebbRubinEOS(mass, sig, eps)
    mb.set_temperature(temperature)
    rho = mb.solve_densities_from_pressures(P)[:, 0]
    for _ in range(newton):
        h = 1e-7 * rho
        slope = (mb.compute_pressure(rho + h) - mb.compute_pressure(rho - h)) / (2 * h)
        rho = rho - (mb.compute_pressure(rho) - P) / slope
    return mb.compute_chempot(rho), rho


def eos_derivatives(pressures, temperature, guest, rel=1e-6):
    """d mu / d theta and d rho_bulk / d theta [B, 2] (theta = guest epsilon,
    guest sigma) at fixed pressures, by implicit differentiation of the MBWR
    root p(rho*) = P (eos.py:209-215)."""
    from .eos import ModifiedBenedictWebbRubinEOS
    sig, eps, mass = guest
    rho = eos_inputs(pressures, temperature, guest)[1]

    def pm(r, s_, e_):
        m = ModifiedBenedictWebbRubinEOS(mass, s_, e_)
        m.set_temperature(temperature)
        return m.compute_pressure(r), m.compute_chempot(r)
    hr = rel * rho
    (pp, mp), (pq, mq) = pm(rho + hr, sig, eps), pm(rho - hr, sig, eps)
    p_r, m_r = (pp - pq) / (2 * hr), (mp - mq) / (2 * hr)
    dmu, drho = np.zeros((len(rho), 2)), np.zeros((len(rho), 2))
    for k, (ds, de) in enumerate(((0.0, rel * eps), (rel * sig, 0.0))):
        h = ds + de
        (pp, mp), (pq, mq) = pm(rho, sig + ds, eps + de), pm(rho, sig - ds, eps - de)
        p_t, m_t = (pp - pq) / (2 * h), (mp - mq) / (2 * h)
        drho[:, k] = -p_t / p_r
        dmu[:, k] = m_t + m_r * drho[:, k]
    return dmu, drho


def _mfa_values(fn, kst, rhohat, B, buf):
    """(MFA part of C1 [B, npts], F_MFA per instance) for kernel spectrum kst."""
    plan = fn.plan
    ch = plan.new_spec(B)
    check(L.lib().cmm_fmt_c1(plan.handle, B, None, fn.R, fn.beta, L.NOHS, None, ptr(kst), ptr(fn.wtab),
                             ptr(rhohat), ptr(ch), ptr(buf.work), ptr(buf.part), buf.nslot, 1, None, _stream()),
          "cmm_fmt_c1")
    return plan.irfft_yz(ch).reshape(B, plan.npts)


def _excess_values(fn, rhohat, B, wda_only=False):
    """(C1 - V fields [B, npts], F_HS + F_MFA (+ F_WDA) per instance) of a
    functional; wda_only: the free energy of the WDA part alone."""
    plan = fn.plan
    buf = E.Buffers(plan, B, nwork=fn.nwork)
    chat = plan.new_spec(B)
    fn.c1(buf, rhohat, chat, want=3)
    E.finalize(buf, (1 << L.NSTAT) - 1)
    st = buf.stats.cpu().numpy()
    Fw = st[:, L.STAT_WDA] * plan.dr if fn.wda is not None else np.zeros(B)
    F = Fw if wda_only else st[:, L.STAT_PHI] * plan.dr / fn.beta + 0.5 * st[:, L.STAT_MFA] * plan.dr + Fw
    return plan.irfft_yz(chat).reshape(B, plan.npts), F


def _wda_values(fn, guest, temperature, mfa_cutoff, rep, rhohat, B, zero_k):
    """(C1 of the WDA part [B, npts], F_WDA per instance) of the functional
    rebuilt for guest (sigma, epsilon, mass): R_hs, the mean-field EOS a from
    the MFA kernel of that guest, the WDA EOS; the MFA convolution is off and
    the hard-sphere part at the same R is subtracted."""
    plan = fn.plan
    sig, eps, mass = guest
    R = W.hardsphere_radius(sig, eps, temperature)
    _, a = E.mfa_kernel_spectrum(plan, sig, eps, mfa_cutoff, rep=rep)
    wda = W.wda_struct(sig, eps, mass, temperature, R, a)
    fw = E.Functional(plan, R, fn.beta, fn.wavelength, fn.V, fn.version, zero_k, a, wda=wda)
    fh = E.Functional(plan, R, fn.beta, fn.wavelength, fn.V, fn.version & ~L.WDA, zero_k)
    cw, Fw = _excess_values(fw, rhohat, B, wda_only=True)
    ch, _ = _excess_values(fh, rhohat, B)
    return cw - ch, Fw


def helium_fraction(plan, host, temperature, cutoff=12 * angstrom):
    """Helium void fraction: integral clip(exp(-V_He / kT), 0, 1) / V_cell."""
    kT = boltzmann * temperature
    hs, he = W.host_type_arrays(host)
    Vhe = E.external_potential(plan, host.recentred_pos(), host.ffatype_ids, hs, he, HELIUM['sigma'] * angstrom,
                               HELIUM['epsilon_K'] * boltzmann, cutoff, float('inf'))
    return float(torch.clamp(torch.exp(-Vhe / kT), 0, 1).sum().item()) * plan.dr / host.volume


def adjoint_gradients(fn, host, guest, temperature, pressures, mus, rho, cutoff=12 * angstrom,
                      mfa_cutoff=12 * angstrom, limit_potential=1e4 * kjmol, tailcorrections=False,
                      fd_rel=1e-3, tol=1e-11, maxiter=300, excess=True):
    """dN/dtheta, dOmega/dtheta (and the excess uptake's) at converged densities.

    rho: converged densities [B, N1, N2, N3] (device) of chemical potentials
    mus at ``pressures`` (atomic units) for functional ``fn`` of (host, guest).
    Returns a dict of N, Omega, dN, dOmega [B, K] (and Nex, dNex), the
    parameter names, and the adjoint solves' iteration counts and residuals.
    """
    if fn.version & L.NOHS:
        raise NotImplementedError("adjoint gradients: MFA-only functionals are not supported")
    if fn.wda is not None and fn.wda.D < 0:
        raise NotImplementedError("adjoint gradients: the LDA part's explicit parameter derivatives are not built")
    plan = fn.plan
    B = rho.shape[0]
    n = plan.npts
    dV = plan.dr
    beta = fn.beta
    rho = rho.reshape((B,) + plan.npoints).contiguous()
    rho2 = rho.view(B, n)
    rhohat = plan.rfft_yz(rho)
    # weighted densities of rho: where the Hessian is evaluated
    buf = E.Buffers(plan, B, nwork=fn.nwork)
    wd = torch.empty((fn.nwd, B) + plan.npoints, dtype=torch.float64, device="cuda")
    fn.c1(buf, rhohat, None, want=8, wd=wd)
    # dOmega/drho of Solver._get_Omega at rho, term by term (not through the
    # fixed-point relation, which the smallest densities satisfy least):
    # dV [ideal' - mu + V + C1 + (K^T - K) rho / 2], ideal' = ln(Lambda^3 rho)/beta
    # where rho >= 1e-12 and 0 where _get_Omega clips it; C1 (the pipeline's,
    # with K rho) plus (K^T - K) rho / 2 is the gradient of F_HS + rho^T K rho / 2
    mfa = [_mfa_values(fn, k, rhohat, B, buf) for k in (fn.kst, _conj_spectrum(fn.kst))]
    chat = plan.new_spec(B)
    fn.c1(buf, rhohat, chat, want=1)
    C1 = plan.irfft_yz(chat).reshape(B, n)
    mu_t = torch.as_tensor(np.asarray(mus, dtype=np.float64), device="cuda").view(B, 1)
    keep = rho2 >= 1e-12
    ideal_d = torch.where(keep, torch.log(fn.lambda3 * torch.where(keep, rho2, torch.ones_like(rho2))) / beta,
                          torch.zeros_like(rho2))
    rhs_om = dV * (ideal_d - mu_t + fn.V.reshape(1, n) + C1 + 0.5 * (mfa[1] - mfa[0]))
    solver = _BiCGStab(fn, rho, wd)
    lam_n = solver.solve(torch.full((B, n), dV, dtype=torch.float64, device="cuda"), tol=tol, maxiter=maxiter)
    it_n, res_n = solver.iterations, solver.residual
    lam_o = solver.solve(rhs_om, tol=tol, maxiter=maxiter)
    it_o, res_o = solver.iterations, solver.residual
    # explicit dV/dtheta contracted with lambda_N, lambda_Omega and rho
    gsig, geps, _ = guest
    D = torch.cat([_dv_fields(plan, host, gsig, geps, cutoff, limit_potential),
                   torch.ones((1, n), dtype=torch.float64, device="cuda")])
    K = D.shape[0] - 1
    S = _contract(torch.cat([lam_n, lam_o, rho2]), D)
    G_n, sum_n = S[:B, :K], S[:B, K]
    G_o, sum_o = S[B:2 * B, :K], S[B:2 * B, K]
    H, N = S[2 * B:, :K], S[2 * B:, K] * dV
    # explicit guest partials of the excess functional and of the EOS
    Gx_n, Gx_o, dF, dmu, dbulk = (np.zeros((B, K)) for _ in range(5))
    _, F0 = _excess_values(fn, rhohat, B)
    # f' = [8 (f(h) - f(-h)) - (f(2h) - f(-2h))] / (12 h)
    stencil = ((1.0, 8.0), (-1.0, -8.0), (2.0, -1.0), (-2.0, 1.0))
    gsig, geps, _ = guest
    # hard-sphere part: d/dR at fixed (zero) MFA kernel, chained with dR/dtheta
    zero_k = torch.zeros_like(fn.kst)
    hR = fd_rel * fn.R
    dC_R = torch.zeros((B, n), dtype=torch.float64, device="cuda")
    dF_R = np.zeros(B)
    for step, wgt in stencil:
        fr = E.Functional(plan, fn.R + step * hR, fn.beta, fn.wavelength, fn.V, fn.version & ~L.WDA, zero_k)
        c1x, F = _excess_values(fr, rhohat, B)
        dC_R += (wgt / (12 * hR)) * c1x
        dF_R += (wgt / (12 * hR)) * F
    dR = np.zeros(2)
    for k, idx in ((0, 1), (1, 0)):   # theta_0: guest epsilon (guest[1]); theta_1: guest sigma (guest[0])
        h = 1e-4 * guest[idx]
        for step, wgt in stencil:
            g = list(guest)
            g[idx] = guest[idx] + step * h
            dR[k] += wgt / (12 * h) * W.hardsphere_radius(g[0], g[1], temperature)
    # MFA part: linear in epsilon; sigma by a small central difference
    rep = 2 if tailcorrections else 1
    c_mfa = _mfa_values(fn, fn.kst, rhohat, B, buf)
    hs_ = 1e-7 * gsig
    kp, _ = E.mfa_kernel_spectrum(plan, gsig + hs_, geps, mfa_cutoff, rep=rep)
    km, _ = E.mfa_kernel_spectrum(plan, gsig - hs_, geps, mfa_cutoff, rep=rep)
    dC_ms = (_mfa_values(fn, kp, rhohat, B, buf) - _mfa_values(fn, km, rhohat, B, buf)) / (2 * hs_)
    half_rho = 0.5 * dV * rho2
    D_eps = dR[0] * dC_R + c_mfa / geps
    D_sig = dR[1] * dC_R + dC_ms
    dF_wda = np.zeros((B, 2))
    if fn.wda is not None:
        # the WDA part moves with the guest through R_hs (weight diameter,
        # Carnahan-Starling eta), the MBWR coefficients and the mean-field
        # EOS a; it is smooth, so its explicit partials are central
        # differences (fourth order, relative step 1e-5) of the functional
        # rebuilt at the shifted parameters, less its hard-sphere part
        for k, idx in ((0, 1), (1, 0)):
            h = 1e-5 * guest[idx]
            dCw = torch.zeros((B, n), dtype=torch.float64, device="cuda")
            for step, wgt in stencil:
                g = list(guest)
                g[idx] = guest[idx] + step * h
                cw, Fw = _wda_values(fn, g, temperature, mfa_cutoff, rep, rhohat, B, zero_k)
                dCw += (wgt / (12 * h)) * cw
                dF_wda[:, k] += (wgt / (12 * h)) * Fw
            if k == 0:
                D_eps = D_eps + dCw
            else:
                D_sig = D_sig + dCw
    for k, Dk in ((0, D_eps), (1, D_sig)):
        Gx_n[:, k] = _pair_dots(lam_n, Dk)
        Gx_o[:, k] = _pair_dots(lam_o, Dk)
    dF[:, 0] = dR[0] * dF_R + _pair_dots(half_rho, c_mfa) / geps + dF_wda[:, 0]
    dF[:, 1] = dR[1] * dF_R + _pair_dots(half_rho, dC_ms) + dF_wda[:, 1]
    # EOS
    dmu[:, :2], dbulk[:, :2] = eos_derivatives(pressures, temperature, guest)
    dN = -beta * (G_n + Gx_n) + beta * dmu * sum_n[:, None]
    dOm = dV * H + dF - N[:, None] * dmu - beta * (G_o + Gx_o) + beta * dmu * sum_o[:, None]
    # Omega at rho as Solver._get_Omega forms it
    rr = torch.where(rho2 < 1e-12, torch.full_like(rho2, 1e-30), rho2)
    ideal = (rr * (torch.log(fn.lambda3 * rr) - 1)).sum(dim=1).cpu().numpy() * dV / beta
    ext = _contract(rho2, fn.V.reshape(1, n))[:, 0] * dV
    Om = ideal + F0 + ext - np.asarray(mus) * N
    out = dict(names=param_names(host), N=N, Omega=Om, dN=dN, dOmega=dOm,
               dOmega_explicit=dV * H + dF - N[:, None] * dmu,
               iterations=(it_n, it_o), residual=(res_n, res_o))
    if excess:
        kT = 1.0 / beta
        he_sig, he_eps = HELIUM['sigma'] * angstrom, HELIUM['epsilon_K'] * boltzmann
        hs, he = W.host_type_arrays(host)
        Vhe = E.external_potential(plan, host.recentred_pos(), host.ffatype_ids, hs, he, he_sig, he_eps, cutoff,
                                   float('inf')).reshape(1, n)
        ehe = torch.exp(-Vhe / kT)
        vol = host.volume
        he_frac = float(torch.clamp(ehe, 0, 1).sum().item()) * dV / vol
        w = torch.where((Vhe > 0) & torch.isfinite(Vhe), -ehe / kT, torch.zeros_like(Vhe))
        dhe = _contract(w, _dv_fields(plan, host, he_sig, he_eps, cutoff, float('inf')))[0] * dV / vol
        dhe[:2] = 0.0   # the helium probe's own parameters are not in theta
        bulks = eos_inputs(pressures, temperature, guest)[1]
        out['Nex'] = N - bulks * he_frac * vol
        out['dNex'] = dN - vol * (dbulk * he_frac + bulks[:, None] * dhe[None, :])
        out['he_frac'] = he_frac
    return out


class IsothermModel(object):
    """An isotherm of one host and guest as a differentiable function of the
    LJ parameters theta (``param_names``).

    ``model(theta)`` (a float64 tensor with requires_grad) returns the excess
    (``quantity='excess'``) or absolute (``'absolute'``) uptakes, or the grand
    potentials (``'omega'``), per pressure; backward runs the adjoint.
    """

    def __init__(self, host, guest, temperature, npoints, pressures, quantity='excess', threshold=1e-12,
                 criterion='res', nsteps=1000, method='hybridanderson', version='WBII', tailcorrections=False,
                 cutoff=12 * angstrom, mfa_cutoff=12 * angstrom, limit_potential=1e4 * kjmol, fd_rel=1e-3,
                 tol=1e-11, wda=False):
        assert quantity in ('excess', 'absolute', 'omega')
        self.host, self.guest = host, guest
        self.T = float(temperature)
        self.npoints = tuple(npoints)
        self.pressures = np.asarray(pressures, dtype=np.float64)
        self.quantity = quantity
        self.solve_kw = dict(threshold=threshold, criterion=criterion, nsteps=nsteps, method=method)
        self.version, self.tail, self.wda = version, tailcorrections, bool(wda)
        self.cutoff, self.mfa_cutoff, self.vcap = cutoff, mfa_cutoff, limit_potential
        self.fd_rel, self.tol = fd_rel, tol
        self.theta0 = pack_params(host, guest)
        self.plan = E.GridPlan(self.npoints, host.rvecs)
        self.last = None

    def solve(self, theta):
        """Converged isotherm at parameters theta (no derivatives): chemical
        potentials from the polished EOS root (``eos_inputs``), Ninit = rho_bulk
        start, the native batched solver."""
        from .batch import GroupedSolve
        host, guest = unpack_params(theta, self.host, self.guest)
        fn = W.build_functional(host, self.npoints, self.T, guest, version=self.version,
                                tailcorrections=self.tail, cutoff=self.cutoff, mfa_cutoff=self.mfa_cutoff,
                                limit_potential=self.vcap, plan=self.plan, wda=self.wda)
        mus, bulks = eos_inputs(self.pressures, self.T, guest)
        rho0 = W.initial_density(fn, mus, ninit=bulks)
        s = GroupedSolve(fn, mus, groups=1, divergence_guard=True, **self.solve_kw)
        N, rho, conv = s.solve(rho0)
        return dict(mu=mus, rho_bulk=bulks, N=np.array(N), converged=np.array(conv), solver=s, host=host,
                    guest=guest, fn=fn, rho=rho)

    def quantity_values(self, sol):
        """The model's quantity at a solution, without derivatives."""
        if self.quantity == 'absolute':
            return np.asarray(sol['N'], dtype=np.float64)
        if self.quantity == 'omega':
            return np.asarray(sol['solver'].omega0)
        he = helium_fraction(self.plan, sol['host'], self.T, self.cutoff)
        return np.asarray(sol['N']) - np.asarray(sol['rho_bulk']) * he * sol['host'].volume

    def values(self, sol):
        """(values [B], Jacobian [B, K], all outputs) of the model's quantity."""
        g = adjoint_gradients(sol['fn'], sol['host'], sol['guest'], self.T, self.pressures, sol['mu'], sol['rho'],
                              cutoff=self.cutoff, mfa_cutoff=self.mfa_cutoff, limit_potential=self.vcap,
                              tailcorrections=self.tail, fd_rel=self.fd_rel, tol=self.tol,
                              excess=self.quantity == 'excess')
        key = {'excess': 'Nex', 'absolute': 'N', 'omega': 'Omega'}[self.quantity]
        return g[key], g['d' + key], g

    def __call__(self, theta):
        return IsothermFunction.apply(theta, self)


class IsothermFunction(torch.autograd.Function):
    """theta [K] -> uptakes (or Omega) [B]; the backward pass is the adjoint."""

    @staticmethod
    def forward(ctx, theta, model):
        sol = model.solve(theta.detach().cpu().numpy())
        if not np.all(sol['converged']):
            raise RuntimeError("isotherm points did not converge: %s" % np.where(~sol['converged'])[0])
        ctx.model, ctx.sol = model, sol
        model.last = sol
        vals = model.quantity_values(sol)
        return torch.as_tensor(np.asarray(vals, dtype=np.float64), dtype=theta.dtype, device=theta.device)

    @staticmethod
    def backward(ctx, grad):
        _, jac, _ = ctx.model.values(ctx.sol)
        J = torch.as_tensor(jac, dtype=grad.dtype, device=grad.device)
        return grad @ J, None
