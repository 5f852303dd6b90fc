"""Device-side objects: grid plans, the functional pipeline and its buffers.

Everything here drives the CUDA library through its C ABI (``_lib``) with
torch tensors as device memory and the current torch stream.  There is no CPU
path: every method requires a CUDA device.
"""
import ctypes

import numpy as np
import torch

from . import _lib as L
from ._lib import check, ptr


def _stream():
    """The calling thread's current CUDA stream (torch's) as a void*."""
    return ctypes.c_void_p(torch._C._cuda_getCurrentRawStream(torch._C._cuda_getDevice()))


def require_cuda():
    if not torch.cuda.is_available():
        raise L.CmmError("cmmdft_b200 needs a CUDA device (sm_100a); there is no CPU fallback")


class GridPlan(object):
    """A grid plan for an N1 x N2 x N3 grid of the cell ``rvecs`` (rows, bohr).

    Wraps ``cmm_grid_create``; owns the plan's device tables.
    """

    def __init__(self, npoints, rvecs, schedule=None):
        """schedule: None (the default FFT schedule) or the five entries of
        cmm_grid_create_sched (x, y, z radix order, plane-pass form, column
        tile), e.g. as chosen by cmmdft_b200.autotune."""
        require_cuda()
        self.lib = L.lib()
        n1, n2, n3 = [int(n) for n in npoints]
        self.npoints = (n1, n2, n3)
        self.rvecs = np.ascontiguousarray(rvecs, dtype=np.float64).reshape(3, 3)
        h = ctypes.c_void_p()
        rv = (ctypes.c_double * 9)(*self.rvecs.ravel().tolist())
        if schedule is None:
            check(self.lib.cmm_grid_create(n1, n2, n3, rv, ctypes.byref(h)), "cmm_grid_create")
        else:
            sc = (ctypes.c_int * 5)(*[int(x) for x in schedule])
            check(self.lib.cmm_grid_create_sched(n1, n2, n3, rv, sc, ctypes.byref(h)), "cmm_grid_create_sched")
        self.handle = h
        ns = ctypes.c_longlong()
        h3 = ctypes.c_int()
        check(self.lib.cmm_grid_spectrum_size(h, ctypes.byref(ns), ctypes.byref(h3)))
        self.nspec = int(ns.value)
        self.h3 = int(h3.value)
        self.npts = n1 * n2 * n3
        k1 = (ctypes.c_int * n1)()
        k2 = (ctypes.c_int * n2)()
        k3 = (ctypes.c_int * self.h3)()
        check(self.lib.cmm_spectrum_index(h, k1, k2, k3))
        self.k1 = np.array(k1[:], dtype=np.int64)
        self.k2 = np.array(k2[:], dtype=np.int64)
        self.k3 = np.array(k3[:], dtype=np.int64)
        self.volume = float(abs(np.linalg.det(self.rvecs)))
        self.dr = self.volume / self.npts

    def schedule(self):
        """(sched[5], radices per axis) of the plan (cmm_grid_schedule)."""
        sc = (ctypes.c_int * 5)()
        rd = (ctypes.c_int * 48)()
        check(self.lib.cmm_grid_schedule(self.handle, sc, rd), "cmm_grid_schedule")
        r = np.array(rd[:]).reshape(3, 16)
        return list(sc[:]), [[int(x) for x in row if x] for row in r]

    def set_staging(self, mode):
        """0: fused plane passes where the plane fits in shared memory, the
        functional's plane split over a CTA pair (default); 1: always the
        staged y pass + z-row form; 2: fused, the functional's plane in one
        CTA (cmm_grid_set_staging)."""
        check(self.lib.cmm_grid_set_staging(self.handle, int(mode)), "cmm_grid_set_staging")

    def __del__(self):
        try:
            if getattr(self, "handle", None) is not None:
                self.lib.cmm_grid_destroy(self.handle)
                self.handle = None
        except Exception:
            pass

    # ---- spectra -------------------------------------------------------
    def new_spec(self, batch=1):
        return torch.empty((batch, self.nspec * 2), dtype=torch.float64, device="cuda")

    def rfft(self, x):
        """Half spectrum (plan layout, unnormalised) of real fields [B, N1, N2, N3]."""
        x = x.contiguous()
        B = x.shape[0]
        out = self.new_spec(B)
        check(self.lib.cmm_rfft3d(self.handle, B, ptr(x), ptr(out), _stream()), "cmm_rfft3d")
        return out

    def irfft(self, spec):
        """Inverse of :meth:`rfft` times N (unnormalised), as real fields."""
        s = spec.clone()
        B = s.shape[0]
        out = torch.empty((B,) + self.npoints, dtype=torch.float64, device="cuda")
        check(self.lib.cmm_irfft3d(self.handle, B, ptr(s), ptr(out), _stream()), "cmm_irfft3d")
        return out

    def rfft_yz(self, x):
        """yz-spectrum (x real, y/z half spectrum) of real fields [B, N1, N2, N3]."""
        x = x.contiguous()
        out = self.new_spec(x.shape[0])
        check(self.lib.cmm_rfft_yz(self.handle, x.shape[0], ptr(x), ptr(out), _stream()), "cmm_rfft_yz")
        return out

    def irfft_yz(self, spec):
        """Real fields from yz-spectra (unnormalised inverse of :meth:`rfft_yz`)."""
        B = spec.shape[0]
        out = torch.empty((B,) + self.npoints, dtype=torch.float64, device="cuda")
        check(self.lib.cmm_irfft_yz(self.handle, B, ptr(spec), ptr(out), _stream()), "cmm_irfft_yz")
        return out

    def spec_to_full(self, spec):
        """Full numpy spectrum [B, N1, N2, N3] (scipy fftn order) from a plan-layout spectrum."""
        n1, n2, n3 = self.npoints
        s = spec.detach().cpu().numpy().view(np.complex128).reshape(-1, n1, n2, self.h3)
        B = s.shape[0]
        full = np.zeros((B, n1, n2, n3), dtype=np.complex128)
        k2 = self.k2[None, :, None]
        k3 = self.k3[None, None, :]
        k1 = self.k1[:, None, None]
        for b in range(B):
            full[b][k1, k2, k3] = s[b]
            # Hermitian completion
            kk1 = (-k1) % n1
            kk2 = (-k2) % n2
            kk3 = (-k3) % n3
            full[b][kk1, kk2, kk3] = np.conj(s[b])
            full[b][k1, k2, k3] = s[b]
        return full


class Buffers(object):
    """Workspace of one shape group of ``batch`` instances."""

    def __init__(self, plan, batch, nhist=0, nwork=12):
        self.plan = plan
        self.batch = batch
        n1, n2, n3 = plan.npoints
        dev = "cuda"
        f64 = torch.float64
        fs = plan.nspec * 2
        # intermediate spectra of the functional pipeline (Functional.nwork)
        self.work = torch.empty((nwork, batch, fs), dtype=f64, device=dev)
        self.nslot = int(L.lib().cmm_part_slots(plan.handle))  # planes or column tiles written per pass
        self.part = torch.zeros((batch, L.NSTAT, self.nslot), dtype=f64, device=dev)
        self.stats = torch.zeros((batch, L.NSTAT), dtype=f64, device=dev)
        self.active = torch.ones(batch, dtype=torch.int32, device=dev)


class Functional(object):
    """Device data of the WBII/FMT + MFA + external-potential functional of one
    host, guest, grid and temperature.

    Mirrors the part list FreeEnergy builds with add_hard_sphere,
    add_mean_field and add_external_potential (cmmdft/functionals.py:176-337).
    """

    def __init__(self, plan, R, beta, wavelength, V, version=L.WBII, kst=None, vdw_a=None, wda=None):
        self.plan = plan
        self.R = float(R)
        self.beta = float(beta)
        self.wavelength = float(wavelength)
        self.lambda3 = float(wavelength) ** 3
        self.V = V.contiguous()                       # [N1, N2, N3] device
        self.version = int(version)
        self.kst = kst                                # MFA kernel spectrum (or zeros)
        if self.kst is None:
            self.kst = torch.zeros(plan.nspec * 2, dtype=torch.float64, device="cuda")
        self.vdw_a = vdw_a
        # optional WDA correlation part (an _lib.WdaEos); sets the CMM_WDA bit
        self.wda = wda
        if wda is not None:
            self.version |= L.WDA
        # (kw0, kw3) table for this grid and radius, L2-resident during the solve
        # intermediate spectra of one pipeline launch per instance
        self.nwork = 24 if (self.version & L.TENSOR) else 12
        self.wtab = None
        if not (self.version & L.NOHS):
            self.wtab = torch.empty(plan.nspec * 2, dtype=torch.float64, device="cuda")
            check(L.lib().cmm_fmt_weights(plan.handle, self.R, ptr(self.wtab), _stream()), "cmm_fmt_weights")

    @property
    def nwd(self):
        """Number of weighted-density fields (n0, n3, nv2 x/y/z, WDA, tensor)."""
        return 5 + (1 if self.version & L.WDA else 0) + (6 if self.version & L.TENSOR else 0)

    def c1(self, buf, rhohat, chat, want=1, active=None, batch=None, wd=None):
        """yz-spectrum of C1 - V (HardSphere.derive + MFA.derive) for every instance;
        want bit 3 also stores the weighted densities into ``wd`` [nwd, B, N1, N2, N3]."""
        B = buf.batch if batch is None else batch
        wda = ctypes.byref(self.wda) if self.wda is not None else None
        check(L.lib().cmm_fmt_c1(self.plan.handle, B, ptr(active), self.R, self.beta, self.version, wda,
                                 ptr(self.kst), ptr(self.wtab), ptr(rhohat), ptr(chat), ptr(buf.work),
                                 ptr(buf.part), buf.nslot, int(want), ptr(wd), _stream()), "cmm_fmt_c1")

    # ---- hybrid line search (Picard.update_rho_hybrid without trial transforms)
    def ls_prepare(self, buf, r, rhohat, wd_rho, rhat, wd_r, ls_part, active=None):
        wda = ctypes.byref(self.wda) if self.wda is not None else None
        check(L.lib().cmm_ls_prepare(self.plan.handle, buf.batch, ptr(active), self.R, self.version, wda,
                                     ptr(self.kst), ptr(self.wtab), ptr(r), ptr(rhohat), ptr(wd_rho), ptr(rhat),
                                     ptr(buf.work), ptr(wd_r), ptr(ls_part), buf.nslot, _stream()),
              "cmm_ls_prepare")

    def ls_omega(self, buf, n3a, coefs, rho, r, wd_rho, wd_r, ls_part, alpha, active=None, vstride=0):
        """n3a: per-instance max n3 of rho, a (strided) device vector, e.g. params[:, 3]
        or the N3MAX column of the finalized stats."""
        wda = ctypes.byref(self.wda) if self.wda is not None else None
        c0, c1, c2 = [float(c) for c in coefs]
        check(L.lib().cmm_ls_omega(self.plan.handle, buf.batch, ptr(active), ptr(n3a), int(n3a.stride(0)), c0, c1,
                                   c2, self.R, self.lambda3, self.version, wda, ptr(rho), ptr(r), ptr(self.V),
                                   int(vstride), ptr(wd_rho), ptr(wd_r), ptr(ls_part), buf.nslot, ptr(alpha),
                                   _stream()), "cmm_ls_omega")

    def ls_finalize(self, buf, ls_part, ls, active=None):
        check(L.lib().cmm_ls_finalize(buf.batch, ptr(active), ptr(ls_part), buf.nslot, ptr(ls), _stream()),
              "cmm_ls_finalize")


def mfa_kernel_spectrum(plan, sigma, epsilon, cutoff, rmin=None, limit=0.0, rep=1):
    """MFA kernel spectrum for MFAFunctional.generate_potential_lj and its vdW ``a``."""
    lib = L.lib()
    if rmin is None:
        rmin = sigma
    cut = -1.0 if cutoff is None else float(cutoff)
    need = ctypes.c_size_t(0)
    check(lib.cmm_mfa_kernel(plan.handle, sigma, epsilon, cut, rmin, limit, rep, None, None,
                             ctypes.byref(need), None, _stream()), "cmm_mfa_kernel(size)")
    work = torch.empty(int(need.value) // 8 + 1, dtype=torch.float64, device="cuda")
    kst = torch.empty(plan.nspec * 2, dtype=torch.float64, device="cuda")
    a = ctypes.c_double(0.0)
    check(lib.cmm_mfa_kernel(plan.handle, sigma, epsilon, cut, rmin, limit, rep, ptr(kst), ptr(work),
                             ctypes.byref(need), ctypes.byref(a), _stream()), "cmm_mfa_kernel")
    return kst, float(a.value)


def external_potential(plan, pos, type_ids, type_sigma, type_epsilon, guest_sigma, guest_epsilon,
                       cutoff, v_cap):
    """LJ external potential of a host on the plan's grid (device tensor [N1,N2,N3])."""
    dev = "cuda"
    pos_t = torch.as_tensor(np.ascontiguousarray(pos, dtype=np.float64), device=dev)
    typ_t = torch.as_tensor(np.ascontiguousarray(type_ids, dtype=np.int32), device=dev)
    sig_t = torch.as_tensor(np.ascontiguousarray(type_sigma, dtype=np.float64), device=dev)
    eps_t = torch.as_tensor(np.ascontiguousarray(type_epsilon, dtype=np.float64), device=dev)
    V = torch.empty(plan.npoints, dtype=torch.float64, device=dev)
    check(L.lib().cmm_extpot_lj(plan.handle, ptr(pos_t), ptr(typ_t), int(len(pos_t)), ptr(sig_t), ptr(eps_t),
                                int(len(sig_t)), float(guest_sigma), float(guest_epsilon), float(cutoff),
                                float(v_cap), ptr(V), _stream()), "cmm_extpot_lj")
    return V


def effective_potential(plan, pos, type_ids, type_sigma, type_epsilon, guest_pos, guest_masses, site_sigma,
                        site_epsilon, rotations, weights, cutoff, beta, v_limit):
    """Orientation-averaged LJ potential of a rigid multi-site guest on the
    plan's grid (device tensor [N1,N2,N3], uncapped; cmm_extpot_rot)."""
    dev = "cuda"
    f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
    pos_t, sig_t, eps_t = f64(pos), f64(type_sigma), f64(type_epsilon)
    typ_t = torch.as_tensor(np.ascontiguousarray(type_ids, dtype=np.int32), device=dev)
    rot_t, w_t = f64(np.asarray(rotations).reshape(-1, 9)), f64(weights)
    gp = np.ascontiguousarray(guest_pos, dtype=np.float64).reshape(-1)
    gm, gs, ge = (np.ascontiguousarray(a, dtype=np.float64) for a in (guest_masses, site_sigma, site_epsilon))
    ns = len(gm)
    if not (len(gp) == 3 * ns and len(gs) == ns and len(ge) == ns and len(w_t) == len(rot_t)):
        raise ValueError("guest arrays or rotations/weights have inconsistent lengths")
    cd = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    V = torch.empty(plan.npoints, dtype=torch.float64, device=dev)
    check(L.lib().cmm_extpot_rot(plan.handle, ptr(pos_t), ptr(typ_t), int(len(pos_t)), ptr(sig_t), ptr(eps_t),
                                 int(len(sig_t)), cd(gp), cd(gm), cd(gs), cd(ge), ns, ptr(rot_t), ptr(w_t),
                                 int(len(w_t)), float(cutoff), float(beta), float(v_limit), ptr(V), _stream()),
          "cmm_extpot_rot")
    return V


def external_potential_derivatives(rvecs, npoints, spacings, pos, type_ids, type_sigma, type_epsilon, guest_sigma,
                                   guest_epsilon, cutoff, v_max, out=None):
    """The eight LJ channels (V and its derivatives in unit-cube scaling) of
    one guest atom type on an npoints grid over the cell: device tensor
    [8, n1, n2, n3] (cmm_extpot_lj_deriv)."""
    dev = "cuda"
    f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
    pos_t, sig_t, eps_t = f64(pos), f64(type_sigma), f64(type_epsilon)
    typ_t = torch.as_tensor(np.ascontiguousarray(type_ids, dtype=np.int32), device=dev)
    n1, n2, n3 = (int(n) for n in npoints)
    if out is None:
        out = torch.empty((8, n1, n2, n3), dtype=torch.float64, device=dev)
    rv = (ctypes.c_double * 9)(*np.asarray(rvecs, dtype=np.float64).ravel().tolist())
    sp = (ctypes.c_double * 3)(*[float(s) for s in spacings])
    check(L.lib().cmm_extpot_lj_deriv(rv, n1, n2, n3, sp, ptr(pos_t), ptr(typ_t), int(len(pos_t)), ptr(sig_t),
                                      ptr(eps_t), int(len(sig_t)), float(guest_sigma), float(guest_epsilon),
                                      float(cutoff), float(v_max), ptr(out), _stream()), "cmm_extpot_lj_deriv")
    return out


def effective_potential_interpolated(plan, tables, site_tab, origin, spacing, guest_pos, guest_masses, rotations,
                                     weights, beta, v_limit):
    """Orientation-averaged potential with tricubically interpolated site
    potentials (cmm_extpot_rot_interp).  ``tables``: device tensor
    [ntab, 8, f1, f2, f3] of channel grids; ``site_tab[s]``: the table of
    site s; ``origin``/``spacing``: the interpolator's."""
    dev = "cuda"
    f64 = lambda a: torch.as_tensor(np.ascontiguousarray(a, dtype=np.float64), device=dev)
    tables = tables.contiguous()
    if tables.dim() != 5 or tables.shape[1] != 8:
        raise ValueError("tables must be [ntab, 8, f1, f2, f3]")
    rot_t, w_t = f64(np.asarray(rotations).reshape(-1, 9)), f64(weights)
    gp = np.ascontiguousarray(guest_pos, dtype=np.float64).reshape(-1)
    gm = np.ascontiguousarray(guest_masses, dtype=np.float64)
    st = np.ascontiguousarray(site_tab, dtype=np.int32)
    ns = len(gm)
    if not (len(gp) == 3 * ns and len(st) == ns and len(w_t) == len(rot_t)):
        raise ValueError("guest arrays or rotations/weights have inconsistent lengths")
    cd = lambda a: np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(ctypes.POINTER(ctypes.c_double))
    fn = (ctypes.c_int * 3)(*[int(n) for n in tables.shape[2:]])
    org, spc = np.asarray(origin, dtype=np.float64), np.asarray(spacing, dtype=np.float64)
    V = torch.empty(plan.npoints, dtype=torch.float64, device=dev)
    check(L.lib().cmm_extpot_rot_interp(plan.handle, ptr(tables), int(tables.shape[0]), fn, cd(org), cd(spc),
                                        cd(gp), cd(gm), st.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), ns,
                                        ptr(rot_t), ptr(w_t), int(len(w_t)), float(beta), float(v_limit), ptr(V),
                                        _stream()), "cmm_extpot_rot_interp")
    return V


def finalize(buf, mask, active=None):
    check(L.lib().cmm_stats_finalize(buf.batch, ptr(active), ptr(buf.part), buf.nslot, ctypes.c_uint(mask),
                                     ptr(buf.stats), _stream()), "cmm_stats_finalize")


def picard_static_step(fn, buf, params, thr, chat, rho, rho_out, rhohat_out, active=None, vstride=0,
                       tol=(1e-6, 1e-4)):
    """tol = (a_tol, r_tol) of the DER criterion (Solver, cmmdft/solver.py:25-26)."""
    check(L.lib().cmm_picard_static_step(fn.plan.handle, buf.batch, ptr(active), ptr(params), fn.beta,
                                         fn.lambda3, float(thr), float(tol[0]), float(tol[1]), ptr(chat), ptr(rho), ptr(fn.V), int(vstride),
                                         ptr(rho_out), ptr(rhohat_out), ptr(buf.part), buf.nslot, _stream()),
          "cmm_picard_static_step")


def residual_step(fn, buf, params, chat, rho, r_out, hist=(), hstride=0, active=None, vstride=0,
                  tol=(1e-6, 1e-4)):
    n = len(hist)
    arr = (ctypes.c_void_p * max(n, 1))(*[h.data_ptr() for h in hist]) if n else None
    check(L.lib().cmm_residual_step(fn.plan.handle, buf.batch, ptr(active), ptr(params), fn.beta, fn.lambda3,
                                    float(tol[0]), float(tol[1]), ptr(chat),
                                    ptr(rho), ptr(fn.V), int(vstride), ptr(r_out), arr, n, int(hstride),
                                    ptr(buf.part), buf.nslot, _stream()), "cmm_residual_step")


def mix_step(fn, buf, coef, fields, strides, clip, ref, rho_out, rhohat_out, thr=0.0, active=None,
             refstride=None, vstride=0):
    n = len(fields)
    arr = (ctypes.c_void_p * n)(*[f.data_ptr() for f in fields])
    st = (ctypes.c_longlong * n)(*[int(s) for s in strides])
    if refstride is None:
        refstride = fn.plan.npts
    check(L.lib().cmm_mix_step(fn.plan.handle, buf.batch, ptr(active), ptr(coef), arr, st, n, int(clip),
                               float(thr), fn.lambda3, ptr(ref), int(refstride), ptr(fn.V), int(vstride),
                               ptr(rho_out), ptr(rhohat_out), ptr(buf.part), buf.nslot, _stream()),
          "cmm_mix_step")
