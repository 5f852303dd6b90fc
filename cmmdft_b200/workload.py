"""Assemble the device functional of a host/guest/grid/temperature.

``build_functional`` performs, on the GPU, what FreeEnergy.add_hard_sphere,
add_mean_field and add_external_potential set up in the reference
(cmmdft/functionals.py:176-337): the capped LJ external potential, the MFA
kernel spectrum and the hard-sphere radius.  ``isotherm_inputs`` gives the
chemical potentials and bulk densities of a pressure list from the MBWR
equation of state, as the reference's example notebook does.
"""
import numpy as np

from . import _lib as L
from . import engine as E
from .eos import ModifiedBenedictWebbRubinEOS
from .units import angstrom, kjmol, boltzmann, planck

# version strings of cmmdft/functionals.py:375-377: base with 'a' and/or 't'
HS_VERSIONS = {}
for _base, _code in (('FMT', L.FMT), ('MFMT', L.MFMT), ('WBII', L.WBII)):
    for _pre, _bits in (('', 0), ('a', L.ANTISYM), ('t', L.TENSOR), ('at', L.ANTISYM | L.TENSOR),
                        ('ta', L.ANTISYM | L.TENSOR)):
        HS_VERSIONS[_pre + _base] = _code | _bits


def hardsphere_radius(sigma, epsilon, temperature):
    """Barker-Henderson fit of SphericalLJGuest (cmmdft/system.py:154-158)."""
    beta = 1 / (boltzmann * temperature)
    Tt = 1 / beta / epsilon
    return sigma * (1 + 0.2977 * Tt) / (1 + 0.33163 * Tt + 0.0010477 * Tt ** 2) / 2


def thermal_wavelength(mass, temperature):
    """Guest.wavelength (cmmdft/system.py:115-117)."""
    kT = boltzmann * temperature
    return planck / np.sqrt(2 * np.pi * mass * kT)


def hs_version_code(version):
    if version not in HS_VERSIONS:
        raise ValueError("Unknown hard sphere functional version: %r" % version)
    return HS_VERSIONS[version]


def host_type_arrays(host, guest_types=None):
    sig = np.array([host.ff[t][0] for t in host.ffatypes])
    eps = np.array([host.ff[t][1] for t in host.ffatypes])
    return sig, eps


def wda_struct(sigma, epsilon, mass, temperature, R, vdw_a):
    """cmm_wda_eos of add_correlation_wda_lj (cmmdft/functionals.py:339-362):
    SumOfEOS([MBWR, CS(Rhs), MFA(a)], factors=[1, -1, -1]) at ``temperature``."""
    from .eos import ModifiedBenedictWebbRubinEOS, CarnahanStarlingEOS, MFAEOS
    mb = ModifiedBenedictWebbRubinEOS(mass, sigma, epsilon)
    cs = CarnahanStarlingEOS(mass, R)
    mf = MFAEOS(mass, sigma, epsilon, a=vdw_a)
    for e in (mb, cs, mf):
        e.set_temperature(temperature)
    w = L.WdaEos()
    w.D = 2 * R
    w.sigma3 = sigma ** 3
    w.epsilon = epsilon
    w.gamma = mb.gamma
    for i in range(8):
        w.a[i] = mb.a[i]
    for i in range(6):
        w.b[i] = mb.b[i]
    w.eta = cs.eta
    w.kT = boltzmann * temperature
    w.a_mfa = mf.a
    for i, f in enumerate((1, -1, -1)):
        w.factors[i] = f
    return w


def build_functional(host, npoints, temperature, guest, version='WBII', tailcorrections=False,
                     cutoff=12 * angstrom, mfa_cutoff=12 * angstrom, limit_potential=1e4 * kjmol, plan=None,
                     wda=False):
    """Device Functional for ``host`` (SyntheticHost-like) at ``npoints``.

    guest = (sigma, epsilon, mass) in atomic units; wda=True adds the WDA
    correlation part of add_correlation_wda_lj.
    """
    sigma, epsilon, mass = guest
    if plan is None:
        plan = E.GridPlan(npoints, host.rvecs)
    sig, eps = host_type_arrays(host)
    V = E.external_potential(plan, host.recentred_pos(), host.ffatype_ids, sig, eps, sigma, epsilon,
                             cutoff, limit_potential)
    kst, a = E.mfa_kernel_spectrum(plan, sigma, epsilon, mfa_cutoff, rep=2 if tailcorrections else 1)
    R = hardsphere_radius(sigma, epsilon, temperature)
    beta = 1.0 / (boltzmann * temperature)
    lam = thermal_wavelength(mass, temperature)
    w = wda_struct(sigma, epsilon, mass, temperature, R, a) if wda else None
    return E.Functional(plan, R, beta, lam, V, hs_version_code(version), kst, a, wda=w)


def isotherm_inputs(pressures, temperature, guest):
    """(mu, rho_bulk) per pressure from the MBWR EOS (eos.py:209-215, calculator.py:129-131)."""
    sigma, epsilon, mass = guest
    mb = ModifiedBenedictWebbRubinEOS(mass, sigma, epsilon)
    mus = mb.calculate_mu(temperature, np.asarray(pressures, dtype=float).ravel())
    return mus, mb.bulk_density(temperature, mus)


def initial_density(fn, chempots, ninit=None):
    """Initial guesses [B, N1, N2, N3] on the device (cmmdft/program.py:219-305).

    ninit None -> ideal gas exp(beta (mu - V)) / Lambda^3;
    ninit array of floats -> ninit[b] * exp(-max(V, 0) / kT) (Ninit=float branch).
    """
    import torch
    mu = torch.as_tensor(np.asarray(chempots, dtype=np.float64), device='cuda').view(-1, 1, 1, 1)
    V = fn.V.unsqueeze(0)
    if ninit is None:
        return torch.exp(fn.beta * (mu - V)) / fn.lambda3
    n0 = torch.as_tensor(np.asarray(ninit, dtype=np.float64), device='cuda').view(-1, 1, 1, 1)
    kT = 1.0 / fn.beta
    return n0 * torch.exp(-torch.clamp(V, min=0.0) / kT)
