"""The batched EOS root search against scipy.optimize.brentq (CPU).

The reference solves p(rho) = p and mu(rho) = mu one bracket at a time with
scipy's brentq (cmmdft/eos.py:85-157).  EquationOfState solves all brackets
of a pressure or chemical-potential list together (brentq_lanes); the roots
must be the very same floats.
"""
import numpy as np
import pytest
from scipy.optimize import brentq

from cmmdft_b200.eos import ModifiedBenedictWebbRubinEOS, SumOfEOS, CarnahanStarlingEOS, MFAEOS
from cmmdft_b200.hosts import methane_guest_params
from cmmdft_b200.units import bar, boltzmann


def _scalar_pressure_roots(e, p, n=10000):
    kT = boltzmann * e.temperature
    grid = e.get_rough_density_grid(n)
    iv = e._brackets([p], kT * grid + grid ** 2 * e.derivative_excess_free_energy_particle(grid), grid)[0]
    f = lambda r: kT * r + r ** 2 * e.derivative_excess_free_energy_particle(r) - p
    return sorted(brentq(f, a, b) for a, b in iv)


def _scalar_chempot_roots(e, mu, n=1000):
    kT = boltzmann * e.temperature
    grid = e.get_rough_density_grid(n)
    g = lambda r: kT * np.log(e.wvl ** 3 * r) + e.excess_free_energy_particle(r) + \
        r * e.derivative_excess_free_energy_particle(r)
    iv = e._brackets([mu], g(grid), grid)[0]
    return sorted(brentq(lambda r: g(r) - mu, a, b) for a, b in iv)


@pytest.mark.parametrize("kind,T", [("mbwr", 150.0), ("mbwr", 300.0), ("sum", 300.0)])
def test_lanes_match_scalar_brentq(kind, T):
    sig, eps, mass = methane_guest_params()
    mb = ModifiedBenedictWebbRubinEOS(mass, sig, eps)
    e = mb if kind == "mbwr" else SumOfEOS(mass, [mb, CarnahanStarlingEOS(mass, 3.5), MFAEOS(mass, sig, eps)],
                                           [1, -1, -1])
    e.set_temperature(T)
    P = np.concatenate([np.logspace(-3, 2, 24), 10 ** np.random.default_rng(3).uniform(-4, 3, 16)]) * bar
    allp = e.solve_densities_from_pressures(P)
    for i, p in enumerate(P):
        got = allp[i][~np.isnan(allp[i])]
        assert np.array_equal(np.array(_scalar_pressure_roots(e, p)), got)
    mus = e.compute_chempot(allp[:, 0])
    allc = e.solve_densities_from_chempots(mus)
    for i, mu in enumerate(mus):
        got = allc[i][~np.isnan(allc[i])]
        assert np.array_equal(np.array(_scalar_chempot_roots(e, mu)), got)


def test_scalar_and_array_forms_agree():
    sig, eps, mass = methane_guest_params()
    mb = ModifiedBenedictWebbRubinEOS(mass, sig, eps)
    P = np.logspace(-3, 2, 6) * bar
    mus = mb.calculate_mu(300.0, P)
    assert [mb.calculate_mu(300.0, p) for p in P] == list(mus)
    assert [mb.bulk_density(300.0, m) for m in mus] == list(mb.bulk_density(300.0, mus))


def test_isotherm_inputs_equal_reference(golden32, golden64):
    """mu(P) and the bulk density as the reference computes them, to the bit."""
    from cmmdft_b200 import workload as W
    guest = methane_guest_params()
    mus, bulks = W.isotherm_inputs(golden64["pressures"] * bar, 300.0, guest)
    assert np.array_equal(mus, golden64["mu"])
    assert np.array_equal(bulks, golden64["rho_bulk"])
    mu1, b1 = W.isotherm_inputs(np.array([1.0]) * bar, 300.0, guest)
    assert mu1[0] == float(golden32["mu"]) and b1[0] == float(golden32["rho_bulk"])
