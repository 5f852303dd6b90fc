"""Pin the numpy oracle against fixtures produced by the unmodified reference.

The fixtures in tests/golden were written by tests/golden/make_golden.py,
which ran the reference package itself.  Tolerances are stated per check.
"""
import numpy as np
import pytest

from cmmdft_b200.hosts import cubic_host_276, methane_guest_params, HELIUM
from cmmdft_b200.units import angstrom, kjmol, bar, boltzmann
from oracle import cmm_oracle as O
from tests._common import relerr, scalar_rel, oracle_case


@pytest.fixture(scope="module")
def case32(golden32):
    return oracle_case(32)


def test_host_generator_is_pinned(golden32):
    h = cubic_host_276(0)
    assert np.array_equal(h.pos, golden32["host_pos"])
    assert np.array_equal(h.ffatype_ids, golden32["host_ids"])
    assert np.array_equal(h.rvecs, golden32["host_rvecs"])


def test_scalars(golden32):
    sig, eps, mass = methane_guest_params()
    T = float(golden32["T"])
    assert scalar_rel(O.hardsphere_radius(sig, eps, T), golden32["Rhs"]) == 0.0
    assert scalar_rel(O.thermal_wavelength(mass, T), golden32["wavelength"]) == 0.0
    mb = O.MBWR(mass, sig, eps)
    mu = O.eos_calculate_mu(mb, T, 1.0 * bar)
    assert scalar_rel(mu, golden32["mu"]) < 1e-14
    mb.set_temperature(T)
    rb = np.nanmin(O.eos_densities_from_chempots(mb, [mu]), axis=1)[0]
    assert scalar_rel(rb, golden32["rho_bulk"]) < 1e-12


def test_external_potential(golden32, case32):
    grid, fe = case32
    V = fe.part_dict["ExtPot"].potential
    # elementwise, relative to the capped maximum (1e4 kJ/mol)
    assert relerr(V, golden32["V"]) < 1e-14


def test_helium_fraction(golden32, case32):
    grid, fe = case32
    h = cubic_host_276(0)
    f = O.helium_void_fraction(grid, h.recentred_pos(), h.ff, h.ffatypes, h.ffatype_ids, h.rvecs,
                               300.0, HELIUM["sigma"] * angstrom, HELIUM["epsilon_K"] * boltzmann)
    assert scalar_rel(f, golden32["he_frac"]) < 1e-13


@pytest.mark.parametrize("tag", ["a", "b"])
def test_functional_derivatives_and_values(golden32, case32, tag):
    grid, fe = case32
    rho = golden32["rho_" + tag]
    mu = float(golden32["mu"])
    k = grid.fft(rho)
    hs, mfa, ext = fe.parts
    beta = fe.beta
    # The WBII phi3 branch just above n3 = 1e-8 cancels catastrophically, so
    # 1-ulp input differences give ~1e-8 RELATIVE noise in the (tiny) HS
    # derivative in dilute regions.  What the fixed point sees is
    # exp(-beta*C1): the tolerance is on beta*|dC1| (relative change of rho).
    # Measured floor of the reference against itself under 1-ulp input
    # perturbations: 1.1e-10 on the ideal-gas profile 'a', 3.4e-8 on the
    # sharp-edged dense profile 'b'; weighted by rho/max(rho): 3e-13 / 2.6e-10.
    floor = {"a": 5e-10, "b": 1e-7}[tag]
    dC = beta * np.abs(hs.derive(k) - golden32["dHS_" + tag])
    assert dC.max() < floor
    assert (dC * rho).max() / rho.max() < 1e-9
    assert relerr(mfa.derive(k), golden32["dMFA_" + tag]) < 1e-13
    vals = [p.value(k) for p in fe.parts]
    for v, g in zip(vals, golden32["values_" + tag]):
        assert scalar_rel(v, g) < 1e-12
    s = O.Picard(fe, nsteps=1, method="static")
    s._initiate_solving(mu)
    assert scalar_rel(s._get_Omega(rho, k), golden32["omega_" + tag]) < 1e-12
    assert beta * np.max(np.abs(s._get_C1(rho, k) - golden32["C1_" + tag])) < floor
    assert relerr(hs.get_n3(k), golden32["n3_" + tag]) < 1e-13


def test_static_picard_trajectory(golden32, case32):
    grid, fe = case32
    mu = float(golden32["mu"])
    rho0 = golden32["rho_a"]
    s = O.Picard(fe, nsteps=3, alpha_mix=0.1, method="static", criterion="res", threshold=1e-8)
    N, rho, conv = s.solve(mu, rho0.copy())
    assert relerr(rho, golden32["picard3_rho"]) < 1e-10
    s = O.Picard(fe, nsteps=500, alpha_mix=0.1, method="static", criterion="res", threshold=1e-8)
    N, rho, conv = s.solve(mu, rho0.copy())
    assert conv and s.curr_step == int(golden32["picard_steps"])
    assert relerr(rho, golden32["picard_rho"]) < 1e-10
    assert scalar_rel(N, golden32["picard_N"]) < 1e-10


def test_static_picard_der_criterion(golden32, case32):
    grid, fe = case32
    s = O.Picard(fe, nsteps=500, alpha_mix=0.1, method="static", criterion=["der"], threshold=[1e-3])
    N, rho, conv = s.solve(float(golden32["mu"]), golden32["rho_a"].copy())
    assert conv and s.curr_step == int(golden32["der_steps"])
    # near convergence dOmega is a difference of O(10 kT) terms that cancel to
    # ~1e-4 kT, so the C1 noise floor (~1e-9 kT) shows at ~1e-5 relative
    assert scalar_rel(s.DER, golden32["der_value"]) < 1e-4
    assert relerr(rho, golden32["der_rho"]) < 1e-10


def test_hybrid_anderson_converged(golden32, case32):
    grid, fe = case32
    mu = float(golden32["mu"])
    s = O.Anderson(fe, nsteps=500, m=5, criterion=["res", "riue"], threshold=[1e-13, 1e-12])
    N, rho, conv = s.solve(mu, golden32["rho_a"].copy())
    assert conv
    # converged solutions (RES < 1e-13, RIUE < 1e-12 on both sides)
    assert relerr(rho, golden32["and_rho"]) < 1e-10
    assert scalar_rel(N, golden32["and_N"]) < 1e-10


def test_mfa_tailcorrections(golden32):
    grid, fe = oracle_case(32, tail=True)
    k = grid.fft(golden32["rho_b"])
    mfa = fe.part_dict["MFA"]
    assert relerr(mfa.derive(k), golden32["dMFA_tail_b"]) < 1e-13
    assert scalar_rel(mfa.value(k), golden32["vMFA_tail_b"]) < 1e-12


@pytest.mark.parametrize("tag", ["a", "b"])
def test_wda_part(golden32, tag):
    grid, fe = oracle_case(32, V=golden32["V"])
    sig, eps, mass = methane_guest_params()
    w = O.add_wda(fe, sig, eps, mass, 300.0)
    rho = golden32["rho_" + tag]
    k = grid.fft(rho)
    assert fe.beta * np.max(np.abs(w.derive(k) - golden32["wda_dWDA_" + tag])) < 1e-12
    assert scalar_rel(w.value(k), golden32["wda_values_" + tag][3]) < 1e-12


TENSOR_CASES = [("atWBII", "a"), ("atWBII", "b"), ("tWBII", "a"), ("tWBII", "b"), ("atFMT", "b"), ("tMFMT", "b")]


@pytest.mark.parametrize("ver,tag", TENSOR_CASES)
def test_tensor_hard_sphere(golden32, case32, ver, tag):
    """Tensor FMT variants (functionals.py:457-487, 534-552, 620-717)."""
    grid, fe = case32
    hs = O.HardSphere(grid, float(golden32["Rhs"]), 300.0, version=ver)
    k = grid.fft(golden32["rho_" + tag])
    # the beta-scaled noise floor of the WBII closed forms (see the plain case)
    floor = {"a": 2e-9, "b": 1e-7}[tag]
    assert hs.beta * np.max(np.abs(hs.derive(k) - golden32["hs_%s_d_%s" % (ver, tag)])) < floor
    assert scalar_rel(hs.value(k), golden32["hs_%s_v_%s" % (ver, tag)]) < 1e-12
