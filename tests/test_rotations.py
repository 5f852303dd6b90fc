"""Multi-site guests on the CPU: the oracle's orientational average and the
package's rotation sets against the unmodified reference
(tests/golden/rot20.npz, rigid CO2 in the 276-atom host at 300 K)."""
import numpy as np
import pytest

import cmmdft_b200 as cd
from cmmdft_b200.hosts import cubic_host_276
from cmmdft_b200.rotations import combined_rotations, generate_rotation_matrix, lebedev_degree
from cmmdft_b200.units import boltzmann
from oracle import cmm_oracle as O


def site_params(ref):
    ids = ref["guest_ffatype_ids"]
    return ref["guest_sigma"][ids], ref["guest_epsilon"][ids]


@pytest.mark.parametrize("deg", [9, 11])
def test_oracle_effective_potential_is_bit_exact(golden_rot, deg):
    """The oracle's restatement with the reference's own rotation matrices
    reproduces the reference's effective potential bit for bit at 40
    seeded grid points (including non-finite values inside host atoms)."""
    ref = golden_rot
    h = cubic_host_276(0)
    n = int(ref["n"])
    g = np.linspace(-0.5, 0.5, n, endpoint=False)
    idx = np.random.default_rng(5).integers(0, n, size=(40, 3))
    pts = np.einsum('ab,ia->ib', h.rvecs, g[idx])
    ss, se = site_params(ref)
    Vo = O.effective_potential(pts, ref["guest_pos"], ref["guest_masses"], ss, se, ref["rot%d" % deg],
                               ref["w%d" % deg], 1 / float(ref["T"]) / boltzmann, h.ff, h.recentred_pos(),
                               h.ffatypes, h.ffatype_ids, h.rvecs)
    Vr = ref["V%d" % deg][idx[:, 0], idx[:, 1], idx[:, 2]]
    assert np.array_equal(Vo, Vr)


@pytest.mark.parametrize("deg", [9, 11])
def test_rotation_sets_match_reference(golden_rot, deg):
    """combined_rotations (Lebedev points from scipy) holds the reference's
    matrices and weights (its tabulated Lebedev rule, its contraction of the
    3D and 2D sets) up to ordering: every matrix within 1e-15, weights within
    1e-15 of 1/nrot-scale values."""
    rot, w = combined_rotations(deg)
    rr, wr = golden_rot["rot%d" % deg], golden_rot["w%d" % deg]
    assert rot.shape == rr.shape and w.shape == wr.shape
    d = np.abs(rr.reshape(len(rr), 1, 9) - rot.reshape(1, len(rot), 9)).max(axis=2)
    j = d.argmin(axis=1)
    assert len(set(j.tolist())) == len(rr)           # a one-to-one matching
    assert d[np.arange(len(rr)), j].max() < 1e-15
    assert np.abs(w[j] - wr).max() < 1e-15
    assert abs(w.sum() - 1.0) < 1e-13


def test_lebedev_degree_rounds_up():
    assert lebedev_degree(9) == 9 and lebedev_degree(10) == 11 and lebedev_degree(32) == 35
    assert len(generate_rotation_matrix(10, 3)[0]) == 50
    with pytest.raises(ValueError):
        lebedev_degree(200)


def test_product_form_is_a_rotation_set():
    rot, w = combined_rotations(9, form='product')
    eye = np.einsum('nij,nkj->nik', rot, rot)
    assert np.abs(eye - np.eye(3)).max() < 1e-14
    with pytest.raises(ValueError):
        combined_rotations(9, form='other')


def test_guest_classes(golden_rot):
    ref = golden_rot
    types = [str(t) for t in ref["guest_ffatypes"]]
    ff = {t: (s, e) for t, s, e in zip(types, ref["guest_sigma"], ref["guest_epsilon"])}
    g = cd.NonSphericalGuest('CO2', pos=ref["guest_pos"], masses=ref["guest_masses"], ffatypes=types,
                             ffatype_ids=ref["guest_ffatype_ids"], ff=ff)
    assert g.natom == 3 and g.mass == ref["guest_masses"].sum()
    s, e = g.site_parameters()
    assert np.array_equal(s, site_params(ref)[0]) and np.array_equal(e, site_params(ref)[1])
    with pytest.raises(NotImplementedError):
        g.compute_hardsphere_radius(300.0)
    d = cd.DualModelGuest('CO2', 1.0, 3.7 * 1.8897261254578281, 200 * boltzmann, pos=ref["guest_pos"],
                          masses=ref["guest_masses"], ffatypes=types, ffatype_ids=ref["guest_ffatype_ids"], ff=ff)
    d.compute_hardsphere_radius(300.0)
    assert d.Rhs > 0 and d.natom == 3 and d.mass == ref["guest_masses"].sum()
    c = d.copy()
    assert type(c) is cd.DualModelGuest and c.sigma == d.sigma and np.array_equal(c.mol.pos, d.mol.pos)
    with pytest.raises(ValueError):
        cd.NonSphericalGuest('X', pos=ref["guest_pos"], masses=None, ffatypes=types,
                             ffatype_ids=ref["guest_ffatype_ids"], ff=ff)


def _fine_points(h, idx, fine_n):
    g = idx * (1.0 / fine_n) + (-0.5)
    return np.einsum('ab,ia->ib', h.rvecs, g)


def test_oracle_derivative_channels_are_bit_exact(golden_rotinterp):
    """get_external_potential_derivatives restated: the eight channels at
    3000 seeded points of the 0.15 A grid, per guest atom type."""
    ref = golden_rotinterp
    h = cubic_host_276(0)
    pts = _fine_points(h, ref["deriv_idx"], ref["fine_npoints"])
    for t, s, e in zip(ref["guest_ffatypes"], ref["guest_sigma"], ref["guest_epsilon"]):
        d = O.external_potential_derivatives(pts, h.ff, s, e, h.recentred_pos(), h.ffatypes, h.ffatype_ids,
                                             h.rvecs, ref["fine_spacings"])
        assert np.array_equal(d, ref["deriv_" + str(t)])


def test_oracle_interpolated_potential_is_bit_exact(golden_rotinterp):
    """The tricubic path (derivative grids at 0.15 A, Hermite tensor-product
    interpolation, the package's rotation set) against the reference's
    ExternalPotential.generate_potential(interpolate=True) at 12 seeded
    points of its 12^3 grid."""
    ref = golden_rotinterp
    h = cubic_host_276(0)
    n = int(ref["n"])
    g = np.linspace(-0.5, 0.5, n, endpoint=False)
    idx = np.random.default_rng(3).integers(0, n, size=(12, 3))
    pts = np.einsum('ab,ia->ib', h.rvecs, g[idx])
    types = [str(t) for t in ref["guest_ffatypes"]]
    tp = {t: (s, e) for t, s, e in zip(types, ref["guest_sigma"], ref["guest_epsilon"])}
    st = [types[i] for i in ref["guest_ffatype_ids"]]
    rot, w = combined_rotations(int(ref["degree"]))
    Vo = O.interpolated_effective_potential(pts, ref["guest_pos"], ref["guest_masses"], st, tp, rot, w,
                                            1 / float(ref["T"]) / boltzmann, h.ff, h.recentred_pos(), h.ffatypes,
                                            h.ffatype_ids, h.rvecs, ref["fine_npoints"], ref["origin"],
                                            ref["interp_spacing"])
    assert np.array_equal(Vo, ref["V"][idx[:, 0], idx[:, 1], idx[:, 2]])


def test_co2_trappe_guest_matches_reference_files(golden_rot):
    """The rigid TraPPE CO2 of the rotation-average benchmark line has the
    geometry and site LJ parameters of the reference's own guest files
    (positions to 1e-15 bohr; masses from standard atomic weights, within
    2e-7 relative of the reference's)."""
    from cmmdft_b200.hosts import co2_trappe_guest
    ref = golden_rot
    g = co2_trappe_guest()
    ids = ref["guest_ffatype_ids"]
    assert np.abs(g["pos"] - ref["guest_pos"]).max() < 1e-15
    assert np.array_equal(g["site_sigma"], ref["guest_sigma"][ids])
    assert np.array_equal(g["site_epsilon"], ref["guest_epsilon"][ids])
    assert [g["ffatypes"][i] for i in g["ffatype_ids"]] == [str(ref["guest_ffatypes"][i]) for i in ids]
    assert np.abs(g["masses"] / ref["guest_masses"] - 1).max() < 2e-7
