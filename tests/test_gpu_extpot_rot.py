"""Orientation-averaged external potential of a rigid multi-site guest
(cmm_extpot_rot) against the unmodified reference: rigid CO2 (TraPPE) in the
276-atom host on a 20^3 grid at 300 K, Lebedev degrees 9 and 11
(tests/golden/rot20.npz, from the reference's own
generate_effective_potential).

The reference stores site potentials in float32, so a rounding difference in
a float64 site sum can move a float32 value by one unit in the last place;
tolerance: per point 1e-6 relative (float32 has 6e-8) with an absolute floor
of 1e-12 Hartree, non-finite values (sites inside host atoms) where the
reference has them, and after the capping of add_external_potential 1e-9 of
the cap."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

import cmmdft_b200 as cd
from cmmdft_b200 import engine as E
from cmmdft_b200 import workload as W
from cmmdft_b200.hosts import cubic_host_276
from cmmdft_b200.rotations import combined_rotations
from cmmdft_b200.units import angstrom, boltzmann, kjmol

CAP = 1e4 * kjmol


@pytest.fixture(scope="module")
def cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return True


def site_params(ref):
    ids = ref["guest_ffatype_ids"]
    return ref["guest_sigma"][ids], ref["guest_epsilon"][ids]


def compare(V, Vr):
    fin = np.isfinite(Vr)
    assert np.array_equal(np.isfinite(V), fin)
    mod = fin & (np.abs(Vr) < CAP)
    d = np.abs(V[mod] - Vr[mod])
    rel = float(np.max(d / (np.abs(Vr[mod]) + 1e-12 / 1e-6)))
    exact = int(np.sum(V == Vr))
    cap = lambda a: np.minimum(np.where(np.isfinite(a), a, CAP), CAP)
    capped = float(np.max(np.abs(cap(V) - cap(Vr)))) / CAP
    return rel, capped, exact


@pytest.mark.parametrize("deg", [9, 11])
@pytest.mark.parametrize("rotations", ["reference", "package"])
def test_effective_potential_against_reference(cuda, golden_rot, deg, rotations):
    ref = golden_rot
    h = cubic_host_276(0)
    n = int(ref["n"])
    plan = E.GridPlan((n, n, n), h.rvecs)
    sig, eps = W.host_type_arrays(h)
    ss, se = site_params(ref)
    rot, w = (ref["rot%d" % deg], ref["w%d" % deg]) if rotations == "reference" else combined_rotations(deg)
    V = E.effective_potential(plan, h.recentred_pos(), h.ffatype_ids, sig, eps, ref["guest_pos"],
                              ref["guest_masses"], ss, se, rot, w, 12 * angstrom, 1 / float(ref["T"]) / boltzmann,
                              CAP).cpu().numpy()
    rel, capped, exact = compare(V, ref["V%d" % deg])
    print("CO2 degree %d, %s rotations: max rel %.2e, capped %.2e of the cap, %d of %d bit-identical"
          % (deg, rotations, rel, capped, exact, V.size))
    assert rel < 1e-6 and capped < 1e-9


def test_dual_model_guest_through_program(cuda, golden_rot, tmp_path):
    """Program -> FreeEnergy.add_external_potential(temperature=T, degree=11)
    with a DualModelGuest: the capped potential against the reference's, the
    eff_epot_<T>K.npy file in the reference's directory layout, a second
    Program served from it, and set_temperature generating the potential of
    a new temperature (functionals.py:213-251, 1019-1025)."""
    ref = golden_rot
    h = cubic_host_276(0)
    types = [str(t) for t in ref["guest_ffatypes"]]
    ff = {t: (s, e) for t, s, e in zip(types, ref["guest_sigma"], ref["guest_epsilon"])}
    T = float(ref["T"])

    def program():
        host = cd.NanoporousHost('synthetic', pos=h.pos, ffatypes=h.ffatypes, ffatype_ids=h.ffatype_ids,
                                 rvecs=h.rvecs, ff=h.ff, masses=h.masses)
        guest = cd.DualModelGuest('CO2', 44.0 * cd.amu, 3.9 * angstrom, 200 * boltzmann, pos=ref["guest_pos"],
                                  masses=ref["guest_masses"], ffatypes=types, ffatype_ids=ref["guest_ffatype_ids"],
                                  ff=ff)
        prog = cd.Program(prefix=str(tmp_path), hostname='synthetic', guestname='CO2', ff_suffix='trappe')
        prog.set_system(host, guest)
        prog.set_grid(npoints=int(ref["n"]))
        prog.init_free_energy(T)
        prog.fener.add_hard_sphere(version='WBII')
        prog.fener.add_external_potential(temperature=T, cutoff=12 * angstrom, degree=11)
        return prog

    prog = program()
    ext = prog.fener.part_dict['ExtPot']
    V300 = ext.potential.copy()
    Vr = ref["V11"]
    Vr_c = np.minimum(np.where(np.isfinite(Vr), Vr, CAP), CAP)
    err = float(np.max(np.abs(ext.potential - Vr_c))) / CAP
    print("DualModelGuest through Program: %.2e of the cap" % err)
    assert err < 1e-9
    fn = tmp_path / 'synthetic' / 'CO2' / 'trappe' / '' / '' / 'eff_epot_300.00K.npy'
    assert fn.is_file() and (prog.workdir / 'ExtPots').is_symlink()
    again = program()                                    # loaded from the file
    assert np.array_equal(again.fener.part_dict['ExtPot'].potential, ext.potential)
    prog.fener.set_temperature(350.0)                    # a new temperature: generated and written
    assert (tmp_path / 'synthetic' / 'CO2' / 'trappe' / 'eff_epot_350.00K.npy').is_file()
    V350 = prog.fener.part_dict['ExtPot'].potential
    assert np.all(V350 <= CAP) and not np.array_equal(V350, V300)


def test_derivative_channels_against_reference(cuda, golden_rotinterp):
    """cmm_extpot_lj_deriv on the 0.15 A grid (114^3) against the reference's
    get_external_potential_derivatives at 3000 seeded points per guest atom
    type: 1e-12 of each channel's largest magnitude there."""
    ref = golden_rotinterp
    h = cubic_host_276(0)
    sig, eps = W.host_type_arrays(h)
    fn = [int(x) for x in ref["fine_npoints"]]
    idx = ref["deriv_idx"]
    for t, s, e in zip(ref["guest_ffatypes"], ref["guest_sigma"], ref["guest_epsilon"]):
        d = E.external_potential_derivatives(h.rvecs, fn, ref["fine_spacings"], h.recentred_pos(), h.ffatype_ids,
                                             sig, eps, s, e, 12 * angstrom, 1e6 * kjmol)
        got = d[:, idx[:, 0], idx[:, 1], idx[:, 2]].cpu().numpy()
        r = ref["deriv_" + str(t)]
        errs = [float(np.max(np.abs(got[c] - r[c])) / max(np.max(np.abs(r[c])), 1e-300)) for c in range(8)]
        print("channels of %s: %s" % (t, " ".join("%.1e" % x for x in errs)))
        assert max(errs) < 1e-12


def test_interpolated_potential_through_program(cuda, golden_rotinterp, tmp_path):
    """add_external_potential(temperature=T, degree=9, interpolate=True) with a
    NonSphericalGuest on the 12^3 grid against the reference's
    ExternalPotential.generate_potential(interpolate=True), capped as
    add_external_potential caps: 1e-9 of the cap, and per point 1e-6
    relative below the cap."""
    ref = golden_rotinterp
    h = cubic_host_276(0)
    types = [str(t) for t in ref["guest_ffatypes"]]
    ff = {t: (s, e) for t, s, e in zip(types, ref["guest_sigma"], ref["guest_epsilon"])}
    host = cd.NanoporousHost('synthetic', pos=h.pos, ffatypes=h.ffatypes, ffatype_ids=h.ffatype_ids, rvecs=h.rvecs,
                             ff=h.ff)
    guest = cd.DualModelGuest('CO2', 44.0 * cd.amu, 3.9 * angstrom, 200 * boltzmann, pos=ref["guest_pos"],
                              masses=ref["guest_masses"], ffatypes=types, ffatype_ids=ref["guest_ffatype_ids"], ff=ff)
    prog = cd.Program(prefix=str(tmp_path), hostname='synthetic', guestname='CO2')
    prog.set_system(host, guest)
    prog.set_grid(npoints=int(ref["n"]))
    prog.init_free_energy(float(ref["T"]))
    prog.fener.add_external_potential(temperature=float(ref["T"]), cutoff=12 * angstrom, degree=int(ref["degree"]),
                                      interpolate=True)
    V = prog.fener.part_dict['ExtPot'].potential
    Vr = ref["V"]
    Vr_c = np.minimum(np.where(np.isfinite(Vr), Vr, CAP), CAP)
    err = float(np.max(np.abs(V - Vr_c))) / CAP
    mod = np.abs(Vr_c) < CAP
    rel = float(np.max(np.abs(V[mod] - Vr_c[mod]) / (np.abs(Vr_c[mod]) + 1e-6)))
    print("interpolated CO2 potential: %.2e of the cap, %.2e relative, %d of %d bit-identical"
          % (err, rel, int(np.sum(V == Vr_c)), V.size))
    assert err < 1e-9 and rel < 1e-6


@pytest.mark.parametrize("interpolate", [False, True])
def test_large_rotation_set_against_oracle(cuda, golden_rotinterp, interpolate, tmp_path):
    """Lebedev degree 29 (8758 rotations): more rotations than one block's
    shared memory holds, so the rotation energies go through the global
    scratch of one row per grid point.  The 4^3 grid through
    ExternalPotential.generate_potential against the oracle at 4 seeded
    points: per point 1e-6 relative (the float32 storage of the site
    potentials), non-finite values where the oracle has them."""
    from oracle import cmm_oracle as O
    ref = golden_rotinterp
    h = cubic_host_276(0)
    types = [str(t) for t in ref["guest_ffatypes"]]
    tp = {t: (s, e) for t, s, e in zip(types, ref["guest_sigma"], ref["guest_epsilon"])}
    guest = cd.NonSphericalGuest('CO2', pos=ref["guest_pos"], masses=ref["guest_masses"], ffatypes=types,
                                 ffatype_ids=ref["guest_ffatype_ids"], ff=tp)
    host = cd.NanoporousHost('synthetic', pos=h.pos, ffatypes=h.ffatypes, ffatype_ids=h.ffatype_ids, rvecs=h.rvecs,
                             ff=h.ff)
    n, deg, T = 4, 29, float(ref["T"])
    prog = cd.Program(prefix=str(tmp_path), hostname='synthetic', guestname='CO2')
    prog.set_system(host, guest)
    prog.set_grid(npoints=n)
    ext = cd.ExternalPotential(prog.grid, prog.system, cutoff=12 * angstrom, degree=deg,
                                           interpolate=interpolate)
    ext.generate_potential(temperature=T)
    V = ext._V.cpu().numpy()
    rot, w = combined_rotations(deg)
    assert len(w) == 8758
    g = np.linspace(-0.5, 0.5, n, endpoint=False)
    idx = np.random.default_rng(11).integers(0, n, size=(4, 3))
    pts = np.einsum('ab,ia->ib', h.rvecs, g[idx])
    beta = 1 / T / boltzmann
    if interpolate:
        st = [types[i] for i in ref["guest_ffatype_ids"]]
        fine_n = [int(np.ceil(l / ext.INTERP_SPACING)) for l in np.linalg.norm(h.rvecs, axis=1)]
        Vo = O.interpolated_effective_potential(pts, ref["guest_pos"], ref["guest_masses"], st, tp, rot, w, beta,
                                                h.ff, h.recentred_pos(), h.ffatypes, h.ffatype_ids, h.rvecs, fine_n,
                                                prog.grid.points[0, 0, 0, :3], np.full(3, ext.INTERP_SPACING),
                                                limit_potential=ext.limit_potential)
    else:
        ids = ref["guest_ffatype_ids"]
        Vo = O.effective_potential(pts, ref["guest_pos"], ref["guest_masses"], ref["guest_sigma"][ids],
                                   ref["guest_epsilon"][ids], rot, w, beta, h.ff, h.recentred_pos(), h.ffatypes,
                                   h.ffatype_ids, h.rvecs, limit_potential=ext.limit_potential)
    Vg = V[idx[:, 0], idx[:, 1], idx[:, 2]]
    fin = np.isfinite(Vo) & (np.abs(Vo) < ext.limit_potential)
    assert np.array_equal(np.isfinite(Vg) & (np.abs(Vg) < ext.limit_potential), fin)
    rel = float(np.max(np.abs(Vg[fin] - Vo[fin]) / (np.abs(Vo[fin]) + 1e-6))) if fin.any() else 0.0
    print("degree 29, interpolate=%s: %d finite points, max rel %.2e" % (interpolate, int(fin.sum()), rel))
    assert fin.any() and rel < 1e-6


def test_five_site_guest_against_oracle(cuda):
    """A five-site guest (tetrahedral CH4-like: a centre and four sites at
    1.09 A) takes the kernel's any-guest form (more than three sites in
    registers): the 4^3 grid at Lebedev degree 5 against the oracle at every
    point, per point 1e-6 relative (float32 site sums), non-finite values
    where the oracle has them."""
    from oracle import cmm_oracle as O
    h = cubic_host_276(0)
    sig, eps = W.host_type_arrays(h)
    d = 1.09 * angstrom / np.sqrt(3.0)
    gpos = np.array([[0, 0, 0], [d, d, d], [-d, -d, d], [-d, d, -d], [d, -d, -d]], dtype=float)
    gm = np.array([12.011, 1.008, 1.008, 1.008, 1.008])
    ss = np.array([3.40, 2.65, 2.65, 2.65, 2.65]) * angstrom
    se = np.array([55.0, 7.9, 7.9, 7.9, 7.9]) * boltzmann
    n = 4
    plan = E.GridPlan((n, n, n), h.rvecs)
    rot, w = combined_rotations(5)
    beta = 1 / 300.0 / boltzmann
    V = E.effective_potential(plan, h.recentred_pos(), h.ffatype_ids, sig, eps, gpos, gm, ss, se, rot, w,
                              12 * angstrom, beta, CAP).cpu().numpy().ravel()
    g = np.linspace(-0.5, 0.5, n, endpoint=False)
    idx = np.stack(np.meshgrid(np.arange(n), np.arange(n), np.arange(n), indexing='ij'), -1).reshape(-1, 3)
    pts = np.einsum('ab,ia->ib', h.rvecs, g[idx])
    Vo = O.effective_potential(pts, gpos, gm, ss, se, rot, w, beta, h.ff, h.recentred_pos(), h.ffatypes,
                               h.ffatype_ids, h.rvecs, limit_potential=CAP)
    rel, capped, exact = compare(V, Vo)
    print("five-site guest, degree 5: max rel %.2e, capped %.2e of the cap, %d of %d bit-identical"
          % (rel, capped, exact, V.size))
    assert rel < 1e-6 and capped < 1e-9
