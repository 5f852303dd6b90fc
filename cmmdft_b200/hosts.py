"""Seeded synthetic hosts and the LJ parameter sets of the benchmark workloads.

The reference reads hosts from yaff checkpoints plus an ``LJ:PARS`` file
(cmmdft/system.py:54-73, cmmdft/extpot_calculator.py:705-716).  The benchmark
workloads use synthetic hosts instead: atoms placed by random sequential
addition (RSA) in an orthorhombic cell with a minimum nearest-image
separation, and atom types drawn as a seeded permutation of fixed counts.
The four atom types carry the UFF sigma/epsilon of a ZIF-8-like framework
(C, H, N, Zn), and the guest is united-atom TraPPE methane.
"""

import numpy as np

from .units import angstrom, boltzmann, amu

# (sigma [angstrom], epsilon/kB [K]) per host atom type.
HOST_LJ_TYPES = {
    "C": (3.43, 52.8),
    "H": (2.57, 22.1),
    "N": (3.26, 34.7),
    "Zn": (2.46, 62.4),
}
# Type counts of the 276-atom cell; larger cells keep these fractions.
HOST_TYPE_COUNTS = {"C": 96, "H": 120, "N": 48, "Zn": 12}

# Standard atomic weights [amu] of the host atom types (for unit conversions
# of loadings only; the grid solve does not use host masses).
ATOM_MASSES = {"C": 12.011, "H": 1.008, "N": 14.007, "Zn": 65.38}

# United-atom methane: sigma [angstrom], epsilon/kB [K], mass [amu].
METHANE = {"sigma": 3.73, "epsilon_K": 148.0, "mass": 16.04}
# Helium probe for the void fraction (Hirschfelder, Curtiss and Bird).
HELIUM = {"sigma": 2.576, "epsilon_K": 10.22}


def lj_type_table(types=HOST_LJ_TYPES):
    """Return ``{name: (sigma, epsilon)}`` in atomic units (bohr, Hartree)."""
    return {k: (s * angstrom, e * boltzmann) for k, (s, e) in types.items()}


def type_counts_for(natom, counts=HOST_TYPE_COUNTS):
    """Split ``natom`` over the types in the ratio of ``counts`` (largest remainder)."""
    names = list(counts)
    w = np.array([counts[n] for n in names], dtype=float)
    exact = natom * w / w.sum()
    base = np.floor(exact).astype(int)
    rem = natom - base.sum()
    order = np.argsort(-(exact - base), kind="stable")
    base[order[:rem]] += 1
    return dict(zip(names, base.tolist()))


class SyntheticHost(object):
    """A periodic orthorhombic host cell with typed LJ atoms.

    Attributes mirror what the reference's spherical external-potential path
    reads from a yaff ``System`` (cmmdft/extpot_calculator.py:199-209):
    ``pos`` (natom x 3, bohr), ``ffatypes`` (names), ``ffatype_ids``,
    ``rvecs`` (3 x 3 cell vectors as rows, bohr) and ``ff`` (type name ->
    (sigma, epsilon) in atomic units).
    """

    def __init__(self, pos, ffatypes, ffatype_ids, rvecs, ff):
        self.pos = np.asarray(pos, dtype=np.float64)
        self.ffatypes = list(ffatypes)
        self.ffatype_ids = np.asarray(ffatype_ids, dtype=np.int32)
        self.rvecs = np.asarray(rvecs, dtype=np.float64)
        self.ff = dict(ff)

    @property
    def natom(self):
        return len(self.pos)

    @property
    def volume(self):
        return float(abs(np.linalg.det(self.rvecs)))

    @property
    def masses(self):
        """Atomic masses (atomic units) from the type names' standard weights."""
        w = np.array([ATOM_MASSES.get(t, np.nan) for t in self.ffatypes])
        return w[self.ffatype_ids] * amu

    def recentred_pos(self):
        """Positions shifted so their mean is the origin (cmmdft/system.py:70)."""
        return self.pos - self.pos.sum(axis=0) / len(self.pos)


def random_sequential_host(lengths_A, natom, seed, min_sep_A=1.3,
                           counts=HOST_TYPE_COUNTS, types=HOST_LJ_TYPES,
                           max_tries=2000000):
    """Place ``natom`` atoms uniformly in the cell by RSA.

    A trial position is rejected when its nearest-image distance to any
    accepted atom is below ``min_sep_A``.  Types are a seeded permutation of
    the counts returned by :func:`type_counts_for`.  Positions are returned in
    bohr and are not recentred (the host wrapper recentres, as the reference
    does for checkpoint hosts).
    """
    rng = np.random.default_rng(seed)
    L = np.asarray(lengths_A, dtype=float).reshape(3)
    accepted = np.zeros((natom, 3))
    n = 0
    tries = 0
    min2 = min_sep_A ** 2
    # Large cells test a trial only against the accepted atoms of the 27 bins
    # (edge >= min_sep) around it: the same accept/reject decisions as the
    # test against every atom, since no other atom is within min_sep.
    nb = np.floor(L / min_sep_A).astype(int)
    binned = natom > 2000 and bool(np.all(nb >= 3))
    if binned:
        bins = {}
        off = np.array([(a, b, c) for a in (-1, 0, 1) for b in (-1, 0, 1) for c in (-1, 0, 1)])
    while n < natom:
        tries += 1
        if tries > max_tries:
            raise RuntimeError("RSA could not place %d atoms" % natom)
        trial = rng.uniform(0.0, 1.0, 3) * L
        if binned:
            bt = np.minimum((trial / L * nb).astype(int), nb - 1)
            near = [i for o in off for i in bins.get(tuple((bt + o) % nb), ())]
            if near:
                d = accepted[near] - trial
                d -= L * np.round(d / L)
                if np.min(np.einsum("ij,ij->i", d, d)) < min2:
                    continue
            bins.setdefault(tuple(bt), []).append(n)
        elif n:
            d = accepted[:n] - trial
            d -= L * np.round(d / L)
            if np.min(np.einsum("ij,ij->i", d, d)) < min2:
                continue
        accepted[n] = trial
        n += 1
    cnt = type_counts_for(natom, counts)
    names = list(cnt)
    ids = np.concatenate([np.full(cnt[k], i, dtype=np.int32) for i, k in enumerate(names)])
    ids = rng.permutation(ids).astype(np.int32)
    rvecs = np.diag(L) * angstrom
    ff = lj_type_table({k: types[k] for k in names})
    return SyntheticHost(accepted * angstrom, names, ids, rvecs, ff)


def cubic_host_276(seed=0):
    """The 276-atom cubic cell (a = 17.0 angstrom) used at 32^3 and 64^3."""
    return random_sequential_host((17.0, 17.0, 17.0), 276, seed)


def uneven_hosts(nhost=8, seed=2, density_A3=0.056, edge_range=(12.0, 40.0)):
    """Orthorhombic hosts with edges drawn from U(edge_range), seeded."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(nhost):
        L = rng.uniform(edge_range[0], edge_range[1], 3)
        natom = int(round(density_A3 * float(np.prod(L))))
        out.append(random_sequential_host(tuple(L), natom, seed * 1000 + i))
    return out


def methane_guest_params():
    """(sigma, epsilon, mass) of the methane guest in atomic units."""
    return (METHANE["sigma"] * angstrom, METHANE["epsilon_K"] * boltzmann,
            METHANE["mass"] * amu)


def cubic_host_779(seed=0):
    """The 276-atom cell's atom density at a = 24.0 angstrom (779 atoms, 96^3)."""
    return random_sequential_host((24.0, 24.0, 24.0), 779, seed)


def cubic_host_64(seed=4, density_A3=0.056):
    """The large cubic cell of the 256^3 WDA workload: a = 64 angstrom at the
    276-atom cell's atom density (14,680 atoms, the same type mix)."""
    natom = int(round(density_A3 * 64.0 ** 3))
    return random_sequential_host((64.0, 64.0, 64.0), natom, seed)


# Rigid TraPPE CO2 (Potoff and Siepmann, AIChE J. 47, 1676 (2001)): C-O bond
# 1.16 angstrom, site (sigma [angstrom], epsilon/kB [K]) and mass [amu].
CO2_TRAPPE = {"bond": 1.16, "types": {"O_CD": (3.05, 79.0), "C_CD": (2.80, 27.0)},
              "masses": {"O_CD": 15.9994, "C_CD": 12.0107}}


def co2_trappe_guest():
    """Sites of rigid linear CO2 along z (O, C, O): dict with pos [3, 3],
    masses [3], ffatypes, ffatype_ids, ff {type: (sigma, epsilon)} and the
    per-site sigma/epsilon arrays, all in atomic units."""
    b = CO2_TRAPPE["bond"] * angstrom
    types = ["O_CD", "C_CD"]
    ids = np.array([0, 1, 0], dtype=np.int32)
    ff = {t: (CO2_TRAPPE["types"][t][0] * angstrom, CO2_TRAPPE["types"][t][1] * boltzmann) for t in types}
    pos = np.array([[0.0, 0.0, b], [0.0, 0.0, 0.0], [0.0, 0.0, -b]])
    masses = np.array([CO2_TRAPPE["masses"][types[i]] * amu for i in ids])
    return dict(pos=pos, masses=masses, ffatypes=types, ffatype_ids=ids, ff=ff,
                site_sigma=np.array([ff[types[i]][0] for i in ids]),
                site_epsilon=np.array([ff[types[i]][1] for i in ids]))
