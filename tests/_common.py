"""Shared helpers for the test suite (builds the oracle side of a case)."""
import numpy as np

from cmmdft_b200.hosts import cubic_host_276, methane_guest_params
from cmmdft_b200.units import angstrom, kjmol


def relerr(a, b, scale=None):
    """Max abs difference relative to max|b| (or ``scale``)."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    s = np.max(np.abs(b)) if scale is None else scale
    if s == 0:
        return float(np.max(np.abs(a - b)))
    return float(np.max(np.abs(a - b)) / s)


def scalar_rel(a, b):
    return abs(float(a) - float(b)) / max(abs(float(b)), 1e-300)


def oracle_case(npts=32, T=300.0, host=None, V=None, hs_version='WBII', tail=False, guest=None):
    """Oracle functional for the 276-atom cubic host at ``npts``^3."""
    from oracle import cmm_oracle as O
    host = cubic_host_276(0) if host is None else host
    sig, eps, mass = methane_guest_params() if guest is None else guest
    grid = O.OGrid(host.rvecs, npoints=npts)
    if V is None:
        pos = host.recentred_pos()
        V = O.external_potential(grid.points[..., :3].reshape(-1, 3), host.ff, sig, eps, pos,
                                 host.ffatypes, host.ffatype_ids, host.rvecs).reshape(grid.npoints)
        V = O.cap_potential(V, 1e4 * kjmol)
    fe = O.build_functional(grid, sig, eps, mass, T, V, hs_version=hs_version,
                            tailcorrections=tail)
    return grid, fe
