"""Synthetic hosts (CPU): the binned random sequential addition makes the
same decisions as the all-atom test, and the 64 angstrom workload host has
the stated size, type mix and minimum separation."""
import numpy as np
import pytest
from scipy.spatial import cKDTree

from cmmdft_b200 import hosts as H
from cmmdft_b200.units import angstrom


def test_binned_rsa_equals_all_atom_rsa(monkeypatch):
    a = H.random_sequential_host((30.0, 26.0, 22.0), 2400, seed=7)
    # force the all-atom test by making every axis too short for the bins
    real_floor = np.floor

    def no_bins(x, *k):
        r = real_floor(x, *k)
        return np.minimum(r, 2) if np.ndim(r) == 1 and len(r) == 3 else r
    monkeypatch.setattr(H.np, "floor", no_bins)
    b = H.random_sequential_host((30.0, 26.0, 22.0), 2400, seed=7)
    monkeypatch.undo()
    assert np.array_equal(a.pos, b.pos) and np.array_equal(a.ffatype_ids, b.ffatype_ids)


def test_cubic_host_64():
    h = H.cubic_host_64()
    assert h.natom == 14680
    assert np.allclose(np.diag(h.rvecs), 64.0 * angstrom) and np.count_nonzero(h.rvecs - np.diag(np.diag(h.rvecs))) == 0
    counts = np.bincount(h.ffatype_ids, minlength=4)
    w = np.array([H.HOST_TYPE_COUNTS[k] for k in h.ffatypes], dtype=float)
    assert np.all(np.abs(counts - h.natom * w / w.sum()) < 1)
    L = 64.0 * angstrom
    tree = cKDTree(np.mod(h.pos, L), boxsize=L)
    d, _ = tree.query(np.mod(h.pos, L), k=2)
    assert d[:, 1].min() >= 1.3 * angstrom * (1 - 1e-12)
