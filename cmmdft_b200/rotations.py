"""Rotation sets for orientational averages of non-spherical guests
(cmmdft/extpot_calculator.py:341-383, 616-655).

``generate_rotation_matrix(degree, 2)``: ``degree`` rotations about z at
angles 2 pi k / degree, with the common weight 1 / (degree 4 pi).
``generate_rotation_matrix(degree, 3)``: one rotation per point of the
Lebedev rule of the smallest tabulated degree >= ``degree`` (the rule the
reference's AngularGrid picks; points and weights here from
``scipy.integrate.lebedev_rule``, the weights sum to 4 pi), the rotation
taking z to the point by the polar angle phi1 and the azimuth phi2 of the
point.  The 4D (Stroud) rule of the reference is not provided.

``combined_rotations(degree)`` forms the nrot = n3 * n2 matrices and weights
w3 * w2 that generate_effective_potential hands to the orientational
average.  The reference combines the sets there with the contraction
``einsum('aij,bjk->abij', R3, R2)``, i.e. R3[a] times diag of the row sums
of R2[b], which is not a product of the two rotations; that is the default
here so that the effective potentials agree with the reference's.
``form='product'`` gives the products R3 R2 (the contraction of the
reference's single-point effective_potential, :551-567).
"""
import bisect

import numpy as np

__all__ = ['LEBEDEV_DEGREES', 'lebedev_degree', 'generate_rotation_matrix', 'combined_rotations']

# degrees of the tabulated Lebedev rules (cmmdft/rotations/AngGrid.py:38-71)
LEBEDEV_DEGREES = (3, 5, 7, 9, 11, 13, 15, 17, 19, 21, 23, 25, 27, 29, 31, 35, 41, 47, 53, 59, 65, 71, 77, 83,
                   89, 95, 101, 107, 113, 119, 125, 131)


def lebedev_degree(degree):
    """The tabulated degree used for ``degree``: itself or the next larger one."""
    if degree < 0 or degree > LEBEDEV_DEGREES[-1]:
        raise ValueError("Argument degree should be a positive integer <= %d, got %r"
                         % (LEBEDEV_DEGREES[-1], degree))
    return LEBEDEV_DEGREES[bisect.bisect_left(LEBEDEV_DEGREES, degree)]


def generate_rotation_matrix(degree, dimension):
    """(rotations [n, 3, 3], weights) as the reference's generate_rotation_matrix."""
    if dimension == 2:
        theta = np.linspace(0, 2 * np.pi, degree, endpoint=False)
        c, s = np.cos(theta), np.sin(theta)
        z, o = np.zeros_like(c), np.ones_like(c)
        rot = np.array([[c, -s, z], [s, c, z], [z, z, o]])
        return rot.transpose(2, 0, 1), 1 / (degree * 4 * np.pi)
    if dimension == 3:
        from scipy.integrate import lebedev_rule
        pts, w = lebedev_rule(lebedev_degree(degree))
        x, y, zz = pts
        phi1 = np.arctan2(np.sqrt(y ** 2 + x ** 2), zz)
        phi2 = np.arctan2(y, x)
        c1, s1 = np.cos(phi1), np.sin(phi1)
        c2, s2 = np.cos(phi2), np.sin(phi2)
        z = np.zeros(len(phi1))
        rot = np.array([[c1 * c2, -s2, s1 * c2], [c1 * s2, c2, s1 * s2], [-s1, z, c1]])
        return rot.transpose(2, 0, 1), np.asarray(w)
    raise NotImplementedError("rotation sets of dimension %r" % dimension)


def combined_rotations(degree, form='reference'):
    """(matrices [n3 * n2, 3, 3], weights [n3 * n2]) of the orientational average."""
    r1, w1 = generate_rotation_matrix(degree, 3)
    r2, w2 = generate_rotation_matrix(degree, 2)
    if form == 'reference':
        rot = np.einsum('aij,bjk->abij', r1, r2).reshape(-1, 3, 3)
    elif form == 'product':
        rot = np.einsum('nij,mjk->nmik', r1, r2).reshape(-1, 3, 3)
    else:
        raise ValueError("form must be 'reference' or 'product', got %r" % (form,))
    return rot, np.repeat(w1 * w2, len(r2))
