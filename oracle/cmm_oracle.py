"""CPU oracle for the CmmDFT grid solve (TEST INFRASTRUCTURE ONLY).

This module restates, in plain numpy/scipy, the reference algorithm of the
path that cmmdft_b200 implements on the GPU.  It is the checker: only the test
suite, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` / ``--impl
reference`` legs of ``bench.py`` may import it.  Nothing in the product path
(``cmmdft_b200``) imports, calls or falls back to this file.

Parity of this restatement is pinned against the unmodified reference run
in the build container: ``tests/golden/make_golden.py`` imports the reference
through import shims and writes the fixtures that ``tests/test_oracle_golden.py``
compares this module with.

Every function cites the reference file:line (paths inside the reference
project) whose arithmetic it follows.  FFTs use full complex spectra with the
reference's phase convention so that rounding follows the reference closely.
"""

import numpy as np
import scipy.fft as sfft
import scipy.optimize as opt
from scipy.optimize import brentq

from cmmdft_b200.units import angstrom, kjmol, boltzmann, planck

FFT_WORKERS = 1

FMT_NAMES = ['FMT', 'aFMT', 'tFMT', 'atFMT', 'taFMT']        # functionals.py:375-377
MFMT_NAMES = ['MFMT', 'aMFMT', 'tMFMT', 'atMFMT', 'taMFMT']
WBII_NAMES = ['WBII', 'aWBII', 'tWBII', 'atWBII', 'taWBII']


# ---------------------------------------------------------------- grid ----
class OGrid(object):
    """Centred periodic grid; cmmdft/system.py:231-295 and :307-332."""

    def __init__(self, rvecs, npoints=None, spacing=0.25 * angstrom):
        self.rvecs = np.asarray(rvecs, dtype=np.float64)
        lengths = np.linalg.norm(self.rvecs, axis=1)
        if npoints is None:  # system.py:252-255
            self.npoints = [int(np.ceil(l / spacing)) for l in lengths]
        elif isinstance(npoints, int):
            self.npoints = [npoints] * 3
        else:
            self.npoints = [int(n) for n in npoints]
        n = self.npoints
        # column norms, system.py:262-266
        self.spacings = [np.linalg.norm(self.rvecs[:, a]) / n[a] for a in range(3)]
        self.volume = float(abs(np.linalg.det(self.rvecs)))
        self.dr = self.volume / np.prod(n)
        self.points = np.zeros(n + [4])
        g = [np.linspace(-0.5, 0.5, num=n[a], endpoint=False) for a in range(3)]
        gp = np.asarray(np.meshgrid(g[0], g[1], g[2], indexing='ij'))
        self.points[..., :3] = np.einsum('ab,aijk->ijkb', self.rvecs, gp)
        self.points[..., 3] = np.sqrt(self.points[..., 0] ** 2 + self.points[..., 1] ** 2
                                      + self.points[..., 2] ** 2)
        self.kpoints = np.zeros(n + [4])
        kg = [np.fft.fftfreq(n[a], d=self.spacings[a]) for a in range(3)]
        kp = np.meshgrid(kg[0], kg[1], kg[2], indexing='ij')
        for a in range(3):
            self.kpoints[..., a] = 2 * np.pi * kp[a]
        self.kpoints[..., 3] = np.sqrt(self.kpoints[..., 0] ** 2 + self.kpoints[..., 1] ** 2
                                       + self.kpoints[..., 2] ** 2)
        self.scalprod = (self.kpoints[..., 0] * self.spacings[0] * n[0]
                         + self.kpoints[..., 1] * self.spacings[1] * n[1]
                         + self.kpoints[..., 2] * self.spacings[2] * n[2])
        kcut = 2 * np.pi / np.array(self.spacings)  # system.py:293-295
        self.sigma_lanczos = (np.sinc(self.kpoints[..., 0] / kcut[0])
                              * np.sinc(self.kpoints[..., 1] / kcut[1])
                              * np.sinc(self.kpoints[..., 2] / kcut[2]))
        self._phase = np.exp(1j * np.pi * self.scalprod)
        self._iphase = np.exp(-1j * np.pi * self.scalprod)

    def supercell(self, rep):
        rep = np.asarray(rep)
        return OGrid(self.rvecs * rep, npoints=list(np.asarray(self.npoints) * rep))

    def integrate(self, data):  # system.py:307-308
        return np.sum(data) * self.dr

    def fft(self, rdata):  # system.py:310-311
        return sfft.fftn(rdata, workers=FFT_WORKERS) * self._phase / np.prod(self.npoints)

    def fftn(self, rdata):  # system.py:313-321
        F = sfft.fftn(rdata, axes=(0, 1, 2), workers=FFT_WORKERS)
        return F * (self._phase / np.prod(self.npoints))[..., None]

    def ifft(self, fdata):  # system.py:323-324
        return sfft.ifftn(fdata * self._iphase, workers=FFT_WORKERS).real * np.prod(self.npoints)

    def ifftn(self, fdata):  # system.py:326-332
        F = sfft.ifftn(fdata * self._iphase[..., None], axes=(0, 1, 2), workers=FFT_WORKERS)
        return F.real * np.prod(self.npoints)


# --------------------------------------------------------------- guest ----
def hardsphere_radius(sigma, epsilon, temperature):
    """Barker-Henderson fit, cmmdft/system.py:154-158."""
    beta = 1 / (boltzmann * temperature)
    Tt = 1 / beta / epsilon
    return sigma * (1 + 0.2977 * Tt) / (1 + 0.33163 * Tt + 0.0010477 * Tt ** 2) / 2


def thermal_wavelength(mass, temperature):
    """cmmdft/system.py:115-117."""
    kT = boltzmann * temperature
    return planck / np.sqrt(2 * np.pi * mass * kT)


# ------------------------------------------------------ external pot ----
def lennard_jones(r, sigma, epsilon, cutoff):
    """Cut-and-shifted LJ, cmmdft/extpot_calculator.py:156-183."""
    inside = r < cutoff
    V = np.zeros_like(r)
    r6 = (sigma / r[inside]) ** 6
    r12 = r6 * r6
    rc6 = (sigma / cutoff) ** 6
    shift = 4 * epsilon * (rc6 ** 2 - rc6)
    V[inside] = 4 * epsilon * (r12 - r6) - shift
    return V


def external_potential(points, ff, sig_g, eps_g, pos, ffatypes, ffatype_ids, rvecs,
                       cutoff=12 * angstrom):
    """Host-atom loop with Lorentz-Berthelot mixing and per-axis minimum image,
    cmmdft/extpot_calculator.py:186-222.  ``pos`` must already be recentred."""
    Vext = np.zeros(len(points))
    X, Y, Z = points.T
    L = np.linalg.norm(rvecs, axis=1)  # rows, extpot_calculator.py:202
    for i, tid in enumerate(ffatype_ids):
        s, e = ff[ffatypes[tid]]
        sm = 0.5 * (s + sig_g)
        em = np.sqrt(e * eps_g)
        rx = X - pos[i, 0]
        ry = Y - pos[i, 1]
        rz = Z - pos[i, 2]
        rx -= L[0] * (rx / L[0]).round()
        ry -= L[1] * (ry / L[1]).round()
        rz -= L[2] * (rz / L[2]).round()
        R = np.sqrt(rx ** 2 + ry ** 2 + rz ** 2 + 1e-16)
        Vext[:] += lennard_jones(R, sm, em, cutoff)
    return Vext


def effective_potential(points, guest_pos, guest_masses, site_sigma, site_epsilon, rotations, weights, beta,
                        ff, pos, ffatypes, ffatype_ids, rvecs, cutoff=12 * angstrom,
                        limit_potential=1e4 * kjmol):
    """Orientation-averaged potential of a rigid multi-site guest at
    ``points`` [m, 3] (effective_potential_vectorized as
    generate_effective_potential calls it, cmmdft/extpot_calculator.py:
    569-655): the guest moved to each point and centred on its centre of
    mass, each rotation applied about it, the site potentials (the host-atom
    LJ sum of external_potential with the site's own sigma/epsilon) stored in
    float32 and summed there, then -logsumexp(-beta pot, b=weights) / beta,
    NaN -> limit_potential.  ``pos`` must already be recentred."""
    from scipy.special import logsumexp
    m, nsite, nrot = len(points), len(guest_pos), len(rotations)
    masses = np.asarray(guest_masses, dtype=np.float64).reshape(nsite, 1)
    neutral = guest_pos[None, :, :] + points[:, None, :]
    com = np.sum(neutral * masses[None, :, :], axis=1) / np.sum(masses)
    rel = neutral - com[:, None, :]
    rotated = np.einsum('rij,mnj->mnri', rotations, rel) + com[:, None, None, :]
    pot = np.zeros((m, nsite, nrot), dtype=np.float32)
    for a in range(nsite):
        coords = rotated[:, a, :, :].reshape(m * nrot, 3)
        pot[:, a, :] = external_potential(coords, ff, site_sigma[a], site_epsilon[a], pos, ffatypes, ffatype_ids,
                                          rvecs, cutoff).reshape(m, nrot)
    pot = np.sum(pot, axis=1)
    res = -logsumexp(-float(beta) * pot, b=weights, axis=1) / beta
    return np.where(np.isnan(res), limit_potential, res)


def lennard_jones_derivatives(r, sigma, epsilon, cutoff):
    """V and the radial factors dV, ddV, dddV of lennard_jones(derivative=True)
    (cmmdft/extpot_calculator.py:156-183)."""
    inside = r < cutoff
    V, dV, ddV, dddV = (np.zeros_like(r) for _ in range(4))
    ri = r[inside]
    r6 = (sigma / ri) ** 6
    r12 = r6 * r6
    rc6 = (sigma / cutoff) ** 6
    V[inside] = 4 * epsilon * (r12 - r6) - 4 * epsilon * (rc6 ** 2 - rc6)
    dV[inside] = 24 * epsilon * (r6 - 2 * r12) / ri ** 2
    ddV[inside] = 96 * epsilon * (7 * r12 - 2 * r6) / ri ** 4
    dddV[inside] = 384 * epsilon * (5 * r6 - 28 * r12) / ri ** 6
    return V, dV, ddV, dddV


def external_potential_derivatives(points, ff, sig_g, eps_g, pos, ffatypes, ffatype_ids, rvecs, spacings,
                                   cutoff=12 * angstrom):
    """[8, m]: V, dV/dx, dV/dy, dV/dz, d2V/dxdy, d2V/dxdz, d2V/dydz, d3V/dxdydz
    at ``points`` in the unit-cube scaling of a grid with ``spacings``, with
    the clipping of get_external_potential_derivatives
    (cmmdft/extpot_calculator.py:264-338).  ``pos`` must already be recentred."""
    n = len(points)
    out = np.zeros((8, n))
    X, Y, Z = points.T
    L = np.linalg.norm(rvecs, axis=1)
    for i, tid in enumerate(ffatype_ids):
        s, e = ff[ffatypes[tid]]
        sm = 0.5 * (s + sig_g)
        em = np.sqrt(e * eps_g)
        rx = X - pos[i, 0]
        ry = Y - pos[i, 1]
        rz = Z - pos[i, 2]
        rx -= L[0] * (rx / L[0]).round()
        ry -= L[1] * (ry / L[1]).round()
        rz -= L[2] * (rz / L[2]).round()
        R = np.sqrt(rx ** 2 + ry ** 2 + rz ** 2 + 1e-16)
        V, dV, ddV, dddV = lennard_jones_derivatives(R, sm, em, cutoff)
        out[0] += V
        out[1] += dV * rx
        out[2] += dV * ry
        out[3] += dV * rz
        out[4] += ddV * rx * ry
        out[5] += ddV * rx * rz
        out[6] += ddV * ry * rz
        out[7] += dddV * rx * ry * rz
    vmax = 1e+6 * kjmol
    mask = out[0] > vmax
    for c in range(4):
        out[c] = np.clip(out[c], -vmax, vmax)
    out[4:, mask] = 0.0
    dx, dy, dz = spacings
    for c, f in ((1, dx), (2, dy), (3, dz), (4, dx * dy), (5, dx * dz), (6, dy * dz), (7, dx * dy * dz)):
        out[c] *= f
    return out


# corner offsets and derivative orders of the tricubic scheme
# (cmmdft/extpot_calculator.py:408-413 and the channel order above)
TRICUBIC_CORNERS = ((0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0), (0, 0, 1), (1, 0, 1), (0, 1, 1), (1, 1, 1))
TRICUBIC_ORDERS = ((0, 0, 0), (1, 0, 0), (0, 1, 0), (0, 0, 1), (1, 1, 0), (1, 0, 1), (0, 1, 1), (1, 1, 1))


def _hermite(c, o, t):
    """Cubic Hermite basis on [0, 1]: value (o = 0) or slope (o = 1) at end c."""
    if o == 0:
        return (1 - t) ** 2 * (1 + 2 * t) if c == 0 else t * t * (3 - 2 * t)
    return t * (1 - t) ** 2 if c == 0 else t * t * (t - 1)


def tricubic(deriv_at, positions, origin, spacing, npoints):
    """Interpolator.tricubic_interpolation (cmmdft/extpot_calculator.py:
    391-549) of the channel values that ``deriv_at(idx [m, 3]) -> [8, m]``
    gives at fine-grid indices: cell of each position by floor((p - origin)
    / spacing), periodic corner indices, and the tricubic polynomial fixed by
    the 64 corner values -- the tensor product of cubic Hermite interpolants,
    which is what the reference's 64 x 64 matrix encodes."""
    s = (positions - origin) / spacing
    ix = np.floor(s).astype(int)
    r = s - ix
    npoints = np.asarray(npoints)
    res = np.zeros(len(positions))
    for (cx, cy, cz) in TRICUBIC_CORNERS:
        idx = (ix + np.array([cx, cy, cz])) % npoints
        vals = deriv_at(idx)
        for d, (ox, oy, oz) in enumerate(TRICUBIC_ORDERS):
            res += vals[d] * _hermite(cx, ox, r[:, 0]) * _hermite(cy, oy, r[:, 1]) * _hermite(cz, oz, r[:, 2])
    return res


def interpolated_effective_potential(points, guest_pos, guest_masses, site_types, type_params, rotations, weights,
                                     beta, ff, pos, ffatypes, ffatype_ids, rvecs, fine_npoints, origin, spacing,
                                     cutoff=12 * angstrom, limit_potential=1e4 * kjmol):
    """The orientational average of ``effective_potential`` with the site
    potentials interpolated tricubically from per-type derivative grids
    (ExternalPotential.generate_potential(interpolate=True),
    cmmdft/functionals.py:1032-1055): the fine grid has ``fine_npoints`` points
    per axis over the cell (Grid points, spacing |a_i| / n_i), the
    interpolator takes ``origin`` and ``spacing``.  Channel values are
    computed at the corners that are needed only."""
    from scipy.special import logsumexp
    fine_npoints = np.asarray(fine_npoints)
    fine_sp = np.linalg.norm(rvecs, axis=0) / fine_npoints          # Grid.spacings (columns)
    m, nsite, nrot = len(points), len(guest_pos), len(rotations)
    masses = np.asarray(guest_masses, dtype=np.float64).reshape(nsite, 1)
    neutral = guest_pos[None, :, :] + points[:, None, :]
    com = np.sum(neutral * masses[None, :, :], axis=1) / np.sum(masses)
    rel = neutral - com[:, None, :]
    rotated = np.einsum('rij,mnj->mnri', rotations, rel) + com[:, None, None, :]
    pot = np.zeros((m, nsite, nrot), dtype=np.float32)

    def grid_points(idx):
        g = idx * (1.0 / fine_npoints) + (-0.5)     # linspace(-0.5, 0.5, n, endpoint=False)[i]
        return np.einsum('ab,ia->ib', rvecs, g)

    for a in range(nsite):
        sg, eg = type_params[site_types[a]]
        at = lambda idx: external_potential_derivatives(grid_points(idx), ff, sg, eg, pos, ffatypes, ffatype_ids,
                                                        rvecs, fine_sp, cutoff)
        coords = rotated[:, a, :, :].reshape(m * nrot, 3)
        pot[:, a, :] = tricubic(at, coords, origin, spacing, fine_npoints).reshape(m, nrot)
    pot = np.sum(pot, axis=1)
    res = -logsumexp(-float(beta) * pot, b=weights, axis=1) / beta
    return np.where(np.isnan(res), limit_potential, res)


def cap_potential(V, limit):
    """cmmdft/functionals.py:247-251 (non-finite and > limit -> limit)."""
    V = V.copy()
    V[~np.isfinite(V)] = limit
    V[V > limit] = limit
    return V


# ---------------------------------------------------------- hard sphere --
class HardSphere(object):
    """White-Bear / Rosenfeld / modified FMT, cmmdft/functionals.py:375-618."""
    name = 'HardSphere'

    def __init__(self, grid, R, temperature, version='WBII'):
        assert version in FMT_NAMES + MFMT_NAMES + WBII_NAMES, version
        self.grid, self.R, self.version = grid, R, version
        self.beta = 1 / (boltzmann * temperature)
        self.krho = None
        self._init_weights()

    def _init_weights(self):  # functionals.py:421-455
        g, R = self.grid, self.R
        om = g.kpoints[..., 3] * R
        mask = ~np.isclose(om, 0)
        kw0 = np.ones_like(om, dtype=np.complex128)
        kw0[mask] = np.sinc(om[mask] / np.pi)
        kw0 *= g.sigma_lanczos
        kw1 = R * kw0
        kw2 = 4.0 * np.pi * R ** 2 * kw0
        j2 = np.ones_like(om, dtype=np.complex128)
        j2[mask] = 3 * (np.sin(om[mask]) - om[mask] * np.cos(om[mask])) / om[mask] ** 3
        j2 *= g.sigma_lanczos
        kw3 = (4.0 * np.pi * R ** 3 / 3.0) * j2
        kwv2 = -1.j * kw3[..., None] * g.kpoints[..., :3]
        kwv2[~mask] = 0.0
        kwv1 = kwv2 / (4 * np.pi * R)
        self.sw = [kw0, kw1, kw2, kw3]
        self.vw = [kwv1, kwv2]
        self.tw = None
        if 't' in self.version:  # tensor weights, functionals.py:457-487
            KX, KY, KZ, K = (g.kpoints[..., i] for i in range(4))
            K2 = K ** 2
            with np.errstate(invalid='ignore', divide='ignore'):
                H = [np.where(K > 0, (KX * KX) / K2, 1 / 3), np.where(K > 0, (KX * KY) / K2, 0.0),
                     np.where(K > 0, (KX * KZ) / K2, 0.0), np.where(K > 0, (KY * KY) / K2, 1 / 3),
                     np.where(K > 0, (KY * KZ) / K2, 0.0), np.where(K > 0, (KZ * KZ) / K2, 1 / 3)]
            B = -4 * np.pi * R ** 2 * (j2 - kw0)
            delta = [1 / 3, 0.0, 0.0, 1 / 3, 0.0, 1 / 3]
            self.tw = [B * (h - d) for h, d in zip(H, delta)]

    def densities(self, krho):  # functionals.py:489-532
        g = self.grid
        n0 = g.ifft(krho * self.sw[0])
        n1 = g.ifft(krho * self.sw[1])
        n2 = g.ifft(krho * self.sw[2])
        n3 = np.clip(g.ifft(krho * self.sw[3]), 1e-30, 0.99)
        nv1 = g.ifftn(krho[..., None] * self.vw[0])
        nv2 = g.ifftn(krho[..., None] * self.vw[1])
        xi = None
        if 'a' in self.version:
            xi = np.clip((nv2[..., 0] ** 2 + nv2[..., 1] ** 2 + nv2[..., 2] ** 2)
                         / (n2 ** 2 + 1e-16), 0.0, 1)
        ln = np.log(1 - n3)
        n32 = n3 * n3
        return n0, n1, n2, n3, ln, n32, n32 * n3, nv1, nv2, xi

    def tensor_densities(self, krho):  # functionals.py:534-548
        xx, xy, xz, yy, yz, zz = (self.grid.ifft(krho * w) for w in self.tw)
        tr2 = xx ** 2 + yy ** 2 + zz ** 2 + 2 * (xy ** 2 + xz ** 2 + yz ** 2)
        tr3 = (xx ** 3 + yy ** 3 + zz ** 3 + 3 * (xx * xy * xy + xx * xz * xz + yy * xy * xy + yy * yz * yz
                                                  + zz * xz * xz + zz * yz * yz) + 6 * xy * xz * yz)
        return [xx, xy, xz, yy, yz, zz, tr2, tr3]

    def get_n3(self, krho):  # functionals.py:554-556 (unclipped)
        return self.grid.ifft(krho * self.sw[3])

    def set_density(self, krho):  # functionals.py:565-572
        if self.krho is not None and np.array_equal(krho, self.krho):
            return
        self.krho = krho
        self.wd = self.densities(krho)
        self.nt = self.tensor_densities(krho) if 't' in self.version else None

    def derive(self, krho):  # functionals.py:574-609
        self.set_density(krho)
        g, v, wd = self.grid, self.version, self.wd
        nt = self.nt
        tot = 0.0
        for f, w in zip([dphi_n0, dphi_n1, dphi_n2, dphi_n3], self.sw):
            tot += g.fft(f(*wd, nt=nt, version=v)) * w
        for f, w in zip([dphi_nv1, dphi_nv2], self.vw):
            kd = g.fftn(f(*wd, nt=nt, version=v))
            tot += -(kd[..., 0] * w[..., 0] + kd[..., 1] * w[..., 1] + kd[..., 2] * w[..., 2])
        if 't' in v:
            kd = g.fftn(dphi_nt(*wd, nt=nt, version=v))
            for c in range(6):
                tot += kd[..., c] * self.tw[c]
        return g.ifft(tot) / self.beta

    def value(self, krho):  # functionals.py:611-618
        self.set_density(krho)
        return self.grid.integrate(phi_total(*self.wd, nt=self.nt, version=self.version)) / self.beta


def _phi1(n3, ln):  # functionals.py:720-721
    return -ln


def _dphi1(n3):  # functionals.py:723-724
    return 1.0 / (1.0 - n3)


def _phi2(n3, ln, n32, v):  # functionals.py:726-732
    if v in FMT_NAMES or v in MFMT_NAMES:
        return 1 / (1.0 - n3)
    return np.where(n3 <= 1e-8, (1 + n32 / 9) / (1 - n3),
                    (5 * n3 - n32 + 2 * (1 - n3) * ln) / (3 * (n3 - n32)))


def _dphi2(n3, ln, n32, v):  # functionals.py:734-741
    q = (1 - 2 * n3 + n32)
    if v in FMT_NAMES or v in MFMT_NAMES:
        return 1 / q
    return np.where(n3 <= 1e-8, (1 + 2 * n3 / 9 + n32 / 18) / q,
                    -2 * (n3 - 3 * n32 + q * ln) / (3 * n32 * q))


def _phi3(n3, ln, n32, n33, v):  # functionals.py:743-754
    q = (1 - 2 * n3 + n32)
    if v in FMT_NAMES:
        return 1 / (24 * np.pi * q)
    if v in MFMT_NAMES:
        return np.where(n3 <= 1e-8, (1.0 - 2 * n3 / 9 - n32 / 18) / (24 * np.pi * q),
                        (n3 + q * ln) / (36 * np.pi * n32 * q))
    return np.where(n3 <= 1e-8, (1 - 4 * n3 / 9 + n32 / 18) / (24 * np.pi * q),
                    -2 * (n3 - 3 * n32 + n33 + ln * q) / ((3 * n32) * 24 * np.pi * q))


def _dphi3(n3, ln, n32, n33, v):  # functionals.py:756-767
    c = (1 - 3 * n3 + 3 * n32 - n33)
    if v in FMT_NAMES:
        return 1 / (12 * np.pi * c)
    if v in MFMT_NAMES:
        return np.where(n3 <= 1e-8, (8 / 3 - 0.5 * n3 - 0.1 * n32) / (36 * np.pi * c),
                        -(2 * n3 - 5 * n32 + n33 + 2 * c * ln) / (36 * np.pi * n33 * c))
    return np.where(n3 <= 1e-8, (7 / 3 - n3 / 2 + n32 / 10) / (36 * np.pi * c),
                    (2 * n3 - 5 * n32 + 6 * n33 - n32 * n32 + 2 * c * ln) / (36 * np.pi * n33 * c))


def _dot3(a, b):
    return a[..., 0] * b[..., 0] + a[..., 1] * b[..., 1] + a[..., 2] * b[..., 2]


def _pref3(n2, nv2, xi, v, nt=None):  # functionals.py:629-639 / 664-673
    if 'a' in v:
        p = (n2 ** 3) * ((1 - xi) ** 3)
    else:
        p = n2 ** 3 - 3.0 * n2 * _dot3(nv2, nv2)
    if 't' in v:
        xx, xy, xz, yy, yz, zz, tr2, tr3 = nt
        vx, vy, vz = nv2[..., 0], nv2[..., 1], nv2[..., 2]
        p += (9 / 2) * (xx * vx ** 2 + yy * vy ** 2 + zz * vz ** 2
                        + 2 * xy * vx * vy + 2 * xz * vx * vz + 2 * yz * vy * vz)
        p -= (9 / 2) * tr3
    return p


def phi_total(n0, n1, n2, n3, ln, n32, n33, nv1, nv2, xi, nt=None, version=None):  # :620-641
    phi = n0 * _phi1(n3, ln)
    phi += (n1 * n2 - _dot3(nv1, nv2)) * _phi2(n3, ln, n32, version)
    phi += _pref3(n2, nv2, xi, version, nt) * _phi3(n3, ln, n32, n33, version)
    return phi


def dphi_n0(n0, n1, n2, n3, ln, n32, n33, nv1, nv2, xi, nt=None, version=None):  # :643-644
    return _phi1(n3, ln)


def dphi_n1(n0, n1, n2, n3, ln, n32, n33, nv1, nv2, xi, nt=None, version=None):  # :646-647
    return n2 * _phi2(n3, ln, n32, version)


def dphi_n2(n0, n1, n2, n3, ln, n32, n33, nv1, nv2, xi, nt=None, version=None):  # :649-656
    d = n1 * _phi2(n3, ln, n32, version)
    if 'a' in version:
        d += (3 * (n2 ** 2) * (1 + xi) * ((1 - xi) ** 2)) * _phi3(n3, ln, n32, n33, version)
    else:
        d += 3 * (n2 ** 2 - _dot3(nv2, nv2)) * _phi3(n3, ln, n32, n33, version)
    return d


def dphi_n3(n0, n1, n2, n3, ln, n32, n33, nv1, nv2, xi, nt=None, version=None):  # :658-676
    d = n0 * _dphi1(n3)
    d += (n1 * n2 - _dot3(nv2, nv1)) * _dphi2(n3, ln, n32, version)
    d += _pref3(n2, nv2, xi, version, nt) * _dphi3(n3, ln, n32, n33, version)
    return d


def dphi_nv1(n0, n1, n2, n3, ln, n32, n33, nv1, nv2, xi, nt=None, version=None):  # :678-680
    return -nv2 * _phi2(n3, ln, n32, version)[..., None]


def dphi_nv2(n0, n1, n2, n3, ln, n32, n33, nv1, nv2, xi, nt=None, version=None):  # :682-701
    d = -nv1 * _phi2(n3, ln, n32, version)[..., None]
    p3 = _phi3(n3, ln, n32, n33, version)
    if 'a' in version:
        d += nv2 * (-6 * n2 * ((1 - xi) ** 2) * p3)[..., None]
    else:
        d += nv2 * (-6 * n2 * p3)[..., None]
    if 't' in version:
        xx, xy, xz, yy, yz, zz, tr2, tr3 = nt
        vx, vy, vz = nv2[..., 0], nv2[..., 1], nv2[..., 2]
        gn = np.empty_like(nv2)
        gn[..., 0] = 2 * (xx * vx + xy * vy + xz * vz)
        gn[..., 1] = 2 * (xy * vx + yy * vy + yz * vz)
        gn[..., 2] = 2 * (xz * vx + yz * vy + zz * vz)
        d += (9 / 2) * gn * p3[..., None]
    return d


def dphi_nt(n0, n1, n2, n3, ln, n32, n33, nv1, nv2, xi, nt=None, version=None):  # :703-717
    xx, xy, xz, yy, yz, zz, tr2, tr3 = nt
    vx, vy, vz = nv2[..., 0], nv2[..., 1], nv2[..., 2]
    g = np.stack([vx * vx - 3 * (xx * xx + xy * xy + xz * xz),
                  (vx * vy - 3 * (xx * xy + yy * xy + xz * yz)) * 2,
                  (vx * vz - 3 * (xx * xz + zz * xz + xy * yz)) * 2,
                  vy * vy - 3 * (yy * yy + xy * xy + yz * yz),
                  (vy * vz - 3 * (yy * yz + zz * yz + xy * xz)) * 2,
                  vz * vz - 3 * (zz * zz + xz * xz + yz * yz)], axis=-1)
    return (9 / 2) * g * _phi3(n3, ln, n32, n33, version)[..., None]


# ----------------------------------------------------------------- MFA ----
def mfa_lj_potential(grid, sigma, epsilon, cutoff=None, rmin=None, limit=0.0):
    """Sampled cut-and-shifted LJ kernel, cmmdft/functionals.py:878-910."""
    if rmin is None:
        rmin = sigma
    r = grid.points[..., 3]
    pot = np.full(r.shape, limit, dtype=np.float64)
    m = r > rmin
    x = np.zeros_like(r)
    x[m] = sigma / r[m]
    pot[m] = 4 * epsilon * (x[m] ** 12 - x[m] ** 6)
    if cutoff is not None:
        rc = r <= cutoff
        rc6 = (sigma / cutoff) ** 6
        pot[rc] -= 4 * epsilon * (rc6 ** 2 - rc6)
        pot[~rc] = 0.0
    return pot


class MFA(object):
    """Mean-field attraction, cmmdft/functionals.py:770-939."""
    name = 'MFA'

    def __init__(self, grid, sigma, epsilon, cutoff=12 * angstrom, tailcorrections=False,
                 repetitions=(2, 2, 2)):
        self.tail = tailcorrections
        self.rep = tuple(repetitions)
        self.small = grid
        self.big = grid.supercell(self.rep) if tailcorrections else grid
        self.potential = mfa_lj_potential(self.big, sigma, epsilon, cutoff=cutoff)
        self.kpotential = self.big.fft(self.potential) * self.big.sigma_lanczos

    def vdw_a(self):  # functionals.py:814-822
        return 0.5 * self.big.integrate(self.potential)

    def derive(self, krho):  # functionals.py:912-926
        if self.tail:
            r0, r1, r2 = self.rep
            return self.small.ifft(krho * self.kpotential[::r0, ::r1, ::r2]) * self.big.volume
        return self.small.ifft(krho * self.kpotential) * self.big.volume

    def value(self, krho):  # functionals.py:928-939
        rho = self.small.ifft(krho)
        return 0.5 * self.small.integrate(rho * self.derive(krho))


class ExtPot(object):
    """External potential part, cmmdft/functionals.py:941-1083."""
    name = 'ExtPot'

    def __init__(self, grid, potential):
        self.grid = grid
        self.potential = potential

    def derive(self, krho):  # functionals.py:1073-1075
        return self.potential

    def value(self, krho):  # functionals.py:1077-1083
        return self.grid.integrate(self.grid.ifft(krho) * self.potential)


# ----------------------------------------------------------------- EOS ----
class MBWR(object):
    """Modified Benedict-Webb-Rubin LJ EOS (Johnson, Zollweg, Gubbins 1993),
    cmmdft/eos.py:295-469; regression parameters of their Table 10."""
    X = [0.8623085097507421, 2.976218765822098, -8.402230115796038, 0.1054136629203555,
         -0.8564583828174598, 1.582759470107601, 0.7639421948305453, 1.753173414312048,
         2.798291772190376e+3, -4.8394220260857657e-2, 0.9963265197721935,
         -3.698000291272493e+1, 2.084012299434647e+1, 8.305402124717285e+1,
         -9.574799715203068e+2, -1.477746229234994e+2, 6.398607852471505e+1,
         1.603993673294834e+1, 6.805916615864377e+1, -2.791293578795945e+3,
         -6.245128304568454, -8.116836104958410e+3, 1.488735559561229e+1,
         -1.059346754655084e+4, -1.131607632802822e+2, -8.867771540418822e+3,
         -3.986982844450543e+1, -4.689270299917261e+3, 2.593535277438717e+2,
         -2.694523589434903e+3, -7.218487631550215e+2, 1.721802063863269e+2]
    gamma = 3.0

    def __init__(self, mass, sigma, epsilon):
        self.mass, self.sigma, self.epsilon = mass, sigma, epsilon

    def set_temperature(self, T):  # eos.py:27-29, 340-366
        self.T = T
        self.wvl = planck / np.sqrt(2 * np.pi * self.mass * boltzmann * T)
        x = [None] + self.X
        Tr = boltzmann * T / self.epsilon
        self.a = [x[1] * Tr + x[2] * np.sqrt(Tr) + x[3] + x[4] / Tr + x[5] / Tr ** 2,
                  x[6] * Tr + x[7] + x[8] / Tr + x[9] / Tr ** 2,
                  x[10] * Tr + x[11] + x[12] / Tr,
                  x[13],
                  x[14] / Tr + x[15] / Tr ** 2,
                  x[16] / Tr,
                  x[17] / Tr + x[18] / Tr ** 2,
                  x[19] / Tr ** 2]
        self.b = [x[20] / Tr ** 2 + x[21] / Tr ** 3,
                  x[22] / Tr ** 2 + x[23] / Tr ** 4,
                  x[24] / Tr ** 2 + x[25] / Tr ** 3,
                  x[26] / Tr ** 2 + x[27] / Tr ** 4,
                  x[28] / Tr ** 2 + x[29] / Tr ** 3,
                  x[30] / Tr ** 2 + x[31] / Tr ** 3 + x[32] / Tr ** 4]

    def _G(self, rho):  # eos.py:368-378
        rr = rho * self.sigma ** 3
        F = np.exp(-self.gamma * rr ** 2)
        ig = 1.0 / (2 * self.gamma)
        G = [ig * (1 - F)]
        for n in range(2, 7):
            G.append(-ig * (F * rr ** (2 * (n - 1)) - 2 * (n - 1) * G[-1]))
        return G

    def fex_particle(self, rho):  # eos.py:395-409
        Ar = 0.0
        rr = rho * self.sigma ** 3
        for i, ai in enumerate(self.a):
            Ar += ai / (i + 1) * rr ** (i + 1)
        for bi, Gi in zip(self.b, self._G(rho)):
            Ar += bi * Gi
        return Ar * self.epsilon

    def dfex_particle(self, rho):  # eos.py:411-422
        dA = 0.0
        rr = rho * self.sigma ** 3
        for i, ai in enumerate(self.a):
            dA += ai * rr ** i * self.sigma ** 3
        F = np.exp(-self.gamma * rr ** 2)
        for t, bi in enumerate(self.b):
            dA += bi * self.sigma ** 3 * rr ** (2 * t + 1) * F
        return dA * self.epsilon

    def rough_grid(self, n):  # eos.py:448-450
        return np.logspace(-10, 0, n) * 1.5 / self.sigma ** 3


class CarnahanStarling(object):
    """cmmdft/eos.py:471-520 (constant Rhs)."""

    def __init__(self, mass, R):
        self.mass, self.R = mass, R
        self.eta = 4 * np.pi * R ** 3 / 3

    def set_temperature(self, T):
        self.T = T
        self.wvl = planck / np.sqrt(2 * np.pi * self.mass * boltzmann * T)

    def fex_particle(self, rho):  # eos.py:503-505
        kT = boltzmann * self.T
        return kT * (4 * self.eta * rho - 3 * (self.eta * rho) ** 2) / (1 - self.eta * rho) ** 2

    def dfex_particle(self, rho):  # eos.py:507-509
        kT = boltzmann * self.T
        return 2 * kT * self.eta * (2 - self.eta * rho) / (1 - self.eta * rho) ** 3


class MFAEOS(object):
    """Mean-field EOS, cmmdft/eos.py:523-546."""

    def __init__(self, mass, sigma=None, epsilon=None, a=None):
        self.mass = mass
        self.a = a if a is not None else -16 / 9 * np.pi * epsilon * sigma ** 3

    def set_temperature(self, T):
        self.T = T

    def fex_particle(self, rho):
        return self.a * rho

    def dfex_particle(self, rho):
        return self.a


def eos_fex_volume(eos, rho):
    """excess_free_energy_volume, eos.py:46-48."""
    return rho * eos.fex_particle(rho)


def eos_dfex_volume(eos, rho):
    """derivative_excess_free_energy_volume, eos.py:54-58."""
    v = rho * eos.dfex_particle(rho)
    v += eos.fex_particle(rho)
    return v


class SumOfEOS(object):
    """cmmdft/eos.py:226-265 (volume forms summed with factors)."""

    def __init__(self, list_eos, factors):
        self.list_eos, self.factors = list_eos, factors

    def set_temperature(self, T):
        for e in self.list_eos:
            e.set_temperature(T)

    def fex_volume(self, rho):
        r = rho * 0.0
        for e, f in zip(self.list_eos, self.factors):
            r += f * eos_fex_volume(e, rho)
        return r

    def dfex_volume(self, rho):
        r = rho * 0.0
        for e, f in zip(self.list_eos, self.factors):
            r += f * eos_dfex_volume(e, rho)
        return r


class WDA(object):
    """WDAVFunctional, cmmdft/functionals.py:1116-1184."""
    name = 'WDA-V'

    def __init__(self, grid, R, eos, temperature):
        self.grid, self.R, self.eos = grid, R, eos
        eos.set_temperature(temperature)
        om = grid.kpoints[..., 3] * (2 * R)
        mask = ~np.isclose(om, 0)
        self.kw = np.zeros_like(om, dtype=np.complex128)
        self.kw[mask] = 3 * (np.sin(om[mask]) - om[mask] * np.cos(om[mask])) / om[mask] ** 3
        self.kw[~mask] = 1.0
        self.kw *= grid.sigma_lanczos

    def wd(self, krho):  # functionals.py:1157-1158
        return self.grid.ifft(krho * self.kw)

    def derive(self, krho):  # functionals.py:1160-1174
        dphi = self.eos.dfex_volume(self.wd(krho))
        return self.grid.ifft(self.grid.fft(dphi) * self.kw)

    def value(self, krho):  # functionals.py:1176-1184
        return self.grid.integrate(self.eos.fex_volume(self.wd(krho)))


def add_wda(fener, sigma, epsilon, mass, temperature):
    """FreeEnergy.add_correlation_wda_lj, cmmdft/functionals.py:339-362."""
    R = fener.part_dict['HardSphere'].R
    a = fener.part_dict['MFA'].vdw_a() if 'MFA' in fener.part_dict else None
    eos = SumOfEOS([MBWR(mass, sigma, epsilon), CarnahanStarling(mass, R), MFAEOS(mass, sigma, epsilon, a=a)],
                   [1, -1, -1])
    w = WDA(fener.grid, R, eos, temperature)
    fener.parts.append(w)
    fener.part_names.append(w.name)
    fener.part_dict[w.name] = w
    return w


def eos_chempot(eos, rho):
    """eos.py:31-33."""
    kT = boltzmann * eos.T
    return kT * np.log(eos.wvl ** 3 * rho) + (rho * eos.dfex_particle(rho) + eos.fex_particle(rho))


def eos_densities_from_pressures(eos, pressures, n_rough=10000):
    """Bracket on a rough log grid then brentq, cmmdft/eos.py:121-157."""
    grid = eos.rough_grid(n_rough)
    kT = boltzmann * eos.T
    pg = kT * grid + grid ** 2 * eos.dfex_particle(grid)
    out = np.zeros([len(pressures), 3]) * np.nan
    for i, p in enumerate(pressures):
        sols = []
        f = lambda r: kT * r + r ** 2 * eos.dfex_particle(r) - p
        for j in range(1, n_rough):
            if pg[j - 1] <= p <= pg[j]:
                sols.append(brentq(f, grid[j - 1], grid[j]))
        if sols:
            out[i, :len(sols)] = np.array(sorted(sols))
    return out


def eos_densities_from_chempots(eos, chempots, n_rough=1000):
    """cmmdft/eos.py:85-119."""
    grid = eos.rough_grid(n_rough)
    kT = boltzmann * eos.T
    mg = kT * np.log(eos.wvl ** 3 * grid) + eos.fex_particle(grid) + grid * eos.dfex_particle(grid)
    out = np.zeros([len(chempots), 2]) * np.nan
    for i, mu in enumerate(chempots):
        sols = []
        f = lambda r: kT * np.log(eos.wvl ** 3 * r) + eos.fex_particle(r) + r * eos.dfex_particle(r) - mu
        for j in range(1, n_rough):
            if mg[j - 1] <= mu <= mg[j]:
                sols.append(brentq(f, grid[j - 1], grid[j]))
        if sols:
            out[i, :len(sols)] = np.array(sorted(sols))
    return out


def eos_calculate_mu(eos, T, pressure):
    """eos.py:209-215."""
    eos.set_temperature(T)
    rho = eos_densities_from_pressures(eos, [pressure])[0][0]
    return eos_chempot(eos, rho)


# ------------------------------------------------------------ free energy -
class FreeEnergy(object):
    """The part list the solver sums over (cmmdft/functionals.py:25-174)."""

    def __init__(self, grid, temperature, wavelength, parts):
        self.grid = grid
        self.temperature = temperature
        self.beta = 1.0 / (boltzmann * temperature)
        self.wavelength = wavelength
        self.parts = parts
        self.part_names = [p.name for p in parts]
        self.part_dict = dict((p.name, p) for p in parts)


class NoSolutionError(Exception):
    pass


class Solver(object):
    """Fixed-point driver, cmmdft/solver.py:18-345 (criteria RES/RIUE/DER)."""
    name = 'SOLVER'

    def __init__(self, fener, nsteps=500, threshold=1e-6, criterion='RIUE', min_iter=1, a_tol=1e-6, r_tol=1e-4):
        self.grid = fener.grid
        self.fener = fener
        self.nsteps = nsteps
        crit = criterion if isinstance(criterion, list) else [criterion]
        thr = threshold if isinstance(threshold, list) else [threshold] * len(crit)
        if not isinstance(criterion, list) and criterion.lower() == 'der':
            thr = [1]  # solver.py:72-73
        self.criterion = [c.lower() for c in crit]
        self.threshold = thr
        self.a_tol, self.r_tol = a_tol, r_tol
        self.lower_density = 1e-12
        self.iphase = 0
        self.curr_step = 0
        self.correction_factor = 1
        self.omega_calls = 0

    def _initiate_solving(self, chempot):  # solver.py:90-101
        f = self.fener
        self.fugacity = np.exp(f.beta * chempot) / f.beta / f.wavelength ** 3
        self.chempot = chempot
        self.curr_step = 0
        self.omega0 = None

    def get_new_rho(self, C1, fugacity):  # solver.py:128-129
        return self.fener.beta * np.exp(-self.fener.beta * C1) * fugacity

    def _clip_density(self, rho):  # solver.py:146-148
        return np.where(rho < self.lower_density, 1e-30, rho)

    def _get_C1(self, rho, krho=None):  # solver.py:137-144
        if krho is None:
            krho = self.grid.fft(rho)
        C1 = np.zeros(self.grid.npoints)
        for p in self.fener.parts:
            C1 += p.derive(krho)
        return C1

    def _get_Omega(self, rho, krho):  # solver.py:103-119
        self.omega_calls += 1
        N = self.grid.integrate(rho)
        rr = self._clip_density(rho)
        Fid = self.grid.integrate(rr * (np.log(self.fener.wavelength ** 3 * rr) - 1.0)).real / self.fener.beta
        G = Fid - self.chempot * N
        for p in self.fener.parts:
            G += p.value(krho)
        self.omega0 = G
        return G

    def _get_alpha_max(self, rho, krho, Grho):  # solver.py:150-165
        krho_new = self.grid.fft(Grho)
        hs = self.fener.part_dict['HardSphere']
        a = np.max(hs.get_n3(krho)).real
        b = np.max(hs.get_n3(krho_new)).real
        return np.min([abs((1 - a) / ((b - a) + 1e-16)), 1])

    def _check_convergence(self, rho_new, C1_new, rho, N_new):  # solver.py:167-234
        ok = True
        self.IUE = self.grid.integrate(np.abs(rho_new - rho)).real
        self.RIUE = np.nan
        self.RES = np.nan
        if N_new > 0:
            self.RIUE = self.IUE / N_new
        for c, t in zip(self.criterion, self.threshold):
            if c == 'riue':
                v = self.RIUE
            elif c == 'res':
                G = self.get_new_rho(C1_new, self.fugacity)
                self.RES = np.linalg.norm(G - rho_new) / np.sqrt(N_new) / np.sqrt(np.prod(self.grid.npoints))
                v = self.RES
            elif c == 'der':  # solver.py:200-205 with _get_dOmega :131-135
                beta = self.fener.beta
                rr = self._clip_density(rho_new)
                dO = np.log(self.fener.wavelength ** 3 * rr) / beta + C1_new - self.chempot
                keep = ~np.isclose(rho_new, 0)
                w = np.abs(rho_new) * beta * dO / (self.a_tol + self.r_tol * np.abs(rho_new))
                self.DER = np.linalg.norm(w[keep]) / np.sqrt(np.prod(self.grid.npoints))
                v = self.DER
            else:
                raise NotImplementedError(c)
            ok *= (v < t)
        if self.IUE == 0 and np.isnan(self.RIUE):
            ok = True
        return bool(ok)

    def _solve(self, chempot, rho):  # solver.py:236-315
        self._initiate_solving(chempot)
        krho = self.grid.fft(rho)
        C1 = self._get_C1(rho, krho)
        self.omega0 = self._get_Omega(rho, krho)
        converged = False
        self.history = []
        for istep in range(self.nsteps):
            self.curr_step = istep + 1
            rho_new, krho_new, C1_new = self.update_rho(rho, krho, C1)
            if not np.all(np.isfinite(rho_new)):
                raise FloatingPointError
            N_new = self.grid.integrate(rho_new).real
            if self._check_convergence(rho_new, C1_new, rho, N_new):
                converged = True
                self.history.append((N_new, self.RES, self.RIUE))
                break
            self.history.append((N_new, self.RES, self.RIUE))
            rho, C1, krho = rho_new.copy(), C1_new.copy(), krho_new.copy()
        return N_new, rho_new, converged

    def solve(self, chempot, rho):  # solver.py:317-345
        self.correction_factor = 1
        while self.correction_factor >= 1 / 4:
            try:
                return self._solve(chempot, rho)
            except FloatingPointError:
                self.correction_factor /= 2
                self.iphase += 1
        self.correction_factor = 1
        raise NoSolutionError('not converged')


class Picard(Solver):
    """cmmdft/solver.py:348-457."""
    name = 'PICARD'

    def __init__(self, fener, nsteps=500, alpha_mix=0.1, method='hybrid', **kw):
        Solver.__init__(self, fener, nsteps, **kw)
        self.alpha_mix = alpha_mix
        self.thresh = 1 * kjmol
        self.update_rho = self.update_rho_hybrid if method == 'hybrid' else self.update_rho_static

    def update_rho_static(self, rho, krho, C1):  # solver.py:392-401
        G = self.get_new_rho(C1, self.fugacity)
        a = self.alpha_mix * self.correction_factor
        rho_new = (1.0 - a) * rho + a * G
        rho_new[rho_new < 1e-10 / angstrom ** 3] = 0.0
        k = self.grid.fft(rho_new)
        return rho_new, k, self._get_C1(rho_new, k)

    def update_rho_hybrid(self, rho, krho, C1):  # solver.py:403-457
        prev = self.omega0
        G = self.get_new_rho(C1, self.fugacity)
        amax = self._get_alpha_max(rho, krho, G)
        if np.isclose(amax, 0):
            aopt = 0
            mn = mx = 0
        else:
            a1 = 0.45 * amax
            r1 = (1 - a1) * rho + a1 * G
            o1 = self._get_Omega(r1, self.grid.fft(r1))
            a2 = 0.9 * amax if o1 <= prev else 0.225 * amax
            r2 = (1 - a2) * rho + a2 * G
            o2 = self._get_Omega(r2, self.grid.fft(r2))
            c, b, a = np.polyfit([0, a1, a2], [prev, o1, o2], 2)
            al = np.linspace(-max(a1, a2) / 4, max(a1, a2), 10000)
            om = a + b * al + c * al ** 2
            aopt = al[np.where(om == np.min(om))[0][0]]
            mn = np.min(om) / kjmol
            mx = np.max(om) / kjmol
        if aopt <= 0:
            if mx - mn > self.thresh:
                def fun(alpha):
                    rt = (1 - alpha) * rho + alpha * G
                    return self._get_Omega(rt, self.grid.fft(rt))
                bnd = opt.Bounds(0.01 * amax, 0.9 * amax)
                aopt = opt.minimize(fun, [self.alpha_mix * amax], bounds=bnd, method='SLSQP',
                                    options={'ftol': 1e-8}).x
            else:
                aopt = self.alpha_mix * amax
        if aopt <= 0 or np.isclose(aopt, 0):
            aopt = self.alpha_mix * amax
        rho_new = (1 - aopt * self.correction_factor) * rho + aopt * self.correction_factor * G
        rho_new = self._clip_density(rho_new)
        k = self.grid.fft(rho_new)
        C1n = self._get_C1(rho_new, k)
        self._get_Omega(rho_new, k)
        return rho_new, k, C1n


class Anderson(Picard):
    """cmmdft/solver.py:459-604 (SLSQP-constrained mixing coefficients)."""
    name = 'ANDERSON'

    def __init__(self, fener, nsteps=500, method='hybridanderson', m=5, damping=0.3, delta=0.2,
                 damping_max=0.8, damping_min=0.01, adaptive_damping=True,
                 damping_factors=(1.5, 0.5), alpha_mix=0.1, **kw):
        Picard.__init__(self, fener, nsteps, alpha_mix=alpha_mix, method='hybrid', **kw)
        self.Anderson_method = method
        self.m = m
        self.damping = self.original_damping = damping
        self.damping_max, self.damping_min = damping_max, damping_min
        self.adaptive_damping = adaptive_damping
        self.damping_factors = damping_factors
        self.delta = delta
        self.update_rho = self.update_rho_anderson_driver

    def _initiate_solving(self, chempot):  # solver.py:518-525
        Picard._initiate_solving(self, chempot)
        n = int(np.prod(self.grid.npoints))
        self.prev_rhos = np.zeros((self.m, n))
        self.prev_Grhos = np.zeros((self.m, n))
        self.And_true = False
        self.it_eps0 = np.nan
        self.damping = self.original_damping

    def _save(self, rho, G):  # solver.py:527-535
        self.prev_rhos = np.roll(self.prev_rhos, -1, axis=0)
        self.prev_rhos[-1] = rho.ravel()
        self.prev_Grhos = np.roll(self.prev_Grhos, -1, axis=0)
        self.prev_Grhos[-1] = G.ravel()

    def _damping(self):  # solver.py:537-544
        r = np.linalg.norm(self.prev_Grhos[-1] - self.prev_rhos[-1])
        p = np.linalg.norm(self.prev_Grhos[-2] - self.prev_rhos[-2])
        if r < p:
            self.damping = min(self.damping * self.damping_factors[0], self.damping_max)
        else:
            self.damping = max(self.damping * self.damping_factors[1], self.damping_min)

    def update_rho_anderson_driver(self, rho, krho, C1):  # solver.py:546-579
        prev = self.omega0
        G = self.get_new_rho(C1, self.fugacity)
        res = np.linalg.norm(G - rho)
        self._save(rho, G)
        self.it_eps = res / self.grid.integrate(rho)
        if self.curr_step < 3:
            self.it_eps0 = self.it_eps
        cond = ('hybrid' not in self.Anderson_method.lower()) or \
               ((self.it_eps <= self.it_eps0 * self.delta) and self.curr_step > 4) or self.And_true
        if cond:
            rho_new, k, C1n = self.update_rho_Anderson()
            Gn = self.get_new_rho(C1n, self.fugacity)
            self.And_true = True
            if np.isinf(Gn).any() or np.isnan(Gn).any():
                return self.update_rho_hybrid(rho, krho, C1)
            On = self._get_Omega(rho_new, k)
            if On > prev * 0.8:
                return self.update_rho_hybrid(rho, krho, C1)
            return rho_new, k, C1n
        return self.update_rho_hybrid(rho, krho, C1)

    def anderson_coefficients(self, residuals):  # solver.py:582-591
        mk = len(residuals)

        def f(a):
            return np.linalg.norm(np.einsum('i,ij->j', a, residuals))
        return opt.minimize(f, np.full(mk, 1 / mk), method='SLSQP', tol=1e-10,
                            bounds=opt.Bounds(0, 1),
                            constraints=opt.LinearConstraint(np.ones(mk), 1, 1)).x

    def update_rho_Anderson(self):  # solver.py:581-604
        mk = min(self.curr_step, self.m)
        R = self.prev_Grhos[-mk:] - self.prev_rhos[-mk:]
        al = self.anderson_coefficients(R)
        rr = np.einsum('i,ij->j', al, self.prev_rhos[-mk:]).reshape(self.grid.npoints)
        gr = np.einsum('i,ij->j', al, self.prev_Grhos[-mk:]).reshape(self.grid.npoints)
        if self.adaptive_damping:
            self._damping()
        d = self.correction_factor * self.damping
        rho_new = self._clip_density((1 - d) * rr + d * gr)
        k = self.grid.fft(rho_new)
        return rho_new, k, self._get_C1(rho_new, k)


# ------------------------------------------------------------ builders ----
def build_functional(grid, sigma, epsilon, mass, temperature, V, hs_version='WBII',
                     mfa_cutoff=12 * angstrom, tailcorrections=False):
    """WBII + MFA + ExtPot in the order of cmmdft/functionals.py:283-337 / 176-254."""
    R = hardsphere_radius(sigma, epsilon, temperature)
    lam = thermal_wavelength(mass, temperature)
    parts = [HardSphere(grid, R, temperature, hs_version),
             MFA(grid, sigma, epsilon, cutoff=mfa_cutoff, tailcorrections=tailcorrections),
             ExtPot(grid, V)]
    return FreeEnergy(grid, temperature, lam, parts)


def initial_density(fener, chempot):
    """Ideal gas in the external potential, cmmdft/program.py:296-305."""
    V = fener.part_dict['ExtPot'].potential
    return np.exp(fener.beta * (chempot - V)) / fener.wavelength ** 3


def helium_void_fraction(grid, host_pos, ff, ffatypes, ffatype_ids, rvecs, temperature,
                         he_sigma, he_eps, cutoff=12 * angstrom):
    """He void fraction (intent of cmmdft/calculator.py:152-167)."""
    pts = grid.points[..., :3].reshape(-1, 3)
    V = external_potential(pts, ff, he_sigma, he_eps, host_pos, ffatypes, ffatype_ids, rvecs,
                           cutoff)
    e = np.clip(np.exp(-V / boltzmann / temperature), 0, 1)
    return grid.integrate(e).real / grid.volume
