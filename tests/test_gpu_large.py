"""The large-cell WDA workload against the oracle: the a = 64 A cubic host
(14,680 atoms), 256^3 FP64, WBII + MFA + the WDA correlation part + LJ
external potential (the staged plane passes: a 256 x 256 plane of 6 fields
does not fit in shared memory).

The oracle cannot afford the whole solve at this size (its external
potential alone takes hours, one functional derivative a minute), so it
receives the GPU's external potential (checked separately at 4096 points in
test_gpu_parity.py) and runs static Picard steps from Ninit = rho_bulk at
1 bar: one step on the 256^3 grid of the workload, two on a 128^3 grid of
the same host (also staged).  Tolerances: the grand potential of the start
density 1e-11 relative; the density after the steps 1e-10 relative to its
maximum; N 1e-10.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from cmmdft_b200 import batch as BT, workload as W
from cmmdft_b200.hosts import cubic_host_64, methane_guest_params
from cmmdft_b200.units import bar
from tests._common import relerr, scalar_rel


@pytest.mark.parametrize("n,steps", [(128, 2), (256, 1)])
def test_large_wda_picard_steps(n, steps):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from oracle import cmm_oracle as O
    host = cubic_host_64()
    sig, eps, mass = guest = methane_guest_params()
    T = 300.0
    fn = W.build_functional(host, (n, n, n), T, guest, wda=True)
    mus, bulks = W.isotherm_inputs([1.0 * bar], T, guest)
    r0 = W.initial_density(fn, mus, ninit=bulks)
    s = BT.NativeBatchSolve(fn, mus, method='static', nsteps=steps, threshold=1e-30, criterion='res')
    N, rho, conv = s.solve(r0)
    rho_gpu = rho[0].cpu().numpy()
    om_gpu = float(s.omega0[0])
    V = fn.V.cpu().numpy()
    r0n = r0[0].cpu().numpy()
    del rho, r0, s
    grid = O.OGrid(host.rvecs, npoints=n)
    fe = O.build_functional(grid, sig, eps, mass, T, V)
    O.add_wda(fe, sig, eps, mass, T)
    op = O.Picard(fe, nsteps=steps, alpha_mix=0.1, method='static', criterion='res', threshold=1e-30)
    No, rho_o, _ = op.solve(float(mus[0]), r0n.copy())
    e_rho = relerr(rho_gpu, rho_o)
    e_om = scalar_rel(om_gpu, op.omega0)
    e_N = scalar_rel(N[0], No)
    print("%d^3 WDA, %d static Picard step(s) vs the oracle: rho %.2e, N %.2e, Omega(start) %.2e"
          % (n, steps, e_rho, e_N, e_om))
    assert e_rho < 1e-10 and e_N < 1e-10
    assert e_om < 1e-11
