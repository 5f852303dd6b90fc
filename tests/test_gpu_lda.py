"""The LDA part (LDAFunctional, cmmdft/functionals.py:1085-1114) through the
drop-in API against the unmodified reference (tests/golden/lda32.npz): the
32^3 case with WBII + MFA + ExtPot + LDA of SumOfEOS([MBWR, CS, MFA],
[1, -1, -1]).  The GPU evaluates it inside the fused pipeline as the WDA
machinery with weight 1.  Tolerances as the other C1 checks: beta |dC1| at
the reference's WBII noise floor (2e-9 ideal gas, 1e-7 dense), the LDA
derivative alone 1e-12 relative, free-energy parts and Omega 1e-11, three
static Picard steps 1e-10 (N) and max(1e-10, 3 x the reference's own floor on
that trajectory) for rho."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

import cmmdft_b200 as cd
from cmmdft_b200 import batch as BT, engine as E, _lib as L
from cmmdft_b200.hosts import cubic_host_276, methane_guest_params
from cmmdft_b200.units import angstrom
from tests._common import relerr, scalar_rel

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _program(tmp_path):
    h = cubic_host_276(0)
    host = cd.NanoporousHost('synthetic', pos=h.pos, ffatypes=h.ffatypes, ffatype_ids=h.ffatype_ids,
                             rvecs=h.rvecs, ff=h.ff)
    sig, eps, mass = methane_guest_params()
    guest = cd.SphericalLJGuest('CH4', mass, sig, eps)
    prog = cd.Program(prefix=str(tmp_path), hostname='synthetic', guestname='CH4')
    prog.set_system(host, guest)
    prog.set_grid(npoints=32)
    prog.init_free_energy(300.0)
    prog.fener.add_hard_sphere(version='WBII')
    prog.fener.add_mean_field(cutoff=12 * angstrom)
    prog.fener.add_external_potential(cutoff=12 * angstrom)
    prog.fener.set_temperature(300.0)
    a = prog.fener.part_dict['MFA'].compute_vdw_a()
    S = cd.SumOfEOS(mass, [cd.ModifiedBenedictWebbRubinEOS(mass, sig, eps), cd.CarnahanStarlingEOS(mass, guest.Rhs),
                           cd.MFAEOS(mass, sig, eps, a=a)], factors=[1, -1, -1])
    prog.fener.add_lda(S)
    return prog


def test_lda_part_against_reference(golden32, tmp_path):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    ref = dict(np.load(os.path.join(ROOT, "tests", "golden", "lda32.npz")))
    prog = _program(tmp_path)
    fe = prog.fener
    fn = fe.device()
    assert fn.wda is not None and fn.wda.D < 0
    plan = fn.plan
    mu = float(ref["mu"])
    for tag, floor in (('a', 2e-9), ('b', 1e-7)):
        rho = torch.as_tensor(golden32["rho_" + tag][None], device="cuda")
        buf = E.Buffers(plan, 1, nwork=fn.nwork)
        buf.part[:, L.STAT_N3MAX, :] = -np.inf
        chat = plan.new_spec(1)
        fn.c1(buf, plan.rfft_yz(rho), chat, want=3)
        E.finalize(buf, (1 << L.NSTAT) - 1)
        st = buf.stats.cpu().numpy()[0]
        C1 = plan.irfft_yz(chat)[0].cpu().numpy() + fn.V.cpu().numpy()
        beta = fn.beta
        err = np.abs(C1 - ref["C1_" + tag])
        at = np.unravel_index(int(np.argmax(err)), err.shape)
        assert beta * err[at] < floor, ("C1 error at", at, "rho", golden32["rho_" + tag][at], "V",
                                        float(fn.V[at].item()), "dLDA", ref["dLDA_" + tag][at], "a", fn.vdw_a,
                                        "eos", (fn.wda.eta, fn.wda.kT, fn.wda.a_mfa, fn.wda.sigma3, fn.wda.epsilon,
                                                list(fn.wda.factors)), "points above floor",
                                        int(np.sum(beta * err >= floor)))
        # the LDA part alone: the pipeline with and without it (same HS and MFA arithmetic)
        fh = E.Functional(plan, fn.R, fn.beta, fn.wavelength, fn.V, fn.version & ~L.WDA, fn.kst, fn.vdw_a)
        chat_h = plan.new_spec(1)
        fh.c1(E.Buffers(plan, 1, nwork=fh.nwork), plan.rfft_yz(rho), chat_h, want=1)
        d_lda = (plan.irfft_yz(chat)[0] - plan.irfft_yz(chat_h)[0]).cpu().numpy()
        e_d = relerr(d_lda, ref["dLDA_" + tag])
        F_lda = st[L.STAT_WDA] * plan.dr
        e_F = scalar_rel(F_lda, ref["values_" + tag][3])
        print("LDA profile %s: beta|dC1| %.2e, dF_LDA %.2e, F_LDA %.2e" % (tag, beta * np.max(np.abs(C1 - ref["C1_" + tag])),
                                                                      e_d, e_F))
        assert e_d < 1e-12 and e_F < 1e-11
    s = BT.NativeBatchSolve(fn, [mu], method='static', nsteps=3, threshold=1e-30, criterion='res')
    N, rho, conv = s.solve(torch.as_tensor(golden32["rho_a"][None], device="cuda"))
    # the target 1e-10, or three times the reference's own floor on this
    # trajectory (the same steps from a start one ulp above) where larger
    e_rho = relerr(rho[0].cpu().numpy(), ref["picard3_rho"])
    e_N = scalar_rel(N[0], ref["picard3_N"])
    print("LDA three static Picard steps: rho %.2e (floor %.2e), N %.2e" % (e_rho, ref["picard3_floor"], e_N))
    assert e_rho < max(1e-10, 3 * float(ref["picard3_floor"]))
    assert e_N < 1e-10
