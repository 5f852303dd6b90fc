"""The allocation-free functional pipeline against the allocating one.

cmm_fmt_c1_noalloc serves callers that cannot allocate device memory at the
point of evaluation (plugin hosts that forbid allocation in a callback,
fixed device-memory budgets, bindings that cannot own CUDA allocations); its
scratch is a static device array shared by all calls.  This file is
collected last so a failure here leaves every other test already run.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

from cmmdft_b200 import _lib as L, engine as E, workload as W
from cmmdft_b200.hosts import cubic_host_276, methane_guest_params


@pytest.fixture(scope="module")
def case(golden32):
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    fn = W.build_functional(cubic_host_276(0), (32, 32, 32), 300.0, methane_guest_params())
    rho = torch.as_tensor(np.stack([golden32["rho_b"], golden32["rho_a"]]), device="cuda")
    return fn, fn.plan.rfft_yz(rho)


def _stream():
    return ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)


def test_noalloc_matches_allocating_pipeline_twice(case):
    fn, spec = case
    plan, lib, B = fn.plan, L.lib(), spec.shape[0]
    assert lib.cmm_fmt_c1_noalloc_capacity(plan.handle) >= B
    # the allocating entry point, with caller-provided workspace
    buf = E.Buffers(plan, B)
    buf.part[:, L.STAT_N3MAX, :] = -np.inf
    chat_ref = plan.new_spec(B)
    fn.c1(buf, spec, chat_ref, want=7)
    E.finalize(buf, (1 << L.NSTAT) - 1)
    st_ref = buf.stats.cpu().numpy()
    ref = chat_ref.cpu().numpy()
    # two calls in a row of the allocation-free entry point
    for call in range(2):
        chat = plan.new_spec(B)
        stats = torch.full((B, L.NSTAT), np.nan, dtype=torch.float64, device="cuda")
        rc = lib.cmm_fmt_c1_noalloc(plan.handle, B, None, fn.R, fn.beta, fn.version, None, L.ptr(fn.kst),
                                    L.ptr(fn.wtab), L.ptr(spec), L.ptr(chat), L.ptr(stats), 7, _stream())
        assert rc == 0, lib.cmm_status_string(rc)
        got = chat.cpu().numpy()
        st = stats.cpu().numpy()
        assert np.max(np.abs(got - ref)) <= 1e-13 * np.max(np.abs(ref))
        for q in (L.STAT_PHI, L.STAT_MFA, L.STAT_N3MAX):
            assert np.allclose(st[:, q], st_ref[:, q], rtol=1e-13, atol=0)


def test_noalloc_rejects_batches_beyond_its_scratch(case):
    fn, spec = case
    lib = L.lib()
    cap = int(lib.cmm_fmt_c1_noalloc_capacity(fn.plan.handle))
    rc = lib.cmm_fmt_c1_noalloc(fn.plan.handle, cap + 1, None, fn.R, fn.beta, fn.version, None, L.ptr(fn.kst),
                                L.ptr(fn.wtab), L.ptr(spec), L.ptr(spec), L.ptr(spec), 1, _stream())
    assert rc == 6  # CMM_ERR_WORKSPACE, before any device work


def test_mfa_only_rejects_hard_sphere_outputs(case):
    """CMM_NOHS (the MFA convolution alone) has no hard-sphere sums: both
    entry points reject any want bit beyond the C1 spectrum with CMM_ERR_ARG
    before any device work, and accept want = 1."""
    fn, spec = case
    plan, lib, B = fn.plan, L.lib(), spec.shape[0]
    chat = plan.new_spec(B)
    stats = torch.zeros((B, L.NSTAT), dtype=torch.float64, device="cuda")
    buf = E.Buffers(plan, B)
    for want in (3, 5, 7):
        rc = lib.cmm_fmt_c1_noalloc(plan.handle, B, None, fn.R, fn.beta, L.NOHS, None, L.ptr(fn.kst), None,
                                    L.ptr(spec), L.ptr(chat), L.ptr(stats), want, _stream())
        assert rc == 1, (want, rc)   # CMM_ERR_ARG
        rc = lib.cmm_fmt_c1(plan.handle, B, None, fn.R, fn.beta, L.NOHS, None, L.ptr(fn.kst), None, L.ptr(spec),
                            L.ptr(chat), L.ptr(buf.work), L.ptr(buf.part), buf.nslot, want, None, _stream())
        assert rc == 1, (want, rc)
    rc = lib.cmm_fmt_c1_noalloc(plan.handle, B, None, fn.R, fn.beta, L.NOHS, None, L.ptr(fn.kst), None,
                                L.ptr(spec), L.ptr(chat), None, 1, _stream())
    assert rc == 0, lib.cmm_status_string(rc)
