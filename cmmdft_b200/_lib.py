"""ctypes binding of libcmmdft_b200.so (the C ABI declared in include/cmmdft_b200.h).

The product path has no CPU fallback: importing this module on a machine
without the built library, or calling a kernel without a CUDA device, raises.
"""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libcmmdft_b200.so")

# cmm_stat_* slots (include/cmmdft_b200.h)
STAT_N, STAT_IUE, STAT_NONFIN, STAT_FID, STAT_FEXT, STAT_RES2, STAT_PHI, STAT_MFA, \
    STAT_N3MAX, STAT_GNONFIN, STAT_GRAM0 = range(11)
STAT_WDA, STAT_DER = 18, 19
NSTAT = 20
# hybrid line-search sums (cmm_ls_*)
LS_MFA_RR, LS_MFA_XR, LS_N3MAX_G, LS_SUM_R, LS_SUM_RV, LS_FID, LS_PHI, LS_WDA, NLS = 0, 1, 2, 3, 4, 5, 8, 11, 16
MAX_HIST = 8
MAX_FIELDS = 12
FMT, MFMT, WBII, ANTISYM, NOHS, WDA, TENSOR = 0, 1, 2, 8, 16, 32, 64


class WdaEos(ctypes.Structure):
    """cmm_wda_eos of include/cmmdft_b200.h."""
    _fields_ = [("D", ctypes.c_double), ("sigma3", ctypes.c_double), ("epsilon", ctypes.c_double),
                ("gamma", ctypes.c_double), ("a", ctypes.c_double * 8), ("b", ctypes.c_double * 6),
                ("eta", ctypes.c_double), ("kT", ctypes.c_double), ("a_mfa", ctypes.c_double),
                ("factors", ctypes.c_double * 3)]
CLIP_NONE, CLIP_PICARD, CLIP_DENSITY = 0, 1, 2
SOLVE_HYBRID, SOLVE_ANDERSON, SOLVE_HYBRIDANDERSON, SOLVE_STATIC = 1, 2, 3, 4
CRIT_RES, CRIT_RIUE, CRIT_DER = 0, 1, 2
COEF_SLSQP, COEF_EXACT = 0, 1
BICG_RHO, BICG_ALPHA, BICG_OMEGA, BICG_BETA, BICG_D0, BICG_D1, BICG_RR, BICG_FIRST, BICG_NS = range(9)

_vp, _d, _i = ctypes.c_void_p, ctypes.c_double, ctypes.c_int


class FunctionalDesc(ctypes.Structure):
    """cmm_functional_desc."""
    _fields_ = [("grid", _vp), ("R", _d), ("beta", _d), ("lambda3", _d), ("version", _i), ("wda", _vp),
                ("d_kst", _vp), ("d_wtab", _vp), ("d_V", _vp)]


class SolveOpts(ctypes.Structure):
    """cmm_solve_opts."""
    _fields_ = [("method", _i), ("nsteps", _i), ("m", _i), ("ncrit", _i), ("crit", _i * 3), ("thr", _d * 3),
                ("alpha_mix", _d), ("damping", _d), ("delta", _d), ("damping_max", _d), ("damping_min", _d),
                ("damping_up", _d), ("damping_down", _d), ("adaptive_damping", _i), ("divergence_guard", _i),
                ("a_tol", _d), ("r_tol", _d), ("ls_thresh", _d), ("kjmol", _d), ("coefs", _i),
                ("picard_thr", _d), ("device_loop", _i)]


class SolveWs(ctypes.Structure):
    """cmm_solve_ws."""
    _fields_ = [(n, _vp) for n in ("ring", "rres", "trial", "rho0", "result", "spec_ring", "wd_ring", "wd_r", "rhat",
                                   "chat", "chat2", "that", "work", "part", "stats", "params", "coef", "active",
                                   "ls_part", "ls", "ls_alpha")] + \
               [("nslot", _i), ("h_stats", _vp), ("h_ls", _vp), ("h_alpha", _vp), ("h_stage", _vp),
                ("h_result", _vp)]


class SolveOut(ctypes.Structure):
    """cmm_solve_out."""
    _fields_ = [(n, _vp) for n in ("N", "omega", "converged", "steps", "diverged", "failed", "history")] + \
               [("launches", ctypes.c_longlong), ("omega_evals", ctypes.c_longlong), ("pipe_log", _vp),
                ("pipe_cap", _i), ("pipe_n", _i), ("cf", _vp)]


FALLBACK_FN = ctypes.CFUNCTYPE(ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                               ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double))


class CmmError(RuntimeError):
    """A cmm_* entry point returned a non-zero status."""


_lib = None

c_int, c_double, c_void_p, c_ll = ctypes.c_int, ctypes.c_double, ctypes.c_void_p, ctypes.c_longlong
P = ctypes.POINTER

_SIGS = {
    "cmm_version": ([], c_int),
    "cmm_status_string": ([c_int], ctypes.c_char_p),
    "cmm_grid_create": ([c_int, c_int, c_int, P(c_double), P(c_void_p)], c_int),
    "cmm_grid_destroy": ([c_void_p], c_int),
    "cmm_grid_create_sched": ([c_int, c_int, c_int, P(c_double), P(c_int), P(c_void_p)], c_int),
    "cmm_grid_schedule": ([c_void_p, P(c_int), P(c_int)], c_int),
    "cmm_grid_set_staging": ([c_void_p, c_int], c_int),
    "cmm_part_slots": ([c_void_p], c_int),
    "cmm_grid_spectrum_size": ([c_void_p, P(c_ll), P(c_int)], c_int),
    "cmm_spectrum_index": ([c_void_p, P(c_int), P(c_int), P(c_int)], c_int),
    "cmm_plane_smem_bytes": ([c_void_p, c_int, P(ctypes.c_size_t)], c_int),
    "cmm_extpot_lj": ([c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, c_double, c_double,
                       c_double, c_double, c_void_p, c_void_p], c_int),
    "cmm_extpot_set_mode": ([c_int], c_int),
    "cmm_extpot_rot": ([c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, P(c_double), P(c_double),
                        P(c_double), P(c_double), c_int, c_void_p, c_void_p, c_int, c_double, c_double, c_double,
                        c_void_p, c_void_p], c_int),
    "cmm_extpot_lj_deriv": ([P(c_double), c_int, c_int, c_int, P(c_double), c_void_p, c_void_p, c_int, c_void_p,
                             c_void_p, c_int, c_double, c_double, c_double, c_double, c_void_p, c_void_p], c_int),
    "cmm_extpot_rot_interp": ([c_void_p, c_void_p, c_int, P(c_int), P(c_double), P(c_double), P(c_double),
                               P(c_double), P(c_int), c_int, c_void_p, c_void_p, c_int, c_double, c_double, c_void_p,
                               c_void_p], c_int),
    "cmm_rfft3d": ([c_void_p, c_int, c_void_p, c_void_p, c_void_p], c_int),
    "cmm_irfft3d": ([c_void_p, c_int, c_void_p, c_void_p, c_void_p], c_int),
    "cmm_rfft_yz": ([c_void_p, c_int, c_void_p, c_void_p, c_void_p], c_int),
    "cmm_irfft_yz": ([c_void_p, c_int, c_void_p, c_void_p, c_void_p], c_int),
    "cmm_mfa_kernel": ([c_void_p, c_double, c_double, c_double, c_double, c_double, c_int, c_void_p,
                        c_void_p, P(ctypes.c_size_t), P(c_double), c_void_p], c_int),
    "cmm_fmt_c1": ([c_void_p, c_int, c_void_p, c_double, c_double, c_int, c_void_p, c_void_p, c_void_p,
                    c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_int, c_void_p, c_void_p], c_int),
    "cmm_ls_prepare": ([c_void_p, c_int, c_void_p, c_double, c_int, c_void_p, c_void_p, c_void_p, c_void_p,
                        c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p], c_int),
    "cmm_ls_omega": ([c_void_p, c_int, c_void_p, c_void_p, c_ll, c_double, c_double, c_double, c_double, c_double,
                      c_int, c_void_p, c_void_p, c_void_p, c_void_p, c_ll, c_void_p, c_void_p, c_void_p, c_int,
                      c_void_p, c_void_p], c_int),
    "cmm_ls_finalize": ([c_int, c_void_p, c_void_p, c_int, c_void_p, c_void_p], c_int),
    "cmm_solve_stage_bytes": ([c_int], ctypes.c_size_t),
    "cmm_anderson_slsqp": ([P(c_double), c_int, P(c_double), P(c_int), P(c_int)], c_int),
    "cmm_fmt_hvp": ([c_void_p, c_int, c_void_p, c_double, c_double, c_int, c_void_p, c_int, c_void_p, c_void_p,
                     c_void_p, c_void_p, c_void_p, c_void_p, c_void_p], c_int),
    "cmm_extpot_lj_grad": ([c_void_p, c_void_p, c_void_p, c_int, c_void_p, c_void_p, c_int, c_double, c_double,
                            c_double, c_double, c_void_p, c_void_p], c_int),
    "cmm_contract": ([c_void_p, c_ll, c_int, c_void_p, c_ll, c_int, c_ll, c_void_p, c_int, c_void_p], c_int),
    "cmm_bicg_vec": ([c_int, c_ll, c_int, c_void_p, c_void_p, c_void_p, c_double, c_void_p, c_void_p, c_void_p,
                      c_void_p, c_void_p, c_void_p, c_void_p, c_int, c_void_p], c_int),
    "cmm_bicg_scalars": ([c_int, c_void_p, c_void_p, c_int, c_void_p, c_int, c_void_p], c_int),
    "cmm_solve_batched": ([P(FunctionalDesc), P(SolveOpts), c_int, c_void_p, c_void_p, c_void_p, P(SolveWs),
                           P(SolveOut), FALLBACK_FN, c_void_p, c_void_p], c_int),
    "cmm_fmt_weights": ([c_void_p, c_double, c_void_p, c_void_p], c_int),
    "cmm_picard_static_step": ([c_void_p, c_int, c_void_p, c_void_p, c_double, c_double, c_double, c_double,
                                c_double, c_void_p,
                                c_void_p, c_void_p, c_ll, c_void_p, c_void_p, c_void_p, c_int, c_void_p], c_int),
    "cmm_residual_step": ([c_void_p, c_int, c_void_p, c_void_p, c_double, c_double, c_double, c_double, c_void_p, c_void_p, c_void_p,
                           c_ll, c_void_p, P(c_void_p), c_int, c_ll, c_void_p, c_int, c_void_p], c_int),
    "cmm_mix_step": ([c_void_p, c_int, c_void_p, c_void_p, P(c_void_p), P(c_ll), c_int, c_int, c_double,
                      c_double, c_void_p, c_ll, c_void_p, c_ll, c_void_p, c_void_p, c_void_p, c_int,
                      c_void_p], c_int),
    "cmm_fmt_c1_noalloc_capacity": ([c_void_p], ctypes.c_size_t),
    "cmm_fmt_c1_noalloc": ([c_void_p, c_int, c_void_p, c_double, c_double, c_int, c_void_p, c_void_p, c_void_p,
                            c_void_p, c_void_p, c_void_p, c_int, c_void_p], c_int),
    "cmm_stats_finalize": ([c_int, c_void_p, c_void_p, c_int, ctypes.c_uint, c_void_p, c_void_p], c_int),
}


def lib():
    """Load the library (once) and declare every exported signature."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise CmmError("%s is missing: build it with `python -m cmmdft_b200.build` "
                       "(there is no CPU fallback)" % LIB_PATH)
    L = ctypes.CDLL(LIB_PATH)
    for name, (args, res) in _SIGS.items():
        fn = getattr(L, name)
        fn.argtypes = args
        fn.restype = res
    _lib = L
    return L


def exported_symbols():
    return list(_SIGS)


def check(rc, what=""):
    if rc != 0:
        msg = lib().cmm_status_string(rc).decode()
        raise CmmError("%s failed: %s (status %d)" % (what or "cmm call", msg, rc))


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())
