"""ctypes binding of libnegf_b200.so (the C ABI declared in include/negf_b200.h).

The shared library is built in-tree by ``libnegf.jl_b200/build.py``.  There is
no CPU fallback: if the library is missing or no CUDA device is usable, the
first call raises.
"""

import ctypes
import os

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libnegf_b200.so")

NEGF_SUCCESS = 0
NEGF_ERR_INVALID = 1
NEGF_ERR_CUDA = 2
NEGF_ERR_SINGULAR = 3
NEGF_ERR_NOMEM = 4
NEGF_ERR_TIMEOUT = 5
NEGF_DDRGF_MAX_LEVELS = 6

c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_void_pp = ctypes.POINTER(ctypes.c_void_p)
c_double_p = ctypes.POINTER(ctypes.c_double)


class ZGemmProblem(ctypes.Structure):
    _fields_ = [("A", ctypes.c_void_p), ("B", ctypes.c_void_p), ("Cin", ctypes.c_void_p), ("C", ctypes.c_void_p),
                ("m", ctypes.c_int32), ("n", ctypes.c_int32), ("k", ctypes.c_int32),
                ("lda", ctypes.c_int32), ("ldb", ctypes.c_int32), ("ldc", ctypes.c_int32), ("ldcin", ctypes.c_int32),
                ("alpha", ctypes.c_double * 2), ("beta", ctypes.c_double * 2), ("diag", ctypes.c_double * 2)]


class SolveOpts(ctypes.Structure):
    _fields_ = [("eta", ctypes.c_double), ("mu_l", ctypes.c_double), ("mu_r", ctypes.c_double),
                ("kT", ctypes.c_double), ("want_gr", ctypes.c_int32), ("want_gl", ctypes.c_int32),
                ("want_t", ctypes.c_int32), ("max_chunk", ctypes.c_int32), ("hbm_budget_gb", ctypes.c_double),
                ("precision", ctypes.c_int32), ("gemm_form", ctypes.c_int32), ("gj_nb", ctypes.c_int32),
                ("sigma_per_energy", ctypes.c_int32), ("gj_update", ctypes.c_int32)]


NEGF_PREC_FP64 = 0
NEGF_PREC_MIXED = 1
NEGF_METHOD_RGF = 0
NEGF_METHOD_DDRGF = 1
NEGF_METHOD_SELINV = 2


class CCscMatrix(ctypes.Structure):
    _fields_ = [("m", ctypes.c_int32), ("n", ctypes.c_int32), ("nnz", ctypes.c_int32),
                ("colptr", c_int32_p), ("rowval", c_int32_p), ("nzval", ctypes.c_void_p)]


# exported symbol -> (restype, argtypes)
PROTOTYPES = {
    "negf_last_error": (ctypes.c_char_p, []),
    "negf_version": (ctypes.c_int, []),
    "negf_zgemm_batched": (ctypes.c_int, [ctypes.c_char, ctypes.c_char, ctypes.c_int32,
                                          ctypes.POINTER(ZGemmProblem), ctypes.c_void_p]),
    "negf_zgemm_batched_mixed": (ctypes.c_int, [ctypes.c_char, ctypes.c_char, ctypes.c_int32,
                                                ctypes.POINTER(ZGemmProblem), ctypes.c_void_p]),
    "negf_zcopy_batched": (ctypes.c_int, [ctypes.c_char, ctypes.c_int32, c_int32_p, c_int32_p, c_void_pp, c_int32_p,
                                          c_void_pp, c_int32_p, ctypes.c_void_p]),
    "negf_set_tensor_wait_limit": (ctypes.c_int, [ctypes.c_double]),
    "negf_zfill_batched": (ctypes.c_int, [ctypes.c_int32, c_int32_p, c_int32_p, c_void_pp, c_int32_p, c_double_p,
                                          ctypes.c_void_p]),
    "negf_zinv_batched": (ctypes.c_int, [ctypes.c_int32, c_int32_p, c_void_pp, c_int32_p, c_void_pp, c_int32_p,
                                         c_int32_p, ctypes.c_void_p]),
    "negf_zinv_batched_noalloc": (ctypes.c_int, [ctypes.c_int32, c_int32_p, c_void_pp, c_int32_p, c_void_pp,
                                                 c_int32_p, c_int32_p, ctypes.c_void_p]),
    "negf_zgetrf_batched": (ctypes.c_int, [ctypes.c_int32, c_int32_p, c_void_pp, c_int32_p, c_void_pp, c_int32_p,
                                           ctypes.c_void_p]),
    "negf_ztrsm_batched": (ctypes.c_int, [ctypes.c_char, ctypes.c_char, ctypes.c_char, ctypes.c_char, c_double_p,
                                          ctypes.c_int32, c_int32_p, c_int32_p, c_void_pp, c_int32_p, c_void_pp,
                                          c_int32_p, ctypes.c_void_p]),
    "negf_zgetri_nopiv_batched": (ctypes.c_int, [ctypes.c_int32, c_int32_p, c_void_pp, c_int32_p, ctypes.c_void_p]),
    "negf_rgf": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_int32_p, c_void_pp, c_void_pp, c_void_pp,
                                c_void_pp, c_void_pp, c_void_pp, c_void_pp, ctypes.c_void_p]),
    "negf_keldysh": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_int32_p, c_void_pp, c_void_pp, c_void_pp,
                                    c_void_pp, c_void_pp, ctypes.c_void_p]),
    "negf_general_rgf": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_void_pp,
                                        c_void_pp, ctypes.c_void_p]),
    "negf_selected_inverse": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_void_pp, ctypes.POINTER(ctypes.c_uint8),
                                             ctypes.c_int32, ctypes.c_void_p]),
    "negf_ddrgf": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_int32_p, c_void_pp, c_void_pp, c_void_pp,
                                  ctypes.c_int32, c_void_pp, c_void_pp, c_void_pp, ctypes.c_void_p]),
    "negf_selected_inverse_batched": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_void_pp,
                                                     ctypes.POINTER(ctypes.c_uint8), ctypes.c_int32, ctypes.c_int32,
                                                     ctypes.c_int32, ctypes.c_void_p]),
    "negf_ddrgf_levels_ex": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_int32_p, c_void_pp, c_void_pp,
                                            c_void_pp, ctypes.c_int32, c_int32_p, c_void_pp, c_void_pp, c_void_pp,
                                            ctypes.c_int32, ctypes.c_void_p]),
    "negf_device_selected_inverse": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, c_double_p,
                                                    ctypes.POINTER(SolveOpts), ctypes.c_int32, ctypes.c_int32,
                                                    c_int32_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                    ctypes.c_int32, ctypes.c_void_p]),
    "negf_ddrgf_get_nr_tasks": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p]),
    "negf_ddrgf_choose_d1": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_int32_p]),
    "negf_ddrgf_levels": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_int32_p, c_void_pp, c_void_pp, c_void_pp,
                                         ctypes.c_int32, c_int32_p, c_void_pp, c_void_pp, c_void_pp, ctypes.c_void_p]),
    "negf_ddrgf_choose_levels": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                                c_int32_p, c_int32_p]),
    "negf_server_create": (ctypes.c_int, [ctypes.POINTER(SolveOpts), ctypes.c_double, ctypes.POINTER(ctypes.c_void_p)]),
    "negf_server_create_ex": (ctypes.c_int, [ctypes.POINTER(SolveOpts), ctypes.c_double, ctypes.c_int32,
                                             ctypes.POINTER(ctypes.c_void_p)]),
    "negf_server_stats_ex": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64), c_int32_p, c_int32_p,
                                            c_double_p]),
    "negf_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, c_int32_p, c_void_pp, c_void_pp,
                                          ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, c_double_p,
                                          ctypes.c_void_p, ctypes.c_void_p, c_double_p,
                                          ctypes.POINTER(ctypes.c_int64)]),
    "negf_server_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, c_int32_p]),
    "negf_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64, ctypes.c_double, c_double_p]),
    "negf_server_stats": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64),
                                         ctypes.POINTER(ctypes.c_int64), c_double_p, c_double_p]),
    "negf_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "negf_server_group_sizes": (ctypes.c_int, [ctypes.c_int32, ctypes.POINTER(ctypes.c_int64), ctypes.c_double,
                                               c_int32_p, c_int32_p]),
    "negf_ddrgf_cost_rgf": (ctypes.c_int, [ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_int32,
                                           c_double_p]),
    "negf_ddrgf_cost_ddrgf": (ctypes.c_int, [ctypes.c_double, ctypes.c_double, ctypes.c_int32, ctypes.c_int32,
                                             ctypes.c_int32, c_double_p]),
    "negf_ddrgf_check_nr_threads": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p,
                                                   c_int32_p]),
    "negf_ddrgf_opt_params": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double,
                                             ctypes.c_double, c_int32_p, c_int32_p, c_int32_p, c_double_p]),
    "negf_device_create": (ctypes.c_int, [ctypes.c_int32, c_int32_p, c_void_pp, c_void_pp, ctypes.c_void_p,
                                          ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    "negf_device_upload": (ctypes.c_int, [ctypes.c_void_p, c_void_pp, c_void_pp, ctypes.c_void_p, ctypes.c_void_p]),
    "negf_device_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "negf_solve": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, c_double_p, ctypes.POINTER(SolveOpts),
                                  ctypes.c_void_p, ctypes.c_void_p, c_double_p, ctypes.c_int32, ctypes.c_void_p]),
    "negf_solver_create": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int32, ctypes.POINTER(SolveOpts),
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "negf_solver_create_batch": (ctypes.c_int, [ctypes.c_int32, c_void_pp, ctypes.POINTER(ctypes.c_int32),
                                                ctypes.POINTER(SolveOpts), c_void_pp]),
    "negf_batch_bytes": (ctypes.c_int, [ctypes.c_int32, c_void_pp, ctypes.POINTER(ctypes.c_int32),
                                        ctypes.POINTER(SolveOpts), ctypes.POINTER(ctypes.c_int64)]),
    "negf_solver_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "negf_device_set_overlap": (ctypes.c_int, [ctypes.c_void_p, c_void_pp, c_void_pp]),
    "negf_solver_set_self_energies": (ctypes.c_int, [ctypes.c_void_p, c_void_pp, c_void_pp, ctypes.c_void_p]),
    "negf_solver_set_energies": (ctypes.c_int, [ctypes.c_void_p, c_double_p, ctypes.c_void_p]),
    "negf_solver_run": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "negf_solver_outputs": (ctypes.c_int, [ctypes.c_void_p, c_void_pp, c_void_pp,
                                           ctypes.POINTER(ctypes.POINTER(ctypes.c_double))]),
    "negf_solver_check": (ctypes.c_int, [ctypes.c_void_p]),
    "negf_solver_download": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, c_double_p,
                                            ctypes.c_void_p]),
    "negf_solver_run_download": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, c_double_p,
                                            ctypes.c_void_p]),
    "negf_solver_run_profiled": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    "negf_solver_profile_read": (ctypes.c_int, [ctypes.c_void_p, c_double_p, c_double_p,
                                                ctypes.POINTER(ctypes.c_int64), ctypes.c_int32]),
    "negf_solver_stats": (ctypes.c_int, [ctypes.c_void_p, c_double_p, ctypes.POINTER(ctypes.c_int64),
                                         ctypes.POINTER(ctypes.c_int64)]),
    "negf_bndiag_of_inv_direct": (ctypes.c_int, [ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p,
                                                 ctypes.c_void_p, ctypes.c_int32, c_int32_p, ctypes.c_int32,
                                                 ctypes.POINTER(CCscMatrix)]),
    "run_bndiag_wrapper": (CCscMatrix, [ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, c_int32_p, c_int32_p,
                                        ctypes.c_void_p, ctypes.c_int32, c_int32_p, ctypes.c_int32,
                                        ctypes.POINTER(ctypes.c_char_p), c_int32_p, ctypes.c_int32]),
    "negf_probe_fp64_peak": (ctypes.c_int, [c_double_p, c_double_p]),
    "negf_probe_int8_peak": (ctypes.c_int, [c_double_p]),
    "negf_release_cached_memory": (ctypes.c_int, []),
    "negf_probe_fp64_int8_overlap": (ctypes.c_int, [c_double_p, c_double_p, c_double_p]),
}

_lib = None


class NegfError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("libnegf_b200 error %d: %s" % (code, msg))
        self.code = code


class SingularError(NegfError):
    pass


def load(path=None):
    """Load the shared library (once) and declare its prototypes."""
    global _lib
    if _lib is not None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError("libnegf_b200.so not found at %s; build it with libnegf.jl_b200/build.py" % p)
    lib = ctypes.CDLL(p)
    for name, (res, args) in PROTOTYPES.items():
        f = getattr(lib, name, None)
        if f is None:
            MISSING.append(name)
            continue
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


MISSING = []


def check(rc):
    if rc != NEGF_SUCCESS:
        msg = load().negf_last_error().decode()
        if rc == NEGF_ERR_SINGULAR:
            raise SingularError(rc, msg)
        raise NegfError(rc, msg)


def ptr_array(ptrs):
    arr = (ctypes.c_void_p * max(1, len(ptrs)))()
    for i, p in enumerate(ptrs):
        arr[i] = p
    return arr


def int_array(vals):
    arr = (ctypes.c_int32 * max(1, len(vals)))()
    for i, v in enumerate(vals):
        arr[i] = int(v)
    return arr
