"""ctypes binding of libnegfgpu.so (include/negf_gpu.h).

The library must have been built (``negftrans_b200.build.build()``); there is
no fallback: a missing library raises instead of computing anything on the
CPU.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "libnegfgpu.so")

NEGF_OK = 0
NEGF_ERR_ARG = -1
NEGF_ERR_CUDA = -2
NEGF_ERR_NOMEM = -3
NEGF_ERR_UNSUPPORTED = -4
NEGF_ERR_TOO_LARGE = -5
NEGF_FP64 = 0
NEGF_MIXED = 1

# every symbol include/negf_gpu.h declares
EXPORTS = (
    "negf_basis_size", "negf_basis", "negf_kmesh", "negf_vhat", "negf_ctx_create",
    "negf_ctx_destroy", "negf_tri_solve", "negf_transmission", "negf_transmission_device",
    "negf_density", "negf_ldos_matrix", "negf_ptor", "negf_version", "negf_transmission_noalloc",
    "negf_density_real", "negf_ldos", "negf_basis_k", "negf_transmission_batch",
    "negf_density_neq", "negf_dm_real", "negf_set_variant", "negf_autotune", "negf_vhat_gpu",
    "negf_density_accumulate", "negf_tc_product_check", "negf_tc_inverse_check",
    "negf_set_mixed_policy", "negf_get_mixed_policy", "negf_get_mixed_stats", "negf_dm_real_slab",
)
# every symbol include/negf_mlp.h declares
MLP_EXPORTS = (
    "negf_mlp_create", "negf_mlp_destroy", "negf_mlp_param_count", "negf_mlp_set_params",
    "negf_mlp_get_params", "negf_mlp_forward", "negf_mlp_grad", "negf_mlp_train",
)

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)


class Problem(C.Structure):
    _fields_ = [("N", C.c_int32), ("Nz", C.c_int32), ("ngx", C.c_int32), ("ngy", C.c_int32),
                ("nx", _ip), ("ny", _ip), ("vhat", _dp), ("Lx", C.c_double), ("Ly", C.c_double),
                ("Lz", C.c_double), ("V_L", C.c_double), ("V_R", C.c_double), ("eta", C.c_double),
                ("nk", C.c_int32), ("kpt", _dp), ("lead_model", C.c_int32)]


class MixedPolicy(C.Structure):
    _fields_ = [("threshold_window", C.c_double), ("eta_fp64_below", C.c_double), ("tau_tolerance", C.c_double),
                ("max_refinements", C.c_int32), ("ctas_per_job", C.c_int32)]


class MixedStats(C.Structure):
    _fields_ = [("n_jobs", C.c_int32), ("n_mixed", C.c_int32), ("n_fp64_policy", C.c_int32),
                ("n_fp64_rejected", C.c_int32), ("jobs_per_wave", C.c_int32), ("ctas_per_job", C.c_int32),
                ("max_correction", C.c_double), ("mixed_ms", C.c_double), ("fp64_ms", C.c_double)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Stats(C.Structure):
    _fields_ = [("n_jobs", C.c_int32), ("n_singular", C.c_int32), ("first_bad_job", C.c_int32),
                ("info", C.c_int32), ("device_ms", C.c_double)]


class NegfError(RuntimeError):
    def __init__(self, where, code):
        names = {NEGF_ERR_ARG: "invalid argument", NEGF_ERR_CUDA: "CUDA error",
                 NEGF_ERR_NOMEM: "out of device memory", NEGF_ERR_UNSUPPORTED: "unsupported",
                 NEGF_ERR_TOO_LARGE: "problem larger than the fixed scratch"}
        super().__init__(f"{where}: {names.get(code, code)} ({code})")
        self.code = code


_lib = None


def lib():
    """Load libnegfgpu.so; raises if it was not built."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(f"{LIB_PATH} is missing: build it with negftrans_b200.build.build()")
    L = C.CDLL(LIB_PATH)
    L.negf_version.restype = C.c_char_p
    L.negf_basis_size.argtypes = [C.c_double, C.c_double, C.c_double, _ip]
    L.negf_basis.argtypes = [C.c_double, C.c_double, C.c_double, C.c_int32, _ip, _ip]
    L.negf_kmesh.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double, _dp]
    L.negf_vhat.argtypes = [_dp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _dp]
    L.negf_ctx_create.argtypes = [C.POINTER(Problem), C.c_int32, C.POINTER(C.c_void_p)]
    L.negf_ctx_destroy.argtypes = [C.c_void_p]
    L.negf_tri_solve.argtypes = [C.c_void_p, _dp, C.c_int32, C.c_int32, C.c_char_p, _dp, _dp, _dp]
    L.negf_transmission.argtypes = [C.c_void_p, _dp, C.c_int32, C.c_int32, _dp, C.POINTER(Stats)]
    L.negf_transmission_device.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int32, C.c_void_p,
                                           C.c_void_p, C.c_void_p, C.c_void_p]
    L.negf_transmission_noalloc.argtypes = (
        [C.c_int32] * 4 + [C.c_void_p] * 3 + [C.c_double] * 6 + [C.c_int32] + [C.c_void_p] * 2
        + [C.c_int32] + [C.c_void_p] * 3)
    L.negf_density.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                               C.c_double, _dp, C.POINTER(Stats)]
    L.negf_ldos_matrix.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int32, C.c_int32,
                                   C.c_int32, _dp, C.POINTER(Stats)]
    L.negf_density_real.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_int32, C.c_int32, C.c_double, _dp, _dp,
                                    C.POINTER(Stats)]
    L.negf_ldos.argtypes = [C.c_void_p, C.c_double, C.c_double, C.c_int32, _ip, C.c_int32, C.c_int32, _dp,
                            C.c_double, _dp, C.POINTER(Stats)]
    L.negf_basis_k.argtypes = [C.c_double] * 5 + [C.c_int32, _ip, _ip, _ip]
    L.negf_transmission_batch.argtypes = [C.POINTER(C.c_void_p), C.c_int32, _dp, C.c_int32, _dp,
                                          C.POINTER(Stats)]
    L.negf_ptor.argtypes = [_dp, _ip, _ip, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _dp]
    L.negf_density_neq.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                                   C.c_double, C.c_double, _dp, C.POINTER(Stats)]
    L.negf_dm_real.argtypes = [C.c_void_p, _dp, C.c_int32, C.c_int32, C.c_double, _dp]
    L.negf_dm_real_slab.argtypes = [C.c_void_p, _dp, C.c_int32, C.c_int32, C.c_int32, C.c_double, _dp]
    L.negf_set_variant.argtypes = [C.c_void_p, C.c_int32]
    L.negf_density_accumulate.argtypes = [C.c_void_p, _dp, _dp, C.c_int32, _dp, C.POINTER(Stats)]
    L.negf_vhat_gpu.argtypes = [_dp, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_int32, _dp]
    L.negf_autotune.argtypes = [C.c_void_p, _dp, C.c_int32, _ip, _dp]
    L.negf_tc_product_check.argtypes = [C.c_void_p, C.c_int32, C.c_void_p, C.c_int32, C.c_void_p, C.c_void_p,
                                        C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_void_p]
    L.negf_tc_inverse_check.argtypes = [C.c_void_p, C.c_int32, C.c_int32, C.c_void_p, C.c_void_p, C.c_void_p]
    L.negf_set_mixed_policy.argtypes = [C.c_void_p, C.POINTER(MixedPolicy)]
    L.negf_get_mixed_policy.argtypes = [C.c_void_p, C.POINTER(MixedPolicy)]
    L.negf_get_mixed_stats.argtypes = [C.c_void_p, C.POINTER(MixedStats)]
    _fp = C.POINTER(C.c_float)
    L.negf_mlp_create.argtypes = [C.c_int32, _ip, C.c_int32, C.c_int32, C.POINTER(C.c_void_p)]
    L.negf_mlp_destroy.argtypes = [C.c_void_p]
    L.negf_mlp_param_count.argtypes = [C.c_void_p]
    L.negf_mlp_param_count.restype = C.c_int64
    L.negf_mlp_set_params.argtypes = [C.c_void_p, _fp]
    L.negf_mlp_get_params.argtypes = [C.c_void_p, _fp]
    L.negf_mlp_forward.argtypes = [C.c_void_p, _fp, C.c_int32, _fp]
    L.negf_mlp_grad.argtypes = [C.c_void_p, _fp, _fp, _fp, C.c_int32, _dp, _fp]
    L.negf_mlp_train.argtypes = [C.c_void_p, _fp, _fp, _fp, C.c_int64, C.c_int32, C.c_int32, C.c_float,
                                 C.c_uint64, _dp]
    _lib = L
    return L


def check(where, rc):
    if rc < 0:
        raise NegfError(where, rc)
    return rc
