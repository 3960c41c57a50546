"""The C-ABI library loads and exports every symbol include/negf_gpu.h and
include/negf_mlp.h declare; argument errors come back as status codes (no GPU needed)."""
import ctypes as C
import os
import re

import pytest

from negftrans_b200 import _lib

INC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "include")


def declared_symbols(header="negf_gpu.h"):
    src = open(os.path.join(INC, header)).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char \*)\s*(negf_\w+)\s*\(", src, re.M)))


def test_header_and_binding_agree():
    assert sorted(_lib.EXPORTS) == declared_symbols()
    assert sorted(_lib.MLP_EXPORTS) == declared_symbols("negf_mlp.h")


def test_library_exports_all(built_lib):
    L = C.CDLL(built_lib)
    for name in declared_symbols() + declared_symbols("negf_mlp.h"):
        assert hasattr(L, name), name


def test_version(built_lib):
    assert b"sm_100a" in _lib.lib().negf_version()


def test_argument_errors_without_gpu(built_lib):
    L = _lib.lib()
    assert L.negf_basis_size(1.0, 1.0, 1.0, None) == _lib.NEGF_ERR_ARG
    assert L.negf_kmesh(0, 1, 1.0, 1.0, None) == _lib.NEGF_ERR_ARG
    assert L.negf_ctx_create(None, 0, C.byref(C.c_void_p())) == _lib.NEGF_ERR_ARG
    assert L.negf_transmission(None, None, 0, 0, None, None) == _lib.NEGF_ERR_ARG
    assert L.negf_density(None, 4, 4, 0.0, 0.0, 0.0, 1.0, None, None) == _lib.NEGF_ERR_ARG
    assert L.negf_set_variant(None, 0) == _lib.NEGF_ERR_ARG
    assert L.negf_density_accumulate(None, None, None, 0, None, None) == _lib.NEGF_ERR_ARG
    assert L.negf_autotune(None, None, 0, None, None) == _lib.NEGF_ERR_ARG
    assert L.negf_density_neq(None, 4, 4, 0.0, 0.0, 0.0, 1.0, 1.0, None, None) == _lib.NEGF_ERR_ARG
    buf = (C.c_double * 8)()
    # N_z = 1: the reference indexes generator_r(:,:,0); rejected here
    assert L.negf_tri_solve(None, buf, 1, 1, b"F", buf, None, None) == _lib.NEGF_ERR_ARG


def test_problem_validation_rejects_small_table(built_lib):
    """Pair differences outside the V table would read out of bounds."""
    L = _lib.lib()
    p = _lib.Problem()
    nx = (C.c_int32 * 2)(0, 3)
    ny = (C.c_int32 * 2)(0, 0)
    vh = (C.c_double * (2 * 3 * 3 * 2))()
    kp = (C.c_double * 3)(0, 0, 1)
    p.N, p.Nz, p.ngx, p.ngy = 2, 2, 1, 1
    p.nx, p.ny = C.cast(nx, _lib._ip), C.cast(ny, _lib._ip)
    p.vhat = C.cast(vh, _lib._dp)
    p.Lx = p.Ly = p.Lz = 1.0
    p.nk, p.kpt = 1, C.cast(kp, _lib._dp)
    assert L.negf_ctx_create(C.byref(p), 0, C.byref(C.c_void_p())) == _lib.NEGF_ERR_ARG


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "nope.so"))
    with pytest.raises(RuntimeError):
        _lib.lib()
