"""The C ABI library loads and exports every symbol of include/fhs_b200.h;
CPU-only entry points and error paths work without a GPU."""
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "fhs_b200.h")).read()
    return sorted(set(re.findall(r"FHS_API\s+[^;(]*?\b(fhs_\w+)\s*\(", src)))


def test_every_declared_symbol_is_exported():
    from fhs_b200 import _lib
    L = _lib.lib()
    names = _declared()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_abi_version_and_cpu_only_calls():
    from fhs_b200 import _lib
    from oracle import wavelets
    L = _lib.lib()
    assert L.fhs_abi_version() == 1
    for n0, n1 in ((64, 64), (37, 29), (1024, 1024)):
        assert L.fhs_sara_n_coefs(n0, n1, 4) == wavelets.n_coefs_sara(n0, n1)
    assert L.fhs_sara_n_coefs(8, 8, 0) == -1
    assert L.fhs_solver_stage_count() == 15
    assert L.fhs_solver_stage_name(2) == b"degrid_dual"
    assert L.fhs_solver_stage_name(4) == b"ellipse_fb"


def test_errors_are_reported_not_raised():
    import ctypes as C

    import numpy as np
    from fhs_b200 import _lib
    L = _lib.lib()
    h = C.c_void_p()
    st = L.fhs_measop_create(0, 16, 16, 2, 2, 7, 7, 1, C.byref(h))
    if st == 7:  # no device here
        assert b"no CUDA device" in L.fhs_last_error()
    else:
        assert st == 0
        L.fhs_measop_destroy(h)
    assert L.fhs_measop_create(0, 15, 16, 2, 2, 7, 7, 1, C.byref(h)) in (6, 7)  # odd size: unsupported
    assert L.fhs_solver_destroy(None) == 0
    x = np.zeros(2)
    assert L.fhs_proj_l2ball(0, -1, _lib.dptr(x), 1.0, _lib.dptr(x), _lib.dptr(x)) == 1
    assert L.fhs_proj_l2ball_noalloc(0, 1 << 40, None, 1.0, None, None, None) == 6
    assert b"static scratch limit" in L.fhs_last_error()


def test_package_fails_loudly_without_library(tmp_path, monkeypatch):
    from fhs_b200 import _lib
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "missing.so"))
    with pytest.raises(ImportError):
        _lib.lib()


def test_null_handles_of_the_dr_and_solver_accessors():
    """The entry points added for visibility gridding and the noise adjustment
    reject null handles and buffers with a status, without touching a GPU."""
    import ctypes as C

    import numpy as np
    from fhs_b200 import _lib
    L = _lib.lib()
    out = C.c_void_p()
    buf = np.zeros(4)
    cells = np.zeros(4, dtype=np.int64)
    assert L.fhs_measop_create_dr(None, C.byref(out)) == 1 and not out.value
    assert L.fhs_measop_create_dr(None, None) == 1
    assert L.fhs_measop_is_dr(None) == -1
    assert L.fhs_measop_dr_cells(None, 0, cells.ctypes.data_as(C.POINTER(C.c_int64))) == 1
    assert L.fhs_measop_dr_lambda(None, 0, _lib.dptr(buf)) == 1
    for fn in (L.fhs_solver_epsilon, L.fhs_solver_set_epsilon):
        assert fn(None, _lib.dptr(buf)) != 0
    assert L.fhs_solver_regularization(None, _lib.dptr(buf), None) != 0
    assert L.fhs_last_error() != b""
