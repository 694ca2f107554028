"""The C ABI library loads on a machine without a GPU and exports every
entry point include/ct2b200.h declares (no compute calls)."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    src = open(os.path.join(ROOT, "include", "ct2b200.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ct2_\w+)\s*\(", src)))


def test_header_declares_entry_points():
    names = declared_symbols()
    assert "ct2_view_proj3D_sinoproj_linear" in names
    assert "ct2_dev_view_proj3D_sinobackproject_linear" in names
    assert len(names) >= 20


def test_library_exports_every_declared_symbol():
    from ct2b200 import _lib
    L = _lib.lib()
    missing = [n for n in declared_symbols() if not hasattr(L, n)]
    assert not missing, missing


def test_every_declared_symbol_has_a_python_signature():
    from ct2b200 import _lib
    _lib.lib()
    bound = set()
    for name in _lib.SIGS:
        bound.add("ct2_" + name)
        bound.add("ct2_dev_" + name)
    for name in _lib.DEV_ONLY:
        bound.add("ct2_dev_" + name)
    for name in _lib.HOST_ONLY:
        bound.add("ct2_" + name)
    extra = {"ct2_last_error", "ct2_version"}
    unbound = [n for n in declared_symbols() if n not in bound and n not in extra]
    assert not unbound, unbound


def test_version_and_error_strings():
    from ct2b200 import _lib
    L = _lib.lib()
    assert b"sm_100a" in L.ct2_version()
    assert isinstance(L.ct2_last_error(), bytes)


def test_invalid_arguments_rejected_without_gpu_work():
    """Argument validation runs before any CUDA call, so it works here."""
    import numpy as np
    import pytest
    import view_proj3D
    fv = np.zeros((2, 18), np.float32)
    with pytest.raises(ValueError):
        view_proj3D.sinoproj_linear(None, fv, 2, 4, 4, 1.0, 1.0, -2.0, -2.0,
                                    np.zeros((3, 3, 3), np.float32), -1.0, 1.0, 1.0, 0, 0, 0,
                                    3, 3, 3)


def test_window_overrun_is_an_argument_error_before_any_device_work():
    """sinoave / sinodist windows past the sinogram are rejected by the C ABI
    (the Fortran would read or write past its array)."""
    import numpy as np
    from ct2b200 import _lib
    s = np.zeros((4, 4, 4), np.float32)
    o = np.zeros((2, 2, 2), np.float32)
    rc = _lib.lib().ct2_tomo3Dfort_sinoave(s.ctypes.data, o.ctypes.data, 4, 4, 4, 2, 2, 2, 2, 2, 2,
                                           3, 2, 2)
    assert rc == _lib.CT2_EINVAL
    assert "windows reach past" in _lib.last_error()


def test_set_backprojector_rejects_unknown_kind():
    """The backprojector switch checks its argument before any CUDA call."""
    from ct2b200 import _lib
    L = _lib.lib()
    assert L.ct2_set_backprojector(2) == _lib.CT2_EINVAL
    assert L.ct2_set_backprojector(-1) == _lib.CT2_EINVAL


def test_wait_selftest_rejects_bad_spin_counts():
    """Argument checks of the bounded-wait self-test run before any CUDA call."""
    from ct2b200 import _lib
    L = _lib.lib()
    assert L.ct2_wait_selftest(0) == _lib.CT2_EINVAL
    assert L.ct2_wait_selftest((1 << 20) + 1) == _lib.CT2_EINVAL


def test_launch_count_is_host_bookkeeping():
    """The launch counter answers without a GPU: no kernel has run here, so
    after a reset it reads zero, and a null pointer is an argument error."""
    import ctypes
    from ct2b200 import _lib
    L = _lib.lib()
    n = ctypes.c_ulonglong(123)
    assert L.ct2_launch_count(ctypes.byref(n), 1) == _lib.CT2_OK
    assert L.ct2_launch_count(ctypes.byref(n), 0) == _lib.CT2_OK
    assert n.value == 0
    assert L.ct2_launch_count(None, 0) == _lib.CT2_EINVAL


def test_batch_entry_points_check_arguments_first():
    """The batch engine rejects bad arguments before any CUDA call."""
    import ctypes
    from ct2b200 import _lib
    L = _lib.lib()
    h = ctypes.c_void_p()
    assert L.ct2_batch_create(0, ctypes.byref(h)) == _lib.CT2_EINVAL
    assert L.ct2_batch_create(257, ctypes.byref(h)) == _lib.CT2_EINVAL
    assert L.ct2_batch_create(4, None) == _lib.CT2_EINVAL
    assert L.ct2_batch_commit(None, None, None) == _lib.CT2_EINVAL
    assert L.ct2_batch_em_iteration(None, None) == _lib.CT2_EINVAL
    assert L.ct2_batch_clear(None, 0, None) == _lib.CT2_EINVAL
    assert L.ct2_batch_destroy(None) == _lib.CT2_OK


def test_many_entry_points_check_arguments_first():
    """The multi-volume projector and backprojector validate the volume
    count, the view and the grid before any CUDA call, and an empty batch is
    no work."""
    from ct2b200 import _lib
    L = _lib.lib()
    view = [2, 4, 4, 1.0, 1.0, -2.0, -2.0]
    grid = [1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 3, 3, 3]
    for fn in (L.ct2_dev_view_proj3D_sinoproj_linear_many,
               L.ct2_dev_view_proj3D_sinobackproject_linear_many):
        assert fn(-1, None, None, *view, None, *grid, None) == _lib.CT2_EINVAL
        assert fn(4097, None, None, *view, None, *grid, None) == _lib.CT2_EINVAL
        assert b"nvol" in L.ct2_last_error()
        assert fn(2, None, None, 2, -4, 4, 1.0, 1.0, -2.0, -2.0, None, *grid,
                  None) == _lib.CT2_EINVAL
        assert fn(2, None, None, *view, None, 1.0, 0.0, 1.0, 0.0, 0.0, 0.0, 3, 3, 3,
                  None) == _lib.CT2_EINVAL
        assert fn(0, None, None, *view, None, *grid, None) == _lib.CT2_OK
