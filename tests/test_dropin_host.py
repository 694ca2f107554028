"""The drop-in modules' argument marshalling on the host path (NumPy
inputs), without a GPU: conversion to the Fortran types as f2py converts,
shape checks raising ValueError, intent(in,out) arrays copied rather than
updated in place, empty arrays passed as null pointers, and the surface
table's argument order."""
import numpy as np
import pytest

from ct2b200 import _dropin as D


def test_host_path_chosen_for_numpy():
    m = D.Marshal("sinoproj_linear", [np.zeros(3), None, 1.0])
    assert not m.dev and m.device is None


def test_f32_converts_and_checks_shapes():
    m = D.Marshal("f", [])
    x = np.arange(24, dtype=np.float64).reshape(2, 3, 4)[:, :, ::2]  # strided, FP64
    a = m.f32(x, (2, 3, 2), "smat")
    assert a.dtype == np.float32 and a.flags.c_contiguous
    assert np.array_equal(a, x.astype(np.float32))
    assert m.f32([1, 2, 3], None, "v").dtype == np.float32
    with pytest.raises(ValueError, match=r"f: argument smat has shape \(2, 3, 2\), "
                                         r"expected \(2, 3, 3\)"):
        m.f32(x, (2, 3, 3), "smat")
    with pytest.raises(ValueError, match="argument v must be an array"):
        m.f32(1.5, (3,), "v")
    assert m.f32(1.5, (1,), "v").shape == (1,)  # a scalar for a one-element array


def test_i32_converts_and_passes_none():
    m = D.Marshal("f", [])
    assert m.i32(None, (2,), "ind") is None
    a = m.i32(np.array([[1, 0], [0, 1]], dtype=np.int64), (2, 2), "ind")
    assert a.dtype == np.int32 and a.flags.c_contiguous
    with pytest.raises(ValueError, match="argument ind has shape"):
        m.i32(np.ones((2, 3)), (3, 2), "ind")


def test_out_and_copy():
    m = D.Marshal("f", [])
    o = m.out((2, 5))
    assert o.shape == (2, 5) and o.dtype == np.float32 and not o.any()
    src = np.ones((3, 3), np.float32)
    c = m.copy(src, (3, 3), "smat")
    c[0, 0] = 7.0
    assert src[0, 0] == 1.0  # the caller's array is not updated in place
    ro = np.ones(4, np.float32)
    ro.setflags(write=False)
    assert m.copy(ro, (4,), "x").flags.writeable


def test_ptr_of_empty_arrays_is_null():
    assert D.Marshal.ptr(None) is None
    assert D.Marshal.ptr(np.zeros(0, np.float32)) is None
    a = np.zeros(3, np.float32)
    assert D.Marshal.ptr(a) == a.ctypes.data


def test_arguments_are_kept_alive():
    m = D.Marshal("f", [])
    a = m.f32(np.ones(3), (3,), "v")
    o = m.out((3,))
    assert any(k is a for k in m.keep) and any(k is o for k in m.keep)


def test_shape_table_order_and_checks():
    m = D.Marshal("gen_shape_proj", [])
    nsurf = 2
    frames = [np.full(nsurf, i, np.float64) for i in range(12)]
    ell = [np.ones(1), np.ones(1) * 2, np.ones(1) * 3]
    cyl = [np.zeros(0), np.zeros(0)]
    cone = [np.ones(1) * 4, np.ones(1) * 5]
    args = D.shape_table(m, nsurf, frames, 0, 1, ell, 0, cyl, 1, cone)
    assert args[0] == 2
    assert [float(a[0]) for a in args[1:13]] == [float(i) for i in range(12)]
    assert args[13] == 0                                   # planes
    assert args[14] == 1 and [float(a[0]) for a in args[15:18]] == [1.0, 2.0, 3.0]
    assert args[18] == 0 and [a.size for a in args[19:21]] == [0, 0]
    assert args[21] == 1 and [float(a[0]) for a in args[22:24]] == [4.0, 5.0]
    with pytest.raises(ValueError, match="argument ax_ell has shape"):
        D.shape_table(m, nsurf, frames, 0, 2, ell, 0, cyl, 1, cone)
    with pytest.raises(ValueError, match="argument yu2 has shape"):
        bad = list(frames)
        bad[4] = np.zeros(3)
        D.shape_table(m, nsurf, bad, 0, 1, ell, 0, cyl, 1, cone)


def test_int_and_float_helpers():
    assert D.ints(1.0, np.int64(2), "3") == [1, 2, 3]
    assert D.floats(1, np.float32(0.5)) == [1.0, 0.5]
