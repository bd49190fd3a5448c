"""Argument checks of the Python mirror that run before any library call (no device)."""
import numpy as np
import pytest

import rls_b200 as R
from rls_b200.solvers import _checked


def test_checked_inputs_are_converted_and_sized():
    Z = np.arange(6, dtype=np.float64)[::2]                     # strided, wrong dtype
    a = _checked(Z, np.complex128, 3, "rec.Z")
    assert a.dtype == np.complex128 and a.flags.c_contiguous and np.array_equal(a.real, [0, 2, 4])
    with pytest.raises(R.DimensionMismatch):
        _checked(Z, np.complex128, 4, "rec.Z")


def test_checked_outputs_must_be_writable_in_place():
    sigma = np.zeros(5)
    assert _checked(sigma, np.float64, 5, "sigma", writable=True) is sigma
    with pytest.raises(R.ArgumentError):
        _checked(np.zeros(5, dtype=np.float32), np.float64, 5, "sigma", writable=True)
    with pytest.raises(R.ArgumentError):
        _checked(np.zeros(10)[::2], np.float64, 5, "sigma", writable=True)
    ro = np.zeros(5)
    ro.flags.writeable = False
    with pytest.raises(R.ArgumentError):
        _checked(ro, np.float64, 5, "sigma", writable=True)
    with pytest.raises(R.DimensionMismatch):
        _checked(np.zeros(4), np.float64, 5, "sigma", writable=True)
