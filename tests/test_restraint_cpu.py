"""Harmonic restraint handle through the C ABI without a device: argument
checks of the setters (include/HarmonicRestraintForce.h and
src/HarmonicRestraintForce.cu:36-160 raise on the same inputs)."""
import numpy as np
import pytest

from apocharmm_b200 import api
from apocharmm_b200._lib import ApoCharmmError


def test_setters_check_sizes_and_values():
    n = 10
    h = api.HarmonicRestraintForce(n)
    h.setSelection([0, 3, 9])
    h.setForceConstant(2.5)
    h.setForceConstants(np.ones(n))
    h.setReferenceCoordinates(np.zeros((n, 3)))
    h.setMasses(np.full(n, 12.0))
    with pytest.raises(ApoCharmmError, match="out of range"):
        h.setSelection([0, n])
    with pytest.raises(ApoCharmmError, match="out of range"):
        h.setSelection([-1])
    with pytest.raises(ApoCharmmError, match="expected 10 values"):
        h.setForceConstants(np.ones(n + 1))
    with pytest.raises(ApoCharmmError, match="expected 30 values"):
        h.setReferenceCoordinates(np.zeros((n - 1, 3)))
    with pytest.raises(ApoCharmmError, match="non-finite"):
        h.setMasses(np.full(n, np.nan))
    with pytest.raises(ApoCharmmError, match="finite"):
        h.setForceConstant(np.inf)
    h.close()


def test_create_rejects_bad_sizes():
    with pytest.raises(ApoCharmmError):
        api.HarmonicRestraintForce(0)
