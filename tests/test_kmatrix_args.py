"""Host-side argument checks of `KMatrix.gemv_device` (no library call is
made: each case is rejected before the C ABI is reached)."""
import pytest
import torch

from __graft_entry__ import import_package


@pytest.fixture(scope="module")
def eqd():
    return import_package()


def _matrix(eqd, n):
    M = object.__new__(eqd.KMatrix)   # no device K: only the checks run
    M.n, M._h = n, None
    return M


def test_rejects_wrong_length(eqd):
    M = _matrix(eqd, 10)
    s = torch.zeros(3, 9, dtype=torch.float64)
    with pytest.raises(eqd.EqdArgumentError):
        M.gemv_device(s, torch.zeros_like(s))


def test_rejects_float32_and_noncontiguous(eqd):
    M = _matrix(eqd, 10)
    with pytest.raises(eqd.EqdArgumentError):
        M.gemv_device(torch.zeros(2, 10, dtype=torch.float32), torch.zeros(2, 10, dtype=torch.float64))
    s = torch.zeros(10, 4, dtype=torch.float64).t()   # (4, 10), not contiguous
    with pytest.raises(eqd.EqdArgumentError):
        M.gemv_device(s, torch.zeros(4, 10, dtype=torch.float64))


def test_rejects_mismatched_vector_counts(eqd):
    M = _matrix(eqd, 10)
    with pytest.raises(eqd.EqdArgumentError):
        M.gemv_device(torch.zeros(3, 10, dtype=torch.float64), torch.zeros(2, 10, dtype=torch.float64))
    with pytest.raises(eqd.EqdArgumentError):
        M.gemv_device((0, 3), (0, 4))
