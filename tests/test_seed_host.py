"""Host-side pieces of the learned-seed path that need no GPU: the batched
potential generator used for training data reproduces the well family of
``operators.wells_potential``, and argument checks of the Python front end."""
import numpy as np
import pytest

from nutrlan_b200 import operators as ops
from nutrlan_b200.seed_train import potentials
from nutrlan_b200.seednet import _ptr


def test_batched_potentials_match_wells_family():
    seeds = [1, 2, 3, 1000003]
    V = potentials(seeds, 64, device="cpu").numpy()
    for i, s in enumerate(seeds):
        np.testing.assert_allclose(V[i], ops.wells_potential(64, s), rtol=1e-12, atol=1e-12)
        assert V[i].min() < -4.0 and V[i].max() <= 0.0


def test_output_buffers_must_match_exactly():
    with pytest.raises(ValueError):
        _ptr(np.zeros(8, np.float64), np.float32, (8,), output=True)
    with pytest.raises(ValueError):
        _ptr(np.zeros(8, np.float32), np.float32, (9,))
    p, keep = _ptr([1.0, 2.0], np.float32)
    assert keep.dtype == np.float32 and p.value == keep.ctypes.data
