"""
The standalone nearest-dot search (cms_nearest_dots) against SciPy's
cdist(ref, query, 'sqeuclidean').min(axis=0) / .argmin(axis=0), the CPU
computation the reference's min_sqdist primitive replaces
(cms-cuda/_gpu_kernels.py:508-566): bit-identical minima and first-index
argmins, exact ties included.
"""

import numpy as np
import pytest
from scipy.spatial.distance import cdist

from parity import exact, load_case

pytestmark = pytest.mark.gpu


def _ctx():
    from cms_cuda import _lib
    return _lib.Context(0)


def test_random_points_with_ties():
    rng = np.random.default_rng(0)
    q = rng.uniform(-30, 30, (3000, 3))
    r = rng.uniform(-30, 30, (7000, 3))
    r[4100] = r[50]            # duplicate reference: the first index must win
    q[7] = r[50]               # a query sitting on it (distance 0)
    q[8] = (r[10] + r[20]) / 2
    d2, idx = _ctx().nearest_dots(q, r)
    ref = cdist(r, q, metric="sqeuclidean")
    exact("min d2", d2, ref.min(axis=0))
    exact("argmin", idx, ref.argmin(axis=0))
    assert idx[7] == 50 and d2[7] == 0.0


def test_golden_buried_dots():
    """Buried target dots against buried binder dots of the reference's golden complex."""
    c = load_case("golden_pkl")
    q = c["dots1_coor"][c["dots1_buried"] == 1]
    r = c["dots0_coor"][c["dots0_buried"] == 1]
    d2, idx = _ctx().nearest_dots(q, r)
    ref = cdist(r, q, metric="sqeuclidean")
    exact("min d2", d2, ref.min(axis=0))
    exact("argmin", idx, ref.argmin(axis=0))


def test_far_offset_coordinates():
    """Large absolute coordinates (FP32 staging relative to the box centre)."""
    rng = np.random.default_rng(1)
    base = np.array([5000.0, -3000.0, 12000.0])
    q = base + rng.normal(0, 10, (500, 3))
    r = base + rng.normal(0, 10, (900, 3))
    d2, idx = _ctx().nearest_dots(q, r)
    ref = cdist(r, q, metric="sqeuclidean")
    exact("min d2", d2, ref.min(axis=0))
    exact("argmin", idx, ref.argmin(axis=0))
