"""Host-side logic of the rollout server (no GPU): the device-footprint
estimate used for admission, request compatibility for union handles, and the
poke workload's helpers."""
import math

import numpy as np

from sors_b200 import serving


def _req(n_cells=4, **kw):
    rng = np.random.default_rng(0)
    r = serving.poke_cube_request(rng, n_cells, steps=kw.pop("steps", 10))
    for k, v in kw.items():
        setattr(r, k, v)
    return r


def test_footprint_estimate_grows_with_size_and_precision():
    a = serving.estimate_device_bytes(1000, 5000, 4, "mixed")
    b = serving.estimate_device_bytes(2000, 10000, 4, "mixed")
    c = serving.estimate_device_bytes(1000, 5000, 4, "fp64")
    h = serving.estimate_device_bytes(1000, 5000, 8, "mixed")
    assert 0 < a < b and a < c and a < h
    # roughly linear in the mesh size once past the fixed 1 MiB
    assert 1.8 < (b - (1 << 20)) / (a - (1 << 20)) < 2.2


def test_compatible_requests():
    a, b = _req(), _req()
    assert serving.compatible(a, b)
    assert not serving.compatible(a, _req(steps=11))
    assert not serving.compatible(a, _req(precision="fp64"))
    assert not serving.compatible(a, _req(planes=([[0, 0, 0.001]], [[0, 0, 1.0]])))
    assert not serving.compatible(a, _req(disks=None))


def test_cube_surface_nodes():
    for n in (1, 2, 5):
        s = serving.cube_surface_nodes(n)
        assert s.size == (n + 1) ** 3 - max(n - 1, 0) ** 3
        assert s.min() >= 0 and s.max() < (n + 1) ** 3
        assert np.all(np.diff(s) > 0)


def test_poke_request_shape():
    r = _req(n_cells=3)
    assert r.vertices.shape == (64, 3) and r.elements.shape == (6 * 27, 4)
    assert r.planes is not None and r.disks is not None
    assert set(np.asarray(r.surface).tolist()) <= set(range(64))


def test_percentile_empty_is_nan():
    assert math.isnan(serving.percentile([], 50))
    assert serving.percentile([1.0, 2.0, 3.0], 50) == 2.0
