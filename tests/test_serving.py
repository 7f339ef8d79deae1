"""Rollout serving: results alone == results in the mix, admission, latencies."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _requests(n, steps=5, seed=3):
    from sors_b200.serving import poke_cube_request
    rng = np.random.default_rng(seed)
    return [poke_cube_request(rng, int(rng.integers(4, 9)), tag=i, steps=steps, dt=1e-2) for i in range(n)]


def test_alone_equals_mix():
    from sors_b200.serving import RolloutServer
    reqs = _requests(6)
    alone = {}
    for r in _requests(6):
        srv = RolloutServer(max_slots=1)
        srv.submit(r)
        res = srv.close()
        assert res[0].error is None, res[0].error
        alone[r.tag] = res[0].final
    srv = RolloutServer(max_slots=4)
    for r in reqs:
        srv.submit(r)
    mixed = {r.tag: r for r in srv.close()}
    assert sorted(mixed) == sorted(alone)
    for tag, res in mixed.items():
        assert res.error is None, res.error
        assert len(res.step_latencies) == 5
        # independent handles and deterministic kernels: bitwise the same
        assert np.array_equal(res.final, alone[tag])
        assert np.abs(res.final - reqs[tag].vertices.ravel()).max() > 1e-5


def test_memory_admission_rejects_oversize():
    from sors_b200.serving import RolloutServer
    srv = RolloutServer(max_slots=2, memory_budget_bytes=1 << 20)
    srv.submit(_requests(1)[0])
    res = srv.close()
    assert res[0].error is not None and "budget" in res[0].error
