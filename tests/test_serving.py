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
        srv = RolloutServer(max_slots=1, max_blocks=296)
        srv.submit(r)
        res = srv.close()
        assert res[0].error is None, res[0].error
        alone[r.tag] = res[0].final
    srv = RolloutServer(max_slots=4, max_blocks=296)
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


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_served_poke_matches_oracle(precision):
    # one poke rollout (ground plane + moving disk) through the server against
    # the oracle's SQP rollout: FP64 1e-8 m, mixed 1e-6 of the displacement
    from oracle import oracle as orc
    from oracle import contact as oc
    from sors_b200.serving import RolloutServer, poke_cube_request
    rng = np.random.default_rng(5)
    req = poke_cube_request(rng, 4, tag=0, steps=8, dt=1e-2, precision=precision)
    srv = RolloutServer(max_slots=2)
    srv.submit(req)
    res = srv.close()[0]
    assert res.error is None, res.error
    o = orc.System(req.vertices, req.elements, rho=req.density, youngs=req.youngs, nu=req.poisson,
                   grav=req.gravity, scheme="backward_euler", method="minimize_SQP", dt=req.dt, substeps=1)
    dk = oc.DiskContact(req.disks[0], req.disks[1], req.disks[2], req.surface)
    sq = oc.SQPOracle(o, oc.PlaneContact(req.planes[0], req.planes[1], req.surface), dk)
    q = req.vertices.ravel().copy()
    held = 0
    for t in range(req.steps):
        dk.set_disk(req.disks[0][0] + req.disk_velocity[0] * req.dt * t, req.disks[1][0], req.disks[2][0])
        q = sq.step(q, req.dt)
        held += sq.last_active
    assert held > 0
    disp = np.abs(q - req.vertices.ravel()).max()
    err = np.abs(res.final - q).max()
    assert err <= (1e-8 if precision == "fp64" else 1e-6 * disp), (err, disp)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batched_equals_alone(precision):
    # six pokes packed into one union handle against each run alone
    from sors_b200.serving import RolloutServer, poke_cube_request

    def reqs():
        rng = np.random.default_rng(8)
        return [poke_cube_request(rng, int(rng.integers(3, 7)), tag=i, steps=6, dt=1e-2, precision=precision)
                for i in range(6)]
    alone = {}
    for r in reqs():
        srv = RolloutServer(max_slots=1)
        srv.submit(r)
        res = srv.close()[0]
        assert res.error is None, res.error
        alone[r.tag] = res.final
    rs = reqs()
    srv = RolloutServer(max_slots=2, batch_max=6)
    for r in rs:
        srv.submit(r)
    out = {r.tag: r for r in srv.close()}
    assert sorted(out) == sorted(alone)
    assert max(r.batch for r in out.values()) > 1
    for tag, res in out.items():
        assert res.error is None, res.error
        disp = np.abs(alone[tag] - rs[tag].vertices.ravel()).max()
        err = np.abs(res.final - alone[tag]).max()
        # FP64: within the SQP stopping tolerance ||dx|| < 1e-9 m; mixed: 1e-6 of the displacement
        assert err <= (1e-9 if precision == "fp64" else 1e-6 * disp), (tag, err, disp)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_member_segmented_pcg_equals_alone(precision):
    # three cantilevers of different lengths in one handle, declared as three
    # members: each member's trajectory equals its run alone
    import ctypes as C

    from sors_b200 import _lib, meshes
    from tests.helpers import make_pair
    parts = [meshes.cantilever_tets(n, 2, 2, (0.005 * n, 0.01, 0.01)) for n in (4, 8, 12)]
    alone = []
    for X, T in parts:
        en, sol, _, _ = make_pair(X, T, dt=1e-3, precision=precision, res_tol=1e-8)
        q = X.ravel().copy()
        for _ in range(5):
            q = sol.step(q, en)
        alone.append(q)
    offs = np.cumsum([0] + [X.shape[0] for X, _ in parts]).astype(np.int32)
    Xu = np.vstack([X for X, _ in parts])
    Tu = np.vstack([T + offs[k] for k, (_, T) in enumerate(parts)]).astype(np.int32)
    en, sol, _, _ = make_pair(Xu, Tu, dt=1e-3, precision=precision, res_tol=1e-8)
    _lib.check(_lib.load().sors_set_members(en.handle(), offs.ctypes.data_as(C.POINTER(C.c_int32)), len(parts)))
    q = Xu.ravel().copy()
    for _ in range(5):
        q = sol.step(q, en)
    for k, (X, _) in enumerate(parts):
        qk = q[3 * offs[k]:3 * offs[k + 1]]
        disp = np.abs(alone[k] - X.ravel()).max()
        err = np.abs(qk - alone[k]).max()
        assert err <= (1e-9 if precision == "fp64" else 1e-6 * disp), (k, err, disp)


def test_members_reject_a_coupling_element():
    import ctypes as C

    from sors_b200 import _lib, meshes
    from tests.helpers import make_pair
    X, T = meshes.cantilever_tets(4, 2, 2, (0.02, 0.01, 0.01))
    en, _, _, _ = make_pair(X, T, dt=1e-3)
    offs = np.array([0, 10, X.shape[0]], np.int32)  # cuts through the beam
    st = _lib.load().sors_set_members(en.handle(), offs.ctypes.data_as(C.POINTER(C.c_int32)), 2)
    assert st == 1 and "joins two members" in _lib.last_error()
