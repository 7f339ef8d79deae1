"""maxDistance pairs in the GPU SQP step against the oracle's SQP
(oracle/contact.py, exact QP solves with the pair rows of
cpp/src/constraints/maxDistance.cpp:4-80).

Two cubes fly apart joined by a 2.5 mm pair (the two-sphere rope of
cpp/demos/08_multiple_constraints_sphere.cpp): the pair goes taut, is held,
and releases.  Trajectories agree to 1e-9 m in FP64 and 1e-6 of the
displacement in mixed precision; the held pairs agree step by step.
"""
import numpy as np
import pytest

from tests.helpers import contact_pair, two_cubes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_rope_between_cubes(precision, kind):
    X, T, a, b, n1 = two_cubes(kind=kind)
    dt = 5e-4
    en, sol, sq, _ = contact_pair(X, T, dt=dt, rho=1000.0, E=2e4, nu=0.4, precision=precision,
                                  max_distance=([a], [b], [0.0025]))
    v = np.zeros_like(X); v[:n1, 0] = -0.2; v[n1:, 0] = 0.2
    en.set_initial_velocity(v.ravel())
    sq.s.set_initial_velocity(v.ravel())
    x = X.ravel().copy(); xo = x.copy()
    held = []
    for _ in range(14):
        x = sol.step(x, en)
        xo = sq.step(xo, dt)
        hp = en.held_pairs()
        if precision == "fp64":
            assert list(hp) == list(sq.held_pairs)
        held.append(len(hp))
        L = np.linalg.norm(x.reshape(-1, 3)[a] - x.reshape(-1, 3)[b])
        assert L <= 0.0025 + 1e-9
    assert max(held) == 1 and held[-1] == 0
    disp = np.abs(xo - X.ravel()).max()
    err = np.abs(x - xo).max()
    assert err <= (1e-9 if precision == "fp64" else 1e-6 * disp), (err, disp)


def test_rope_and_ground():
    # the demo's combination: plane contact and a maxDistance pair in one QP
    X, T, a, b, n1 = two_cubes(kind="tet")
    X = X + np.array([0.0, 0.0, 0.0002])
    dt = 5e-4
    en, sol, sq, surf = contact_pair(X, T, planes=([[0, 0, 0]], [[0, 0, 1.0]]), dt=dt, rho=1000.0, E=2e4, nu=0.4,
                                     max_distance=([a], [b], [0.0025]))
    v = np.zeros_like(X); v[:n1, 0] = -0.2; v[n1:, 0] = 0.2; v[:, 2] = -0.3
    en.set_initial_velocity(v.ravel())
    sq.s.set_initial_velocity(v.ravel())
    x = X.ravel().copy(); xo = x.copy()
    touched = held = 0
    for _ in range(12):
        x = sol.step(x, en)
        xo = sq.step(xo, dt)
        assert en.active_contacts() == sq.last_active
        assert list(en.held_pairs()) == list(sq.held_pairs)
        touched += sq.last_active
        held += len(sq.held_pairs)
        assert x.reshape(-1, 3)[surf, 2].min() > -1e-9
    assert touched > 0 and held > 0
    assert np.abs(x - xo).max() < 1e-9


def test_adjoint_rope_vs_fd():
    # gradient of a loss on the final state w.r.t. per-element Young's moduli
    # through steps that hold the pair, against central differences of the
    # oracle's SQP rollout (h = 1e-6 relative)
    import torch
    from oracle import oracle as orc
    from oracle import contact as oc
    from sors_b200.adjoint import rollout
    X, T, a, b, n1 = two_cubes(kind="tet")
    ne = T.shape[0]
    rng = np.random.default_rng(5)
    E = np.exp(rng.uniform(np.log(1e4), np.log(4e4), ne))
    dt, steps = 5e-4, 6
    v0 = np.zeros_like(X); v0[:n1, 0] = -0.2; v0[n1:, 0] = 0.2
    en, sol, _, _ = contact_pair(X, T, dt=dt, rho=1000.0, E=E, nu=0.4, max_distance=([a], [b], [0.0025]))
    c = rng.standard_normal(X.size)

    def oracle_final(Ev):
        o = orc.System(X, T, rho=1000.0, youngs=Ev, nu=0.4, grav=(0, 0, -9.81), scheme="backward_euler",
                       method="minimize_SQP", dt=dt, substeps=1)
        o.set_initial_velocity(v0.ravel())
        sq = oc.SQPOracle(o, max_distance=oc.MaxDistance([a], [b], [0.0025]))
        q = X.ravel().copy()
        held = 0
        for _ in range(steps):
            q = sq.step(q, dt)
            held += len(sq.held_pairs)
        return q, held

    qo, held = oracle_final(E)
    assert held >= 3
    Et = torch.tensor(E, requires_grad=True)
    qT = rollout(en, sol, Et, None, steps, dt, v0=v0.ravel(), poisson=0.4, checkpoint_every=4)
    assert np.abs(qT.detach().numpy() - qo).max() < 1e-9
    (qT * torch.tensor(c)).sum().backward()
    gE = Et.grad.numpy()
    h = 1e-6
    for _ in range(3):
        r = rng.standard_normal(ne)
        d_adj = gE @ (E * r)
        d_fd = c @ (oracle_final(E * (1 + h * r))[0] - oracle_final(E * (1 - h * r))[0]) / (2 * h)
        assert abs(d_adj - d_fd) <= 1e-5 * abs(d_fd), (d_adj, d_fd)
