"""Adjoint of Crank-Nicolson steps (sors_adjoint_step_cn through
sors_b200.adjoint) against central finite differences of the oracle's
Crank-Nicolson rollout (FP64).

The CN residual holds half of the previous step's internal force, which the
forward carries as state (zero at the start, as the reference's integrator);
the adjoint chains its cotangent from step to step and the velocity as
v_{t+1} = 2 (q_{t+1} - q_t) / dt - v_t.  Directional derivatives along seeded
directions in (E, act) agree with the oracle's central differences to 1e-5
relative, and checkpointed recomputation (which restores that force) gives the
same gradients as storing every state."""
import numpy as np
import pytest

from sors_b200 import meshes
from tests.helpers import make_pair

pytestmark = pytest.mark.gpu

DT = 2e-3


def _case(steps=6, seed=0, clamp=True):
    X, T = meshes.hex_bar(6, 2, 2, (0.03, 0.01, 0.01))
    ne = T.shape[0]
    rng = np.random.default_rng(seed)
    E = np.exp(rng.uniform(np.log(1e5), np.log(3e5), ne))
    mus = {"group": np.arange(ne, dtype=np.int32), "k": np.full(ne, 3e4), "dir": np.tile([1.0, 0, 0], (ne, 1))}
    en, sol, o, s = make_pair(X, T, rho=1070.0, E=E, nu=0.45, dt=DT, clamp=clamp, muscles=mus,
                              scheme="crank_nicolson")
    act = rng.uniform(0, 1, (steps, ne))
    w = rng.standard_normal(3 * X.shape[0])
    return X, T, E, mus, en, sol, act, w


def _oracle_loss(oracle, X, T, E, mus, act, w, clamp=True):
    o = oracle.System(X, T, rho=1070.0, youngs=E, nu=0.45, grav=(0, 0, -9.81), scheme="crank_nicolson",
                      method="minimize_newton", dt=DT, substeps=1)
    if clamp:
        m, v = meshes.clamp_mask(X)
        o.set_neumann(m, v)
    o.set_muscles(mus["group"], mus["k"], mus["dir"], T.shape[0])
    q = X.ravel().copy()
    for t in range(act.shape[0]):
        o.set_muscle_act(act[t])
        q, st = o.step(q)
        assert st == 0
    return float(w @ q)


@pytest.mark.parametrize("clamp", [True, False])
def test_cn_adjoint_vs_oracle_fd(oracle, clamp):
    from sors_b200.adjoint import RolloutAdjoint
    X, T, E, mus, en, sol, act, w = _case(clamp=clamp)
    r = RolloutAdjoint(en, sol, act.shape[0], DT, poisson=0.45)
    assert r.cn
    qT = r.forward(E, act)
    gE, gA, _, _ = r.backward(w)
    assert abs(float(w @ qT) - _oracle_loss(oracle, X, T, E, mus, act, w, clamp)) < 1e-9 * np.abs(w).sum()
    rng = np.random.default_rng(7)
    h = 1e-6
    for _ in range(3):
        rE = rng.standard_normal(E.size)
        rA = rng.standard_normal(act.shape)
        d_adj = gE @ (E * rE) + (gA * rA).sum()
        lp = _oracle_loss(oracle, X, T, E * (1 + h * rE), mus, act + h * rA, w, clamp)
        lm = _oracle_loss(oracle, X, T, E * (1 - h * rE), mus, act - h * rA, w, clamp)
        d_fd = (lp - lm) / (2 * h)
        assert abs(d_adj - d_fd) <= 1e-5 * abs(d_fd) + 1e-12, (d_adj, d_fd)


def test_cn_checkpointing_is_exact():
    from sors_b200.adjoint import RolloutAdjoint
    X, T, E, mus, en, sol, act, w = _case(steps=7)
    grads = []
    for k in (1, 3):
        r = RolloutAdjoint(en, sol, act.shape[0], DT, poisson=0.45, checkpoint_every=k)
        qT = r.forward(E, act)
        grads.append((qT,) + tuple(r.backward(w)))
    for a, b in zip(*grads):
        assert np.array_equal(a, b)
