"""Adjoint of the implicit step (sors_adjoint_step, sors_b200.adjoint) against
central finite differences of the oracle's forward rollout (FP64).

Directional derivatives along seeded random directions in (E, act) agree with
the oracle's central differences (h = 1e-6 relative) to 1e-5 relative.
"""
import numpy as np
import pytest
import torch

from sors_b200 import meshes
from tests.helpers import make_pair

pytestmark = pytest.mark.gpu

DT = 2e-3


def _case(clamp=True, steps=8, seed=0, precision="fp64"):
    X, T = meshes.hex_bar(6, 2, 2, (0.03, 0.01, 0.01))
    ne = T.shape[0]
    rng = np.random.default_rng(seed)
    E = np.exp(rng.uniform(np.log(1e5), np.log(3e5), ne))
    mus = {"group": np.arange(ne, dtype=np.int32), "k": np.full(ne, 3e4), "dir": np.tile([1.0, 0, 0], (ne, 1))}
    en, sol, o, s = make_pair(X, T, rho=1070.0, E=E, nu=0.45, dt=DT, clamp=clamp, muscles=mus,
                              precision=precision, res_tol=1e-10 if precision == "mixed" else 0.0)
    act = rng.uniform(0, 1, (steps, ne))
    w = rng.standard_normal(3 * X.shape[0])
    return X, T, E, mus, en, sol, act, w


def _oracle_loss(oracle, X, T, E, mus, act, w, clamp):
    o = oracle.System(X, T, rho=1070.0, youngs=E, nu=0.45, grav=(0, 0, -9.81), scheme="backward_euler",
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
def test_adjoint_vs_oracle_fd(oracle, clamp):
    from sors_b200.adjoint import rollout
    X, T, E, mus, en, sol, act, w = _case(clamp=clamp)
    Et = torch.tensor(E, requires_grad=True)
    At = torch.tensor(act, requires_grad=True)
    qT = rollout(en, sol, Et, At, act.shape[0], DT, poisson=0.45)
    loss = (torch.tensor(w) * qT).sum()
    loss.backward()
    gE, gA = Et.grad.numpy(), At.grad.numpy()
    # the GPU forward matches the oracle's
    assert abs(loss.item() - _oracle_loss(oracle, X, T, E, mus, act, w, clamp)) < 1e-9 * np.abs(w).sum()
    rng = np.random.default_rng(42)
    h = 1e-6
    for _ in range(4):
        rE = rng.standard_normal(E.size)
        rA = rng.standard_normal(act.shape)
        d_adj = gE @ (E * rE) + (gA * rA).sum()
        lp = _oracle_loss(oracle, X, T, E * (1 + h * rE), mus, act + h * rA, w, clamp)
        lm = _oracle_loss(oracle, X, T, E * (1 - h * rE), mus, act - h * rA, w, clamp)
        d_fd = (lp - lm) / (2 * h)
        assert abs(d_adj - d_fd) <= 1e-5 * abs(d_fd) + 1e-12, (d_adj, d_fd)


def test_checkpointing_is_exact():
    from sors_b200.adjoint import RolloutAdjoint
    X, T, E, mus, en, sol, act, w = _case(steps=7)
    grads = []
    for k in (1, 3):
        r = RolloutAdjoint(en, sol, act.shape[0], DT, poisson=0.45, checkpoint_every=k)
        qT = r.forward(E, act)
        gE, gA, gq0, gv0 = r.backward(w)
        grads.append((qT, gE, gA, gq0, gv0))
    for a, b in zip(*grads):
        np.testing.assert_array_equal(a, b)


def test_adjoint_mixed_precision():
    from sors_b200.adjoint import RolloutAdjoint
    out = []
    for precision in ("fp64", "mixed"):
        X, T, E, mus, en, sol, act, w = _case(precision=precision)
        r = RolloutAdjoint(en, sol, act.shape[0], DT, poisson=0.45)
        r.forward(E, act)
        gE, gA, _, _ = r.backward(w)
        out.append(np.concatenate([gE * E, gA.ravel()]))
    err = np.abs(out[1] - out[0]).max() / np.abs(out[0]).max()
    assert err < 1e-4, err


def test_adjoint_neumann_velocity(oracle):
    # one step with a prescribed velocity on the x = 0 face: dL/dneumann by FD
    import ctypes as C
    from sors_b200 import _lib
    X, T = meshes.hex_bar(4, 2, 2, (0.02, 0.01, 0.01))
    mask, val = meshes.clamp_mask(X)
    rng = np.random.default_rng(3)
    val = np.where(mask == 1, rng.uniform(-0.05, 0.05, mask.size), 0.0)
    en, sol, o, s = make_pair(X, T, dt=DT, clamp=True)
    L = _lib.load()
    _lib.check(L.sors_set_neumann(en._h, mask.astype(np.int32).ctypes.data_as(C.POINTER(C.c_int32)),
                                  val.ctypes.data_as(C.POINTER(C.c_double))))
    q1 = sol.step(X.ravel().copy(), en)
    w = rng.standard_normal(q1.size)
    n = q1.size
    dneu = np.zeros(n); dq = np.zeros(n); dv = np.zeros(n)
    p = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
    st = _lib.SorsStepStats()
    _lib.check(L.sors_adjoint_step(en._h, p(q1), DT, p(w), None, None, 0, p(dq), p(dv), None, None, p(dneu),
                                   C.byref(st)))

    def f(v):
        oo = oracle.System(X, T, rho=1070.0, youngs=1e5, nu=0.45, grav=(0, 0, -9.81), dt=DT, substeps=1)
        oo.set_neumann(mask, v)
        qq, st2 = oo.step(X.ravel().copy())
        assert st2 == 0
        return float(w @ qq)
    r = rng.standard_normal(n) * mask
    h = 1e-6
    d_fd = (f(val + h * r) - f(val - h * r)) / (2 * h)
    assert abs(dneu @ r - d_fd) <= 1e-6 * abs(d_fd)
    # dL/dq_n and dL/dv_n against FD of the initial state
    def g(q0, v0):
        oo = oracle.System(X, T, rho=1070.0, youngs=1e5, nu=0.45, grav=(0, 0, -9.81), dt=DT, substeps=1)
        oo.set_neumann(mask, val)
        oo.set_initial_deformation(q0); oo.set_initial_velocity(v0)
        qq, st2 = oo.step(q0.copy())
        assert st2 == 0
        return float(w @ qq)
    rq = rng.standard_normal(n) * 1e-3; rv = rng.standard_normal(n) * 1e-2
    q0 = X.ravel().copy(); v0 = np.zeros(n)
    d_fd = (g(q0 + h * rq, v0 + h * rv) - g(q0 - h * rq, v0 - h * rv)) / (2 * h)
    assert abs(dq @ rq + dv @ rv - d_fd) <= 1e-6 * abs(d_fd)
