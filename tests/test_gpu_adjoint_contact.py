"""Adjoint through contact steps (minimize_SQP): the held contacts act as
equalities in the transpose solve.  Checked against central differences of the
oracle's SQP rollout (FP64, h = 1e-6 relative) along seeded directions."""
import numpy as np
import pytest
import torch

from sors_b200 import meshes
from tests.helpers import contact_pair

pytestmark = pytest.mark.gpu

DT = 2e-3


def _bar():
    X, T = meshes.hex_bar(8, 2, 2, (0.04, 0.01, 0.01))
    return X + np.array([0.0, 0.0, 0.0005]), T


def _oracle_rollout(X, T, E, act, mus, steps, before=None, disks=None, planes=None):
    from oracle import oracle as orc
    from oracle import contact as oc
    groups, _ = meshes.extract_surfaces(X, T)
    surf = np.unique(np.concatenate([g.ravel() for g in groups]))
    o = orc.System(X, T, rho=1070.0, youngs=E, nu=0.45, grav=(0, 0, -9.81), scheme="backward_euler",
                   method="minimize_SQP", dt=DT, substeps=1)
    if mus is not None:
        o.set_muscles(mus["group"], mus["k"], mus["dir"], T.shape[0])
    pl = None if planes is None else oc.PlaneContact(planes[0], planes[1], surf)
    dk = None if disks is None else oc.DiskContact(disks[0], disks[1], disks[2], surf)
    sq = oc.SQPOracle(o, pl, dk)
    q = X.ravel().copy()
    held = 0
    for t in range(steps):
        if before is not None:
            before(t, sq)
        if act is not None:
            o.set_muscle_act(act[t])
        q = sq.step(q, DT)
        held += sq.last_active
    return q, held, o.mass()


def test_adjoint_drop_with_muscles_vs_fd():
    # hex bar with +x fibres dropped onto z = 0: loss (z_com - 0.004)^2 after 14 steps
    from sors_b200.adjoint import rollout
    X, T = _bar()
    ne = T.shape[0]
    rng = np.random.default_rng(1)
    E = np.exp(rng.uniform(np.log(1e5), np.log(3e5), ne))
    steps = 14
    act = rng.uniform(0, 1, (steps, ne))
    mus = {"group": np.arange(ne, dtype=np.int32), "k": np.full(ne, 3e4), "dir": np.tile([1.0, 0, 0], (ne, 1))}
    planes = ([[0, 0, 0]], [[0, 0, 1.0]])
    en, sol, sq, surf = contact_pair(X, T, planes=planes, dt=DT, E=E, muscles=mus)
    qo, held, mass = _oracle_rollout(X, T, E, act, mus, steps, planes=planes)
    assert held > 0
    mz = torch.tensor(mass[2::3])
    Et = torch.tensor(E, requires_grad=True)
    At = torch.tensor(act, requires_grad=True)
    qT = rollout(en, sol, Et, At, steps, DT, poisson=0.45, checkpoint_every=4)
    zc = (qT.view(-1, 3)[:, 2] * mz).sum() / mz.sum()
    loss = (zc - 0.004) ** 2
    loss.backward()
    assert np.abs(qT.detach().numpy() - qo).max() < 1e-8

    def L(Ev, Av):
        q, _, _ = _oracle_rollout(X, T, Ev, Av, mus, steps, planes=planes)
        z = (q[2::3] * mass[2::3]).sum() / mass[2::3].sum()
        return (z - 0.004) ** 2

    gE, gA = Et.grad.numpy(), At.grad.numpy()
    h = 1e-6
    for _ in range(3):
        rE = rng.standard_normal(ne); rA = rng.standard_normal(act.shape)
        d_adj = gE @ (E * rE) + (gA * rA).sum()
        d_fd = (L(E * (1 + h * rE), act + h * rA) - L(E * (1 - h * rE), act - h * rA)) / (2 * h)
        assert abs(d_adj - d_fd) <= 1e-4 * abs(d_fd) + 1e-16, (d_adj, d_fd)


def test_adjoint_disk_poke_vs_fd():
    # tet cube on the ground pressed by a moving disk: d(w . q_T)/dE
    from sors_b200.adjoint import rollout
    from sors_b200 import py_sors as ps
    X, _ = meshes.hex_bar(4, 4, 4, (0.01, 0.01, 0.01))
    T = meshes.kuhn_tet_elements(4, 4, 4)
    ne = T.shape[0]
    rng = np.random.default_rng(2)
    E = rng.uniform(3e4, 8e4, ne)
    c0 = np.array([0.005, 0.005, 0.0102])
    disks = ([c0], [[0, 0, -1.0]], [0.004])
    planes = ([[0, 0, 0]], [[0, 0, 1.0]])
    steps = 8
    en, sol, sq, surf = contact_pair(X, T, planes=planes, disks=disks, dt=DT, E=E, nu=0.45, rho=1000.0)
    disk = ps.get_disk_contact_constraint(en, 1)

    def center(t):
        return c0 - np.array([0, 0, 0.08 * DT * t])

    w = rng.standard_normal(X.size)
    Et = torch.tensor(E, requires_grad=True)
    qT = rollout(en, sol, Et, None, steps, DT, poisson=0.45, checkpoint_every=3,
                 before_step=lambda t: disk.set_disk(center(t), [0, 0, -1.0], 0.004))
    (torch.tensor(w) * qT).sum().backward()

    def L(Ev):
        def before(t, s):
            s.disks.set_disk(center(t), [0, 0, -1.0], 0.004)
        from oracle import oracle as orc
        q, held, _ = _oracle_rollout_rho(X, T, Ev, steps, before, disks, planes)
        return float(w @ q), held

    l0, held = L(E)
    assert held > 0
    assert abs(float(w @ qT.detach().numpy()) - l0) < 1e-9 * np.abs(w).sum()
    gE = Et.grad.numpy()
    h = 1e-6
    for _ in range(3):
        r = rng.standard_normal(ne)
        d_fd = (L(E * (1 + h * r))[0] - L(E * (1 - h * r))[0]) / (2 * h)
        assert abs(gE @ (E * r) - d_fd) <= 1e-4 * abs(d_fd) + 1e-14, (gE @ (E * r), d_fd)


def _oracle_rollout_rho(X, T, E, steps, before, disks, planes):
    from oracle import oracle as orc
    from oracle import contact as oc
    groups, _ = meshes.extract_surfaces(X, T)
    surf = np.unique(np.concatenate([g.ravel() for g in groups]))
    o = orc.System(X, T, rho=1000.0, youngs=E, nu=0.45, grav=(0, 0, -9.81), scheme="backward_euler",
                   method="minimize_SQP", dt=DT, substeps=1)
    sq = oc.SQPOracle(o, oc.PlaneContact(planes[0], planes[1], surf),
                      oc.DiskContact(disks[0], disks[1], disks[2], surf))
    q = X.ravel().copy()
    held = 0
    for t in range(steps):
        before(t, sq)
        q = sq.step(q, DT)
        held += sq.last_active
    return q, held, o.mass()
