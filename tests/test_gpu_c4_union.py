"""Several differentiated rollouts in one union handle (the C4 batching).

bench.py's c4 workload differentiates 64 activation seeds of the SoftCon hex
bar in one union handle: the copies share no element, so the union's SQP
steps, contacts and adjoint are the direct sum of the copies'.  Here a union
of three copies of a small bar, each with its own activations and Young's
moduli, is dropped onto z = 0 (planeContact, minimize_SQP) and differentiated
once; each copy's final state must equal its rollout alone, and its gradient
must match central differences of the ORACLE's SQP forward (FP64, h = 1e-6
relative) along a seeded direction.
"""
import numpy as np
import pytest

import bench
from sors_b200 import meshes
from tests.test_gpu_adjoint_contact import DT, _bar, _oracle_rollout

pytestmark = pytest.mark.gpu

STEPS = 14
SEEDS = 3


def test_union_adjoint_matches_oracle_fd():
    import torch
    from sors_b200.adjoint import RolloutAdjoint
    torch.cuda.set_device(0)
    X, T = _bar()
    n1, e1 = X.shape[0], T.shape[0]
    groups, _ = meshes.extract_surfaces(X, T)
    surf = np.unique(np.concatenate([g.ravel() for g in groups])).astype(np.int32)
    rng = np.random.default_rng(21)
    Es = [np.exp(rng.uniform(np.log(1e5), np.log(3e5), e1)) for _ in range(SEEDS)]
    acts = [rng.uniform(0, 1, (STEPS, e1)) for _ in range(SEEDS)]
    mus = {"group": np.arange(e1, dtype=np.int32), "k": np.full(e1, 5e4), "dir": np.tile([1.0, 0, 0], (e1, 1))}
    mass = None

    def oracle_loss(E, act):
        nonlocal mass
        q, held, mass = _oracle_rollout(X, T, E, act, mus, STEPS, planes=([[0, 0, 0]], [[0, 0, 1.0]]))
        m = mass[2::3]
        return ((q[2::3] * m).sum() / m.sum() - 0.004) ** 2, q, held

    refs = [oracle_loss(Es[k], acts[k]) for k in range(SEEDS)]
    assert all(r[2] > 0 for r in refs)  # every copy touched the plane
    m = mass[2::3]
    # union handle of the three copies (bench.c4_energy builds it), one forward and one backward
    en, sol = bench.c4_energy(X, T, np.concatenate(Es), surf, members=SEEDS)
    r = RolloutAdjoint(en, sol, STEPS, DT, poisson=0.45, checkpoint_every=5)
    qT = r.forward(np.concatenate(Es), np.concatenate(acts, axis=1)).reshape(SEEDS, n1, 3)
    for k in range(SEEDS):
        assert np.abs(qT[k].ravel() - refs[k][1]).max() < 1e-8
    z = (qT[:, :, 2] * m).sum(axis=1) / m.sum()
    dq = np.zeros((SEEDS, n1, 3))
    dq[:, :, 2] = (2 * (z - 0.004))[:, None] * m[None, :] / m.sum()
    gE, gA, _, _ = r.backward(dq.ravel())
    h = 1e-6
    for k in (0, SEEDS - 1):
        rE = rng.standard_normal(e1); rA = rng.standard_normal((STEPS, e1))
        d_adj = gE[k * e1:(k + 1) * e1] @ (Es[k] * rE) + (gA[:, k * e1:(k + 1) * e1] * rA).sum()
        lp = oracle_loss(Es[k] * (1 + h * rE), acts[k] + h * rA)[0]
        lm = oracle_loss(Es[k] * (1 - h * rE), acts[k] - h * rA)[0]
        d_fd = (lp - lm) / (2 * h)
        assert abs(d_adj - d_fd) <= 1e-4 * abs(d_fd) + 1e-16, (k, d_adj, d_fd)
