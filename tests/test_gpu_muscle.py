"""SoftCon fibre terms (cpp/src/energies/softconMuscle.cpp) on the GPU against the oracle.

The GPU path uses the energy k/2 (|F m| - (1 - e))^2, whose gradient is the
reference's gradient, with its exact Hessian; the oracle is run in the same
(consistent) form.  Element quantities agree to 1e-10 relative; trajectories to
the displacement tolerances stated per test.
"""
import numpy as np
import pytest

from sors_b200 import meshes
from tests.helpers import deform, make_pair, rel_err

pytestmark = pytest.mark.gpu


def _hex_bar():
    X, H = meshes.hex_bar(8, 2, 2, (0.04, 0.01, 0.01))
    return X, H


def _muscles(ne, rng, frac=1.0):
    group = np.where(rng.uniform(size=ne) < frac, np.arange(ne), -1).astype(np.int32)
    k = rng.uniform(2e4, 2e5, ne)
    d = rng.standard_normal((ne, 3))
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    return {"group": group, "k": k, "dir": d}


@pytest.mark.parametrize("kind", ["tet", "hex"])
@pytest.mark.parametrize("project", [False, True])
def test_muscle_element_parity(oracle, kind, project):
    from sors_b200 import py_sors as ps
    if kind == "tet":
        X, T = meshes.cantilever_tets(4, 2, 2, (0.02, 0.01, 0.01))
    else:
        X, T = _hex_bar()
    rng = np.random.default_rng(3)
    ne = T.shape[0]
    mus = _muscles(ne, rng, frac=0.7)
    en, _, _, _ = make_pair(X, T, E=2e5, nu=0.45, project=project, clamp=False, muscles=mus)
    act = rng.uniform(0.0, 1.0, ne)
    en._apply_actuation(ps.Params(["softconMuscle"], [act.reshape(-1, 1)]))
    for trial in range(2):
        q = deform(X, rng, amp=0.1)
        psi, g, H = en.compute_element_data(q, project=project)
        x = q.reshape(-1, 3)
        for e in range(ne):
            Xe, xe = X[T[e]], x[T[e]]
            if mus["group"][e] >= 0:
                opsi, og, oH, st = oracle.elem_eval_muscle(Xe, xe, 2e5, 0.45, mus["k"][e], mus["dir"][e], act[e],
                                                           form=oracle.MUSCLE_CONSISTENT, project=project)
            else:
                opsi, og, oH, st = oracle.elem_eval(Xe, xe, 2e5, 0.45, project=project)
            assert st == 0
            assert abs(psi[e] - opsi) <= 1e-10 * abs(opsi) + 1e-14
            assert rel_err(g[e], og) < 1e-10
            tol = 1e-9 if project else 1e-10
            assert np.abs(H[e] - oH).max() <= tol * np.abs(oH).max()


def test_softcon_contraction(golden, oracle):
    # TestCube::test_softcon_muscle (cpp/src/_test.cpp:563-625): the first two
    # tets of the 5-tet cube carry fibres along z, all actuations ramp as
    # 2 i / 10, BE dt = 0.01, no gravity; the cube's z-extent must shrink.
    from sors_b200 import py_sors as ps
    d = golden["test_cube"]
    X = np.array(d["vertices"], float); T = np.array(d["elements"], np.int32)
    ne = T.shape[0]
    mus = {"group": np.array([0, 1] + [-1] * (ne - 2), np.int32), "k": np.full(ne, 1e5),
           "dir": np.tile([0.0, 0.0, 1.0], (ne, 1))}
    en, sol, o, s = make_pair(X, T, rho=1000.0, E=1e6, nu=0.4, grav=(0, 0, 0), dt=d["dt"], clamp=False,
                              project=False, muscles=mus)
    q = X.ravel().copy(); qo = q.copy()
    for i in range(1, 10):
        act = np.full((ne, 1), 2.0 * i / 10)
        q = sol.step(q, en, ps.Params(["softconMuscle"], [act]))
        o.set_muscle_act(act.ravel()[:2])
        qo, st = o.step(qo)
        assert st == 0
    z0 = X[:, 2].max() - X[:, 2].min()
    z1 = q.reshape(-1, 3)[:, 2].max() - q.reshape(-1, 3)[:, 2].min()
    assert z1 < z0
    assert np.abs(q - qo).max() < 1e-9


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_muscle_hex_trajectory(oracle, precision):
    # fibre +x in every hex, per-element activation U[0,1] redrawn every step,
    # gravity, x = 0 clamped, BE dt = 2e-3.
    from sors_b200 import py_sors as ps
    X, T = _hex_bar()
    ne = T.shape[0]
    rng = np.random.default_rng(7)
    mus = {"group": np.arange(ne, dtype=np.int32), "k": np.full(ne, 5e4), "dir": np.tile([1.0, 0, 0], (ne, 1))}
    en, sol, o, s = make_pair(X, T, rho=1070.0, E=2e5, nu=0.45, dt=2e-3, precision=precision, muscles=mus,
                              res_tol=1e-9 if precision == "mixed" else 0.0)
    q = X.ravel().copy(); qo = q.copy()
    for step in range(15):
        act = rng.uniform(0, 1, ne)
        q = sol.step(q, en, ps.Params(["softconMuscle"], [act.reshape(-1, 1)]))
        o.set_muscle_act(act)
        qo, st = o.step(qo)
        assert st == 0
    disp = np.abs(qo - X.ravel()).max()
    err = np.abs(q - qo).max()
    assert disp > 1e-5
    assert err <= (1e-9 if precision == "fp64" else 1e-6 * disp), (err, disp)
