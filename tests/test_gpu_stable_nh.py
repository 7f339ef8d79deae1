"""Stable Neo-Hookean elements (cpp/src/energies/stableNeoHookean.cpp) on the
GPU against the oracle: element energy, gradient and Hessian to 1e-10
relative (projected Hessians 1e-9), inverted elements included; trajectories
to 1e-9 m (FP64) and 1e-6 of the displacement (mixed)."""
import numpy as np
import pytest

from sors_b200 import meshes
from tests.helpers import deform, make_pair, rel_err

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", ["tet", "hex"])
@pytest.mark.parametrize("project", [False, True])
def test_stable_nh_element_parity(oracle, kind, project):
    if kind == "tet":
        X, T = meshes.cantilever_tets(4, 2, 2, (0.02, 0.01, 0.01))
    else:
        X, T = meshes.hex_bar(4, 2, 2, (0.02, 0.01, 0.01))
    rng = np.random.default_rng(9)
    ne = T.shape[0]
    E = rng.uniform(5e4, 5e5, ne)
    nu = rng.uniform(0.3, 0.48, ne)
    en, _, _, _ = make_pair(X, T, E=E, nu=nu, project=project, clamp=False, energy="stableneohookean")
    for trial in range(3):
        q = deform(X, rng, amp=0.15 if trial < 2 else 0.6)   # the last draw inverts some elements
        psi, g, H = en.compute_element_data(q, project=project)
        x = q.reshape(-1, 3)
        for e in range(ne):
            opsi, og, oH, st = oracle.elem_eval_material(X[T[e]], x[T[e]], E[e], nu[e],
                                                         oracle.MAT_STABLE_NEOHOOKEAN, project=project)
            assert st == 0
            assert abs(psi[e] - opsi) <= 1e-10 * abs(opsi) + 1e-14
            assert rel_err(g[e], og) < 1e-10
            tol = 1e-9 if project else 1e-10
            assert np.abs(H[e] - oH).max() <= tol * np.abs(oH).max(), e


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_stable_nh_cantilever(oracle, precision):
    X, T = meshes.cantilever_tets()
    en, sol, o, s = make_pair(X, T, E=1e5, nu=0.45, dt=1e-3, precision=precision, energy="stableneohookean",
                              res_tol=1e-9 if precision == "mixed" else 0.0)
    q = X.ravel().copy(); qo = q.copy()
    for _ in range(40):
        q = sol.step(q, en)
        qo, st = o.step(qo)
        assert st == 0
    disp = np.abs(qo - X.ravel()).max()
    err = np.abs(q - qo).max()
    assert disp > 1e-4
    assert err <= (1e-9 if precision == "fp64" else 1e-6 * disp), (err, disp)
