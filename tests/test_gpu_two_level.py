"""Two-level PCG preconditioner (block Jacobi + exact coarse correction on
per-aggregate rigid-body modes): same Newton roots as block Jacobi alone,
fewer PCG iterations, bit-reproducible runs."""
import numpy as np
import pytest

from sors_b200 import meshes
from tests.helpers import make_pair

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_two_level_block_trajectory(oracle, precision):
    # a jittered 6-tet block large enough for several aggregates (12k nodes)
    X, T, E = meshes.jittered_block_tets(40, 10, 10, (0.4, 0.1, 0.1), seed=2)
    runs = {}
    for tl in (False, True):
        en, sol, o, s = make_pair(X, T, E=E, nu=0.45, dt=5e-3, precision=precision, two_level=tl,
                                  res_tol=1e-9 if precision == "mixed" else 0.0)
        q = X.ravel().copy()
        pcg = 0
        for _ in range(4):
            q = sol.step(q, en)
            pcg += sol.last_stats.pcg_iters
        runs[tl] = (q, pcg)
    (q0, it0), (q1, it1) = runs[False], runs[True]
    disp = np.abs(q0 - X.ravel()).max()
    assert disp > 1e-4
    assert np.abs(q1 - q0).max() <= (1e-9 if precision == "fp64" else 1e-6 * disp)
    assert it1 < it0, (it1, it0)


def test_two_level_c1_matches_oracle(c1_mesh, oracle):
    X, T = c1_mesh
    en, sol, o, s = make_pair(X, T, two_level=True)
    q = X.ravel().copy(); qo = q.copy()
    for _ in range(30):
        q = sol.step(q, en)
        qo, st = o.step(qo)
        assert st == 0
    assert np.abs(q - qo).max() < 1e-8


def test_two_level_deterministic():
    X, T, E = meshes.jittered_block_tets(24, 8, 8, (0.24, 0.08, 0.08), seed=4)
    outs = []
    for _ in range(2):
        en, sol, o, s = make_pair(X, T, E=E, two_level=True, precision="mixed", res_tol=1e-9)
        q = X.ravel().copy()
        for _ in range(3):
            q = sol.step(q, en)
        outs.append(q)
    np.testing.assert_array_equal(outs[0], outs[1])


@pytest.fixture(scope="module")
def c1_mesh():
    return meshes.cantilever_tets()


def test_two_level_with_contact():
    # SQP subproblems run the projected PCG; the two-level correction is
    # projected as well and must give the same contact step as block Jacobi
    X, H = meshes.hex_bar(12, 6, 6, (0.03, 0.015, 0.015))
    X = X + np.array([0.0, 0.0, 0.0003])
    from tests.helpers import contact_pair
    out = {}
    for tl in (False, True):
        en, sol, sq, surf = contact_pair(X, H, planes=([[0, 0, 0]], [[0, 0, 1.0]]), dt=2e-3, two_level=tl)
        x = X.ravel().copy()
        pcg = 0
        for _ in range(10):
            x = sol.step(x, en)
            pcg += sol.last_stats.pcg_iters
        out[tl] = (x, pcg, en.active_contacts())
    assert out[True][2] == out[False][2] and out[True][2] > 0
    assert np.abs(out[True][0] - out[False][0]).max() < 1e-9
