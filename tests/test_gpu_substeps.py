"""Substepping and the CFL time step of Solver::step (cpp/src/solver.cpp:5-44,
300-331) on the GPU against the oracle.

With CFLtimeSteppingFlag the step is split into ceil(dt / dt_CFL) substeps,
dt_CFL = (shortest element edge at q) / max |v_prev| (Courant number 1,
Element::compute_minimal_edge_length, cpp/headers/geometries/element.h:131-142).
"""
import numpy as np
import pytest

from sors_b200 import meshes
from tests.helpers import make_pair

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def c1():
    return meshes.cantilever_tets()


def _cfl_substeps(q, v, T, dt):
    """ceil(dt / min(dt, l_min / max|v|)) with the element edges at q."""
    x = q.reshape(-1, 3)[T]
    lmin = min(np.linalg.norm(x[:, i] - x[:, j], axis=1).min() for i in range(4) for j in range(i + 1, 4))
    vmax = np.abs(v).max()
    dtc = lmin / vmax if vmax > 0 else np.inf
    return int(np.ceil(dt / min(dt, dtc)))


def test_fixed_substeps(c1, oracle):
    """Clamped cantilever, dt = 3e-3 split into 3 backward-Euler substeps."""
    X, T = c1
    en, sol, o, _ = make_pair(X, T, dt=3e-3, substeps=3)
    q = X.ravel().copy(); qo = q.copy()
    for _ in range(8):
        q = sol.step(q, en)
        assert sol.last_stats.substeps == 3
        qo, st = o.step(qo)
        assert st == 0
    assert np.abs(qo - X.ravel()).max() > 1e-5
    assert np.abs(q - qo).max() < 1e-8


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_cfl_substeps_spinning_beam(c1, oracle, precision):
    """Free cantilever beam spun about its centre (25 rad/s about z: |v_y| up
    to 1.25 m/s at the tips) with 5 mm edges: dt = 1e-2 needs
    ceil(1e-2 / 4e-3) = 3 substeps in the first step.  Every step's substep
    count follows the CFL rule on the oracle's state, and the trajectory
    follows the oracle."""
    X, T = c1
    en, sol, o, _ = make_pair(X, T, dt=1e-2, clamp=False, cfl=True, precision=precision)
    c = X.mean(axis=0)
    w = np.array([0.0, 0.0, 25.0])
    v0 = np.cross(w, X - c).ravel()
    en.set_initial_velocity(v0.reshape(-1, 3))
    o.set_initial_velocity(v0)
    q = X.ravel().copy(); qo = q.copy()
    counts = []
    worst = disp = 0.0
    for _ in range(6):
        _, vprev, _ = o.state()
        expect = _cfl_substeps(qo, vprev, T, 1e-2)
        q = sol.step(q, en)
        counts.append(sol.last_stats.substeps)
        assert counts[-1] == expect, (counts, expect)
        qo, st = o.step(qo)
        assert st == 0
        worst = max(worst, float(np.abs(q - qo).max()))
        disp = max(disp, float(np.abs(qo - X.ravel()).max()))
    assert counts[0] == 3, counts
    if precision == "fp64":
        assert worst < 1e-8, worst
    else:
        assert worst <= 1e-6 * disp, (worst, disp)
