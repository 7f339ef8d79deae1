"""Contact step on the GPU (minimize_SQP with planeContact / diskContact)
against the oracle's SQP (oracle/contact.py, exact QP solves).

Trajectories agree to 1e-8 m in FP64; mixed precision to 1e-6 of the
displacement.  The active contact sets agree step by step.
"""
import numpy as np
import pytest

from sors_b200 import meshes
from tests.helpers import contact_pair

pytestmark = pytest.mark.gpu


def test_plane_contact_no_penetration(golden):
    # TestConstraint::test_plane_contact_no_penetration (cpp/src/_test.cpp:629-697)
    d = golden["test_constraint"]
    X = np.array(d["vertices"]); T = np.array([[0, 1, 2, 3]])
    en, sol, sq, surf = contact_pair(X, T, planes=([[0, 0, 0]], [[0, 0, 1.0]]), surface=[0, 1, 2, 3], rho=1.0,
                                     E=1e5, nu=0.3, dt=1e-2)
    x = sol.step(X.ravel().copy(), en)
    assert (x.reshape(-1, 3)[:, 2] >= -d["tol"]).all()
    xo = sq.step(X.ravel().copy(), 1e-2)
    assert np.abs(x - xo).max() < 1e-9


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_drop_on_plane(precision, kind):
    X, H = meshes.hex_bar(4, 3, 3, (0.012, 0.009, 0.009))
    T = H if kind == "hex" else meshes.kuhn_tet_elements(4, 3, 3)
    X = X + np.array([0.0, 0.0, 0.0003])
    en, sol, sq, surf = contact_pair(X, T, planes=([[0, 0, 0]], [[0, 0, 1.0]]), dt=2e-3, precision=precision)
    x = X.ravel().copy(); xo = x.copy()
    touched = 0
    for step in range(20):
        x = sol.step(x, en)
        xo = sq.step(xo, 2e-3)
        assert en.active_contacts() == sq.last_active
        touched += sq.last_active
        assert x.reshape(-1, 3)[surf, 2].min() > -1e-8
    assert touched > 0
    disp = np.abs(xo - X.ravel()).max()
    err = np.abs(x - xo).max()
    assert err <= (1e-8 if precision == "fp64" else 1e-6 * disp), (err, disp)


def test_disk_poke_on_ground():
    # a tet cube resting on z = 0, pressed by a disk (r = 4 mm) moving down at 0.05 m/s
    X, _ = meshes.hex_bar(5, 5, 5, (0.01, 0.01, 0.01))
    T = meshes.kuhn_tet_elements(5, 5, 5)
    dt = 2e-3
    top = 0.01
    center = np.array([0.005, 0.005, top + 0.0002])
    en, sol, sq, surf = contact_pair(X, T, planes=([[0, 0, 0]], [[0, 0, 1.0]]),
                                     disks=([center], [[0, 0, -1.0]], [0.004]), dt=dt, E=5e4, nu=0.4, rho=1000.0)
    from sors_b200 import py_sors as ps
    disk = ps.get_disk_contact_constraint(en, 1)
    x = X.ravel().copy(); xo = x.copy()
    for step in range(12):
        c = center - np.array([0, 0, 0.05 * dt * step])
        disk.set_disk(c, [0, 0, -1.0], 0.004)
        sq.disks.set_disk(c, [0, 0, -1.0], 0.004)
        x = sol.step(x, en)
        xo = sq.step(xo, dt)
        assert en.active_contacts() == sq.last_active
    assert np.abs(x - xo).max() < 1e-8
    # the disk pushed the top down
    assert x.reshape(-1, 3)[:, 2].max() < top


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_drop_within_osqp_tolerance_of_reference_qp(kind):
    # The reference solves each SQP subproblem with OSQP (max_iter 250, absolute
    # tolerance 1e-3, solver.cpp:116-176), restated in oracle/contact.py.  The
    # device solves the subproblem exactly: its contacts stay on the plane, the
    # OSQP-restated step leaves them up to the tolerance below it, and the two
    # trajectories differ by less than that tolerance.
    from oracle import contact as oc
    X, H = meshes.hex_bar(4, 3, 3, (0.012, 0.009, 0.009))
    T = H if kind == "hex" else meshes.kuhn_tet_elements(4, 3, 3)
    X = X + np.array([0.0, 0.0, 0.0003])
    en, sol, sq, surf = contact_pair(X, T, planes=([[0, 0, 0]], [[0, 0, 1.0]]), dt=2e-3)
    sq.qp = "osqp"
    x = X.ravel().copy(); xo = x.copy()
    worst = 0.0
    for step in range(20):
        x = sol.step(x, en)
        xo = sq.step(xo, 2e-3)
        worst = max(worst, float(np.abs(x - xo).max()))
        assert x.reshape(-1, 3)[surf, 2].min() > -1e-9
        assert xo.reshape(-1, 3)[surf, 2].min() > -oc.OSQP_EPS_ABS
    assert worst < oc.OSQP_EPS_ABS
