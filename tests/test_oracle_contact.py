"""Oracle of the contact step (oracle/contact.py) on the CPU: the reference's
own contact test (cpp/src/_test.cpp:629-697) and KKT properties of the SQP."""
import numpy as np
import pytest


def test_plane_contact_no_penetration_oracle(golden):
    # TestConstraint::test_plane_contact_no_penetration: one SQP step of a tet
    # whose vertex 0 starts 0.1 below the plane z = 0.
    from oracle import oracle as orc
    from oracle import contact as oc
    d = golden["test_constraint"]
    X = np.array(d["vertices"]); T = np.array([[0, 1, 2, 3]])
    o = orc.System(X, T, rho=1.0, youngs=1e5, nu=0.3, grav=(0, 0, -9.81), scheme="backward_euler",
                   method="minimize_SQP", dt=1e-2, substeps=1, nthreads=1)
    pl = oc.PlaneContact([[0, 0, 0]], [[0, 0, 1.0]], [0, 1, 2, 3])
    sq = oc.SQPOracle(o, pl)
    x = sq.step(X.ravel(), 1e-2)
    assert (x.reshape(-1, 3)[:, 2] >= -d["tol"]).all()


def test_cube_drop_kkt():
    # a hex cube dropped onto z = 0: every active contact holds after each step
    from oracle import oracle as orc
    from oracle import contact as oc
    from sors_b200 import meshes
    X, T = meshes.hex_bar(3, 3, 3, (0.01, 0.01, 0.01))
    X = X + np.array([0, 0, 0.0004])
    groups, _ = meshes.extract_surfaces(X, T)
    surf = np.unique(np.concatenate([g.ravel() for g in groups]))
    o = orc.System(X, T, rho=1070.0, youngs=1e5, nu=0.45, grav=(0, 0, -9.81), scheme="backward_euler",
                   method="minimize_SQP", dt=2e-3, substeps=1, nthreads=2)
    sq = oc.SQPOracle(o, oc.PlaneContact([[0, 0, 0]], [[0, 0, 1.0]], surf))
    x = X.ravel().copy()
    touched = False
    for _ in range(15):
        x = sq.step(x, 2e-3)
        touched |= sq.last_active > 0
        assert x.reshape(-1, 3)[surf, 2].min() > -1e-9
    assert touched
