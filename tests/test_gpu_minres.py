"""MINRES Newton solves of the exact (indefinite) Hessian against the oracle.

The reference solves every Newton system with LDL^T (cpp/src/solver.cpp:65-84),
indefinite ones included.  CG cannot; `linearSolver = "minres"` takes the same
exact Newton step on the device.  The cases: a bar compressed by 10 % between
two clamped ends and stepped dynamically (its first Newton iterates have four
or five negative eigenvalues, and the oracle's LDL^T Newton converges in 6-8
iterations), and the short chamber cylinder under follower pressure."""
from __future__ import annotations

import numpy as np
import pytest

from sors_b200 import meshes

pytestmark = pytest.mark.gpu


def _compressed_bar(comp=0.1, pert=1e-4, L=0.08):
    X, T = meshes.cantilever_tets(8, 2, 2, (L, 0.02, 0.02))
    N = X.shape[0]
    mask = np.zeros(3 * N, np.int32)
    ends = (np.abs(X[:, 0]) < 1e-12) | (np.abs(X[:, 0] - L) < 1e-12)
    mask[np.repeat(ends, 3)] = 1
    rng = np.random.default_rng(0)
    q0 = (X * np.array([1 - comp, 1, 1])).ravel() + pert * rng.standard_normal(3 * N) * (1 - mask)
    return X, T, mask, q0


def _hessian_min_eig(o, q, dt):
    import scipy.sparse as sp
    A, _ = o.hessian_csr(q, dt)
    A = (sp.tril(A) + sp.tril(A, -1).T).toarray()   # the lower triangle defines the operator
    return np.linalg.eigvalsh(A)[0]


@pytest.mark.parametrize("precision,two_level", [("fp64", False), ("fp64", True), ("mixed", False)])
def test_minres_indefinite_steps_match_oracle(oracle, precision, two_level):
    from sors_b200 import py_sors as ps
    X, T, mask, q0 = _compressed_bar()
    dt = 1e-2
    o = oracle.System(X, T, rho=1000.0, youngs=1e5, nu=0.45, grav=(0, 0, 0), dt=dt, scheme="backward_euler")
    o.set_neumann(mask, np.zeros(mask.size))
    o.set_initial_deformation(q0)
    assert _hessian_min_eig(o, q0, dt) < -100.0   # the first Newton system is indefinite

    s = ps.SimulationSettings()
    s.meshType = "Tetrahedron"; s.dt = dt; s.timeSteppingScheme = "backward_euler"
    s.precision = precision; s.hessianProjection = False; s.linearSolver = "minres"
    s.twoLevelPreconditioner = two_level; s.newtonResidualTol = 1e-10
    ne = T.shape[0]
    params = [ps.Params(["density", "youngsModulus", "poissonsRatio"], [1000.0, 1e5, 0.45])] * ne
    cp = ps.Params(["neumannBCmask", "neumannBCvalue"], [mask.astype(float), np.zeros(mask.size)])
    en = ps.Energy(X, T, s, np.zeros(3), 0.0, [{"neohookean"}] * ne, params, ["neumannBC"], cp, [], ps.Params())
    en.set_initial_deformation(q0)
    sol = ps.Solver(s)
    q, qo = q0.copy(), q0.copy()
    for _ in range(3):
        qo, st = o.step(qo, dt=dt)
        assert st == 0
        q = sol.step(q, en)
        assert sol.last_stats.newton_iters >= 2
    u = np.abs(qo - q0).max()
    assert u > 1e-4
    tol = 1e-8 if precision == "fp64" else 1e-6 * u
    assert np.abs(q - qo).max() < tol, np.abs(q - qo).max()


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_minres_c3_chamber_pressure_matches_oracle(oracle, precision):
    """The short chamber cylinder under follower pressure (hexes, dt = 0) with
    the exact Hessian, as the reference solves it."""
    from sors_b200 import py_sors as ps
    X, H = meshes.voxel_cylinder(length=0.015, h=2.5e-3, cap_layers=2)
    groups, _ = meshes.extract_surfaces(X, H)
    faces = np.concatenate(groups)
    gid = np.concatenate([np.full(len(g), k) for k, g in enumerate(groups)])
    ng = len(groups)
    mask = np.repeat((np.abs(X[:, 2]) < 1e-12).astype(np.int32), 3)
    o = oracle.System(X, H, rho=1070.0, youngs=3e5, nu=0.48, grav=(0, 0, 0), dt=0.0)
    o.set_neumann(mask, np.zeros(mask.size)); o.set_pressure(faces, gid)
    s = ps.SimulationSettings()
    s.meshType = "Hexahedron"; s.dt = 0.0; s.timeSteppingScheme = "backward_euler"
    s.precision = precision; s.newtonResidualTol = 1e-10
    s.hessianProjection = False; s.linearSolver = "minres"
    ne = H.shape[0]
    params = [ps.Params(["density", "youngsModulus", "poissonsRatio"], [1070.0, 3e5, 0.48])] * ne
    cp = ps.Params(["neumannBCmask", "neumannBCvalue"], [mask.astype(float), np.zeros(mask.size)])
    fp = ps.Params(["surfaceVertexIdx", "surfaceGroups"], [faces.astype(float), gid.astype(float)])
    en = ps.Energy(X, H, s, np.zeros(3), 0.0, [{"neohookean"}] * ne, params, ["neumannBC"], cp, ["pressure"], fp)
    sol = ps.Solver(s)
    q, qo = X.ravel().copy(), X.ravel().copy()
    for level in (1, 2, 3):
        pr = np.zeros(ng); pr[1] = 5e3 * level
        qo, st = o.step(qo, dt=0.0, pressure=pr)
        assert st == 0
        q = sol.step(q, en, ps.Params(["pressure"], [pr.reshape(-1, 1)]), 0.0)
    u = np.abs(qo - X.ravel()).max()
    assert u > 1e-5
    tol = 1e-8 if precision == "fp64" else 1e-6 * u
    assert np.abs(q - qo).max() < tol, np.abs(q - qo).max()


def test_exact_quad_pressure_jacobian_same_solution(oracle):
    """pressureJacobian = "exact" (p/8 for quads in the Newton matrix) changes
    the Newton iterates, not the solution: the chamber cylinder ends where the
    oracle's LDL^T Newton with the reference's p/6 ends."""
    from sors_b200 import py_sors as ps
    X, H = meshes.voxel_cylinder(length=0.015, h=2.5e-3, cap_layers=2)
    groups, _ = meshes.extract_surfaces(X, H)
    faces = np.concatenate(groups)
    gid = np.concatenate([np.full(len(g), k) for k, g in enumerate(groups)])
    ng = len(groups)
    mask = np.repeat((np.abs(X[:, 2]) < 1e-12).astype(np.int32), 3)
    o = oracle.System(X, H, rho=1070.0, youngs=3e5, nu=0.48, grav=(0, 0, 0), dt=0.0)
    o.set_neumann(mask, np.zeros(mask.size)); o.set_pressure(faces, gid)
    s = ps.SimulationSettings()
    s.meshType = "Hexahedron"; s.dt = 0.0; s.timeSteppingScheme = "backward_euler"
    s.precision = "fp64"; s.newtonResidualTol = 1e-10; s.pressureJacobian = "exact"
    ne = H.shape[0]
    params = [ps.Params(["density", "youngsModulus", "poissonsRatio"], [1070.0, 3e5, 0.48])] * ne
    cp = ps.Params(["neumannBCmask", "neumannBCvalue"], [mask.astype(float), np.zeros(mask.size)])
    fp = ps.Params(["surfaceVertexIdx", "surfaceGroups"], [faces.astype(float), gid.astype(float)])
    en = ps.Energy(X, H, s, np.zeros(3), 0.0, [{"neohookean"}] * ne, params, ["neumannBC"], cp, ["pressure"], fp)
    sol = ps.Solver(s)
    q, qo = X.ravel().copy(), X.ravel().copy()
    for level in (1, 2, 3):
        pr = np.zeros(ng); pr[1] = 5e3 * level
        qo, st = o.step(qo, dt=0.0, pressure=pr)
        assert st == 0
        q = sol.step(q, en, ps.Params(["pressure"], [pr.reshape(-1, 1)]), 0.0)
    assert np.abs(qo - X.ravel()).max() > 1e-5
    assert np.abs(q - qo).max() < 1e-8, np.abs(q - qo).max()
