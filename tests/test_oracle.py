"""The CPU oracle pinned against the reference's own known answers.

Fixtures come from the reference tests (cpp/src/_test.cpp, parsed into
tests/golden/reference_known_answers.json) and, for the Neo-Hookean formulas,
from torch autograd in FP64 (the method of python/_autodiff_check.py).
"""
import numpy as np
import pytest
import torch

pytestmark = []


def _quartic_system(oracle, golden, dt=0.0, method="minimize_newton"):
    d = golden["test_energy"]
    X = np.array(d["vertices"]); T = np.array(d["elements"])
    return oracle.System(X, T, rho=1.0, youngs=1.0, nu=0.3, grav=(0, 0, 0), method=method,
                         material=oracle.MAT_TEST_QUARTIC, nthreads=1), X


def test_energy_known_answers(oracle, golden):
    # TestEnergy::test_energy / test_gradient / test_hessian (cpp/src/_test.cpp:136-176)
    d = golden["test_energy"]
    sysm, X = _quartic_system(oracle, golden)
    q = X.ravel()
    assert sysm.energy(q, 0.0) == d["energy"]
    g = sysm.gradient(q, 0.0)
    np.testing.assert_allclose(g, np.array(d["gradient"]).ravel(), rtol=1e-12, atol=1e-12)
    H, st = sysm.hessian_dense(q, 0.0)
    assert st == 0
    np.testing.assert_allclose(H, np.diag(np.array(d["hessian_diag"]).ravel()), rtol=1e-12, atol=1e-12)


def test_optimization_known_answer(oracle, golden):
    # TestOptimization::test_optimization (cpp/src/_test.cpp:180-199): Newton at dt=1
    d = golden["test_energy"]
    sysm, X = _quartic_system(oracle, golden)
    q, st = sysm.minimize(X.ravel(), dt=d["optimization_dt"])
    assert st == 0
    g = sysm.gradient(q, d["optimization_dt"])
    assert float(g @ g) < d["tol"]


def test_tetrahedron_dFdx(oracle, golden):
    # TestTetrahedron::test_deformationHessian (cpp/src/_test.cpp:217-235)
    d = golden["test_tetrahedron"]
    B, inv, vol = oracle.tet_init(np.array(d["undeformed"]))
    np.testing.assert_allclose(B, np.array(d["dFdx"]), atol=0, rtol=0)
    assert abs(vol - 1.0 / 6.0) < 1e-15


def test_tetrahedron_rest(oracle, golden):
    # test_energy_zero / test_gradient_zero (cpp/src/_test.cpp:238-286), TOL 1e-9
    d = golden["test_tetrahedron"]
    X = np.array(d["undeformed"])
    m = d["material"]
    psi, g, H, st = oracle.elem_eval(X, X, m["youngsModulus"], m["poissonsRatio"])
    assert abs(psi) < d["tol"]
    assert np.abs(g).max() < d["tol"]


# --- Neo-Hookean formulas against torch autograd (FP64) --------------------

def _torch_nh(X, x, E, nu):
    """Psi*V for a tet (1 qp) or hex (8 qp, weights 1/8, 5-tet volume)."""
    from oracle import oracle as orc
    nv = X.shape[0]
    lam = E * nu / ((1 + nu) * (1 - 2 * nu)); mu = E / (2 * (1 + nu))
    xt = torch.tensor(x, dtype=torch.float64, requires_grad=True)
    if nv == 4:
        Dm = torch.tensor((X[:3] - X[3]).T)
        Ds = (xt[:3] - xt[3]).T
        Fs = [Ds @ torch.linalg.inv(Dm)]
        V = abs(np.linalg.det(X[:3] - X[3])) / 6
    else:
        G, _, V = orc.hex_init(X)
        Fs = [xt.T @ torch.tensor(G[s]) for s in range(8)]
    psi = 0
    for F in Fs:
        J = torch.det(F); lJ = torch.log(J)
        psi = psi + (0.5 * mu * ((F * F).sum() - 3) - mu * lJ + 0.5 * lam * lJ * lJ) / len(Fs)
    return psi * V, xt


@pytest.mark.parametrize("nv", [4, 8])
def test_neohookean_vs_autograd(oracle, nv):
    rng = np.random.default_rng(7 + nv)
    if nv == 4:
        X = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float) * 0.01 + rng.uniform(-1e-3, 1e-3, (4, 3))
    else:
        from sors_b200.meshes import hex_grid_elements, grid_nodes
        X = grid_nodes(1, 1, 1, (0.01, 0.012, 0.009))[hex_grid_elements(1, 1, 1)[0]]
        X = X + rng.uniform(-5e-4, 5e-4, X.shape)
    for trial in range(5):
        x = X @ (np.eye(3) + rng.uniform(-0.2, 0.2, (3, 3))).T + rng.uniform(-1, 1, 3)
        E, nu = 1e5 * (1 + trial), 0.3 + 0.04 * trial
        psi, g, H, st = oracle.elem_eval(X, x, E, nu, project=False)
        assert st == 0
        tpsi, xt = _torch_nh(X, x, E, nu)
        tg = torch.autograd.grad(tpsi, xt, create_graph=True)[0]
        tH = torch.stack([torch.autograd.grad(tg.reshape(-1)[i], xt, retain_graph=True)[0].reshape(-1)
                          for i in range(3 * nv)])
        assert abs(psi - tpsi.item()) <= 1e-12 * abs(tpsi.item()) + 1e-18
        np.testing.assert_allclose(g, tg.detach().numpy().ravel(), rtol=1e-10, atol=1e-10 * np.abs(g).max())
        np.testing.assert_allclose(H, tH.numpy(), rtol=1e-9, atol=1e-10 * np.abs(H).max())


def test_projection_is_psd_and_identity_on_psd(oracle):
    rng = np.random.default_rng(3)
    A = rng.normal(size=(9, 9)); A = A + A.T
    P = oracle.project_psd9(A)
    w = np.linalg.eigvalsh(P)
    assert w.min() > -1e-12 * np.abs(w).max()
    wA, VA = np.linalg.eigh(A)
    ref = (VA * np.maximum(wA, 0)) @ VA.T
    np.testing.assert_allclose(P, ref, atol=1e-12 * np.abs(A).max())
    S = A @ A.T
    np.testing.assert_allclose(oracle.project_psd9(S), S, atol=1e-12 * np.abs(S).max())


# --- TestCube dynamics (cpp/src/_test.cpp:290-560) --------------------------

def _cube(oracle, golden, params, grav, method="minimize_newton"):
    d = golden["test_cube"]
    X = np.array(d["vertices"]); T = np.array(d["elements"])
    s = oracle.System(X, T, rho=params["density"], youngs=params["youngsModulus"], nu=params["poissonsRatio"],
                      grav=grav, scheme="backward_euler", method=method, dt=d["dt"], substeps=1, nthreads=1)
    return s, X, d


def _com_accel(series, dt):
    y = np.asarray(series)
    n = len(y)
    acc = (-2 * y[1:n - 1] + y[2:] + y[:n - 2]) / (dt * dt)
    return acc[1:n - 3].mean()


def test_cube_gravity(oracle, golden):
    p = golden["test_cube"]["gravity_test"]
    s, X, d = _cube(oracle, golden, p, p["gravity"])
    q = X.ravel().copy(); zs = [X[:, 2].mean()]
    for _ in range(1, d["num_steps"]):
        q, st = s.step(q); assert st == 0
        zs.append(q.reshape(-1, 3)[:, 2].mean())
    assert abs(_com_accel(zs, d["dt"]) - d["expected_acceleration"]) < d["tol"]


def test_cube_pressure(oracle, golden):
    p = golden["test_cube"]["pressure_test"]
    s, X, d = _cube(oracle, golden, p, (0, 0, 0))
    s.set_pressure(np.array(p["faces"]), np.array(p["groups"]))
    q = X.ravel().copy(); ys = [X[:, 1].mean()]
    act = np.array([p["pressure"]])
    for _ in range(1, d["num_steps"]):
        q, st = s.step(q, pressure=act); assert st == 0
        ys.append(q.reshape(-1, 3)[:, 1].mean())
    assert abs(_com_accel(ys, d["dt"]) - d["expected_acceleration"]) < d["tol"]


def test_cube_vertex_force(oracle, golden):
    p = golden["test_cube"]["vertex_force_test"]
    s, X, d = _cube(oracle, golden, p, (0, 0, 0))
    s.set_vertex_force(True)
    f = np.zeros((8, 3)); f[:, 2] = p["force_per_vertex_z"]
    q = X.ravel().copy(); zs = [X[:, 2].mean()]
    for _ in range(1, d["num_steps"]):
        q, st = s.step(q, vforce=f.ravel()); assert st == 0
        zs.append(q.reshape(-1, 3)[:, 2].mean())
    assert abs(_com_accel(zs, d["dt"]) - d["expected_acceleration"]) < d["tol"]


def test_cube_energy_decreases(oracle, golden):
    # TestCube::test_energy_min: Neumann mask written at DOFs 3*i, i = 0..3
    p = golden["test_cube"]["energy_min_test"]
    s, X, d = _cube(oracle, golden, p, p["gravity"])
    mask = np.zeros(24, np.int32)
    for i in p["masked_vertices"]:
        mask[3 * i:3 * i + 3] = 1
    s.set_neumann(mask, np.zeros(24))
    s.set_pressure(np.array(p["faces"]), np.array(p["groups"]))
    q = X.ravel().copy()
    for i in range(1, p["num_steps"]):
        pr = min(p["max_pressure"] * 2 * i / p["num_steps"], p["max_pressure"])
        act = np.array([pr])
        e0 = s.energy(q, d["dt"], pressure=act)
        q, st = s.step(q, pressure=act); assert st == 0
        e1 = s.energy(q, d["dt"], pressure=act)
        assert e1 <= e0


def test_ldl_matches_dense_solve(oracle):
    from sors_b200.meshes import cantilever_tets, clamp_mask
    X, T = cantilever_tets(6, 2, 2, (0.03, 0.01, 0.01))
    s = oracle.System(X, T, rho=1070, youngs=1e5, nu=0.45, grav=(0, 0, -9.81), dt=1e-3, nthreads=2)
    m, v = clamp_mask(X)
    s.set_neumann(m, v)
    rng = np.random.default_rng(0)
    q = X.ravel() + rng.uniform(-1e-4, 1e-4, X.size)
    H, st = s.hessian_dense(q, 1e-3)
    b = rng.normal(size=X.size)
    Hs = np.tril(H) + np.tril(H, -1).T
    from oracle.oracle import lib, _pd
    x = b.copy()
    lib().orc_solve_with_hessian(s.h, _pd(q), 1e-3, None, _pd(x))
    np.testing.assert_allclose(x, np.linalg.solve(Hs, b), rtol=1e-9, atol=1e-12 * np.abs(x).max())


# --- SoftCon fibre term (cpp/src/energies/softconMuscle.cpp) ----------------

def _torch_muscle(X, x, k, m, act):
    """Consistent fibre energy k/2 (|F m| - (1 - e))^2 x V, tet or hex."""
    from oracle import oracle as orc
    nv = X.shape[0]
    xt = torch.tensor(x, dtype=torch.float64, requires_grad=True)
    if nv == 4:
        Dm = torch.tensor((X[:3] - X[3]).T)
        Fs = [(xt[:3] - xt[3]).T @ torch.linalg.inv(Dm)]
        V = abs(np.linalg.det(X[:3] - X[3])) / 6
    else:
        G, _, V = orc.hex_init(X)
        Fs = [xt.T @ torch.tensor(G[s]) for s in range(8)]
    mt = torch.tensor(m, dtype=torch.float64)
    psi = 0
    for F in Fs:
        ll = torch.linalg.norm(F @ mt)
        psi = psi + 0.5 * k * (ll - (1 - act)) ** 2 / len(Fs)
    return psi * V, xt


@pytest.mark.parametrize("nv", [4, 8])
def test_muscle_consistent_vs_autograd(oracle, nv):
    rng = np.random.default_rng(21 + nv)
    if nv == 4:
        X = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float) * 0.01
    else:
        from sors_b200.meshes import hex_grid_elements, grid_nodes
        X = grid_nodes(1, 1, 1, (0.01, 0.012, 0.009))[hex_grid_elements(1, 1, 1)[0]]
    for trial in range(4):
        x = X @ (np.eye(3) + rng.uniform(-0.2, 0.2, (3, 3))).T
        m = rng.standard_normal(3); m /= np.linalg.norm(m)
        k, act = 1e4 * (1 + trial), 0.3 * trial
        psi_nh, g_nh, H_nh, _ = oracle.elem_eval(X, x, 1e5, 0.4)
        psi, g, H, st = oracle.elem_eval_muscle(X, x, 1e5, 0.4, k, m, act, form=oracle.MUSCLE_CONSISTENT)
        assert st == 0
        tpsi, xt = _torch_muscle(X, x, k, m, act)
        tg = torch.autograd.grad(tpsi, xt, create_graph=True)[0]
        tH = torch.stack([torch.autograd.grad(tg.reshape(-1)[i], xt, retain_graph=True)[0].reshape(-1)
                          for i in range(3 * nv)])
        assert abs((psi - psi_nh) - tpsi.item()) <= 1e-10 * abs(tpsi.item()) + 1e-18
        np.testing.assert_allclose(g - g_nh, tg.detach().numpy().ravel(), rtol=1e-9,
                                   atol=1e-10 * np.abs(g - g_nh).max())
        np.testing.assert_allclose(H - H_nh, tH.numpy(), rtol=1e-8, atol=1e-9 * np.abs(H - H_nh).max())


def test_muscle_reference_forms(oracle):
    # The reference's gradient is shared by both forms; its energy |l-(1-e)| and
    # its Hessian differ from the consistent ones (the deviation this build records).
    rng = np.random.default_rng(5)
    X = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float) * 0.01
    x = X @ (np.eye(3) + rng.uniform(-0.1, 0.1, (3, 3))).T
    m = np.array([0.0, 0.0, 1.0])
    a = oracle.elem_eval_muscle(X, x, 1e5, 0.4, 1e5, m, 0.4, form=oracle.MUSCLE_REFERENCE)
    b = oracle.elem_eval_muscle(X, x, 1e5, 0.4, 1e5, m, 0.4, form=oracle.MUSCLE_CONSISTENT)
    np.testing.assert_array_equal(a[1], b[1])
    assert abs(a[0] - b[0]) > 1e-6 * abs(b[0])
    assert np.abs(a[2] - b[2]).max() > 1e-6 * np.abs(b[2]).max()


def test_softcon_contraction_oracle(oracle, golden):
    # TestCube::test_softcon_muscle (cpp/src/_test.cpp:563-625), reference forms.
    d = golden["test_cube"]
    X = np.array(d["vertices"]); T = np.array(d["elements"])
    ne = T.shape[0]
    s = oracle.System(X, T, rho=1000.0, youngs=1e6, nu=0.4, grav=(0, 0, 0), scheme="backward_euler",
                      method="minimize_newton", dt=d["dt"], substeps=1, nthreads=1)
    s.set_muscles(np.array([0, 1] + [-1] * (ne - 2)), np.full(ne, 1e5), np.tile([0, 0, 1.0], (ne, 1)), 2,
                  form=oracle.MUSCLE_REFERENCE)
    q = X.ravel().copy()
    for i in range(1, 10):
        s.set_muscle_act(np.full(2, 2.0 * i / 10))
        q, st = s.step(q)
        assert st == 0
    z = q.reshape(-1, 3)[:, 2]
    assert z.max() - z.min() < X[:, 2].max() - X[:, 2].min()


# --- Stable Neo-Hookean (cpp/src/energies/stableNeoHookean.cpp) -------------

def _torch_snh(X, x, E, nu):
    """Psi*V of the stable Neo-Hookean energy with the reference's
    reparameterisation (stableNeoHookean.cpp:10-15), as python/_autodiff_check.py."""
    from oracle import oracle as orc
    nv = X.shape[0]
    lam = E * nu / ((1 + nu) * (1 - 2 * nu)); mu = E / (2 * (1 + nu))
    mu_s = 4.0 / 3.0 * mu; lam_s = lam + 5.0 / 8.0 * mu_s; alpha = 1 + 0.75 * mu_s / lam_s
    xt = torch.tensor(x, dtype=torch.float64, requires_grad=True)
    if nv == 4:
        Dm = torch.tensor((X[:3] - X[3]).T)
        Fs = [(xt[:3] - xt[3]).T @ torch.linalg.inv(Dm)]
        V = abs(np.linalg.det(X[:3] - X[3])) / 6
    else:
        G, _, V = orc.hex_init(X)
        Fs = [xt.T @ torch.tensor(G[s]) for s in range(8)]
    psi = 0
    for F in Fs:
        J = torch.det(F); IC = (F * F).sum()
        psi = psi + (0.5 * mu_s * (IC - 3) + 0.5 * lam_s * (J - alpha) ** 2 - 0.5 * mu_s * torch.log(IC + 1)) / len(Fs)
    return psi * V, xt


@pytest.mark.parametrize("nv", [4, 8])
def test_stable_neohookean_vs_autograd(oracle, nv):
    rng = np.random.default_rng(31 + nv)
    if nv == 4:
        X = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1]], float) * 0.01
    else:
        from sors_b200.meshes import hex_grid_elements, grid_nodes
        X = grid_nodes(1, 1, 1, (0.01, 0.012, 0.009))[hex_grid_elements(1, 1, 1)[0]]
    for trial in range(5):
        A = np.eye(3) + rng.uniform(-0.3, 0.3, (3, 3))
        if trial == 4:
            A[:, 0] *= -1.0   # an inverted element: the energy stays finite
        x = X @ A.T
        E, nu = 1e5 * (1 + trial), 0.3 + 0.04 * trial
        psi, g, H, st = oracle.elem_eval_material(X, x, E, nu, oracle.MAT_STABLE_NEOHOOKEAN)
        assert st == 0
        tpsi, xt = _torch_snh(X, x, E, nu)
        tg = torch.autograd.grad(tpsi, xt, create_graph=True)[0]
        tH = torch.stack([torch.autograd.grad(tg.reshape(-1)[i], xt, retain_graph=True)[0].reshape(-1)
                          for i in range(3 * nv)])
        assert abs(psi - tpsi.item()) <= 1e-12 * abs(tpsi.item()) + 1e-18
        np.testing.assert_allclose(g, tg.detach().numpy().ravel(), rtol=1e-10, atol=1e-10 * np.abs(g).max())
        np.testing.assert_allclose(H, tH.numpy(), rtol=1e-9, atol=1e-10 * np.abs(H).max())
