"""GPU path (libsors_b200.so through the py_sors API / C ABI) against the oracle.

Tolerances: element-level and assembled FP64 quantities agree with the oracle
to 1e-10 relative (the reference's per-element criterion); trajectories agree
within the displacement tolerances stated in each test.
"""
import numpy as np
import pytest

from sors_b200 import meshes
from tests.helpers import deform, make_pair, rel_err

pytestmark = pytest.mark.gpu

ELEM_TOL = 1e-10


@pytest.fixture(scope="module")
def c1():
    return meshes.cantilever_tets()


def _hex_mesh():
    X, H = meshes.hex_bar(6, 2, 2, (0.03, 0.01, 0.01))
    rng = np.random.default_rng(5)
    X = meshes.jitter_interior(X, 0.005, 0.1, rng)
    return X, H


@pytest.mark.parametrize("kind", ["tet", "hex"])
@pytest.mark.parametrize("project", [False, True])
def test_element_parity(c1, oracle, kind, project):
    X, T = (c1 if kind == "tet" else _hex_mesh())
    rng = np.random.default_rng(11)
    ne = T.shape[0]
    E = np.exp(rng.uniform(np.log(5e4), np.log(5e5), ne))
    nu = rng.uniform(0.3, 0.48, ne)
    en, _, _, _ = make_pair(X, T, E=E, nu=nu, project=project, clamp=False)
    for trial in range(3):
        q = deform(X, rng, amp=0.15)
        psi, g, H = en.compute_element_data(q, project=project)
        opsi, og, oH, st = oracle.elem_eval_batch(X, T, q.reshape(-1, 3), E, nu, project=project)
        assert st == 0
        assert rel_err(psi, opsi) < ELEM_TOL
        assert rel_err(g, og) < ELEM_TOL
        # per-element relative error of the Hessian
        scale = np.abs(oH).reshape(ne, -1).max(1)
        err = np.abs(H - oH).reshape(ne, -1).max(1) / scale
        assert err.max() < (ELEM_TOL if not project else 1e-9), err.max()


def test_rest_state_zero(golden):
    # TestTetrahedron::test_energy_zero / test_gradient_zero on the GPU (TOL 1e-9)
    d = golden["test_tetrahedron"]
    X = np.array(d["undeformed"]); T = np.array([[0, 1, 2, 3]])
    m = d["material"]
    en, _, _, _ = make_pair(X, T, rho=m["density"], E=m["youngsModulus"], nu=m["poissonsRatio"], clamp=False,
                            grav=(0, 0, 0))
    psi, g, H = en.compute_element_data(X.ravel(), project=False)
    assert abs(psi[0]) < d["tol"]
    assert np.abs(g).max() < d["tol"]


def test_quartic_known_answers(golden):
    # TestEnergy (cpp/src/_test.cpp:136-176) through the GPU assembly
    from sors_b200 import py_sors as ps
    d = golden["test_energy"]
    X = np.array(d["vertices"]); T = np.array(d["elements"])
    s = ps.SimulationSettings(); s.meshType = "Tetrahedron"; s._material_override = 1
    en = ps.Energy(X, T, s, np.zeros(3), 0.0, [set()] * 2,
                   [ps.Params(["density"], [1.0]) for _ in range(2)], [], ps.Params(), [], ps.Params())
    q = X.ravel()
    assert en.compute_energy(q, 0.0) == d["energy"]
    np.testing.assert_allclose(en.compute_gradient(q, 0.0), np.array(d["gradient"]).ravel(), atol=1e-12)
    H = en.compute_hessian(q, 0.0).toarray()
    np.testing.assert_allclose(H, np.diag(np.array(d["hessian_diag"]).ravel()), atol=1e-12)


@pytest.mark.parametrize("scheme", ["backward_euler", "crank_nicolson"])
@pytest.mark.parametrize("dt", [0.0, 1e-3])
def test_assembly_parity(c1, oracle, scheme, dt):
    X, T = c1
    rng = np.random.default_rng(3)
    en, _, o, _ = make_pair(X, T, scheme=scheme, dt=dt if dt else 1e-3, project=False, alpha=0.5)
    q = deform(X, rng, amp=0.05)
    # the same previous state on both sides
    vprev = rng.uniform(-0.01, 0.01, q.size)
    en.set_initial_velocity(vprev); o.set_initial_velocity(vprev)
    e_gpu = en.compute_energy(q, dt)
    e_orc = o.energy(q, dt)
    assert abs(e_gpu - e_orc) <= 1e-10 * max(abs(e_orc), 1e-12)
    g_gpu = en.compute_gradient(q, dt)
    g_orc = o.gradient(q, dt)
    assert rel_err(g_gpu, g_orc) < ELEM_TOL
    Hg = en.compute_hessian(q, dt)
    Ho, st = o.hessian_csr(q, dt)
    assert st == 0
    D = (Hg - Ho).tocoo()
    assert np.abs(D.data).max(initial=0.0) <= ELEM_TOL * np.abs(Ho.data).max()


def test_pressure_assembly_cube(golden, oracle):
    # TestCube mesh with the follower load: force, Jacobian (lower triangle mirrored)
    d = golden["test_cube"]; p = d["pressure_test"]
    X = np.array(d["vertices"]); T = np.array(d["elements"])
    faces = np.array(p["faces"]); groups = np.array(p["groups"])
    en, _, o, _ = make_pair(X, T, rho=p["density"], E=p["youngsModulus"], nu=p["poissonsRatio"], grav=(0, 0, 0),
                            dt=d["dt"], project=False, clamp=False, faces=faces, groups=groups)
    from sors_b200 import py_sors as ps
    act = ps.Params(["pressure"], [np.array([[p["pressure"]]])])
    rng = np.random.default_rng(2)
    q = deform(X, rng, amp=0.05)
    pr = np.array([p["pressure"]])
    assert rel_err(en.compute_gradient(q, d["dt"], act), o.gradient(q, d["dt"], pressure=pr)) < ELEM_TOL
    e_g = en.compute_energy(q, d["dt"], act); e_o = o.energy(q, d["dt"], pressure=pr)
    assert abs(e_g - e_o) <= 1e-10 * abs(e_o)
    Hg = en.compute_hessian(q, d["dt"], act).toarray()
    Ho, _ = o.hessian_dense(q, d["dt"], pressure=pr)
    Hsym = np.tril(Ho) + np.tril(Ho, -1).T
    assert rel_err(Hg, Hsym) < ELEM_TOL


def _com_accel(series, dt):
    y = np.asarray(series); n = len(y)
    acc = (-2 * y[1:n - 1] + y[2:] + y[:n - 2]) / (dt * dt)
    return acc[1:n - 3].mean()


@pytest.mark.parametrize("case", ["gravity", "pressure", "vertex_force"])
def test_cube_dynamics(golden, case):
    # TestCube::test_gravity_force / test_pressure_force / test_external_force on the GPU
    from sors_b200 import py_sors as ps
    d = golden["test_cube"]
    X = np.array(d["vertices"]); T = np.array(d["elements"])
    key = {"gravity": "gravity_test", "pressure": "pressure_test", "vertex_force": "vertex_force_test"}[case]
    p = d[key]
    grav = p.get("gravity", [0, 0, 0])
    kw = {}
    if case == "pressure":
        kw = dict(faces=np.array(p["faces"]), groups=np.array(p["groups"]))
    en, sol, _, _ = make_pair(X, T, rho=p["density"], E=p["youngsModulus"], nu=p["poissonsRatio"], grav=grav,
                              dt=d["dt"], clamp=False, vertex_force=(case == "vertex_force"), **kw)
    act = None
    axis = 2
    if case == "pressure":
        act = ps.Params(["pressure"], [np.array([[p["pressure"]]])]); axis = 1
    if case == "vertex_force":
        f = np.zeros((8, 3)); f[:, 2] = p["force_per_vertex_z"]
        act = ps.Params(["vertexForce"], [f])
    q = X.ravel().copy(); ys = [X[:, axis].mean()]
    for _ in range(1, d["num_steps"]):
        q = sol.step(q, en, act)
        ys.append(q.reshape(-1, 3)[:, axis].mean())
    assert abs(_com_accel(ys, d["dt"]) - d["expected_acceleration"]) < d["tol"]


def test_c1_trajectory_fp64(c1, oracle):
    """Cantilever, 200 BE steps at dt=1e-3, FP64, Newton residual tol 1e-8."""
    X, T = c1
    en, sol, o, _ = make_pair(X, T, dt=1e-3, res_tol=1e-8)
    q = X.ravel().copy(); qo = q.copy()
    worst = 0.0
    for step in range(200):
        q = sol.step(q, en)
        qo, st = o.step(qo)
        assert st == 0
        worst = max(worst, np.abs(q - qo).max())
    disp = np.abs(qo - X.ravel()).max()
    assert disp > 1e-5  # the beam moved
    assert worst < 1e-8, worst


@pytest.mark.parametrize("project", [True, "adaptive"])
def test_c1_trajectory_mixed(c1, oracle, project):
    """Mixed precision (FP32 Hessian/PCG, FP64 residual), all 200 steps of the
    cantilever: the largest error over the trajectory stays within 1e-6 of the
    largest displacement, for the always-projected and the adaptive Hessian."""
    X, T = c1
    en, sol, o, _ = make_pair(X, T, dt=1e-3, precision="mixed", res_tol=1e-8, project=project)
    q = X.ravel().copy(); qo = q.copy()
    worst = disp = 0.0
    for step in range(200):
        q = sol.step(q, en)
        qo, st = o.step(qo)
        assert st == 0
        worst = max(worst, float(np.abs(q - qo).max()))
        disp = max(disp, float(np.abs(qo - X.ravel()).max()))
    assert worst <= 1e-6 * disp, (worst, disp)


@pytest.mark.parametrize("method", ["minimize_newton_linesearch", "minimize_frozenhessian"])
def test_other_methods(c1, oracle, method):
    X, T = c1
    en, sol, o, _ = make_pair(X, T, dt=1e-3, method=method, clamp=(method != "minimize_newton_linesearch"))
    q = X.ravel().copy(); qo = q.copy()
    for _ in range(5):
        q = sol.step(q, en)
        qo, st = o.step(qo)
        assert st == 0
    assert np.abs(q - qo).max() < 1e-8


def test_crank_nicolson_trajectory(c1, oracle):
    X, T = c1
    en, sol, o, _ = make_pair(X, T, dt=2e-3, scheme="crank_nicolson", alpha=2.0)
    q = X.ravel().copy(); qo = q.copy()
    for _ in range(20):
        q = sol.step(q, en)
        qo, st = o.step(qo)
        assert st == 0
    assert np.abs(q - qo).max() < 1e-8


def test_hex_trajectory(oracle):
    X, H = _hex_mesh()
    en, sol, o, _ = make_pair(X, H, E=2e5, dt=2e-3)
    q = X.ravel().copy(); qo = q.copy()
    for _ in range(10):
        q = sol.step(q, en)
        qo, st = o.step(qo)
        assert st == 0
    assert np.abs(q - qo).max() < 1e-8


def test_inverted_element_raises(c1):
    X, T = c1
    en, _, _, _ = make_pair(X, T)
    q = X.ravel().copy().reshape(-1, 3)
    q[T[0, 0]] = q[T[0, 1]] + (q[T[0, 1]] - q[T[0, 0]])  # fold a vertex through the opposite side
    with pytest.raises(RuntimeError, match="Inverted Elements"):
        en.compute_hessian(q.ravel(), 1e-3)


def test_deterministic(c1):
    X, T = c1
    outs = []
    for _ in range(2):
        en, sol, _, _ = make_pair(X, T, dt=1e-3)
        q = X.ravel().copy()
        for _ in range(3):
            q = sol.step(q, en)
        outs.append(q)
    assert np.array_equal(outs[0], outs[1])


def _c3_case(length=0.015, h=2.5e-3):
    """Voxel cylinder (R 20 mm) with three closed chambers; base clamped."""
    X, H = meshes.voxel_cylinder(length=length, h=h, cap_layers=2)
    groups, _ = meshes.extract_surfaces(X, H)
    faces = np.concatenate(groups)
    gid = np.concatenate([np.full(len(g), k) for k, g in enumerate(groups)])
    return X, H, faces, gid, len(groups)


C3_LEVELS = (1, 2, 3)


@pytest.fixture(scope="module")
def c3_reference(oracle):
    X, H, faces, gid, ng = _c3_case()
    mask = np.repeat((np.abs(X[:, 2]) < 1e-12).astype(np.int32), 3)
    o = oracle.System(X, H, rho=1070.0, youngs=3e5, nu=0.48, grav=(0, 0, 0), dt=0.0)
    o.set_neumann(mask, np.zeros(mask.size)); o.set_pressure(faces, gid)
    qo = X.ravel().copy()
    for level in C3_LEVELS:
        pr = np.zeros(ng); pr[1] = 5e3 * level   # one chamber
        qo, st = o.step(qo, dt=0.0, pressure=pr)
        assert st == 0
    return qo


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_c3_chamber_pressure_static(c3_reference, precision):
    """Pressure-actuated arm, hexes, quasistatic (dt = 0): GPU vs oracle over a load ramp."""
    from sors_b200 import py_sors as ps
    X, H, faces, gid, ng = _c3_case()
    assert ng == 4  # outer surface + three chambers
    mask = np.repeat((np.abs(X[:, 2]) < 1e-12).astype(np.int32), 3)
    s = ps.SimulationSettings()
    s.meshType = "Hexahedron"; s.dt = 0.0; s.timeSteppingScheme = "backward_euler"
    s.precision = precision; s.newtonResidualTol = 1e-10
    ne = H.shape[0]
    params = [ps.Params(["density", "youngsModulus", "poissonsRatio"], [1070.0, 3e5, 0.48])] * ne
    cp = ps.Params(["neumannBCmask", "neumannBCvalue"], [mask.astype(float), np.zeros(mask.size)])
    fp = ps.Params(["surfaceVertexIdx", "surfaceGroups"], [faces.astype(float), gid.astype(float)])
    en = ps.Energy(X, H, s, np.zeros(3), 0.0, [{"neohookean"}] * ne, params, ["neumannBC"], cp, ["pressure"], fp)
    sol = ps.Solver(s)
    q = X.ravel().copy()
    for level in C3_LEVELS:
        pr = np.zeros(ng); pr[1] = 5e3 * level   # one chamber
        q = sol.step(q, en, ps.Params(["pressure"], [pr.reshape(-1, 1)]), 0.0)
    qo = c3_reference
    u = qo - X.ravel()
    assert np.abs(u).max() > 1e-5
    tol = 1e-8 if precision == "fp64" else 1e-6 * np.abs(u).max()
    assert np.abs(q - qo).max() < tol, np.abs(q - qo).max()


def _fan_ball(r=0.01):
    """Tets fanned from a centre vertex to a once-subdivided icosahedron (42
    surface vertices, 80 tets): the centre's block-row has 43 blocks, more
    than the widest SpMV lane group (32 lanes), which then loops over the row."""
    t = (1 + 5 ** 0.5) / 2
    V = [[-1, t, 0], [1, t, 0], [-1, -t, 0], [1, -t, 0], [0, -1, t], [0, 1, t], [0, -1, -t], [0, 1, -t],
         [t, 0, -1], [t, 0, 1], [-t, 0, -1], [-t, 0, 1]]
    F = [[0, 11, 5], [0, 5, 1], [0, 1, 7], [0, 7, 10], [0, 10, 11], [1, 5, 9], [5, 11, 4], [11, 10, 2],
         [10, 7, 6], [7, 1, 8], [3, 9, 4], [3, 4, 2], [3, 2, 6], [3, 6, 8], [3, 8, 9], [4, 9, 5], [2, 4, 11],
         [6, 2, 10], [8, 6, 7], [9, 8, 1]]
    V = [list(np.asarray(v, float) / np.linalg.norm(v)) for v in V]
    mid = {}

    def m(a, b):
        k = (min(a, b), max(a, b))
        if k not in mid:
            v = np.asarray(V[a]) + np.asarray(V[b])
            V.append(list(v / np.linalg.norm(v)))
            mid[k] = len(V) - 1
        return mid[k]
    F2 = []
    for a, b, c in F:
        ab, bc, ca = m(a, b), m(b, c), m(c, a)
        F2 += [[a, ab, ca], [b, bc, ab], [c, ca, bc], [ab, bc, ca]]
    X = np.vstack([np.asarray(V) * r, [[0.0, 0.0, 0.0]]])
    c = X.shape[0] - 1
    T = []
    for a, b, d in F2:
        # positive orientation, the centre as vertex 3
        v = np.dot(np.cross(X[b] - X[a], X[d] - X[a]), X[c] - X[a])
        T.append([a, b, d, c] if v > 0 else [a, d, b, c])
    return X, np.asarray(T, np.int32)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_long_block_rows(oracle, precision):
    # a block-row longer than 32 blocks (several blocks per SpMV lane, and a
    # long assembly row); the trajectory still matches the oracle
    X, T = _fan_ball()
    en, sol, o, _ = make_pair(X, T, E=5e4, nu=0.4, dt=2e-3, precision=precision)
    q = X.ravel().copy(); qo = q.copy()
    for _ in range(8):
        q = sol.step(q, en)
        qo, st = o.step(qo)
        assert st == 0
    disp = np.abs(qo - X.ravel()).max()
    assert disp > 1e-6
    assert np.abs(q - qo).max() < (1e-9 if precision == "fp64" else 1e-6 * disp)
