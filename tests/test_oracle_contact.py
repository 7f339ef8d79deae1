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


def test_max_distance_rope_oracle():
    # two cubes flying apart (+-0.2 m/s) joined by a maxDistance pair of 2.5 mm
    # (the two-sphere rope of cpp/demos/08_multiple_constraints_sphere.cpp): the
    # pair goes taut, holds at its bound with a non-negative multiplier, then
    # releases when the bodies rebound.
    from oracle import oracle as orc
    from oracle import contact as oc
    from tests.helpers import two_cubes
    X, T, a, b, n1 = two_cubes()
    dt = 5e-4
    o = orc.System(X, T, rho=1000.0, youngs=np.full(T.shape[0], 2e4), nu=0.4, grav=(0, 0, -9.81),
                   scheme="backward_euler", method="minimize_SQP", dt=dt, substeps=1, nthreads=1)
    v = np.zeros_like(X); v[:n1, 0] = -0.2; v[n1:, 0] = 0.2
    o.set_initial_velocity(v.ravel())
    sq = oc.SQPOracle(o, max_distance=oc.MaxDistance([a], [b], [0.0025]))
    x = X.ravel().copy()
    held = []
    for _ in range(14):
        x = sq.step(x, dt)
        L = np.linalg.norm(x.reshape(-1, 3)[a] - x.reshape(-1, 3)[b])
        assert L <= 0.0025 + 1e-12
        held.append(len(sq.held_pairs))
        if held[-1]:
            assert abs(L - 0.0025) < 1e-12
    assert held[0] == 0 and max(held) == 1 and held[-1] == 0


def test_max_distance_qp_kkt():
    # one QP with a pair row: stationarity H dx + g = mu a, mu >= 0, a.dx = l
    from oracle import contact as oc
    import scipy.sparse as sp
    rng = np.random.default_rng(3)
    n = 12
    M = rng.standard_normal((n, n)); H = sp.csr_matrix(M @ M.T + n * np.eye(n))
    g = rng.standard_normal(n)
    x = rng.standard_normal(n)
    md = oc.MaxDistance([0, 1], [2, 3], [0.1, 50.0])
    A, l = md.rows(x, n)
    dx, work, mu = oc.solve_qp(H, g, sp.csr_matrix((0, n)), np.zeros(0), A, l)
    assert work[0] and not work[1]
    assert mu[0] >= 0.0 and abs((A @ dx)[0] - l[0]) < 1e-10
    assert np.abs(H @ dx + g - A.T @ mu).max() < 1e-9


def test_max_distance_adjoint_needs_constraint_curvature():
    # One SQP step of the rope scene with the pair held: the step's sensitivity
    # to the Young's moduli, from the KKT system with the Lagrangian Hessian
    # H + (mu / L)(I - u u^T) on (x_i - x_j), matches central differences of
    # the oracle's step; the energy Hessian alone is off by about 1 %.  (This
    # is the transpose system sors_adjoint_step solves for held pairs.)
    from oracle import oracle as orc
    from oracle import contact as oc
    from tests.helpers import two_cubes
    X, T, a, b, n1 = two_cubes(kind="tet")
    ne = T.shape[0]
    rng = np.random.default_rng(5)
    E = np.exp(rng.uniform(np.log(1e4), np.log(4e4), ne))
    dt = 5e-4
    v0 = np.zeros_like(X); v0[:n1, 0] = -0.2; v0[n1:, 0] = 0.2

    def system(Ev):
        return orc.System(X, T, rho=1000.0, youngs=Ev, nu=0.4, grav=(0, 0, -9.81), scheme="backward_euler",
                          method="minimize_SQP", dt=dt, substeps=1, nthreads=1)

    o = system(E)
    o.set_initial_velocity(v0.ravel())
    sq = oc.SQPOracle(o, max_distance=oc.MaxDistance([a], [b], [0.0025]))
    q = X.ravel().copy()
    for _ in range(3):
        q = sq.step(q, dt)
    qP, vP, _ = o.state()

    def one_step(Ev):
        s = system(Ev)
        s.set_initial_deformation(qP); s.set_initial_velocity(vP)
        sqs = oc.SQPOracle(s, max_distance=oc.MaxDistance([a], [b], [0.0025]))
        return sqs.step(qP.copy(), dt), sqs

    q1, sq1 = one_step(E)
    assert list(sq1.held_pairs) == [0]
    s0 = system(E); s0.set_initial_deformation(qP); s0.set_initial_velocity(vP)
    H = s0.hessian_csr(q1, dt)[0].toarray()
    g = s0.gradient(q1, dt)
    n = q1.size
    xs = q1.reshape(-1, 3); d = xs[a] - xs[b]; L = np.linalg.norm(d); u = d / L
    arow = np.zeros(n); arow[3 * a:3 * a + 3] = -u; arow[3 * b:3 * b + 3] = u
    mu = (arow @ g) / (arow @ arow)
    assert mu > 0 and np.abs(g - mu * arow).max() < 1e-6 * np.abs(g).max()
    C = np.zeros((n, n)); M = (np.eye(3) - np.outer(u, u)) * mu / L
    for p, sp_ in ((a, 1), (b, -1)):
        for r, sr in ((a, 1), (b, -1)):
            C[3 * p:3 * p + 3, 3 * r:3 * r + 3] += sp_ * sr * M
    c = rng.standard_normal(n)
    r = rng.standard_normal(ne)
    h = 1e-6

    def grad_at(Ev):
        s = system(Ev); s.set_initial_deformation(qP); s.set_initial_velocity(vP)
        return s.gradient(q1, dt)

    dg = (grad_at(E * (1 + h * r)) - grad_at(E * (1 - h * r))) / (2 * h)
    d_fd = c @ (one_step(E * (1 + h * r))[0] - one_step(E * (1 - h * r))[0]) / (2 * h)
    errs = []
    for HL in (H + C, H):
        K = np.block([[HL, arow[:, None]], [arow[None, :], np.zeros((1, 1))]])
        lam = np.linalg.solve(K, np.concatenate([c, [0.0]]))[:n]
        errs.append(abs(-lam @ dg - d_fd) / abs(d_fd))
    assert errs[0] < 1e-5, errs
    assert errs[1] > 1e-3, errs


# --- OSQP restatement (oracle/contact.py osqp_solve) -------------------------

def test_osqp_restatement_solves_a_convex_qp():
    # well-scaled convex QP with equality and one-sided rows: OSQP's ADMM meets
    # its termination test and lands on the exact KKT point
    import scipy.sparse as sp
    from oracle import contact as oc
    rng = np.random.default_rng(0)
    n = 30
    B = rng.standard_normal((n, n))
    P = sp.csr_matrix(B @ B.T + n * np.eye(n)); q = rng.standard_normal(n)
    A = sp.csr_matrix(rng.standard_normal((8, n))); lo = rng.standard_normal(8) - 1
    up = np.full(8, np.inf); up[:2] = lo[:2]
    x, it, conv = oc.osqp_solve(P, q, A, lo, up)
    dx, _, _ = oc.solve_qp(P, q, A[:2], lo[:2], A[2:], lo[2:])
    assert conv and it <= oc.MAX_ITER_QP
    assert np.abs(x - dx).max() <= 1e-6 * np.abs(dx).max()


def test_osqp_restatement_rejects_nonconvex():
    # OSQP's set-up refuses an indefinite P; minimize_SQP turns that into "OSQP solver failed"
    import scipy.sparse as sp
    from oracle import contact as oc
    n = 6
    P = sp.diags([1.0, 2.0, -3.0, 1.0, 1.0, 1.0]).tocsr()
    A = sp.csr_matrix(np.eye(n)[:2])
    with pytest.raises(oc.OSQPNonConvex):
        oc.osqp_solve(P, np.ones(n), A, np.zeros(2), np.full(2, np.inf))


def test_plane_contact_no_penetration_osqp(golden):
    # the reference's contact test with the QP solved as the reference does
    # (OSQP, max_iter 250): within the test's 1e-4 tolerance, but not exactly
    # on the plane, as OSQP's 1e-3 absolute tolerance allows
    from oracle import oracle as orc
    from oracle import contact as oc
    d = golden["test_constraint"]
    X = np.array(d["vertices"]); T = np.array([[0, 1, 2, 3]])
    o = orc.System(X, T, rho=1.0, youngs=1e5, nu=0.3, grav=(0, 0, -9.81), scheme="backward_euler",
                   method="minimize_SQP", dt=1e-2, substeps=1, nthreads=1)
    sq = oc.SQPOracle(o, oc.PlaneContact([[0, 0, 0]], [[0, 0, 1.0]], [0, 1, 2, 3]), qp="osqp")
    z = sq.step(X.ravel(), 1e-2).reshape(-1, 3)[:, 2]
    assert z.min() >= -d["tol"]


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_osqp_and_exact_contact_steps_agree_to_osqp_tolerance(kind):
    # a small body dropped onto z = 0: the exact QP keeps every contact on the
    # plane; OSQP stops at its first termination check with up to
    # eps_abs = 1e-3 m of primal residual, so its contacts sink slightly and the
    # two trajectories differ by less than that tolerance
    from oracle import oracle as orc
    from oracle import contact as oc
    from sors_b200 import meshes
    if kind == "hex":
        X, T = meshes.hex_bar(3, 3, 3, (0.01, 0.01, 0.01))
    else:
        X, T = meshes.cantilever_tets(6, 3, 3, (0.012, 0.006, 0.006))
    X = X + np.array([0, 0, 0.0004])
    groups, _ = meshes.extract_surfaces(X, T)
    surf = np.unique(np.concatenate([g.ravel() for g in groups]))
    out = {}
    for qp in ("exact", "osqp"):
        o = orc.System(X, T, rho=1070.0, youngs=1e5, nu=0.45, grav=(0, 0, -9.81), scheme="backward_euler",
                       method="minimize_SQP", dt=2e-3, substeps=1, nthreads=2)
        sq = oc.SQPOracle(o, oc.PlaneContact([[0, 0, 0]], [[0, 0, 1.0]], surf), qp=qp)
        x = X.ravel().copy(); tr = []
        for _ in range(20):
            x = sq.step(x, 2e-3); tr.append(x.copy())
        out[qp] = np.array(tr)
    zmin = lambda tr: tr[:, 2::3].reshape(len(tr), -1)[:, surf].min()
    assert zmin(out["exact"]) > -1e-12
    assert -oc.OSQP_EPS_ABS < zmin(out["osqp"]) < 0.0
    assert np.abs(out["exact"] - out["osqp"]).max() < oc.OSQP_EPS_ABS
