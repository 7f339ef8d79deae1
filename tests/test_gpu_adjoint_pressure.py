"""Adjoint of steps under follower pressure (sors_adjoint_step with pressure
faces, sors_adjoint_pressure_grad) against central finite differences of the
oracle's forward rollout (FP64).

The pressure term's exact Jacobian is not the Newton matrix's: the reference
(and the device's forward Newton) mirror its lower triangle and use p/6 for
quads where the exact coefficient is p/8.  The adjoint solves the transpose
system of the exact Jacobian, so directional derivatives along seeded
directions in (E, pressure) agree with the oracle's central differences to
1e-5 relative, for quads (hex bar) and triangles (tet bar)."""
import numpy as np
import pytest

from sors_b200 import meshes
from tests.helpers import make_pair

pytestmark = pytest.mark.gpu

DT = 2e-3
STEPS = 6


def _case(kind, seed=0):
    if kind == "hex":
        X, T = meshes.hex_bar(6, 2, 2, (0.03, 0.01, 0.01))
    else:
        X, T = meshes.cantilever_tets(6, 2, 2, (0.03, 0.01, 0.01))
    groups, _ = meshes.extract_surfaces(X, T)
    faces = np.concatenate(groups)
    gid = np.concatenate([np.full(len(g), k) for k, g in enumerate(groups)])
    ne = T.shape[0]
    rng = np.random.default_rng(seed)
    E = np.exp(rng.uniform(np.log(1e5), np.log(3e5), ne))
    pres = rng.uniform(2e3, 8e3, (STEPS, len(groups)))
    w = rng.standard_normal(3 * X.shape[0])
    return X, T, faces, gid, E, pres, w


def _oracle_loss(oracle, X, T, faces, gid, E, pres, w):
    o = oracle.System(X, T, rho=1070.0, youngs=E, nu=0.45, grav=(0, 0, -9.81), scheme="backward_euler",
                      method="minimize_newton", dt=DT, substeps=1)
    m, v = meshes.clamp_mask(X)
    o.set_neumann(m, v)
    o.set_pressure(faces, gid)
    q = X.ravel().copy()
    for t in range(pres.shape[0]):
        q, st = o.step(q, pressure=pres[t])
        assert st == 0
    return float(w @ q)


@pytest.mark.parametrize("kind", ["hex", "tet"])
def test_pressure_adjoint_vs_oracle_fd(oracle, kind):
    from sors_b200.adjoint import RolloutAdjoint
    X, T, faces, gid, E, pres, w = _case(kind)
    en, sol, o, s = make_pair(X, T, rho=1070.0, E=E, nu=0.45, dt=DT, faces=faces, groups=gid)
    r = RolloutAdjoint(en, sol, STEPS, DT, poisson=0.45)
    qT = r.forward(E, None, pressure=pres)
    gE, _, _, _ = r.backward(w)
    gP = r.grad_pressure
    assert gP.shape == pres.shape
    lo = _oracle_loss(oracle, X, T, faces, gid, E, pres, w)
    assert abs(float(w @ qT) - lo) < 1e-9 * np.abs(w).sum()
    rng = np.random.default_rng(42)
    h = 1e-6
    for _ in range(3):
        rE = rng.standard_normal(E.size)
        rP = rng.standard_normal(pres.shape)
        d_adj = gE @ (E * rE) + (gP * pres * rP).sum()
        lp = _oracle_loss(oracle, X, T, faces, gid, E * (1 + h * rE), pres * (1 + h * rP), w)
        lm = _oracle_loss(oracle, X, T, faces, gid, E * (1 - h * rE), pres * (1 - h * rP), w)
        d_fd = (lp - lm) / (2 * h)
        assert abs(d_adj - d_fd) <= 1e-5 * abs(d_fd) + 1e-12, (d_adj, d_fd)


def test_pressure_grad_needs_an_adjoint_step():
    from sors_b200 import _lib
    import ctypes as C
    X, T, faces, gid, E, pres, w = _case("hex")
    en, sol, o, s = make_pair(X, T, rho=1070.0, E=E, nu=0.45, dt=DT, faces=faces, groups=gid)
    out = np.zeros(pres.shape[1])
    L = _lib.load()
    st = L.sors_adjoint_pressure_grad(en._h, out.ctypes.data_as(C.POINTER(C.c_double)), out.size)
    assert st == 1  # SORS_ERR_ARG: no adjoint step yet
