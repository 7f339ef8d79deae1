"""ctypes front-end of the CPU oracle (oracle/sors_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
cpu_baseline / reference arm of bench.py, as the checker.  The product
package (sors_b200) never imports this module.

The oracle restates the SORS reference path in FP64 on the CPU; the C source
cites the reference file:line of every step.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libsors_oracle.so")
_lib = None

SCHEME = {"backward_euler": 0, "crank_nicolson": 1}
METHOD = {"minimize_newton": 0, "minimize_newton_linesearch": 1, "minimize_frozenhessian": 2, "minimize_SQP": 3}
MAT_NEOHOOKEAN = 0
MAT_TEST_QUARTIC = 1
MAT_STABLE_NEOHOOKEAN = 2

_dp = C.POINTER(C.c_double)
_ip = C.POINTER(C.c_int32)
_lp = C.POINTER(C.c_int64)


def build(force: bool = False) -> str:
    """Compile the oracle with its Makefile (gcc + OpenMP)."""
    src = os.path.join(_HERE, "sors_oracle.c")
    if force or not os.path.exists(_LIB_PATH) or os.path.getmtime(_LIB_PATH) < os.path.getmtime(src):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        L.orc_tet_init.argtypes = [_dp, _dp, _dp, _dp]
        L.orc_hex_init.argtypes = [_dp, _dp, _dp, _dp]
        L.orc_elem_eval.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_int, _dp, _dp, _dp]
        L.orc_elem_eval_batch.argtypes = [C.c_int, C.c_int, _dp, _ip, _dp, _dp, _dp, C.c_int, _dp, _dp, _dp]
        L.orc_project_psd9.argtypes = [_dp]
        L.orc_elem_eval_material.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_int, C.c_int, _dp, _dp,
                                              _dp]
        L.orc_elem_eval_muscle.argtypes = [C.c_int, _dp, _dp, C.c_double, C.c_double, C.c_double, _dp, C.c_double,
                                           C.c_int, C.c_int, _dp, _dp, _dp]
        L.orc_set_muscles.argtypes = [C.c_void_p, _ip, _dp, _dp, C.c_int, C.c_int]
        L.orc_set_muscle_act.argtypes = [C.c_void_p, _dp]
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int, C.c_int, _dp, C.c_int, _ip, _dp, _dp, _dp, _dp, C.c_double, C.c_int,
                                 C.c_int, C.c_int, C.c_int, C.c_int]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_set_neumann.argtypes = [C.c_void_p, _ip, _dp]
        L.orc_set_pressure.argtypes = [C.c_void_p, C.c_int, C.c_int, _ip, _ip]
        L.orc_set_vertex_force.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_step_settings.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_int]
        L.orc_set_method.argtypes = [C.c_void_p, C.c_int]
        L.orc_set_initial_deformation.argtypes = [C.c_void_p, _dp]
        L.orc_set_initial_velocity.argtypes = [C.c_void_p, _dp]
        L.orc_get_state.argtypes = [C.c_void_p, _dp, _dp, _dp]
        L.orc_get_mass.argtypes = [C.c_void_p, _dp]
        L.orc_energy.restype = C.c_double
        L.orc_energy.argtypes = [C.c_void_p, _dp, C.c_double, _dp, _dp]
        L.orc_gradient.argtypes = [C.c_void_p, _dp, C.c_double, _dp, _dp, _dp]
        L.orc_hessian_dense.argtypes = [C.c_void_p, _dp, C.c_double, _dp, _dp]
        L.orc_hessian_csr.argtypes = [C.c_void_p, _dp, C.c_double, _dp, _lp, _lp, _ip, _dp]
        L.orc_step.argtypes = [C.c_void_p, _dp, C.c_double, C.c_int, _dp, _dp]
        L.orc_minimize.argtypes = [C.c_void_p, _dp, C.c_double, _dp, _dp]
        L.orc_update_state.argtypes = [C.c_void_p, _dp, C.c_double]
        L.orc_solve_with_hessian.argtypes = [C.c_void_p, _dp, C.c_double, _dp, _dp]
        L.orc_last_newton_iters.argtypes = [C.c_void_p]
        L.orc_num_threads.restype = C.c_int
        _lib = L
    return _lib


def _d(a):
    return None if a is None else np.ascontiguousarray(a, dtype=np.float64)


def _pd(a):
    return None if a is None else a.ctypes.data_as(_dp)


def _i(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def _pi(a):
    return a.ctypes.data_as(_ip)


def tet_init(X):
    X = _d(X).reshape(4, 3)
    B = np.zeros((9, 12)); inv = np.zeros((3, 3)); vol = np.zeros(1)
    lib().orc_tet_init(_pd(X), _pd(B), _pd(inv), _pd(vol))
    return B, inv, float(vol[0])


def hex_init(X):
    X = _d(X).reshape(8, 3)
    G = np.zeros((8, 8, 3)); B = np.zeros((8, 9, 24)); vol = np.zeros(1)
    lib().orc_hex_init(_pd(X), _pd(G), _pd(B), _pd(vol))
    return G, B, float(vol[0])


def elem_eval(X, x, youngs, nu, project=False):
    """Psi*V, grad*V, hess*V of one element (tet: 4x3, hex: 8x3)."""
    X = _d(X); x = _d(x)
    nv = X.shape[0]
    n = 3 * nv
    psi = np.zeros(1); g = np.zeros(n); H = np.zeros((n, n))
    st = lib().orc_elem_eval(nv, _pd(X), _pd(x), float(youngs), float(nu), int(project), _pd(psi), _pd(g), _pd(H))
    return float(psi[0]), g, H, st


def elem_eval_material(X, x, youngs, nu, material, project=False):
    """Psi*V, grad*V, hess*V of one element for a material model (MAT_*)."""
    X = _d(X); x = _d(x)
    n = 3 * X.shape[0]
    psi = np.zeros(1); g = np.zeros(n); H = np.zeros((n, n))
    st = lib().orc_elem_eval_material(X.shape[0], _pd(X), _pd(x), float(youngs), float(nu), int(material),
                                      int(project), _pd(psi), _pd(g), _pd(H))
    return float(psi[0]), g, H, st


MUSCLE_REFERENCE = 0   # the reference's energy and Hessian forms (softconMuscle.cpp:30-31, :115-127)
MUSCLE_CONSISTENT = 1  # energy k/2 (|Fm| - (1-e))^2 and its exact Hessian


def elem_eval_muscle(X, x, youngs, nu, k, m, act, form=MUSCLE_CONSISTENT, project=False):
    """Neo-Hookean + SoftCon fibre element: Psi*V, grad*V, hess*V, status."""
    X = _d(X); x = _d(x)
    nv = X.shape[0]
    n = 3 * nv
    psi = np.zeros(1); g = np.zeros(n); H = np.zeros((n, n))
    st = lib().orc_elem_eval_muscle(nv, _pd(X), _pd(x), float(youngs), float(nu), float(k), _pd(_d(m)), float(act),
                                    int(form), int(project), _pd(psi), _pd(g), _pd(H))
    return float(psi[0]), g, H, st


def elem_eval_batch(Xn, conn, xn, youngs, nu, project=False, want_hess=True):
    Xn = _d(Xn); xn = _d(xn); conn = _i(conn)
    ne, nv = conn.shape
    n = 3 * nv
    youngs = _d(np.broadcast_to(youngs, (ne,)).copy()); nu = _d(np.broadcast_to(nu, (ne,)).copy())
    psi = np.zeros(ne); g = np.zeros((ne, n))
    H = np.zeros((ne, n, n)) if want_hess else None
    st = lib().orc_elem_eval_batch(nv, ne, _pd(Xn), _pi(conn), _pd(xn), _pd(youngs), _pd(nu), int(project),
                                   _pd(psi), _pd(g), _pd(H))
    return psi, g, H, st


def project_psd9(A):
    A = _d(A).reshape(9, 9).copy()
    lib().orc_project_psd9(_pd(A))
    return A


class System:
    """CPU restatement of Energy<3,E> + Solver<3,E> (minimize_newton & co)."""

    def __init__(self, X, conn, rho, youngs, nu, grav=(0, 0, 0), alpha=0.0, scheme="backward_euler",
                 method="minimize_newton", project=False, material=MAT_NEOHOOKEAN, nthreads=None,
                 dt=0.0, substeps=1, cfl=False):
        self.X = _d(X).reshape(-1, 3)
        self.conn = _i(conn)
        ne, nv = self.conn.shape
        self.nv = nv
        self.N = self.X.shape[0]
        self.ndof = 3 * self.N
        bc = lambda a: _d(np.broadcast_to(np.asarray(a, dtype=np.float64), (ne,)).copy())
        self._rho, self._E, self._nu = bc(rho), bc(youngs), bc(nu)
        g = _d(np.asarray(grav, dtype=np.float64))
        if nthreads is None:
            nthreads = os.cpu_count() or 1
        self.nthreads = nthreads
        self.h = lib().orc_create(nv, self.N, _pd(self.X), ne, _pi(self.conn), _pd(self._rho), _pd(self._E),
                                  _pd(self._nu), _pd(g), float(alpha), SCHEME[scheme], METHOD[method],
                                  int(project), int(material), int(nthreads))
        lib().orc_set_step_settings(self.h, float(dt), int(substeps), int(cfl))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_destroy(h)
            self.h = None

    def set_neumann(self, mask, value):
        self._mask = _i(mask); self._mval = _d(value)
        lib().orc_set_neumann(self.h, _pi(self._mask), _pd(self._mval))

    def set_pressure(self, faces, groups):
        self._faces = _i(faces); self._groups = _i(groups)
        lib().orc_set_pressure(self.h, self._faces.shape[0], self._faces.shape[1], _pi(self._faces),
                               _pi(self._groups))

    def set_muscles(self, group, stiffness, direction, n_groups, form=MUSCLE_CONSISTENT):
        """SoftCon fibre terms: group per element (-1 none), stiffness, direction (E x 3)."""
        self._mgroup = _i(group); self._mk = _d(stiffness); self._mdir = _d(direction).reshape(-1, 3)
        lib().orc_set_muscles(self.h, _pi(self._mgroup), _pd(self._mk), _pd(self._mdir), int(n_groups), int(form))

    def set_muscle_act(self, act):
        self._mact = _d(act).ravel()
        lib().orc_set_muscle_act(self.h, _pd(self._mact))

    def set_vertex_force(self, enabled=True):
        lib().orc_set_vertex_force(self.h, int(enabled))

    def set_method(self, method):
        lib().orc_set_method(self.h, METHOD[method])

    def set_initial_deformation(self, q):
        q = _d(q).ravel(); lib().orc_set_initial_deformation(self.h, _pd(q))

    def set_initial_velocity(self, v):
        v = _d(v).ravel(); lib().orc_set_initial_velocity(self.h, _pd(v))

    def state(self):
        qp = np.zeros(self.ndof); vp = np.zeros(self.ndof); gp = np.zeros(self.ndof)
        lib().orc_get_state(self.h, _pd(qp), _pd(vp), _pd(gp))
        return qp, vp, gp

    def mass(self):
        m = np.zeros(self.ndof)
        lib().orc_get_mass(self.h, _pd(m))
        return m

    def energy(self, q, dt, pressure=None, vforce=None):
        q = _d(q).ravel()
        return lib().orc_energy(self.h, _pd(q), float(dt), _pd(_d(pressure)), _pd(_d(vforce)))

    def gradient(self, q, dt, pressure=None, vforce=None):
        q = _d(q).ravel(); g = np.zeros(self.ndof)
        lib().orc_gradient(self.h, _pd(q), float(dt), _pd(_d(pressure)), _pd(_d(vforce)), _pd(g))
        return g

    def hessian_dense(self, q, dt, pressure=None):
        q = _d(q).ravel(); H = np.zeros((self.ndof, self.ndof))
        st = lib().orc_hessian_dense(self.h, _pd(q), float(dt), _pd(_d(pressure)), _pd(H))
        return H, st

    def hessian_csr(self, q, dt, pressure=None):
        import scipy.sparse as sp
        q = _d(q).ravel()
        nnz = np.zeros(1, dtype=np.int64)
        pa = _d(pressure)
        lib().orc_hessian_csr(self.h, _pd(q), float(dt), _pd(pa), nnz.ctypes.data_as(_lp), None, None, None)
        rp = np.zeros(self.ndof + 1, dtype=np.int64)
        col = np.zeros(int(nnz[0]), dtype=np.int32)
        val = np.zeros(int(nnz[0]))
        st = lib().orc_hessian_csr(self.h, _pd(q), float(dt), _pd(pa), nnz.ctypes.data_as(_lp),
                                   rp.ctypes.data_as(_lp), _pi(col), _pd(val))
        return sp.csr_matrix((val, col, rp), shape=(self.ndof, self.ndof)), st

    def step(self, q, dt=0.0, substeps=0, pressure=None, vforce=None):
        """Solver::step: returns (new q, status)."""
        q = _d(q).ravel().copy()
        st = lib().orc_step(self.h, _pd(q), float(dt), int(substeps), _pd(_d(pressure)), _pd(_d(vforce)))
        return q, st

    def minimize(self, q, dt, pressure=None, vforce=None):
        """Solver::minimize_<method> without update_state: returns (q, status)."""
        q = _d(q).ravel().copy()
        st = lib().orc_minimize(self.h, _pd(q), float(dt), _pd(_d(pressure)), _pd(_d(vforce)))
        return q, st

    def update_state(self, q, dt):
        q = _d(q).ravel(); lib().orc_update_state(self.h, _pd(q), float(dt))

    def newton_iters(self):
        return lib().orc_last_newton_iters(self.h)
