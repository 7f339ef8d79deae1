"""Oracle for the contact step (Solver::minimize_SQP with PlaneContact / DiskContact).

TEST INFRASTRUCTURE ONLY: used by tests/ as the checker, never by the product.

Restates, on top of the oracle's FP64 system (oracle.System with method
"minimize_SQP": element terms on every DOF, no Neumann override,
cpp/src/energy.cpp:275,:337):
  - PlaneContact::update_active_constraints (cpp/src/constraints/planeContact.cpp:89-124)
  - DiskContact::update_active_constraints  (cpp/src/constraints/diskContact.cpp:94-205)
  - Energy::compute_constraint_bounds / compute_constraint_matrix_qp (cpp/src/energy.cpp:394-474):
      Neumann rows  dx_i = -(x_i - qPrev_i - dt val_i)            (neumannBC.cpp:4-21)
      contact rows  n . dx_v >= -n . (x_v - p)                      (planeContact.cpp:4-42)
  - Solver::minimize_SQP (cpp/src/solver.cpp:109-197): x += dx until ||dx|| < 1e-9, at most 100 iterations.
The reference solves each QP with OSQP (cpp/src/solver.cpp:116-176: scaling
off, max_iter = MAX_ITER_QP = 250, verbose off, other settings default).  OSQP
is an un-vendored submodule (external/osqp, v1.x API; its pinned commit is not
recorded in the mounted tree), so two QP solvers are restated here:
  - qp="exact": the KKT point itself (primal-dual active set on the KKT
    system, SuperLU), the point OSQP approximates;
  - qp="osqp": the published OSQP algorithm (B. Stellato, G. Banjac,
    P. Goulart, A. Bemporad, S. Boyd, "OSQP: an operator splitting solver for
    quadratic programs", Math. Prog. Comp. 12, 2020: Algorithm 1 with the
    direct KKT solve, termination of section 3.4, step-size update of
    section 5.2) with OSQP's default parameters and the reference's settings,
    including OSQP's rejection of a non-convex problem at set-up (the KKT
    matrix must have n positive and m negative pivots), which minimize_SQP
    turns into "OSQP solver failed" (solver.cpp:160-163).  OSQP schedules its
    step-size updates by measured run time (not reproducible); this
    restatement updates at each termination check (every 25 iterations).
"""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

PLANE_CONSTRAINT_THRESHOLD = 0.01      # cpp/headers/common.h:29
DISK_PLANAR_CONSTRAINT_THRESHOLD = 0.01  # common.h:33
DISK_RADIAL_CONSTRAINT_THRESHOLD = 0.001  # common.h:35
MAX_ITER = 100
DX_TOL = 1e-9


class PlaneContact:
    def __init__(self, points, normals, surface):
        self.p = np.asarray(points, float).reshape(-1, 3)
        self.n = np.asarray(normals, float).reshape(-1, 3)
        self.surf = np.asarray(surface, int).ravel()
        self.mask = -np.ones(self.surf.size, int)

    def update(self, x):
        xs = x.reshape(-1, 3)[self.surf]
        for i in range(self.surf.size):
            best, idx = np.inf, -1
            for k in range(self.p.shape[0]):
                d = float(self.n[k] @ (xs[i] - self.p[k]))
                if d < PLANE_CONSTRAINT_THRESHOLD and d < best:
                    best, idx = d, k
            self.mask[i] = idx

    def rows(self):
        return [(int(self.surf[i]), self.p[k], self.n[k]) for i, k in enumerate(self.mask) if k >= 0]


class DiskContact:
    def __init__(self, centers, normals, radii, surface):
        self.c = np.asarray(centers, float).reshape(-1, 3).copy()
        n = np.asarray(normals, float).reshape(-1, 3)
        self.n = n / np.linalg.norm(n, axis=1, keepdims=True)
        self.r = np.asarray(radii, float).ravel().copy()
        self.surf = np.asarray(surface, int).ravel()
        self.mask = -np.ones(self.surf.size, int)
        self.frozen = False

    def set_disk(self, center, normal, radius, idx=0):
        self.c[idx] = center
        self.n[idx] = np.asarray(normal, float) / np.linalg.norm(normal)
        self.r[idx] = radius

    def _pd(self, d, x):
        return float(self.n[d] @ (x - self.c[d]))

    def _rd(self, d, x):
        v = x - self.c[d]
        return float(np.linalg.norm(v - (self.n[d] @ v) * self.n[d]))

    def update(self, x):
        xs = x.reshape(-1, 3)[self.surf]
        clear = 3.0 * DISK_PLANAR_CONSTRAINT_THRESHOLD
        depth = 5.0 * DISK_PLANAR_CONSTRAINT_THRESHOLD
        if self.frozen:
            if all(self._pd(d, xs[i]) >= clear for i, d in enumerate(self.mask) if d >= 0):
                self.frozen = False
                self.mask[:] = -1
            return
        hit = np.zeros(self.c.shape[0], bool)
        for i in range(self.surf.size):
            for d in range(self.c.shape[0]):
                if self._pd(d, xs[i]) >= DISK_PLANAR_CONSTRAINT_THRESHOLD:
                    continue
                if self._rd(d, xs[i]) > self.r[d] + DISK_RADIAL_CONSTRAINT_THRESHOLD:
                    continue
                hit[d] = True
        self.mask[:] = -1
        if not hit.any():
            return
        active = 0
        for d in range(self.c.shape[0]):
            if not hit[d]:
                continue
            for i in range(self.surf.size):
                pd = self._pd(d, xs[i])
                if pd > DISK_PLANAR_CONSTRAINT_THRESHOLD or pd < -depth:
                    continue
                if self._rd(d, xs[i]) > self.r[d] + DISK_RADIAL_CONSTRAINT_THRESHOLD:
                    continue
                if self.mask[i] == -1:
                    self.mask[i] = d
                    active += 1
                elif abs(pd) < abs(self._pd(self.mask[i], xs[i])):
                    self.mask[i] = d
        if active:
            self.frozen = True

    def rows(self):
        return [(int(self.surf[i]), self.c[d], self.n[d]) for i, d in enumerate(self.mask) if d >= 0]


class MaxDistance:
    """MaxDistance (cpp/src/constraints/maxDistance.cpp:4-80): g_k = d_k - |x_i - x_j| >= 0 for every
    pair, always active (fixed constraint flag, maxDistance.h:26-33); QP row -u.dx_i + u.dx_j >= |x_i - x_j| - d_k
    with u = (x_i - x_j) / |x_i - x_j| (a zero u when the vertices coincide, as Eigen's normalized())."""

    def __init__(self, vertex1, vertex2, max_distance):
        self.i = np.asarray(vertex1, int).ravel()
        self.j = np.asarray(vertex2, int).ravel()
        self.d = np.asarray(max_distance, float).ravel()

    def rows(self, x, n):
        xs = x.reshape(-1, 3)
        diff = xs[self.i] - xs[self.j]
        L = np.linalg.norm(diff, axis=1)
        u = np.where(L[:, None] > 0.0, diff / np.where(L > 0.0, L, 1.0)[:, None], 0.0)
        ri, ci, vi = [], [], []
        for r in range(self.d.size):
            for k in range(3):
                ri += [r, r]; ci += [3 * self.i[r] + k, 3 * self.j[r] + k]; vi += [-u[r, k], u[r, k]]
        return sp.csr_matrix((vi, (ri, ci)), shape=(self.d.size, n)), L - self.d


def solve_qp(H, g, Aeq, beq, Ain, bin_, max_iter=50):
    """min 1/2 dx'H dx + g'dx s.t. Aeq dx = beq, Ain dx >= bin_ (exact, active set)."""
    n = H.shape[0]
    m = Ain.shape[0]
    work = bin_ > 0.0
    for _ in range(max_iter):
        A = sp.vstack([Aeq, Ain[work]]).tocsr()
        b = np.concatenate([beq, bin_[work]])
        K = sp.bmat([[H, A.T], [A, None]]).tocsc()
        z = spla.spsolve(K, np.concatenate([-g, b]))
        dx = z[:n]
        y = -z[n:]
        mu = np.zeros(m)
        mu[work] = y[Aeq.shape[0]:]
        slack = Ain @ dx - bin_
        scale_s = 1e-12 + 1e-9 * (np.abs(bin_).max() if m else 0.0)
        scale_mu = 1e-14 + 1e-8 * (np.abs(mu).max() if m else 0.0)
        add = (~work) & (slack < -scale_s)
        drop = work & (mu < -scale_mu)
        if not add.any() and not drop.any():
            return dx, work, mu
        work = (work | add) & ~drop
    return dx, work, mu


# OSQP defaults (published with the solver) and the reference's settings
OSQP_RHO = 0.1
OSQP_SIGMA = 1e-6
OSQP_ALPHA = 1.6
OSQP_EPS_ABS = 1e-3
OSQP_EPS_REL = 1e-3
OSQP_CHECK_TERMINATION = 25
OSQP_RHO_EQ_OVER_INEQ = 1e3     # equality rows (|u - l| < 1e-4) get a 1e3 times larger step size
OSQP_RHO_TOL = 1e-4
OSQP_ADAPTIVE_RHO_TOLERANCE = 5.0
OSQP_RHO_MIN, OSQP_RHO_MAX = 1e-6, 1e6
MAX_ITER_QP = 250               # cpp/headers/common.h:23


class OSQPNonConvex(RuntimeError):
    """OSQP's set-up rejects the problem: P + sigma I + A' diag(rho) A is not
    positive definite (the KKT matrix lacks n positive pivots)."""


def _osqp_factor(P, A, rho_vec):
    n = P.shape[0]
    M = (P + OSQP_SIGMA * sp.identity(n) + (A.T @ sp.diags(rho_vec) @ A if A.shape[0] else 0)).tocsc()
    lu = spla.splu(M, permc_spec="MMD_AT_PLUS_A", diag_pivot_thresh=0.0, options={"SymmetricMode": True})
    # symmetric pivoting: the signs of U's diagonal are the inertia of M
    if not (lu.U.diagonal() > 0.0).all():
        raise OSQPNonConvex("non-convex problem")
    return lu


def osqp_solve(P, q, A, l, u, max_iter=MAX_ITER_QP):
    """min 1/2 x'Px + q'x s.t. l <= Ax <= u by OSQP's ADMM (cold start, no
    scaling, no polishing).  Returns (x, iterations, converged)."""
    P = sp.csr_matrix(P)
    A = sp.csr_matrix(A) if A is not None and A.shape[0] else sp.csr_matrix((0, P.shape[0]))
    n, m = P.shape[0], A.shape[0]
    l = np.asarray(l, float); u = np.asarray(u, float)
    eq = np.abs(u - l) < OSQP_RHO_TOL
    rho = OSQP_RHO

    def rho_vec(r):
        v = np.full(m, r)
        v[eq] *= OSQP_RHO_EQ_OVER_INEQ
        return v

    rv = rho_vec(rho)
    lu = _osqp_factor(P, A, rv)
    x = np.zeros(n); z = np.zeros(m); y = np.zeros(m)
    converged = False
    it = 0
    for it in range(1, max_iter + 1):
        # KKT solve with nu eliminated: (P + sigma I + A' R A) xt = sigma x - q + A'(R z - y), zt = A xt
        xt = lu.solve(OSQP_SIGMA * x - q + (A.T @ (rv * z - y) if m else 0.0))
        zt = A @ xt if m else np.zeros(0)
        x = OSQP_ALPHA * xt + (1.0 - OSQP_ALPHA) * x
        zr = OSQP_ALPHA * zt + (1.0 - OSQP_ALPHA) * z
        z_new = np.clip(zr + y / rv, l, u) if m else z
        y = y + rv * (zr - z_new) if m else y
        z = z_new
        if it % OSQP_CHECK_TERMINATION == 0 or it == max_iter:
            Ax = A @ x if m else np.zeros(0)
            Px = P @ x
            Aty = A.T @ y if m else np.zeros(n)
            r_prim = np.abs(Ax - z).max(initial=0.0)
            r_dual = np.abs(Px + q + Aty).max(initial=0.0)
            s_prim = max(np.abs(Ax).max(initial=0.0), np.abs(z).max(initial=0.0))
            s_dual = max(np.abs(Px).max(initial=0.0), np.abs(Aty).max(initial=0.0), np.abs(q).max(initial=0.0))
            if r_prim <= OSQP_EPS_ABS + OSQP_EPS_REL * s_prim and r_dual <= OSQP_EPS_ABS + OSQP_EPS_REL * s_dual:
                converged = True
                break
            if m:
                num = r_prim / (s_prim + 1e-30)
                den = r_dual / (s_dual + 1e-30)
                new = min(max(rho * np.sqrt(num / (den + 1e-30)), OSQP_RHO_MIN), OSQP_RHO_MAX)
                if new > OSQP_ADAPTIVE_RHO_TOLERANCE * rho or new < rho / OSQP_ADAPTIVE_RHO_TOLERANCE:
                    rho = new
                    rv = rho_vec(rho)
                    lu = _osqp_factor(P, A, rv)
    return x, it, converged


class SQPOracle:
    """One rollout of Solver::step with minimize_SQP (backward Euler)."""

    def __init__(self, system, planes=None, disks=None, neumann=None, max_distance=None, qp="exact"):
        if qp not in ("exact", "osqp"):
            raise ValueError(qp)
        self.qp = qp
        self.qp_unconverged = 0   # OSQP solves that stopped at MAX_ITER_QP (the reference uses them anyway)
        self.s = system
        self.planes = planes
        self.disks = disks
        self.max_distance = max_distance
        self.held_pairs = np.zeros(0, int)
        self.mask = None if neumann is None else np.asarray(neumann[0]).ravel().astype(bool)
        self.val = None if neumann is None else np.asarray(neumann[1], float).ravel()
        self.last_iters = 0
        self.last_active = 0

    def minimize(self, q, dt):
        x = np.array(q, float).ravel().copy()
        n = x.size
        for c in (self.planes, self.disks):
            if c is not None:
                c.update(x)
        rows = []
        taken = set()
        fixed_nodes = set() if self.mask is None else set(np.nonzero(self.mask.reshape(-1, 3).any(1))[0].tolist())
        for c in (self.planes, self.disks):
            if c is None:
                continue
            for v, p, nn in c.rows():
                if v in taken or v in fixed_nodes:
                    continue
                taken.add(v)
                rows.append((v, p, nn))
        self.last_active = len(rows)
        qPrev, _, _ = self.s.state()
        eq = np.nonzero(self.mask)[0] if self.mask is not None else np.zeros(0, int)
        Aeq = sp.csr_matrix((np.ones(eq.size), (np.arange(eq.size), eq)), shape=(eq.size, n))
        ri, ci, vi = [], [], []
        for r, (v, p, nn) in enumerate(rows):
            for k in range(3):
                ri.append(r); ci.append(3 * v + k); vi.append(nn[k])
        Ain = sp.csr_matrix((vi, (ri, ci)), shape=(len(rows), n))
        for it in range(MAX_ITER):
            g = self.s.gradient(x, dt)
            H, st = self.s.hessian_csr(x, dt)
            assert st == 0, "inverted element"
            beq = -(x[eq] - qPrev[eq] - dt * self.val[eq]) if eq.size else np.zeros(0)
            bin_ = np.array([-(nn @ (x[3 * v:3 * v + 3] - p)) for v, p, nn in rows])
            A_all, b_all = Ain, bin_
            if self.max_distance is not None:
                Ap, bp = self.max_distance.rows(x, n)
                A_all = sp.vstack([Ain, Ap]).tocsr()
                b_all = np.concatenate([bin_, bp])
            if self.qp == "osqp":
                # rows as Energy::compute_constraint_bounds: equalities l = u, inequalities [l, inf)
                A_q = sp.vstack([Aeq, A_all]).tocsr()
                l_q = np.concatenate([beq, b_all])
                u_q = np.concatenate([beq, np.full(b_all.size, np.inf)])
                try:
                    dx, _, ok = osqp_solve(H, g, A_q, l_q, u_q)
                except OSQPNonConvex:
                    raise RuntimeError("OSQP solver failed")
                self.qp_unconverged += not ok
                x += dx
                if np.isnan(dx).any():
                    raise RuntimeError("SQP method diverged")
                if np.linalg.norm(dx) < DX_TOL:
                    self.last_iters = it + 1
                    return x
                continue
            dx, work, _ = solve_qp(H, g, Aeq, beq, A_all, b_all)
            self.held_pairs = np.nonzero(work[len(rows):])[0]
            x += dx
            if np.isnan(dx).any():
                raise RuntimeError("SQP method diverged")
            if np.linalg.norm(dx) < DX_TOL:
                self.last_iters = it + 1
                return x
        raise RuntimeError("SQP method did not converge")

    def step(self, q, dt):
        x = self.minimize(q, dt)
        self.s.update_state(x, dt)
        return x
