"""Differentiable rollouts: the adjoint of the implicit backward-Euler step.

No reference counterpart: SORS has no differentiation.  A rollout runs T steps
of `Solver.step` from (q0, v0) with per-element Young's moduli E and per-step
SoftCon activations act[t] (one per muscle group), and returns the final
positions.  Its gradient runs backwards through the steps: each step's
implicit residual g(q_{t+1}; q_t, v_t, E, act_t) = 0 is differentiated by
`sors_adjoint_step` (one transpose solve with the step's exact Hessian plus
element-level derivatives on the GPU), chained through the state
(q_{t+1}, v_{t+1} = (q_{t+1} - q_t) / dt).

States are checkpointed every `checkpoint_every` steps during the forward pass
(positions, velocities and the disk contacts' state); the backward pass
recomputes each segment from its checkpoint (the GPU path is deterministic, so
the recomputed states equal the forward ones bit for bit).  Contact steps
(minimize_SQP) are differentiated with the contacts they held as equalities;
held maxDistance pairs enter as equalities too, with their constraint
curvature (the multiplier times the Hessian of |x_i - x_j|) in the transpose
system.

Crank-Nicolson rollouts (`timeSteppingScheme = "crank_nicolson"`) chain the
state's previous-step force as well (`sors_adjoint_step_cn`; checkpoints keep
it).

`rollout(...)` is the torch entry point: a torch.autograd.Function whose inputs
are float64 tensors E (E,) and act (T, G).  Follower-load pressures per step
(`RolloutAdjoint.forward(..., pressure=...)`) are differentiated too
(`grad_pressure` after `backward`).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def _p(a, ct=C.c_double):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


class RolloutAdjoint:
    """Forward rollout with checkpoints, and its adjoint, on one Energy/Solver pair."""

    def __init__(self, energy, solver, steps: int, dt: float, q0=None, v0=None, poisson=None,
                 checkpoint_every: int = 1, before_step=None):
        self.en = energy
        self.sol = solver
        self.steps = int(steps)
        self.dt = float(dt)
        n = energy.ndof
        self.q0 = np.ascontiguousarray(energy.undeformedVertices.ravel() if q0 is None else q0, dtype=np.float64)
        self.v0 = np.zeros(n) if v0 is None else np.ascontiguousarray(v0, dtype=np.float64).ravel()
        ne = energy.numElements
        self.poisson = np.ascontiguousarray(np.broadcast_to(
            np.asarray(0.45 if poisson is None else poisson, np.float64), (ne,)))
        self.k = max(1, int(checkpoint_every))
        self.before_step = before_step  # callable(t): moves disks etc. before step t
        self._ckpt = {}
        self._held = {}
        self._cstate0 = None
        self._E = None
        self._act = None
        self._pressure = None
        self.grad_pressure = None  # dL/d pressure (T, groups) after backward, with a pressure schedule
        self.last_pcg_iters = 0
        # Crank-Nicolson: the state carries the previous step's internal force
        # (zero at the start), and v_{t+1} = 2 (q_{t+1} - q_t) / dt - v_t
        self.cn = int(energy._settings_c.time_stepping) == 1

    # -- helpers --------------------------------------------------------------
    def _set_material(self, E):
        L = _lib.load()
        E = np.ascontiguousarray(E, dtype=np.float64)
        _lib.check(L.sors_set_material(self.en._h, _p(E), _p(self.poisson)))

    def _set_act(self, a):
        if a is None or a.size == 0:
            return
        a = np.ascontiguousarray(a, dtype=np.float64)
        _lib.check(_lib.load().sors_set_actuation(self.en._h, b"softconMuscle", _p(a), a.size))

    def _set_pressure(self, p):
        if p is None or p.size == 0:
            return
        p = np.ascontiguousarray(p, dtype=np.float64)
        _lib.check(_lib.load().sors_set_actuation(self.en._h, b"pressure", _p(p), p.size))

    def _contact_state(self):
        L = _lib.load()
        k = L.sors_get_contact_state(self.en._h, None, 0)
        st = np.zeros(k, np.int32)
        L.sors_get_contact_state(self.en._h, _p(st, C.c_int32), k)
        return st

    def _restore(self, q, v, cstate, g=None):
        self.en.set_initial_deformation(q)
        self.en.set_initial_velocity(v)
        if self.cn:
            g = np.zeros(self.en.ndof) if g is None else np.ascontiguousarray(g, dtype=np.float64)
            _lib.check(_lib.load().sors_set_prev_force(self.en._h, _p(g)))
        _lib.check(_lib.load().sors_set_contact_state(self.en._h, _p(cstate, C.c_int32), cstate.size))

    def _prev_force(self):
        if not self.cn:
            return None
        g = np.zeros(self.en.ndof)
        _lib.check(_lib.load().sors_get_prev_force(self.en._h, _p(g)))
        return g

    def _held_now(self):
        L = _lib.load()
        k = L.sors_held_contacts(self.en._h, None, None, 0)
        nodes = np.zeros(max(k, 1), np.int32); normals = np.zeros((max(k, 1), 3))
        if k:
            L.sors_held_contacts(self.en._h, _p(nodes, C.c_int32), _p(normals), k)
        kp = L.sors_held_pairs(self.en._h, None, None, 0)
        pairs = np.zeros(max(kp, 1), np.int32); mu = np.zeros(max(kp, 1))
        if kp:
            L.sors_held_pairs(self.en._h, _p(pairs, C.c_int32), _p(mu), kp)
        return nodes[:k].copy(), normals[:k].copy(), pairs[:kp].copy(), mu[:kp].copy()

    def _step(self, q, t):
        if self.before_step is not None:
            self.before_step(t)
        self._set_act(None if self._act is None else self._act[t])
        self._set_pressure(None if self._pressure is None else self._pressure[t])
        qn = self.sol.step(q, self.en, None, self.dt)
        self._held[t] = self._held_now()
        return qn

    # -- forward ----------------------------------------------------------------
    def forward(self, E, act=None, pressure=None):
        """Runs the rollout; returns q_T.  E: (E,), act: (T, G) or None,
        pressure: (T, pressure groups) follower-load pressures per step or None."""
        self._E = np.array(E, dtype=np.float64)
        self._act = None if act is None else np.array(act, dtype=np.float64).reshape(self.steps, -1)
        self._pressure = None if pressure is None else np.array(pressure, dtype=np.float64).reshape(self.steps, -1)
        self._set_material(self._E)
        self._restore(self.q0, self.v0, self._contact_state() if self._cstate0 is None else self._cstate0)
        if self._cstate0 is None:
            self._cstate0 = self._contact_state()
        q = self.q0.copy()
        v = self.v0.copy()
        self._ckpt = {}
        self._held = {}
        for t in range(self.steps):
            if t % self.k == 0:
                self._ckpt[t] = (q.copy(), v.copy(), self._contact_state(), self._prev_force())
            qn = self._step(q, t)
            v = 2.0 * (qn - q) / self.dt - v if self.cn else (qn - q) / self.dt
            q = qn
        return q

    # -- backward ---------------------------------------------------------------
    def backward(self, dL_dqT, dL_dvT=None):
        """Gradient of L(q_T, v_T): returns (dL/dE, dL/dact or None, dL/dq0, dL/dv0)."""
        L = _lib.load()
        n = self.en.ndof
        ne = self.en.numElements
        G = 0 if self._act is None else self._act.shape[1]
        Qb = np.array(dL_dqT, dtype=np.float64).ravel().copy()
        Vb = np.zeros(n) if dL_dvT is None else np.array(dL_dvT, dtype=np.float64).ravel().copy()
        gE = np.zeros(ne)
        gA = None if self._act is None else np.zeros_like(self._act)
        dq = np.zeros(n); dv = np.zeros(n); dE = np.zeros(ne); dA = np.zeros(max(G, 1))
        Gb = np.zeros(n); dG = np.zeros(n)  # Crank-Nicolson: cotangent of the state's previous-step force
        P = 0 if self._pressure is None else self._pressure.shape[1]
        self.grad_pressure = None if P == 0 else np.zeros_like(self._pressure)
        dP = np.zeros(max(P, 1))
        stats = _lib.SorsStepStats()
        self.last_pcg_iters = 0
        self._set_material(self._E)
        starts = sorted(self._ckpt)
        for s in reversed(starts):
            e = min(s + self.k, self.steps)
            q, v, cst, g = self._ckpt[s]
            self._restore(q, v, cst, g)
            qs = [q.copy()]
            for t in range(s, e):
                qs.append(self._step(qs[-1], t))
            for t in range(e - 1, s - 1, -1):
                self._set_act(None if self._act is None else self._act[t])
                self._set_pressure(None if self._pressure is None else self._pressure[t])
                # v_{t+1} = (q_{t+1} - q_t) / dt, or 2 (q_{t+1} - q_t) / dt - v_t (Crank-Nicolson)
                cv = 2.0 / self.dt if self.cn else 1.0 / self.dt
                b = Qb + cv * Vb
                hn, hv, hp, hmu = self._held[t]
                hv = np.ascontiguousarray(hv)
                _lib.check(L.sors_adjoint_set_pairs(self.en._h, _p(hp, C.c_int32) if hp.size else None,
                                                    _p(hmu) if hp.size else None, hp.size))
                if self.cn:
                    _lib.check(L.sors_adjoint_step_cn(self.en._h, _p(qs[t + 1 - s]), self.dt, _p(b), _p(Gb),
                                                      _p(hn, C.c_int32) if hn.size else None,
                                                      _p(hv) if hn.size else None, hn.size, _p(dq), _p(dv), _p(dG),
                                                      _p(dE), _p(dA) if G else None, None, C.byref(stats)))
                    Gb = dG.copy()
                else:
                    _lib.check(L.sors_adjoint_step(self.en._h, _p(qs[t + 1 - s]), self.dt, _p(b),
                                                   _p(hn, C.c_int32) if hn.size else None,
                                                   _p(hv) if hn.size else None, hn.size, _p(dq), _p(dv), _p(dE),
                                                   _p(dA) if G else None, None, C.byref(stats)))
                self.last_pcg_iters += stats.pcg_iters
                gE += dE
                if G:
                    gA[t] = dA[:G]
                if P:
                    _lib.check(L.sors_adjoint_pressure_grad(self.en._h, _p(dP), P))
                    self.grad_pressure[t] = dP[:P]
                Qb = dq - cv * Vb
                Vb = dv - Vb if self.cn else dv.copy()
        return gE, gA, Qb, Vb


def rollout(energy, solver, E, act, steps, dt, q0=None, v0=None, poisson=None, checkpoint_every=1,
            before_step=None):
    """Differentiable final positions q_T (torch float64, shape (3N,)).

    E: torch tensor (E,) of Young's moduli; act: torch tensor (T, G) of SoftCon
    activations or None.  Gradients flow to E and act."""
    import torch

    runner = RolloutAdjoint(energy, solver, steps, dt, q0=q0, v0=v0, poisson=poisson,
                            checkpoint_every=checkpoint_every, before_step=before_step)

    class _Rollout(torch.autograd.Function):
        @staticmethod
        def forward(ctx, Et, At):
            qT = runner.forward(Et.detach().cpu().numpy(), None if At is None else At.detach().cpu().numpy())
            return torch.from_numpy(qT)

        @staticmethod
        def backward(ctx, gq):
            gE, gA, _, _ = runner.backward(gq.detach().cpu().numpy())
            return torch.from_numpy(gE), (None if gA is None else torch.from_numpy(gA))

    out = _Rollout.apply(E, act)
    out.runner = runner
    return out
