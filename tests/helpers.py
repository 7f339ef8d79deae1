"""Shared builders: the same mesh and settings for the GPU path and the oracle."""
from __future__ import annotations

import numpy as np

from sors_b200 import meshes


def make_pair(X, T, *, rho=1070.0, E=1e5, nu=0.45, grav=(0.0, 0.0, -9.81), alpha=0.0, dt=1e-3,
              scheme="backward_euler", method="minimize_newton", precision="fp64", project=True,
              clamp=True, res_tol=0.0, faces=None, groups=None, vertex_force=False, oracle_project=False,
              muscles=None):
    """(gpu_energy, gpu_solver, oracle_system, X) on one mesh."""
    from oracle import oracle as orc
    from sors_b200 import py_sors as ps
    X = np.asarray(X, float)
    T = np.asarray(T, np.int32)
    ne = T.shape[0]
    Ev = np.broadcast_to(np.asarray(E, float), (ne,)).copy()
    nuv = np.broadcast_to(np.asarray(nu, float), (ne,)).copy()
    rhov = np.broadcast_to(np.asarray(rho, float), (ne,)).copy()
    s = ps.SimulationSettings()
    s.meshType = "Tetrahedron" if T.shape[1] == 4 else "Hexahedron"
    s.dt = dt
    s.substeps = 1
    s.timeSteppingScheme = scheme
    s.solverMethod = method
    s.precision = precision
    s.hessianProjection = project
    s.newtonResidualTol = res_tol
    energies = [{"neohookean"}] * ne
    params = [ps.Params(["density", "youngsModulus", "poissonsRatio"], [rhov[i], Ev[i], nuv[i]]) for i in range(ne)]
    if muscles is not None:
        # per-element "softconMuscle" energies with their Params (tetrahedron.cpp:82-88)
        energies = list(energies)
        for i in range(ne):
            if muscles["group"][i] >= 0:
                energies[i] = {"neohookean", "softconMuscle"}
                params[i].set_param("muscleGroup", float(muscles["group"][i]))
                params[i].set_param("softconStiffness", float(muscles["k"][i]))
                params[i].set_param("softconDirection", np.asarray(muscles["dir"][i], float).reshape(1, 3))
    ctypes_, cparams = [], ps.Params()
    mask = val = None
    if clamp:
        mask, val = meshes.clamp_mask(X)
        ctypes_.append("neumannBC")
        cparams.set_param("neumannBCmask", mask.astype(float))
        cparams.set_param("neumannBCvalue", val)
    ftypes, fparams = [], ps.Params()
    if faces is not None:
        ftypes.append("pressure")
        fparams.set_param("surfaceVertexIdx", np.asarray(faces, float))
        fparams.set_param("surfaceGroups", np.asarray(groups, float))
    if vertex_force:
        ftypes.append("vertexForce")
    en = ps.Energy(X, T, s, np.asarray(grav, float), alpha, energies, params, ctypes_, cparams, ftypes, fparams)
    sol = ps.Solver(s)
    o = orc.System(X, T, rho=rhov, youngs=Ev, nu=nuv, grav=grav, alpha=alpha, scheme=scheme, method=method,
                   project=oracle_project, dt=dt, substeps=1)
    if clamp:
        o.set_neumann(mask, val)
    if faces is not None:
        o.set_pressure(np.asarray(faces), np.asarray(groups))
    if vertex_force:
        o.set_vertex_force(True)
    if muscles is not None:
        o.set_muscles(muscles["group"], muscles["k"], muscles["dir"], int(max(muscles["group"])) + 1)
    return en, sol, o, s


def rel_err(a, b):
    a = np.asarray(a, float); b = np.asarray(b, float)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def deform(X, rng, amp=0.05, scale=None):
    X = np.asarray(X, float)
    L = np.ptp(X, axis=0).max() if scale is None else scale
    A = np.eye(3) + rng.uniform(-amp, amp, (3, 3))
    return (X @ A.T + rng.uniform(-amp, amp, X.shape) * L * 0.02).ravel()
