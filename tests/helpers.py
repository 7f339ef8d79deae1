"""Shared builders: the same mesh and settings for the GPU path and the oracle."""
from __future__ import annotations

import numpy as np

from sors_b200 import meshes


def make_pair(X, T, *, rho=1070.0, E=1e5, nu=0.45, grav=(0.0, 0.0, -9.81), alpha=0.0, dt=1e-3,
              scheme="backward_euler", method="minimize_newton", precision="fp64", project=True,
              clamp=True, res_tol=0.0, faces=None, groups=None, vertex_force=False, oracle_project=False,
              muscles=None, energy="neohookean", two_level=False, substeps=1, cfl=False):
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
    s.substeps = substeps
    s.CFLtimeSteppingFlag = cfl
    s.timeSteppingScheme = scheme
    s.solverMethod = method
    s.precision = precision
    s.hessianProjection = project
    s.newtonResidualTol = res_tol
    s.twoLevelPreconditioner = two_level
    energies = [{energy}] * ne
    params = [ps.Params(["density", "youngsModulus", "poissonsRatio"], [rhov[i], Ev[i], nuv[i]]) for i in range(ne)]
    if muscles is not None:
        # per-element "softconMuscle" energies with their Params (tetrahedron.cpp:82-88)
        energies = list(energies)
        for i in range(ne):
            if muscles["group"][i] >= 0:
                energies[i] = {energy, "softconMuscle"}
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
                   project=oracle_project, dt=dt, substeps=substeps, cfl=cfl,
                   material=orc.MAT_STABLE_NEOHOOKEAN if energy == "stableneohookean" else orc.MAT_NEOHOOKEAN)
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


def contact_pair(X, T, *, planes=None, disks=None, surface=None, rho=1070.0, E=1e5, nu=0.45,
                 grav=(0.0, 0.0, -9.81), dt=1e-3, precision="fp64", project=True, neumann=None, muscles=None,
                 two_level=False, max_distance=None):
    """GPU Energy/Solver with minimize_SQP and the oracle's SQP on the same scene.

    planes: (points (k,3), normals (k,3)); disks: (centers, normals, radii);
    max_distance: (vertex1, vertex2, distances);
    surface: candidate contact vertices (all surface vertices when None);
    neumann: (mask 3N, value 3N) or None."""
    from oracle import oracle as orc
    from oracle import contact as oc
    from sors_b200 import py_sors as ps
    X = np.asarray(X, float)
    T = np.asarray(T, np.int32)
    ne = T.shape[0]
    if surface is None:
        groups, _ = meshes.extract_surfaces(X, T)
        surface = np.unique(np.concatenate([g.ravel() for g in groups]))
    surface = np.asarray(surface, np.int32)
    Ev = np.broadcast_to(np.asarray(E, float), (ne,)).copy()
    s = ps.SimulationSettings()
    s.meshType = "Tetrahedron" if T.shape[1] == 4 else "Hexahedron"
    s.dt = dt
    s.timeSteppingScheme = "backward_euler"
    s.solverMethod = "minimize_SQP"
    s.precision = precision
    s.hessianProjection = project
    s.twoLevelPreconditioner = two_level
    ctypes_, cp = [], ps.Params()
    if neumann is not None:
        ctypes_.append("neumannBC")
        cp.set_param("neumannBCmask", np.asarray(neumann[0], float))
        cp.set_param("neumannBCvalue", np.asarray(neumann[1], float))
    if planes is not None:
        ctypes_.append("planeContact")
        cp.set_param("positionVectorListPlanes", np.asarray(planes[0], float).ravel())
        cp.set_param("normalVectorListPlanes", np.asarray(planes[1], float).ravel())
    if disks is not None:
        ctypes_.append("diskContact")
        cp.set_param("diskCenterVectorList", np.asarray(disks[0], float).ravel())
        cp.set_param("diskNormalVectorList", np.asarray(disks[1], float).ravel())
        cp.set_param("diskRadiusList", np.asarray(disks[2], float).ravel())
    if planes is not None or disks is not None:
        cp.set_param("surfaceVerticesIdx", surface.astype(float))
    if max_distance is not None:
        ctypes_.append("maxDistance")
        cp.set_param("maxDistanceVertex1Indices", np.asarray(max_distance[0], float))
        cp.set_param("maxDistanceVertex2Indices", np.asarray(max_distance[1], float))
        cp.set_param("maxDistanceList", np.asarray(max_distance[2], float))
    en = ps.EnergyTet.from_arrays if T.shape[1] == 4 else ps.EnergyHex.from_arrays
    en = en(X, T, s, np.asarray(grav, float), 0.0, density=rho, youngsModulus=Ev, poissonsRatio=nu,
            muscleGroup=None if muscles is None else muscles["group"],
            softconStiffness=None if muscles is None else muscles["k"],
            softconDirection=None if muscles is None else muscles["dir"])
    en._setup_constraints_forces(ctypes_, cp, (), None)
    sol = ps.Solver(s)
    o = orc.System(X, T, rho=rho, youngs=Ev, nu=nu, grav=grav, scheme="backward_euler", method="minimize_SQP",
                   project=False, dt=dt, substeps=1)
    if muscles is not None:
        o.set_muscles(muscles["group"], muscles["k"], muscles["dir"], int(max(muscles["group"])) + 1)
    pl = None if planes is None else oc.PlaneContact(planes[0], planes[1], surface)
    dk = None if disks is None else oc.DiskContact(disks[0], disks[1], disks[2], surface)
    md = None if max_distance is None else oc.MaxDistance(*max_distance)
    sq = oc.SQPOracle(o, pl, dk, neumann, max_distance=md)
    return en, sol, sq, surface


def two_cubes(n=2, s=0.004, gap=0.002, kind="hex"):
    """Two n^3-cell cubes of side s, gap apart along x; returns (X, T, a, b, n1) with
    a the max-x vertex of the first cube and b the min-x vertex of the second, both at
    mid height and mid depth (the pair of a maxDistance rope), n1 the first cube's
    vertex count."""
    X, H = meshes.hex_bar(n, n, n, (s, s, s))
    T = H if kind == "hex" else meshes.kuhn_tet_elements(n, n, n)
    X2 = X + np.array([s + gap, 0.0, 0.0])
    off = 1e-3 * (np.abs(X[:, 1] - s / 2) + np.abs(X[:, 2] - s / 2))
    a = int(np.argmax(X[:, 0] - off))
    b = X.shape[0] + int(np.argmin(X[:, 0] + off))
    return np.vstack([X, X2]), np.vstack([T, T + X.shape[0]]).astype(np.int32), a, b, X.shape[0]
