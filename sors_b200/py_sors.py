"""Drop-in for the reference's Python module `py_sors` (cpp/py_sors.cpp:25-262).

Same names, argument meaning and error behaviour for the implicit-Euler path:
  Energy(undeformedVertices, eleIdx, settings, gravAcceleration, dampingAlpha,
         elementEnergiesList, elementParameterList, constraintTypesList,
         constraintParameterList, forceTypesList, forceParameterList)
      -> EnergyTet | EnergyHex                       (cpp/py_sors.cpp:30-95)
  Solver(settings) -> SolverTet | SolverHex; .step(solution, systemEnergy,
      act, dt=0.0, substeps=0) and .step(solution, systemEnergy, dt, substeps)
                                                      (cpp/py_sors.cpp:99-148)
  Params, SimulationSettings                          (cpp/py_sors.cpp:151-177)

Everything below the calls runs in libsors_b200.so on the GPU.  Errors the
reference raises as std::runtime_error (surfacing as RuntimeError through
pybind11) are raised as RuntimeError with the same message.  Element energies,
constraints and forces this build does not implement raise NotImplementedError
instead of the reference's exit(1) for unknown names.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

from . import _lib
from . import meshes as _meshes

_SCHEMES = {"backward_euler": 0, "crank_nicolson": 1}
_METHODS = {"minimize_newton": 0, "minimize_newton_linesearch": 1, "minimize_frozenhessian": 2, "minimize_SQP": 3}
_REF_ONLY_METHODS = set()
_REF_ENERGIES = {"neohookean", "stableneohookean", "pseudostrain", "softconMuscle"}
_REF_CONSTRAINTS = {"neumannBC", "planeContact", "diskContact", "maxDistance"}
_REF_FORCES = {"pressure", "vertexForce"}


class SimulationSettings:
    """cpp/headers/simulationSettings.h:18-71, plus the device-solver options."""

    def __init__(self):
        self.description = ""
        self.verbose = 1
        self.meshFilePath = ""
        self.outputFolder = ""
        self.meshFileName = ""
        self.meshType = ""
        self.dt = float("nan")
        self.numSteps = -1
        self.substeps = 1
        self.CFLtimeSteppingFlag = False
        self.timeSteppingScheme = "crank_nicolson"
        self.solverMethod = "minimize_newton"
        self.numThreads = 1
        # device-solver options (no reference counterpart)
        self.precision = "fp64"            # "fp64" | "mixed"
        # SPD projection of dP/dF per quadrature point: True always, False never,
        # "adaptive" (default) the exact Hessian unless PCG meets negative curvature
        self.hessianProjection = "adaptive"
        self.maxBlocksPerKernel = 0        # grid cap per kernel (0: whole GPU)
        self.newtonSafeguard = False       # halve Newton steps that raise ||g|| (adaptive Hessian only)
        # block Jacobi + coarse rigid-body correction: True, False or "auto"
        # (on for meshes of 20,000 nodes or more)
        self.twoLevelPreconditioner = "auto"
        # Newton linear solver of "minimize_newton": "pcg", or "minres" for the
        # exact Newton step of an indefinite Hessian (the reference's LDL^T step)
        self.linearSolver = "pcg"
        # follower-load coefficient of the Newton matrix for quads: "reference"
        # (p/6, as pressureForce.cpp) or "exact" (p/8); the solution is the same
        self.pressureJacobian = "reference"
        self.newtonResidualTol = 0.0       # absolute ||gradient|| stop; 0 = reference dx test only
        self.newtonDxTol = 1e-9            # reference DX_TOL (cpp/headers/common.h:25)
        self.newtonMaxIter = 100           # reference MAX_ITER (cpp/headers/common.h:21)
        self.pcgRelTol = 1e-10
        self.pcgMaxIter = 20000
        self.device = 0
        self.newtonPredictor = True        # start Newton from q + dt v_prev (same solution, fewer iterations)

    def verbose_print(self):
        print("Simulation Description:", self.description or "not indicated")
        for k in ("meshFilePath", "outputFolder", "meshFileName", "meshType", "dt", "numSteps", "substeps",
                  "CFLtimeSteppingFlag", "timeSteppingScheme", "solverMethod", "precision"):
            print(f"{k + ':':25s}{getattr(self, k)}")


class Params:
    """String -> matrix dictionary (cpp/headers/params.h:30-175)."""

    def __init__(self, keys=None, values=None):
        self._d: dict[str, np.ndarray] = {}
        if keys is not None:
            if values is None or len(keys) != len(values):
                raise ValueError("keys and values must have the same length")
            for k, v in zip(keys, values):
                self.set_param(k, v)

    def get_value(self, key):
        if key not in self._d:
            raise KeyError(f"Key not found in the parameter list: {key}")
        return self._d[key].copy()

    def has(self, key):
        return key in self._d

    def set_param(self, key, value=None):
        if value is None:
            return self._load_csv(key)
        if np.isscalar(value):
            m = np.array([[float(value)]])
        else:
            a = np.asarray(value, dtype=np.float64)
            m = a.reshape(-1, 1) if a.ndim == 1 else a.reshape(a.shape[0], -1)
        if key in self._d and self._d[key].size != m.size:
            raise ValueError(f"size mismatch for parameter {key}")
        self._d[key] = m

    def _load_csv(self, filename):
        if not filename.endswith(".csv") or not os.path.exists(filename):
            raise RuntimeError(f"Could not open the file: {filename}")
        with open(filename) as f:
            for line in f:
                cells = line.strip().split(",")
                if len(cells) < 2:
                    continue
                vals = [float(c) for c in cells[1:]]
                self.set_param(cells[0], vals if len(vals) > 1 else vals[0])

    def keys(self):
        return list(self._d.keys())


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct))


class _EnergyBase:
    NV = 0
    MESH = ""

    def __init__(self, undeformedVertices, eleIdx, settings, gravAcceleration, dampingAlpha=0.0,
                 elementEnergiesList=None, elementParameterList=None, constraintTypesList=(),
                 constraintParameterList=None, forceTypesList=(), forceParameterList=None):
        L = _lib.load()
        X = np.ascontiguousarray(np.asarray(undeformedVertices, dtype=np.float64).reshape(-1, 3))
        T = np.ascontiguousarray(np.asarray(eleIdx, dtype=np.int32).reshape(-1, self.NV))
        ne = T.shape[0]
        self.settings = settings
        self.undeformedVertices = X
        self.eleIdx = T
        elementEnergiesList = elementEnergiesList if elementEnergiesList is not None else [set()] * ne
        elementParameterList = elementParameterList if elementParameterList is not None else [Params()] * ne
        if len(elementEnergiesList) != ne or len(elementParameterList) != ne:
            raise ValueError("one energy set and one Params per element are required")
        rho = np.empty(ne); E = np.empty(ne); nu = np.empty(ne)
        mgroup = mk = mdir = None
        material = None
        for i, (es, pr) in enumerate(zip(elementEnergiesList, elementParameterList)):
            es = set(es)
            for name in es:
                if name not in _REF_ENERGIES:
                    raise RuntimeError(f"Unknown energy type: {name}")
            if es - {"neohookean", "stableneohookean", "softconMuscle"}:
                raise NotImplementedError(
                    f"element energies {sorted(es - {'neohookean', 'stableneohookean', 'softconMuscle'})} "
                    "are not built on the GPU path")
            if {"neohookean", "stableneohookean"} <= es:
                raise NotImplementedError("an element with both Neo-Hookean energies is not supported")
            if "softconMuscle" in es:
                # tetrahedron.cpp:82-88 / hexahedron.cpp:51-57
                if mgroup is None:
                    mgroup = np.full(ne, -1, np.int32); mk = np.zeros(ne); mdir = np.zeros((ne, 3))
                mgroup[i] = int(pr.get_value("muscleGroup")[0, 0])
                mk[i] = float(pr.get_value("softconStiffness")[0, 0])
                mdir[i] = np.asarray(pr.get_value("softconDirection"), dtype=np.float64).ravel()[:3]
            rho[i] = float(pr.get_value("density")[0, 0])
            if "neohookean" in es or "stableneohookean" in es:
                E[i] = float(pr.get_value("youngsModulus")[0, 0])
                nu[i] = float(pr.get_value("poissonsRatio")[0, 0])
                kind = 2 if "stableneohookean" in es else 0
                material = kind if material in (None, kind) else -1
            else:
                E[i] = 0.0; nu[i] = 0.0
                material = 1 if material in (None, 1) else -1
        if material == -1:
            raise NotImplementedError("a mesh mixing elastic energy models (or elements without one) is not supported")
        if material == 1:
            # elements without energies only carry mass (Energy with empty sets)
            material = 0
        self._init_arrays(X, T, settings, gravAcceleration, dampingAlpha, rho, E, nu, material or 0)
        if mgroup is not None:
            self.set_muscles(mgroup, mk, mdir)
        self._setup_constraints_forces(constraintTypesList, constraintParameterList, forceTypesList,
                                       forceParameterList)

    def _setup_constraints_forces(self, constraintTypesList, constraintParameterList, forceTypesList,
                                  forceParameterList):
        """Constraint and force set-up of Energy<3,E>::Energy (cpp/src/energy.cpp:58-174)."""
        L = _lib.load()
        cp = constraintParameterList if constraintParameterList is not None else Params()
        fp = forceParameterList if forceParameterList is not None else Params()
        self._forces = list(forceTypesList)
        self._constraints = list(constraintTypesList)
        for c in constraintTypesList:
            if c not in _REF_CONSTRAINTS:
                raise RuntimeError(f"Unknown constraint type: {c}")
            if c == "neumannBC":
                mask = np.ascontiguousarray(cp.get_value("neumannBCmask").ravel().astype(np.int32))
                val = np.ascontiguousarray(cp.get_value("neumannBCvalue").ravel().astype(np.float64))
                if mask.size != self.ndof or val.size != self.ndof:
                    raise ValueError("neumannBCmask/neumannBCvalue must have 3N entries")
                _lib.check(L.sors_set_neumann(self._h, _p(mask, C.c_int32), _p(val, C.c_double)))
            elif c == "planeContact":
                # energy.cpp:69-84
                pts = np.ascontiguousarray(cp.get_value("positionVectorListPlanes").ravel().astype(np.float64))
                nrm = np.ascontiguousarray(cp.get_value("normalVectorListPlanes").ravel().astype(np.float64))
                surf = np.ascontiguousarray(cp.get_value("surfaceVerticesIdx").ravel().astype(np.int32))
                if pts.size != nrm.size or pts.size % 3:
                    raise ValueError("plane points and normals must be lists of 3-vectors of the same length")
                _lib.check(L.sors_set_plane_contact(self._h, _p(pts, C.c_double), _p(nrm, C.c_double), pts.size // 3,
                                                    _p(surf, C.c_int32), surf.size))
            elif c == "diskContact":
                # energy.cpp:85-108
                cen = np.ascontiguousarray(cp.get_value("diskCenterVectorList").ravel().astype(np.float64))
                nrm = np.ascontiguousarray(cp.get_value("diskNormalVectorList").ravel().astype(np.float64))
                rad = np.ascontiguousarray(cp.get_value("diskRadiusList").ravel().astype(np.float64))
                surf = np.ascontiguousarray(cp.get_value("surfaceVerticesIdx").ravel().astype(np.int32))
                if cen.size != nrm.size or cen.size % 3 or rad.size != cen.size // 3:
                    raise ValueError("DiskContact: centers/normals must be same length and multiples of 3")
                _lib.check(L.sors_set_disk_contact(self._h, _p(cen, C.c_double), _p(nrm, C.c_double),
                                                   _p(rad, C.c_double), rad.size, _p(surf, C.c_int32), surf.size))
            elif c == "maxDistance":
                # energy.cpp:109-120
                v1 = np.ascontiguousarray(cp.get_value("maxDistanceVertex1Indices").ravel().astype(np.int32))
                v2 = np.ascontiguousarray(cp.get_value("maxDistanceVertex2Indices").ravel().astype(np.int32))
                dm = np.ascontiguousarray(cp.get_value("maxDistanceList").ravel().astype(np.float64))
                if not (v1.size == v2.size == dm.size):
                    raise ValueError("MaxDistance constraint parameters must have the same size.")
                if v1.size == 0:
                    raise ValueError("MaxDistance constraint pair is empty. Remove this constraint.")
                _lib.check(L.sors_set_max_distance(self._h, _p(v1, C.c_int32), _p(v2, C.c_int32),
                                                   _p(dm, C.c_double), v1.size))
            else:
                raise NotImplementedError(f"constraint {c} is not built on the GPU path")
        for f in forceTypesList:
            if f not in _REF_FORCES:
                raise RuntimeError(f"Unknown force type: {f}")
            if f == "pressure":
                faces = np.ascontiguousarray(fp.get_value("surfaceVertexIdx").astype(np.int32))
                groups = np.ascontiguousarray(fp.get_value("surfaceGroups").ravel().astype(np.int32))
                self._n_groups = int(groups.max()) + 1 if groups.size else 0
                _lib.check(L.sors_set_pressure_faces(self._h, _p(faces, C.c_int32), faces.shape[0], faces.shape[1],
                                                     _p(groups, C.c_int32), self._n_groups))
            elif f == "vertexForce":
                _lib.check(L.sors_enable_vertex_force(self._h, 1))

    def _init_arrays(self, X, T, settings, gravAcceleration, dampingAlpha, rho, E, nu, material=0):
        L = _lib.load()
        X = np.ascontiguousarray(np.asarray(X, dtype=np.float64).reshape(-1, 3))
        T = np.ascontiguousarray(np.asarray(T, dtype=np.int32).reshape(-1, self.NV))
        ne = T.shape[0]
        rho = np.ascontiguousarray(np.broadcast_to(np.asarray(rho, np.float64), (ne,)))
        E = np.ascontiguousarray(np.broadcast_to(np.asarray(E, np.float64), (ne,)))
        nu = np.ascontiguousarray(np.broadcast_to(np.asarray(nu, np.float64), (ne,)))
        self.settings = settings
        self.undeformedVertices = X
        self.eleIdx = T
        self._material = material
        self._forces = []
        self._n_groups = 0
        s = _lib.default_settings()
        if settings.timeSteppingScheme not in _SCHEMES:
            raise RuntimeError(f"Unknown time stepping scheme: {settings.timeSteppingScheme}")
        s.time_stepping = _SCHEMES[settings.timeSteppingScheme]
        if settings.solverMethod in _REF_ONLY_METHODS:
            raise NotImplementedError(f"{settings.solverMethod} is not built on the GPU path")
        s.solver_method = _METHODS.get(settings.solverMethod, 0)
        s.dt = 0.0 if (settings.dt is None or math.isnan(settings.dt)) else float(settings.dt)
        s.substeps = int(settings.substeps)
        s.cfl = int(bool(settings.CFLtimeSteppingFlag))
        g = np.asarray(gravAcceleration, dtype=np.float64).ravel()
        for k in range(3):
            s.grav[k] = float(g[k])
        s.damping_alpha = float(dampingAlpha)
        s.precision = 1 if getattr(settings, "precision", "fp64") == "mixed" else 0
        hp = getattr(settings, "hessianProjection", "adaptive")
        s.project_spd = 2 if (isinstance(hp, str) and hp == "adaptive") else int(bool(hp))
        s.material = int(getattr(settings, "_material_override", self._material))
        s.newton_dx_tol = float(getattr(settings, "newtonDxTol", 1e-9))
        s.newton_res_tol = float(getattr(settings, "newtonResidualTol", 0.0))
        s.newton_max_iter = int(getattr(settings, "newtonMaxIter", 100))
        s.pcg_rel_tol = float(getattr(settings, "pcgRelTol", 1e-10))
        s.pcg_max_iter = int(getattr(settings, "pcgMaxIter", 20000))
        s.device = int(getattr(settings, "device", 0))
        s.newton_predictor = int(bool(getattr(settings, "newtonPredictor", True)))
        s.max_blocks = int(getattr(settings, "maxBlocksPerKernel", 0))
        s.newton_safeguard = int(bool(getattr(settings, "newtonSafeguard", False)))
        tl = getattr(settings, "twoLevelPreconditioner", "auto")
        s.two_level = 2 if (isinstance(tl, str) and tl == "auto") else int(bool(tl))
        ls = getattr(settings, "linearSolver", "pcg")
        if ls not in ("pcg", "minres"):
            raise ValueError(f"linearSolver must be 'pcg' or 'minres', not {ls!r}")
        s.linear_solver = 1 if ls == "minres" else 0
        pj = getattr(settings, "pressureJacobian", "reference")
        if pj not in ("reference", "exact"):
            raise ValueError(f"pressureJacobian must be 'reference' or 'exact', not {pj!r}")
        s.pressure_jac_exact = 1 if pj == "exact" else 0
        self._settings_c = s
        h = C.c_void_p()
        _lib.check(L.sors_create(_p(X, C.c_double), X.shape[0], _p(T, C.c_int32), ne, self.NV, _p(rho, C.c_double),
                                 _p(E, C.c_double), _p(nu, C.c_double), C.byref(s), C.byref(h)))
        self._h = h
        self.numVertices = X.shape[0]
        self.numElements = ne
        self.ndof = 3 * X.shape[0]

    @classmethod
    def from_arrays(cls, undeformedVertices, eleIdx, settings, gravAcceleration, dampingAlpha=0.0, *, density,
                    youngsModulus, poissonsRatio, neumannBCmask=None, neumannBCvalue=None, forceTypesList=(),
                    forceParameterList=None, muscleGroup=None, softconStiffness=None, softconDirection=None,
                    energy="neohookean"):
        """Neo-Hookean mesh from per-element arrays instead of one Params per element.

        Same system as the reference-style constructor; meant for meshes with
        millions of elements where building Python Params objects dominates set-up."""
        obj = cls.__new__(cls)
        if energy not in ("neohookean", "stableneohookean"):
            raise NotImplementedError(f"element energy {energy} is not built on the GPU path")
        obj._init_arrays(undeformedVertices, eleIdx, settings, gravAcceleration, dampingAlpha, density,
                         youngsModulus, poissonsRatio, 2 if energy == "stableneohookean" else 0)
        if muscleGroup is not None:
            obj.set_muscles(muscleGroup, softconStiffness, softconDirection)
        ctypes_, cp = [], Params()
        if neumannBCmask is not None:
            ctypes_ = ["neumannBC"]
            cp.set_param("neumannBCmask", np.asarray(neumannBCmask, dtype=np.float64).ravel())
            cp.set_param("neumannBCvalue", np.asarray(neumannBCvalue, dtype=np.float64).ravel())
        obj._setup_constraints_forces(ctypes_, cp, forceTypesList, forceParameterList)
        return obj

    def set_muscles(self, muscleGroup, softconStiffness, softconDirection, n_groups=None):
        """SoftCon fibre terms per element (group -1 = none); activations via act["softconMuscle"]."""
        L = _lib.load()
        g = np.ascontiguousarray(np.asarray(muscleGroup).ravel().astype(np.int32))
        k = np.ascontiguousarray(np.broadcast_to(np.asarray(softconStiffness, np.float64), g.shape))
        d = np.ascontiguousarray(np.broadcast_to(np.asarray(softconDirection, np.float64).reshape(-1, 3), (g.size, 3)))
        if g.size != self.numElements:
            raise ValueError("one muscle group per element is required")
        self._n_mgroups = int(n_groups if n_groups is not None else max(int(g.max()) + 1, 1))
        _lib.check(L.sors_set_muscles(self._h, _p(g, C.c_int32), _p(k, C.c_double), _p(d, C.c_double),
                                      self._n_mgroups))

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            try:
                _lib.load().sors_destroy(h)
            except Exception:
                pass
            self._h = None

    # -- actuation (Params), cpp/src/energy.cpp:233-240, :284-291 -------------
    def _apply_actuation(self, act):
        if act is None:
            return
        L = _lib.load()
        if "pressure" in self._forces and act.has("pressure"):
            p = np.ascontiguousarray(act.get_value("pressure").T.ravel())
            _lib.check(L.sors_set_actuation(self._h, b"pressure", _p(p, C.c_double), p.size))
        if getattr(self, "_n_mgroups", 0) and act.has("softconMuscle"):
            a = np.ascontiguousarray(np.asarray(act.get_value("softconMuscle"), np.float64).ravel())
            _lib.check(L.sors_set_actuation(self._h, b"softconMuscle", _p(a, C.c_double), a.size))
        if "vertexForce" in self._forces and act.has("vertexForce"):
            v = np.ascontiguousarray(act.get_value("vertexForce").ravel())  # (N,3) row-major = transpose().reshaped()
            _lib.check(L.sors_set_actuation(self._h, b"vertexForce", _p(v, C.c_double), v.size))

    def _q(self, q):
        q = np.ascontiguousarray(np.asarray(q, dtype=np.float64).ravel())
        if q.size != self.ndof:
            raise ValueError(f"expected {self.ndof} DOFs, got {q.size}")
        return q

    # -- Energy<3,E> methods -------------------------------------------------
    def compute_energy(self, q, dt, act=None):
        self._apply_actuation(act)
        q = self._q(q); out = C.c_double()
        _lib.check(_lib.load().sors_energy(self._h, _p(q, C.c_double), float(dt), C.byref(out)))
        return out.value

    def compute_gradient(self, q, dt, act=None):
        self._apply_actuation(act)
        q = self._q(q); g = np.empty(self.ndof)
        _lib.check(_lib.load().sors_gradient(self._h, _p(q, C.c_double), float(dt), _p(g, C.c_double)))
        return g

    def compute_hessian_bsr(self, q, dt, act=None):
        """(row_ptr, col, blocks[nnzb,3,3]) of the assembled Hessian."""
        self._apply_actuation(act)
        L = _lib.load()
        q = self._q(q)
        nnzb = C.c_int64()
        _lib.check(L.sors_hessian_bsr(self._h, None, 0.0, None, None, None, C.byref(nnzb)))
        rp = np.empty(self.numVertices + 1, np.int32); col = np.empty(nnzb.value, np.int32)
        val = np.empty(nnzb.value * 9)
        _lib.check(L.sors_hessian_bsr(self._h, _p(q, C.c_double), float(dt), _p(rp, C.c_int32), _p(col, C.c_int32),
                                      _p(val, C.c_double), C.byref(nnzb)))
        return rp, col, val.reshape(-1, 3, 3)

    def compute_hessian(self, q, dt, act=None):
        """Energy::compute_hessian as a scipy.sparse CSR matrix."""
        import scipy.sparse as sp
        rp, col, blocks = self.compute_hessian_bsr(q, dt, act)
        return sp.bsr_matrix((blocks, col, rp), shape=(self.ndof, self.ndof)).tocsr()

    def compute_element_data(self, q, project=None):
        """Per-element (Psi V, grad V, hess V) from the same device code as the assembly."""
        q = self._q(q)
        n = 3 * self.NV
        psi = np.empty(self.numElements); g = np.empty((self.numElements, n)); H = np.empty((self.numElements, n, n))
        proj = int(self._settings_c.project_spd == 1) if project is None else int(bool(project))
        _lib.check(_lib.load().sors_elem_eval(self._h, _p(q, C.c_double), proj, _p(psi, C.c_double),
                                              _p(g, C.c_double), _p(H, C.c_double)))
        return psi, g, H

    def update_state(self, q, dt):
        q = self._q(q)
        _lib.check(_lib.load().sors_update_state(self._h, _p(q, C.c_double), float(dt)))

    def set_initial_velocity(self, velocities):
        v = np.ascontiguousarray(np.asarray(velocities, dtype=np.float64).ravel())
        _lib.check(_lib.load().sors_set_initial_velocity(self._h, _p(v, C.c_double)))

    def set_initial_deformation(self, vertices):
        v = np.ascontiguousarray(np.asarray(vertices, dtype=np.float64).ravel())
        _lib.check(_lib.load().sors_set_initial_deformation(self._h, _p(v, C.c_double)))

    def get_qPrev(self):
        q = np.empty(self.ndof)
        _lib.check(_lib.load().sors_get_state(self._h, _p(q, C.c_double), None))
        return q

    def get_vPrev(self):
        v = np.empty(self.ndof)
        _lib.check(_lib.load().sors_get_state(self._h, None, _p(v, C.c_double)))
        return v

    def device_bytes(self):
        return int(_lib.load().sors_device_bytes(self._h))

    def active_contacts(self):
        """Contact constraints active in the last SQP step."""
        return int(_lib.load().sors_active_contacts(self._h))

    def held_pairs(self):
        """Indices of the maxDistance pairs held at their bound by the last SQP step."""
        L = _lib.load()
        k = int(L.sors_held_pairs(self._h, None, None, 0))
        out = np.zeros(max(k, 1), np.int32)
        L.sors_held_pairs(self._h, _p(out, C.c_int32), None, k)
        return out[:k]

    def handle(self):
        return self._h


class EnergyTet(_EnergyBase):
    NV = 4
    MESH = "Tetrahedron"


class EnergyHex(_EnergyBase):
    NV = 8
    MESH = "Hexahedron"


class DiskContact:
    """Handle on an Energy's diskContact constraint (cpp/py_sors.cpp:230-245)."""

    def __init__(self, energy):
        self._energy = energy

    def set_disk(self, center, normal, radius, diskIdx=0):
        c = np.ascontiguousarray(np.asarray(center, np.float64).ravel())
        n = np.ascontiguousarray(np.asarray(normal, np.float64).ravel())
        _lib.check(_lib.load().sors_set_disk(self._energy._h, int(diskIdx), _p(c, C.c_double), _p(n, C.c_double),
                                             float(radius)))


def get_disk_contact_constraint(energy, idx):
    """cpp/py_sors.cpp:248-261: the diskContact constraint at index idx of constraintTypesList."""
    cons = getattr(energy, "_constraints", [])
    if idx < 0 or idx >= len(cons):
        raise IndexError("constraint index out of range")
    if cons[idx] != "diskContact":
        raise ValueError("constraint at index is not DiskContact")
    return DiskContact(energy)


def Energy(undeformedVertices, eleIdx, settings, gravAcceleration, dampingAlpha=0.0, elementEnergiesList=None,
           elementParameterList=None, constraintTypesList=(), constraintParameterList=None, forceTypesList=(),
           forceParameterList=None):
    """Factory by settings.meshType (cpp/py_sors.cpp:30-62)."""
    args = (undeformedVertices, eleIdx, settings, gravAcceleration, dampingAlpha, elementEnergiesList,
            elementParameterList, constraintTypesList, constraintParameterList, forceTypesList, forceParameterList)
    if settings.meshType == "Tetrahedron":
        return EnergyTet(*args)
    if settings.meshType == "Hexahedron":
        return EnergyHex(*args)
    raise RuntimeError("Unknown mesh type: " + str(settings.meshType))


class _SolverBase:
    ENERGY = _EnergyBase

    def __init__(self, settings=None):
        self.settings = settings
        self.last_stats = None

    def step(self, solution, systemEnergy, act=None, dt=0.0, substeps=0, out=None):
        """Solver<3,E>::step (cpp/src/solver.cpp:5-52): returns the new solution.

        `out` (optional, 3N float64, e.g. pinned host memory) receives the result."""
        if isinstance(act, (int, float)) and not isinstance(act, bool):
            # step(solution, systemEnergy, dt, substeps) overload (cpp/py_sors.cpp:124-130)
            act, dt, substeps = None, float(act), int(dt) if dt else 0
        if not isinstance(systemEnergy, self.ENERGY):
            raise TypeError("systemEnergy does not match the solver's mesh type")
        systemEnergy._apply_actuation(act)
        q = systemEnergy._q(solution)
        if out is None:
            out = np.empty_like(q)
        elif out.dtype != np.float64 or out.size != q.size or not out.flags.c_contiguous:
            raise ValueError("out must be a contiguous float64 array of 3N entries")
        st = _lib.SorsStepStats()
        _lib.check(_lib.load().sors_step(systemEnergy._h, _p(q, C.c_double), _p(out, C.c_double), float(dt),
                                         int(substeps), C.byref(st)))
        self.last_stats = st
        return out

    def step_device(self, q_device_ptr, systemEnergy, act=None, dt=0.0, substeps=0):
        """Step a device-resident FP64 solution (pointer, e.g. torch tensor.data_ptr()) in place."""
        systemEnergy._apply_actuation(act)
        st = _lib.SorsStepStats()
        _lib.check(_lib.load().sors_step_device(systemEnergy._h, C.c_void_p(int(q_device_ptr)), float(dt),
                                                int(substeps), C.byref(st)))
        self.last_stats = st
        return st


class SolverTet(_SolverBase):
    ENERGY = EnergyTet


class SolverHex(_SolverBase):
    ENERGY = EnergyHex


def Solver(settings):
    """Factory by settings.meshType (cpp/py_sors.cpp:99-111)."""
    if settings.meshType == "Tetrahedron":
        return SolverTet(settings)
    if settings.meshType == "Hexahedron":
        return SolverHex(settings)
    raise RuntimeError("Unknown mesh type: " + str(settings.meshType))


class IO:
    """Mesh utilities of IO (cpp/py_sors.cpp:180-198) that the FEM set-up uses."""

    @staticmethod
    def extract_tet_surfaces(vertices, eleIdx, verboseFlag=False):
        return _meshes.extract_surfaces(np.asarray(vertices, float), np.asarray(eleIdx))

    @staticmethod
    def extract_hex_surfaces(vertices, eleIdx, verboseFlag=False):
        return _meshes.extract_surfaces(np.asarray(vertices, float), np.asarray(eleIdx))

    @staticmethod
    def read_tet_MSH(filename, verboseFlag=False):
        """IO::read_tet_MSH (cpp/src/io.cpp:380-471): (vertices (N,3), tets (E,4)), MSH 4.1 / 2.2."""
        from . import msh
        return msh.read_tet_msh(filename)

    @staticmethod
    def read_hex_MSH(filename, verboseFlag=False):
        """IO::read_hex_MSH (cpp/src/io.cpp:473-569): (vertices (N,3), hexes (E,8))."""
        from . import msh
        return msh.read_hex_msh(filename)

    @staticmethod
    def hex_to_5_tets(hexElements):
        """cpp/src/io.cpp:899-929."""
        h = np.asarray(hexElements, dtype=np.int32)
        if h.shape[0] == 0 or h.shape[1] != 8:
            return np.zeros((0, 4), np.int32)
        idx = np.array([[0, 1, 3, 4], [1, 2, 3, 6], [1, 4, 5, 6], [3, 4, 6, 7], [1, 3, 4, 6]])
        return h[:, idx].reshape(-1, 4)
