"""Rollout serving: many independent rollouts resident on one GPU.

Requests (a mesh, its material, boundary conditions and a number of steps)
arrive at any time.  The server admits a request when a slot is free and its
estimated device footprint fits the memory budget; every admitted rollout
keeps its mesh, state and Hessian pattern resident in its own library handle
(one CUDA stream each) and is stepped by a worker thread, so the steps of
different rollouts overlap on the device.  When a rollout finishes its slot
and memory are released and the next waiting request is admitted at once
(continuous admission).  Per-step and per-rollout latencies are recorded.

The library calls release the GIL (ctypes), so worker threads really run
their steps concurrently.
"""
from __future__ import annotations

import queue
import threading
import time
from dataclasses import dataclass, field

import numpy as np

from . import py_sors as ps


@dataclass
class RolloutRequest:
    """One rollout: a tet (4) or hex (8) Neo-Hookean mesh stepped `steps` times."""
    vertices: np.ndarray
    elements: np.ndarray
    density: object
    youngs: object
    poisson: object
    steps: int
    dt: float
    gravity: tuple = (0.0, 0.0, -9.81)
    neumann_mask: np.ndarray | None = None
    neumann_value: np.ndarray | None = None
    precision: str = "mixed"
    scheme: str = "backward_euler"
    newton_res_tol: float = 1e-8
    tag: object = None
    submitted: float = field(default=0.0)
    # contact (minimize_SQP): planes (points, normals), disks (centers, normals,
    # radii) moving at disk_velocity (m/s, per disk) and the candidate surface vertices
    planes: tuple | None = None
    disks: tuple | None = None
    disk_velocity: np.ndarray | None = None
    surface: np.ndarray | None = None


@dataclass
class RolloutResult:
    tag: object
    final: np.ndarray | None
    step_latencies: list
    queue_wait: float
    latency: float            # submit -> done
    newton_iters: int
    pcg_iters: int
    error: str | None = None


def estimate_device_bytes(n_nodes: int, n_elems: int, nodes_per_elem: int, precision: str) -> int:
    """Footprint of one handle before creating it (pattern + vectors + Hessian).

    Block-CSR blocks are estimated from the element count (each element adds
    its vertex pairs, shared across neighbours): tets ~ 2.6 blocks per
    element, hexes ~ 3.5; the estimate is conservative by ~10 %.
    """
    hs = 4 if precision == "mixed" else 8
    nv = nodes_per_elem
    nnzb = int((2.7 if nv == 4 else 3.6) * n_elems + n_nodes)
    b = 0
    b += 8 * 3 * n_nodes * 12             # FP64 state vectors
    b += 3 * n_nodes * hs * 6 + 9 * n_nodes * hs   # PCG vectors + block-Jacobi
    b += 9 * nnzb * hs                     # Hessian values
    b += 4 * nnzb * 2 + 4 * n_nodes * 4    # pattern + slot pointers
    b += 4 * n_elems * nv * 2 + 2 * n_elems * nv * nv + 16 * n_elems  # conn, pairs, slot items, materials
    return int(b * 1.1) + (1 << 20)


class RolloutServer:
    """Continuous-admission server for independent rollouts on one GPU."""

    def __init__(self, max_slots: int = 8, memory_budget_bytes: int | None = None, device: int = 0):
        import torch
        self.device = device
        if memory_budget_bytes is None:
            free, _total = torch.cuda.mem_get_info(device)
            memory_budget_bytes = int(free * 0.8)
        self.budget = memory_budget_bytes
        self.max_slots = max_slots
        self._in_use = 0
        self._active = 0
        self._lock = threading.Condition()
        self._pending: "queue.Queue[RolloutRequest | None]" = queue.Queue()
        self._results: list[RolloutResult] = []
        self._threads: list[threading.Thread] = []
        self._closed = False
        self._dispatcher = threading.Thread(target=self._dispatch, daemon=True)
        self._dispatcher.start()

    # -- public -------------------------------------------------------------
    def submit(self, req: RolloutRequest) -> None:
        if self._closed:
            raise RuntimeError("server is closed")
        req.submitted = time.perf_counter()
        self._pending.put(req)

    def close(self, wait: bool = True) -> list[RolloutResult]:
        self._closed = True
        self._pending.put(None)
        if wait:
            self._dispatcher.join()
            for t in list(self._threads):
                t.join()
        return list(self._results)

    def results(self) -> list[RolloutResult]:
        return list(self._results)

    # -- internals ----------------------------------------------------------
    def _dispatch(self):
        while True:
            req = self._pending.get()
            if req is None:
                return
            need = estimate_device_bytes(req.vertices.shape[0], req.elements.shape[0], req.elements.shape[1],
                                         req.precision)
            if need > self.budget:
                self._results.append(RolloutResult(req.tag, None, [], 0.0, 0.0, 0, 0,
                                                   error=f"rollout needs ~{need} bytes, budget is {self.budget}"))
                continue
            with self._lock:
                while self._active >= self.max_slots or self._in_use + need > self.budget:
                    self._lock.wait()
                self._active += 1
                self._in_use += need
            t = threading.Thread(target=self._run, args=(req, need), daemon=True)
            self._threads.append(t)
            t.start()

    def _run(self, req: RolloutRequest, need: int):
        import torch
        torch.cuda.set_device(self.device)
        started = time.perf_counter()
        steps_lat = []
        newton = pcg = 0
        final = None
        err = None
        try:
            en, sol = build_rollout(req, self.device)
            disk = None
            if req.disks is not None:
                disk = ps.get_disk_contact_constraint(en, en._constraints.index("diskContact"))
                c0 = np.asarray(req.disks[0], float).reshape(-1, 3)
                nrm = np.asarray(req.disks[1], float).reshape(-1, 3)
                rad = np.asarray(req.disks[2], float).ravel()
                vel = np.zeros_like(c0) if req.disk_velocity is None else np.asarray(req.disk_velocity,
                                                                                       float).reshape(-1, 3)
            q = np.ascontiguousarray(req.vertices, dtype=np.float64).ravel().copy()
            for t in range(req.steps):
                t0 = time.perf_counter()
                if disk is not None:
                    for d in range(c0.shape[0]):
                        disk.set_disk(c0[d] + vel[d] * req.dt * t, nrm[d], rad[d], d)
                q = sol.step(q, en)
                steps_lat.append(time.perf_counter() - t0)
                newton += sol.last_stats.newton_iters
                pcg += sol.last_stats.pcg_iters
            final = q
            del en
        except Exception as ex:  # reported per rollout, the server keeps running
            err = str(ex)
        done = time.perf_counter()
        self._results.append(RolloutResult(req.tag, final, steps_lat, started - req.submitted, done - req.submitted,
                                           newton, pcg, err))
        with self._lock:
            self._active -= 1
            self._in_use -= need
            self._lock.notify_all()


def build_rollout(req: RolloutRequest, device: int = 0):
    """Energy and Solver for one request (the reference-style py_sors objects)."""
    s = ps.SimulationSettings()
    s.meshType = "Tetrahedron" if req.elements.shape[1] == 4 else "Hexahedron"
    s.dt = req.dt
    s.timeSteppingScheme = req.scheme
    contact = req.planes is not None or req.disks is not None
    s.solverMethod = "minimize_SQP" if contact else "minimize_newton"
    s.precision = req.precision
    s.newtonResidualTol = 0.0 if contact else req.newton_res_tol
    s.device = device
    cls = ps.EnergyTet if req.elements.shape[1] == 4 else ps.EnergyHex
    en = cls.from_arrays(req.vertices, req.elements, s, np.asarray(req.gravity, float), 0.0,
                         density=req.density, youngsModulus=req.youngs, poissonsRatio=req.poisson,
                         neumannBCmask=req.neumann_mask, neumannBCvalue=req.neumann_value)
    if contact:
        types, cp = [], ps.Params()
        if req.neumann_mask is not None:
            types.append("neumannBC")
            cp.set_param("neumannBCmask", np.asarray(req.neumann_mask, float).ravel())
            cp.set_param("neumannBCvalue", np.asarray(req.neumann_value, float).ravel())
        if req.planes is not None:
            types.append("planeContact")
            cp.set_param("positionVectorListPlanes", np.asarray(req.planes[0], float).ravel())
            cp.set_param("normalVectorListPlanes", np.asarray(req.planes[1], float).ravel())
        if req.disks is not None:
            types.append("diskContact")
            cp.set_param("diskCenterVectorList", np.asarray(req.disks[0], float).ravel())
            cp.set_param("diskNormalVectorList", np.asarray(req.disks[1], float).ravel())
            cp.set_param("diskRadiusList", np.asarray(req.disks[2], float).ravel())
        cp.set_param("surfaceVerticesIdx", np.asarray(req.surface, float).ravel())
        en._setup_constraints_forces(types, cp, (), None)
    return en, ps.Solver(s)


def percentile(values, p):
    if not values:
        return float("nan")
    return float(np.percentile(np.asarray(values, float), p))


def cube_surface_nodes(n_cells: int) -> np.ndarray:
    """Boundary node ids of an n^3-cell grid (vid = i + NX (j + NY k))."""
    n1 = n_cells + 1
    k, j, i = np.meshgrid(np.arange(n1), np.arange(n1), np.arange(n1), indexing="ij")
    on = (i == 0) | (i == n_cells) | (j == 0) | (j == n_cells) | (k == 0) | (k == n_cells)
    return np.nonzero(on.ravel())[0].astype(np.int32)


def poke_cube_request(rng: np.random.Generator, n_cells: int, tag=None, steps: int = 100, dt: float = 1e-2,
                      precision: str = "mixed") -> RolloutRequest:
    """A poke rollout: a 6-tet cube (side U[30, 60] mm, n_cells^3 cells) resting on
    the ground plane z = 0 under gravity, pressed by a rigid disk (radius 10 mm,
    normal -z) that starts 1 mm above the top face at a seeded (x, y) offset and
    moves 10 mm down over the rollout (the PokeFlex set-up, planeContact +
    diskContact with minimize_SQP)."""
    from . import meshes
    side = float(rng.uniform(0.03, 0.06))
    X = meshes.grid_nodes(n_cells, n_cells, n_cells, (side, side, side))
    T = meshes.kuhn_tet_elements(n_cells, n_cells, n_cells)
    E = float(rng.uniform(2e4, 2e5))
    nu = float(rng.uniform(0.30, 0.48))
    cx, cy = rng.uniform(0.3 * side, 0.7 * side, size=2)
    travel = 0.01
    vz = -travel / (steps * dt)
    return RolloutRequest(X, T, 1000.0, E, nu, steps, dt, gravity=(0.0, 0.0, -9.81), precision=precision, tag=tag,
                          planes=(np.zeros((1, 3)), np.array([[0.0, 0.0, 1.0]])),
                          disks=(np.array([[cx, cy, side + 0.001]]), np.array([[0.0, 0.0, -1.0]]), np.array([0.01])),
                          disk_velocity=np.array([[0.0, 0.0, vz]]), surface=cube_surface_nodes(n_cells))
