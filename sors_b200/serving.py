"""Rollout serving: many independent rollouts resident on one GPU.

Requests (a mesh, its material, boundary conditions and a number of steps)
arrive at any time.  The server admits work when a slot is free and its
estimated device footprint fits the memory budget (continuous admission).

Batching: compatible small requests waiting at admission time (same element
type, step count, dt, scheme, precision, gravity and planes; at most
`batch_small` elements each) are packed into one union mesh, up to
`batch_max` requests and `batch_elems` elements: one library
handle whose nodes and elements are the concatenation of theirs.  The meshes
share no element, so the union's gradient, Hessian and contact constraints are
the direct sum of theirs; one Newton / SQP iteration, one PCG kernel sequence
and one captured CUDA graph per chunk then serve all of them at once (each
kernel launch does the work of the whole batch).  Each rollout keeps its own
disk indenter (an independent disk contact group).  Results are sliced back
per request; they equal the rollout run alone up to the solver tolerances
(the union's Newton / SQP iterations continue until every member has
converged, and its dot products are summed in a different order).

Inside a union every linear solve runs one preconditioned CG per member
(sors_set_members): the members share each kernel launch but keep their own
step lengths, tolerances and convergence, so a union's solves take as many
iterations as its slowest member alone, not those of the joined system.

Every admitted batch keeps its union mesh, state and Hessian pattern resident
in its own handle (one CUDA stream) and is stepped by a worker thread, so the
batches overlap on the device.  Per-step and per-rollout latencies are
recorded per request.  The library calls release the GIL (ctypes).
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
    batch: int = 1            # requests stepped together in one union handle


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
    b += (3 * 4 + 4 * 2) * n_nodes * hs + 9 * n_nodes * hs   # PCG vectors (p padded) + block-Jacobi
    b += 9 * nnzb * hs                     # Hessian values
    b += 4 * nnzb * 2 + 4 * n_nodes * 4    # pattern + slot pointers
    b += 4 * n_elems * nv * 2 + 2 * n_elems * nv * nv + 16 * n_elems  # conn, pairs, slot items, materials
    if nv == 4:
        # element-owner assembly: tet shapes, node chunks (chunk element lists
        # hold each element ~1.5 times with its owned-vertex slots) and items
        b += 80 * n_elems + 4 * n_nodes + int(1.5 * n_elems) * 12 + 2 * n_elems * nv * nv
    return int(b * 1.1) + (1 << 20)


class RolloutServer:
    """Continuous-admission server for independent rollouts on one GPU."""

    def __init__(self, max_slots: int = 8, memory_budget_bytes: int | None = None, device: int = 0,
                 batch_max: int = 1, batch_elems: int = 400_000, batch_small: int = 50_000,
                 max_blocks: int | None = None):
        import torch
        self.device = device
        # kernels of concurrent handles share the GPU: cap each grid so that
        # several run side by side (0 = the whole GPU, used for one slot)
        self.max_blocks = (max(148, 2 * 1184 // max_slots) if max_slots > 1 else 0) if max_blocks is None \
            else int(max_blocks)
        self.batch_max = max(1, int(batch_max))
        self.batch_elems = int(batch_elems)
        # only meshes up to batch_small elements are packed: larger ones already
        # fill the GPU alone, and a union's iterations are those of its hardest member
        self.batch_small = int(batch_small)
        self._held: list[RolloutRequest] = []
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
    def _next(self, block: bool):
        if self._held:
            return self._held.pop(0)
        try:
            return self._pending.get(block=block)
        except queue.Empty:
            return False

    def _dispatch(self):
        closing = False
        while True:
            if closing:
                if not self._held:
                    return
                req = self._held.pop(0)
            else:
                req = self._next(block=True)
            if req is None:
                closing = True
                continue
            batch = [req]
            if self.batch_max > 1 and req.elements.shape[0] <= self.batch_small:
                # pack compatible requests that are waiting now (no waiting for new arrivals)
                rest = []
                while len(batch) < self.batch_max:
                    nxt = self._held.pop(0) if (closing and self._held) else (False if closing else self._next(False))
                    if nxt is False:
                        break
                    if nxt is None:
                        closing = True
                        break
                    if (compatible(batch[0], nxt) and nxt.elements.shape[0] <= self.batch_small and
                            sum(r.elements.shape[0] for r in batch) + nxt.elements.shape[0] <= self.batch_elems):
                        batch.append(nxt)
                    else:
                        rest.append(nxt)
                self._held = rest + self._held
            need = sum(estimate_device_bytes(r.vertices.shape[0], r.elements.shape[0], r.elements.shape[1],
                                             r.precision) for r in batch)
            if need > self.budget:
                for r in batch:
                    self._results.append(RolloutResult(r.tag, None, [], 0.0, 0.0, 0, 0,
                                                       error=f"rollout needs ~{need} bytes, budget is {self.budget}"))
                continue
            with self._lock:
                while self._active >= self.max_slots or self._in_use + need > self.budget:
                    self._lock.wait()
                self._active += 1
                self._in_use += need
            t = threading.Thread(target=self._run, args=(batch, need), daemon=True)
            self._threads.append(t)
            t.start()

    def _run(self, batch, need: int):
        import torch
        torch.cuda.set_device(self.device)
        self._run_batch(batch, time.perf_counter())
        with self._lock:
            self._active -= 1
            self._in_use -= need
            self._lock.notify_all()

    def _run_batch(self, batch, started):
        """Steps one union; if it fails and holds several rollouts, each is run
        again on its own so that one failing rollout does not fail the others."""
        steps_lat = []
        newton = pcg = 0
        finals = [None] * len(batch)
        err = None
        en = sol = None
        try:
            en, sol, slices, disks = build_union(batch, self.device, self.max_blocks)
            ref = batch[0]
            q = np.concatenate([np.ascontiguousarray(r.vertices, dtype=np.float64).ravel() for r in batch])
            for t in range(ref.steps):
                t0 = time.perf_counter()
                for d, (c0, nrm, rad, vel) in enumerate(disks):
                    _lib_set_disk(en, d, c0 + vel * ref.dt * t, nrm, rad)
                q = sol.step(q, en)
                steps_lat.append(time.perf_counter() - t0)
                newton += sol.last_stats.newton_iters
                pcg += sol.last_stats.pcg_iters
            finals = [q[a:b].copy() for a, b in slices]
            del en
        except Exception as ex:  # reported per rollout, the server keeps running
            err = str(ex)
            if en is not None:
                err += curvature_note(en)
        en = sol = None  # release the union's device memory before any re-run
        if err is not None and len(batch) > 1:
            for r in batch:
                self._run_batch([r], started)
            return
        done = time.perf_counter()
        for r, f in zip(batch, finals):
            self._results.append(RolloutResult(r.tag, f, list(steps_lat), started - r.submitted, done - r.submitted,
                                               newton, pcg, err, batch=len(batch)))


def curvature_note(en) -> str:
    """' (exact Hessian indefinite: ...)' when the last step's PCG met
    non-positive curvature, else ''.  A Rayleigh quotient below -0.1 (OSQP's
    default step size on contact rows, plus sigma) means the reference's OSQP
    set-up would reject that step's QP as non-convex."""
    import ctypes as C
    from . import _lib
    rq = C.c_double(); n = C.c_int32()
    if _lib.load().sors_last_step_curvature(en._h, C.byref(rq), C.byref(n)) != 0 or n.value == 0:
        return ""
    return f" (exact Hessian indefinite in {n.value} solves of the step, min p'Hp/p'p = {rq.value:.3e})"


def compatible(a: RolloutRequest, b: RolloutRequest) -> bool:
    """Requests that can share one union handle."""
    def planes_key(r):
        return None if r.planes is None else (np.asarray(r.planes[0], float).tobytes(),
                                              np.asarray(r.planes[1], float).tobytes())
    return (a.elements.shape[1] == b.elements.shape[1] and a.steps == b.steps and a.dt == b.dt and
            a.scheme == b.scheme and a.precision == b.precision and tuple(a.gravity) == tuple(b.gravity) and
            planes_key(a) == planes_key(b) and (a.disks is None) == (b.disks is None) and
            (a.neumann_mask is None) == (b.neumann_mask is None) and a.newton_res_tol == b.newton_res_tol)


def _lib_set_disk(en, d, c, n, r):
    import ctypes as C
    from . import _lib
    c = np.ascontiguousarray(c, dtype=np.float64); n = np.ascontiguousarray(n, dtype=np.float64)
    _lib.check(_lib.load().sors_set_disk(en._h, int(d), c.ctypes.data_as(C.POINTER(C.c_double)),
                                         n.ctypes.data_as(C.POINTER(C.c_double)), float(r)))


def build_union(batch, device: int = 0, max_blocks: int = 0):
    """One Energy/Solver over the union of the batch's meshes.

    Returns (energy, solver, slices, disks): slices[k] = (a, b) DOF range of
    request k; disks: (center0, normal, radius, velocity) per disk, in the
    order of the handle's disk contact groups."""
    import ctypes as C
    from . import _lib
    if len(batch) == 1 and batch[0].disks is None:
        en, sol = build_rollout(batch[0], device, max_blocks=max_blocks)
        return en, sol, [(0, batch[0].vertices.size)], []
    ref = batch[0]
    offs = np.cumsum([0] + [r.vertices.shape[0] for r in batch])
    X = np.concatenate([np.asarray(r.vertices, float) for r in batch])
    T = np.concatenate([np.asarray(r.elements, np.int32) + offs[k] for k, r in enumerate(batch)])
    bc = lambda v, r: np.broadcast_to(np.asarray(v, float), (r.elements.shape[0],))
    rho = np.concatenate([bc(r.density, r) for r in batch])
    E = np.concatenate([bc(r.youngs, r) for r in batch])
    nu = np.concatenate([bc(r.poisson, r) for r in batch])
    mask = val = None
    if ref.neumann_mask is not None:
        mask = np.concatenate([np.asarray(r.neumann_mask).ravel() for r in batch])
        val = np.concatenate([np.asarray(r.neumann_value, float).ravel() for r in batch])
    surf = None
    if ref.surface is not None:
        surf = np.concatenate([np.asarray(r.surface) + offs[k] for k, r in enumerate(batch)])
    union = RolloutRequest(X, T, rho, E, nu, ref.steps, ref.dt, gravity=ref.gravity, neumann_mask=mask,
                           neumann_value=val, precision=ref.precision, scheme=ref.scheme,
                           newton_res_tol=ref.newton_res_tol, planes=ref.planes, disks=None, surface=surf)
    # the meshes of a union overlap in space: aggregates would mix them, so the
    # union runs block Jacobi (its members are small)
    en, sol = build_rollout(union, device, sqp=ref.planes is not None or ref.disks is not None,
                            max_blocks=max_blocks, two_level=len(batch) == 1 and "auto")
    disks = []
    if ref.disks is not None:
        cen, nrm, rad, ptr, dsurf = [], [], [], [0], []
        for k, r in enumerate(batch):
            c0 = np.asarray(r.disks[0], float).reshape(-1, 3)
            nn = np.asarray(r.disks[1], float).reshape(-1, 3)
            rr = np.asarray(r.disks[2], float).ravel()
            vel = (np.zeros_like(c0) if r.disk_velocity is None
                   else np.asarray(r.disk_velocity, float).reshape(-1, 3))
            s_k = np.asarray(r.surface, np.int32) + offs[k]
            for d in range(c0.shape[0]):
                cen.append(c0[d]); nrm.append(nn[d]); rad.append(rr[d])
                dsurf.append(s_k); ptr.append(ptr[-1] + s_k.size)
                disks.append((c0[d], nn[d], rr[d], vel[d]))
        cen = np.ascontiguousarray(cen, dtype=np.float64); nrm = np.ascontiguousarray(nrm, dtype=np.float64)
        rad = np.ascontiguousarray(rad, dtype=np.float64)
        dsurf = np.ascontiguousarray(np.concatenate(dsurf), dtype=np.int32)
        ptr = np.ascontiguousarray(ptr, np.int32)
        dp = lambda a: a.ctypes.data_as(C.POINTER(C.c_double))
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int32))
        _lib.check(_lib.load().sors_set_disk_contact_groups(en._h, dp(cen), dp(nrm), dp(rad), len(disks), ip(dsurf),
                                                            ip(ptr)))
        en._constraints = list(en._constraints) + ["diskContact"]
    if len(batch) > 1:
        # one PCG per member inside the shared launches (batched.cu)
        node_offsets = np.ascontiguousarray(offs, dtype=np.int32)
        _lib.check(_lib.load().sors_set_members(en._h, node_offsets.ctypes.data_as(C.POINTER(C.c_int32)),
                                                len(batch)))
    slices = [(3 * offs[k], 3 * offs[k + 1]) for k in range(len(batch))]
    return en, sol, slices, disks


def build_rollout(req: RolloutRequest, device: int = 0, sqp: bool | None = None, max_blocks: int = 0,
                  two_level="auto"):
    """Energy and Solver for one request (the reference-style py_sors objects)."""
    s = ps.SimulationSettings()
    s.meshType = "Tetrahedron" if req.elements.shape[1] == 4 else "Hexahedron"
    s.dt = req.dt
    s.timeSteppingScheme = req.scheme
    contact = (req.planes is not None or req.disks is not None) if sqp is None else sqp
    s.solverMethod = "minimize_SQP" if contact else "minimize_newton"
    s.precision = req.precision
    s.newtonResidualTol = 0.0 if contact else req.newton_res_tol
    s.device = device
    s.maxBlocksPerKernel = max_blocks
    s.twoLevelPreconditioner = two_level
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
        if req.surface is not None:
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
