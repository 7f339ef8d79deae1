#!/usr/bin/env python
"""Implicit-Euler FEM step throughput on the jittered Neo-Hookean tet block.

Workload (one "step" = one backward-Euler time step, i.e. one full Newton
solve with block-Jacobi PCG linear solves, of the whole mesh):
  beam 1.0 x 0.25 x 0.25 m as a 200 x 50 x 50 cell grid, 6 tets per cell
  (3,000,000 tets, 522,801 nodes, 1,568,403 DOF); interior nodes jittered by
  seeded U(+-10% h); per-element Young's modulus log-uniform in [5e4, 5e5] Pa,
  nu = 0.45, rho = 1070; the x = 0 face clamped; gravity; dt = 5e-3 s.
  Mixed precision (FP32 Hessian, SpMV and PCG vectors; FP64 residual, energy,
  dots and log J) is the headline; the plain FP64 path is timed beside it.

value   = elements x steps / s with the state resident in HBM (Solver.step_device)
e2e     = the same through Solver.step with pinned host buffers (H2D of q and
          D2H of the result inside every timed step)
Inputs are larger than L2 (the assembled system is ~1.1 GB), so no flush.

--impl reference times the CPU restatement of the reference path (oracle/,
FP64, OpenMP element loops + sparse LDL^T Newton, all host threads) on a
bounded sample of the same workload (a 24 x 12 x 12 cell block with the same
spacing, jitter and material distribution), in the same unit.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "fem_step_throughput"
UNIT = "elem*steps/s"
SIZE = (1.0, 0.25, 0.25)
CELLS = (200, 50, 50)
SAMPLE_CELLS = (24, 12, 12)
DT = 5e-3


def workload_name(cells, precision):
    nx, ny, nz = cells
    return (f"jittered 6-tet Neo-Hookean block {nx}x{ny}x{nz} cells ({6 * nx * ny * nz:,} tets, "
            f"{(nx + 1) * (ny + 1) * (nz + 1):,} nodes), E log-uniform [5e4,5e5], nu 0.45, rho 1070, "
            f"x=0 clamped, gravity, backward Euler dt 5e-3, {precision}")


_shuffle = False


def block_mesh(cells, seed=0, shuffle=None):
    """The jittered block; with shuffle, its nodes and elements renumbered by a
    seeded random permutation (the numbering of a mesh read from a file)."""
    from sors_b200 import meshes
    nx, ny, nz = cells
    h = SIZE[0] / CELLS[0]
    X, T, E = meshes.jittered_block_tets(nx, ny, nz, (nx * h, ny * h, nz * h), jitter=0.1, seed=seed)
    if _shuffle if shuffle is None else shuffle:
        rng = np.random.default_rng(seed + 1000)
        perm = rng.permutation(X.shape[0])
        inv = np.empty_like(perm)
        inv[perm] = np.arange(perm.size)
        eperm = rng.permutation(T.shape[0])
        X = X[perm]
        T = inv[T[eperm]].astype(np.int32)
        E = E[eperm]
    mask, val = meshes.clamp_mask(X)
    return X, T, E, mask, val


PROJECTION = {"true": True, "false": False, "adaptive": "adaptive"}
_projection = "adaptive"
_two_level = True


def make_settings(precision):
    from sors_b200 import py_sors as ps
    s = ps.SimulationSettings()
    s.meshType = "Tetrahedron"
    s.dt = DT
    s.substeps = 1
    s.timeSteppingScheme = "backward_euler"
    s.solverMethod = "minimize_newton"
    s.precision = precision
    s.hessianProjection = PROJECTION[_projection]
    s.twoLevelPreconditioner = _two_level
    s.newtonResidualTol = 1e-8
    return s


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.path = os.path.join("/tmp", f"sors_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "200", "-i", str(self.gpu)], stdout=open(self.path, "w"),
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        try:
            rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        except Exception:
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1])); mx = float(r[2])
            except (ValueError, IndexError):
                continue
            for nm, v in zip(names, r[5:9]):
                if v.strip().lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        try:
            return float(json.load(open(p))["hbm_gbs"]), "measured"
        except Exception:
            pass
    return 6650.0, "fallback"


def ncu_traffic(kernel_key, units):
    """DRAM bytes per launch of a kernel from the committed ncu summary, scaled to `units`."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    try:
        d = json.load(open(p)).get(kernel_key)
        return float(d["dram_bytes_per_launch"]) * units / float(d["units"])
    except Exception:
        return None


# ---------------------------------------------------------------------------
# CPU restatement (oracle) on a bounded sample
# ---------------------------------------------------------------------------
def cpu_sample_run(steps, warmup, threads=None):
    from oracle import oracle as orc
    X, T, E, mask, val = block_mesh(SAMPLE_CELLS, seed=0, shuffle=False)
    nthreads = threads or os.cpu_count() or 1
    o = orc.System(X, T, rho=1070.0, youngs=E, nu=0.45, grav=(0, 0, -9.81), scheme="backward_euler",
                   method="minimize_newton", dt=DT, substeps=1, nthreads=nthreads)
    o.set_neumann(mask, val)
    q = X.ravel().copy()
    for _ in range(warmup):
        q, st = o.step(q)
        if st != 0:
            raise RuntimeError(f"oracle step failed ({st})")
    t0 = time.perf_counter()
    for _ in range(steps):
        q, st = o.step(q)
        if st != 0:
            raise RuntimeError(f"oracle step failed ({st})")
    dt_wall = time.perf_counter() - t0
    ne = T.shape[0]
    return {"value": ne * steps / dt_wall, "unit": UNIT, "cores": nthreads, "kind": "port",
            "sample": f"{SAMPLE_CELLS[0]}x{SAMPLE_CELLS[1]}x{SAMPLE_CELLS[2]} cells of the same block "
                      f"({ne:,} tets, same spacing/jitter/material distribution), {steps} full implicit steps "
                      f"after {warmup} warm-up, FP64 OpenMP assembly + sparse LDL^T Newton (||dx||<1e-9)",
            "ms_per_step": 1e3 * dt_wall / steps, "elements": ne}


def cpu_phases(threads=None):
    """The reference's element and assembly phases at full size, on the host
    cores: one Energy::compute_gradient (cpp/src/energy.cpp:252-308) and one
    Energy::compute_hessian with triplets -> CSR (cpp/src/energy.cpp:312-390)
    of the whole 3.0M-tet block, by the CPU restatement (FP64, OpenMP)."""
    from oracle import oracle as orc
    X, T, E, mask, val = block_mesh(CELLS, seed=0, shuffle=False)
    nthreads = threads or os.cpu_count() or 1
    o = orc.System(X, T, rho=1070.0, youngs=E, nu=0.45, grav=(0, 0, -9.81), scheme="backward_euler",
                   method="minimize_newton", dt=DT, substeps=1, nthreads=nthreads)
    o.set_neumann(mask, val)
    q = X.ravel().copy()
    t0 = time.perf_counter()
    o.gradient(q, DT)
    t1 = time.perf_counter()
    H, st = o.hessian_csr(q, DT)
    t2 = time.perf_counter()
    nnz = int(H.nnz)
    del H, o
    return {"workload": workload_name(CELLS, "FP64"), "cores": nthreads, "kind": "port",
            "gradient_s": t1 - t0, "hessian_csr_s": t2 - t1, "hessian_nnz": nnz,
            "what": "one full-size gradient assembly and one Hessian assembly (element Hessians, triplets, "
                    "triplets -> CSR with duplicate sums), FP64, all host threads"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    steps, warmup = args.steps, args.warmup
    cb = cpu_sample_run(steps, warmup)
    ne = cb["elements"]
    line = {"metric": METRIC, "value": cb["value"], "unit": UNIT, "n_gpus": world, "steps": steps,
            "warmup": warmup, "ms_per_step": cb["ms_per_step"], "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "impl": "reference",
            "config": {"workload": workload_name(SAMPLE_CELLS, "FP64 CPU restatement of the reference path "
                                                 "(sparse LDL^T Newton)") +
                       f"; a bounded sample of the {workload_name(CELLS, 'GPU')} workload, same spacing, jitter "
                       "and material distribution, compared per element",
                       "elements": ne, "precision": "fp64", "parallelism": "host cores"},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_phases:
        line["cpu_baseline"]["phases"] = cpu_phases()
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
_asm_variant = 0


def build_energy(precision, X, T, E, mask, val, device):
    from sors_b200 import _lib
    from sors_b200 import py_sors as ps
    s = make_settings(precision)
    s.device = device
    en = ps.EnergyTet.from_arrays(X, T, s, np.array([0.0, 0.0, -9.81]), 0.0, density=1070.0, youngsModulus=E,
                                  poissonsRatio=0.45, neumannBCmask=mask, neumannBCvalue=val)
    if _asm_variant:
        _lib.check(_lib.load().sors_set_assembly_variant(en.handle(), _asm_variant))
    return en, ps.Solver(s)


def timed_device_steps(torch, L, en, sol, q_dev, steps, stream):
    """Device-resident steps timed with CUDA events on the library's stream."""
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    newton = pcg = 0
    for _ in range(steps):
        st = sol.step_device(q_dev.data_ptr(), en)
        newton += st.newton_iters
        pcg += st.pcg_iters
    ev1.record(stream)
    ev1.synchronize()
    return ev0.elapsed_time(ev1), newton, pcg


def max_over_ranks(value, dist, device=None):
    """The largest of each rank's value (every rank calls it, same order)."""
    if dist is None:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_gpu(args, rank, world, local_rank):
    import torch
    from sors_b200 import _lib
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local_rank)
    L = _lib.load()
    cells = tuple(args.cells)
    X, T, E, mask, val = block_mesh(cells, seed=0)
    ne = T.shape[0]
    nn = X.shape[0]
    en, sol = build_energy(args.precision, X, T, E, mask, val, local_rank)
    stream = torch.cuda.ExternalStream(L.sors_stream(en.handle()), device=local_rank)
    q_dev = torch.tensor(X.ravel(), dtype=torch.float64, device=f"cuda:{local_rank}")
    for _ in range(args.warmup):
        sol.step_device(q_dev.data_ptr(), en)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    launches0 = L.sors_kernel_launch_count()
    hess0 = L.sors_evaluation_count(en.handle(), 1)
    with Clocks(local_rank) as clk:
        ms, newton, pcg = timed_device_steps(torch, L, en, sol, q_dev, args.steps, stream)
    launches = L.sors_kernel_launch_count() - launches0
    hess_evals = L.sors_evaluation_count(en.handle(), 1) - hess0
    torch.cuda.synchronize()
    if dist:
        ms = max_over_ranks(ms, dist, f"cuda:{local_rank}")
        dist.barrier()
    value = world * ne * args.steps / (ms / 1e3)
    # kernel roofline on the final assembled system
    prof = _lib.SorsKernelProfile()
    _lib.check(L.sors_profile_kernels(en.handle(), 20, __import__("ctypes").byref(prof)))
    # per PCG iteration: the SpMV and either the block-Jacobi update or the two
    # two-level kernels (update + restriction, coarse solve + prolongation)
    two_level = prof.tl_restrict_ms > 0.0
    it_kernels = {"tl_restrict": (prof.tl_restrict_ms, prof.tl_restrict_bytes),
                  "tl_coarse_z": (prof.tl_coarse_z_ms, prof.tl_coarse_z_bytes)} if two_level else \
        {"pcg_update": (prof.pcg_update_ms, prof.pcg_update_bytes)}
    kern = {"form_p": (prof.form_p_ms, prof.form_p_bytes), "pcg_spmv": (prof.spmv_ms, prof.spmv_bytes), **it_kernels,
            "assemble": (prof.assemble_ms, prof.assemble_bytes)}
    per_step = {k: (hess_evals if k == "assemble" else pcg) / args.steps * v[0] for k, v in kern.items()}
    dom = max(per_step, key=per_step.get)
    dur, bytes_ = kern[dom]
    peak, peak_src = measured_peak_hbm()
    achieved = bytes_ / (dur / 1e3) / 1e9
    traffic = ncu_traffic(f"{dom}_{args.precision}", nn)
    # end-to-end through Solver.step with pinned host buffers
    # the solver steps the pinned host solution in place (q_in == q_out)
    q_host = torch.empty(3 * nn, dtype=torch.float64, pin_memory=True).numpy()
    q_host[:] = q_dev.cpu().numpy()
    e2e_steps = args.steps
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True); ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(e2e_steps):
        sol.step(q_host, en, out=q_host)
    ev1.record(stream)
    ev1.synchronize()
    e2e_ms = ev0.elapsed_time(ev1)
    if dist:
        e2e_ms = max_over_ranks(e2e_ms, dist, f"cuda:{local_rank}")
    e2e_value = world * ne * e2e_steps / (e2e_ms / 1e3)
    steps_done = args.warmup + args.steps + e2e_steps
    q_mixed = q_host.copy()
    # plain FP64 drop-in beside it, then advanced untimed to the same step count
    # from the same start, for the mixed-precision error
    fp64 = None
    if not args.no_fp64 and args.precision == "mixed":
        del en  # free the mixed handle's memory first
        en64, sol64 = build_energy("fp64", X, T, E, mask, val, local_rank)
        q64 = torch.tensor(X.ravel(), dtype=torch.float64, device=f"cuda:{local_rank}")
        for _ in range(args.warmup):
            sol64.step_device(q64.data_ptr(), en64)
        stream64 = torch.cuda.ExternalStream(L.sors_stream(en64.handle()), device=local_rank)
        ms64, n64, p64 = timed_device_steps(torch, L, en64, sol64, q64, args.steps, stream64)
        prof64 = _lib.SorsKernelProfile()
        _lib.check(L.sors_profile_kernels(en64.handle(), 20, __import__("ctypes").byref(prof64)))
        for _ in range(steps_done - args.warmup - args.steps):
            sol64.step_device(q64.data_ptr(), en64)
        torch.cuda.synchronize()
        q64h = q64.cpu().numpy()
        disp64 = float(np.abs(q64h - X.ravel()).max())
        fp64 = {"value": ne * args.steps / (ms64 / 1e3), "ms_per_step": ms64 / args.steps,
                "newton_iters_per_step": n64 / args.steps, "pcg_iters_per_step": p64 / args.steps,
                "spmv_gbs": prof64.spmv_bytes / (prof64.spmv_ms / 1e3) / 1e9,
                "assemble_gbs": prof64.assemble_bytes / (prof64.assemble_ms / 1e3) / 1e9,
                "assemble_ms": prof64.assemble_ms,
                "final_disp_max": disp64}
        error_vs_fp64 = {"steps": steps_done, "max_abs_m": float(np.abs(q_mixed - q64h).max()),
                         "rel_to_max_disp": float(np.abs(q_mixed - q64h).max()) / max(disp64, 1e-300),
                         "what": "max |q_mixed - q_fp64| over all DOFs after the same number of steps from "
                                 "the same start, relative to the FP64 run's largest displacement"}
        del en64
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64" if args.precision == "mixed" else "f64", "data": "synthetic",
        "config": {"workload": workload_name(cells, "mixed precision" if args.precision == "mixed" else "FP64"),
                   "elements": ne, "nodes": nn, "dofs": 3 * nn, "precision": args.precision,
                   "newton": "||dx||<1e-9 or ||g||<1e-8, Eisenstat-Walker PCG forcing",
                   "hessian_projection": _projection,
                   "preconditioner": "two-level" if _two_level else "block Jacobi",
                   "numbering": "random permutation" if _shuffle else "grid order (x fastest)",
                   "assembly": ["chunked element-owner", "row-owner", "chunked, two passes"][_asm_variant],
                   "parallelism": "replicas" if world > 1 else "single GPU",
                   "l2": "inputs larger than L2 (assembled system ~1 GB resident), no flush"},
        "newton_steps_per_s": world * args.steps / (ms / 1e3),
        "newton_iters_per_step": newton / args.steps,
        "hessian_assemblies_per_step": hess_evals / args.steps, "pcg_iters_per_step": pcg / args.steps,
        "assembly_gbs": prof.assemble_bytes / (prof.assemble_ms / 1e3) / 1e9,
        "kernels": {**{f"{k}_ms": v[0] for k, v in kern.items()},
                    **{f"{k}_gbs": v[1] / (v[0] / 1e3) / 1e9 for k, v in kern.items()},
                    "share_ms_per_step": per_step},
        "roofline": {"kernel": dom, "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "peak_source": peak_src, "traffic": traffic,
                     "algorithmic_bytes_per_launch": bytes_},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 8 * 3 * nn, "d2h_bytes_per_step": 8 * 3 * nn},
        "gpu_launches": int(launches),
        "clocks": clk.summary(),
    }
    if fp64:
        line["fp64"] = fp64
        line["error_vs_fp64"] = error_vs_fp64
    if world == 1 and not args.no_cpu:
        try:
            cb = cpu_sample_run(steps=3, warmup=1)
            line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")}
        except Exception as ex:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
                                    "sample": f"failed: {ex}"}
        if not args.no_phases:
            try:
                ph = cpu_phases()
                # the GPU does both phases in one assembly launch (gradient rows and Hessian)
                ph["gpu_assemble_ms"] = {"mixed": prof.assemble_ms,
                                         "fp64": fp64["assemble_ms"] if fp64 else None}
                line["cpu_baseline"]["phases"] = ph
            except Exception as ex:
                line["cpu_baseline"]["phases"] = {"failed": str(ex)}
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def run_c3(args):
    """Pressure-actuated arm: voxelised cylinder (R 20 mm, L 200 mm, h 1.25 mm) with
    three closed chambers, base clamped, E 3e5, nu 0.48; static Newton solve per
    load level, 10 levels 0 -> 50 kPa, on one chamber and on all three.  As in
    python/d04_sopra.py:73-85 the largest surface group (the outer skin) is
    dropped and the remaining groups (the chamber walls) are the pressure
    groups.  One line per (load case, precision)."""
    import torch
    from sors_b200 import meshes
    from sors_b200 import py_sors as ps
    torch.cuda.set_device(0)
    X, H = meshes.voxel_cylinder(radius=0.02, length=0.2, h=1.25e-3, cap_layers=2)
    groups, _ = meshes.extract_surfaces(X, H)
    groups.pop(int(np.argmax([len(g) for g in groups])))
    faces = np.concatenate(groups)
    gid = np.concatenate([np.full(len(g), k) for k, g in enumerate(groups)])
    mask = np.repeat((np.abs(X[:, 2]) < 1e-12).astype(np.int32), 3)
    if args.profile_only:
        # the hex kernels at rest, 5 launches each (short ncu capture target)
        import ctypes
        from sors_b200 import _lib
        L = _lib.load()
        for precision in ("mixed", "fp64"):
            s = ps.SimulationSettings()
            s.meshType = "Hexahedron"; s.dt = 0.0; s.precision = precision
            s.hessianProjection = PROJECTION[args.c3_projection]
            fp = ps.Params(["surfaceVertexIdx", "surfaceGroups"], [faces.astype(float), gid.astype(float)])
            en = ps.EnergyHex.from_arrays(X, H, s, np.zeros(3), 0.0, density=1070.0, youngsModulus=3e5,
                                          poissonsRatio=0.48, neumannBCmask=mask,
                                          neumannBCvalue=np.zeros(mask.size), forceTypesList=["pressure"],
                                          forceParameterList=fp)
            prof = _lib.SorsKernelProfile()
            _lib.check(L.sors_profile_kernels(en.handle(), 5, ctypes.byref(prof)))
            print(json.dumps({"workload": "c3 kernels at rest", "precision": precision,
                              "hessian_projection": args.c3_projection, "hexes": int(H.shape[0]),
                              **{k: getattr(prof, k) for k, _ in _lib.SorsKernelProfile._fields_
                                 if k.endswith("_ms")}}),
                  flush=True)
            del en
        return
    for case, chambers in (("one chamber", [0]), ("all three chambers", list(range(len(groups))))):
        for precision in ("mixed", "fp64"):
            s = ps.SimulationSettings()
            s.meshType = "Hexahedron"; s.dt = 0.0; s.timeSteppingScheme = "backward_euler"
            s.precision = precision; s.newtonResidualTol = 1e-8
            s.hessianProjection = PROJECTION[args.c3_projection]
            s.linearSolver = args.c3_solver
            s.pressureJacobian = args.c3_pressure_jac
            fp = ps.Params(["surfaceVertexIdx", "surfaceGroups"], [faces.astype(float), gid.astype(float)])
            en = ps.EnergyHex.from_arrays(X, H, s, np.zeros(3), 0.0, density=1070.0, youngsModulus=3e5,
                                          poissonsRatio=0.48, neumannBCmask=mask,
                                          neumannBCvalue=np.zeros(mask.size), forceTypesList=["pressure"],
                                          forceParameterList=fp)
            sol = ps.Solver(s)
            q = X.ravel().copy()
            levels, newton, pcg = 10, 0, 0
            err = None
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            try:
                for lvl in range(1, levels + 1):
                    pr = np.zeros((len(groups), 1)); pr[chambers, 0] = 5e3 * lvl
                    q = sol.step(q, en, ps.Params(["pressure"], [pr]), 0.0)
                    newton += sol.last_stats.newton_iters; pcg += sol.last_stats.pcg_iters
            except RuntimeError as ex:
                err = f"level {lvl}: {ex}"
            wall = time.perf_counter() - t0
            print(json.dumps({"workload": f"c3 pressure-actuated hex arm, static 10-level ramp to 50 kPa ({case})",
                              "precision": precision, "hessian_projection": args.c3_projection,
                              "linear_solver": args.c3_solver, "pressure_jacobian": args.c3_pressure_jac,
                              "hexes": int(H.shape[0]), "nodes": int(X.shape[0]), "chambers": len(groups),
                              "s_per_load_level": wall / levels, "newton_iters_per_level": newton / levels,
                              "pcg_iters_per_level": pcg / levels, "error": err,
                              "tip_displacement_max_m": float(np.abs(q - X.ravel()).max())}), flush=True)
            del en


def c4_case(seed, steps):
    """Differentiation workload: hex bar 0.2 x 0.04 x 0.04 m (40 x 8 x 8 hexes),
    fibres +x in every element, a_e(t) ~ U[0, 1] seeded, E 2e5, nu 0.45, rho
    1070, dropped from 0.05 m onto the plane z = 0 (planeContact, minimize_SQP),
    backward Euler dt 2e-3.  Loss (z_com(T) - 0.08)^2."""
    from sors_b200 import meshes
    X, H = meshes.hex_bar(40, 8, 8, (0.2, 0.04, 0.04))
    X = X + np.array([0.0, 0.0, 0.05])
    ne = H.shape[0]
    rng = np.random.default_rng(seed)
    act = rng.uniform(0.0, 1.0, (steps, ne))
    E = np.full(ne, 2e5)
    groups, _ = meshes.extract_surfaces(X, H)
    surf = np.unique(np.concatenate([g.ravel() for g in groups]))
    return X, H, E, act, surf


def c4_energy(X, H, E, surf, precision="fp64", members=1):
    """Energy/Solver of `members` copies of the C4 bar in one handle (a union:
    the copies share no element, so the system, its contacts and its adjoint
    are the direct sum of the copies'; every kernel launch serves all of them,
    and each linear solve runs one PCG per copy).  Each element is its own
    muscle group."""
    from sors_b200 import py_sors as ps
    s = ps.SimulationSettings()
    s.meshType = "Hexahedron"; s.dt = 2e-3; s.timeSteppingScheme = "backward_euler"
    s.solverMethod = "minimize_SQP"; s.precision = precision
    n1, e1 = X.shape[0], H.shape[0]
    Xu = np.tile(X, (members, 1))
    Hu = np.concatenate([H + k * n1 for k in range(members)]).astype(np.int32)
    su = np.concatenate([surf + k * n1 for k in range(members)])
    ne = e1 * members
    Eu = np.broadcast_to(np.asarray(E, float), (ne,)).copy() if np.size(E) in (1, ne) else np.tile(E, members)
    en = ps.EnergyHex.from_arrays(Xu, Hu, s, np.array([0.0, 0.0, -9.81]), 0.0, density=1070.0, youngsModulus=Eu,
                                  poissonsRatio=0.45, muscleGroup=np.arange(ne), softconStiffness=np.full(ne, 5e4),
                                  softconDirection=np.tile([1.0, 0.0, 0.0], (ne, 1)))
    cp = ps.Params()
    cp.set_param("positionVectorListPlanes", np.zeros(3))
    cp.set_param("normalVectorListPlanes", np.array([0.0, 0.0, 1.0]))
    cp.set_param("surfaceVerticesIdx", su.astype(float))
    en._setup_constraints_forces(["planeContact"], cp, (), None)
    if members > 1:
        # one PCG per copy in shared launches (member-segmented solves)
        import ctypes
        from sors_b200 import _lib
        offs = np.arange(members + 1, dtype=np.int32) * n1
        _lib.check(_lib.load().sors_set_members(en._h, offs.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)),
                                                members))
    return en, ps.Solver(s)


def c4_mass(X, H):
    """Lumped node masses of the C4 bar (uniform hexes: rho V / 8 per corner)."""
    m = np.zeros(X.shape[0])
    np.add.at(m, H.ravel(), 1070.0 * (0.2 * 0.04 * 0.04 / H.shape[0]) / 8)
    return m


def run_c4(args):
    """Gradient of the C4 loss w.r.t. per-element E and a_e(t) by the adjoint,
    for `seeds` activation seeds in one union handle (one forward and one
    backward pass serve all of them).  The directional derivative of seed 0
    along `fd_dirs` seeded directions is checked against central differences
    (h = 1e-6) of the GPU FP64 forward, all directions in one union of
    2 x fd_dirs perturbed copies."""
    import torch
    from sors_b200.adjoint import RolloutAdjoint
    torch.cuda.set_device(0)
    steps, dt, S = args.c4_steps, 2e-3, args.seeds
    X, H, E, _, surf = c4_case(0, steps)
    n1, e1 = X.shape[0], H.shape[0]
    acts = [c4_case(sd, steps)[3] for sd in range(S)]
    act_u = np.concatenate(acts, axis=1)                      # (T, S * e1): group = union element
    E_u = np.tile(E, S)
    m = c4_mass(X, H)

    def losses(qT, members):
        z = (qT.reshape(members, n1, 3)[:, :, 2] * m).sum(axis=1) / m.sum()
        return (z - 0.08) ** 2, z

    en, sol = c4_energy(X, H, E, surf, members=S)
    r = RolloutAdjoint(en, sol, steps, dt, poisson=0.45, checkpoint_every=args.checkpoint_every)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    qT = r.forward(E_u, act_u)
    t1 = time.perf_counter()
    Ls, z = losses(qT, S)
    dq = np.zeros((S, n1, 3))
    dq[:, :, 2] = (2 * (z - 0.08))[:, None] * m[None, :] / m.sum()
    gE, gA, _, _ = r.backward(dq.ravel())
    t2 = time.perf_counter()
    fwd_iters = r.last_pcg_iters
    del r, en, sol
    # central differences for seed 0: member 2d = +h r_d, member 2d + 1 = -h r_d
    D, h = args.fd_dirs, 1e-6
    rng = np.random.default_rng(99)
    dirs = [(rng.standard_normal(e1), rng.standard_normal((steps, e1))) for _ in range(D)]
    d_adj = np.array([gE[:e1] @ (E * rE) + (gA[:, :e1] * rA).sum() for rE, rA in dirs])
    Efd = np.concatenate([E * (1 + sg * h * rE) for rE, _ in dirs for sg in (1, -1)])
    Afd = np.concatenate([acts[0] + sg * h * rA for _, rA in dirs for sg in (1, -1)], axis=1)
    en2, sol2 = c4_energy(X, H, Efd, surf, members=2 * D)
    r2 = RolloutAdjoint(en2, sol2, steps, dt, poisson=0.45, checkpoint_every=steps)
    t3 = time.perf_counter()
    qfd = r2.forward(Efd, Afd)
    t4 = time.perf_counter()
    Lfd, _ = losses(qfd, 2 * D)
    d_fd = (Lfd[0::2] - Lfd[1::2]) / (2 * h)
    errs = np.abs(d_adj - d_fd) / np.maximum(np.abs(d_fd), 1e-300)
    print(json.dumps({"workload": f"c4 SoftCon hex bar 40x8x8 dropped from 0.05 m on z=0, adjoint of E and a_e(t), "
                                  f"FP64, {S} seeds in one union handle",
                      "hexes_per_seed": int(e1), "nodes_per_seed": int(n1), "hexes_total": int(e1 * S),
                      "steps": steps, "seeds": S, "gradients_per_s": S / (t2 - t0), "wall_s": t2 - t0,
                      "forward_ms_per_step": 1e3 * (t1 - t0) / steps, "backward_ms_per_step": 1e3 * (t2 - t1) / steps,
                      "adjoint_pcg_iters_per_step": fwd_iters / steps, "checkpoint_every": args.checkpoint_every,
                      "loss_seed0": float(Ls[0]), "loss_mean": float(Ls.mean()),
                      "fd_directions": D, "fd_h": h, "fd_forward_s": t4 - t3,
                      "fd_max_rel_err": float(errs.max()) if D else None,
                      "fd_vs": "central differences of the GPU FP64 forward (union of 2 x fd_directions copies)",
                      "directional_derivatives": d_adj.tolist()}), flush=True)


def run_serve(args):
    """Mixed-size poke sweep (C5): `rollouts` requests with Poisson arrivals at
    `rate` per second, each a 6-tet cube (log-uniform 5k-250k tets, side
    U[30, 60] mm, E U[2e4, 2e5], nu U[0.30, 0.48], rho 1000) on z = 0 pressed by
    a 10 mm disk moving 10 mm down, 100 steps of 1e-2 s, minimize_SQP.
    Served form: mixed precision, continuous admission by HBM footprint,
    `slots` handles in flight.  Baseline: the plain FP64 drop-in, one rollout at
    a time, on every k-th request of the same set (k = rollouts / baseline
    sample, the same size distribution); its rollouts/s is the subsample's
    count over its summed rollout times."""
    import torch
    from sors_b200 import serving
    torch.cuda.set_device(0)

    def make(precision):
        r = np.random.default_rng(11)
        out = []
        for i in range(args.rollouts):
            tets = float(np.exp(r.uniform(np.log(5e3), np.log(args.tets_max))))
            n = max(2, int(round((tets / 6.0) ** (1.0 / 3.0))))
            out.append(serving.poke_cube_request(r, n, tag=i, steps=args.rollout_steps, dt=1e-2, precision=precision))
        return out

    def summary(res, wall, reqs):
        steps = [x for r in res for x in r.step_latencies]
        lat = [r.latency for r in res]
        failed = sorted((r.tag, r.error) for r in res if r.error)
        return {"rollouts": len(res), "rollouts_per_s": len(res) / wall, "makespan_s": wall,
                "mean_batch": float(np.mean([r.batch for r in res])) if res else 0.0,
                "failures": len(failed), "failed": [{"tag": t, "tets": int(reqs[t].elements.shape[0]), "error": e}
                                                    for t, e in failed],
                "step_latency_p50_ms": 1e3 * serving.percentile(steps, 50),
                "step_latency_p99_ms": 1e3 * serving.percentile(steps, 99),
                "rollout_latency_p50_s": serving.percentile(lat, 50),
                "rollout_latency_p99_s": serving.percentile(lat, 99),
                "tets_total": int(sum(q.elements.shape[0] for q in reqs.values()))}

    rng = np.random.default_rng(7)
    gaps = rng.exponential(1.0 / args.rate, size=args.rollouts)
    arrivals = np.cumsum(gaps) - gaps[0]
    reqs_m = make("mixed")
    by_tag = {q.tag: q for q in reqs_m}
    srv = serving.RolloutServer(max_slots=args.slots, batch_max=args.batch)
    t0 = time.perf_counter()
    for req, at in zip(reqs_m, arrivals):
        now = time.perf_counter() - t0
        if at > now:
            time.sleep(at - now)
        srv.submit(req)
    res_m = srv.close()
    served = summary(res_m, time.perf_counter() - t0, by_tag)
    # plain FP64 drop-in, one rollout at a time, on every k-th request
    k = max(1, args.rollouts // max(1, args.baseline_sample))
    reqs_p = make("fp64")[::k]
    plain_res, busy = [], 0.0
    for req in reqs_p:
        srv1 = serving.RolloutServer(max_slots=1, batch_max=1)
        t1 = time.perf_counter()
        srv1.submit(req)
        plain_res += srv1.close()
        busy += time.perf_counter() - t1
    plain = summary(plain_res, busy, {q.tag: q for q in reqs_p})
    plain["every_kth_request"] = k
    # accuracy of the served form against the plain FP64 path on the subsample
    final_p = {r.tag: r.final for r in plain_res if r.final is not None}
    rel = [float(np.abs(r.final - final_p[r.tag]).max() /
                 max(np.abs(final_p[r.tag] - by_tag[r.tag].vertices.ravel()).max(), 1e-30))
           for r in res_m if r.final is not None and r.tag in final_p]
    print(json.dumps({"workload": f"poke sweep: {args.rollouts} rollouts x {args.rollout_steps} steps, "
                                  f"Poisson arrivals at {args.rate}/s, 6-tet cubes 5k-{args.tets_max / 1e3:.0f}k "
                                  f"tets (log-uniform) on z=0 "
                                  f"pressed by a 10 mm disk moving 10 mm down (minimize_SQP contact)",
                      "slots": args.slots, "batch_max": args.batch, "served_mixed": served,
                      "plain_fp64_sequential": plain,
                      "speedup_rollouts_per_s": served["rollouts_per_s"] / plain["rollouts_per_s"],
                      "max_rel_diff_vs_fp64": max(rel) if rel else None,
                      "compared_rollouts": len(rel)}), flush=True)


def run_profile_only(args):
    """Builds the workload and runs only the kernel profiler (3 launches each)."""
    import ctypes

    import torch
    from sors_b200 import _lib
    torch.cuda.set_device(0)
    L = _lib.load()
    X, T, E, mask, val = block_mesh(tuple(args.cells), seed=0)
    en, sol = build_energy(args.precision, X, T, E, mask, val, 0)
    prof = _lib.SorsKernelProfile()
    _lib.check(L.sors_profile_kernels(en.handle(), 3, ctypes.byref(prof)))
    out = {f: getattr(prof, f) for f, _ in _lib.SorsKernelProfile._fields_}
    out["elements"] = T.shape[0]
    out["nodes"] = X.shape[0]
    print(json.dumps(out), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--cells", type=int, nargs=3, default=list(CELLS))
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-two-level", dest="two_level", action="store_false",
                    help="block Jacobi alone instead of the two-level PCG preconditioner")
    ap.add_argument("--projection", default="adaptive", choices=sorted(PROJECTION),
                    help="SPD projection of the element Hessians: always, never, or only where PCG meets "
                         "negative curvature")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--assembly", type=int, default=0, choices=[0, 1, 2],
                    help="assembly kernel: 0 chunked element-owner, 1 row-owner, 2 chunked in two passes")
    ap.add_argument("--shuffle", action="store_true",
                    help="renumber the block's nodes and elements by a seeded random permutation")
    ap.add_argument("--no-phases", action="store_true",
                    help="skip the full-size CPU gradient / Hessian assembly timing (about 30 s of host work)")
    ap.add_argument("--workload", default="c2", choices=["c2", "c3", "c4", "serve"],
                    help="c2: the 3.0M-tet block (default); c3: pressure-actuated hex arm, static load ramp; "
                         "serve: Poisson stream of poke rollouts")
    ap.add_argument("--rollouts", type=int, default=512)
    ap.add_argument("--rollout-steps", type=int, default=100)
    ap.add_argument("--rate", type=float, default=2.0, help="serve: Poisson arrival rate (rollouts/s)")
    ap.add_argument("--tets-max", type=float, default=2.5e5, help="serve: upper end of the log-uniform tet counts")
    ap.add_argument("--slots", type=int, default=16, help="serve: concurrent handles")
    ap.add_argument("--batch", type=int, default=1, help="serve: rollouts packed into one union handle (1: none; unions measured slower on the poke mix)")
    ap.add_argument("--baseline-sample", type=int, default=64,
                    help="serve: measure the sequential FP64 baseline on every (rollouts / K)-th request")
    ap.add_argument("--c3-pressure-jac", default="reference", choices=["reference", "exact"],
                    help="c3: follower-load coefficient of the Newton matrix for quads (p/6 as the reference, or p/8)")
    ap.add_argument("--c3-solver", default="pcg", choices=["pcg", "minres"],
                    help="c3: Newton linear solver (minres takes the exact-Hessian step, with --c3-projection false)")
    ap.add_argument("--c3-projection", default="true", choices=sorted(PROJECTION),
                    help="c3: SPD projection of the element Hessians")
    ap.add_argument("--seeds", type=int, default=64, help="c4: activation seeds differentiated in one union handle")
    ap.add_argument("--c4-steps", type=int, default=100, help="c4: steps per rollout")
    ap.add_argument("--fd-dirs", type=int, default=20, help="c4: finite-difference directions checked")
    ap.add_argument("--checkpoint-every", type=int, default=10, help="c4: checkpoint interval (steps)")
    ap.add_argument("--profile-only", action="store_true",
                    help="assemble once at rest and launch each hot kernel 3 times (short ncu capture target)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    global _projection, _two_level, _shuffle, _asm_variant
    _asm_variant = args.assembly
    _projection = args.projection
    _two_level = args.two_level
    _shuffle = args.shuffle
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
    elif args.workload == "c3":
        run_c3(args)
    elif args.workload == "c4":
        run_c4(args)
    elif args.workload == "serve":
        run_serve(args)
    elif args.profile_only:
        run_profile_only(args)
    else:
        run_gpu(args, rank, world, local_rank)


if __name__ == "__main__":
    main()
