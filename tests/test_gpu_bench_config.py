"""The bench's own configuration against the oracle.

bench.py times the jittered 6-tet block with mixed precision, the adaptive
Hessian (exact unless PCG meets negative curvature), the two-level PCG
preconditioner, the Newton residual stop 1e-8 (which enables the gradient-only
probe and the chord step near convergence) and the Newton predictor.  These
tests run exactly those settings (bench.build_energy) on the 24 x 12 x 12-cell
sample of the same block, with its per-element log-uniform Young's modulus,
and compare every step with the oracle's FP64 LDL^T Newton (the reference's
Solver::step, cpp/src/solver.cpp:5-105): FP64 within 1e-8 m, mixed precision
within 1e-6 of the largest displacement.
"""
import numpy as np
import pytest

import bench

pytestmark = pytest.mark.gpu

STEPS = 6


@pytest.fixture(scope="module")
def sample_trajectory():
    from oracle import oracle as orc
    X, T, E, mask, val = bench.block_mesh(bench.SAMPLE_CELLS, seed=0)
    o = orc.System(X, T, rho=1070.0, youngs=E, nu=0.45, grav=(0, 0, -9.81), scheme="backward_euler",
                   method="minimize_newton", dt=bench.DT, substeps=1)
    o.set_neumann(mask, val)
    q = X.ravel().copy()
    traj = []
    for _ in range(STEPS):
        q, st = o.step(q)
        assert st == 0
        traj.append(q.copy())
    return (X, T, E, mask, val), traj


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_bench_settings_match_oracle(sample_trajectory, precision):
    import torch
    (X, T, E, mask, val), traj = sample_trajectory
    torch.cuda.set_device(0)
    assert bench._projection == "adaptive" and bench._two_level
    en, sol = bench.build_energy(precision, X, T, E, mask, val, 0)
    s = bench.make_settings(precision)
    assert s.hessianProjection == "adaptive" and s.twoLevelPreconditioner is True
    assert s.newtonResidualTol == 1e-8 and s.newtonPredictor
    q = X.ravel().copy()
    worst = disp = 0.0
    newton = 0
    for k in range(STEPS):
        q = sol.step(q, en)
        newton += sol.last_stats.newton_iters
        worst = max(worst, float(np.abs(q - traj[k]).max()))
        disp = max(disp, float(np.abs(traj[k] - X.ravel()).max()))
    assert disp > 1e-4  # the block sags under gravity
    assert newton >= 2 * STEPS
    if precision == "fp64":
        assert worst < 1e-8, worst
    else:
        assert worst <= 1e-6 * disp, (worst, disp)
