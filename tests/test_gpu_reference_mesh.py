"""A reference demo mesh through the GPU step: the PokeFlex foam dice.

tests/golden/pokeflex_T1P2_mesh.npz holds cpp/demos/meshes/pokeflexFoamDice/
T1P2_mesh.msh as read by sors_b200.msh (tests/golden/make_mesh_fixture.py).
The scene is python/d03_pokeflex.py's, built through the same py_sors calls:
mesh scaled mm -> m, centred in x and z, lowest point moved to y = 0
(d03_pokeflex.py:65-70, python/_utils.py:256-330); stable Neo-Hookean,
E 1345.6 Pa, nu 0.0177, density = 0.14 kg / volume, mass damping 170, gravity
-y; vertices below y = 2 mm clamped (neumannBC); a 20 mm disk facing -y moving
down as 0.25 - 0.17 sin(pi t / 50) m (diskContact, set_disk every frame);
Crank-Nicolson, dt = 1/30 s, minimize_SQP (d03_pokeflex.py:20-31, 99-135,
225-262).  The disk reaches the dice at frame 9; the first 14 frames are
compared with the oracle's SQP step by step.
"""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
FRAMES = 14
DT = 1.0 / 30.0


def dice_scene():
    d = np.load(os.path.join(HERE, "golden", "pokeflex_T1P2_mesh.npz"))
    X = d["vertices"] * 1e-3
    for ax in (0, 2):
        X[:, ax] -= 0.5 * (X[:, ax].min() + X[:, ax].max())
    X[:, 1] -= X[:, 1].min()
    T = d["tets"].astype(np.int32)
    a, b, c, e = (X[T[:, k]] for k in range(4))
    volume = float(np.abs(np.einsum("ij,ij->i", b - a, np.cross(c - a, e - a))).sum() / 6.0)
    return X, T, 0.14 / volume


def disk_center(t):
    return np.array([0.0, 0.25 - 0.17 * np.sin(np.pi * t / 50.0), 0.0])


E_YOUNG, NU, ALPHA = 1345.6024023489897, 0.017728278261516663, 169.99039484049894
GRAV = np.array([0.0, -9.81, 0.0])
NORMAL = [0.0, -1.0, 0.0]


@pytest.fixture(scope="module")
def dice():
    from oracle import contact as oc
    from oracle import oracle as orc
    from sors_b200 import py_sors as ps
    X, T, rho = dice_scene()
    N = X.shape[0]
    groups, _ = ps.IO.extract_tet_surfaces(X, T)
    surf = np.unique(np.vstack(groups))
    mask = np.zeros(3 * N); val = np.zeros(3 * N)
    mask[np.repeat(X[:, 1] < 0.002, 3)] = 1.0
    assert 0 < mask.sum() < 3 * N
    o = orc.System(X, T, rho=rho, youngs=E_YOUNG, nu=NU, grav=GRAV, alpha=ALPHA, scheme="crank_nicolson",
                   method="minimize_SQP", material=orc.MAT_STABLE_NEOHOOKEAN, dt=DT, substeps=1)
    odisk = oc.DiskContact(disk_center(0), NORMAL, [0.02], surf)
    sq = oc.SQPOracle(o, None, odisk, (mask, val))
    qo = X.ravel().copy()
    traj, active = [], []
    for t in range(1, FRAMES + 1):
        odisk.set_disk(disk_center(t), NORMAL, 0.02, 0)
        qo = sq.step(qo, DT)
        traj.append(qo.copy())
        active.append(sq.last_active)
    return X, T, rho, surf, mask, val, traj, active


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_pokeflex_dice_matches_oracle(dice, precision):
    from sors_b200 import py_sors as ps
    X, T, rho, surf, mask, val, traj, active = dice
    ne = T.shape[0]
    assert sum(a > 0 for a in active) >= 3  # the disk pressed the dice in the last frames
    s = ps.SimulationSettings()
    s.meshType = "Tetrahedron"; s.dt = DT; s.substeps = 1; s.CFLtimeSteppingFlag = False
    s.timeSteppingScheme = "crank_nicolson"; s.solverMethod = "minimize_SQP"; s.precision = precision
    energies = [{"stableneohookean"}] * ne
    params = [ps.Params(["density", "youngsModulus", "poissonsRatio"], [rho, E_YOUNG, NU]) for _ in range(ne)]
    cp = ps.Params(["neumannBCmask", "neumannBCvalue", "diskCenterVectorList", "diskNormalVectorList",
                    "diskRadiusList", "surfaceVerticesIdx"],
                   [mask, val, disk_center(0).tolist(), NORMAL, [0.02], surf.tolist()])
    en = ps.Energy(X, T, s, GRAV, ALPHA, energies, params, ["neumannBC", "diskContact"], cp, [], ps.Params())
    sol = ps.Solver(s)
    disk = ps.get_disk_contact_constraint(en, 1)
    q = X.ravel().copy()
    worst = disp = 0.0
    for t in range(1, FRAMES + 1):
        disk.set_disk(disk_center(t), NORMAL, 0.02, diskIdx=0)
        q = sol.step(q, en)
        worst = max(worst, float(np.abs(q - traj[t - 1]).max()))
        disp = max(disp, float(np.abs(traj[t - 1] - X.ravel()).max()))
    # the disk's footprint (captured at first contact and then frozen, as
    # DiskContact::update_active_constraints does) is held on the disk face;
    # other vertices inside its radius are not constrained
    x = q.reshape(-1, 3)[surf]
    on_face = (np.hypot(x[:, 0], x[:, 2]) < 0.02) & (np.abs(x[:, 1] - disk_center(FRAMES)[1]) < 1e-6)
    assert on_face.sum() == active[-1] > 0
    if precision == "fp64":
        assert worst < 1e-8, (worst, disp)
    else:
        assert worst <= 1e-6 * disp, (worst, disp)
