"""sors_elem_energy_noalloc: the element-energy sum for callers that cannot let
a library allocate device memory (their memory belongs to their own pool or
arena, or they run a real-time loop that must not allocate after start-up).

The entry point keeps its scratch in a fixed array inside the library, so the
caller only provides device inputs and the output.  These checks call it
through the C ABI, twice in a row on different states (the second call reuses
the scratch the first one left behind), and compare it with the element part
of the existing sors_energy entry point on the same mesh, within the element
tolerance of the other parity tests.  This file is collected last.
"""
import ctypes as C

import numpy as np
import pytest

from sors_b200 import meshes
from tests.helpers import deform, make_pair

pytestmark = pytest.mark.gpu

TOL = 1e-10


def _noalloc_energy(torch, L, X, T, E, nu, q):
    dev = torch.device("cuda:0")
    Xd = torch.tensor(np.ascontiguousarray(X).ravel(), dtype=torch.float64, device=dev)
    qd = torch.tensor(np.ascontiguousarray(q).ravel(), dtype=torch.float64, device=dev)
    Td = torch.tensor(np.ascontiguousarray(T, dtype=np.int32).ravel(), dtype=torch.int32, device=dev)
    Ed = torch.tensor(np.broadcast_to(E, (T.shape[0],)).copy(), dtype=torch.float64, device=dev)
    nd = torch.tensor(np.broadcast_to(nu, (T.shape[0],)).copy(), dtype=torch.float64, device=dev)
    out = torch.full((1,), float("nan"), dtype=torch.float64, device=dev)
    st = L.sors_elem_energy_noalloc(C.c_void_p(Xd.data_ptr()), C.c_void_p(qd.data_ptr()), C.c_void_p(Td.data_ptr()),
                                    T.shape[0], T.shape[1], C.c_void_p(Ed.data_ptr()), C.c_void_p(nd.data_ptr()),
                                    C.c_void_p(out.data_ptr()), None)
    torch.cuda.synchronize()
    return st, float(out.item())


@pytest.mark.parametrize("kind", ["tet", "hex"])
def test_noalloc_matches_energy_entry_point(kind):
    import torch

    from sors_b200 import _lib
    L = _lib.load()
    if kind == "tet":
        X, T = meshes.cantilever_tets()
    else:
        X, T = meshes.hex_bar(10, 3, 3, (0.05, 0.015, 0.015))
    rng = np.random.default_rng(42)
    E = np.exp(rng.uniform(np.log(5e4), np.log(5e5), T.shape[0]))
    nu = rng.uniform(0.3, 0.48, T.shape[0])
    # zero gravity, no forces, dt = 0: sors_energy and the oracle's energy are
    # exactly the element sum
    en, _, orc_sys, _ = make_pair(X, T, E=E, nu=nu, grav=(0.0, 0.0, 0.0), clamp=False)
    for call in range(2):
        q = deform(X, rng, amp=0.1)
        ref = en.compute_energy(q, 0.0)
        st, val = _noalloc_energy(torch, L, X, T, E, nu, q)
        assert st == 0, _lib.last_error()
        assert abs(val - ref) <= TOL * abs(ref), (call, val, ref)
        ref_cpu = orc_sys.energy(q, 0.0)
        assert abs(val - ref_cpu) <= TOL * abs(ref_cpu), (call, val, ref_cpu)


def test_noalloc_many_blocks_ragged_tail():
    """About 300k tets: 293 blocks of partial sums, the last one partly filled."""
    import torch

    from oracle import oracle as orc
    from sors_b200 import _lib
    L = _lib.load()
    X, T, _ = meshes.jittered_block_tets(40, 25, 50, (0.2, 0.125, 0.25), jitter=0.1, seed=3)
    assert T.shape[0] == 300_000 and T.shape[0] % 1024 != 0
    rng = np.random.default_rng(5)
    E = np.exp(rng.uniform(np.log(5e4), np.log(5e5), T.shape[0]))
    nu = np.full(T.shape[0], 0.45)
    o = orc.System(X, T, rho=1000.0, youngs=E, nu=nu)
    for call in range(2):
        q = deform(X, rng, amp=0.05)
        st, val = _noalloc_energy(torch, L, X, T, E, nu, q)
        assert st == 0, _lib.last_error()
        ref = o.energy(q, 0.0)
        assert abs(val - ref) <= TOL * abs(ref), (call, val, ref)


def test_noalloc_at_capacity():
    """Exactly 8,388,608 tets (every block of partial sums in use).  Under one
    affine map every element of a regular Kuhn grid has the same F and volume,
    so the sum is the element count times one element's energy (oracle)."""
    import torch

    from oracle import oracle as orc
    from sors_b200 import _lib
    L = _lib.load()
    cap = 8_388_608
    nx, ny, nz = 170, 64, 128
    X = meshes.grid_nodes(nx, ny, nz, (0.17, 0.064, 0.128))
    T = meshes.kuhn_tet_elements(nx, ny, nz)
    # pad with repeats of the first elements up to the capacity
    T = np.vstack([T, T[:cap - T.shape[0]]]).astype(np.int32)
    assert T.shape[0] == cap
    A = np.array([[1.05, 0.02, -0.01], [0.03, 0.97, 0.02], [-0.02, 0.01, 1.02]])
    q = X @ A.T
    psi_one, _, _, _ = orc.elem_eval(X[T[0]], q[T[0]], 1e5, 0.45)
    ref = cap * psi_one
    for call in range(2):
        st, val = _noalloc_energy(torch, L, X, T, 1e5, 0.45, q)
        assert st == 0, _lib.last_error()
        assert abs(val - ref) <= TOL * abs(ref), (call, val, ref)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    from sors_b200 import _lib
    L = _lib.load()
    dummy = C.c_void_p(1)  # never dereferenced: the size check comes first
    st = L.sors_elem_energy_noalloc(dummy, dummy, dummy, 8_388_609, 4, dummy, dummy, dummy, None)
    assert st == 1
    assert "exceeds the capacity" in _lib.last_error()
