"""The element-owner tet assembly over node chunks against the row-owner
assembly and the oracle.

Both kernels evaluate the same element terms in the same Hessian type and sum
each CSR block's items in the same order, so their Hessians agree to the last
bits (FP64 1e-14 relative, FP32 blocks 1e-6 relative); gradients agree to
rounding.  The chunked kernel is checked against the oracle's triplet -> CSR
assembly (cpp/src/energy.cpp:252-390) at 1e-10 in FP64, on the jittered
block, on the same block with its nodes randomly renumbered (chunks are cut in
Morton order of the positions, whatever the numbering), with Neumann rows, for
backward Euler and Crank-Nicolson, and for stable Neo-Hookean elements.
"""
import numpy as np
import pytest

from sors_b200 import meshes
from tests.helpers import deform, make_pair, rel_err

pytestmark = pytest.mark.gpu

ELEM_TOL = 1e-10


def _block(shuffle):
    X, T, E = meshes.jittered_block_tets(10, 5, 6, (0.1, 0.05, 0.06), jitter=0.1, seed=4)
    if shuffle:
        perm = np.random.default_rng(8).permutation(X.shape[0])
        inv = np.empty_like(perm); inv[perm] = np.arange(perm.size)
        X = X[perm]
        T = inv[T].astype(np.int32)
    return X, T, E


def _hessians(en, q, dt):
    from sors_b200 import _lib
    L = _lib.load()
    assert L.sors_assembly_chunks(en.handle()) > 0
    g_chunk = en.compute_gradient(q, dt)
    H_chunk = en.compute_hessian(q, dt)
    _lib.check(L.sors_set_assembly_variant(en.handle(), 1))
    g_row = en.compute_gradient(q, dt)
    H_row = en.compute_hessian(q, dt)
    _lib.check(L.sors_set_assembly_variant(en.handle(), 0))
    return g_chunk, H_chunk, g_row, H_row


@pytest.mark.parametrize("shuffle", [False, True])
@pytest.mark.parametrize("scheme,dt", [("backward_euler", 5e-3), ("crank_nicolson", 5e-3), ("backward_euler", 0.0)])
@pytest.mark.parametrize("energy", ["neohookean", "stableneohookean"])
def test_chunked_matches_row_owner_and_oracle(oracle, shuffle, scheme, dt, energy):
    X, T, E = _block(shuffle)
    rng = np.random.default_rng(11)
    en, _, o, _ = make_pair(X, T, E=E, scheme=scheme, dt=dt if dt else 1e-3, project=False, alpha=0.3,
                            energy=energy)
    q = deform(X, rng, amp=0.04)
    vprev = rng.uniform(-0.01, 0.01, q.size)
    en.set_initial_velocity(vprev); o.set_initial_velocity(vprev)
    g_chunk, H_chunk, g_row, H_row = _hessians(en, q, dt)
    scale = np.abs(H_row.data).max()
    assert np.abs((H_chunk - H_row).data).max(initial=0.0) <= 1e-14 * scale
    assert rel_err(g_chunk, g_row) < 1e-14
    Ho, st = o.hessian_csr(q, dt)
    assert st == 0
    assert np.abs((H_chunk - Ho).data).max(initial=0.0) <= ELEM_TOL * np.abs(Ho.data).max()
    assert rel_err(g_chunk, o.gradient(q, dt)) < ELEM_TOL


@pytest.mark.parametrize("energy", ["neohookean", "stableneohookean"])
def test_chunked_mixed_precision_blocks(oracle, energy):
    X, T, E = _block(True)
    rng = np.random.default_rng(12)
    en, _, o, _ = make_pair(X, T, E=E, dt=5e-3, project=False, precision="mixed", energy=energy)
    q = deform(X, rng, amp=0.04)
    g_chunk, H_chunk, g_row, H_row = _hessians(en, q, 5e-3)
    scale = np.abs(H_row.data).max()
    assert np.abs((H_chunk - H_row).data).max(initial=0.0) <= 1e-6 * scale
    assert rel_err(g_chunk, g_row) < 1e-14
    Ho, _ = o.hessian_csr(q, 5e-3)
    assert np.abs((H_chunk - Ho).data).max(initial=0.0) <= 1e-6 * np.abs(Ho.data).max()


def test_chunked_is_bit_reproducible(oracle):
    X, T, E = _block(True)
    en, _, _, _ = make_pair(X, T, E=E, dt=5e-3, project=False)
    q = deform(X, np.random.default_rng(13), amp=0.04)
    a = en.compute_hessian(q, 5e-3)
    b = en.compute_hessian(q, 5e-3)
    assert (a != b).nnz == 0
    assert np.array_equal(en.compute_gradient(q, 5e-3), en.compute_gradient(q, 5e-3))


def test_inverted_element_reported(oracle):
    X, T, E = _block(False)
    en, _, _, _ = make_pair(X, T, E=E, dt=5e-3, project=False)
    q = X.copy()
    a, b = T[7, 0], T[7, 1]
    q[[a, b]] = q[[b, a]]  # swapping two vertices of one tet inverts it
    with pytest.raises(RuntimeError, match="Inverted Elements"):
        en.compute_hessian(q.ravel(), 5e-3)


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("energy", ["neohookean", "stableneohookean"])
def test_two_pass_chunked_matches_one_pass(oracle, precision, energy):
    # variant 2: every element evaluated once into device records, then the
    # chunks load them; the same generators, so the same sums
    from sors_b200 import _lib
    L = _lib.load()
    X, T, E = _block(True)
    rng = np.random.default_rng(14)
    en, _, o, _ = make_pair(X, T, E=E, dt=5e-3, project=False, precision=precision, energy=energy)
    q = deform(X, rng, amp=0.04)
    g1 = en.compute_gradient(q, 5e-3)
    H1 = en.compute_hessian(q, 5e-3)
    _lib.check(L.sors_set_assembly_variant(en.handle(), 2))
    g2 = en.compute_gradient(q, 5e-3)
    H2 = en.compute_hessian(q, 5e-3)
    _lib.check(L.sors_set_assembly_variant(en.handle(), 0))
    assert np.abs((H2 - H1).data).max(initial=0.0) <= 1e-6 * np.abs(H1.data).max()
    assert rel_err(g2, g1) < 1e-14
    if precision == "fp64":
        Ho, _ = o.hessian_csr(q, 5e-3)
        assert np.abs((H2 - Ho).data).max(initial=0.0) <= ELEM_TOL * np.abs(Ho.data).max()
