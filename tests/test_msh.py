"""MSH reader (sors_b200.msh, IO.read_tet_MSH / read_hex_MSH) on the CPU."""
import os

import numpy as np
import pytest

from sors_b200 import meshes, msh

# The reference project's root, when a checkout is available (no default):
# its demo meshes live under cpp/demos/meshes.
_REF_ROOT = os.environ.get("SORS_REFERENCE_ROOT", "")
REF_MESHES = os.path.join(_REF_ROOT, "cpp", "demos", "meshes") if _REF_ROOT else ""


@pytest.mark.parametrize("version", ["4.1", "2.2"])
@pytest.mark.parametrize("binary", [False, True])
@pytest.mark.parametrize("kind", ["tet", "hex"])
def test_round_trip(tmp_path, version, binary, kind):
    X = meshes.grid_nodes(3, 2, 2, (0.03, 0.02, 0.02))
    T = meshes.kuhn_tet_elements(3, 2, 2) if kind == "tet" else meshes.hex_grid_elements(3, 2, 2)
    f = tmp_path / "m.msh"
    msh.write_msh(f, X, T, version=version, binary=binary)
    Xr, Tr = msh.read_tet_msh(f) if kind == "tet" else msh.read_hex_msh(f)
    np.testing.assert_array_equal(Xr, X)
    np.testing.assert_array_equal(Tr, T)


def test_tag_mapping_and_type_filter(tmp_path):
    # non-contiguous node tags and a mixed element list: only tets come back,
    # mapped to 0-based vertex indices in node order
    f = tmp_path / "m.msh"
    f.write_text("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n5\n10 0 0 0\n20 1 0 0\n30 0 1 0\n40 0 0 1\n"
                 "50 1 1 1\n$EndNodes\n$Elements\n3\n1 2 2 0 0 10 20 30\n2 4 2 0 0 10 20 30 40\n"
                 "3 4 2 0 0 20 30 40 50\n$EndElements\n")
    X, T = msh.read_tet_msh(f)
    assert X.shape == (5, 3)
    np.testing.assert_array_equal(T, [[0, 1, 2, 3], [1, 2, 3, 4]])


@pytest.mark.skipif(not REF_MESHES or not os.path.isdir(REF_MESHES),
                    reason="SORS_REFERENCE_ROOT not set to a reference checkout")
def test_reference_demo_meshes():
    # the MSH 4.1 binary meshes that ship with the reference's demos
    for name in ("duck.msh", "sphere1.msh"):
        X, T = msh.read_tet_msh(os.path.join(REF_MESHES, name))
        assert T.shape[0] > 0 and T.min() >= 0 and T.max() < X.shape[0]
        a, b, c, d = (X[T[:, k]] for k in range(4))
        vol = np.einsum("ij,ij->i", b - a, np.cross(c - a, d - a)) / 6.0
        assert (np.abs(vol) > 0).all()
