"""CPU checks of the C ABI library and the host-side API (no GPU needed)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            names |= set(re.findall(r"^\w[\w\s\*]*?\b(sors_\w+)\(", src, re.M))
    return names


def test_library_exports_every_declared_symbol():
    from sors_b200 import _lib
    L = _lib.load()
    declared = _declared()
    assert declared, "no declarations found"
    assert all(hasattr(L, n) for n in declared), sorted(n for n in declared if not hasattr(L, n))
    bound = {n for n, _, _ in _lib.SIGNATURES}
    assert declared == bound


def test_default_settings_match_reference_constants():
    from sors_b200 import _lib
    s = _lib.default_settings()
    assert s.newton_dx_tol == 1e-9        # cpp/headers/common.h:25
    assert s.newton_max_iter == 100       # cpp/headers/common.h:21
    assert s.time_stepping == 1           # SimulationSettings default "crank_nicolson"
    assert s.substeps == 1


def test_struct_layout_matches_header():
    from sors_b200 import _lib
    # the C struct is naturally aligned: check the ctypes size against a gcc-compiled probe
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "sors_b200.h"
int main(void){printf("%zu %zu %zu %zu\n", sizeof(SorsSettings), offsetof(SorsSettings, device),
 sizeof(SorsStepStats), offsetof(SorsStepStats, dx_norm));return 0;}
'''
    import subprocess
    import tempfile
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "probe.c")
        open(p, "w").write(src)
        exe = os.path.join(d, "probe")
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), p, "-o", exe], check=True,
                       env={k: v for k, v in os.environ.items() if k not in ("CC",)})
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    assert int(out[0]) == C.sizeof(_lib.SorsSettings)
    assert int(out[1]) == _lib.SorsSettings.device.offset
    assert int(out[2]) == C.sizeof(_lib.SorsStepStats)
    assert int(out[3]) == _lib.SorsStepStats.dx_norm.offset


def test_params_semantics(tmp_path):
    from sors_b200.py_sors import Params
    p = Params(["density", "youngsModulus"], [1000.0, 2e5])
    assert p.get_value("density").shape == (1, 1)
    p.set_param("v", [1.0, 2.0, 3.0])
    assert p.get_value("v").shape == (3, 1)
    with pytest.raises(ValueError):
        p.set_param("v", [1.0, 2.0])
    with pytest.raises(KeyError):
        p.get_value("missing")
    f = tmp_path / "p.csv"
    f.write_text("density,1070\nsoftconDirection,0,0,1\n")
    q = Params(); q.set_param(str(f))
    assert q.get_value("density")[0, 0] == 1070
    assert q.get_value("softconDirection").ravel().tolist() == [0, 0, 1]


def test_unknown_mesh_type_raises():
    from sors_b200 import py_sors as ps
    s = ps.SimulationSettings(); s.meshType = "Prism"
    with pytest.raises(RuntimeError, match="Unknown mesh type"):
        ps.Solver(s)
    with pytest.raises(RuntimeError, match="Unknown mesh type"):
        ps.Energy(np.zeros((4, 3)), np.zeros((1, 4)), s, np.zeros(3))


def test_hex_to_5_tets_and_surfaces():
    from sors_b200 import meshes
    from sors_b200.py_sors import IO
    X, H = meshes.hex_bar(2, 1, 1, (2.0, 1.0, 1.0))
    T = IO.hex_to_5_tets(H)
    assert T.shape == (10, 4)
    groups, fe = IO.extract_hex_surfaces(X, H)
    assert len(groups) == 1 and groups[0].shape == (10, 4)
    # outward normals: (b-a)x(c-a) points away from the element
    for f, e in zip(groups[0], fe[0]):
        a, b, c = X[f[0]], X[f[1]], X[f[2]]
        n = np.cross(b - a, c - a)
        assert n @ (X[H[e]].mean(0) - a) < 0
    Xt, Tt = meshes.cantilever_tets(2, 1, 1, (2.0, 1.0, 1.0))
    gt, _ = IO.extract_tet_surfaces(Xt, Tt)
    assert sum(len(g) for g in gt) == 2 * 10  # 10 boundary quads, 2 triangles each


def test_kuhn_mesh_is_conforming():
    from sors_b200 import meshes
    X, T = meshes.cantilever_tets(3, 2, 2, (3.0, 2.0, 2.0))
    assert T.shape[0] == 6 * 12
    # every interior face is shared by exactly two tets, boundary faces by one
    f = np.sort(T[:, [[0, 1, 2], [0, 1, 3], [0, 2, 3], [1, 2, 3]]].reshape(-1, 3), 1)
    _, c = np.unique(f, axis=0, return_counts=True)
    assert set(c.tolist()) <= {1, 2}
    vol = np.abs(np.einsum("ij,ij->i", X[T[:, 1]] - X[T[:, 0]],
                           np.cross(X[T[:, 2]] - X[T[:, 0]], X[T[:, 3]] - X[T[:, 0]]))) / 6
    assert abs(vol.sum() - 12.0) < 1e-12
