"""Store one of the reference's demo meshes as a compact test fixture.

Reads cpp/demos/meshes/pokeflexFoamDice/T1P2_mesh.msh (the PokeFlex foam dice
that python/d03_pokeflex.py pokes; Gmsh MSH 4.1 binary) of a reference checkout
with this package's MSH reader (sors_b200.msh, the counterpart of
IO::read_tet_MSH, cpp/src/io.cpp:380-471) and writes the vertices (as read,
in millimetres) and the 0-based tets to tests/golden/pokeflex_T1P2_mesh.npz,
with the SHA-256 of the source file.  The GPU tests load the .npz, so they need
no reference checkout.

Run from the repository root:
    python tests/golden/make_mesh_fixture.py <REFERENCE_ROOT>
(or set SORS_REFERENCE_ROOT).
"""
from __future__ import annotations

import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

REL = os.path.join("cpp", "demos", "meshes", "pokeflexFoamDice", "T1P2_mesh.msh")
OUT = os.path.join(HERE, "pokeflex_T1P2_mesh.npz")


def main() -> None:
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SORS_REFERENCE_ROOT")
    if not ref:
        sys.exit("usage: make_mesh_fixture.py <reference project root> (or set SORS_REFERENCE_ROOT)")
    from sors_b200 import msh
    src = os.path.join(ref, REL)
    X, T = msh.read_tet_msh(src)
    digest = hashlib.sha256(open(src, "rb").read()).hexdigest()
    np.savez_compressed(OUT, vertices=np.asarray(X, np.float64), tets=np.asarray(T, np.int32),
                        source=np.array(REL), sha256=np.array(digest))
    print(f"wrote {OUT}: {X.shape[0]} vertices, {T.shape[0]} tets, source sha256 {digest}")


if __name__ == "__main__":
    main()
