"""Extract the known-answer fixtures of the SORS reference tests into JSON.

Reads cpp/src/_test.cpp and cpp/headers/_test.h of the reference *as text*
(the reference cannot be compiled here: its Eigen submodule is empty) and
writes tests/golden/reference_known_answers.json.  Every literal below is
parsed from the reference source, and the scalar settings of each test are
recorded with the line they come from.

Run from the repository root:
    python tests/golden/extract_reference_fixtures.py [REFERENCE_ROOT]
"""
from __future__ import annotations

import json
import os
import re
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def _numbers_after(text: str, anchor: str, count: int, start: int = 0) -> tuple[list[float], int]:
    """Return the first `count` numeric literals after `anchor` (and after `start`)."""
    pos = text.index(anchor, start) + len(anchor)
    nums: list[float] = []
    for m in re.finditer(r"-?\d+(?:\.\d*)?(?:[eE][-+]?\d+)?", text[pos:]):
        nums.append(float(m.group(0)))
        if len(nums) == count:
            return nums, pos + m.end()
    raise ValueError(f"not enough numbers after {anchor!r}")


def _line_of(text: str, anchor: str, start: int = 0) -> int:
    return text.count("\n", 0, text.index(anchor, start)) + 1


def extract(ref_root: str) -> dict:
    path = os.path.join(ref_root, "cpp", "src", "_test.cpp")
    hpath = os.path.join(ref_root, "cpp", "headers", "_test.h")
    # line comments are blanked (newlines kept, so line numbers stay valid)
    text = re.sub(r"//[^\n]*", "", open(path).read())
    htext = open(hpath).read()
    out: dict = {"source": "cpp/src/_test.cpp (SORS reference tests), parsed as text"}

    # --- TestEnergy: 5-vertex, 2-tet mesh with the quartic mock element ----
    v, _ = _numbers_after(text, "vertices_ <<", 15)
    e, _ = _numbers_after(text, "eleIdx_ <<", 8)
    g, _ = _numbers_after(text, "gradGT <<", 15)
    h, _ = _numbers_after(text, "hessDiagGT <<", 15)
    out["test_energy"] = {
        "vertices": [v[i:i + 3] for i in range(0, 15, 3)],
        "elements": [[int(x) for x in e[i:i + 4]] for i in range(0, 8, 4)],
        "energy": 3.0,  # `return (energy == 3)`
        "energy_line": _line_of(text, "return (energy == 3)"),
        "gradient": [g[i:i + 3] for i in range(0, 15, 3)],
        "gradient_line": _line_of(text, "gradGT <<"),
        "hessian_diag": [h[i:i + 3] for i in range(0, 15, 3)],
        "hessian_line": _line_of(text, "hessDiagGT <<"),
        "dt": 0.0,
        "gravity": [0.0, 0.0, 0.0],
        "optimization_dt": 1.0,  # solver.minimize_newton(..., 1.0, ...)
        "optimization_line": _line_of(text, "solver.minimize_newton(reshapedVertices, systemEnergy_, 1.0"),
        "tol": 1e-9,
    }

    # --- TestTetrahedron: unit tet, exact 9x12 dF/dx, zero energy at rest ----
    und, p = _numbers_after(text, "undeformedVertices_ <<", 12)
    cur, _ = _numbers_after(text, "currentVertices_ <<", 12, p)
    dh, _ = _numbers_after(text, "deformationHessianCalc <<", 108)
    tol_tet = float(re.search(r"class TestTetrahedron[\s\S]*?TOL = ([0-9.eE-]+)", htext).group(1))
    out["test_tetrahedron"] = {
        "undeformed": [und[i:i + 3] for i in range(0, 12, 3)],
        "current": [cur[i:i + 3] for i in range(0, 12, 3)],
        "dFdx": [dh[i:i + 12] for i in range(0, 108, 12)],
        "dFdx_line": _line_of(text, "deformationHessianCalc <<"),
        "material": {"density": 1.0, "youngsModulus": 1.0, "poissonsRatio": 0.3},
        "tol": tol_tet,
    }

    # --- TestCube: unit cube as 5 tets ------------------------------------
    cv, _ = _numbers_after(text, "vertices_ = (MatrixXd(8, 3) <<", 24)
    ce, _ = _numbers_after(text, "elements_ = (MatrixXi(5, 4) <<", 20)
    tol_cube = float(re.search(r"class TestCube[\s\S]*?TOL = ([0-9.eE-]+)", htext).group(1))
    dt_cube = float(re.search(r"TestCube::TestCube\(\) : dt_\(([0-9.eE-]+)\)", text).group(1))
    out["test_cube"] = {
        "vertices": [cv[i:i + 3] for i in range(0, 24, 3)],
        "elements": [[int(x) for x in ce[i:i + 4]] for i in range(0, 20, 4)],
        "dt": dt_cube,
        "tol": tol_cube,
        "expected_acceleration": -10.0,
        "gravity_test": {"density": 1.0, "youngsModulus": 500000.0, "poissonsRatio": 0.4,
                         "gravity": [0.0, 0.0, -10.0], "line": _line_of(text, "bool TestCube::test_gravity_force")},
        "pressure_test": {"density": 1.0, "youngsModulus": 500000.0, "poissonsRatio": 0.4, "pressure": 10.0,
                          "faces": [[1, 5, 6], [1, 6, 2]], "groups": [0, 0],
                          "line": _line_of(text, "bool TestCube::test_pressure_force")},
        "vertex_force_test": {"density": 1.0, "youngsModulus": 500000.0, "poissonsRatio": 0.4,
                              "force_per_vertex_z": -10.0 / 8,
                              "line": _line_of(text, "bool TestCube::test_external_force")},
        "energy_min_test": {"density": 1000.0, "youngsModulus": 250000.0, "poissonsRatio": 0.4,
                            "gravity": [0.0, 0.0, -9.81], "max_pressure": 1000.0, "num_steps": 10,
                            "faces": [[1, 5, 6], [1, 6, 2]], "groups": [0, 0],
                            # the reference writes the mask at DOFs 3*i for i in 0..3 (not the vertex ids)
                            "masked_vertices": [0, 1, 2, 3],
                            "line": _line_of(text, "bool TestCube::test_energy_min")},
        "num_steps": 10,
    }

    # --- TestConstraint: penetrating tet vs plane z=0 ----------------------
    cstart = text.index("bool TestConstraint::test_plane_contact_no_penetration")
    pv, _ = _numbers_after(text, "vertices <<", 12, cstart)
    out["test_constraint"] = {
        "vertices": [pv[i:i + 3] for i in range(0, 12, 3)],
        "tol": float(re.search(r"class TestConstraint[\s\S]*?TOL = ([0-9.eE-]+)", htext).group(1)),
        "line": _line_of(text, "bool TestConstraint::test_plane_contact_no_penetration"),
    }
    return out


def main() -> None:
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("SORS_REFERENCE_ROOT")
    if not ref:
        sys.exit("usage: extract_reference_fixtures.py <reference project root> "
                 "(or set SORS_REFERENCE_ROOT)")
    data = extract(ref)
    dst = os.path.join(HERE, "reference_known_answers.json")
    with open(dst, "w") as f:
        json.dump(data, f, indent=1)
    print("wrote", dst)


if __name__ == "__main__":
    main()
