"""Host-side checks of the device-solver settings (no GPU): the py_sors
mirror rejects unknown values before any handle is created, and the C struct
carries what it was given."""
import numpy as np
import pytest

from sors_b200 import meshes


def _energy(**fields):
    from sors_b200 import py_sors as ps
    X, T = meshes.cantilever_tets(2, 1, 1, (0.02, 0.01, 0.01))
    s = ps.SimulationSettings()
    s.meshType = "Tetrahedron"; s.dt = 1e-2
    for k, v in fields.items():
        setattr(s, k, v)
    ne = T.shape[0]
    params = [ps.Params(["density", "youngsModulus", "poissonsRatio"], [1000.0, 1e5, 0.45])] * ne
    return ps.Energy(X, T, s, np.zeros(3), 0.0, [{"neohookean"}] * ne, params, [], ps.Params(), [], ps.Params())


@pytest.mark.parametrize("field,value", [("linearSolver", "gmres"), ("pressureJacobian", "p7")])
def test_unknown_solver_settings_are_rejected(field, value):
    with pytest.raises(ValueError, match=field):
        _energy(**{field: value})


def test_default_settings_keep_the_reference_solver_choices():
    from sors_b200 import _lib
    s = _lib.default_settings()
    assert s.linear_solver == 0          # PCG
    assert s.pressure_jac_exact == 0     # the reference's p/6 quad coefficient
    assert s.project_spd == 2            # exact Hessian unless PCG meets negative curvature
