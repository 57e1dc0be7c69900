"""Symmetry-reduced meshes on the GPU: the representatives' weighted device sum, projected onto
the group-invariant tensors, equals the oracle's full-mesh sum (FP64 bar, 1e-10 relative) and
the engine's own full-mesh sum."""
import itertools

import numpy as np
import pytest

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import synthetic_orthogonal_model
from wanniernlqg_b200.symmetry import SymmetryOperation, kmesh_orbits, symmetrize_model, tetrahedral_group

pytestmark = pytest.mark.gpu
ALL27 = ["".join(c) for c in itertools.product("xyz", repeat=3)]


@pytest.fixture(scope="module")
def engine_cls():
    from wanniernlqg_b200 import build
    build.build()
    from wanniernlqg_b200.engine import ResponseEngine
    return ResponseEngine


def rel_err(got, ref):
    return np.max(np.abs(got - ref)) / np.max(np.abs(ref))


@pytest.mark.parametrize("group,mesh,nw", [("td", (8, 8, 8), 8), ("grey_mm2", (8, 6, 4), 6)])
def test_reduced_mesh_matches_oracle_full_mesh(engine_cls, oracle_mod, group, mesh, nw):
    if group == "td":
        ops = [SymmetryOperation.from_fractional(W) for W in tetrahedral_group()]
    else:
        mm2 = [np.diag(d) for d in ([1, 1, 1], [-1, -1, 1], [-1, 1, 1], [1, -1, 1])]
        ops = [SymmetryOperation.from_fractional(W, antiunitary=a) for W in mm2 for a in (False, True)]
    model = symmetrize_model(synthetic_orthogonal_model(nw, 2, seed=7, full_position=True), ops)
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ALL27), (_abi.INJECTION_CURRENT, ALL27)],
                           broadening_type=_abi.LORENTZIAN, broadening=0.03, photon_energies=np.linspace(0.05, 3, 40))
    orbits = kmesh_orbits(mesh, ops)
    assert len(orbits.representatives) < np.prod(mesh) // 3
    with engine_cls(model, task) as eng:
        red = eng.integrate_mesh_reduced(mesh, ops, orbits=orbits)
        full_gpu = eng.integrate_mesh(mesh)
    full = oracle_mod.integrate_mesh(model, task, mesh)
    for r, g, f in zip(task.split(red), task.split(full_gpu), task.split(full)):
        assert rel_err(r, f) < 1e-10
        assert rel_err(g, f) < 1e-10
