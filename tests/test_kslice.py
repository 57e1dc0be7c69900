"""K-slice geometry and writer (CalculationUtils.jl:295-392, ResultWriters.jl:91-121), with the
oracle as the per-point evaluator."""
import numpy as np
import pytest

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.kslice import kslice_indices, kslice_map, make_kslice_grid, make_kslice_points, write_kslice
from wanniernlqg_b200.model import reference_workload_model


def test_kslice_points_order_and_half_open():
    pts, coords, nu, nv = make_kslice_points([4, 3, 7], [1, 2], [0.1, 0.0, 0.5], [1.0, 0.0, 0.0], [0.0, 0.5, 0.0])
    assert (nu, nv) == (4, 3) and pts.shape == (12, 3)
    assert np.allclose(pts[1], [0.35, 0.0, 0.5]) and np.allclose(pts[4], [0.1, 0.5 / 3, 0.5])
    assert tuple(coords[5]) == (2, 2)
    grid, _, _ = make_kslice_grid([4, 3, 7], [1, 2], [0, 0, 0], [1, 0, 0], [0, 1, 0])
    assert kslice_indices(grid, 6) == (2, 2)
    with pytest.raises(IndexError):
        kslice_indices(grid, 13)


def test_kslice_map_and_writer(oracle_mod, tmp_path):
    model = reference_workload_model("nw4")
    task = _abi.TaskArrays([(_abi.QUANTUM_METRIC, ["xx"])])
    data = kslice_map(lambda k: oracle_mod.point_values(model, task, k), [5, 3], [0, 0, 0.25], [1, 0, 0], [0, 1, 0])
    assert data.shape == (5, 3)
    ref = oracle_mod.point_values(model, task, [[2 / 5, 1 / 3, 0.25]])[0, 0].real
    assert data[2, 1] == ref
    path = write_kslice(data, [5, 3], str(tmp_path / "out"), "metric_xx.dat")
    back = np.loadtxt(path)
    assert np.array_equal(back, data)
    with pytest.raises(ValueError):
        write_kslice(data.T, [5, 3], str(tmp_path), "bad.dat")
