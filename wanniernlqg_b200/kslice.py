"""K-slice maps: per-k responses on a planar half-open grid and their text output.

Mirrors the reference's slice geometry and writer:
  KSliceGrid2D, kslice_indices, kslice_kpoint!, make_kslice_grid, make_kslice_points
      (src/Core/CalculationUtils.jl:295-392)
  kslice_output_size, write_kslice (src/IO/ResultWriters.jl:91-121)
The values come from the engine's batched point evaluation (wnlqg_b200_eval_points), one device
call for the whole slice.
"""
from __future__ import annotations

import dataclasses
import os
from typing import Callable, Sequence

import numpy as np


@dataclasses.dataclass
class KSliceGrid2D:
    """Sample counts, fractional reciprocal origin and two spanning vectors of a half-open planar
    mesh; u varies fastest and both coordinates exclude their upper endpoint."""
    num_u_points: int
    num_v_points: int
    origin: np.ndarray
    vector_1: np.ndarray
    vector_2: np.ndarray

    def __len__(self) -> int:
        return self.num_u_points * self.num_v_points


def kslice_indices(grid: KSliceGrid2D, kpoint_index: int):
    """One-based (u_index, v_index) of a one-based linear index, u fastest."""
    if not 1 <= kpoint_index <= len(grid):
        raise IndexError(f"k-slice index {kpoint_index} outside 1:{len(grid)}")
    ik0 = kpoint_index - 1
    return ik0 % grid.num_u_points + 1, ik0 // grid.num_u_points + 1


def make_kslice_grid(k_mesh: Sequence[int], active_axes: Sequence[int], origin, vector_1, vector_2):
    """(grid, num_u_points, num_v_points) with the counts taken from k_mesh at the two active
    axes (one-based, as in the reference)."""
    nu, nv = int(k_mesh[active_axes[0] - 1]), int(k_mesh[active_axes[1] - 1])
    grid = KSliceGrid2D(nu, nv, np.array(origin, dtype=np.float64), np.array(vector_1, dtype=np.float64),
                        np.array(vector_2, dtype=np.float64))
    return grid, nu, nv


def make_kslice_points(k_mesh: Sequence[int], active_axes: Sequence[int], origin, vector_1, vector_2):
    """(points [n, 3] fractional, coordinates [n, 2] one-based (u, v), nu, nv) in u-fastest order:
    k = origin + (u-1)/nu * vector_1 + (v-1)/nv * vector_2."""
    grid, nu, nv = make_kslice_grid(k_mesh, active_axes, origin, vector_1, vector_2)
    idx = np.arange(nu * nv)
    ui, vi = idx % nu, idx // nu
    points = grid.origin[None, :] + (ui / nu)[:, None] * grid.vector_1[None, :] + (vi / nv)[:, None] * grid.vector_2[None, :]
    coords = np.stack([ui + 1, vi + 1], axis=1)
    return points, coords, nu, nv


def kslice_map(point_values: Callable, k_mesh: Sequence[int], origin, vector_1, vector_2, *,
               active_axes: Sequence[int] = (1, 2), value: int = 0, part: str = "real") -> np.ndarray:
    """data[u, v] (shape (nu, nv)) of one value of `point_values(points) -> [n, value_count]`
    (for example ResponseEngine.point_values) on the slice."""
    points, _, nu, nv = make_kslice_points(k_mesh, active_axes, origin, vector_1, vector_2)
    vals = np.asarray(point_values(points))[:, value]
    vals = vals.real if part == "real" else vals.imag
    return vals.reshape(nv, nu).T.copy()


def kslice_output_size(k_mesh: Sequence[int]):
    if len(k_mesh) != 2:
        raise ValueError(f"k-resolved output expects k_mesh with length 2, got length={len(k_mesh)}")
    return int(k_mesh[0]), int(k_mesh[1])


def write_kslice(data: np.ndarray, k_mesh: Sequence[int], directory: str, filename: str) -> str:
    """One text row per first index, values space-separated (shortest round-trip decimals), no
    unit conversion; the shape must equal the two mesh counts.  Returns the path."""
    expected = kslice_output_size(k_mesh)
    if data.shape != expected:
        raise ValueError(f"Dimension mismatch: data has size {data.shape}, expected {expected}.")
    os.makedirs(directory, exist_ok=True)
    path = os.path.join(directory, filename)
    with open(path, "w") as fh:
        for row in data:
            fh.write(" ".join(repr(float(x)) for x in row) + "\n")
    return path
