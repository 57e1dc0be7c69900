"""Deterministic sharding of a k-mesh over ranks (one process per GPU).

Mirrors the reference's lane scheme: min(Nk, 64) contiguous lanes
(_deterministic_integral_lane_range, Runtime/Setup/BundleAssembly.jl:35-48), lane L owned by
rank L mod size (_local_deterministic_integral_lanes, :51-53), lanes reduced in lane order
(_reduce_integral_states!, Runtime/Reduction/DeterministicReduction.jl:2-38).  Every rank
evaluates only its own lanes (no data-path collective); one all-reduce of the zero-padded
[lanes, values] tensor then gives every rank all lane tensors exactly (x + 0 = x), and the
lane-ordered sum makes the result bit-identical for any number of ranks.
"""
from __future__ import annotations

from typing import Callable, List, Sequence, Tuple

import numpy as np

LANE_LIMIT = 64


def lane_count(nk: int) -> int:
    return min(nk, LANE_LIMIT)


def lane_range(nk: int, lanes: int, lane: int) -> Tuple[int, int]:
    """0-based half-open [first, last) of lane `lane` (0-based)."""
    if not 0 <= lane < lanes:
        raise IndexError(lane)
    return (lane * nk) // lanes, ((lane + 1) * nk) // lanes


def local_lanes(lanes: int, rank: int, size: int) -> List[int]:
    return list(range(rank, lanes, size))


def distributed_integrate_mesh(evaluate_range: Callable[[int, int], np.ndarray], mesh: Sequence[int],
                               value_count: int, group=None, device=None) -> np.ndarray:
    """Lane-deterministic mesh integral over the ranks of `group` (torch.distributed).

    evaluate_range(first, last) returns sum_{k in [first,last)} value(k)/Nk (complex
    [value_count]); it is called once per lane this rank owns.
    """
    import torch
    import torch.distributed as dist
    nk = int(np.prod(mesh))
    lanes = lane_count(nk)
    if dist.is_available() and dist.is_initialized():
        rank, size = dist.get_rank(group), dist.get_world_size(group)
    else:
        rank, size = 0, 1
    buf = np.zeros((lanes, value_count), dtype=np.complex128)
    for lane in local_lanes(lanes, rank, size):
        first, last = lane_range(nk, lanes, lane)
        buf[lane] = evaluate_range(first, last)
    if size > 1:
        t = torch.from_numpy(buf.view(np.float64).copy())
        if device is not None:
            t = t.to(device)
        dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
        buf = t.cpu().numpy().view(np.complex128)
    out = np.zeros(value_count, dtype=np.complex128)
    for lane in range(lanes):
        out += buf[lane]
    return out
