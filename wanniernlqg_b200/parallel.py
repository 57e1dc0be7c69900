"""Deterministic work sharing over ranks (one process per GPU).

Uniform meshes mirror the reference's lane scheme: min(Nk, 64) contiguous lanes
(_deterministic_integral_lane_range, Runtime/Setup/BundleAssembly.jl:35-48), lane L owned by
rank L mod size (_local_deterministic_integral_lanes, :51-53), lanes reduced in lane order
(_reduce_integral_states!, Runtime/Reduction/DeterministicReduction.jl:2-38).  Every rank
evaluates only its own lanes (no data-path collective); one all-reduce of the zero-padded
[lanes, values] tensor then gives every rank all lane tensors exactly (x + 0 = x), and the
lane-ordered sum makes the result bit-identical for any number of ranks.

Adaptive integration mirrors integrate_response_mpi (Runtime/Execution/ResponseIntegration.jl:
200-387): rank 0 alone runs the unchanged controller (heap, error estimate, budget); each batch
of rule nodes it asks for is broadcast, node i of the run's global sequence is evaluated by rank
i mod size (one batched evaluator call per rank and packet), the values are gathered back to
rank 0 and handed to the controller in the original order, so the controller's arithmetic is
the one-rank arithmetic.  A collective preflight first checks that every rank holds a valid and
identical contract; an evaluator failure on any rank ends the run on every rank with the
failing ranks' messages.
"""
from __future__ import annotations

from typing import Callable, List, Optional, Sequence, Tuple

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


def _world(group):
    import torch.distributed as dist
    if dist.is_available() and dist.is_initialized():
        return dist.get_rank(group), dist.get_world_size(group)
    return 0, 1


def _contract(domain, algorithm, normalization, batched, boxes_per_step, pending_memory_limit_bytes):
    """This rank's view of the global contract, validated (the preflight packet)."""
    from . import integration
    try:
        if not isinstance(algorithm, integration.HAdaptiveCubature):
            raise TypeError("distributed adaptive integration requires HAdaptiveCubature")
        if not (isinstance(pending_memory_limit_bytes, int) and pending_memory_limit_bytes > 0):
            raise ValueError("positive adaptive pending-memory limit required")
        integration.validate_integration_budget(domain, algorithm)
        integration._normalization(domain, normalization)
        value = (domain.lower, domain.upper, domain.coordinates, algorithm.atol, algorithm.rtol,
                 algorithm.max_evaluations, algorithm.initial_divisions, normalization, bool(batched),
                 int(boxes_per_step), pending_memory_limit_bytes)
        return {"ok": True, "value": value, "error": ""}
    except Exception as exc:   # noqa: BLE001 - every rank must reach the collective
        return {"ok": False, "value": None, "error": f"{type(exc).__name__}: {exc}"}


def distributed_integrate_response(batch_evaluator: Callable[[np.ndarray], np.ndarray], domain, algorithm, *,
                                   normalization: str = "domain_average", batched: bool = False,
                                   boxes_per_step: int = 256, group=None,
                                   pending_memory_limit_bytes: int = 1 << 30):
    """Adaptive integral over the ranks of `group` (torch.distributed, gloo or NCCL object
    collectives); every rank calls it with the same contract and its own evaluator (normally its
    GPU's ResponseEngine.point_values) and every rank returns the same ResponseIntegralResult.

    batched=False runs the serial HCubature controller (integration.integrate_response),
    batched=True the GPU-oriented integrate_response_batched (boxes_per_step boxes per step).
    A packet holds at most as many nodes as pending_memory_limit_bytes admits at four times the
    first value's size (the reference's bounded pending packet)."""
    import torch.distributed as dist
    from . import integration
    rank, size = _world(group)
    local = _contract(domain, algorithm, normalization, batched, boxes_per_step, pending_memory_limit_bytes)
    if size == 1:
        if not local["ok"]:
            raise ValueError(local["error"])
        return _run_controller(batch_evaluator, domain, algorithm, normalization, batched, boxes_per_step)
    contracts = [None] * size
    dist.all_gather_object(contracts, local, group=group)
    failed = [f"rank {r}: {c['error']}" for r, c in enumerate(contracts) if not c["ok"]]
    if failed:
        raise ValueError("adaptive collective preflight failed: " + "; ".join(failed))
    if any(c["value"] != contracts[0]["value"] for c in contracts):
        raise ValueError("adaptive ranks supplied different global contracts")
    src = _global_rank(group, 0)

    def evaluate_packet(command):
        nodes = command["nodes"]
        owned = [i for i in range(len(nodes)) if (command["first_sequence"] + i) % size == rank]
        packet = {"ok": True, "rank": rank, "ordinals": owned, "values": None, "error": ""}
        if owned:
            try:
                vals = np.asarray(batch_evaluator(np.asarray(nodes)[owned]), dtype=np.complex128)
                if vals.shape[0] != len(owned):
                    raise ValueError("incomplete cubature node batch")
                packet["values"] = vals
            except Exception as exc:   # noqa: BLE001 - reported through the gather
                packet.update(ok=False, values=None, error=f"{type(exc).__name__}: {exc}")
        gathered = [None] * size if rank == 0 else None
        dist.gather_object(packet, gathered, dst=src, group=group)
        return gathered

    if rank == 0:
        state = {"sequence": 0, "value_bytes": 0}

        def distributed_batch(nodes):
            nodes = np.asarray(nodes, dtype=np.float64)
            out = None
            first = 0
            while first < len(nodes):
                if state["value_bytes"] == 0:
                    capacity = 1
                else:
                    capacity = pending_memory_limit_bytes // state["value_bytes"]
                    if capacity <= 0:
                        raise ValueError("adaptive node result exceeds pending-memory limit")
                last = min(len(nodes), first + capacity)
                command = {"operation": "evaluate_batch", "nodes": nodes[first:last],
                           "first_sequence": state["sequence"]}
                dist.broadcast_object_list([command], src=src, group=group)
                packets = evaluate_packet(command)
                failures = [p for p in packets if not p["ok"]]
                if failures:
                    raise RuntimeError("adaptive evaluator failed: " +
                                       "; ".join(f"rank {p['rank']}: {p['error']}" for p in failures))
                seen = np.zeros(last - first, dtype=bool)
                chunk = None
                for p in packets:
                    if not p["ordinals"]:
                        continue
                    if chunk is None:
                        chunk = np.zeros((last - first,) + p["values"].shape[1:], dtype=np.complex128)
                    for j, o in enumerate(p["ordinals"]):
                        if seen[o]:
                            raise RuntimeError("adaptive node ownership mismatch")
                        chunk[o] = p["values"][j]
                        seen[o] = True
                if not seen.all():
                    raise RuntimeError("incomplete adaptive node values")
                state["sequence"] += last - first
                if state["value_bytes"] == 0:
                    state["value_bytes"] = 4 * chunk[0].nbytes
                out = chunk if out is None else np.concatenate([out, chunk])
                first = last
            return out

        try:
            result = _run_controller(distributed_batch, domain, algorithm, normalization, batched, boxes_per_step)
            terminal = {"operation": "finish", "ok": True, "value": result, "error": ""}
        except Exception as exc:   # noqa: BLE001 - broadcast to every rank
            terminal = {"operation": "finish", "ok": False, "value": None, "error": f"{type(exc).__name__}: {exc}"}
        dist.broadcast_object_list([terminal], src=src, group=group)
    else:
        while True:
            box = [None]
            dist.broadcast_object_list(box, src=src, group=group)
            command = box[0]
            if command["operation"] == "finish":
                terminal = command
                break
            if command["operation"] != "evaluate_batch":
                raise RuntimeError("invalid adaptive operation")
            evaluate_packet(command)
    if not terminal["ok"]:
        raise RuntimeError(terminal["error"])
    return terminal["value"]


def _global_rank(group, group_rank: int) -> int:
    import torch.distributed as dist
    if group is None:
        return group_rank
    return dist.get_global_rank(group, group_rank)


def _run_controller(batch_evaluator, domain, algorithm, normalization, batched, boxes_per_step):
    from . import integration
    if batched:
        return integration.integrate_response_batched(batch_evaluator, domain, algorithm,
                                                      normalization=normalization, boxes_per_step=boxes_per_step)
    return integration.integrate_response(None, domain, algorithm, normalization=normalization,
                                          batch_evaluator=batch_evaluator)
