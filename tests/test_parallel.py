"""Rank sharding of the mesh (host logic) with world_size-2 gloo process groups on CPU.

The per-lane evaluator is the CPU oracle here; on GPUs it is ResponseEngine.integrate_mesh.
"""
import os
import socket

import numpy as np
import pytest

from wanniernlqg_b200 import _abi, parallel
from wanniernlqg_b200.model import reference_workload_model


def _task():
    return _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.BERRY_CURVATURE, ["xy"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.02, photon_energies=np.linspace(0, 3, 8))


def test_lane_ranges_match_reference_rule():
    # fld((L-1)*Nk, NL)+1 .. fld(L*Nk, NL) (1-based) == [(L*Nk)//NL, ((L+1)*Nk)//NL) 0-based
    for nk in (1, 7, 64, 65, 1000, 32768):
        lanes = parallel.lane_count(nk)
        covered = []
        for lane in range(lanes):
            a, b = parallel.lane_range(nk, lanes, lane)
            covered.extend(range(a, b))
        assert covered == list(range(nk))
    assert parallel.local_lanes(64, 1, 4) == list(range(1, 64, 4))


def _worker(rank, world, port, mesh, out_path):
    import torch.distributed as dist
    from oracle import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    model = reference_workload_model("nw4")
    task = _task()
    res = parallel.distributed_integrate_mesh(
        lambda a, b: oracle.integrate_mesh(model, task, mesh, a, b, threads=1), mesh, task.value_count())
    np.save(out_path + f".{rank}.npy", res)
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def test_two_rank_gloo_sharding_is_bitwise_identical(tmp_path, oracle_mod):
    import torch.multiprocessing as mp
    mesh = (5, 4, 4)
    out = str(tmp_path / "res")
    mp.start_processes(_worker, args=(2, _free_port(), mesh, out), nprocs=2, start_method="spawn", join=True)
    r0 = np.load(out + ".0.npy")
    r1 = np.load(out + ".1.npy")
    model = reference_workload_model("nw4")
    single = oracle_mod.integrate_mesh(model, _task(), mesh, threads=1)
    assert np.array_equal(r0, r1)
    assert np.array_equal(r0, single)


# ---- adaptive integration over ranks (integrate_response_mpi, ResponseIntegration.jl:200-387) ----

def _adaptive_setup():
    from wanniernlqg_b200 import integration
    model = reference_workload_model("nw4")
    task = _abi.TaskArrays([(_abi.BERRY_CURVATURE, ["xy"]), (_abi.QUANTUM_METRIC, ["xx"])])
    domain = integration.IntegrationDomain((0.0, 0.0, 0.0), (1.0, 1.0, 1.0))
    algorithm = integration.HAdaptiveCubature(atol=0.0, rtol=2e-3, max_evaluations=1500)
    return model, task, domain, algorithm


def _adaptive_worker(rank, world, port, mode, out_path):
    import pickle
    import torch.distributed as dist
    from oracle import oracle
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    model, task, domain, algorithm = _adaptive_setup()
    evaluated = []

    def evaluator(nodes):
        evaluated.append(len(nodes))
        if mode == "fail" and rank == 1 and np.any(nodes[:, 0] > 0.6):
            raise ValueError("planted failure")
        return oracle.point_values(model, task, nodes, threads=1)

    if mode == "contract" and rank == 1:
        from wanniernlqg_b200 import integration
        algorithm = integration.HAdaptiveCubature(atol=0.0, rtol=1e-3, max_evaluations=1500)
    try:
        # "chunked": a pending-packet limit of a few values, so every rule travels in several packets.
        limit = 2048 if mode == "chunked" else 1 << 30
        res = parallel.distributed_integrate_response(evaluator, domain, algorithm, batched=(mode == "batched"),
                                                      pending_memory_limit_bytes=limit)
        outcome = {"value": res.value, "evaluations": res.evaluations, "estimate": res.embedded_estimate,
                   "local_nodes": int(sum(evaluated))}
    except Exception as exc:   # noqa: BLE001 - recorded for the test
        outcome = {"error": f"{type(exc).__name__}: {exc}", "local_nodes": int(sum(evaluated))}
    with open(out_path + f".{rank}.pkl", "wb") as fh:
        pickle.dump(outcome, fh)
    dist.barrier()
    dist.destroy_process_group()


def _run_adaptive(tmp_path, world, mode):
    import pickle
    import torch.multiprocessing as mp
    out = str(tmp_path / f"adaptive_{mode}_{world}")
    mp.start_processes(_adaptive_worker, args=(world, _free_port(), mode, out), nprocs=world, start_method="spawn",
                       join=True)
    res = []
    for r in range(world):
        with open(out + f".{r}.pkl", "rb") as fh:
            res.append(pickle.load(fh))
    return res


@pytest.mark.parametrize("world,mode", [(2, "serial"), (3, "serial"), (2, "batched"), (2, "chunked")])
def test_adaptive_over_ranks_is_bitwise_the_single_rank_run(tmp_path, oracle_mod, world, mode):
    """Rank 0's controller sees the one-rank values in the one-rank order: value, estimate and
    evaluation count are identical to the single-process run, on every rank, and the rule nodes
    are shared out round-robin (every rank evaluates about 1/world of them)."""
    from wanniernlqg_b200 import integration
    model, task, domain, algorithm = _adaptive_setup()
    ev = lambda nodes: oracle_mod.point_values(model, task, nodes, threads=1)   # noqa: E731
    if mode == "batched":
        single = integration.integrate_response_batched(ev, domain, algorithm)
    else:
        single = integration.integrate_response(None, domain, algorithm, batch_evaluator=ev)
    res = _run_adaptive(tmp_path, world, mode)
    for r in res:
        assert "error" not in r, r
        assert np.array_equal(r["value"], single.value)
        assert r["evaluations"] == single.evaluations and r["estimate"] == single.embedded_estimate
    shares = [r["local_nodes"] for r in res]
    assert sum(shares) == single.evaluations
    if mode != "chunked":
        assert max(shares) - min(shares) <= len(res) * 40   # one rule (33 nodes) of imbalance per packet at most


def test_adaptive_over_ranks_reports_evaluator_failure_everywhere(tmp_path, oracle_mod):
    res = _run_adaptive(tmp_path, 2, "fail")
    for r in res:
        assert "error" in r and "rank 1: ValueError: planted failure" in r["error"], r


def test_adaptive_over_ranks_refuses_different_contracts(tmp_path, oracle_mod):
    res = _run_adaptive(tmp_path, 2, "contract")
    for r in res:
        assert "error" in r and "different global contracts" in r["error"], r
        assert r["local_nodes"] == 0
