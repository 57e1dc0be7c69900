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
