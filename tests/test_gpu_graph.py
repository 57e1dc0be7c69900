"""CUDA graphs of whole calls and the autotuner, through the C ABI.

A graph replays exactly the launches of the call it captured, so its results are bitwise those of
the direct call; refilled device inputs give the direct call's results for the new inputs.  The
autotuner only chooses among configurations the library runs anyway: results after tuning agree
with those before to the FP64 path's 1e-11 (the team size can change the last bits of the
eigensolve; the contraction tile cannot change any bit).
"""
import numpy as np
import pytest

from wanniernlqg_b200 import _abi, _lib
from wanniernlqg_b200.model import kramers_doubled_model, reference_workload_model, synthetic_orthogonal_model

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch_and_engine():
    from wanniernlqg_b200 import build
    build.build()
    import torch
    from wanniernlqg_b200 import engine
    return torch, engine


def _task(nom=64, **kw):
    return _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.BERRY_CURVATURE, ["xy"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.02,
                           photon_energies=np.linspace(0, 3, nom), **kw)


def test_mesh_many_graph_replays_the_direct_call(torch_and_engine):
    torch, eng = torch_and_engine
    models = [synthetic_orthogonal_model(nw, 1, seed=40 + nw, full_position=True) for nw in (6, 12, 32)]
    models.append(kramers_doubled_model(models[0], 1e-3, seed=3))
    engines = [eng.ResponseEngine(m, _task(), max_batch=2048) for m in models]
    try:
        meshes = [(8, 8, 8), (10, 6, 4), (12, 12, 12), (6, 6, 6)]
        ranges = [(0, 512), (17, 240), (0, 1728), (5, 216)]
        direct = [torch.zeros(2 * e.value_count, dtype=torch.float64, device="cuda") for e in engines]
        graphed = [torch.zeros_like(d) for d in direct]
        stream = torch.cuda.current_stream().cuda_stream
        eng.integrate_meshes_many(engines, meshes, ranges, [d.data_ptr() for d in direct], stream)
        torch.cuda.synchronize()
        with eng.CapturedGraph.mesh_many(engines, meshes, ranges, [g.data_ptr() for g in graphed]) as graph:
            assert graph.kernel_count >= 4 * len(engines)
            for _ in range(2):
                for g in graphed:
                    g.zero_()
                graph.launch(stream)
                torch.cuda.synchronize()
                graph.status()
                for d, g in zip(direct, graphed):
                    assert torch.equal(d, g)
            # A plan held by a graph is not destroyed (its model stays alive with it).
            with pytest.raises(_lib.EngineError):
                engines[0].close()
            # A direct call that outgrows the staged buffers retires them; the graph still replays.
            big = torch.zeros_like(direct[2])
            engines[2].integrate_mesh_device((4, 4, 128), 0, 2048, big.data_ptr(), stream)
            graph.launch(stream)
            torch.cuda.synchronize()
            for d, g in zip(direct, graphed):
                assert torch.equal(d, g)
    finally:
        for e in engines:
            e.close()


def test_points_graph_refills_and_pads(torch_and_engine):
    torch, eng = torch_and_engine
    model = reference_workload_model("nw4")
    rng = np.random.default_rng(21)
    n = 96
    with eng.ResponseEngine(model, _task()) as e:
        k_dev = torch.zeros((n, 3), dtype=torch.float64, device="cuda")
        w_dev = torch.zeros(n, dtype=torch.float64, device="cuda")
        out = torch.zeros(2 * e.value_count, dtype=torch.float64, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        with eng.CapturedGraph.points_weighted(e, k_dev.data_ptr(), w_dev.data_ptr(), n, out.data_ptr()) as graph:
            for trial in range(3):
                k = rng.random((n, 3))
                w = rng.random(n)
                if trial == 2:
                    w[70:] = 0.0   # an uneven cell padded to the captured count
                k_dev.copy_(torch.from_numpy(k))
                w_dev.copy_(torch.from_numpy(w))
                graph.launch(stream)
                torch.cuda.synchronize()
                graph.status()
                got = out.cpu().numpy().view(np.complex128)
                m = 70 if trial == 2 else n
                ref = e.weighted_sum(k[:m], w[:m])
                scale = np.max(np.abs(ref))
                if trial < 2:
                    assert np.array_equal(got, e.weighted_sum(k, w))
                assert np.max(np.abs(got - ref)) <= 1e-12 * scale


@pytest.mark.parametrize("nw,precision", [(32, _abi.PRECISION_FP64), (6, _abi.PRECISION_FP64),
                                          (32, _abi.PRECISION_MIXED)])
def test_autotune_keeps_results(torch_and_engine, nw, precision):
    _, eng = torch_and_engine
    model = (reference_workload_model("nw32") if nw == 32
             else synthetic_orthogonal_model(nw, 2, seed=7, full_position=True))
    task = _task(nom=512, precision=precision)
    mesh = (32, 32, 32)
    with eng.ResponseEngine(model, task, max_batch=8192) as e:
        before = e.integrate_mesh(mesh, 0, 8192)
        rep = e.autotune(mesh, 0, 8192)
        assert rep["eigh_team"] in (32, 64, 128) and rep["energies_per_thread"] in (1, 2, 4)
        assert sorted(rep["eigh_ms"]) == [32, 64, 128] and sorted(rep["response_ms"]) == [1, 2, 4]
        assert all(v > 0 for v in list(rep["eigh_ms"].values()) + list(rep["response_ms"].values()))
        assert rep["warm_start"] in (0, 1) and set(rep["start_ms"]) == {"cold", "warm"}
        if nw == 32 and precision == _abi.PRECISION_FP64:
            assert rep["response_threads"] in (256, 512) and set(rep["width_ms"]) == {256, 512}
        else:
            assert rep["response_threads"] == -1
        after = e.integrate_mesh(mesh, 0, 8192)
        tol = 1e-11 if precision == _abi.PRECISION_FP64 else 1e-6
        for a, b in zip(task.split(after), task.split(before)):
            assert np.max(np.abs(a - b)) <= tol * max(np.max(np.abs(b)), 1e-300)
    with eng.ResponseEngine(model, task, max_batch=8192) as e2:
        again = e2.autotune(mesh, 0, 8192)
        assert again["from_cache"] and again["eigh_team"] == rep["eigh_team"]
        assert again["energies_per_thread"] == rep["energies_per_thread"]
        assert again["warm_start"] == rep["warm_start"]
        assert again["response_threads"] == rep["response_threads"]


def test_graph_of_the_berry_dipole_stencils_replays_the_direct_call(torch_and_engine):
    """The Fermi-sea dipole's stencil (shifted fronts through the staged contraction with the
    shifted tile sets) and its analytic backend inside a captured graph: bitwise the direct call."""
    torch, eng = torch_and_engine
    model = synthetic_orthogonal_model(8, 1, seed=5, full_position=True)
    engines = []
    for backend in ("finite_difference", "analytic"):
        task = _abi.TaskArrays([(_abi.BERRY_DIPOLE_SEA, ["xyz", "yzx"]), (_abi.BERRY_DIPOLE, ["xyz"])],
                               fermi_energies=[-0.2, 0.3], temperature=100.0, degeneracy_threshold=1e-7,
                               derivative_backend=backend)
        engines.append(eng.ResponseEngine(model, task, max_batch=1024))
    try:
        meshes = [(12, 10, 8), (12, 10, 8)]
        ranges = [(0, 960), (100, 700)]
        direct = [torch.zeros(2 * e.value_count, dtype=torch.float64, device="cuda") for e in engines]
        graphed = [torch.zeros_like(d) for d in direct]
        stream = torch.cuda.current_stream().cuda_stream
        eng.integrate_meshes_many(engines, meshes, ranges, [d.data_ptr() for d in direct], stream)
        torch.cuda.synchronize()
        with eng.CapturedGraph.mesh_many(engines, meshes, ranges, [g.data_ptr() for g in graphed]) as graph:
            for g in graphed:
                g.zero_()
            graph.launch(stream)
            torch.cuda.synchronize()
            graph.status()
            for d, g in zip(direct, graphed):
                assert torch.equal(d, g)
        a = direct[0].cpu().numpy().view(np.complex128)
        b = direct[1].cpu().numpy().view(np.complex128)
        assert np.all(np.isfinite(a)) and np.all(np.isfinite(b))
    finally:
        for e in engines:
            e.close()
