"""Host side of the B200 engine: a device-resident model plus a compiled task (plan).

``ResponseEngine`` is the drop-in for the reference's per-worker k loop: ``integrate_mesh``
returns the lane tensor sum_k value(k)/Nk over a range of the Gamma-centred mesh (the
contract of consume_point!, Runtime/Execution/IntegralDriver.jl:820-874), ``point_values`` is
the batched ResponsePointEvaluator / ResponseNodeEvaluator
(Runtime/Execution/ResponsePointEvaluation.jl:8-64), and ``spectrum`` exposes compute_spectrum!
(MatrixElements/Interpolated/HamiltonianMatrixElements.jl:279-300).
"""
from __future__ import annotations

import ctypes
from typing import Optional, Sequence

import numpy as np

from . import _abi, _lib
from .model import TightBindingModel


class ResponseEngine:
    def __init__(self, model: TightBindingModel, task: _abi.TaskArrays, *, device: int = 0, max_batch: int = 0):
        L = _lib.load()
        self._L = L
        self.model = model
        self.task = task
        self._marrays = _abi.ModelArrays(model)
        self._model = ctypes.c_void_p()
        self._plan = ctypes.c_void_p()
        _lib.check(L.wnlqg_b200_model_create(ctypes.byref(self._marrays.desc), device, ctypes.byref(self._model)))
        try:
            _lib.check(L.wnlqg_b200_plan_create(self._model, ctypes.byref(task.desc), max_batch,
                                                ctypes.byref(self._plan)))
        except Exception:
            L.wnlqg_b200_model_destroy(self._model)
            self._model = ctypes.c_void_p()
            raise
        self.value_count = int(L.wnlqg_b200_plan_value_count(self._plan))

    # -- lifetime ------------------------------------------------------------------------
    def close(self) -> None:
        if self._plan:
            # Refused while a CUDA graph holds the plan: the model then stays alive too.
            _lib.check(self._L.wnlqg_b200_plan_destroy(self._plan))
            self._plan = ctypes.c_void_p()
        if self._model:
            self._L.wnlqg_b200_model_destroy(self._model)
            self._model = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- evaluation ----------------------------------------------------------------------
    def integrate_mesh(self, mesh: Sequence[int], k_begin: int = 0, k_end: Optional[int] = None) -> np.ndarray:
        """sum over mesh indices [k_begin, k_end) of value(k)/Nk, complex [value_count]."""
        mesh_a = np.ascontiguousarray(np.asarray(mesh, dtype=np.int64))
        if mesh_a.shape != (3,):
            raise ValueError("mesh must have three counts")
        if k_end is None:
            k_end = int(np.prod(mesh_a))
        out = np.zeros(self.value_count, dtype=np.complex128)
        _lib.check(self._L.wnlqg_b200_eval_mesh(self._plan, mesh_a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                                int(k_begin), int(k_end),
                                                out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def integrate_mesh_device(self, mesh: Sequence[int], k_begin: int, k_end: int, out_device_ptr: int,
                              stream_ptr: int = 0) -> None:
        """Asynchronous variant writing value_count complex values to a device pointer."""
        mesh_a = np.ascontiguousarray(np.asarray(mesh, dtype=np.int64))
        _lib.check(self._L.wnlqg_b200_eval_mesh_device(self._plan,
                                                       mesh_a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                                       int(k_begin), int(k_end), ctypes.c_void_p(out_device_ptr),
                                                       ctypes.c_void_p(stream_ptr)))

    def point_values(self, kpoints) -> np.ndarray:
        """Per-point values at fractional k-points [n, 3] -> complex [n, value_count]."""
        k = np.ascontiguousarray(np.asarray(kpoints, dtype=np.float64).reshape(-1, 3))
        out = np.zeros((k.shape[0], self.value_count), dtype=np.complex128)
        _lib.check(self._L.wnlqg_b200_eval_points(self._plan, k.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                  k.shape[0], out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def weighted_sum(self, kpoints, weights) -> np.ndarray:
        """sum_i weights[i] * value(k_i) over host k-points [n, 3], complex [value_count]."""
        k = np.ascontiguousarray(np.asarray(kpoints, dtype=np.float64).reshape(-1, 3))
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).reshape(-1))
        if w.shape[0] != k.shape[0]:
            raise ValueError("one weight per k-point")
        out = np.zeros(self.value_count, dtype=np.complex128)
        _lib.check(self._L.wnlqg_b200_eval_points_weighted(
            self._plan, k.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), k.shape[0],
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def weighted_sum_device(self, kpoints_ptr: int, weights_ptr: int, n: int, out_device_ptr: int,
                            stream_ptr: int = 0) -> None:
        """Asynchronous weighted sum over n device-resident k-points ([n, 3] doubles) and weights,
        writing value_count complex values to a device pointer."""
        _lib.check(self._L.wnlqg_b200_eval_points_weighted_device(
            self._plan, ctypes.c_void_p(kpoints_ptr), ctypes.c_void_p(weights_ptr), int(n),
            ctypes.c_void_p(out_device_ptr), ctypes.c_void_p(stream_ptr)))

    def mesh_weighted_sum(self, mesh: Sequence[int], indices, weights) -> np.ndarray:
        """sum_i weights[i] * value(mesh point indices[i]) from host arrays, complex [value_count]."""
        mesh_a = np.ascontiguousarray(np.asarray(mesh, dtype=np.int64))
        idx = np.ascontiguousarray(np.asarray(indices, dtype=np.int64).reshape(-1))
        w = np.ascontiguousarray(np.asarray(weights, dtype=np.float64).reshape(-1))
        if idx.shape != w.shape:
            raise ValueError("one weight per index")
        out = np.zeros(self.value_count, dtype=np.complex128)
        ip = ctypes.POINTER(ctypes.c_int64)
        _lib.check(self._L.wnlqg_b200_eval_mesh_weighted(
            self._plan, mesh_a.ctypes.data_as(ip), idx.ctypes.data_as(ip),
            w.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), idx.shape[0],
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        return out

    def integrate_mesh_reduced(self, mesh: Sequence[int], operations, *, orbits=None) -> np.ndarray:
        """Mesh average of a shift / injection current task evaluated on the symmetry-reduced
        mesh (representatives weighted by orbit size, then projected onto the group-invariant
        tensors); see wanniernlqg_b200.symmetry.integrate_mesh_reduced."""
        from .symmetry import integrate_mesh_reduced
        return integrate_mesh_reduced(self.mesh_weighted_sum, self.task, mesh, operations, orbits=orbits)

    def spectrum(self, kpoints, vectors: bool = True):
        """(energies [n, nw], canonical eigenvectors [n, nw, nw] or None when ``vectors`` is
        false) at fractional k-points."""
        k = np.ascontiguousarray(np.asarray(kpoints, dtype=np.float64).reshape(-1, 3))
        nw = self.model.num_orbitals
        e = np.zeros((k.shape[0], nw))
        # Column-major per k: store as [n, col, row] and transpose.
        u = np.zeros((k.shape[0], nw, nw), dtype=np.complex128) if vectors else None
        dp = ctypes.POINTER(ctypes.c_double)
        _lib.check(self._L.wnlqg_b200_eval_spectrum(self._plan, k.ctypes.data_as(dp), k.shape[0], e.ctypes.data_as(dp),
                                                    u.ctypes.data_as(dp) if vectors else None))
        return e, (np.ascontiguousarray(u.transpose(0, 2, 1)) if vectors else None)

    def last_timing(self):
        """Device milliseconds (fourier, eigen, response, total) of the last mesh evaluation."""
        vals = [ctypes.c_double() for _ in range(4)]
        _lib.check(self._L.wnlqg_b200_plan_last_timing(self._plan, *[ctypes.byref(v) for v in vals]))
        return tuple(v.value for v in vals)

    def last_launch_count(self) -> int:
        return int(self._L.wnlqg_b200_plan_last_launch_count(self._plan))

    def status(self) -> None:
        """After synchronising the stream of an asynchronous call (``*_device``, the many-plan
        call): raises on a bounded device wait that gave up or on a k-point that failed the task's
        spectral isolation contract (wnlqg_b200_plan_status)."""
        _lib.check(self._L.wnlqg_b200_plan_status(self._plan))

    def autotune(self, mesh: Sequence[int], k_begin: int = 0, k_end: Optional[int] = None) -> dict:
        """Pick the eigensolver team size and the contraction tile by timing them on a block of
        ``mesh`` (wnlqg_b200_plan_autotune); the choice stays in this plan and in the process
        cache.  Returns the report as a dict."""
        mesh_a = np.ascontiguousarray(np.asarray(mesh, dtype=np.int64))
        if k_end is None:
            k_end = int(np.prod(mesh_a))
        rep = _abi.AutotuneReport()
        _lib.check(self._L.wnlqg_b200_plan_autotune(self._plan, mesh_a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)),
                                                    int(k_begin), int(k_end), ctypes.byref(rep)))
        return {"eigh_team": rep.eigh_team, "energies_per_thread": rep.energies_per_thread,
                "eigh_ms": {t: rep.eigh_ms[i] for i, t in enumerate((32, 64, 128)) if rep.eigh_ms[i] >= 0},
                "response_ms": {t: rep.response_ms[i] for i, t in enumerate((1, 2, 4)) if rep.response_ms[i] >= 0},
                "warm_start": rep.warm_start,
                "start_ms": ({"cold": rep.start_ms[0], "warm": rep.start_ms[1]} if rep.warm_start >= 0 else {}),
                "response_threads": rep.response_threads,
                "width_ms": ({256: rep.width_ms[0], 512: rep.width_ms[1]} if rep.response_threads > 0 else {}),
                "metric_shg_grid": rep.metric_shg_grid,
                "metric_shg_grid_ms": list(rep.metric_shg_grid_ms) if rep.metric_shg_grid > 0 else [],
                "shg_grid": rep.shg_grid,
                "shg_grid_ms": list(rep.shg_grid_ms) if rep.shg_grid > 0 else [],
                "response_grid": rep.response_grid,
                "response_grid_ms": list(rep.response_grid_ms) if rep.response_grid >= 0 else [],
                "eigh_grid": rep.eigh_grid,
                "eigh_grid_ms": list(rep.eigh_grid_ms) if rep.eigh_grid > 0 else [],
                "from_cache": bool(rep.from_cache)}


def integrate_meshes_many(engines, meshes, ranges, outs_device, stream_ptr: int = 0) -> None:
    """Mesh sums of several engines (models) in one asynchronous call (wnlqg_b200_eval_mesh_many):
    engine i sums meshes[i] over ranges[i] = (k_begin, k_end) into the device pointer outs_device[i];
    the engines' kernels overlap on the device.  All engines must use one device."""
    n = len(engines)
    L = _lib.load()
    vp = ctypes.c_void_p
    plans = (vp * n)(*[e._plan for e in engines])
    mesh_a = np.ascontiguousarray(np.asarray(meshes, dtype=np.int64).reshape(n, 3))
    kb = np.ascontiguousarray(np.array([r[0] for r in ranges], dtype=np.int64))
    ke = np.ascontiguousarray(np.array([r[1] for r in ranges], dtype=np.int64))
    outs = (vp * n)(*[vp(o) for o in outs_device])
    ip = ctypes.POINTER(ctypes.c_int64)
    _lib.check(L.wnlqg_b200_eval_mesh_many(plans, n, mesh_a.ctypes.data_as(ip), kb.ctypes.data_as(ip),
                                           ke.ctypes.data_as(ip), outs, vp(stream_ptr)))


class CapturedGraph:
    """One CUDA graph holding a whole call (wnlqg_b200_graph_*): build it with
    :meth:`mesh_many` or :meth:`points_weighted`, replay it with :meth:`launch`.  The engines it
    captured must outlive it; close it before closing them."""

    def __init__(self, handle, engines):
        self._L = _lib.load()
        self._g = handle
        self._engines = list(engines)

    @classmethod
    def mesh_many(cls, engines, meshes, ranges, outs_device) -> "CapturedGraph":
        """The work of :func:`integrate_meshes_many` with these arguments."""
        n = len(engines)
        L = _lib.load()
        vp = ctypes.c_void_p
        plans = (vp * n)(*[e._plan for e in engines])
        mesh_a = np.ascontiguousarray(np.asarray(meshes, dtype=np.int64).reshape(n, 3))
        kb = np.ascontiguousarray(np.array([r[0] for r in ranges], dtype=np.int64))
        ke = np.ascontiguousarray(np.array([r[1] for r in ranges], dtype=np.int64))
        outs = (vp * n)(*[vp(o) for o in outs_device])
        ip = ctypes.POINTER(ctypes.c_int64)
        g = vp()
        _lib.check(L.wnlqg_b200_graph_capture_mesh_many(plans, n, mesh_a.ctypes.data_as(ip), kb.ctypes.data_as(ip),
                                                        ke.ctypes.data_as(ip), outs, ctypes.byref(g)))
        return cls(g, engines)

    @classmethod
    def points_weighted(cls, engine, kpoints_ptr: int, weights_ptr: int, n: int,
                        out_device_ptr: int) -> "CapturedGraph":
        """The work of :meth:`ResponseEngine.weighted_sum_device` on these device buffers."""
        L = _lib.load()
        g = ctypes.c_void_p()
        _lib.check(L.wnlqg_b200_graph_capture_points_weighted(
            engine._plan, ctypes.c_void_p(kpoints_ptr), ctypes.c_void_p(weights_ptr), int(n),
            ctypes.c_void_p(out_device_ptr), ctypes.byref(g)))
        return cls(g, [engine])

    @property
    def kernel_count(self) -> int:
        return int(self._L.wnlqg_b200_graph_kernel_count(self._g))

    def launch(self, stream_ptr: int = 0) -> None:
        _lib.check(self._L.wnlqg_b200_graph_launch(self._g, ctypes.c_void_p(stream_ptr)))

    def status(self) -> None:
        """After synchronising: raises when a bounded device wait of the last launch gave up."""
        _lib.check(self._L.wnlqg_b200_graph_status(self._g))

    def close(self) -> None:
        if self._g:
            _lib.check(self._L.wnlqg_b200_graph_destroy(self._g))
            self._g = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
