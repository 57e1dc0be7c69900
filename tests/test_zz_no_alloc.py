"""The allocation-free spectrum entry point agrees with the planned spectrum path.

wnlqg_b200_spectrum_noalloc exists for callers whose device memory belongs to another pool
allocator under a fixed budget (a Julia CUDA.jl pool, PyTorch's caching allocator, a serving
process that reserves its HBM up front): they cannot let the library call cudaMalloc behind the
pool's back.  Here the test plays such a caller: it owns every device buffer (allocated with
torch) and calls the entry point through the C ABI twice in a row, checking each result against
wnlqg_b200_eval_spectrum with the tolerances of the other spectrum tests.  This file is named
to be collected last.
"""
import ctypes

import numpy as np
import pytest

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import reference_workload_model

pytestmark = pytest.mark.gpu


def test_spectrum_noalloc_matches_planned_spectrum():
    import torch
    from wanniernlqg_b200 import build, _lib
    from wanniernlqg_b200.engine import ResponseEngine
    build.build()
    L = _lib.load()
    model = reference_workload_model("nw32")
    nw, nr = model.num_orbitals, model.num_r_vectors
    task = _abi.TaskArrays([(_abi.QUANTUM_METRIC, ["xx"])], broadening_type=_abi.LORENTZIAN, broadening=0.01)
    dev = torch.device("cuda", 0)
    ham = torch.from_numpy(np.ascontiguousarray(model.hamiltonian_r.transpose(2, 1, 0)).view(np.float64).copy()).to(dev)
    rvec = torch.from_numpy(np.ascontiguousarray(model.r_vectors.T)).to(dev)
    deg = torch.from_numpy(model.r_degeneracies.copy()).to(dev)
    rng = np.random.default_rng(21)
    with ResponseEngine(model, task) as eng:
        for call in range(2):
            k = rng.random((200, 3))
            e_ref, u_ref = eng.spectrum(k)
            kd = torch.from_numpy(k).to(dev)
            e = torch.zeros((200, nw), dtype=torch.float64, device=dev)
            u = torch.zeros((200, nw, nw, 2), dtype=torch.float64, device=dev)
            torch.cuda.synchronize()
            _lib.check(L.wnlqg_b200_spectrum_noalloc(nw, nr, ctypes.c_void_p(ham.data_ptr()),
                                                     ctypes.c_void_p(rvec.data_ptr()), ctypes.c_void_p(deg.data_ptr()),
                                                     ctypes.c_void_p(kd.data_ptr()), 200, ctypes.c_void_p(e.data_ptr()),
                                                     ctypes.c_void_p(u.data_ptr()), None))
            torch.cuda.synchronize()
            e_h = e.cpu().numpy()
            uu = u.cpu().numpy()
            u_h = (uu[..., 0] + 1j * uu[..., 1]).transpose(0, 2, 1)   # column-major per k
            assert np.max(np.abs(e_h - e_ref)) < 1e-12 * max(1.0, np.abs(e_ref).max())
            ov = np.abs(np.sum(u_h.conj() * u_ref, axis=1))
            assert np.max(np.abs(ov - 1.0)) < 1e-9


def test_spectrum_noalloc_rejects_oversized_batch():
    from wanniernlqg_b200 import build, _lib
    build.build()
    L = _lib.load()
    # 8 MiB / ((729 + 1024) * 16 B) is about 299 points; 10_000 must be refused before any launch.
    st = L.wnlqg_b200_spectrum_noalloc(32, 729, ctypes.c_void_p(16), ctypes.c_void_p(16), ctypes.c_void_p(16),
                                       ctypes.c_void_p(16), 10_000, ctypes.c_void_p(16), ctypes.c_void_p(16), None)
    assert st == 1
    assert "8 MiB" in _lib.last_error()
