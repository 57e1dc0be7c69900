"""A model loaded from a Packed HDF5 bundle runs through the C ABI exactly like the model itself.

The bundle is written by this package (the reference's fixture tree is not needed); the device
results from the bundle-loaded model are compared with the oracle on the original model (1e-10
relative, the FP64 bar) and bitwise with the device results of the original model.
"""
import numpy as np
import pytest

from wanniernlqg_b200 import _abi, bundle
from wanniernlqg_b200.model import reference_workload_model

pytestmark = pytest.mark.gpu


def test_bundle_model_matches_oracle_and_direct_model(tmp_path, oracle_mod):
    from wanniernlqg_b200 import build
    build.build()
    from wanniernlqg_b200.engine import ResponseEngine
    model = reference_workload_model("nw4")
    path = bundle.write_model_operator_bundle(str(tmp_path / "nw4.h5"), model, mp_grid=(8, 8, 8))
    loaded = bundle.model_from_operator_bundle(path)
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.INJECTION_CURRENT, ["xyy"]),
                            (_abi.BERRY_CURVATURE, ["xy"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.02,
                           photon_energies=np.linspace(0, 3, 64))
    k = np.random.default_rng(5).random((32, 3))
    with ResponseEngine(loaded, task) as eng:
        from_bundle = eng.point_values(k)
    with ResponseEngine(model, task) as eng:
        direct = eng.point_values(k)
    assert np.array_equal(from_bundle, direct)
    ref = oracle_mod.point_values(model, task, k)
    scale = np.max(np.abs(ref))
    assert np.max(np.abs(from_bundle - ref)) / scale < 1e-10
