"""GPU parity at the workloads' own sizes: the CPU-runnable nw = 4 case on its full 32^3 mesh, a
whole 65,536-point block of the nw = 32 workload mesh (checked point by point on a strided
subsample and through the block sum), and nonorthogonal nw = 64 second harmonic generation on
256 photon energies.  Tolerances: 1e-10 relative for the FP64 path, 1e-4 for the mixed path (max
norm over energies and components, relative to the oracle's max norm).
"""
import numpy as np
import pytest

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import reference_workload_model

pytestmark = pytest.mark.gpu
RTOL = 1e-10
MIXED_RTOL = 1e-4


@pytest.fixture(scope="module")
def engine_cls():
    from wanniernlqg_b200 import build
    build.build()
    from wanniernlqg_b200.engine import ResponseEngine
    return ResponseEngine


def rel_err(got, ref):
    scale = np.max(np.abs(ref))
    return np.max(np.abs(got - ref)) / (scale if scale > 0 else 1.0)


def mesh_points(mesh, idx):
    n1, n2, n3 = mesh
    return np.stack([(idx % n1) / n1, ((idx // n1) % n2) / n2, (idx // (n1 * n2)) / n3], axis=1)


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_nw4_full_32_mesh(engine_cls, oracle_mod, precision):
    """Shift and injection current xyy of the nw = 4 model on its whole 32^3 mesh, 128 energies in
    [0, 3] eV, Lorentzian 0.02 eV, mu = 0, T = 0: the lane-ordered mesh integral."""
    model = reference_workload_model("nw4")
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.INJECTION_CURRENT, ["xyy"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.02, photon_energies=np.linspace(0, 3, 128),
                           precision=precision)
    with engine_cls(model, task) as eng:
        got = eng.integrate_mesh((32, 32, 32))
    ref = oracle_mod.integrate_mesh(model, task, (32, 32, 32))
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < tol


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_nw32_workload_block(engine_cls, oracle_mod, precision):
    """One whole 65,536-point block of the 256^3 workload mesh (shift current xyy on 512
    energies, Berry curvature xy, quantum metric xx): on the FP64 path the block sum equals the sum
    of the engine's own point values of the block (mesh and arbitrary-point Fourier paths), on the
    mixed path it matches the FP64 block; the point values match the oracle on a strided subsample
    of 256 points spread over the block."""
    model = reference_workload_model("nw32")
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.BERRY_CURVATURE, ["xy"]),
                            (_abi.QUANTUM_METRIC, ["xx"])], broadening_type=_abi.LORENTZIAN, broadening=0.01,
                           photon_energies=np.linspace(0.0, 4.0, 512), precision=precision)
    mesh = (256, 256, 256)
    start = 3 * 65536 + 12345
    idx = np.arange(start, start + 65536, dtype=np.int64)
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    with engine_cls(model, task, max_batch=65536) as eng:
        block = eng.integrate_mesh(mesh, start, start + 65536)
        pts = eng.point_values(mesh_points(mesh, idx))
    nk = 256 ** 3
    if precision == _abi.PRECISION_FP64:
        # The mesh path's staged Fourier and the points path's tensor-core Fourier (7 slices, 2^-49
        # of each column's scale) agree to the FP64 bar.
        for g, r in zip(task.split(block), task.split(pts.sum(axis=0) / nk)):
            assert rel_err(g, r) < RTOL
    else:
        # The mixed mesh block against the FP64 block (the points path's 4-slice Fourier is
        # checked point by point against the oracle below).
        task64 = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.BERRY_CURVATURE, ["xy"]),
                                  (_abi.QUANTUM_METRIC, ["xx"])], broadening_type=_abi.LORENTZIAN,
                                 broadening=0.01, photon_energies=np.linspace(0.0, 4.0, 512))
        with engine_cls(model, task64, max_batch=65536) as eng:
            block64 = eng.integrate_mesh(mesh, start, start + 65536)
        for g, r in zip(task.split(block), task.split(block64)):
            assert rel_err(g, r) < MIXED_RTOL
    sub = idx[::256]
    ref = oracle_mod.point_values(model, task, mesh_points(mesh, sub))
    got = pts[::256]
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < tol


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_nonorthogonal_nw64_shg_256_energies(engine_cls, oracle_mod, precision):
    """Metric SHG chi^xxx of the nonorthogonal nw = 64 workload model (|R_i| <= 3) on 256
    energies in [0, 3] eV, Lorentzian 0.02 eV, at four k-points: every (term, quantity) block."""
    model = reference_workload_model("nw64_nonorth")
    task = _abi.TaskArrays([(_abi.SECOND_HARMONIC, ["xxx"])], broadening_type=_abi.LORENTZIAN, broadening=0.02,
                           photon_energies=np.linspace(0.0, 3.0, 256), fermi_energy=0.0, temperature=0.0,
                           degeneracy_threshold=0.002, shg_low_frequency_broadening=0.025,
                           denominator_regularization=0.01, shg_eta_correction=False, precision=precision)
    k = np.random.default_rng(64).random((4, 3))
    with engine_cls(model, task) as eng:
        got = task.split(eng.point_values(k))[0]
    ref = task.split(oracle_mod.point_values(model, task, k))[0]
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    worst = 0.0
    for t in range(7):
        for q in range(2):
            scale = np.max(np.abs(ref[..., t, q]))
            if scale > 0:
                worst = max(worst, np.max(np.abs(got[..., t, q] - ref[..., t, q])) / scale)
    assert worst < tol
