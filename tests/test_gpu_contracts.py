"""GPU checks, through the C ABI, of the reference's error contracts and of known answers:
the spectral isolation contract (geometry_isolated_spectrum_minimum_gap,
OrthogonalBandDerivatives.jl:66-82, at BerryMultipoleGeometry.jl:81 and PositionMatrixElements.jl:
447-452), the zero-temperature rule of the intrinsic AHC (IntrinsicHallOccupations.jl:15-16), the
linear transport Berry channel (LinearTransportKernels.jl:100-163), the Qi-Wu-Zhang Chern number,
and the autotuner's grid dimensions for large orbital counts.
"""
import re
import sys
import os

import numpy as np
import pytest

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import TightBindingModel, kramers_doubled_model, synthetic_orthogonal_model

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from test_parity_pins import two_band_model  # noqa: E402

pytestmark = pytest.mark.gpu
RTOL = 1e-10
MIXED_RTOL = 1e-4
ISO_RE = re.compile(r"GEOMETRY_SINGLE_BAND_SPECTRUM_NOT_ISOLATED: bands=\((\d+),(\d+)\), gap_ev=(\S+), "
                    r"threshold_ev=(\S+) \(k-point row (\d+)\)")


@pytest.fixture(scope="module")
def engine_cls():
    from wanniernlqg_b200 import build
    build.build()
    from wanniernlqg_b200.engine import ResponseEngine
    return ResponseEngine


def rel_err(got, ref):
    scale = np.max(np.abs(ref))
    return np.max(np.abs(got - ref)) / (scale if scale > 0 else 1.0)


def _parsed(msg):
    m = ISO_RE.search(msg)
    assert m, msg
    return int(m.group(1)), int(m.group(2)), float(m.group(3)), float(m.group(4)), int(m.group(5))


def _doubled(model: TightBindingModel) -> TightBindingModel:
    nw, nr = model.num_orbitals, model.num_r_vectors
    ham = np.zeros((2 * nw, 2 * nw, nr), dtype=np.complex128, order="F")
    for r in range(nr):
        ham[:, :, r] = np.kron(model.hamiltonian_r[:, :, r], np.eye(2))
    return TightBindingModel(model.lattice.copy(), model.r_vectors.copy(), model.r_degeneracies.copy(), ham, None)


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_berry_dipole_isolation_error_matches_oracle(engine_cls, oracle_mod, precision):
    """The first failing k-point row, its first failing band pair and the threshold equal the
    oracle's report; points, mesh and weighted calls all refuse, and the plan stays usable."""
    from wanniernlqg_b200._lib import EngineError
    model = synthetic_orthogonal_model(6, 1, 3, full_position=True)
    k = np.random.default_rng(21).random((40, 3))
    e0 = oracle_mod.kpoint_spectrum(model, k[0])[0]
    thr = float(np.median(np.diff(e0)))
    task = _abi.TaskArrays([(_abi.BERRY_DIPOLE, ["xyz"])], fermi_energies=[0.0], fermi_surface_broadening=0.05,
                           degeneracy_threshold=thr, precision=precision)
    with pytest.raises(RuntimeError) as oexc:
        oracle_mod.point_values(model, task, k)
    ref = _parsed(str(oexc.value))
    with engine_cls(model, task) as eng:
        with pytest.raises(EngineError) as gexc:
            eng.point_values(k)
        assert gexc.value.status == 1
        got = _parsed(str(gexc.value))
        assert got[:2] == ref[:2] and got[3] == ref[3] and got[4] == ref[4]
        # Mixed-path energies come out of one FP64 refinement sweep: the gap agrees to ~1e-8.
        assert got[2] == pytest.approx(ref[2], rel=1e-9 if precision == _abi.PRECISION_FP64 else 1e-6)
        with pytest.raises(EngineError):
            eng.weighted_sum(k, np.ones(len(k)))
        with pytest.raises(EngineError, match="NOT_ISOLATED"):
            eng.integrate_mesh((4, 4, 4))
        # A threshold below every gap: the same plan object is gone, a new one evaluates.
    ok = _abi.TaskArrays([(_abi.BERRY_DIPOLE, ["xyz"])], fermi_energies=[0.0], fermi_surface_broadening=0.05,
                         degeneracy_threshold=1e-9, precision=precision)
    with engine_cls(model, ok) as eng:
        vals = eng.point_values(k)
    assert np.all(np.isfinite(vals))


def test_exact_geometry_isolation_and_async_status(engine_cls, oracle_mod):
    """eta = 0 geometry on an exactly doubled model: synchronous calls refuse; the asynchronous
    device call returns OK and the error comes from plan_status after synchronising, once."""
    import torch
    from wanniernlqg_b200._lib import EngineError
    model = _doubled(synthetic_orthogonal_model(3, 1, 4))
    task = _abi.TaskArrays([(_abi.BERRY_CURVATURE, ["xy"])], denominator_regularization=0.0)
    with pytest.raises(RuntimeError) as oexc:
        oracle_mod.integrate_mesh(model, task, (3, 2, 2))
    ref = _parsed(str(oexc.value))
    with engine_cls(model, task) as eng:
        with pytest.raises(EngineError) as gexc:
            eng.integrate_mesh((3, 2, 2))
        got = _parsed(str(gexc.value))
        assert got[0:2] == ref[0:2] == (1, 2) and got[4] == ref[4] == 0 and got[3] == 1e-10
        out = torch.zeros(2 * eng.value_count, dtype=torch.float64, device="cuda")
        eng.integrate_mesh_device((3, 2, 2), 0, 12, out.data_ptr())
        torch.cuda.synchronize()
        with pytest.raises(EngineError, match="NOT_ISOLATED"):
            eng.status()
        eng.status()   # cleared
    reg = _abi.TaskArrays([(_abi.BERRY_CURVATURE, ["xy"])], denominator_regularization=1e-3)
    with engine_cls(model, reg) as eng:
        got = eng.integrate_mesh((3, 2, 2))
    assert rel_err(got, oracle_mod.integrate_mesh(model, reg, (3, 2, 2))) < RTOL


def test_intrinsic_ahc_refuses_finite_temperature(engine_cls):
    from wanniernlqg_b200._lib import EngineError
    model = synthetic_orthogonal_model(4, 1, 2)
    task = _abi.TaskArrays([(_abi.INTRINSIC_AHC, ["xy"])], fermi_energies=[0.0], temperature=50.0)
    with pytest.raises(EngineError, match="INTRINSIC_HALL_REQUIRES_ZERO_TEMPERATURE"):
        engine_cls(model, task)


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
@pytest.mark.parametrize("temperature,gamma", [(0.0, 0.0), (300.0, 0.05)])
def test_linear_transport_berry_matches_oracle(engine_cls, oracle_mod, precision, temperature, gamma):
    model = synthetic_orthogonal_model(12, 1, 31, full_position=True)
    task = _abi.TaskArrays([(_abi.LINEAR_TRANSPORT_BERRY, ["xy", "yz", "zx"])],
                           fermi_energies=[-0.6, -0.1, 0.0, 0.35, 0.8], temperature=temperature,
                           linear_transport_gamma_inter=gamma, precision=precision)
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    k = np.random.default_rng(5).random((24, 3))
    with engine_cls(model, task) as eng:
        pts = eng.point_values(k)
        mesh = eng.integrate_mesh((6, 5, 4))
    assert rel_err(pts, oracle_mod.point_values(model, task, k)) < tol
    assert rel_err(mesh, oracle_mod.integrate_mesh(model, task, (6, 5, 4))) < tol


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_qwz_chern_number_on_device(engine_cls, precision):
    """Known answer independent of the oracle: the occupied Berry curvature (bare denominators)
    and the intrinsic AHC of the Qi-Wu-Zhang model average to C / (2 pi), C = -1 (0 < m < 2),
    +1 (-2 < m < 0), 0 (|m| > 2)."""
    tol = 1e-12 if precision == _abi.PRECISION_FP64 else 1e-5
    for mass, chern in ((1.0, -1), (-1.0, 1), (3.0, 0)):
        model = two_band_model(mass, tz=0.0, sz_x=0.0)
        bc = _abi.TaskArrays([(_abi.BERRY_CURVATURE, ["xy"])], fermi_energy=0.0, denominator_regularization=0.0,
                             precision=precision)
        ahc = _abi.TaskArrays([(_abi.INTRINSIC_AHC, ["xy"])], fermi_energies=[0.0], precision=precision)
        for task in (bc, ahc):
            with engine_cls(model, task) as eng:
                mean = eng.integrate_mesh((64, 64, 1))[0].real
            assert abs(2 * np.pi * mean - chern) <= tol


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_large_orbital_autotuned_grids_keep_results(engine_cls, oracle_mod, precision):
    """nw = 96 (per-CTA global working sets for the response passes and the CTA eigensolver
    stages): the autotuner's grid choices change how points are split among CTAs, and so the
    summation order (FP64: last bits) and, on the mixed path, the FP32 eigensolver's warm-start
    chains (results within the mixed accuracy); tuned point values match the oracle."""
    model = synthetic_orthogonal_model(96, 1, seed=41, full_position=True)
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.BERRY_CURVATURE, ["xy"]),
                            (_abi.QUANTUM_METRIC, ["xx"])], broadening_type=_abi.LORENTZIAN, broadening=0.02,
                           photon_energies=np.linspace(0.1, 3.0, 16), precision=precision)
    mesh = (8, 8, 8)
    with engine_cls(model, task, max_batch=512) as eng:
        before = eng.integrate_mesh(mesh, 0, 512)
        rep = eng.autotune(mesh, 0, 512)
        after = eng.integrate_mesh(mesh, 0, 512)
        k = np.random.default_rng(12).random((3, 3))
        got = eng.point_values(k)
    assert rep["response_grid"] != -1 and len(rep["response_grid_ms"]) == 3
    assert rep["eigh_grid"] != -1 and len(rep["eigh_grid_ms"]) == 3
    # FP64: only the summation order changes; mixed: the FP32 warm-start chains change too.
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    for g, r in zip(task.split(after), task.split(before)):
        assert rel_err(g, r) <= (1e-12 if precision == _abi.PRECISION_FP64 else 1e-5)
    ref = oracle_mod.point_values(model, task, k)
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < tol


def test_measured_peaks_are_plausible(engine_cls):
    """The roofline denominators of the SM-bound stages: positive, FP32 FMA above FP64 FMA, and
    within an order of magnitude of the B200's nominal dense figures (FP64 ~37-40, FP32 ~74-80
    TFLOP/s)."""
    from wanniernlqg_b200 import _lib
    p = _lib.measure_peaks(0)
    assert 4.0 < p["fp64_dmma_tflops"] < 400.0
    assert 4.0 < p["fp64_fma_tflops"] < 400.0
    assert 8.0 < p["fp32_fma_tflops"] < 800.0
    assert p["fp32_fma_tflops"] > p["fp64_fma_tflops"]
