"""Second-harmonic generation on the GPU (shg_kernel) through the C ABI.

Checked three ways: directly against the reference's frozen four-band tables
(test/second_harmonic_unit.jl; the table is the sum of the seven terms), against the CPU oracle
term by term at arbitrary k-points (FP64: 1e-10 relative in the max norm over each term and
quantity block), and through the mesh reduction.
"""
import os

import numpy as np
import pytest

from conftest import GOLDEN, read_complex_lines
from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import read_wannier_tb, reference_workload_model

pytestmark = pytest.mark.gpu
RTOL = 1e-10
MIXED_RTOL = 1e-4
COMPONENTS = [(a, b, c) for a in range(3) for (b, c) in ((0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1))]
OMEGAS = [0.0, 0.1, 0.73, 1.7]


def shg_task(*, gaussian=True, correction=True, T=0.0, mu=0.0, omegas=OMEGAS, components=COMPONENTS,
             precision=_abi.PRECISION_FP64, extra=()):
    return _abi.TaskArrays(list(extra) + [(_abi.SECOND_HARMONIC, components)],
                           broadening_type=_abi.GAUSSIAN if gaussian else _abi.LORENTZIAN, broadening=0.025,
                           photon_energies=omegas, fermi_energy=mu, temperature=T, degeneracy_threshold=0.002,
                           shg_low_frequency_broadening=0.025, shg_intermediate_regularization=0.04,
                           shg_eta_correction=correction, precision=precision)


def block_err(got, ref):
    """Largest relative error over the (term, quantity) blocks of [.., n_omega, nc, 7, 2] arrays."""
    worst = 0.0
    for t in range(7):
        for q in range(2):
            g, r = got[..., t, q], ref[..., t, q]
            scale = np.max(np.abs(r))
            err = np.max(np.abs(g - r))
            worst = max(worst, err / scale if scale > 0 else err)
    return worst


@pytest.fixture(scope="module")
def engine_cls():
    from wanniernlqg_b200 import build
    build.build()
    from wanniernlqg_b200.engine import ResponseEngine
    return ResponseEngine


@pytest.fixture(scope="module")
def tb4():
    return read_wannier_tb(os.path.join(GOLDEN, "synthetic_tb.dat"))


@pytest.mark.parametrize("gaussian", [True, False])
@pytest.mark.parametrize("correction", [True, False])
def test_shg_matches_reference_tables(engine_cls, tb4, gaussian, correction):
    task = shg_task(gaussian=gaussian, correction=correction)
    with engine_cls(tb4, task) as eng:
        got = task.split(eng.point_values([[0.17, 0.23, 0.31], [0.0, 0.0, 0.0]]))[0]
    for i, point in enumerate(["generic", "gamma"]):
        name = f"{point}_{'gaussian' if gaussian else 'lorentzian'}_{'corrected' if correction else 'uncorrected'}.dat"
        ref = read_complex_lines(os.path.join(GOLDEN, "second_harmonic", name)).reshape(4, 18, 2, order="F")
        np.testing.assert_allclose(got[i].sum(axis=2), ref, atol=1e-10, rtol=1e-8)
        assert np.all(got[i][:, :, 5:7, :] == 0)


@pytest.mark.parametrize("T,mu_band", [(0.0, None), (300.0, 1)])
@pytest.mark.parametrize("gaussian", [True, False])
def test_shg_terms_match_oracle_nw4(engine_cls, oracle_mod, tb4, T, mu_band, gaussian):
    rng = np.random.default_rng(21)
    k = np.vstack([[0.17, 0.23, 0.31], rng.random((7, 3))])
    mu = 0.0 if mu_band is None else float(oracle_mod.kpoint_data(tb4, k[0])[0][mu_band])
    task = shg_task(gaussian=gaussian, T=T, mu=mu, omegas=np.linspace(0.0, 3.0, 37))
    with engine_cls(tb4, task) as eng:
        got = task.split(eng.point_values(k))[0]
    ref = task.split(oracle_mod.point_values(tb4, task, k))[0]
    assert block_err(got, ref) < RTOL
    if T > 0:
        assert np.any(got[:, :, :, 5:7, :] != 0)


@pytest.mark.parametrize("T", [0.0, 300.0])
def test_shg_nw32_matches_oracle(engine_cls, oracle_mod, T):
    model = reference_workload_model("nw32")
    rng = np.random.default_rng(22)
    k = rng.random((4, 3))
    comps = [(0, 1, 1), (2, 0, 1), (1, 2, 2), (0, 0, 0)]
    task = shg_task(T=T, omegas=np.linspace(0.0, 4.0, 40), components=comps)
    with engine_cls(model, task) as eng:
        got = task.split(eng.point_values(k))[0]
    ref = task.split(oracle_mod.point_values(model, task, k))[0]
    assert block_err(got, ref) < RTOL


def test_shg_mesh_with_other_responses(engine_cls, oracle_mod, tb4):
    """SHG beside shift-current and quantum-metric components in one task: value offsets, mesh
    lanes, staged Fourier."""
    task = shg_task(gaussian=False, T=150.0, omegas=np.linspace(0.0, 2.5, 21),
                    extra=[(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.QUANTUM_METRIC, ["xx"])])
    mesh = (6, 5, 4)
    with engine_cls(tb4, task, max_batch=37) as eng:
        got = eng.integrate_mesh(mesh)
    ref = oracle_mod.integrate_mesh(tb4, task, mesh)
    g_parts, r_parts = task.split(got), task.split(ref)
    for g, r in zip(g_parts[:2], r_parts[:2]):
        scale = np.max(np.abs(r))
        assert np.max(np.abs(g - r)) <= RTOL * scale
    assert block_err(g_parts[2], r_parts[2]) < RTOL


def test_shg_mixed_precision_within_bound(engine_cls, oracle_mod, tb4):
    rng = np.random.default_rng(23)
    k = rng.random((6, 3))
    task = shg_task(precision=_abi.PRECISION_MIXED, omegas=np.linspace(0.0, 3.0, 13))
    with engine_cls(tb4, task) as eng:
        got = task.split(eng.point_values(k))[0]
    ref = task.split(oracle_mod.point_values(tb4, task, k))[0]
    assert block_err(got, ref) < MIXED_RTOL


def test_shg_invalid_widths_rejected(engine_cls, tb4):
    from wanniernlqg_b200._lib import EngineError
    task = shg_task()
    task.desc.shg_low_frequency_broadening = 0.0
    with pytest.raises(EngineError) as ei:
        engine_cls(tb4, task)
    assert ei.value.status == 1 and "finite and positive" in str(ei.value)


def test_shg_large_nw_matches_oracle(engine_cls, oracle_mod):
    """nw = 48: the SHG matrices live in the per-CTA global working set."""
    from wanniernlqg_b200.model import synthetic_orthogonal_model
    model = synthetic_orthogonal_model(48, 1, seed=9, full_position=True)
    task = shg_task(T=300.0, omegas=np.linspace(0.0, 3.0, 9), components=[(0, 1, 1), (2, 0, 0), (1, 1, 1)])
    k = np.random.default_rng(24).random((2, 3))
    with engine_cls(model, task) as eng:
        got = task.split(eng.point_values(k))[0]
    ref = task.split(oracle_mod.point_values(model, task, k))[0]
    assert block_err(got, ref) < RTOL


# ---- metric (nonorthogonal) SHG --------------------------------------------------------------

def _overlap_model(model, M):
    """The same model in a nonorthogonal basis: S = M^H M at R = 0, H' = M^H H M, A' = M^H A M."""
    import copy
    nw, nr = model.num_orbitals, model.num_r_vectors
    out = copy.deepcopy(model)
    home = int(np.where(np.all(model.r_vectors == 0, axis=0))[0][0])
    S = np.zeros((nw, nw, nr), dtype=np.complex128, order="F")
    S[:, :, home] = M.conj().T @ M
    out.overlap_r = S
    out.hamiltonian_r = np.asfortranarray(np.einsum("ji,jkr,kl->ilr", M.conj(), model.hamiltonian_r, M))
    out.position_r = np.asfortranarray(np.einsum("ji,jkar,kl->ilar", M.conj(), model.position_r, M))
    return out


def metric_task(*, T=300.0, mu=0.1, components=COMPONENTS, omegas=(0.1, 0.6, 1.4)):
    return _abi.TaskArrays([(_abi.SECOND_HARMONIC, components)], broadening_type=_abi.LORENTZIAN, broadening=0.03,
                           photon_energies=omegas, fermi_energy=mu, temperature=T, degeneracy_threshold=0.002,
                           shg_low_frequency_broadening=0.025, shg_intermediate_regularization=0.0,
                           denominator_regularization=0.01, shg_eta_correction=False)


@pytest.mark.parametrize("T", [0.0, 300.0])
def test_metric_shg_matches_oracle(engine_cls, oracle_mod, T):
    """Nonorthogonal model (constant non-unitary basis change of an orthogonal one): GPU metric SHG
    (metric_shg_kernel + shg_kernel) against the oracle term by term, and equal to the orthogonal
    model's SHG (basis invariance)."""
    from wanniernlqg_b200.model import synthetic_orthogonal_model
    base = synthetic_orthogonal_model(6, 1, seed=4, full_position=True)
    rng = np.random.default_rng(9)
    model = _overlap_model(base, np.eye(6) + 0.2 * (rng.standard_normal((6, 6)) + 1j * rng.standard_normal((6, 6))))
    task = metric_task(T=T)
    k = np.random.default_rng(5).random((6, 3))
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
    with engine_cls(base, task) as eng:
        orth = eng.point_values(k)
    ref = oracle_mod.point_values(model, task, k)
    g, r, o = task.split(got)[0], task.split(ref)[0], task.split(orth)[0]
    assert block_err(g, r) < RTOL
    assert block_err(g, o) < 1e-9


def test_metric_shg_identity_overlap_mesh(engine_cls, oracle_mod):
    """Identity overlap: the metric path's mesh integral equals the orthogonal path's and the oracle."""
    from wanniernlqg_b200.model import synthetic_orthogonal_model
    base = synthetic_orthogonal_model(5, 1, seed=6, full_position=True)
    model = _overlap_model(base, np.eye(5))
    task = metric_task(components=[(0, 0, 0), (1, 2, 2), (2, 0, 1)])
    mesh = (4, 3, 3)
    with engine_cls(model, task, max_batch=13) as eng:
        got = eng.integrate_mesh(mesh)
    with engine_cls(base, task) as eng:
        orth = eng.integrate_mesh(mesh)
    ref = oracle_mod.integrate_mesh(model, task, mesh)
    assert block_err(task.split(got)[0], task.split(ref)[0]) < RTOL
    assert block_err(task.split(got)[0], task.split(orth)[0]) < 1e-9


def test_metric_shg_preconditions(engine_cls):
    from wanniernlqg_b200._lib import EngineError
    from wanniernlqg_b200.model import synthetic_orthogonal_model
    model = _overlap_model(synthetic_orthogonal_model(4, 1, seed=1, full_position=True), np.eye(4))
    bad_corr = _abi.TaskArrays([(_abi.SECOND_HARMONIC, [(0, 0, 0)])], broadening=0.03, photon_energies=[0.5],
                               denominator_regularization=0.01, shg_intermediate_regularization=0.01,
                               shg_eta_correction=True)
    bad_eta = _abi.TaskArrays([(_abi.SECOND_HARMONIC, [(0, 0, 0)])], broadening=0.03, photon_energies=[0.5],
                              denominator_regularization=0.0, shg_intermediate_regularization=0.01,
                              shg_eta_correction=False)
    for task, msg in ((bad_corr, "ETA_CORRECTION_UNSUPPORTED"), (bad_eta, "POSITIVE_GEOMETRY_REQUIRED")):
        with pytest.raises(EngineError) as ei:
            engine_cls(model, task)
        assert ei.value.status == 1 and msg in str(ei.value)


def test_metric_shg_nw64_matches_oracle(engine_cls, oracle_mod):
    """64 orbitals with a k-dependent overlap S(R) (the SHG chi^xxx shape of the nonorthogonal
    workload): metric inputs and the SHG kernel's global working set against the oracle."""
    from wanniernlqg_b200.model import synthetic_nonorthogonal_model
    model = synthetic_nonorthogonal_model(64, 1, seed=7, full_position=True)
    task = metric_task(components=[(0, 0, 0), (1, 0, 1)], omegas=(0.4, 1.2), T=300.0, mu=0.0)
    k = np.random.default_rng(8).random((2, 3))
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
    ref = oracle_mod.point_values(model, task, k)
    assert block_err(task.split(got)[0], task.split(ref)[0]) < RTOL


def test_metric_shg_autotuned_grids_keep_results(engine_cls, oracle_mod):
    """The autotuner's grid choices for the metric input kernel (1, 2, 4 CTAs per SM) and the SHG
    kernel's global working set (the L2-resident grid, 1, 2 CTAs per SM) change no result: mesh
    sums before and after tuning agree to 1e-12, and the tuned point values match the oracle."""
    from wanniernlqg_b200.model import synthetic_nonorthogonal_model
    model = synthetic_nonorthogonal_model(64, 1, seed=9, full_position=True)
    task = metric_task(components=[(0, 0, 0)], omegas=(0.4, 1.2), T=0.0, mu=0.0)
    mesh = (8, 8, 8)
    with engine_cls(model, task, max_batch=256) as eng:
        before = eng.integrate_mesh(mesh, 0, 256)
        rep = eng.autotune(mesh, 0, 256)
        after = eng.integrate_mesh(mesh, 0, 256)
        k = np.random.default_rng(10).random((2, 3))
        got = eng.point_values(k)
    assert rep["metric_shg_grid"] > 0 and len(rep["metric_shg_grid_ms"]) == 3
    assert rep["shg_grid"] > 0 and len(rep["shg_grid_ms"]) == 3
    assert np.max(np.abs(after - before)) <= 1e-12 * np.max(np.abs(before))
    ref = oracle_mod.point_values(model, task, k)
    assert block_err(task.split(got)[0], task.split(ref)[0]) < RTOL
