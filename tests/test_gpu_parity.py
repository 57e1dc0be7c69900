"""GPU parity of the FP64 path against the CPU FP64 oracle, through the C ABI.

Tolerance: 1e-10 relative in the max norm over frequencies and components (relative to the
oracle's max norm), the plain-FP64 bar for this path.
"""
import numpy as np
import pytest

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import reference_workload_model, synthetic_orthogonal_model

pytestmark = pytest.mark.gpu
RTOL = 1e-10


def rel_err(got, ref):
    scale = np.max(np.abs(ref))
    return np.max(np.abs(got - ref)) / (scale if scale > 0 else 1.0)


@pytest.fixture(scope="module")
def engine_cls():
    from wanniernlqg_b200 import build
    build.build()
    from wanniernlqg_b200.engine import ResponseEngine
    return ResponseEngine


def nw4_task(kind=_abi.LORENTZIAN, width=0.02, nom=128, **kw):
    return _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.INJECTION_CURRENT, ["xyy"])],
                           broadening_type=kind, broadening=width, photon_energies=np.linspace(0, 3, nom), **kw)


def nw32_task(nom=512, **kw):
    return _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.BERRY_CURVATURE, ["xy"]),
                            (_abi.QUANTUM_METRIC, ["xx"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.01, photon_energies=np.linspace(0, 4, nom), **kw)


@pytest.mark.parametrize("name", ["nw4", "nw32"])
def test_spectrum_matches_oracle(engine_cls, oracle_mod, name):
    model = reference_workload_model(name)
    task = nw4_task() if name == "nw4" else nw32_task()
    rng = np.random.default_rng(11)
    k = rng.random((24, 3))
    with engine_cls(model, task) as eng:
        e, u = eng.spectrum(k)
    for i in range(k.shape[0]):
        eo, uo, _ = oracle_mod.kpoint_spectrum(model, k[i])
        assert np.max(np.abs(e[i] - eo)) < 1e-12 * max(1.0, np.abs(eo).max())
        # Gauge-invariant comparison of eigenvectors: |<u_gpu|u_oracle>| = 1 column by column.
        ov = np.abs(np.sum(u[i].conj() * uo, axis=0))
        assert np.max(np.abs(ov - 1.0)) < 1e-9


@pytest.mark.parametrize("name", ["nw4", "nw32"])
def test_point_values_match_oracle(engine_cls, oracle_mod, name):
    model = reference_workload_model(name)
    task = nw4_task() if name == "nw4" else nw32_task()
    rng = np.random.default_rng(12)
    k = rng.random((16, 3))
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
    ref = oracle_mod.point_values(model, task, k)
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < RTOL


@pytest.mark.parametrize("kind", [_abi.LORENTZIAN, _abi.GAUSSIAN])
def test_nw4_mesh_matches_oracle(engine_cls, oracle_mod, kind):
    model = reference_workload_model("nw4")
    task = nw4_task(kind=kind, width=0.02 if kind == _abi.LORENTZIAN else 0.04)
    mesh = (8, 8, 8)
    with engine_cls(model, task, max_batch=192) as eng:
        got = eng.integrate_mesh(mesh)
    ref = oracle_mod.integrate_mesh(model, task, mesh)
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < RTOL


def test_nw32_mesh_matches_oracle(engine_cls, oracle_mod):
    model = reference_workload_model("nw32")
    task = nw32_task(nom=96)
    mesh = (4, 4, 3)
    with engine_cls(model, task) as eng:
        got = eng.integrate_mesh(mesh)
    ref = oracle_mod.integrate_mesh(model, task, mesh)
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < RTOL


def test_full_shift_tensor_multi_pass(engine_cls, oracle_mod):
    """All 27 shift components and 27 injection components (several response passes)."""
    import itertools
    comps = ["".join(c) for c in itertools.product("xyz", repeat=3)]
    model = synthetic_orthogonal_model(8, 1, 4, full_position=True)
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, comps), (_abi.INJECTION_CURRENT, comps)],
                           broadening_type=_abi.GAUSSIAN, broadening=0.05, photon_energies=np.linspace(0.1, 2.5, 24))
    k = np.random.default_rng(13).random((8, 3))
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
    ref = oracle_mod.point_values(model, task, k)
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < RTOL


def test_sub_range_and_batches(engine_cls, oracle_mod):
    model = reference_workload_model("nw4")
    task = nw4_task(nom=32)
    mesh = (6, 5, 4)
    with engine_cls(model, task, max_batch=64) as eng:
        part = eng.integrate_mesh(mesh, 17, 101)
        whole = eng.integrate_mesh(mesh)
    assert rel_err(part, oracle_mod.integrate_mesh(model, task, mesh, 17, 101)) < RTOL
    assert rel_err(whole, oracle_mod.integrate_mesh(model, task, mesh)) < RTOL


def test_run_to_run_bitwise_deterministic(engine_cls):
    model = reference_workload_model("nw4")
    task = nw4_task()
    with engine_cls(model, task, max_batch=128) as eng:
        a = eng.integrate_mesh((8, 8, 4))
        b = eng.integrate_mesh((8, 8, 4))
    assert np.array_equal(a, b)


def test_nonfinite_model_rejected(engine_cls):
    from wanniernlqg_b200._lib import EngineError
    model = reference_workload_model("nw4")
    model.hamiltonian_r[0, 0, 3] = np.nan
    with pytest.raises(EngineError) as ei:
        engine_cls(model, nw4_task())
    assert ei.value.status == 3


def test_invalid_task_rejected(engine_cls):
    from wanniernlqg_b200._lib import EngineError
    model = reference_workload_model("nw4")
    with pytest.raises(EngineError) as ei:
        engine_cls(model, nw4_task(width=0.0))
    assert ei.value.status == 1


@pytest.mark.parametrize("name,mesh,batch", [("nw4", (5, 3, 4), 7), ("nw4", (16, 2, 3), 40), ("nw32", (9, 2, 2), 10)])
def test_staged_mesh_fourier_batches_crossing_lines(engine_cls, oracle_mod, name, mesh, batch):
    """The staged (separable) mesh contraction, with plan batches that start and end mid-line
    and mid-plane, equals the oracle's direct Fourier sum."""
    model = reference_workload_model(name)
    task = nw4_task(nom=24) if name == "nw4" else nw32_task(nom=24)
    with engine_cls(model, task, max_batch=batch) as eng:
        got = eng.integrate_mesh(mesh)
        part = eng.integrate_mesh(mesh, 3, int(np.prod(mesh)) - 2)
    ref = oracle_mod.integrate_mesh(model, task, mesh)
    ref_part = oracle_mod.integrate_mesh(model, task, mesh, 3, int(np.prod(mesh)) - 2)
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < RTOL
    for g, r in zip(task.split(part), task.split(ref_part)):
        assert rel_err(g, r) < RTOL


# Mixed path (FP32 per-k matrices; FP64 energies, denominators, occupations and k-sums).
# Stated bound: 1e-4 relative (max norm over frequencies/components, relative to the oracle's
# max norm) for every response; the bench workload's sigma^xyy target is 1e-4.
MIXED_RTOL = 1e-4


@pytest.mark.parametrize("name", ["nw4", "nw32"])
def test_mixed_point_values_within_bound(engine_cls, oracle_mod, name):
    model = reference_workload_model(name)
    task = (nw4_task(precision=_abi.PRECISION_MIXED) if name == "nw4"
            else nw32_task(precision=_abi.PRECISION_MIXED))
    k = np.random.default_rng(14).random((16, 3))
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
    ref = oracle_mod.point_values(model, task, k)
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < MIXED_RTOL


@pytest.mark.parametrize("name,mesh", [("nw4", (8, 8, 8)), ("nw32", (9, 4, 3))])
def test_mixed_mesh_within_bound(engine_cls, oracle_mod, name, mesh):
    model = reference_workload_model(name)
    task = (nw4_task(precision=_abi.PRECISION_MIXED) if name == "nw4"
            else nw32_task(nom=64, precision=_abi.PRECISION_MIXED))
    with engine_cls(model, task) as eng:
        got = eng.integrate_mesh(mesh)
    ref = oracle_mod.integrate_mesh(model, task, mesh)
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < MIXED_RTOL


@pytest.mark.parametrize("name", ["nw4", "nw32"])
def test_mixed_eigensolver_refined_to_fp64(engine_cls, oracle_mod, name, monkeypatch):
    """FP32 Jacobi + one FP64 Rayleigh-Ritz refinement reaches FP64-level eigenvalues.  The
    eigensolver is isolated by feeding it the FP64 CUDA-core Fourier sums."""
    monkeypatch.setenv("WNLQG_B200_DIRECT_FOURIER", "1")
    model = reference_workload_model(name)
    task = nw4_task(precision=_abi.PRECISION_MIXED) if name == "nw4" else nw32_task(precision=_abi.PRECISION_MIXED)
    k = np.random.default_rng(15).random((24, 3))
    with engine_cls(model, task) as eng:
        e, u = eng.spectrum(k)
    for i in range(k.shape[0]):
        eo, uo, _ = oracle_mod.kpoint_spectrum(model, k[i])
        err = np.max(np.abs(e[i] - eo))
        assert err < 1e-11 * max(1.0, np.abs(eo).max()), (i, err, np.min(np.diff(eo)))
        ov = np.abs(np.sum(u[i].conj() * uo, axis=0))
        assert np.max(np.abs(ov - 1.0)) < 1e-8, (i, np.max(np.abs(ov - 1.0)), np.min(np.diff(eo)))


@pytest.mark.parametrize("nw", [17, 24, 31])
@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_team_eigensolver_below_32_orbitals(engine_cls, oracle_mod, nw, precision, monkeypatch):
    """17 to 31 orbitals run the 128-thread team eigensolver on np = nw or nw + 1 < 32 (the FP64
    refinement's DMMA row blocks masked at np, a zero-padded row and column for odd nw).  Spectra
    at arbitrary points against the oracle (eigenvalues to 1e-11 of the largest |E|, eigenvectors
    of bands 1 meV from their neighbours parallel to 1e-8), point values and a warm-started mesh
    block to 1e-10 (FP64) or the mixed bound.  The FP64 CUDA-core Fourier sums
    (WNLQG_B200_DIRECT_FOURIER=1) isolate the eigensolver from the tensor-core Fourier.  The
    seeds keep every band gap above 10 meV at the test's points (smallest 17-32 meV), so the
    comparison does not rest on the conditioning of near-degenerate pairs."""
    monkeypatch.setenv("WNLQG_B200_DIRECT_FOURIER", "1")
    model = synthetic_orthogonal_model(nw, 1, seed={17: 87, 24: 92, 31: 101}[nw], full_position=True)
    task = nw32_task(nom=64, precision=precision)
    k = np.random.default_rng(nw).random((8, 3))
    mesh = (6, 5, 4)
    with engine_cls(model, task) as eng:
        e, u = eng.spectrum(k)
        pts = eng.point_values(k)
        got_mesh = eng.integrate_mesh(mesh, 10, 110)
    for i in range(k.shape[0]):
        eo, uo, _ = oracle_mod.kpoint_spectrum(model, k[i])
        assert np.max(np.abs(e[i] - eo)) < 1e-11 * max(1.0, np.abs(eo).max())
        gaps = np.diff(eo)
        isolated = np.ones(nw, dtype=bool)
        isolated[:-1] &= gaps > 1e-3
        isolated[1:] &= gaps > 1e-3
        ov = np.abs(np.sum(u[i].conj() * uo, axis=0))
        assert np.max(np.abs(ov - 1.0)[isolated]) < 1e-8
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    for g, r in zip(task.split(pts), task.split(oracle_mod.point_values(model, task, k))):
        assert rel_err(g, r) < tol
    for g, r in zip(task.split(got_mesh), task.split(oracle_mod.integrate_mesh(model, task, mesh, 10, 110))):
        assert rel_err(g, r) < tol


@pytest.mark.parametrize("name", ["nw4", "nw32"])
def test_fp64_warp_eigensolver_matches_cta_jacobi(engine_cls, name, monkeypatch):
    """FP64 path up to 32 orbitals: FP32 warp Jacobi as preconditioner, then FP64 sweeps to the
    CTA Jacobi's stopping rule.  Same spectrum as the FP64 CTA Jacobi (WNLQG_B200_CTA_EIGH=1) to
    1e-13 of the largest |E|, eigenvectors equal up to phase, and the same mesh response to 1e-12."""
    model = reference_workload_model(name)
    task = nw4_task() if name == "nw4" else nw32_task()
    k = np.random.default_rng(17).random((32, 3))
    mesh = (6, 6, 6)
    with engine_cls(model, task) as eng:
        e_w, u_w = eng.spectrum(k)
        m_w = eng.integrate_mesh(mesh)
    monkeypatch.setenv("WNLQG_B200_CTA_EIGH", "1")
    with engine_cls(model, task) as eng:
        e_c, u_c = eng.spectrum(k)
        m_c = eng.integrate_mesh(mesh)
    assert np.max(np.abs(e_w - e_c)) < 1e-13 * max(1.0, np.abs(e_c).max())
    for i in range(k.shape[0]):
        gaps = np.diff(e_c[i])
        ov = np.abs(np.sum(u_w[i].conj() * u_c[i], axis=0))
        isolated = np.ones(e_c.shape[1], dtype=bool)
        isolated[:-1] &= gaps > 1e-6
        isolated[1:] &= gaps > 1e-6
        assert np.max(np.abs(ov[isolated] - 1.0)) < 1e-10
    for g, r in zip(task.split(m_w), task.split(m_c)):
        assert rel_err(g, r) < 1e-12


@pytest.mark.parametrize("name,precision,slices", [("nw4", _abi.PRECISION_FP64, 7), ("nw32", _abi.PRECISION_FP64, 7),
                                                   ("nw4", _abi.PRECISION_MIXED, 4), ("nw32", _abi.PRECISION_MIXED, 4)])
def test_tensor_core_fourier_eigenvalues_within_slice_bound(engine_cls, oracle_mod, name, precision, slices):
    """Arbitrary k-points take the tcgen05 Fourier on S int8 slices: H(k) carries at most
    16 sqrt(2 NR) 2^(-7S) of each channel column's largest |H(R)|, and so do the eigenvalues
    (Weyl); the FP64 path (S = 7) stays at the FP64 bar."""
    model = reference_workload_model(name)
    task = nw4_task(precision=precision) if name == "nw4" else nw32_task(precision=precision)
    k = np.random.default_rng(16).random((24, 3))
    with engine_cls(model, task) as eng:
        e, _ = eng.spectrum(k)
    colmax = np.max(np.abs(model.hamiltonian_r), axis=2)
    bound = 16.0 * np.sqrt(2 * model.num_r_vectors) * 2.0 ** (-7 * slices) * np.linalg.norm(colmax, 2)
    for i in range(k.shape[0]):
        eo, _, _ = oracle_mod.kpoint_spectrum(model, k[i])
        assert np.max(np.abs(e[i] - eo)) < max(bound, 1e-11 * max(1.0, np.abs(eo).max()))


def test_mesh_weighted_sum_contiguous_and_scattered(engine_cls, oracle_mod):
    """Host mesh indices + weights: a contiguous run (staged path) equals the lane sum, and a
    scattered representative set with multiplicities equals the weighted oracle point sum."""
    model = reference_workload_model("nw4")
    task = nw4_task(nom=32)
    mesh = (8, 6, 4)
    nk = int(np.prod(mesh))
    rng = np.random.default_rng(16)
    with engine_cls(model, task, max_batch=50) as eng:
        idx = np.arange(10, 150)
        got = eng.mesh_weighted_sum(mesh, idx, np.full(idx.size, 1.0 / nk))
        ref = eng.integrate_mesh(mesh, 10, 150)
        assert rel_err(got, ref) < 1e-13
        sidx = rng.choice(nk, 37, replace=False)
        w = rng.integers(1, 9, sidx.size) / nk
        got2 = eng.mesh_weighted_sum(mesh, sidx, w)
    k = np.stack([(sidx % 8) / 8, ((sidx // 8) % 6) / 6, (sidx // 48) / 4], axis=1)
    ref2 = (oracle_mod.point_values(model, task, k) * w[:, None]).sum(axis=0)
    for g, r in zip(task.split(got2), task.split(ref2)):
        assert rel_err(g, r) < RTOL


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
@pytest.mark.parametrize("temperature", [0.0, 50.0])
def test_ahc_and_berry_dipole_match_oracle(engine_cls, oracle_mod, precision, temperature):
    """Fermi-axis responses: the intrinsic AHC at T = 0 (the only temperature the reference's AHC
    accepts), the linear transport Berry channel at T > 0 (with an interband rate), and the Berry
    dipole at a degeneracy threshold below every gap of the sampled spectra."""
    model = synthetic_orthogonal_model(8, 1, 6, full_position=True)
    hall = _abi.INTRINSIC_AHC if temperature == 0.0 else _abi.LINEAR_TRANSPORT_BERRY
    task = _abi.TaskArrays([(hall, ["xy", "zx"]), (_abi.BERRY_DIPOLE, ["xyz", "xzx", "yzy"])],
                           fermi_energies=[-0.5, 0.0, 0.5], temperature=temperature,
                           fermi_surface_broadening=0.05, precision=precision, degeneracy_threshold=1e-8,
                           linear_transport_gamma_inter=0.0 if temperature == 0.0 else 0.01)
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    k = np.random.default_rng(17).random((12, 3))
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
        gm = eng.integrate_mesh((6, 4, 4))
    ref = oracle_mod.point_values(model, task, k)
    rm = oracle_mod.integrate_mesh(model, task, (6, 4, 4))
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < tol
    for g, r in zip(task.split(gm), task.split(rm)):
        assert rel_err(g, r) < tol


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
@pytest.mark.parametrize("kind", [_abi.GAUSSIAN, _abi.LORENTZIAN])
def test_jerk_matches_oracle(engine_cls, oracle_mod, precision, kind):
    import itertools
    comps = ["".join(c) for c in itertools.product("xyz", repeat=4)][::7]
    model = synthetic_orthogonal_model(8, 1, 9, full_position=True)
    task = _abi.TaskArrays([(_abi.JERK_CURRENT, comps)], broadening_type=kind, broadening=0.05,
                           photon_energies=np.linspace(0.2, 3.0, 20), precision=precision)
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    k = np.random.default_rng(18).random((10, 3))
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
        gm = eng.integrate_mesh((5, 3, 3))
    ref = oracle_mod.point_values(model, task, k)
    rm = oracle_mod.integrate_mesh(model, task, (5, 3, 3))
    assert rel_err(got, ref) < tol
    assert rel_err(gm, rm) < tol


@pytest.mark.parametrize("nw,rmax", [(8, 1), (24, 1)])
def test_nonorthogonal_generalized_spectrum_matches_oracle(engine_cls, oracle_mod, nw, rmax):
    from wanniernlqg_b200.model import synthetic_nonorthogonal_model
    model = synthetic_nonorthogonal_model(nw, rmax, 5)
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"])], broadening_type=_abi.LORENTZIAN, broadening=0.01)
    k = np.random.default_rng(19).random((12, 3))
    with engine_cls(model, task) as eng:
        e, c = eng.spectrum(k)
    for i in range(k.shape[0]):
        eo, co, _ = oracle_mod.kpoint_spectrum(model, k[i])
        assert np.max(np.abs(e[i] - eo)) < 1e-11 * max(1.0, np.abs(eo).max())
        ph = np.exp(2j * np.pi * (model.r_vectors.T @ k[i])) / model.r_degeneracies
        sk = np.einsum("ijr,r->ij", model.overlap_r, ph)
        ov = np.abs(np.sum(c[i].conj() * (sk @ co), axis=0))
        assert np.max(np.abs(ov - 1.0)) < 1e-9


def test_nonorthogonal_other_responses_rejected_and_indefinite_overlap_reported(engine_cls):
    """Nonorthogonal models take the shift and injection currents; other kinds are refused at plan
    creation, and a non-positive-definite S(k) is reported, never silently used."""
    from wanniernlqg_b200._lib import EngineError
    from wanniernlqg_b200.model import synthetic_nonorthogonal_model
    model = synthetic_nonorthogonal_model(6, 1, 2)
    with pytest.raises(EngineError) as ei:
        engine_cls(model, _abi.TaskArrays([(_abi.QUANTUM_METRIC, ["xx"])]))
    assert ei.value.status == 6
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"])])
    bad = synthetic_nonorthogonal_model(6, 1, 2)
    home = int(np.where(np.all(bad.r_vectors == 0, axis=0))[0][0])
    bad.overlap_r[:, :, home] -= 2.0 * np.eye(6)       # S(k) = -I + small: not positive definite
    with engine_cls(bad, task) as eng:
        with pytest.raises(EngineError) as ei:
            eng.spectrum(np.array([[0.1, 0.2, 0.3]]))
        assert ei.value.status == 1


def _nonorth_full_position(nw, seed):
    """Nonorthogonal synthetic model with the full off-diagonal position operator."""
    from wanniernlqg_b200.model import synthetic_nonorthogonal_model
    m = synthetic_nonorthogonal_model(nw, 1, seed)
    full = synthetic_orthogonal_model(nw, 1, seed, full_position=True)
    m.position_r = full.position_r
    return m


def _currents_task(precision=_abi.PRECISION_FP64, kind=_abi.LORENTZIAN, width=0.03):
    return _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy", "zxy", "yzz"]), (_abi.INJECTION_CURRENT, ["xyy", "zzx"])],
                           broadening_type=kind, broadening=width, photon_energies=np.linspace(0, 3, 40),
                           precision=precision)


@pytest.mark.parametrize("nw,precision", [(8, _abi.PRECISION_FP64), (8, _abi.PRECISION_MIXED),
                                          (32, _abi.PRECISION_FP64)])
def test_nonorthogonal_currents_match_oracle(engine_cls, oracle_mod, nw, precision):
    """Metric geometry (nonorth_geometry_kernel) + the shared pair contraction against the oracle."""
    model = _nonorth_full_position(nw, 7)
    task = _currents_task(precision)
    k = np.random.default_rng(41).random((5, 3))
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
    ref = oracle_mod.point_values(model, task, k)
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < tol


def test_nonorthogonal_mesh_and_identity_overlap(engine_cls, oracle_mod):
    """Mesh lanes for a nonorthogonal model against the oracle, and an identity overlap giving the
    orthogonal engine's result (two different GPU geometries of one model)."""
    import copy
    model = _nonorth_full_position(8, 3)
    task = _currents_task(kind=_abi.GAUSSIAN, width=0.06)
    mesh = (5, 4, 3)
    with engine_cls(model, task, max_batch=17) as eng:
        got = eng.integrate_mesh(mesh)
    ref = oracle_mod.integrate_mesh(model, task, mesh)
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < RTOL
    orth = synthetic_orthogonal_model(8, 1, 3, full_position=True)
    ident = copy.deepcopy(orth)
    home = int(np.where(np.all(orth.r_vectors == 0, axis=0))[0][0])
    ident.overlap_r = np.zeros((8, 8, orth.num_r_vectors), dtype=np.complex128, order="F")
    ident.overlap_r[:, :, home] = np.eye(8)
    k = np.random.default_rng(42).random((4, 3))
    with engine_cls(orth, task) as eng:
        a = eng.point_values(k)
    with engine_cls(ident, task) as eng:
        b = eng.point_values(k)
    assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(a))


# ---- orbital counts above 32: matrices in a per-CTA global working set ---------------------------

@pytest.mark.parametrize("nw,precision", [(48, _abi.PRECISION_FP64), (64, _abi.PRECISION_FP64),
                                          (64, _abi.PRECISION_MIXED)])
def test_large_nw_point_values_match_oracle(engine_cls, oracle_mod, nw, precision):
    model = synthetic_orthogonal_model(nw, 1, seed=nw, full_position=True)
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy", "zxz"]), (_abi.BERRY_CURVATURE, ["xy"]),
                            (_abi.QUANTUM_METRIC, ["xx"]), (_abi.INJECTION_CURRENT, ["xyy"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.02, photon_energies=np.linspace(0, 3, 24),
                           precision=precision)
    k = np.random.default_rng(nw).random((3, 3))
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
    ref = oracle_mod.point_values(model, task, k)
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < tol


def test_large_nw_mesh_matches_oracle(engine_cls, oracle_mod):
    model = synthetic_orthogonal_model(64, 1, seed=5, full_position=True)
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.QUANTUM_METRIC, ["xx"])],
                           broadening_type=_abi.GAUSSIAN, broadening=0.05, photon_energies=np.linspace(0, 3, 16))
    mesh = (4, 3, 2)
    with engine_cls(model, task, max_batch=10) as eng:
        got = eng.integrate_mesh(mesh)
    ref = oracle_mod.integrate_mesh(model, task, mesh)
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < RTOL


@pytest.mark.parametrize("nw", [96, 128])
def test_large_nw_spectrum_matches_oracle(engine_cls, oracle_mod, nw):
    model = synthetic_orthogonal_model(nw, 1, seed=3)
    task = _abi.TaskArrays([(_abi.QUANTUM_METRIC, ["xx"])])
    k = np.random.default_rng(4).random((4, 3))
    with engine_cls(model, task) as eng:
        e, _ = eng.spectrum(k)
    for i in range(k.shape[0]):
        eo, _, _ = oracle_mod.kpoint_spectrum(model, k[i])
        assert np.max(np.abs(e[i] - eo)) < 1e-11 * max(1.0, np.abs(eo).max())


@pytest.mark.parametrize("nw", [64, 80])
def test_large_nw_nonorthogonal_spectrum_matches_oracle(engine_cls, oracle_mod, nw):
    from wanniernlqg_b200.model import synthetic_nonorthogonal_model
    model = synthetic_nonorthogonal_model(nw, 1, seed=2)
    task = _abi.TaskArrays([(_abi.INJECTION_CURRENT, ["xyy"])])
    k = np.random.default_rng(6).random((3, 3))
    with engine_cls(model, task) as eng:
        e, _ = eng.spectrum(k)
    for i in range(k.shape[0]):
        eo, _, _ = oracle_mod.kpoint_spectrum(model, k[i])
        assert np.max(np.abs(e[i] - eo)) < 1e-10 * max(1.0, np.abs(eo).max())


@pytest.mark.parametrize("name,window,mu", [("nw4", 1, 0.0), ("nw4", 2, 0.0), ("nw4", 1, 5.0), ("nw32", 4, 0.0),
                                             ("nw32", 3, -0.3), ("nw32", 100, 0.0)])
def test_band_window_matches_oracle(engine_cls, oracle_mod, name, window, mu):
    """band_window_size restricts the shift/injection pairs to bands around mu (widened to whole
    degeneracy groups); a window past the spectrum edge leaves no pairs."""
    model = reference_workload_model(name)
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.INJECTION_CURRENT, ["xyy"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.02, photon_energies=np.linspace(0, 3, 32),
                           fermi_energy=mu, band_window_size=window, degeneracy_threshold=0.05)
    full = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.INJECTION_CURRENT, ["xyy"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.02, photon_energies=np.linspace(0, 3, 32),
                           fermi_energy=mu)
    k = np.random.default_rng(31).random((6, 3))
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
    ref = oracle_mod.point_values(model, task, k)
    for g, r in zip(task.split(got), task.split(ref)):
        scale = np.max(np.abs(r))
        assert np.max(np.abs(g - r)) <= RTOL * max(scale, 1e-300)
    ref_full = oracle_mod.point_values(model, full, k)
    if 2 * window > model.num_orbitals:
        assert np.array_equal(ref, ref_full)
    elif mu > 4.0:
        assert np.all(ref == 0)
    else:
        assert not np.allclose(ref, ref_full)


def test_kslice_map_on_gpu_matches_oracle(engine_cls, oracle_mod):
    """A Berry-curvature / metric k-slice through one batched device call."""
    from wanniernlqg_b200.kslice import kslice_map
    model = reference_workload_model("nw32")
    task = _abi.TaskArrays([(_abi.BERRY_CURVATURE, ["xy"]), (_abi.QUANTUM_METRIC, ["xx"])])
    args = ([12, 9], [0.0, 0.0, 0.1], [1.0, 0.0, 0.0], [0.0, 1.0, 0.0])
    with engine_cls(model, task) as eng:
        got = kslice_map(eng.point_values, *args)
    ref = kslice_map(lambda k: oracle_mod.point_values(model, task, k), *args)
    assert rel_err(got, ref) < RTOL


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_eval_mesh_many_uneven_models(engine_cls, oracle_mod, precision):
    """Models of different orbital counts (half Kramers-doubled with an O(1e-3 eV) splitting) in
    one concurrent call: each result equals the model's own evaluation and the oracle, on both
    precision paths (the mixed path's FP64 refinement resolves the near-degenerate pairs)."""
    import torch
    from wanniernlqg_b200.engine import integrate_meshes_many
    from wanniernlqg_b200.model import kramers_doubled_model
    models = []
    for i, nw in enumerate([6, 8, 12, 16]):
        base = synthetic_orthogonal_model(nw, 1, seed=20 + i, full_position=True)
        models.append(kramers_doubled_model(base, 1e-3, seed=i) if i % 2 else base)
    # Finite-temperature Hall response as the reference computes it (the linear transport Berry
    # channel); the Berry dipole at a threshold that counts the O(1e-3 eV) Kramers splittings as
    # isolated (the reference's default 2e-3 eV would refuse these models).
    task = _abi.TaskArrays([(_abi.LINEAR_TRANSPORT_BERRY, ["xy"]), (_abi.BERRY_DIPOLE, ["xzz"])],
                           fermi_energies=[-0.5, 0.0, 0.5], temperature=50.0, degeneracy_threshold=1e-9,
                           precision=precision)
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    engines = [engine_cls(m, task) for m in models]
    try:
        meshes = [(6, 5, 4), (4, 4, 4), (5, 3, 3), (3, 3, 4)]
        ranges = [(0, int(np.prod(ms))) for ms in meshes]
        outs = [torch.zeros(2 * e.value_count, dtype=torch.float64, device="cuda") for e in engines]
        integrate_meshes_many(engines, meshes, ranges, [o.data_ptr() for o in outs])
        torch.cuda.synchronize()
        for e, m, ms, o in zip(engines, models, meshes, outs):
            got = o.cpu().numpy().view(np.complex128)
            single = e.integrate_mesh(ms)
            assert np.array_equal(got, single)
            ref = oracle_mod.integrate_mesh(m, task, ms)
            for g, r in zip(task.split(got), task.split(ref)):
                assert rel_err(g, r) < tol
    finally:
        for e in engines:
            e.close()


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_plans_of_different_sizes_share_kernels(engine_cls, oracle_mod, precision):
    """A smaller plan created after a larger one leaves the larger one usable: kernel attributes
    (dynamic shared memory limits) are per kernel, not per plan."""
    big = reference_workload_model("nw32")
    small = synthetic_orthogonal_model(4, 1, seed=3, full_position=True)
    task = nw32_task(nom=64, precision=precision)
    k = np.random.default_rng(21).random((8, 3))
    with engine_cls(big, task) as eng_big:
        with engine_cls(small, task) as eng_small:
            eng_small.point_values(k)
            got = eng_big.point_values(k)
    ref = oracle_mod.point_values(big, task, k)
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < tol


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_eigensolver_team_sizes_agree(engine_cls, oracle_mod, precision, monkeypatch):
    """Eigensolver stages with one, two or four warps per matrix give the same spectrum (to
    rounding) and the same mesh responses on the nw = 32 workload."""
    model = reference_workload_model("nw32")
    task = nw32_task(nom=64, precision=precision)
    k = np.random.default_rng(18).random((16, 3))
    res = {}
    for team in ("32", "64", "128"):
        monkeypatch.setenv("WNLQG_B200_EIGH_TEAM", team)
        with engine_cls(model, task) as eng:
            res[team] = (eng.spectrum(k)[0], eng.integrate_mesh((6, 5, 4)))
    e32, m32 = res["32"]
    tol = 1e-11 if precision == _abi.PRECISION_FP64 else 1e-6
    for team in ("64", "128"):
        e, m = res[team]
        assert np.max(np.abs(e - e32)) < 1e-12 * np.abs(e32).max()
        for g, r in zip(task.split(m), task.split(m32)):
            assert rel_err(g, r) < tol


@pytest.mark.parametrize("nw,precision", [(48, _abi.PRECISION_MIXED), (64, _abi.PRECISION_FP64),
                                          (96, _abi.PRECISION_FP64), (128, _abi.PRECISION_MIXED)])
def test_large_nw_mixed_precision_eigensolver_matches_cta_jacobi(engine_cls, nw, precision, monkeypatch):
    """Above 32 orbitals (the FP64 path from 60 orbitals): FP32 CTA Jacobi + FP64 CTA refinement
    (shared memory at 48 and 64, a global working set for the FP64 stage at 96 and for both at
    128) against the FP64 CTA Jacobi
    (WNLQG_B200_CTA_EIGH=1): spectra to 1e-12 (FP64 path) / 1e-11 (mixed path, one FP64 sweep)
    of max |E|, FP64 mesh responses to 1e-11.  Both engines take the FP64 CUDA-core Fourier sums,
    which isolates the eigensolver from the mixed path's 4-slice tensor-core Fourier."""
    monkeypatch.setenv("WNLQG_B200_DIRECT_FOURIER", "1")
    model = synthetic_orthogonal_model(nw, 1, seed=nw + 1, full_position=True)
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.QUANTUM_METRIC, ["xx"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.03, photon_energies=np.linspace(0, 3, 16),
                           precision=precision)
    ref_task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.QUANTUM_METRIC, ["xx"])],
                               broadening_type=_abi.LORENTZIAN, broadening=0.03, photon_energies=np.linspace(0, 3, 16))
    k = np.random.default_rng(nw).random((6, 3))
    mesh = (3, 2, 2)
    with engine_cls(model, task) as eng:
        e, _ = eng.spectrum(k)
        m = eng.integrate_mesh(mesh)
    monkeypatch.setenv("WNLQG_B200_CTA_EIGH", "1")
    with engine_cls(model, ref_task) as eng:
        e_ref, _ = eng.spectrum(k)
        m_ref = eng.integrate_mesh(mesh)
    etol = 1e-12 if precision == _abi.PRECISION_FP64 else 1e-11
    assert np.max(np.abs(e - e_ref)) < etol * np.abs(e_ref).max()
    rtol = 1e-11 if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    for g, r in zip(task.split(m), ref_task.split(m_ref)):
        assert rel_err(g, r) < rtol


@pytest.mark.parametrize("nw", [1, 2, 3, 5])
@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_small_orbital_counts_match_oracle(engine_cls, oracle_mod, nw, precision):
    """One to five orbitals (odd counts padded to an even Jacobi size, single-band models with
    no transitions): point values and the spectrum against the oracle."""
    model = synthetic_orthogonal_model(nw, 1, seed=30 + nw, full_position=True)
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.QUANTUM_METRIC, ["xx"]), (_abi.BERRY_CURVATURE, ["xy"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.05, photon_energies=np.linspace(0, 3, 12),
                           precision=precision)
    k = np.random.default_rng(nw).random((5, 3))
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
        e, _ = eng.spectrum(k)
    ref = oracle_mod.point_values(model, task, k)
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < tol
    for i in range(k.shape[0]):
        eo, _, _ = oracle_mod.kpoint_spectrum(model, k[i])
        assert np.max(np.abs(e[i] - eo)) < 1e-6 * max(1.0, np.abs(eo).max())


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_band_selection_matches_oracle(engine_cls, oracle_mod, precision):
    """Explicit interband selection (conduction, valence groups, 1-based): point values and a mesh
    against the oracle (transition threshold on, applied per selection as in the reference), and
    the plan-time checks of the groups."""
    from wanniernlqg_b200._lib import EngineError
    model = reference_workload_model("nw32")
    sel = ([17, 18, 19, 20, 22], [10, 12, 13, 14, 15, 16])
    task = nw32_task(nom=48, precision=precision, band_selection=sel)
    k = np.random.default_rng(19).random((8, 3))
    mesh = (4, 3, 3)
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
        got_mesh = eng.integrate_mesh(mesh)
    ref = oracle_mod.point_values(model, task, k)
    ref_mesh = oracle_mod.integrate_mesh(model, task, mesh)
    tol = RTOL if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < tol
    for g, r in zip(task.split(got_mesh), task.split(ref_mesh)):
        assert rel_err(g, r) < tol
    for bad, status in ((([1, 2], [2, 3]), 1), (([40], [1]), 1)):
        with pytest.raises(EngineError) as ei:
            engine_cls(model, nw32_task(nom=8, band_selection=bad))
        assert ei.value.status == status
    with pytest.raises(EngineError) as ei:
        engine_cls(model, nw32_task(nom=8, band_selection=([3], [1]), band_window_size=4))
    assert ei.value.status == 6


def test_convention_one_matches_oracle(engine_cls, oracle_mod):
    """Wannier-center Convention I (centred connection, R + tau_j - tau_i displacement tiles; the
    D(k) similarity cancels in the band frame and is applied to the returned eigenvectors):
    point values, a mesh and canonical eigenvectors against the oracle on a non-cubic lattice;
    models without an R = 0 block and models with an overlap are rejected."""
    import copy
    from wanniernlqg_b200._lib import EngineError
    from wanniernlqg_b200.model import synthetic_nonorthogonal_model
    model = copy.deepcopy(synthetic_orthogonal_model(6, 1, seed=14, full_position=True))
    model.lattice = np.asfortranarray(np.array([[3.1, 0.0, 0.0], [0.9, 2.7, 0.0], [0.4, 0.6, 3.5]]))
    resp = [(_abi.SHIFT_CURRENT, ["xyy", "zxz"]), (_abi.INJECTION_CURRENT, ["xyy"]),
            (_abi.BERRY_CURVATURE, ["xy"]), (_abi.QUANTUM_METRIC, ["xz"]), (_abi.SECOND_HARMONIC, [(0, 1, 1)])]
    task = _abi.TaskArrays(resp, broadening_type=_abi.LORENTZIAN, broadening=0.05, photon_energies=np.linspace(0.1, 2.5, 8),
                           wannier_center_convention="I", shg_intermediate_regularization=0.04)
    k = np.random.default_rng(21).random((6, 3))
    mesh = (4, 3, 3)
    with engine_cls(model, task) as eng:
        got = eng.point_values(k)
        got_mesh = eng.integrate_mesh(mesh)
        _, u = eng.spectrum(k)
    ref = oracle_mod.point_values(model, task, k)
    ref_mesh = oracle_mod.integrate_mesh(model, task, mesh)
    for g, r in zip(task.split(got), task.split(ref)):
        assert rel_err(g, r) < RTOL
    for g, r in zip(task.split(got_mesh), task.split(ref_mesh)):
        assert rel_err(g, r) < RTOL
    for i in range(k.shape[0]):
        _, uo, _ = oracle_mod.kpoint_spectrum(model, k[i], "I")
        assert np.max(np.abs(u[i] - uo)) < 1e-9
    shifted = copy.deepcopy(model)
    shifted.r_vectors = np.asfortranarray(shifted.r_vectors + np.array([[5], [0], [0]]))
    with pytest.raises(EngineError) as ei:
        engine_cls(shifted, task)
    assert ei.value.status == 1
    with pytest.raises(EngineError) as ei:
        engine_cls(synthetic_nonorthogonal_model(4, 1, seed=2),
                   _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"])], wannier_center_convention="I"))
    assert ei.value.status == 6


@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_morton_ordered_points_match_caller_order(engine_cls, oracle_mod, precision, monkeypatch):
    """Arbitrary k-point batches are evaluated in Morton order (warm-started eigensolver) and
    written back in the caller's order: per-point values and weighted sums agree with the
    caller-order evaluation (WNLQG_B200_POINT_ORDER=0) to 1e-11 (FP64 path; 1e-6 mixed path) and
    with the oracle row by row."""
    model = reference_workload_model("nw32")
    task = nw32_task(nom=64, precision=precision)
    rng = np.random.default_rng(44)
    k = rng.random((1500, 3)) * 2.0 - 0.5       # outside [0, 1) too: the order uses k mod 1
    w = rng.random(1500)
    with engine_cls(model, task) as eng:
        vals = eng.point_values(k)
        wsum = eng.weighted_sum(k, w)
    monkeypatch.setenv("WNLQG_B200_POINT_ORDER", "0")
    with engine_cls(model, task) as eng:
        vals0 = eng.point_values(k)
        wsum0 = eng.weighted_sum(k, w)
    tol = 1e-11 if precision == _abi.PRECISION_FP64 else 1e-6
    for g, r in zip(task.split(vals), task.split(vals0)):
        assert rel_err(g, r) < tol
    assert rel_err(wsum, wsum0) < tol
    pick = rng.choice(1500, 12, replace=False)
    ref = oracle_mod.point_values(model, task, k[pick])
    for g, r in zip(task.split(vals[pick]), task.split(ref)):
        assert rel_err(g, r) < (RTOL if precision == _abi.PRECISION_FP64 else 1e-4)


@pytest.mark.parametrize("nw,precision", [(48, _abi.PRECISION_MIXED), (64, _abi.PRECISION_FP64)])
def test_large_nw_warm_started_ranges_match_cta_jacobi(engine_cls, nw, precision, monkeypatch):
    """Above 32 orbitals each FP32 CTA takes a contiguous range of points and warm-starts along
    it (mesh runs, Morton-ordered point batches): a 2048-point mesh block and a 3000-point
    weighted sum agree with the FP64 CTA Jacobi (WNLQG_B200_CTA_EIGH=1) to 1e-11 (FP64 path) or
    the mixed path's bound."""
    monkeypatch.setenv("WNLQG_B200_DIRECT_FOURIER", "1")
    model = synthetic_orthogonal_model(nw, 1, seed=nw + 5, full_position=True)
    kw = dict(broadening_type=_abi.LORENTZIAN, broadening=0.03, photon_energies=np.linspace(0, 3, 16))
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.QUANTUM_METRIC, ["xx"])], precision=precision, **kw)
    ref_task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.QUANTUM_METRIC, ["xx"])], **kw)
    rng = np.random.default_rng(nw + 9)
    k = rng.random((3000, 3))
    w = rng.random(3000) / 3000
    mesh = (16, 16, 16)
    with engine_cls(model, task) as eng:
        m = eng.integrate_mesh(mesh, 1024, 3072)
        s = eng.weighted_sum(k, w)
    monkeypatch.setenv("WNLQG_B200_CTA_EIGH", "1")
    with engine_cls(model, ref_task) as eng:
        m_ref = eng.integrate_mesh(mesh, 1024, 3072)
        s_ref = eng.weighted_sum(k, w)
    rtol = 1e-11 if precision == _abi.PRECISION_FP64 else MIXED_RTOL
    for g, r in zip(task.split(m), task.split(m_ref)):
        assert rel_err(g, r) < rtol
    for g, r in zip(task.split(s), task.split(s_ref)):
        assert rel_err(g, r) < rtol


def test_wide_fp64_response_matches(engine_cls, oracle_mod, monkeypatch):
    """The 512-thread FP64 response kernel (WNLQG_B200_RESPONSE_WIDE=1) gives the 256-thread
    kernel's mesh sums to 1e-12 (only the order of the per-point block sums changes) and the
    oracle's point values."""
    model = reference_workload_model("nw32")
    task = nw32_task(nom=512)
    k = np.random.default_rng(61).random((12, 3))
    with engine_cls(model, task) as eng:
        base = eng.integrate_mesh((8, 8, 8))
    monkeypatch.setenv("WNLQG_B200_RESPONSE_WIDE", "1")
    with engine_cls(model, task) as eng:
        wide = eng.integrate_mesh((8, 8, 8))
        pts = eng.point_values(k)
    for g, r in zip(task.split(wide), task.split(base)):
        assert rel_err(g, r) < 1e-12
    ref = oracle_mod.point_values(model, task, k)
    for g, r in zip(task.split(pts), task.split(ref)):
        assert rel_err(g, r) < RTOL


@pytest.mark.parametrize("nw", [7, 40, 64])
def test_nonorthogonal_mixed_path_cholesky_reduction(engine_cls, oracle_mod, nw, monkeypatch):
    """Nonorthogonal models on the mixed path: FP64 Cholesky reduction C = L^-1 H L^-H, the
    orthogonal mixed-precision stages on C (team stages at 7 orbitals, CTA stages at 40 and 64),
    U = L^-H V.  Eigenvalues to 1e-11 of max |E| against the oracle's generalised solve,
    U^H S(k) U = I to 1e-11, eigenvectors of well-separated bands S-parallel to the oracle's to
    1e-8; currents at points and on a
    warm-started mesh block against the FP64 generalised path to the mixed bound; a
    non-positive-definite S(k) is reported on this path too.  The FP64 CUDA-core Fourier sums
    (WNLQG_B200_DIRECT_FOURIER=1) isolate the eigensolver from the mixed path's 4-slice
    tensor-core Fourier."""
    from wanniernlqg_b200._lib import EngineError
    monkeypatch.setenv("WNLQG_B200_DIRECT_FOURIER", "1")
    model = _nonorth_full_position(nw, 11)
    task = _currents_task(_abi.PRECISION_MIXED)
    ref_task = _currents_task(_abi.PRECISION_FP64)
    k = np.random.default_rng(nw + 3).random((6, 3))
    with engine_cls(model, task) as eng:
        e, c = eng.spectrum(k)
        pts = eng.point_values(k[:3])
        mesh = eng.integrate_mesh((12, 10, 8), 100, 700)
    with engine_cls(model, ref_task) as eng:
        mesh_ref = eng.integrate_mesh((12, 10, 8), 100, 700)
    for i in range(k.shape[0]):
        eo, co, _ = oracle_mod.kpoint_spectrum(model, k[i])
        assert np.max(np.abs(e[i] - eo)) < 1e-11 * max(1.0, np.abs(eo).max())
        ph = np.exp(2j * np.pi * (model.r_vectors.T @ k[i])) / model.r_degeneracies
        sk = np.einsum("ijr,r->ij", model.overlap_r, ph)
        gram = c[i].conj().T @ sk @ c[i]
        assert np.max(np.abs(gram - np.eye(nw))) < 1e-11
        # Bands 0.05 eV from their neighbours: the one FP64 sweep leaves their vectors S-parallel
        # to the oracle's to second order.
        gaps = np.diff(eo)
        isolated = np.ones(nw, dtype=bool)
        isolated[:-1] &= gaps > 0.05
        isolated[1:] &= gaps > 0.05
        ov = np.abs(np.sum(c[i].conj() * (sk @ co), axis=0))
        if isolated.any():
            assert np.max(np.abs(ov - 1.0)[isolated]) < 1e-8
    ref = oracle_mod.point_values(model, ref_task, k[:3])
    for g, r in zip(task.split(pts), task.split(ref)):
        assert rel_err(g, r) < MIXED_RTOL
    for g, r in zip(task.split(mesh), task.split(mesh_ref)):
        assert rel_err(g, r) < MIXED_RTOL
    bad = _nonorth_full_position(nw, 11)
    home = int(np.where(np.all(bad.r_vectors == 0, axis=0))[0][0])
    bad.overlap_r[:, :, home] -= 2.0 * np.eye(nw)
    with engine_cls(bad, task) as eng:
        with pytest.raises(EngineError) as ei:
            eng.spectrum(np.array([[0.1, 0.2, 0.3]]))
        assert ei.value.status == 1
