"""CPU checks of the FP64 oracle against LAPACK (numpy), direct numpy sums and the reference's
golden vectors."""
import itertools
import os

import numpy as np
import pytest

from conftest import GOLDEN, read_complex_lines
from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import reference_workload_model, synthetic_orthogonal_model


@pytest.mark.parametrize("n", [1, 2, 4, 7, 16, 32])
def test_eigensolver_matches_lapack(oracle_mod, n):
    rng = np.random.default_rng(n)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    h = a + a.conj().T
    e, u = oracle_mod.hermitian_eigen(h)
    en = np.linalg.eigvalsh(h)
    assert np.max(np.abs(e - en)) <= 1e-13 * max(1.0, np.max(np.abs(en)))
    assert np.max(np.abs(h @ u - u * e)) <= 1e-12 * max(1.0, np.max(np.abs(en)))
    assert np.max(np.abs(u.conj().T @ u - np.eye(n))) < 1e-13
    # Canonical phase: largest-magnitude entry of each column is real and non-negative.
    for j in range(n):
        p = int(np.argmax(np.abs(u[:, j])))
        assert abs(u[p, j].imag) < 1e-15 and u[p, j].real > 0


def test_eigensolver_uses_upper_triangle(oracle_mod):
    rng = np.random.default_rng(3)
    a = rng.standard_normal((5, 5)) + 1j * rng.standard_normal((5, 5))
    h = np.triu(a) + np.triu(a, 1).conj().T
    h[np.diag_indices(5)] = h.diagonal().real
    junk = h.copy()
    junk[np.tril_indices(5, -1)] = 99.0   # lower triangle must be ignored (Hermitian(H, :U))
    e1, _ = oracle_mod.hermitian_eigen(h)
    e2, _ = oracle_mod.hermitian_eigen(junk)
    assert np.array_equal(e1, e2)


def _numpy_hk(model, k):
    ph = np.exp(2j * np.pi * (model.r_vectors.T @ np.asarray(k))) / model.r_degeneracies
    return np.einsum("ijr,r->ij", model.hamiltonian_r, ph)


@pytest.mark.parametrize("name", ["nw4", "nw32"])
def test_fourier_and_spectrum_match_numpy(oracle_mod, name):
    model = reference_workload_model(name)
    rng = np.random.default_rng(5)
    for k in rng.random((3, 3)):
        hk = _numpy_hk(model, k)
        e, u, dh = oracle_mod.kpoint_spectrum(model, k)
        en = np.linalg.eigvalsh(hk)
        assert np.max(np.abs(e - en)) < 1e-12 * max(1, np.abs(en).max())
        # dH_a in the Hamiltonian gauge = U^H (sum_R f_R i R_a H_R) U
        rc = model.lattice.T @ model.r_vectors
        ph = np.exp(2j * np.pi * (model.r_vectors.T @ k)) / model.r_degeneracies
        for a in range(3):
            dhw = np.einsum("ijr,r->ij", model.hamiltonian_r, ph * 1j * rc[a])
            ref = u.conj().T @ dhw @ u
            assert np.max(np.abs(dh[:, :, a] - ref)) < 1e-11 * max(1, np.abs(ref).max())


def test_jerk_golden_fixture(oracle_mod):
    """Frozen independent ordered jerk fixture (test/third_order_unit.jl:210-253)."""
    inp = read_complex_lines(os.path.join(GOLDEN, "jerk_input.dat"))
    B = inp[:48].reshape(4, 4, 3, order="F")
    A = inp[48:96].reshape(4, 4, 3, order="F")
    C = inp[96:240].reshape(4, 4, 3, 3, order="F")
    comps = list(itertools.product(range(3), repeat=4))
    out = oracle_mod.jerk_algebra([-1.5, -0.4, 0.7, 1.8], B, A, C, [1.1, 2.2, 3.3], comps,
                                  mu=0.0, T=0.0, width=0.04, gaussian=True, reg=0.001, window=5.0)
    ref = read_complex_lines(os.path.join(GOLDEN, "jerk_reference.dat")).reshape(3, 81, order="F")
    np.testing.assert_allclose(out, ref, atol=1e-12, rtol=4e-15)
    assert np.max(np.abs(out.imag)) > 0.01


SHG_COMPONENTS = [(a, b, c) for a in range(3) for (b, c) in ((0, 0), (1, 1), (2, 2), (1, 2), (0, 2), (0, 1))]
SHG_OPTIONS = dict(mu=0.0, T=0.0, broadening=0.025, low_frequency_broadening=0.025, gaussian=True, eta=0.04,
                   eta_correction=True, degeneracy=0.002)
SHG_OMEGAS = [0.0, 0.1, 0.73, 1.7]


def _shg_block(data, sel):
    e, dh, a, da, ddh = data
    ix = np.ix_(sel, sel)
    return (e[sel], dh[ix + (slice(None),)], a[ix + (slice(None),)], da[ix + (slice(None), slice(None))],
            ddh[ix + (slice(None), slice(None))])


@pytest.mark.parametrize("bands", [2, 3, 4])
@pytest.mark.parametrize("point", ["generic", "gamma"])
@pytest.mark.parametrize("gaussian", [True, False])
@pytest.mark.parametrize("correction", [True, False])
def test_shg_golden_fixtures(oracle_mod, bands, point, gaussian, correction):
    """The reference's 24 frozen SHG tables (test/second_harmonic_unit.jl:29-100): the 4-orbital
    synthetic_runtime model at one generic k and at Gamma, band subsets 2:3, 1:3 and 1:4, both
    delta kernels, with and without the finite-eta correction; the table is the sum of the seven
    terms, flattened (frequency, component, quantity)."""
    from wanniernlqg_b200.model import read_wannier_tb
    model = read_wannier_tb(os.path.join(GOLDEN, "synthetic_tb.dat"))
    k = [0.17, 0.23, 0.31] if point == "generic" else [0.0, 0.0, 0.0]
    sel = [1, 2] if bands == 2 else list(range(bands))
    e, V, A, dA, W = _shg_block(oracle_mod.kpoint_data(model, k), sel)
    opts = dict(SHG_OPTIONS, gaussian=gaussian, eta_correction=correction)
    out = oracle_mod.shg_algebra(e, V, A, dA, W, SHG_OMEGAS, SHG_COMPONENTS, **opts)
    name = ("" if bands == 4 else f"{bands}band_") + point + "_" + ("gaussian" if gaussian else "lorentzian") + \
        "_" + ("corrected" if correction else "uncorrected") + ".dat"
    ref = read_complex_lines(os.path.join(GOLDEN, "second_harmonic", name)).reshape(4, 18, 2, order="F")
    np.testing.assert_allclose(out.sum(axis=2), ref, atol=1e-10, rtol=1e-8)


def test_shg_contract_properties(oracle_mod):
    """Structural checks of second_harmonic_unit.jl:101-131: finite values, no one-band terms at
    T = 0, symmetric incident indices, the 1e-7 K temperature switch, and at 300 K with mu on a
    band both one-band terms present with a vanishing aaa Berry-curvature-dipole term."""
    from wanniernlqg_b200.model import read_wannier_tb
    model = read_wannier_tb(os.path.join(GOLDEN, "synthetic_tb.dat"))
    data = oracle_mod.kpoint_data(model, [0.17, 0.23, 0.31])
    out = oracle_mod.shg_algebra(*data, SHG_OMEGAS, SHG_COMPONENTS, **SHG_OPTIONS)
    assert np.all(np.isfinite(out))
    assert np.all(out[:, :, 5:7, :] == 0)
    swapped = oracle_mod.shg_algebra(*data, SHG_OMEGAS, [(a, c, b) for a, b, c in SHG_COMPONENTS], **SHG_OPTIONS)
    np.testing.assert_allclose(swapped, out, atol=1e-10, rtol=1e-8)
    tiny = oracle_mod.shg_algebra(*data, SHG_OMEGAS, SHG_COMPONENTS, **dict(SHG_OPTIONS, T=1e-7))
    assert np.array_equal(tiny, out)
    metal = oracle_mod.shg_algebra(*data, SHG_OMEGAS, SHG_COMPONENTS, **dict(SHG_OPTIONS, T=300.0, mu=data[0][1]))
    assert np.any(metal[:, :, 6, :] != 0) and np.any(metal[:, :, 5, :] != 0)
    for i, (a, b, c) in enumerate(SHG_COMPONENTS):
        if a == b == c:
            assert np.all(metal[:, i, 5, :] == 0)
    with pytest.raises(RuntimeError, match="finite and positive"):
        oracle_mod.shg_algebra(*data, SHG_OMEGAS, SHG_COMPONENTS, **dict(SHG_OPTIONS, eta=0.0))


def _sc_task(**kw):
    args = dict(broadening_type=_abi.LORENTZIAN, broadening=0.02, photon_energies=np.linspace(0, 3, 16))
    args.update(kw)
    return _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy", "zzz"]), (_abi.INJECTION_CURRENT, ["xyy"]),
                            (_abi.BERRY_CURVATURE, ["xy"]), (_abi.QUANTUM_METRIC, ["xx"])], **args)


def test_mesh_lanes_equal_pointwise_sum(oracle_mod):
    """Lane-ordered mesh integral equals (1/Nk) * sum of per-point values on the Gamma mesh."""
    model = reference_workload_model("nw4")
    task = _sc_task()
    mesh = (3, 4, 2)
    idx = np.arange(np.prod(mesh))
    k = np.stack([(idx % 3) / 3, ((idx // 3) % 4) / 4, (idx // 12) / 2], axis=1)
    pv = oracle_mod.point_values(model, task, k)
    tot = oracle_mod.integrate_mesh(model, task, mesh)
    np.testing.assert_allclose(tot, pv.sum(axis=0) / len(idx), rtol=1e-12, atol=1e-300)
    part = oracle_mod.integrate_mesh(model, task, mesh, 5, 17)
    np.testing.assert_allclose(part, pv[5:17].sum(axis=0) / len(idx), rtol=1e-12, atol=1e-300)


def test_thread_count_does_not_change_mesh_result(oracle_mod):
    model = reference_workload_model("nw4")
    task = _sc_task()
    a = oracle_mod.integrate_mesh(model, task, (4, 4, 4), threads=1)
    b = oracle_mod.integrate_mesh(model, task, (4, 4, 4), threads=4)
    assert np.array_equal(a, b)


def test_ahc_zero_temperature_matches_occupied_curvature(oracle_mod):
    """T=0 intrinsic AHC (bare occupied/empty links) equals the occupied-sum Berry curvature up to
    the eta^2/gap^2 difference between bare and regularised links."""
    model = synthetic_orthogonal_model(6, 1, 2, full_position=True)
    mus = [-0.3, 0.0, 0.4]
    k = np.random.default_rng(8).random((6, 3))
    ahc = _abi.TaskArrays([(_abi.INTRINSIC_AHC, ["xy", "yz"])], fermi_energies=mus)
    a = oracle_mod.point_values(model, ahc, k)
    for i, mu in enumerate(mus):
        bc = _abi.TaskArrays([(_abi.BERRY_CURVATURE, ["xy", "yz"])], fermi_energy=mu, denominator_regularization=1e-7)
        b = oracle_mod.point_values(model, bc, k)
        np.testing.assert_allclose(a[:, [i, 3 + i]].real, b.real, rtol=1e-6, atol=1e-9)


def test_berry_dipole_finite_temperature_weight_integrates_to_one():
    """-f'(E) of the dipole weight (ResponseOccupations.jl:24-36) integrates to one over E."""
    kb = 8.617333262145e-5
    T = 50.0
    e = np.linspace(-1, 1, 200001)
    z = np.exp(-np.abs(e / (kb * T)))
    w = z / (kb * T * (1 + z) ** 2)
    assert abs(np.trapezoid(w, e) - 1.0) < 1e-6


def test_mlp_oracle_gradient_matches_finite_differences():
    """Pins the oracle's backpropagation: with weights that are exact BF16 values, central
    differences of the float64 loss equal the analytic gradient."""
    from oracle import mlp_oracle as M
    rng = np.random.default_rng(4)
    p = M.bf16_round(rng.normal(0, 0.3, M.COUNT).astype(np.float32)).astype(np.float64)
    x = rng.normal(size=(40, M.F))
    t = rng.normal(size=40)

    def loss_at(q):
        y, _ = M.forward(q.astype(np.float32), x)   # q holds exact BF16 values for weights
        return np.mean((y - t) ** 2)

    _, g = M.loss_grad(p.astype(np.float32), x, t)
    # Probe biases (no BF16 rounding) with central differences.
    for name in ("b1", "b2", "b3", "b4"):
        o, size = M.OFF[name]
        for i in range(min(size, 5)):
            e = np.zeros(M.COUNT)
            e[o + i] = 1e-3
            fd = (loss_at(p + e) - loss_at(p - e)) / 2e-3
            assert abs(fd - g[o + i]) < 1e-4 * max(1.0, abs(fd))


@pytest.mark.parametrize("n", [2, 5, 16])
def test_generalized_eigen_matches_lapack(oracle_mod, n):
    import scipy.linalg
    rng = np.random.default_rng(30 + n)
    a = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    h = a + a.conj().T
    b = rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n))
    s = b @ b.conj().T + n * np.eye(n)
    e, c = oracle_mod.generalized_eigen(h, s)
    el = scipy.linalg.eigh(h, s, eigvals_only=True)
    assert np.max(np.abs(e - el)) < 1e-12 * max(1.0, np.abs(el).max())
    assert np.max(np.abs(c.conj().T @ s @ c - np.eye(n))) < 1e-12
    assert np.max(np.abs(h @ c - s @ c * e)) < 1e-11 * max(1.0, np.abs(el).max())


def _overlap_copy(model, M=None):
    """The same model in a nonorthogonal basis: S = M^H M at R = 0, H' = M^H H M, A' = M^H A M
    (M = I: the orthogonal model with an identity overlap)."""
    import copy
    nw, nr = model.num_orbitals, model.num_r_vectors
    M = np.eye(nw) if M is None else M
    out = copy.deepcopy(model)
    home = int(np.where(np.all(model.r_vectors == 0, axis=0))[0][0])
    S = np.zeros((nw, nw, nr), dtype=np.complex128, order="F")
    S[:, :, home] = M.conj().T @ M
    out.overlap_r = S
    out.hamiltonian_r = np.asfortranarray(np.einsum("ji,jkr,kl->ilr", M.conj(), model.hamiltonian_r, M))
    out.position_r = np.asfortranarray(np.einsum("ji,jkar,kl->ilar", M.conj(), model.position_r, M))
    return out


@pytest.mark.parametrize("eta", [0.001, 0.0])
@pytest.mark.parametrize("transform", ["identity", "constant"])
def test_nonorthogonal_currents_equal_orthogonal(oracle_mod, eta, transform):
    """The metric (nonorthogonal) geometry of NonorthogonalMatrixElements.jl:560-817 must give the
    orthogonal shift and injection currents when the overlap is the identity, and must be invariant
    under a constant non-unitary change of the orbital basis (the reference has no numeric fixtures
    for this path; these identities pin it)."""
    model = synthetic_orthogonal_model(6, 1, seed=3, full_position=True)
    rng = np.random.default_rng(4)
    M = None if transform == "identity" else np.eye(6) + 0.2 * (rng.standard_normal((6, 6)) + 1j * rng.standard_normal((6, 6)))
    other = _overlap_copy(model, M)
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyy", "zxy", "yyy"]), (_abi.INJECTION_CURRENT, ["xyy", "zzx"])],
                           broadening_type=_abi.LORENTZIAN, broadening=0.05, photon_energies=np.linspace(0, 3, 16),
                           denominator_regularization=eta)
    k = np.random.default_rng(1).random((5, 3))
    a = oracle_mod.point_values(model, task, k)
    b = oracle_mod.point_values(other, task, k)
    assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(a))


@pytest.mark.parametrize("transform", ["identity", "constant"])
@pytest.mark.parametrize("temperature", [0.0, 300.0])
def test_metric_second_harmonic_equals_orthogonal(oracle_mod, transform, temperature):
    """Metric SHG (normalized source jets of NonorthogonalOpticalCutoffVertices.jl:67-186, metric
    Berry connection as r_eta, metric energy Hessians and isolated-band curvature,
    SecondHarmonicKernels.jl:47-68) gives the orthogonal SHG tables when the overlap is the
    identity and is invariant under a constant non-unitary basis change, all seven terms
    (one-band terms at T > 0) and both quantities.  The geometry width is the SHG width here
    (intermediate regularization 0 selects the denominator regularization)."""
    model = synthetic_orthogonal_model(6, 1, seed=4, full_position=True)
    rng = np.random.default_rng(9)
    M = None if transform == "identity" else np.eye(6) + 0.2 * (rng.standard_normal((6, 6)) + 1j * rng.standard_normal((6, 6)))
    other = _overlap_copy(model, M)
    task = _abi.TaskArrays([(_abi.SECOND_HARMONIC, ["xxx", "xyy", "yzx", "zxz"])], broadening_type=_abi.LORENTZIAN,
                           broadening=0.03, photon_energies=np.linspace(0.1, 2.0, 7), denominator_regularization=0.01,
                           shg_intermediate_regularization=0.0, shg_eta_correction=False, temperature=temperature,
                           fermi_energy=0.1)
    k = np.random.default_rng(3).random((5, 3))
    a = oracle_mod.point_values(model, task, k)
    b = oracle_mod.point_values(other, task, k)
    assert np.max(np.abs(a)) > 0
    assert np.max(np.abs(a - b)) <= 1e-10 * np.max(np.abs(a))


def test_metric_second_harmonic_preconditions(oracle_mod):
    """Metric SHG needs a positive geometry width and no eta correction
    (NonorthogonalMatrixElements.jl:1088-1110)."""
    other = _overlap_copy(synthetic_orthogonal_model(4, 1, seed=1, full_position=True))
    k = np.zeros((1, 3))
    kw = dict(broadening=0.03, photon_energies=[0.5], shg_intermediate_regularization=0.01)
    with pytest.raises(RuntimeError, match="ETA_CORRECTION_UNSUPPORTED"):
        oracle_mod.point_values(other, _abi.TaskArrays([(_abi.SECOND_HARMONIC, ["xxx"])], denominator_regularization=0.01,
                                                       shg_eta_correction=True, **kw), k)
    with pytest.raises(RuntimeError, match="POSITIVE_GEOMETRY_REQUIRED"):
        oracle_mod.point_values(other, _abi.TaskArrays([(_abi.SECOND_HARMONIC, ["xxx"])], denominator_regularization=0.0,
                                                       shg_eta_correction=False, **kw), k)


def test_band_selection_partitions_add_up(oracle_mod):
    """Explicit interband selection (valence n, conduction m): the shift and injection currents of
    all valence x conduction group combinations of a band partition add up to the unselected
    result.  The transition threshold is off (transition_window_factor = 0): with it, a point
    counts only when a selected pair lies near a photon energy, which the reference applies per
    selection, so blocks of a partition may drop Lorentzian tails that the full run keeps."""
    model = synthetic_orthogonal_model(6, 1, seed=8, full_position=True)
    kw = dict(broadening_type=_abi.LORENTZIAN, broadening=0.05, photon_energies=np.linspace(0, 3, 10),
              transition_window_factor=0.0)
    resp = [(_abi.SHIFT_CURRENT, ["xyy", "zxz"]), (_abi.INJECTION_CURRENT, ["xyy"])]
    k = np.random.default_rng(2).random((4, 3))
    full = oracle_mod.point_values(model, _abi.TaskArrays(resp, **kw), k)
    groups = [[1, 2], [3, 4], [5, 6]]
    total = np.zeros_like(full)
    for v in groups:
        for c in groups:
            if v == c:
                continue
            total += oracle_mod.point_values(model, _abi.TaskArrays(resp, band_selection=(c, v), **kw), k)
    # pairs inside one group: each group once as its own halves
    for g in groups:
        total += oracle_mod.point_values(model, _abi.TaskArrays(resp, band_selection=([g[1]], [g[0]]), **kw), k)
        total += oracle_mod.point_values(model, _abi.TaskArrays(resp, band_selection=([g[0]], [g[1]]), **kw), k)
    assert np.max(np.abs(total - full)) <= 1e-12 * np.max(np.abs(full))
    with pytest.raises(RuntimeError, match="overlap"):
        oracle_mod.point_values(model, _abi.TaskArrays(resp, band_selection=([1, 2], [2, 3]), **kw), k)
    with pytest.raises(RuntimeError, match="band window"):
        oracle_mod.point_values(model, _abi.TaskArrays(resp, band_selection=([1], [2]), band_window_size=2, **kw), k)


def _lattice_model(full_position, seed=12, nw=5):
    """A synthetic model on a non-cubic lattice (so that fractional and Cartesian centres differ)."""
    import copy
    model = copy.deepcopy(synthetic_orthogonal_model(nw, 1, seed=seed, full_position=full_position))
    model.lattice = np.asfortranarray(np.array([[3.1, 0.0, 0.0], [0.9, 2.7, 0.0], [0.4, 0.6, 3.5]]))
    return model


def test_convention_one_is_a_gauge_transform_of_convention_two(oracle_mod):
    """Convention I (centred connection, R + tau_j - tau_i displacements, D(k) similarity,
    WannierCenterConventionTransforms.jl) is a k-dependent diagonal gauge transform of Convention
    II: with the complete position operator and bare inverses (eta = 0) the shift and injection
    currents, Berry curvature and quantum metric agree; the eigenvalues agree and each Convention I
    eigenvector is D(k)^H times the Convention II one up to its canonical phase."""
    model = _lattice_model(True)
    resp = [(_abi.SHIFT_CURRENT, ["xyy", "zxz"]), (_abi.INJECTION_CURRENT, ["xyy"]),
            (_abi.BERRY_CURVATURE, ["xy", "yz"]), (_abi.QUANTUM_METRIC, ["xx", "xz"])]
    kw = dict(broadening_type=_abi.LORENTZIAN, broadening=0.05, photon_energies=np.linspace(0, 3, 10),
              denominator_regularization=0.0)
    k = np.random.default_rng(3).random((4, 3))
    two = oracle_mod.point_values(model, _abi.TaskArrays(resp, **kw), k)
    one = oracle_mod.point_values(model, _abi.TaskArrays(resp, wannier_center_convention="I", **kw), k)
    for a, b in zip(_abi.TaskArrays(resp, **kw).split(two), _abi.TaskArrays(resp, **kw).split(one)):
        assert np.max(np.abs(a - b)) <= 1e-9 * np.max(np.abs(a))
    tau = np.real(np.array([np.diag(model.position_r[:, :, x, 13]) for x in range(3)]))   # R = 0 is index 13 of the cube
    assert np.all(model.r_vectors[:, 13] == 0)
    frac = np.linalg.solve(model.lattice.T, tau)          # tau_cart[j] = sum_r frac_r lattice[r, j]
    for kp in k:
        e2, u2, _ = oracle_mod.kpoint_spectrum(model, kp, "II")
        e1, u1, _ = oracle_mod.kpoint_spectrum(model, kp, "I")
        assert np.max(np.abs(e1 - e2)) < 1e-12
        d = np.exp(2j * np.pi * (kp @ frac))
        ov = np.abs(np.sum(u1.conj() * (d.conj()[:, None] * u2), axis=0))
        assert np.max(np.abs(ov - 1.0)) < 1e-10
        piv = np.argmax(np.abs(u1), axis=0)
        assert np.all(np.abs(u1[piv, np.arange(u1.shape[1])].imag) < 1e-12)


def test_convention_one_with_diagonal_positions_and_home_cell_check(oracle_mod):
    """With only the centres on the home-cell diagonal (tight-binding positions) Convention I is
    still a gauge transform of Convention II: the centre terms of r = A + i D cancel exactly with
    bare inverses (eta = 0) and up to the regularization with eta > 0.  A model without an R = 0
    block is rejected under Convention I."""
    import copy
    model = _lattice_model(False)
    resp = [(_abi.SHIFT_CURRENT, ["xyy"]), (_abi.INJECTION_CURRENT, ["zxz"])]
    kw = dict(broadening_type=_abi.LORENTZIAN, broadening=0.05, photon_energies=np.linspace(0.5, 2.5, 6))
    k = np.random.default_rng(4).random((3, 3))
    for eta, tol in ((0.0, 1e-9), (0.001, 1e-5)):
        two = oracle_mod.point_values(model, _abi.TaskArrays(resp, denominator_regularization=eta, **kw), k)
        one = oracle_mod.point_values(model, _abi.TaskArrays(resp, denominator_regularization=eta,
                                                             wannier_center_convention="I", **kw), k)
        assert np.max(np.abs(one - two)) <= tol * np.max(np.abs(two))
    shifted = copy.deepcopy(model)
    shifted.r_vectors = np.asfortranarray(shifted.r_vectors + np.array([[5], [0], [0]]))
    with pytest.raises(RuntimeError, match="R=\\(0,0,0\\)"):
        oracle_mod.point_values(shifted, _abi.TaskArrays(resp, wannier_center_convention="I", **kw), k)
