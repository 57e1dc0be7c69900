"""CPU checks of the oracle's spectral isolation contract, the zero-temperature rule of the
intrinsic AHC and the linear transport Berry channel.

References: geometry_isolated_spectrum_minimum_gap (MatrixElements/Interpolated/
OrthogonalBandDerivatives.jl:66-82) at its Berry-dipole call (BerryMultipoleGeometry.jl:81,
threshold degeneracy_threshold) and its eta = 0 call (PositionMatrixElements.jl:447-452, threshold
spectral_gap_tolerance); intrinsic_hall_fermi_sea (IntrinsicHallOccupations.jl:15-16);
_linear_transport_response (LinearTransport/LinearTransportKernels.jl:100-163).
"""
import re

import numpy as np
import pytest

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import TightBindingModel, kramers_doubled_model, synthetic_orthogonal_model

E_CHARGE = 1.602176634e-19
HBAR_JS = 1.054571817e-34
LT_FACTOR = E_CHARGE ** 2 / HBAR_JS * 1e-20


def _doubled(model: TightBindingModel) -> TightBindingModel:
    """H (x) I_2: every band exactly twofold degenerate."""
    nw, nr = model.num_orbitals, model.num_r_vectors
    ham = np.zeros((2 * nw, 2 * nw, nr), dtype=np.complex128, order="F")
    for r in range(nr):
        ham[:, :, r] = np.kron(model.hamiltonian_r[:, :, r], np.eye(2))
    return TightBindingModel(model.lattice.copy(), model.r_vectors.copy(), model.r_degeneracies.copy(), ham, None)


def _error(oracle_mod, fn):
    with pytest.raises(RuntimeError) as exc:
        fn()
    return str(exc.value)


def test_berry_dipole_requires_isolated_spectrum(oracle_mod):
    """A threshold above some gap of the spectrum makes the point fail with the reference's text;
    the first failing pair in the reference's loop order (m, then l) is reported, 1-based."""
    model = synthetic_orthogonal_model(6, 1, 3, full_position=True)
    k = np.array([[0.11, 0.27, 0.35]])
    e, _, _ = oracle_mod.kpoint_spectrum(model, k[0])
    gaps = np.diff(e)
    thr = float(np.sort(gaps)[1])   # above the smallest adjacent gap, below the others
    task = _abi.TaskArrays([(_abi.BERRY_DIPOLE, ["xyz"])], fermi_energies=[0.0], fermi_surface_broadening=0.05,
                           degeneracy_threshold=thr)
    msg = _error(oracle_mod, lambda: oracle_mod.point_values(model, task, k))
    m = re.search(r"GEOMETRY_SINGLE_BAND_SPECTRUM_NOT_ISOLATED: bands=\((\d+),(\d+)\), gap_ev=(\S+), "
                  r"threshold_ev=(\S+) \(k-point row 0\)", msg)
    assert m, msg
    l, mm = int(m.group(1)), int(m.group(2))
    # Reference loop: for m in 1:n, l in 1:m-1, first pair with gap <= threshold.
    first = next((ll, m2) for m2 in range(1, 7) for ll in range(1, m2) if abs(e[m2 - 1] - e[ll - 1]) <= thr)
    assert (l, mm) == first
    assert float(m.group(3)) == pytest.approx(abs(e[mm - 1] - e[l - 1]), rel=1e-12)
    assert float(m.group(4)) == thr
    # Below every gap the same point evaluates.
    ok = _abi.TaskArrays([(_abi.BERRY_DIPOLE, ["xyz"])], fermi_energies=[0.0], fermi_surface_broadening=0.05,
                         degeneracy_threshold=0.5 * float(gaps.min()))
    assert np.all(np.isfinite(oracle_mod.point_values(model, ok, k)))


def test_exact_geometry_rejects_degenerate_spectrum(oracle_mod):
    """eta = 0 (bare inverses) needs every pair split by more than spectral_gap_tolerance: an exactly
    doubled model fails at its first degenerate pair; eta > 0 evaluates it."""
    model = _doubled(synthetic_orthogonal_model(3, 1, 4))
    k = np.array([[0.2, 0.1, 0.3], [0.4, 0.3, 0.1]])
    exact = _abi.TaskArrays([(_abi.BERRY_CURVATURE, ["xy"])], denominator_regularization=0.0)
    msg = _error(oracle_mod, lambda: oracle_mod.point_values(model, exact, k))
    assert "GEOMETRY_SINGLE_BAND_SPECTRUM_NOT_ISOLATED: bands=(1,2), " in msg
    assert "threshold_ev=1e-10 (k-point row 0)" in msg
    mesh_msg = _error(oracle_mod, lambda: oracle_mod.integrate_mesh(model, exact, (2, 2, 2)))
    assert "GEOMETRY_SINGLE_BAND_SPECTRUM_NOT_ISOLATED" in mesh_msg
    assert "(k-point row 0)" in mesh_msg
    reg = _abi.TaskArrays([(_abi.BERRY_CURVATURE, ["xy"])], denominator_regularization=1e-3)
    assert np.all(np.isfinite(oracle_mod.point_values(model, reg, k)))


def test_kramers_pairs_isolated_at_small_threshold(oracle_mod):
    """Kramers-doubled bands split by O(1e-3 eV) fail the reference's default 2e-3 eV dipole
    threshold at some points and pass a 1e-9 eV threshold."""
    model = kramers_doubled_model(synthetic_orthogonal_model(4, 1, 5, full_position=True), 1e-3, seed=1)
    k = np.random.default_rng(3).random((16, 3))
    default = _abi.TaskArrays([(_abi.BERRY_DIPOLE, ["xzz"])], fermi_energies=[0.0], temperature=50.0)
    assert "NOT_ISOLATED" in _error(oracle_mod, lambda: oracle_mod.point_values(model, default, k))
    small = _abi.TaskArrays([(_abi.BERRY_DIPOLE, ["xzz"])], fermi_energies=[0.0], temperature=50.0,
                            degeneracy_threshold=1e-9)
    assert np.all(np.isfinite(oracle_mod.point_values(model, small, k)))


def test_intrinsic_ahc_requires_zero_temperature(oracle_mod):
    model = synthetic_orthogonal_model(4, 1, 2)
    task = _abi.TaskArrays([(_abi.INTRINSIC_AHC, ["xy"])], fermi_energies=[0.0], temperature=50.0)
    msg = _error(oracle_mod, lambda: oracle_mod.point_values(model, task, np.zeros((1, 3))))
    assert "INTRINSIC_HALL_REQUIRES_ZERO_TEMPERATURE" in msg


def test_linear_transport_berry_clean_limit_is_scaled_berry_curvature(oracle_mod):
    """At gamma_inter = 0 and T = 0 the Berry channel is -e^2/hbar 1e-20 times the occupied-sum
    Berry curvature (contact + 2 Im q over unordered pairs == the Kubo sum over ordered pairs)."""
    model = synthetic_orthogonal_model(6, 1, 7, full_position=True)
    mus = [-0.4, 0.1, 0.6]
    k = np.random.default_rng(9).random((8, 3))
    lt = _abi.TaskArrays([(_abi.LINEAR_TRANSPORT_BERRY, ["xy", "yz", "zx"])], fermi_energies=mus)
    got = oracle_mod.point_values(model, lt, k)
    for i, mu in enumerate(mus):
        bc = _abi.TaskArrays([(_abi.BERRY_CURVATURE, ["xy", "yz", "zx"])], fermi_energy=mu)
        ref = oracle_mod.point_values(model, bc, k)
        np.testing.assert_allclose(got[:, [i, 3 + i, 6 + i]].real, -LT_FACTOR * ref.real, rtol=1e-11,
                                   atol=1e-11 * LT_FACTOR * np.abs(ref).max())


def test_linear_transport_berry_rate_and_temperature(oracle_mod):
    """A finite interband rate multiplies each pair term by gap^2/(gap^2 + gamma^2); at T > 0 the
    occupations are the logistic response_occupation.  Checked against a numpy restatement of the
    Berry channel built from the oracle's Hamiltonian-gauge band data: F^H_ab = dA_b/dk_a -
    dA_a/dk_b - i[A_a, A_b] (rotation commutes with the commutator), r = A + i D with the
    regularized inverse."""
    model = synthetic_orthogonal_model(5, 1, 11, full_position=True)
    k = np.array([0.31, 0.17, 0.44])
    eta, kb = 1e-3, 8.617333262145e-5
    e, dh, a, da, ddh = oracle_mod.kpoint_data(model, k)
    n = e.size
    d = e[:, None] - e[None, :]
    inv = d / (d * d + eta * eta)
    r = [a[:, :, x] + 1j * (-dh[:, :, x] * inv) for x in range(3)]
    f_xy = da[:, :, 1, 0] - da[:, :, 0, 1] - 1j * (a[:, :, 0] @ a[:, :, 1] - a[:, :, 1] @ a[:, :, 0])
    for gamma, T, mu in ((0.07, 300.0, 0.05), (0.0, 50.0, -0.2), (0.02, 0.0, 0.3)):
        def occ(x):
            if T == 0:
                return 1.0 if x < mu else (0.0 if x > mu else 0.5)
            z = (x - mu) / (kb * T)
            return np.exp(-z) / (1 + np.exp(-z)) if z >= 0 else 1 / (1 + np.exp(z))
        contact = -LT_FACTOR * sum(occ(e[i]) * f_xy[i, i].real for i in range(n))
        pair = sum(2 * LT_FACTOR * (occ(e[i]) - occ(e[j])) * (e[j] - e[i]) ** 2 / ((e[j] - e[i]) ** 2 + gamma ** 2)
                   * (r[0][i, j] * r[1][j, i]).imag for i in range(n) for j in range(i + 1, n))
        task = _abi.TaskArrays([(_abi.LINEAR_TRANSPORT_BERRY, ["xy"])], fermi_energies=[mu], temperature=T,
                               linear_transport_gamma_inter=gamma)
        got = oracle_mod.point_values(model, task, k[None])[0, 0]
        assert got.imag == 0.0
        assert got.real == pytest.approx(contact + pair, rel=1e-11, abs=1e-13 * LT_FACTOR)


def test_linear_transport_requires_positive_regularization(oracle_mod):
    model = synthetic_orthogonal_model(4, 1, 2)
    task = _abi.TaskArrays([(_abi.LINEAR_TRANSPORT_BERRY, ["xy"])], fermi_energies=[0.0],
                           denominator_regularization=0.0)
    msg = _error(oracle_mod, lambda: oracle_mod.point_values(model, task, np.zeros((1, 3))))
    assert "spectral position regularization must be finite and positive" in msg


def test_linear_transport_joins_exactly_degenerate_levels(oracle_mod):
    """Exactly doubled levels form one spectral block: no pair term inside a block, and no
    SPECTRAL_CROSS_BLOCK_GAP_UNRESOLVED error; the result is finite."""
    base = synthetic_orthogonal_model(3, 1, 4, full_position=True)
    nw, nr = 3, base.num_r_vectors
    ham = np.zeros((6, 6, nr), dtype=np.complex128, order="F")
    pos = np.zeros((6, 6, 3, nr), dtype=np.complex128, order="F")
    for r in range(nr):
        ham[:, :, r] = np.kron(base.hamiltonian_r[:, :, r], np.eye(2))
        for a in range(3):
            pos[:, :, a, r] = np.kron(base.position_r[:, :, a, r], np.eye(2))
    model = TightBindingModel(base.lattice.copy(), base.r_vectors.copy(), base.r_degeneracies.copy(), ham, pos)
    task = _abi.TaskArrays([(_abi.LINEAR_TRANSPORT_BERRY, ["xy"])], fermi_energies=[0.0])
    vals = oracle_mod.point_values(model, task, np.array([[0.13, 0.29, 0.41]]))
    assert np.all(np.isfinite(vals))
