"""CPU checks of the oracle's Fermi-sea Berry-curvature dipole on the finite-difference geometry.

The reference's default BCD geometry backend (derivative_backend = :finite_difference,
Runtime/Config.jl:113) takes, for the Fermi-sea moment D[mu,a,b,c] = sum_n f(E_n) d_c Omega_n^{ab}
(berry_dipole_moments!, Responses/QuantumGeometry/BerryMultipoleMoments.jl:7-47), the central
difference of the band curvature at k +- delta_c (berry_curvature_dipole_component!,
QuantumGeometryDerivatives.jl:193-228), delta_c the fractional image of the Cartesian step h e_c
(finite_difference_step_matrix, Core/Coordinates.jl:33-44), with every shifted spectrum checked for
isolation (BerryMultipoleGeometry.jl:38-39, 84-147).  The pins here share no code with that
restatement:

* two-band closed form: Omega_-^{ab} = (1/2) d^ . (d_a d^ x d_b d^) of H = e(k) + d(k) . sigma on a
  non-cubic lattice, differenced at the same shifted points, and against the analytic derivative;
* integration by parts: over the whole zone, sum_n f d_c Omega_n equals the Fermi-surface form
  sum_n (-f') Omega_n d_c E_n (BerryMultipoleMoments.jl:7-47, a different formula and code path),
  which converges exponentially on a mesh for a gapped model at finite temperature.
"""
import os
import re
import sys

import numpy as np
import pytest

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import TightBindingModel

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from test_parity_pins import d_vector, dhat_derivatives, two_band_model  # noqa: E402

LATTICE = np.diag([1.7, 0.8, 1.3])
PAULI = [np.eye(2, dtype=complex), np.array([[0, 1], [1, 0]], complex), np.array([[0, -1j], [1j, 0]]),
         np.diag([1.0, -1.0]).astype(complex)]
# H(k) = sum c {cos, sin}(k . R) sigma_p with k . R = 2 pi k_frac . R: a gapped two-band model
# (|d| >= 1.1 eV) without inversion, mirror or rotation symmetry, so that the dipole is nonzero.
ASYM_TERMS = [(1, "s", (1, 0, 0), 1.0), (1, "s", (0, 0, 1), 0.3), (1, "c", (0, 1, 0), 0.2),
              (2, "s", (0, 1, 0), 1.0), (2, "s", (1, 0, 1), 0.25),
              (3, "c", (0, 0, 0), 4.0), (3, "c", (1, 0, 0), 1.0), (3, "c", (0, 1, 0), 1.0), (3, "c", (0, 0, 1), 0.5),
              (3, "s", (1, 0, 0), 0.4),
              (0, "s", (1, 0, 0), 0.6), (0, "c", (0, 1, -1), 0.3), (0, "s", (0, 0, 1), 0.2)]


def asymmetric_two_band_model(lattice=LATTICE) -> TightBindingModel:
    terms = {}

    def add(R, mat):
        terms.setdefault(R, np.zeros((2, 2), complex))
        terms[R] += mat

    for p, kind, R, c in ASYM_TERMS:
        minus = tuple(-x for x in R)
        if kind == "c" and R == (0, 0, 0):
            add(R, c * PAULI[p])
        elif kind == "c":
            add(R, c / 2 * PAULI[p])
            add(minus, c / 2 * PAULI[p])
        else:
            add(R, c / 2j * PAULI[p])
            add(minus, -c / 2j * PAULI[p])
    keys = sorted(terms)
    ham = np.zeros((2, 2, len(keys)), complex, order="F")
    for i, R in enumerate(keys):
        ham[:, :, i] = terms[R]
    rv = np.asfortranarray(np.array(keys, dtype=np.int64).T)
    return TightBindingModel(np.asarray(lattice, float), rv, np.ones(len(keys), dtype=np.int64), ham, None)


def scaled_two_band_model(mass: float) -> TightBindingModel:
    """The d-vector model of the parity pins on the diagonal lattice LATTICE: with k . R = theta . r
    (theta = 2 pi k_frac) a Cartesian derivative along c is s_c d/d theta_c and the Cartesian
    curvature Omega^{ab} is s_a s_b times the theta-space one."""
    base = two_band_model(mass)
    return TightBindingModel(LATTICE.copy(), base.r_vectors, base.r_degeneracies, base.hamiltonian_r, None)


def lower_band_curvature(theta, mass, a, b):
    d, jac = d_vector(theta, mass)
    dh, ddh = dhat_derivatives(d, jac)
    return 0.5 * dh @ np.cross(ddh[a], ddh[b])


def sea_task(comps, mus, h=1e-4, **kw):
    kw.setdefault("degeneracy_threshold", 1e-3)
    kw.setdefault("denominator_regularization", 0.0)
    return _abi.TaskArrays([(_abi.BERRY_DIPOLE_SEA, comps)], fermi_energies=mus, finite_difference_step=h, **kw)


@pytest.mark.parametrize("kfrac", [(0.11, 0.23, 0.37), (0.41, 0.07, 0.83)])
def test_sea_dipole_two_band_closed_form(oracle_mod, kfrac):
    """mu between the bands: D = (Omega_-(k + h e_c) - Omega_-(k - h e_c)) / 2h with the closed-form
    curvature at the same Cartesian shifts; mu below or above both bands: 0 (the bands' curvatures
    cancel).  Bare denominators (the default 1e-3 eV regularization shifts Omega by ~eta^2/gap^2)."""
    mass, h = 1.3, 1e-4
    model = scaled_two_band_model(mass)
    s = np.diag(LATTICE)
    kf = np.array(kfrac)
    comps = ["xyz", "xzx", "yzy", "xyx", "zxy", "yxx"]
    got = oracle_mod.point_values(model, sea_task(comps, [-20.0, 0.0, 20.0], h), kf[None])[0].reshape(len(comps), 3)
    assert np.abs(got.imag).max() == 0.0
    for i, comp in enumerate(comps):
        a, b, c = ["xyz".index(x) for x in comp]
        theta = 2 * np.pi * kf
        tp, tm = theta.copy(), theta.copy()
        tp[c] += s[c] * h
        tm[c] -= s[c] * h
        ref = s[a] * s[b] * (lower_band_curvature(tp, mass, a, b) - lower_band_curvature(tm, mass, a, b)) / (2 * h)
        assert got[i, 1].real == pytest.approx(ref, rel=1e-9, abs=1e-12)
        # The central difference is second order: it agrees with the analytic derivative to O(h^2).
        fd8 = ((1, 4 / 5), (2, -1 / 5), (3, 4 / 105), (4, -1 / 280))
        step = 1e-3
        dtheta = 0.0
        for j, w in fd8:
            tpp, tmm = theta.copy(), theta.copy()
            tpp[c] += j * step
            tmm[c] -= j * step
            dtheta += w * (lower_band_curvature(tpp, mass, a, b) - lower_band_curvature(tmm, mass, a, b)) / step
        assert got[i, 1].real == pytest.approx(s[a] * s[b] * s[c] * dtheta, rel=1e-6, abs=1e-9)
        assert abs(got[i, 0].real) <= 1e-9 and abs(got[i, 2].real) <= 1e-9


def test_sea_dipole_equals_fermi_surface_form_over_the_zone(oracle_mod):
    """Integration by parts over the periodic zone: the Fermi-sea moment (finite-difference
    geometry) equals the Fermi-surface moment (curvature times band velocity times -f'), both at
    T = 3000 K on a 32^3 mesh of a gapped model without inversion (measured: 1e-7 relative;
    16^3 gives 3e-4, so the agreement is the mesh converging, not two copies of one formula)."""
    model = asymmetric_two_band_model()
    comps = ["xyz", "xzx", "yzy", "xyx", "zxx", "xyy"]
    mus = [-3.5, 3.0, 4.5]
    sea = sea_task(comps, mus, temperature=3000.0)
    fs = _abi.TaskArrays([(_abi.BERRY_DIPOLE, comps)], fermi_energies=mus, temperature=3000.0,
                         degeneracy_threshold=1e-3, denominator_regularization=0.0)
    a = oracle_mod.integrate_mesh(model, sea, (32, 32, 32)).real
    b = oracle_mod.integrate_mesh(model, fs, (32, 32, 32)).real
    scale = np.abs(b).max()
    assert scale > 1e-3
    assert np.abs(a - b).max() <= 1e-6 * scale


def test_sea_dipole_checks_isolation_at_shifted_points(oracle_mod):
    """A threshold between the centre's gap and the gap at k + delta_x: the centre passes, the
    shifted spectrum fails, and the error reports that spectrum's pair and gap on the centre's row."""
    model = asymmetric_two_band_model()
    h = 1e-2
    k = np.array([0.13, 0.31, 0.77])
    delta = LATTICE[:, 0] * h / (2 * np.pi)
    e0 = oracle_mod.kpoint_spectrum(model, k)[0]
    ep = oracle_mod.kpoint_spectrum(model, k + delta)[0]
    em = oracle_mod.kpoint_spectrum(model, k - delta)[0]
    g0, gp, gm = e0[1] - e0[0], ep[1] - ep[0], em[1] - em[0]
    assert gp != g0 and gm != g0
    # Fail exactly one shifted spectrum: the smaller of the two shifted gaps, if below the centre's.
    failing = min(gp, gm)
    assert failing < g0
    thr = 0.5 * (failing + min(g0, max(gp, gm)))
    with pytest.raises(RuntimeError) as exc:
        oracle_mod.point_values(model, sea_task(["yzx"], [0.0], h, degeneracy_threshold=thr), np.vstack([k, k]))
    m = re.search(r"GEOMETRY_SINGLE_BAND_SPECTRUM_NOT_ISOLATED: bands=\(1,2\), gap_ev=(\S+), threshold_ev=(\S+) "
                  r"\(k-point row 0\)", str(exc.value))
    assert m, str(exc.value)
    assert float(m.group(1)) == pytest.approx(failing, rel=1e-12)
    # The surface form checks only the centre and evaluates.
    fs = _abi.TaskArrays([(_abi.BERRY_DIPOLE, ["yzx"])], fermi_energies=[0.0], temperature=300.0,
                         degeneracy_threshold=thr)
    assert np.all(np.isfinite(oracle_mod.point_values(model, fs, k[None])))


def test_sea_dipole_argument_errors(oracle_mod):
    model = asymmetric_two_band_model()
    k = np.array([[0.1, 0.2, 0.3]])
    for h in (0.0, -1e-4, np.inf):
        with pytest.raises(RuntimeError, match="finite_difference_step must be finite and positive"):
            oracle_mod.point_values(model, sea_task(["xyz"], [0.0], h), k)
    with pytest.raises(RuntimeError, match="Fermi-energy axis"):
        oracle_mod.point_values(model, sea_task(["xyz"], []), k)
    task = sea_task(["xyz", "yzx"], [0.0, 1.0, 2.0])
    assert oracle_mod.point_values(model, task, k).shape == (1, 6)


# ---- the analytic geometry backend (derivative_backend = :analytic) ---------------------------

def test_analytic_sea_dipole_is_the_limit_of_the_finite_differences(oracle_mod):
    """The six-partition contraction of the band derivatives (OrthogonalGeometryDerivatives.jl:
    24-113) against the central differences of the band curvature: the gap closes as h^2 (a factor
    4 per halving of h), so both restatements compute d_c Omega_n (a model with a full position
    operator, Convention II)."""
    from wanniernlqg_b200.model import synthetic_orthogonal_model
    model = synthetic_orthogonal_model(6, 1, 3, full_position=True)
    k = np.random.default_rng(5).random((6, 3))
    e = oracle_mod.kpoint_spectrum(model, k[0])[0]
    comps = ["xyz", "xzx", "yzy", "xyx", "zxy", "yxx", "xxy", "zzx"]
    kw = dict(fermi_energies=[float(np.median(e)), 50.0], temperature=300.0, degeneracy_threshold=1e-6,
              denominator_regularization=0.0)
    an = oracle_mod.point_values(model, _abi.TaskArrays([(_abi.BERRY_DIPOLE_SEA, comps)], derivative_backend="analytic",
                                                        **kw), k)
    errs = []
    for h in (4e-4, 2e-4, 1e-4):
        fd = oracle_mod.point_values(model, _abi.TaskArrays([(_abi.BERRY_DIPOLE_SEA, comps)], finite_difference_step=h,
                                                            **kw), k)
        errs.append(np.abs(an - fd).max() / np.abs(an).max())
    assert errs[-1] < 5e-7
    for e0, e1 in zip(errs, errs[1:]):
        assert 3.5 < e0 / e1 < 4.5, errs
    # mu above every band: sum_n Omega_n^{ab} = Tr F^{ab} = d_a Tr A_b - d_b Tr A_a (the pair terms
    # cancel, the commutator is traceless), so the moment is d_c of that: a direct Fourier sum of the
    # traces of the position blocks.
    rc = model.lattice.T @ model.r_vectors            # Cartesian R, [3, NR]
    tr = np.einsum("iiar->ar", model.position_r)       # Tr A_R,a, [3, NR]
    for kk, vals in zip(k, an.reshape(len(k), len(comps), 2)[:, :, 1]):
        ph = np.exp(2j * np.pi * (model.r_vectors.T @ kk)) / model.r_degeneracies
        for comp, v in zip(comps, vals):
            a, b, c = ["xyz".index(x) for x in comp]
            ref = np.sum(ph * (-rc[a] * rc[c] * tr[b] + rc[b] * rc[c] * tr[a])).real
            assert v.real == pytest.approx(ref, rel=1e-9, abs=1e-11 * np.abs(an).max())


@pytest.mark.parametrize("kfrac", [(0.11, 0.23, 0.37), (0.41, 0.07, 0.83)])
def test_analytic_sea_dipole_two_band_closed_form(oracle_mod, kfrac):
    """mu between the bands: d_c Omega_- of the closed form, differentiated by an eighth-order
    stencil, on the non-cubic lattice."""
    mass = 1.3
    model = scaled_two_band_model(mass)
    s = np.diag(LATTICE)
    kf = np.array(kfrac)
    comps = ["xyz", "xzx", "yzy", "xyx", "zxy", "yxx"]
    task = _abi.TaskArrays([(_abi.BERRY_DIPOLE_SEA, comps)], fermi_energies=[0.0], degeneracy_threshold=1e-3,
                           denominator_regularization=0.0, derivative_backend="analytic")
    got = oracle_mod.point_values(model, task, kf[None])[0].real
    fd8 = ((1, 4 / 5), (2, -1 / 5), (3, 4 / 105), (4, -1 / 280))
    for i, comp in enumerate(comps):
        a, b, c = ["xyz".index(x) for x in comp]
        theta = 2 * np.pi * kf
        d = 0.0
        for j, w in fd8:
            tp, tm = theta.copy(), theta.copy()
            tp[c] += j * 1e-3
            tm[c] -= j * 1e-3
            d += w * (lower_band_curvature(tp, mass, a, b) - lower_band_curvature(tm, mass, a, b)) / 1e-3
        assert got[i] == pytest.approx(s[a] * s[b] * s[c] * d, rel=1e-9, abs=1e-12)


def test_derivative_backend_must_be_known(oracle_mod):
    model = asymmetric_two_band_model()
    task = _abi.TaskArrays([(_abi.BERRY_DIPOLE_SEA, ["xyz"])], fermi_energies=[0.0])
    task.desc.derivative_backend = 2
    with pytest.raises(RuntimeError, match="derivative_backend must be 0"):
        oracle_mod.point_values(model, task, np.array([[0.1, 0.2, 0.3]]))
    with pytest.raises(ValueError):
        _abi.TaskArrays([(_abi.BERRY_DIPOLE_SEA, ["xyz"])], fermi_energies=[0.0], derivative_backend="spectral")


def test_sea_dipole_is_the_same_in_both_wannier_center_conventions(oracle_mod):
    """Convention I changes the Bloch basis by a k-dependent diagonal phase and the home-cell
    connection by the centres (WannierCenterConventionTransforms.jl:55-113); the band curvature and
    its derivative are physical, so both backends give Convention II's moment (analytic to
    rounding, the finite differences to their rounding amplified by 1/2h)."""
    from wanniernlqg_b200.model import synthetic_orthogonal_model
    model = synthetic_orthogonal_model(6, 1, 3, full_position=True)
    k = np.random.default_rng(5).random((6, 3))
    comps = ["xyz", "xzx", "yzy", "xyx"]
    for backend, tol in (("analytic", 1e-13), ("finite_difference", 1e-10)):
        vals = []
        for conv in ("II", "I"):
            task = _abi.TaskArrays([(_abi.BERRY_DIPOLE_SEA, comps)], fermi_energies=[0.0, 50.0], temperature=300.0,
                                   degeneracy_threshold=1e-6, denominator_regularization=0.0,
                                   wannier_center_convention=conv, derivative_backend=backend)
            vals.append(oracle_mod.point_values(model, task, k))
        assert np.abs(vals[0] - vals[1]).max() <= tol * np.abs(vals[0]).max()
