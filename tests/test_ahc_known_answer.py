"""The reference's intrinsic-AHC known answers (test/intrinsic_hall_real_occupation_unit.jl):
prepared geometry with energies E, velocities v and ambient curvature F, and the independent
velocity-product sum

    sigma^{ab}(mu) = sum_{E_l <= mu} [ Re F_ll^{ab} - sum_{E_m > mu} Im((v^a_lm v^b_ml - v^b_lm v^a_ml) / (E_l - E_m)^2) ]

at several Fermi energies, including one equal to a level (that level is occupied) and gaps of one
and eight ulp.  The reference feeds the geometry to intrinsic_hall_fermi_sea directly; here it
comes out of a tight-binding model built to have exactly that geometry at k = 0:
H(k) = diag(E) + sum_a (e^{i k_a} X_a + h.c.) with X_a = -i v_a / 2 (so H(0) = diag(E) and
dH/dk_a(0) = v_a), and position blocks A_y(R = +-x) = -+ i diag(F_xy) / 2 (so A(0) = 0 and
F_xy = d_x A_y = diag(F_xy)).  The single point k = 0 is the 1 x 1 x 1 mesh; on the device its
Fourier sums are exact on the FP64 CUDA-core path (WNLQG_B200_DIRECT_FOURIER=1), which the test
selects: the tensor-core path keeps 49 bits of each column, which can move the level at 0.04 eV by
more than the ulp that decides whether mu = 0.04 occupies it.
"""
import numpy as np
import pytest

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import TightBindingModel


def fixture(energy):
    """Velocities and curvature of the reference fixture (1-based l < m in its loops)."""
    n = len(energy)
    v = np.zeros((n, n, 3), complex)
    f = np.zeros((n, n, 3, 3), complex)
    for l in range(1, n + 1):
        for m in range(l + 1, n + 1):
            v[l - 1, m - 1, 0] = v[m - 1, l - 1, 0] = 0.3 + 0.1 * l
            v[l - 1, m - 1, 1] = 1j * (0.2 + 0.05 * m)
            v[m - 1, l - 1, 1] = np.conj(v[l - 1, m - 1, 1])
    for l in range(1, n + 1):
        f[l - 1, l - 1, 0, 1] = 0.07 * l
        f[l - 1, l - 1, 1, 0] = -0.07 * l
    return np.asarray(energy, float), v, f


def velocity_sum(energy, v, f, mu):
    n = len(energy)
    out = np.zeros((3, 3))
    for a in range(3):
        for b in range(3):
            for l in range(n):
                if not energy[l] <= mu:
                    continue
                out[a, b] += f[l, l, a, b].real
                for m in range(n):
                    if not energy[m] > mu:
                        continue
                    d = energy[l] - energy[m]
                    out[a, b] -= ((v[l, m, a] * v[m, l, b] - v[l, m, b] * v[m, l, a]) / (d * d)).imag
    return out


def geometry_model(energy, v, f) -> TightBindingModel:
    n = len(energy)
    keys = [(0, 0, 0), (1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1)]
    ham = np.zeros((n, n, len(keys)), complex, order="F")
    pos = np.zeros((n, n, 3, len(keys)), complex, order="F")
    ham[:, :, 0] = np.diag(energy)
    for a in range(3):
        x = -0.5j * v[:, :, a]
        ham[:, :, 1 + 2 * a] = x
        ham[:, :, 2 + 2 * a] = x.conj().T
    c = -0.5j * np.diag(np.diag(f[:, :, 0, 1]))
    pos[:, :, 1, 1] = c
    pos[:, :, 1, 2] = c.conj().T
    rv = np.asfortranarray(np.array(keys, dtype=np.int64).T)
    return TightBindingModel(np.eye(3), rv, np.ones(len(keys), dtype=np.int64), ham, pos)


COMPONENTS = ["xy", "yx", "xz", "zy", "xx"]
MUS = [0.03, 0.04, -1.0, 0.08, 0.03]


def ahc_task(mus, **kw):
    return _abi.TaskArrays([(_abi.INTRINSIC_AHC, COMPONENTS)], fermi_energies=mus, **kw)


def expected(energy, v, f, mus):
    ref = np.array([[velocity_sum(energy, v, f, mu)[("xyz".index(c[0]), "xyz".index(c[1]))] for mu in mus]
                    for c in COMPONENTS])
    return ref.ravel()


def check(values, energy, v, f, mus):
    ref = expected(energy, v, f, mus)
    np.testing.assert_allclose(values.real, ref, rtol=2e-12, atol=2e-12)
    assert np.abs(values.imag).max() == 0.0
    got = values.real.reshape(len(COMPONENTS), len(mus))
    assert np.all(got[:, 2] == 0.0)                    # mu below every level
    assert np.all(got[:, 0] == got[:, 4])              # the same mu twice
    assert got[0, 3] == pytest.approx(sum(0.07 * l for l in (1, 2, 3)), rel=1e-14)   # all occupied: sum Re F
    assert not np.array_equal(got[:, 0], got[:, 1])    # the level at mu = 0.04 is occupied


def test_oracle_reproduces_the_reference_ahc_fixture(oracle_mod):
    energy, v, f = fixture([0.0, 0.04, 0.08])
    model = geometry_model(energy, v, f)
    check(oracle_mod.integrate_mesh(model, ahc_task(MUS), (1, 1, 1)), energy, v, f, MUS)


@pytest.mark.parametrize("delta", [np.finfo(float).eps, 8 * np.finfo(float).eps])
def test_oracle_ahc_at_ulp_gaps(oracle_mod, delta):
    energy, v, f = fixture([1.0, 1.0 + delta, 2.0])
    v[0, 1, 0] = v[1, 0, 0] = delta
    v[0, 1, 1], v[1, 0, 1] = 1j * delta, -1j * delta
    model = geometry_model(energy, v, f)
    got = oracle_mod.integrate_mesh(model, ahc_task([1.0]), (1, 1, 1))
    np.testing.assert_allclose(got.real, expected(energy, v, f, [1.0]), rtol=2e-12, atol=2e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [_abi.PRECISION_FP64, _abi.PRECISION_MIXED])
def test_engine_reproduces_the_reference_ahc_fixture(precision, monkeypatch):
    monkeypatch.setenv("WNLQG_B200_DIRECT_FOURIER", "1")
    from wanniernlqg_b200 import build
    build.build()
    from wanniernlqg_b200.engine import ResponseEngine
    energy, v, f = fixture([0.0, 0.04, 0.08])
    with ResponseEngine(geometry_model(energy, v, f), ahc_task(MUS, precision=precision)) as eng:
        got = eng.integrate_mesh((1, 1, 1))
    if precision == _abi.PRECISION_FP64:
        check(got, energy, v, f, MUS)
    else:
        np.testing.assert_allclose(got.real, expected(energy, v, f, MUS), rtol=1e-6, atol=1e-6)
    for delta in (np.finfo(float).eps, 8 * np.finfo(float).eps):
        energy, v, f = fixture([1.0, 1.0 + delta, 2.0])
        v[0, 1, 0] = v[1, 0, 0] = delta
        v[0, 1, 1], v[1, 0, 1] = 1j * delta, -1j * delta
        with ResponseEngine(geometry_model(energy, v, f), ahc_task([1.0])) as eng:
            got = eng.integrate_mesh((1, 1, 1))
        np.testing.assert_allclose(got.real, expected(energy, v, f, [1.0]), rtol=2e-12, atol=2e-12)
