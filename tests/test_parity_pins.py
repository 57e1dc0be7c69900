"""Parity pins of the headline responses that do not rest on the oracle's own formulas.

The reference's tests hold no numeric values for shift / injection current, Berry curvature or
the quantum metric, so these checks pin the oracle (and through the GPU parity tests, the engine)
to definitions that share no code or algebra with the sum-over-states formulas it restates:

* the generalized derivative r^b_{nm;a} (ConventionalShiftCurrent.jl:191-229, a long sum over
  intermediate states) against its definition, the covariant derivative
  d_a r^b_nm - i (A^a_nn - A^a_mm) r^b_nm, with d_a an eighth-order central difference of r(k)
  in a parallel-transport gauge (theory/ShiftCurrent.md section 3);
* the shift-vector form of the b = c bracket, 2 |r^b_nm|^2 (d_a phi^b_nm - A^a_nn + A^a_mm);
* the interband connection against i <u_n|d u_m> from differenced eigenvectors;
* per-k shift and injection current values assembled in numpy from those differences
  (prefactors of ConventionalCurrentIntegralExecution.jl:241-245, 294-298);
* band Berry curvature against the Berry phase of a small plaquette (a Wilson loop, including
  the line integral of the position operator's diagonal), quantum metric against
  ||(1 - P_n) D_a u_n||^2 with the covariant difference D_a = d_a - i A_W^a;
* two-band closed forms (d-vector formulas) for the metric, the curvature and the injection
  current, and a Chern number: the occupied Berry curvature and the intrinsic AHC of a
  Qi-Wu-Zhang lattice model average over the zone to C / (2 pi) with C = +-1 or 0.
"""
import numpy as np
import pytest

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import TightBindingModel, synthetic_orthogonal_model

FD8 = ((1, 4.0 / 5.0), (2, -1.0 / 5.0), (3, 4.0 / 105.0), (4, -1.0 / 280.0))
E_C = 1.602176634e-19
HBAR_JS = 1.054571817e-34
HBAR_EVS = 6.582119569e-16


class Bands:
    """Numpy Fourier sums and LAPACK eigenvectors of an orthogonal model at Cartesian k."""

    def __init__(self, model: TightBindingModel):
        self.model = model
        self.rc = model.lattice.T @ model.r_vectors   # Cartesian R [3, NR] (lattice rows = vectors)
        self.nw = model.num_orbitals

    def kcart(self, kfrac):
        return 2.0 * np.pi * np.linalg.solve(self.model.lattice, np.asarray(kfrac, dtype=float))

    def parts(self, kc):
        ph = np.exp(1j * (self.rc.T @ kc)) / self.model.r_degeneracies
        H = np.einsum("ijr,r->ij", self.model.hamiltonian_r, ph)
        dH = [np.einsum("ijr,r->ij", self.model.hamiltonian_r, ph * 1j * self.rc[a]) for a in range(3)]
        if self.model.position_r is None:
            A = [np.zeros((self.nw, self.nw), complex) for _ in range(3)]
        else:
            A = [np.einsum("ijr,r->ij", self.model.position_r[:, :, a, :], ph) for a in range(3)]
        return H, dH, A

    def frame(self, kc, ref):
        """Energies, eigenvectors in the parallel-transport gauge of `ref` (<ref_n|u_n> real
        positive), dH and A at Cartesian kc."""
        H, dH, A = self.parts(kc)
        E, U = np.linalg.eigh(H)
        for n in range(self.nw):
            U[:, n] *= np.exp(-1j * np.angle(np.vdot(ref[:, n], U[:, n])))
        return E, U, dH, A


def connection(E, U, dH, A):
    """r^b = U^H A_b U + i D_b with bare inverses, D_nm = -(dH_b)_nm / (E_n - E_m), D_nn = 0."""
    d = E[:, None] - E[None, :]
    inv = np.where(d == 0.0, 0.0, 1.0 / np.where(d == 0.0, 1.0, d))
    return [U.conj().T @ A[b] @ U + 1j * (-(U.conj().T @ dH[b] @ U) * inv) for b in range(3)]


def derivative(fn, kc, a, h):
    """Eighth-order central difference of fn along Cartesian axis a (fn returns a list of arrays)."""
    acc = None
    for j, c in FD8:
        for sgn in (1, -1):
            kk = kc.copy()
            kk[a] += sgn * j * h
            vals = fn(kk)
            term = [sgn * c * v / h for v in vals]
            acc = term if acc is None else [x + y for x, y in zip(acc, term)]
    return acc


def fd_geometry(model, kfrac, oracle_mod, h=5e-3):
    """From differences only: r (oracle frame), d_a r^b, d_a E and the parallel-transport
    eigenvector derivatives, all in the oracle's canonical frame at k."""
    bands = Bands(model)
    kc = bands.kcart(kfrac)
    e, u, r_or, g_or, f_or = oracle_mod.kpoint_geometry(model, kfrac, 0.0)
    E0, U0, dH0, A0 = bands.frame(kc, u)
    r0 = connection(E0, U0, dH0, A0)
    dr = [derivative(lambda kk: connection(*bands.frame(kk, u)), kc, a, h) for a in range(3)]
    dE = [derivative(lambda kk: [bands.frame(kk, u)[0]], kc, a, h)[0] for a in range(3)]
    dU = [derivative(lambda kk: [bands.frame(kk, u)[1]], kc, a, h)[0] for a in range(3)]
    return dict(bands=bands, kc=kc, E=E0, U=U0, A=A0, r=r0, dr=dr, dE=dE, dU=dU, oracle=(e, u, r_or, g_or, f_or))


def fd_gder(geo):
    """r^b_{nm;a} = d_a r^b_nm - i (A^a_nn - A^a_mm) r^b_nm in the parallel-transport gauge
    (where the diagonal Bloch connection vanishes at k), indexed [n, m, b, a]."""
    n = geo["E"].size
    out = np.zeros((n, n, 3, 3), complex)
    for a in range(3):
        Ad = np.real(np.diag(geo["r"][a]))
        for b in range(3):
            out[:, :, b, a] = geo["dr"][a][b] - 1j * (Ad[:, None] - Ad[None, :]) * geo["r"][b]
    return out


MODELS = {
    "nw4_full_position": lambda: synthetic_orthogonal_model(4, 1, 3, full_position=True),
    "nw6_full_position": lambda: synthetic_orthogonal_model(6, 1, 8, full_position=True),
    "nw4_diagonal_position": lambda: synthetic_orthogonal_model(4, 2, 0),
}
KPOINTS = [(0.13, 0.29, 0.41), (0.71, 0.05, 0.33)]


@pytest.mark.parametrize("name", sorted(MODELS))
@pytest.mark.parametrize("kfrac", KPOINTS)
def test_generalized_derivative_matches_finite_difference(oracle_mod, name, kfrac):
    geo = fd_geometry(MODELS[name](), np.array(kfrac), oracle_mod)
    g_or = geo["oracle"][3]
    g_fd = fd_gder(geo)
    off = ~np.eye(geo["E"].size, dtype=bool)
    err = max(np.abs(g_fd[:, :, b, a] - g_or[:, :, b, a])[off].max() for a in range(3) for b in range(3))
    assert err <= 1e-10 * np.abs(g_or).max(), err


@pytest.mark.parametrize("name", sorted(MODELS))
def test_connection_matches_differenced_eigenvectors(oracle_mod, name):
    """r^b_nm (n != m) = (U^H A_b U)_nm + i (U^H d_b U)_nm from differenced eigenvectors."""
    geo = fd_geometry(MODELS[name](), np.array(KPOINTS[0]), oracle_mod)
    r_or = geo["oracle"][2]
    U = geo["U"]
    off = ~np.eye(geo["E"].size, dtype=bool)
    for b in range(3):
        r_fd = U.conj().T @ geo["A"][b] @ U + 1j * (U.conj().T @ geo["dU"][b])
        assert np.abs(r_fd - r_or[:, :, b])[off].max() <= 1e-10 * np.abs(r_or).max()


@pytest.mark.parametrize("name", sorted(MODELS))
def test_shift_vector_identity(oracle_mod, name):
    """Q^{abb}_nm = -i (r^b_{nm;a} r^b_mn - r^b_{mn;a} r^b_nm) = 2 |r^b_nm|^2 R^{a,b}_nm with the
    shift vector R = d_a phi^b_nm - A^a_nn + A^a_mm, phi = arg r^b_nm differenced in the
    parallel-transport gauge."""
    model = MODELS[name]()
    geo = fd_geometry(model, np.array(KPOINTS[1]), oracle_mod)
    e, u, r_or, g_or, _ = geo["oracle"]
    n = e.size
    bands, kc = geo["bands"], geo["kc"]
    phase0 = [np.angle(geo["r"][b]) for b in range(3)]

    def phases(kk):
        rr = connection(*bands.frame(kk, u))
        # unwrap against the central phase
        return [phase0[b] + np.angle(rr[b] * np.exp(-1j * phase0[b])) for b in range(3)]

    for a in range(3):
        dphi = derivative(phases, kc, a, 2.5e-3)
        Ad = np.real(np.diag(geo["r"][a]))
        for b in range(3):
            q_or = -1j * (g_or[:, :, b, a] * r_or[:, :, b].T - g_or[:, :, b, a].T * r_or[:, :, b])
            shift = dphi[b] - Ad[:, None] + Ad[None, :]
            q_sv = 2.0 * np.abs(geo["r"][b]) ** 2 * shift
            off = ~np.eye(n, dtype=bool)
            assert np.abs(q_or.imag[off]).max() <= 1e-12 * np.abs(q_or).max()
            assert np.abs(q_or.real - q_sv)[off].max() <= 1e-9 * np.abs(q_or).max()


def _sc_ic_numpy(geo, omegas, eta, comps, kind, vol):
    """Per-k shift or injection current from the differenced geometry (T = 0, mu = 0)."""
    E = geo["E"]
    n = E.size
    f = (E <= 0.0).astype(float)
    r = geo["r"]
    g = fd_gder(geo)
    P_sc = HBAR_EVS * np.pi * (-E_C) ** 3 / (2.0 * HBAR_JS ** 2 * vol)
    P_ic = -np.pi * E_C ** 3 / (HBAR_JS ** 2 * vol)
    out = np.zeros((len(omegas), len(comps)), complex)
    for ci, comp in enumerate(comps):
        a, b, c = ["xyz".index(x) for x in comp]
        for nn in range(n):
            for mm in range(n):
                fnm = f[nn] - f[mm]
                if nn == mm or abs(fnm) <= 1e-10:
                    continue
                if kind == "sc":
                    q = -1j * (g[nn, mm, c, a] * r[b][mm, nn] - g[mm, nn, b, a] * r[c][nn, mm])
                    pref = P_sc
                else:
                    q = (geo["dE"][a][mm] - geo["dE"][a][nn]) * r[c][nn, mm] * r[b][mm, nn]
                    pref = P_ic
                x = (E[mm] - E[nn]) - np.asarray(omegas)
                out[:, ci] += pref * fnm * (eta / np.pi) / (x * x + eta * eta) * q
    return out


@pytest.mark.parametrize("kind", ["sc", "ic"])
@pytest.mark.parametrize("name", ["nw4_full_position", "nw6_full_position"])
def test_current_point_values_from_finite_differences(oracle_mod, kind, name):
    model = MODELS[name]()
    kfrac = np.array(KPOINTS[0])
    geo = fd_geometry(model, kfrac, oracle_mod)
    omegas = np.linspace(0.05, 4.0, 40)
    comps = ["xyy", "yzx", "zzz"]
    resp = _abi.SHIFT_CURRENT if kind == "sc" else _abi.INJECTION_CURRENT
    task = _abi.TaskArrays([(resp, comps)], broadening_type=_abi.LORENTZIAN, broadening=0.05,
                           photon_energies=omegas, denominator_regularization=0.0, transition_window_factor=1e3)
    got = oracle_mod.point_values(model, task, kfrac[None])[0].reshape(len(comps), len(omegas)).T
    ref = _sc_ic_numpy(geo, omegas, 0.05, comps, kind, abs(np.linalg.det(model.lattice)))
    assert np.abs(got - ref).max() <= 1e-9 * np.abs(ref).max()


def _band_values(oracle_mod, model, kind, comp, kfrac, eta):
    """Per-band Omega_n or g_n from the oracle's occupied sums at Fermi levels between bands."""
    e = oracle_mod.kpoint_spectrum(model, kfrac)[0]
    mids = np.concatenate([[e[0] - 1.0], 0.5 * (e[1:] + e[:-1]), [e[-1] + 1.0]])
    sums = []
    for mu in mids:
        task = _abi.TaskArrays([(kind, [comp])], fermi_energy=mu, denominator_regularization=eta)
        sums.append(oracle_mod.point_values(model, task, kfrac[None])[0, 0].real)
    return np.diff(sums)


def _plaquette_curvature(bands, kc, U0, n, a, b, side):
    """Berry phase of band n around a square of the given side in the (a, b) plane, over its
    area: the Bloch part from the overlap product, the position operator's diagonal by a
    three-point Gauss-Legendre line integral along each edge."""
    ea, eb = np.eye(3)[a], np.eye(3)[b]
    corners = [kc + side / 2 * (-ea - eb), kc + side / 2 * (ea - eb), kc + side / 2 * (ea + eb),
               kc + side / 2 * (-ea + eb)]
    vecs = [bands.frame(q, U0)[1][:, n] for q in corners]
    w = 1.0
    for i in range(4):
        w *= np.vdot(vecs[i], vecs[(i + 1) % 4])
    phase = -np.angle(w)
    gl_x = np.array([-np.sqrt(0.6), 0.0, np.sqrt(0.6)])
    gl_w = np.array([5.0, 8.0, 5.0]) / 9.0
    line = 0.0
    for i in range(4):
        k0, k1 = corners[i], corners[(i + 1) % 4]
        for x, wt in zip(gl_x, gl_w):
            q = 0.5 * (k0 + k1) + 0.5 * x * (k1 - k0)
            E, U, dH, A = bands.frame(q, U0)
            a_diag = np.array([np.real(np.vdot(U[:, n], A[c] @ U[:, n])) for c in range(3)])
            line += 0.5 * wt * a_diag @ (k1 - k0)
    return (phase + line) / side ** 2


@pytest.mark.parametrize("name", ["nw4_full_position", "nw4_diagonal_position"])
def test_band_berry_curvature_matches_plaquette_phase(oracle_mod, name):
    model = MODELS[name]()
    kfrac = np.array(KPOINTS[0])
    bands = Bands(model)
    kc = bands.kcart(kfrac)
    _, u, _, _, _ = oracle_mod.kpoint_geometry(model, kfrac, 0.0)
    for comp in ("xy", "yz"):
        a, b = ["xyz".index(x) for x in comp]
        omega = _band_values(oracle_mod, model, _abi.BERRY_CURVATURE, comp, kfrac, 0.0)
        for n in range(model.num_orbitals):
            # Richardson: the plaquette error is even in the side.
            s = 4e-3
            om = (4.0 * _plaquette_curvature(bands, kc, u, n, a, b, s / 2) -
                  _plaquette_curvature(bands, kc, u, n, a, b, s)) / 3.0
            assert abs(om - omega[n]) <= 1e-7 * max(1.0, np.abs(omega).max())


@pytest.mark.parametrize("name", ["nw4_full_position", "nw6_full_position"])
def test_band_quantum_metric_matches_covariant_differences(oracle_mod, name):
    """g_n^{ab} = Re <D_a u_n|(1 - P_n)|D_b u_n>, D_a = d_a - i A_W^a, from differenced vectors."""
    model = MODELS[name]()
    kfrac = np.array(KPOINTS[1])
    geo = fd_geometry(model, kfrac, oracle_mod)
    U, A = geo["U"], geo["A"]
    for comp in ("xx", "xy", "zy"):
        a, b = ["xyz".index(x) for x in comp]
        g_or = _band_values(oracle_mod, model, _abi.QUANTUM_METRIC, comp, kfrac, 0.0)
        for n in range(model.num_orbitals):
            un = U[:, n]
            proj = np.eye(model.num_orbitals) - np.outer(un, un.conj())
            da = geo["dU"][a][:, n] - 1j * A[a] @ un
            db = geo["dU"][b][:, n] - 1j * A[b] @ un
            g_fd = np.real(np.vdot(da, proj @ db))
            assert abs(g_fd - g_or[n]) <= 1e-10 * max(1.0, np.abs(g_or).max())


# ---- two-band closed forms and a Chern number ------------------------------------------------

PAULI = [np.array([[0, 1], [1, 0]], complex), np.array([[0, -1j], [1j, 0]]), np.diag([1.0, -1.0]).astype(complex)]


def two_band_model(mass: float, tz: float = 0.5, sz_x: float = 0.3) -> TightBindingModel:
    """d(k) = (sin kx + sz_x sin kz, sin ky, mass + cos kx + cos ky + tz cos kz), H = d . sigma,
    lattice = identity (Angstrom); tz = sz_x = 0 gives the Qi-Wu-Zhang model."""
    terms = {}   # R -> 2x2 block

    def add(R, mat):
        terms.setdefault(R, np.zeros((2, 2), complex))
        terms[R] += mat

    add((0, 0, 0), mass * PAULI[2])
    for axis, (sin_coef, sin_pauli), cos_coef in (((1, 0, 0), (1.0, 0), 1.0), ((0, 1, 0), (1.0, 1), 1.0),
                                                   ((0, 0, 1), (sz_x, 0), tz)):
        plus, minus = axis, tuple(-x for x in axis)
        add(plus, sin_coef * PAULI[sin_pauli] / 2j + cos_coef * PAULI[2] / 2)
        add(minus, -sin_coef * PAULI[sin_pauli] / 2j + cos_coef * PAULI[2] / 2)
    keys = sorted(terms)
    ham = np.zeros((2, 2, len(keys)), complex, order="F")
    for i, R in enumerate(keys):
        ham[:, :, i] = terms[R]
    rv = np.asfortranarray(np.array(keys, dtype=np.int64).T)
    return TightBindingModel(np.eye(3), rv, np.ones(len(keys), dtype=np.int64), ham, None)


def d_vector(kc, mass, tz=0.5, sz_x=0.3):
    kx, ky, kz = kc
    d = np.array([np.sin(kx) + sz_x * np.sin(kz), np.sin(ky), mass + np.cos(kx) + np.cos(ky) + tz * np.cos(kz)])
    jac = np.array([[np.cos(kx), 0.0, sz_x * np.cos(kz)],
                    [0.0, np.cos(ky), 0.0],
                    [-np.sin(kx), -np.sin(ky), -tz * np.sin(kz)]])   # jac[i, a] = d d_i / d k_a
    return d, jac


def dhat_derivatives(d, jac):
    norm = np.linalg.norm(d)
    dh = d / norm
    return dh, [(jac[:, a] - dh * (dh @ jac[:, a])) / norm for a in range(3)]


def test_two_band_metric_curvature_injection_closed_forms(oracle_mod):
    mass = 1.3
    model = two_band_model(mass)
    for kfrac in ([0.11, 0.23, 0.37], [0.41, 0.07, 0.83]):
        kfrac = np.array(kfrac)
        kc = 2 * np.pi * kfrac
        d, jac = d_vector(kc, mass)
        dh, ddh = dhat_derivatives(d, jac)
        for comp in ("xy", "yz", "xz", "yy"):
            a, b = ["xyz".index(x) for x in comp]
            g = _band_values(oracle_mod, model, _abi.QUANTUM_METRIC, comp, kfrac, 0.0)
            np.testing.assert_allclose(g, 0.25 * ddh[a] @ ddh[b], rtol=1e-12, atol=1e-14)
            om = _band_values(oracle_mod, model, _abi.BERRY_CURVATURE, comp, kfrac, 0.0)
            ref = 0.5 * dh @ np.cross(ddh[a], ddh[b])
            np.testing.assert_allclose(om, [ref, -ref], rtol=1e-12, atol=1e-14)
        # Injection current xyy: P 2 d_x|d| |r^y_vc|^2 [L(2|d| - w) + L(-2|d| - w)], |r^y|^2 = g^yy.
        omegas = np.linspace(0.5, 6.0, 23)
        eta = 0.03
        task = _abi.TaskArrays([(_abi.INJECTION_CURRENT, ["xyy"])], broadening_type=_abi.LORENTZIAN, broadening=eta,
                               photon_energies=omegas, denominator_regularization=0.0, transition_window_factor=1e3)
        got = oracle_mod.point_values(model, task, kfrac[None])[0]
        norm = np.linalg.norm(d)
        dnorm_x = dh @ jac[:, 0]
        lor = lambda x: (eta / np.pi) / (x * x + eta * eta)
        P_ic = -np.pi * E_C ** 3 / HBAR_JS ** 2
        ref = P_ic * 2 * dnorm_x * 0.25 * (ddh[1] @ ddh[1]) * (lor(2 * norm - omegas) + lor(-2 * norm - omegas))
        np.testing.assert_allclose(got.real, ref, rtol=1e-12, atol=1e-14 * np.abs(ref).max())
        assert np.abs(got.imag).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("mass,chern", [(1.0, -1), (-1.0, 1), (3.0, 0)])
def test_qwz_chern_number_from_mesh_curvature(oracle_mod, mass, chern):
    """The occupied Berry curvature and the intrinsic AHC of the Qi-Wu-Zhang model (mu = 0 in the
    gap) average over a 64 x 64 mesh to C / (2 pi) (Angstrom^2): the curvature is analytic, so the
    mesh average converges exponentially to the integer (C = -1 for 0 < m < 2 in the convention
    Omega = d_x A_y - d_y A_x, A = i <u|grad u>, which the plaquette test above fixes)."""
    model = two_band_model(mass, tz=0.0, sz_x=0.0)
    mesh = (64, 64, 1)
    # Bare denominators: the default 1e-3 eV regularization shifts the curvature by ~eta^2/gap^2.
    bc = _abi.TaskArrays([(_abi.BERRY_CURVATURE, ["xy"])], fermi_energy=0.0, denominator_regularization=0.0)
    ahc = _abi.TaskArrays([(_abi.INTRINSIC_AHC, ["xy"])], fermi_energies=[0.0])
    for task in (bc, ahc):
        mean = oracle_mod.integrate_mesh(model, task, mesh)[0].real
        assert abs(2 * np.pi * mean - chern) <= 1e-12
