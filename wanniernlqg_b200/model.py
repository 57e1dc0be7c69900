"""Tight-binding model container, `_tb.dat` reader/writer and the seeded synthetic models.

The container mirrors ``TightBindingModel`` (src/Core/Models.jl:11-75): row-stored
lattice vectors in Angstrom, integer ``r_vectors[3, NR]``, ``r_degeneracies[NR]``,
``hamiltonian_r[nw, nw, NR]`` in eV and ``position_r[nw, nw, 3, NR]`` in Angstrom.
Arrays are kept in Fortran (column-major) order so that their memory is exactly the
memory of the Julia arrays; the C ABI (``include/wnlqg_b200.h``) reads that layout.

The nonorthogonal variant adds ``overlap_r[nw, nw, NR]`` (S(R)), following
``NonorthogonalLocalizedModel`` (src/Core/NonorthogonalLocalizedModels.jl).
"""
from __future__ import annotations

import dataclasses
import itertools
from typing import Optional

import numpy as np


@dataclasses.dataclass
class TightBindingModel:
    lattice: np.ndarray            # (3, 3) float64, rows are lattice vectors (Angstrom)
    r_vectors: np.ndarray          # (3, NR) int64
    r_degeneracies: np.ndarray     # (NR,) int64
    hamiltonian_r: np.ndarray      # (nw, nw, NR) complex128, Fortran order
    position_r: Optional[np.ndarray] = None   # (nw, nw, 3, NR) complex128, Fortran order
    overlap_r: Optional[np.ndarray] = None    # (nw, nw, NR) complex128, Fortran order

    def __post_init__(self):
        self.lattice = np.asfortranarray(np.asarray(self.lattice, dtype=np.float64))
        self.r_vectors = np.asfortranarray(np.asarray(self.r_vectors, dtype=np.int64))
        self.r_degeneracies = np.ascontiguousarray(np.asarray(self.r_degeneracies, dtype=np.int64))
        self.hamiltonian_r = np.asfortranarray(np.asarray(self.hamiltonian_r, dtype=np.complex128))
        if self.position_r is not None:
            self.position_r = np.asfortranarray(np.asarray(self.position_r, dtype=np.complex128))
        if self.overlap_r is not None:
            self.overlap_r = np.asfortranarray(np.asarray(self.overlap_r, dtype=np.complex128))
        nw = self.num_orbitals
        nr = self.num_r_vectors
        if self.lattice.shape != (3, 3):
            raise ValueError("lattice must be 3x3")
        if self.r_vectors.shape != (3, nr) or self.r_degeneracies.shape != (nr,):
            raise ValueError("r_vectors must be (3, NR) and r_degeneracies (NR,)")
        if self.hamiltonian_r.shape != (nw, nw, nr):
            raise ValueError("hamiltonian_r must be (nw, nw, NR)")
        if self.position_r is not None and self.position_r.shape != (nw, nw, 3, nr):
            raise ValueError("position_r must be (nw, nw, 3, NR)")
        if self.overlap_r is not None and self.overlap_r.shape != (nw, nw, nr):
            raise ValueError("overlap_r must be (nw, nw, NR)")
        if np.any(self.r_degeneracies <= 0):
            raise ValueError("r_degeneracies must be positive")

    @property
    def num_orbitals(self) -> int:
        return int(self.hamiltonian_r.shape[0])

    @property
    def num_r_vectors(self) -> int:
        return int(self.hamiltonian_r.shape[2])

    @property
    def cell_volume(self) -> float:
        """det(lattice), the measure the integral driver divides by (Runtime/NativeModelRuntime.jl:600)."""
        return float(np.linalg.det(self.lattice))

    def real_position(self) -> np.ndarray:
        """position_r, or zeros when the model carries none."""
        if self.position_r is not None:
            return self.position_r
        return np.zeros((self.num_orbitals, self.num_orbitals, 3, self.num_r_vectors),
                        dtype=np.complex128, order="F")


def read_wannier_tb(filename: str) -> TightBindingModel:
    """Read a Wannier90 ``_tb.dat`` file (follows src/IO/WannierTB.jl:53-127).

    Layout: title, three lattice rows, num_wann, nrpts, degeneracies 15 per line, then one
    Hamiltonian block per R (blank line, R, then nw*nw lines ``m n Re Im`` with the row
    index fastest), then one position block per R (blank, R, nw*nw lines with three complex
    Cartesian components).
    """
    with open(filename, "r") as fh:
        lines = fh.read().split("\n")
    pos = 0

    def nextline():
        nonlocal pos
        line = lines[pos]
        pos += 1
        return line

    nextline()
    lattice = np.zeros((3, 3))
    for i in range(3):
        lattice[i, :] = [float(x) for x in nextline().split()]
    nw = int(nextline())
    nr = int(nextline())
    degs = []
    for _ in range((nr + 14) // 15):
        degs.extend(int(x) for x in nextline().split())
    if len(degs) != nr:
        raise ValueError("degeneracy count does not match nrpts")
    rvec = np.zeros((3, nr), dtype=np.int64)
    ham = np.zeros((nw, nw, nr), dtype=np.complex128, order="F")
    pos_r = np.zeros((nw, nw, 3, nr), dtype=np.complex128, order="F")
    for ir in range(nr):
        nextline()
        rvec[:, ir] = [int(x) for x in nextline().split()]
        for col in range(nw):
            for row in range(nw):
                v = nextline().split()
                ham[row, col, ir] = complex(float(v[2]), float(v[3]))
    for ir in range(nr):
        nextline()
        nextline()
        for col in range(nw):
            for row in range(nw):
                v = nextline().split()
                vals = [float(x) for x in v[2:8]]
                for a in range(3):
                    pos_r[row, col, a, ir] = complex(vals[2 * a], vals[2 * a + 1])
    return TightBindingModel(lattice, rvec, np.asarray(degs), ham, pos_r)


def write_wannier_tb(model: TightBindingModel, filename: str, title: str = "wnlqg-b200 synthetic model") -> None:
    """Write the model in the ``_tb.dat`` layout that :func:`read_wannier_tb` (and the Julia reader) parse."""
    nw, nr = model.num_orbitals, model.num_r_vectors
    pos_r = model.real_position()
    out = [title]
    for i in range(3):
        out.append(" ".join(f"{x:.17e}" for x in model.lattice[i]))
    out.append(str(nw))
    out.append(str(nr))
    for start in range(0, nr, 15):
        out.append(" ".join(str(int(d)) for d in model.r_degeneracies[start:start + 15]))
    for ir in range(nr):
        out.append("")
        out.append(" ".join(str(int(x)) for x in model.r_vectors[:, ir]))
        for col in range(nw):
            for row in range(nw):
                h = model.hamiltonian_r[row, col, ir]
                out.append(f"{row + 1} {col + 1} {h.real:.17e} {h.imag:.17e}")
    for ir in range(nr):
        out.append("")
        out.append(" ".join(str(int(x)) for x in model.r_vectors[:, ir]))
        for col in range(nw):
            for row in range(nw):
                p = pos_r[row, col, :, ir]
                out.append(f"{row + 1} {col + 1} " + " ".join(f"{z.real:.17e} {z.imag:.17e}" for z in p))
    with open(filename, "w") as fh:
        fh.write("\n".join(out) + "\n")


# ----------------------------------------------------------------------------------------
# Seeded synthetic models (numpy PCG64 through default_rng).  |R| is the Cartesian norm
# with the identity lattice (Angstrom).  Hermitian pairing H(-R) = H(R)^dagger is exact.
# ----------------------------------------------------------------------------------------

def _cube(rmax: int) -> np.ndarray:
    pts = list(itertools.product(range(-rmax, rmax + 1), repeat=3))
    return np.array(pts, dtype=np.int64).T  # (3, NR), lexicographic with the last index fastest


def _paired_gaussian(rng, nw, rvecs, sigma_of_norm, zero_diag_value=None):
    """Complex Gaussian blocks X(R) ~ CN(0, sigma(|R|)^2) with X(-R) = X(R)^dagger.

    Real and imaginary parts each carry variance sigma^2/2.  R=0 is Hermitian; its diagonal
    is replaced by ``zero_diag_value`` when given (a real vector).
    """
    nr = rvecs.shape[1]
    out = np.zeros((nw, nw, nr), dtype=np.complex128, order="F")
    index = {tuple(rvecs[:, i]): i for i in range(nr)}
    norms = np.linalg.norm(rvecs.astype(np.float64), axis=0)
    for i in range(nr):
        r = tuple(rvecs[:, i])
        neg = tuple(-x for x in r)
        j = index[neg]
        if j < i:
            continue
        sig = sigma_of_norm(norms[i])
        block = (rng.standard_normal((nw, nw)) + 1j * rng.standard_normal((nw, nw))) * (sig / np.sqrt(2.0))
        if j == i:  # R = 0: Hermitian block
            block = np.triu(block, 1)
            block = block + block.conj().T
            if zero_diag_value is not None:
                block[np.diag_indices(nw)] = zero_diag_value
            else:
                block[np.diag_indices(nw)] = rng.standard_normal(nw) * sig
            out[:, :, i] = block
        else:
            out[:, :, i] = block
            out[:, :, j] = block.conj().T
    return out


def synthetic_orthogonal_model(nw: int, rmax: int, seed: int = 0, *, full_position: bool = False,
                               hopping_scale: float = 0.3, position_scale: float = 0.05,
                               position_decay: float = 1.5,
                               onsite_shift: Optional[np.ndarray] = None) -> TightBindingModel:
    """The orthogonal synthetic Wannier model of the reference workloads.

    H(R) entries (except the home-cell diagonal) ~ CN(0, (hopping_scale*exp(-|R|))^2) eV,
    Hermitian-paired; home-cell diagonal ~ U[-1, 1] eV.  Orbital centres tau ~ U[0,1)^3 sit on
    the home-cell diagonal of A(R).  With ``full_position`` every other A(R) entry is
    CN(0, (position_scale*exp(-|R|/position_decay))^2) Angstrom, Hermitian-paired per axis.
    """
    rng = np.random.default_rng(seed)
    rvecs = _cube(rmax)
    nr = rvecs.shape[1]
    onsite = rng.uniform(-1.0, 1.0, nw)
    if onsite_shift is not None:
        onsite = onsite + np.asarray(onsite_shift, dtype=np.float64)
    ham = _paired_gaussian(rng, nw, rvecs, lambda n: hopping_scale * np.exp(-n), zero_diag_value=onsite)
    tau = rng.uniform(0.0, 1.0, (nw, 3))
    pos = np.zeros((nw, nw, 3, nr), dtype=np.complex128, order="F")
    home = int(np.where(np.all(rvecs == 0, axis=0))[0][0])
    for a in range(3):
        if full_position:
            pos[:, :, a, :] = _paired_gaussian(rng, nw, rvecs,
                                               lambda n: position_scale * np.exp(-n / position_decay),
                                               zero_diag_value=tau[:, a])
        else:
            pos[np.arange(nw), np.arange(nw), a, home] = tau[:, a]
    return TightBindingModel(np.eye(3), rvecs, np.ones(nr, dtype=np.int64), ham, pos)


def synthetic_nonorthogonal_model(nw: int, rmax: int, seed: int = 0, *, overlap_scale: float = 0.05,
                                  min_overlap_eig: float = 0.5, full_position: bool = False) -> TightBindingModel:
    """Orthogonal generator plus S(R) = delta_R0 I + overlap_scale*exp(-|R|)*CN, Hermitian-paired.

    The off-identity part is rescaled so that min over k of eig S(k) >= ``min_overlap_eig``
    (a bound from sum_R ||X(R)||_2, which bounds every ||X(k)||_2).
    """
    base = synthetic_orthogonal_model(nw, rmax, seed, full_position=full_position)
    rng = np.random.default_rng(seed + 7919)
    rvecs = base.r_vectors
    x = _paired_gaussian(rng, nw, rvecs, lambda n: overlap_scale * np.exp(-n), zero_diag_value=np.zeros(nw))
    bound = sum(np.linalg.norm(x[:, :, i], 2) for i in range(x.shape[2]))
    limit = 1.0 - min_overlap_eig
    if bound > limit:
        x *= limit / bound
    home = int(np.where(np.all(rvecs == 0, axis=0))[0][0])
    x[:, :, home] += np.eye(nw)
    base.overlap_r = np.asfortranarray(x)
    return base


def kramers_doubled_model(model: TightBindingModel, lam: float = 1e-3, seed: int = 0) -> TightBindingModel:
    """H (x) I_2 plus the home-cell orbital-mixing term i lam (M (x) sigma_z) with a real
    antisymmetric M (Hermitian: (i lam M (x) sigma_z)^H = i lam M (x) sigma_z), which splits the
    doubled bands by O(lam) and so creates near-degenerate pairs; positions A (x) I_2."""
    rng = np.random.default_rng(seed)
    nw, nr = model.num_orbitals, model.num_r_vectors
    x = rng.standard_normal((nw, nw))
    M = (x - x.T) / 2.0
    sz = np.diag([1.0, -1.0])
    ham = np.zeros((2 * nw, 2 * nw, nr), dtype=np.complex128, order="F")
    for r in range(nr):
        ham[:, :, r] = np.kron(model.hamiltonian_r[:, :, r], np.eye(2))
    home = int(np.where(np.all(model.r_vectors == 0, axis=0))[0][0])
    ham[:, :, home] += 1j * lam * np.kron(M, sz)
    pos = None
    if model.position_r is not None:
        pos = np.zeros((2 * nw, 2 * nw, 3, nr), dtype=np.complex128, order="F")
        for r in range(nr):
            for a in range(3):
                pos[:, :, a, r] = np.kron(model.position_r[:, :, a, r], np.eye(2))
    return TightBindingModel(model.lattice.copy(), model.r_vectors.copy(), model.r_degeneracies.copy(), ham, pos)


def crossing_model(nw: int = 16, rmax: int = 2, seed: int = 0, *, grid: int = 20) -> TightBindingModel:
    """The synthetic model with its onsite energies shifted so that two bands cross at the Fermi
    level mu = 0: the adjacent pair (n, n+1) around the middle of the spectrum whose direct gap
    min_k (E_{n+1} - E_n) is smallest on a grid^3 mesh is located, the minimum refined by a
    Nelder-Mead search in k, and every home-cell diagonal energy shifted by the midpoint of the two
    bands there (a uniform shift: the spectrum moves rigidly).  The pair's energies at the
    crossing are then within the minimum gap (a Weyl point in 3D without symmetry: usually below
    1e-3 eV) of mu = 0."""
    from scipy.optimize import minimize

    base = synthetic_orthogonal_model(nw, rmax, seed, full_position=True)
    rv = base.r_vectors.astype(np.float64)

    def energies(kfrac):
        ph = np.exp(2j * np.pi * (rv.T @ np.asarray(kfrac))) / base.r_degeneracies
        return np.linalg.eigvalsh(np.einsum("ijr,r->ij", base.hamiltonian_r, ph))

    g = (np.arange(grid) + 0.5) / grid
    kz, ky, kx = np.meshgrid(g, g, g, indexing="ij")
    ks = np.stack([kx.ravel(), ky.ravel(), kz.ravel()], axis=1)
    ph = np.exp(2j * np.pi * (ks @ rv)) / base.r_degeneracies
    hk = np.einsum("ijr,kr->kij", base.hamiltonian_r, ph)
    ev = np.linalg.eigvalsh(hk)
    mids = range(nw // 2 - 2, nw // 2 + 1)
    best = None
    for n in mids:
        gap = ev[:, n + 1] - ev[:, n]
        i = int(np.argmin(gap))
        res = minimize(lambda k: float(np.diff(energies(k % 1.0))[n]), ks[i], method="Nelder-Mead",
                       options={"xatol": 1e-10, "fatol": 1e-12, "maxiter": 4000})
        if best is None or res.fun < best[0]:
            best = (float(res.fun), n, res.x % 1.0)
    gap, n, kstar = best
    e = energies(kstar)
    shift = 0.5 * (e[n] + e[n + 1])
    ham = base.hamiltonian_r.copy(order="F")
    home = int(np.where(np.all(base.r_vectors == 0, axis=0))[0][0])
    ham[np.arange(nw), np.arange(nw), home] -= shift
    model = TightBindingModel(base.lattice.copy(), base.r_vectors.copy(), base.r_degeneracies.copy(), ham,
                              base.position_r.copy(order="F"))
    model.crossing = {"bands": (n, n + 1), "k": kstar, "gap_ev": gap}
    return model


def reference_workload_model(name: str) -> TightBindingModel:
    """Models of the reference workloads, by the short name used in tests and the bench.

    ``nw4``: nw=4, |R_i|<=2 (125 R), diagonal position operator (CPU-runnable case).
    ``nw32``: nw=32, |R_i|<=4 (729 R), full off-diagonal A(R).
    ``nw16_crossing``: nw=16, |R_i|<=2, onsite energies shifted so that two bands cross at 0 eV
    (:func:`crossing_model`).
    ``nw64_nonorth``: nw=64, |R_i|<=3 (343 R), with S(R).
    """
    if name == "nw4":
        return synthetic_orthogonal_model(4, 2, 0)
    if name == "nw32":
        return synthetic_orthogonal_model(32, 4, 0, full_position=True)
    if name == "nw16_crossing":
        return crossing_model(16, 2, 0)
    if name == "nw64_nonorth":
        return synthetic_nonorthogonal_model(64, 3, 0)
    raise KeyError(name)
