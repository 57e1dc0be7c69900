"""Symmetry-reduced Gamma-centred meshes for the q = 0 shift and injection currents.

Restates the reference's response-symmetry reduction:
  * the final-tensor action of a point-group operation (R x R x R for charge currents,
    R x det(R) R x R x R for spin currents; an antiunitary operation exchanges the two field
    indices and multiplies by +1 / -1 / -1 / +1 for shift / injection / shift spin / injection
    spin), its group average (the projector), the deterministic invariant basis and the
    component relations: src/Responses/Shared/ResponseSymmetry.jl:1-253;
  * the exact integer reciprocal action k' = s W^-T k on the mesh, its check that every
    operation permutes the complete mesh, and the orbits (smallest index as representative,
    orbit size as multiplicity): src/Runtime/ResponseSymmetryRuntime.jl:377-497;
  * the compact component plan (only components in the basis support are evaluated):
    src/Runtime/ResponseSymmetryRuntime.jl:730-800;
  * the reduced integral: representatives weighted by multiplicity / N_full, then X = B B^T of
    the sum, real and imaginary parts through their bases:
    src/Runtime/Execution/IntegralDriver.jl:811-846, src/Runtime/Setup/ExecutionState.jl:512-542,
    src/Runtime/ResponseSymmetryRuntime.jl:1121-1141.
The orbit search runs on the host (numpy, one vectorised pass per operation and sweep); the
representatives go to the device in one weighted call (ResponseEngine.mesh_weighted_sum, i.e.
wnlqg_b200_eval_mesh_weighted).
"""
from __future__ import annotations

import dataclasses
import itertools
import warnings
from typing import Callable, List, Optional, Sequence

import numpy as np

from . import _abi

QUANTITIES = ("shift_current", "injection_current", "shift_spin_current", "injection_spin_current")
_ANTIUNITARY_SIGN = {"shift_current": 1.0, "injection_current": -1.0,
                     "shift_spin_current": -1.0, "injection_spin_current": 1.0}
_KIND_QUANTITY = {_abi.SHIFT_CURRENT: "shift_current", _abi.INJECTION_CURRENT: "injection_current"}


@dataclasses.dataclass
class SymmetryOperation:
    """One point-group operation: integer fractional rotation W (acting on fractional real-space
    coordinates), its Cartesian rotation, and whether it is combined with time reversal."""
    rotation_fractional: np.ndarray
    rotation_cartesian: np.ndarray
    antiunitary: bool = False

    @classmethod
    def from_fractional(cls, W, lattice=None, antiunitary: bool = False) -> "SymmetryOperation":
        """Cartesian rotation A W A^-1 with A the matrix whose columns are the lattice vectors
        (`lattice` as stored by TightBindingModel: rows are lattice vectors; identity if None)."""
        W = np.asarray(W, dtype=np.int64)
        A = np.eye(3) if lattice is None else np.asarray(lattice, dtype=np.float64).T
        return cls(W, A @ W @ np.linalg.inv(A), bool(antiunitary))


def response_symmetry_sign(quantity: str) -> float:
    if quantity not in _ANTIUNITARY_SIGN:
        raise ValueError(f"response symmetry is not defined for quantity={quantity}")
    return _ANTIUNITARY_SIGN[quantity]


def response_component_tuples(quantity: str, spatial_dimension: int) -> List[tuple]:
    """0-based Cartesian tuples in result-column order (the last index varies fastest);
    spin currents carry the spin axis (always over x, y, z) second."""
    d = int(spatial_dimension)
    if d not in (1, 2, 3):
        raise ValueError("spatial_dimension must be 1, 2 or 3")
    response_symmetry_sign(quantity)
    if quantity.endswith("spin_current"):
        return [t for t in itertools.product(range(d), range(3), range(d), range(d))]
    return [t for t in itertools.product(range(d), repeat=3)]


def response_component_labels(quantity: str, spatial_dimension: int) -> List[str]:
    return ["".join("xyz"[i] for i in t) for t in response_component_tuples(quantity, spatial_dimension)]


def response_symmetry_action_matrix(quantity: str, spatial_dimension: int, rotation_cartesian,
                                    antiunitary: bool) -> np.ndarray:
    """Real matrix M with X' = M X on the flattened final tensor (same rule for real and
    imaginary parts): M[(a,b,c),(A,B,C)] = sign R[a,A] R[b',B] R[c',C], (b', c') = (c, b) for
    an antiunitary operation; spin currents insert det(R) R on the spin axis."""
    d = int(spatial_dimension)
    R = np.asarray(rotation_cartesian, dtype=np.float64)
    if R.shape != (3, 3):
        raise ValueError("rotation_cartesian must have shape (3, 3)")
    if not np.all(np.isfinite(R)):
        raise ValueError("rotation_cartesian is non-finite")
    resid = np.max(np.abs(R.T @ R - np.eye(3)))
    if resid > 1e-8:
        warnings.warn(f"rotation_cartesian orthogonality residual {resid} exceeds 1e-8; raw rotation retained")
    if d < 3 and (np.max(np.abs(R[:d, d:]), initial=0.0) > 1e-10 or np.max(np.abs(R[d:, :d]), initial=0.0) > 1e-10):
        raise ValueError("point-group operation rotates the active Cartesian subspace out of itself")
    sign = response_symmetry_sign(quantity) if antiunitary else 1.0
    Rd = R[:d, :d]
    if quantity.endswith("spin_current"):
        S = np.linalg.det(R) * R
        T = np.einsum("aA,sS,bB,cC->asbcASBC", Rd, S, Rd, Rd)
        if antiunitary:
            T = T.transpose(0, 1, 3, 2, 4, 5, 6, 7)
        n = d * 3 * d * d
    else:
        T = np.einsum("aA,bB,cC->abcABC", Rd, Rd, Rd)
        if antiunitary:
            T = T.transpose(0, 2, 1, 3, 4, 5)
        n = d ** 3
    M = sign * T.reshape(n, n)
    M[np.abs(M) < 1e-15] = 0.0
    return M


def response_symmetry_projector(quantity: str, spatial_dimension: int,
                                operations: Sequence[SymmetryOperation]) -> np.ndarray:
    """Group average of the action matrices (the operations must form the complete group)."""
    if not operations:
        raise ValueError("at least one point-group operation is required")
    P = sum(response_symmetry_action_matrix(quantity, spatial_dimension, op.rotation_cartesian, op.antiunitary)
            for op in operations) / len(operations)
    P[np.abs(P) < 1e-15] = 0.0
    return P


def response_symmetry_basis(projector: np.ndarray, tolerance: float = 1e-12) -> np.ndarray:
    """Orthonormal basis of the projector's range: columns of P in order, each orthogonalised
    twice against the accepted ones, kept above the rank floor max(tol, sqrt(eps) ||P||_2, ...),
    normalised and signed so that the first entry above the floor is positive."""
    P = np.asarray(projector, dtype=np.float64)
    if P.ndim != 2 or P.shape[0] != P.shape[1]:
        raise ValueError("response projector must be square")
    if not tolerance > 0.0:
        raise ValueError("basis tolerance must be positive")
    floor = max(float(tolerance), np.sqrt(np.finfo(np.float64).eps) * max(np.linalg.norm(P, 2), 1.0))
    accepted: List[np.ndarray] = []
    for j in range(P.shape[1]):
        v = P[:, j].copy()
        for _ in range(2):
            for b in accepted:
                v -= np.dot(b, v) * b
        nv = np.linalg.norm(v)
        if nv <= floor:
            continue
        v /= nv
        lead = np.nonzero(np.abs(v) > floor)[0]
        if lead.size == 0:
            continue
        if v[lead[0]] < 0.0:
            v = -v
        accepted.append(v)
    B = np.stack(accepted, axis=1) if accepted else np.zeros((P.shape[0], 0))
    B[np.abs(B) < 1e-15] = 0.0
    resid = np.max(np.abs(B @ B.T - P))
    if resid > 10 * floor:
        raise ValueError(f"response symmetry basis does not reconstruct its projector; residual={resid}")
    return B


@dataclasses.dataclass
class ResponseRelations:
    labels: List[str]
    forbidden: List[str]
    equal: List[tuple]
    opposite: List[tuple]
    constraint_matrix: np.ndarray


def response_symmetry_relations(quantity: str, spatial_dimension: int, projector: np.ndarray,
                                tolerance: float = 1e-10) -> ResponseRelations:
    """Forbidden components (zero projector rows), equal / opposite pairs (equal / negated rows)
    and the constraint matrix I - P."""
    labels = response_component_labels(quantity, spatial_dimension)
    P = np.asarray(projector, dtype=np.float64)
    if P.shape != (len(labels), len(labels)):
        raise ValueError("projector dimension disagrees with response tensor")
    forbidden = [labels[i] for i in range(len(labels)) if np.linalg.norm(P[i]) <= tolerance]
    equal, opposite = [], []
    for i in range(len(labels)):
        for j in range(i + 1, len(labels)):
            if np.linalg.norm(P[i] - P[j]) <= tolerance:
                equal.append((labels[i], labels[j]))
            if np.linalg.norm(P[i] + P[j]) <= tolerance:
                opposite.append((labels[i], labels[j]))
    C = np.eye(len(labels)) - P
    C[np.abs(C) < 1e-14] = 0.0
    return ResponseRelations(labels, forbidden, equal, opposite, C)


@dataclasses.dataclass
class ResponseTensorSymmetryPlan:
    quantity: str
    labels: List[str]
    projector: np.ndarray
    imaginary_projector: np.ndarray
    basis: np.ndarray
    imaginary_basis: np.ndarray
    relations: ResponseRelations
    basis_support_indices: List[int]
    raw_component_indices: List[int]
    accumulation_path: str
    idempotence_residual: float


def response_tensor_symmetry_plan(quantity: str, spatial_dimension: int, operations: Sequence[SymmetryOperation],
                                  *, numerical_reduction: bool = True, force_dense: bool = False) -> ResponseTensorSymmetryPlan:
    """Projector, basis (recomputed projector B B^T), relations and the components to evaluate:
    the basis support when it is smaller than the whole tensor (compact plan), else all."""
    raw = response_symmetry_projector(quantity, spatial_dimension, operations)
    resid = float(np.max(np.abs(raw @ raw - raw)))
    if resid > 1e-10:
        warnings.warn(f"response symmetry group-average idempotence residual {resid} exceeds 1e-10 for {quantity}")
    B = response_symmetry_basis(raw)
    Bi = response_symmetry_basis(raw)      # the imaginary-part action is the same matrix
    P, Pi = B @ B.T, Bi @ Bi.T
    support = sorted(set(np.nonzero(np.any(np.abs(B) > 1e-12, axis=1))[0].tolist())
                     | set(np.nonzero(np.any(np.abs(Bi) > 1e-12, axis=1))[0].tolist()))
    n = raw.shape[0]
    compact = numerical_reduction and not force_dense and len(support) < n
    path = ("full_kmesh_explanation_only" if not numerical_reduction else
            "selected_component_kernel_compact_coefficients" if compact else "dense_kernel_compact_coefficients")
    basis_support = np.nonzero(np.any(np.abs(B) > 1e-12, axis=1))[0].tolist()
    return ResponseTensorSymmetryPlan(quantity, response_component_labels(quantity, spatial_dimension), P, Pi, B, Bi,
                                      response_symmetry_relations(quantity, spatial_dimension, P), basis_support,
                                      support if compact else list(range(n)), path, resid)


def project_response_symmetry(tensor: np.ndarray, basis: np.ndarray, imaginary_basis: Optional[np.ndarray] = None) -> np.ndarray:
    """X <- B B^T X per energy slice, real part through `basis`, imaginary part through
    `imaginary_basis` (default: the same); tensor shape (n_energy, n_components)."""
    T = np.asarray(tensor)
    Bi = basis if imaginary_basis is None else imaginary_basis
    re = (T.real @ basis) @ basis.T
    im = (T.imag @ Bi) @ Bi.T
    return re + 1j * im


# -- mesh orbits ----------------------------------------------------------------------------------

def _mesh3(k_mesh) -> tuple:
    m = tuple(int(v) for v in k_mesh)
    if not 1 <= len(m) <= 3:
        raise ValueError("k mesh must have one to three entries")
    return m + (1,) * (3 - len(m))


def integer_action(operation: SymmetryOperation, k_mesh) -> np.ndarray:
    """Integer matrix acting on zero-based mesh coordinates: s W^-T scaled by the mesh
    (entry (o, i) = n_o (s W^-T)[o, i] / n_i, which must be an integer)."""
    mesh = _mesh3(k_mesh)
    W = np.asarray(operation.rotation_fractional, dtype=np.int64)
    G = np.rint(np.linalg.inv(W.astype(np.float64)).T).astype(np.int64)
    if not np.array_equal(W.T @ G, np.eye(3, dtype=np.int64)):
        raise ValueError("response symmetry fractional rotation has no exact integer reciprocal inverse")
    if operation.antiunitary:
        G = -G
    act = np.zeros((3, 3), dtype=np.int64)
    for o in range(3):
        for i in range(3):
            num = mesh[o] * G[o, i]
            if num % mesh[i] != 0:
                raise ValueError(f"response symmetry operation does not close k_mesh={mesh}: axis coefficient "
                                 f"({o + 1},{i + 1})={num}/{mesh[i]} is non-integral")
            act[o, i] = num // mesh[i]
    return act


def mesh_permutation(operation: SymmetryOperation, k_mesh) -> np.ndarray:
    """perm[i] = zero-based linear index (first axis fastest) of the image of mesh point i;
    raises unless the operation permutes the complete mesh."""
    mesh = _mesh3(k_mesh)
    act = integer_action(operation, mesh)
    n = mesh[0] * mesh[1] * mesh[2]
    idx = np.arange(n, dtype=np.int64)
    c = (idx % mesh[0], (idx // mesh[0]) % mesh[1], idx // (mesh[0] * mesh[1]))
    out = np.zeros(n, dtype=np.int64)
    stride = (1, mesh[0], mesh[0] * mesh[1])
    for o in range(3):
        v = act[o, 0] * c[0] + act[o, 1] * c[1] + act[o, 2] * c[2]
        out += np.mod(v, mesh[o]) * stride[o]
    if np.bincount(out, minlength=n).max(initial=0) != 1 or out.size != n:
        raise ValueError(f"response symmetry operation is not a permutation of k_mesh={mesh}")
    return out


@dataclasses.dataclass
class MeshOrbits:
    representatives: np.ndarray    # zero-based linear mesh indices, ascending
    multiplicities: np.ndarray
    full_kpoint_count: int


def is_closed_group(operations: Sequence[SymmetryOperation]) -> bool:
    """True when the (W, antiunitary) pairs are closed under composition and contain the identity."""
    keys = {(np.asarray(op.rotation_fractional, dtype=np.int64).tobytes(), bool(op.antiunitary)) for op in operations}
    if (np.eye(3, dtype=np.int64).tobytes(), False) not in keys:
        return False
    for a in operations:
        for b in operations:
            W = np.asarray(a.rotation_fractional, dtype=np.int64) @ np.asarray(b.rotation_fractional, dtype=np.int64)
            if (W.tobytes(), bool(a.antiunitary) != bool(b.antiunitary)) not in keys:
                return False
    return True


def kmesh_orbits(k_mesh, operations: Sequence[SymmetryOperation]) -> MeshOrbits:
    """Orbits of the mesh under the operations, each point labelled with the smallest index of
    its orbit.  A closed group needs one pass (the orbit of i is {perm_g[i]}); a generating set
    is handled by propagating labels along i -> perm_g[i] in both directions until nothing
    changes.  Every operation is checked to permute the complete mesh."""
    mesh = _mesh3(k_mesh)
    if min(mesh) <= 0:
        raise ValueError("response symmetry k mesh entries must be positive")
    n = mesh[0] * mesh[1] * mesh[2]
    label = np.arange(n, dtype=np.int64)
    if is_closed_group(operations):
        for op in operations:
            np.minimum(label, mesh_permutation(op, mesh), out=label)
    else:
        while True:
            before = label.copy()
            for op in operations:
                p = mesh_permutation(op, mesh)
                np.minimum(label, label[p], out=label)
                label[p] = np.minimum(label[p], label)
            if np.array_equal(label, before):
                break
    reps, counts = np.unique(label, return_counts=True)
    if counts.sum() != n:
        raise ValueError("response symmetry orbit multiplicities do not sum to the full k mesh")
    return MeshOrbits(reps.astype(np.int64), counts.astype(np.int64), n)


# -- reduced integral -----------------------------------------------------------------------------

def _component_index(axes: tuple, quantity: str, d: int) -> int:
    t = response_component_tuples(quantity, d)
    return t.index(tuple(axes))


def integrate_mesh_reduced(weighted_sum: Callable, task: _abi.TaskArrays, k_mesh,
                           operations: Sequence[SymmetryOperation], *, orbits: Optional[MeshOrbits] = None,
                           plans: Optional[dict] = None) -> np.ndarray:
    """Mesh average (1/N_full) sum_k value(k) of a shift / injection current task, evaluated on
    the representatives only: weighted_sum(mesh, indices, weights) returns
    sum_i weights[i] value(indices[i]) (e.g. ResponseEngine.mesh_weighted_sum), called once with
    weights multiplicity / N_full; each response block is then projected with X = B B^T X.
    Every component in a response's basis support must be among the task's components;
    components outside the support come out as zero (forbidden)."""
    mesh = _mesh3(k_mesh)
    plans = {} if plans is None else plans
    for kind, _ in task.responses:
        if kind not in _KIND_QUANTITY:
            raise ValueError("symmetry-reduced meshes apply to the shift and injection currents only")
        q = _KIND_QUANTITY[kind]
        if q not in plans:
            plans[q] = response_tensor_symmetry_plan(q, 3, operations)
    for (kind, _), comps in zip(task.responses, task.components):
        plan = plans[_KIND_QUANTITY[kind]]
        have = {_component_index(c, plan.quantity, 3) for c in comps}
        missing = [plan.labels[i] for i in plan.raw_component_indices if i not in have]
        if missing:
            raise ValueError(f"{plan.quantity}: the task must evaluate the symmetry support components {missing}")
    orb = kmesh_orbits(mesh, operations) if orbits is None else orbits
    weights = orb.multiplicities.astype(np.float64) / float(orb.full_kpoint_count)
    raw = np.asarray(weighted_sum(mesh, orb.representatives, weights))
    out = np.array(raw, dtype=np.complex128, copy=True)
    nw = task.photon_energies.size
    for (off, length), (kind, nc), comps in zip(task.block_offsets(), task.responses, task.components):
        plan = plans[_KIND_QUANTITY[kind]]
        block = raw[off:off + length].reshape(nc, nw)               # [component][energy]
        full = np.zeros((nw, len(plan.labels)), dtype=np.complex128)
        seen = set()
        for c, axes in enumerate(comps):
            j = _component_index(axes, plan.quantity, 3)
            if j not in seen:
                full[:, j] = block[c]
                seen.add(j)
        proj = project_response_symmetry(full, plan.basis, plan.imaginary_basis)
        for c, axes in enumerate(comps):
            out[off + c * nw: off + (c + 1) * nw] = proj[:, _component_index(axes, plan.quantity, 3)]
    return out


# -- groups and symmetric test models ---------------------------------------------------------------

def signed_permutation_group(predicate: Callable[[np.ndarray], bool] = lambda M: True) -> List[np.ndarray]:
    """Integer 3x3 signed permutation matrices (the cubic group O_h, 48) filtered by predicate."""
    out = []
    for perm in itertools.permutations(range(3)):
        for signs in itertools.product((1, -1), repeat=3):
            M = np.zeros((3, 3), dtype=np.int64)
            for r, c in enumerate(perm):
                M[r, c] = signs[r]
            if predicate(M):
                out.append(M)
    return out


def tetrahedral_group() -> List[np.ndarray]:
    """T_d (-43m), 24 operations: signed permutations whose nonzero entries multiply to +1."""
    return signed_permutation_group(lambda M: int(np.prod(M[M != 0])) == 1)


def symmetrize_model(model, operations: Sequence[SymmetryOperation]):
    """Group average of a model whose orbitals all sit at one site and transform trivially
    (s-like): H(R) <- avg_g H~_g(R) with H~_g(R) = H(W^-1 R) (conjugated for antiunitary g) and
    A_a(R) <- avg_g sum_b R_ab A~_b(W^-1 R); Wannier centres are averaged the same way.  The
    R-vector set must be closed under the operations (a cube |R_i| <= r_max is).  Used to
    build test models whose mesh sums obey the group exactly."""
    from .model import TightBindingModel
    rv = np.asarray(model.r_vectors, dtype=np.int64)
    lookup = {tuple(r): i for i, r in enumerate(rv.T)}
    H = np.zeros_like(model.hamiltonian_r)
    A = None if model.position_r is None else np.zeros_like(model.position_r)
    for op in operations:
        Winv = np.rint(np.linalg.inv(np.asarray(op.rotation_fractional, dtype=np.float64))).astype(np.int64)
        src = np.empty(rv.shape[1], dtype=np.int64)
        for i in range(rv.shape[1]):
            key = tuple(Winv @ rv[:, i])
            if key not in lookup:
                raise ValueError("R-vector set is not closed under the operations")
            src[i] = lookup[key]
        h = model.hamiltonian_r[:, :, src]
        H += np.conj(h) if op.antiunitary else h
        if A is not None:
            a = model.position_r[:, :, :, src]
            if op.antiunitary:
                a = np.conj(a)
            A += np.einsum("ab,mnbr->mnar", op.rotation_cartesian, a)
    H /= len(operations)
    if A is not None:
        A /= len(operations)
    return TightBindingModel(lattice=model.lattice.copy(), r_vectors=rv.copy(),
                             r_degeneracies=np.asarray(model.r_degeneracies).copy(), hamiltonian_r=H,
                             position_r=A, overlap_r=None)
