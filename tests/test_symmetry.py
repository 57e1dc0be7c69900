"""Symmetry-reduced meshes: the reference's known answers for orbits, tensor actions, projectors
and compact plans (test/response_symmetry_unit.jl:77-440), and the reduction itself checked on
group-averaged models with the CPU oracle: the full-mesh sum equals the representatives'
multiplicity-weighted sum projected with B B^T."""
import itertools

import numpy as np
import pytest

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import synthetic_orthogonal_model
from wanniernlqg_b200.symmetry import (SymmetryOperation, integrate_mesh_reduced, kmesh_orbits, mesh_permutation,
                                       response_component_labels, response_symmetry_action_matrix,
                                       response_symmetry_basis, response_symmetry_projector,
                                       response_symmetry_relations, response_tensor_symmetry_plan,
                                       symmetrize_model, tetrahedral_group, is_closed_group)

I3 = np.eye(3, dtype=np.int64)
MX = np.diag([-1, 1, 1])
QUANTITIES = ("shift_current", "injection_current", "shift_spin_current", "injection_spin_current")


def op(W, antiunitary=False):
    return SymmetryOperation.from_fractional(W, antiunitary=antiunitary)


def grey_mirror_group():
    return [op(I3), op(MX), op(I3, True), op(MX, True)]


@pytest.mark.parametrize("quantity,sign", [("shift_current", 1.0), ("injection_current", -1.0),
                                           ("shift_spin_current", -1.0), ("injection_spin_current", 1.0)])
def test_antiunitary_final_tensor_rules(quantity, sign):
    labels = response_component_labels(quantity, 2)
    ix = {l: i for i, l in enumerate(labels)}
    M = response_symmetry_action_matrix(quantity, 2, np.eye(3), True)
    if quantity.endswith("spin_current"):
        assert M[ix["xzxy"], ix["xzyx"]] == sign
    else:
        assert M[ix["xxy"], ix["xyx"]] == sign
    assert np.array_equal(M @ M.T, np.eye(M.shape[0]))


def test_mirror_action_on_charge_and_spin_components():
    charge = response_symmetry_action_matrix("shift_current", 2, MX.astype(float), False)
    spin = response_symmetry_action_matrix("shift_spin_current", 2, MX.astype(float), False)
    cl = response_component_labels("shift_current", 2)
    sl = response_component_labels("shift_spin_current", 2)
    assert charge[cl.index("xyy"), cl.index("xyy")] == -1.0
    assert spin[sl.index("xyyy"), sl.index("xyyy")] == 1.0


def test_rotation_out_of_active_subspace_rejected():
    with pytest.raises(ValueError):
        response_symmetry_action_matrix("shift_current", 2, np.array([[0., 0, 1], [0, 1, 0], [1, 0, 0]]), False)


@pytest.mark.parametrize("quantity", QUANTITIES)
def test_projector_basis_and_relations(quantity):
    ops = grey_mirror_group()
    P = response_symmetry_projector(quantity, 2, ops)
    assert np.max(np.abs(P @ P - P)) < 1e-13
    B1 = response_symmetry_basis(P)
    B2 = response_symmetry_basis(P.copy())
    assert np.array_equal(B1, B2)
    assert np.max(np.abs(B1.T @ B1 - np.eye(B1.shape[1]))) < 1e-13
    assert np.max(np.abs(B1 @ B1.T - P)) < 1e-13
    rel = response_symmetry_relations(quantity, 2, P)
    assert rel.constraint_matrix.shape == P.shape
    assert rel.forbidden


def test_shift_current_relations_under_grey_mirror():
    P = response_symmetry_projector("shift_current", 2, grey_mirror_group())
    rel = response_symmetry_relations("shift_current", 2, P)
    assert set(rel.forbidden) == {"xxx", "xyy", "yxy", "yyx"}
    assert ("xxy", "xyx") in rel.equal


def test_compact_and_dense_component_plans():
    ops = grey_mirror_group()
    compact = response_tensor_symmetry_plan("shift_current", 2, ops)
    assert compact.accumulation_path == "selected_component_kernel_compact_coefficients"
    assert compact.raw_component_indices == compact.basis_support_indices
    assert len(compact.raw_component_indices) == 4
    assert compact.basis.shape[1] == 3
    dense = response_tensor_symmetry_plan("shift_current", 2, ops, force_dense=True)
    assert dense.accumulation_path == "dense_kernel_compact_coefficients"
    assert dense.raw_component_indices == list(range(len(dense.labels)))
    assert np.array_equal(dense.projector, compact.projector)
    assert np.array_equal(dense.basis, compact.basis)
    ident = response_tensor_symmetry_plan("shift_current", 2, [op(I3)])
    assert ident.accumulation_path == "dense_kernel_compact_coefficients"
    assert len(ident.raw_component_indices) == 8


def test_gamma_centred_integer_orbits():
    ops = grey_mirror_group()
    odd = kmesh_orbits((3, 3), ops)
    even = kmesh_orbits((4, 4), ops)
    assert len(odd.representatives) == 4 and sorted(odd.multiplicities.tolist()) == [1, 2, 2, 4]
    assert odd.multiplicities.sum() == 9
    assert len(even.representatives) == 9 and even.multiplicities.sum() == 16
    inv = kmesh_orbits((3, 3, 3), [op(I3), op(-I3)])
    assert len(inv.representatives) == 14 and inv.multiplicities.sum() == 27
    r90 = np.array([[0, -1, 0], [1, 0, 0], [0, 0, 1]])
    rots = [op(np.linalg.matrix_power(r90, p)) for p in range(4)]
    square = kmesh_orbits((5, 5), rots)
    assert square.multiplicities.sum() == 25 and len(square.representatives) == 7
    with pytest.raises(ValueError):
        kmesh_orbits((2, 3), rots)


def _partition(perms, n):
    """Orbits by breadth-first search over the permutations (independent of kmesh_orbits)."""
    seen = np.zeros(n, dtype=bool)
    parts = set()
    for s in range(n):
        if seen[s]:
            continue
        stack, orbit = [s], []
        seen[s] = True
        while stack:
            x = stack.pop()
            orbit.append(x)
            for p in perms:
                y = int(p[x])
                if not seen[y]:
                    seen[y] = True
                    stack.append(y)
        parts.add(tuple(sorted(orbit)))
    return parts


@pytest.mark.parametrize("mesh,gens", [((5, 5, 1), "grey"), ((4, 6, 1), "grey"), ((3, 4, 5), "inversion"),
                                       ((6, 6, 6), "td"), ((8, 8, 8), "td-generators")])
def test_orbits_match_breadth_first_partition_and_generators(mesh, gens):
    if gens == "grey":
        ops = grey_mirror_group()
    elif gens == "inversion":
        ops = [op(I3), op(-I3)]
    else:
        ops = [op(W) for W in tetrahedral_group()]
    n = int(np.prod(mesh))
    perms = [mesh_permutation(o, mesh) for o in ops]
    expected = _partition(perms, n)
    if gens == "td-generators":
        # S4 about z and the threefold axis generate T_d; not a closed set, so labels propagate.
        s4 = np.array([[0, 1, 0], [-1, 0, 0], [0, 0, -1]])
        c3 = np.array([[0, 0, 1], [1, 0, 0], [0, 1, 0]])
        ops = [op(s4), op(c3)]
        assert not is_closed_group(ops)
    orb = kmesh_orbits(mesh, ops)
    got = {}
    # rebuild the partition from the representatives of every point
    label = np.arange(n)
    for p in perms:
        label = np.minimum(label, p)
    for i in range(n):
        got.setdefault(int(label[i]), []).append(i)
    assert set(tuple(v) for v in got.values()) == expected
    assert np.array_equal(orb.representatives, np.array(sorted(got)))
    assert np.array_equal(orb.multiplicities, np.array([len(got[r]) for r in sorted(got)]))


def test_ibz_coefficients_equal_projected_full_zone():
    """Covariant synthetic data on a 5 x 5 mesh: the representatives' weighted coefficients
    reconstruct the projected full-zone sum."""
    ops = grey_mirror_group()
    orb = kmesh_orbits((5, 5), ops)
    perms = [mesh_permutation(o, (5, 5)) for o in ops]
    acts = [response_symmetry_action_matrix("shift_current", 2, o.rotation_cartesian, o.antiunitary) for o in ops]
    P = sum(acts) / len(acts)
    B = response_symmetry_basis(P)
    nc = P.shape[0]
    raw = np.array([[np.sin(0.37 * (pt + 1) + 0.19 * (c + 1)) for pt in range(25)] for c in range(nc)])
    cov = np.zeros_like(raw)
    for M, p in zip(acts, perms):
        inv = np.argsort(p)
        cov += M @ raw[:, inv]
    cov /= len(acts)
    projected_full = B @ B.T @ cov.sum(axis=1) / 25
    coef = np.zeros(B.shape[1])
    for r, m in zip(orb.representatives, orb.multiplicities):
        coef += m * (B.T @ cov[:, r]) / 25
    assert np.max(np.abs(B @ coef - projected_full)) < 1e-13


ALL27 = ["".join(c) for c in itertools.product("xyz", repeat=3)]


def _oracle_weighted_sum(oracle_mod, model, task):
    def ws(mesh, idx, w):
        n1, n2, n3 = mesh
        idx = np.asarray(idx)
        k = np.stack([idx % n1 / n1, (idx // n1) % n2 / n2, idx // (n1 * n2) / n3], axis=1)
        return (oracle_mod.point_values(model, task, k) * np.asarray(w)[:, None]).sum(axis=0)
    return ws


@pytest.mark.parametrize("group,mesh", [("td", (6, 6, 6)), ("grey_mm2", (6, 6, 4)), ("c2v", (5, 4, 3))])
def test_reduced_mesh_equals_full_mesh_on_symmetric_model(oracle_mod, group, mesh):
    if group == "td":
        ops = [op(W) for W in tetrahedral_group()]
    else:
        mm2 = [np.diag(d) for d in ([1, 1, 1], [-1, -1, 1], [-1, 1, 1], [1, -1, 1])]
        ops = [op(W, a) for W in mm2 for a in ((False, True) if group == "grey_mm2" else (False,))]
    model = symmetrize_model(synthetic_orthogonal_model(4, 1, seed=5, full_position=True), ops)
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ALL27), (_abi.INJECTION_CURRENT, ALL27)],
                           broadening_type=_abi.GAUSSIAN, broadening=0.05, photon_energies=np.linspace(0.1, 2.5, 12))
    full = oracle_mod.integrate_mesh(model, task, mesh)
    red = integrate_mesh_reduced(_oracle_weighted_sum(oracle_mod, model, task), task, mesh, ops)
    for f, r in zip(task.split(full), task.split(red)):
        assert np.abs(f).max() > 0
        assert np.max(np.abs(f - r)) < 1e-12 * np.abs(f).max()


def test_reduced_mesh_needs_support_components_and_current_kinds(oracle_mod):
    ops = [op(W) for W in tetrahedral_group()]
    model = symmetrize_model(synthetic_orthogonal_model(4, 1, seed=5, full_position=True), ops)
    ws = _oracle_weighted_sum(oracle_mod, model, None)
    with pytest.raises(ValueError, match="support"):
        task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, ["xyz"])], photon_energies=[0.5])
        integrate_mesh_reduced(ws, task, (4, 4, 4), ops)
    with pytest.raises(ValueError, match="shift and injection"):
        task = _abi.TaskArrays([(_abi.BERRY_CURVATURE, ["xy"])])
        integrate_mesh_reduced(ws, task, (4, 4, 4), ops)
    # A forbidden component next to the support comes out exactly zero.
    support = ["xyz", "xzy", "yxz", "yzx", "zxy", "zyx"]
    task = _abi.TaskArrays([(_abi.SHIFT_CURRENT, support + ["xxx"])], broadening_type=_abi.GAUSSIAN,
                           broadening=0.05, photon_energies=[0.5, 1.0])
    red = integrate_mesh_reduced(_oracle_weighted_sum(oracle_mod, model, task), task, (4, 4, 4), ops)
    sc = task.split(red)[0]
    assert np.all(sc[:, -1] == 0)
    assert np.max(np.abs(sc[:, :6] - sc[:, :1])) < 1e-12 * np.abs(sc).max()


def test_symmetrized_model_is_invariant():
    ops = [op(W) for W in tetrahedral_group()]
    model = symmetrize_model(synthetic_orthogonal_model(4, 1, seed=5, full_position=True), ops)
    again = symmetrize_model(model, ops)
    assert np.max(np.abs(again.hamiltonian_r - model.hamiltonian_r)) < 1e-15
    assert np.max(np.abs(again.position_r - model.position_r)) < 1e-15
