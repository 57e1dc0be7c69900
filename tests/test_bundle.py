"""Packed HDF5 operator bundles: the container reader, the manifest rules and the model route.

The known answers come from the reference's own fixtures, read as files where the reference tree
is present: ``examples/fixtures/synthetic_runtime`` holds a Packed bundle written by the reference
(HDF5 library output) whose Hamiltonian and position are, by its generator
(``generate_fixture.jl:85-112``), exactly the values of the paired ``synthetic_tb.dat``, and whose
spin operator is diag((-1)^orbital) on z and 0.1 x axis elsewhere in the home cell;
``test/fixtures/schema_compatibility/packed_6_3.h5`` is a legacy bundle that the current reader
must reject with MODEL_SCHEMA_UNSUPPORTED (``storage_schema_compatibility_unit.jl:36-48``).  The
other cases build bundles with this package's writer and plant one defect each.
"""
import glob
import os

import numpy as np
import pytest

from wanniernlqg_b200 import bundle, hdf5lite
from wanniernlqg_b200.model import read_wannier_tb, synthetic_orthogonal_model

# The reference's source tree, named by the environment (no machine path is assumed).
REFERENCE = os.environ.get("WNLQG_REFERENCE_TREE", "")
RUNTIME = os.path.join(REFERENCE, "examples", "fixtures", "synthetic_runtime") if REFERENCE else ""
needs_reference = pytest.mark.skipif(not (RUNTIME and os.path.isdir(RUNTIME)),
                                     reason="WNLQG_REFERENCE_TREE does not name the reference fixture tree")


def test_lookup3_published_values():
    # Bob Jenkins' lookup3.c self-test values for hashlittle.
    assert hdf5lite.lookup3(b"") == 0xDEADBEEF
    assert hdf5lite.lookup3(b"", 0xDEADBEEF) == 0xBD5B7DDE
    assert hdf5lite.lookup3(b"Four score and seven years ago") == 0x17770551
    assert hdf5lite.lookup3(b"Four score and seven years ago", 1) == 0xCD628161


@needs_reference
def test_reference_bundle_matches_its_paired_tb_file():
    path = os.path.join(RUNTIME, "synthetic_operators.h5")
    loaded = bundle.read_real_space_operator_bundle(path)
    manifest = loaded["manifest"]
    assert manifest.profile == "full"
    assert manifest.inventory == list(bundle.REAL_SPACE_OPERATOR_NAMES)
    assert manifest.num_orbitals == 4 and manifest.mp_grid == (2, 1, 1)
    assert len(manifest.entries) == 1 + 3 + 3 + 3 + 9 + 3 + 9 + 3 + 3 + 9 + 9
    assert manifest.entries[5].component_reference == "wanniernlqg.operator-component/1:2:2:0"
    np.testing.assert_array_equal(manifest.wannier_centers_cartesian,
                                  np.tile([0.25, 0.0, 0.0], (4, 1)))
    tb = read_wannier_tb(os.path.join(RUNTIME, "synthetic_tb.dat"))
    ops = loaded["operators"]
    assert np.array_equal(ops["hamiltonian"].data, tb.hamiltonian_r)
    assert np.array_equal(ops["position"].data, tb.position_r)
    assert np.array_equal(manifest.r_vectors, tb.r_vectors)
    assert np.array_equal(manifest.degeneracies, tb.r_degeneracies)
    assert np.array_equal(manifest.lattice, tb.lattice)
    spin = ops["spin"].data
    expect = np.zeros_like(spin)
    for axis in range(3):
        for orb in range(4):
            expect[orb, orb, axis, 0] = (-1.0) ** (orb + 1) if axis == 2 else 0.1 * (axis + 1)
    assert np.array_equal(spin, expect)
    model = bundle.model_from_operator_bundle(path)
    assert np.array_equal(model.hamiltonian_r, tb.hamiltonian_r)
    assert np.array_equal(model.position_r, tb.position_r)


@needs_reference
def test_reference_legacy_bundles_are_rejected():
    for rel in ("test/fixtures/schema_compatibility/packed_6_3.h5",
                "test/fixtures/legacy_model_1_3/synthetic_operators.h5"):
        path = os.path.join(REFERENCE, rel)
        for reader in (bundle.read_real_space_operator_bundle_manifest,
                       bundle.read_real_space_operator_bundle,
                       bundle.read_operator_bundle_payload,
                       lambda p: bundle.validate_packed_paired_tb(p, __file__)):
            with pytest.raises(ValueError, match="MODEL_SCHEMA_UNSUPPORTED"):
                reader(path)


@needs_reference
def test_reader_walks_every_reference_hdf5_file():
    """Every group, attribute and dataset of the reference's HDF5 fixtures (superblocks 0 and 2,
    symbol-table and dense groups, huge heap objects, chunked data) decodes with all checksums
    verified."""
    files = sorted(glob.glob(os.path.join(REFERENCE, "**", "*.h5"), recursive=True))
    assert files
    counts = {"groups": 0, "datasets": 0}

    def walk(g):
        g.attrs
        counts["groups"] += 1
        for key in g.keys():
            node = g[key]
            if isinstance(node, hdf5lite.Group):
                walk(node)
            else:
                node.attrs
                node.read()
                counts["datasets"] += 1

    for path in files:
        with hdf5lite.open_file(path) as f:
            walk(f)
    assert counts["datasets"] > 100


@needs_reference
def test_reference_bundle_round_trips_through_the_writer(tmp_path):
    path = os.path.join(RUNTIME, "synthetic_operators.h5")
    original = bundle.read_real_space_operator_bundle(path)
    m = original["manifest"]
    geometry = {k: getattr(m, k) for k in (
        "wannier_center_policy", "real_space_replica_policy", "minimum_distance_materialized",
        "mp_grid", "wigner_seitz_tolerance", "wigner_seitz_search_size",
        "replica_mapping_reference")}
    out = bundle.write_real_space_operator_bundle(
        str(tmp_path / "copy.h5"), original["lattice"], original["degeneracies"],
        original["operators"], geometry=geometry, definitions=m.mathematical_definitions)
    again = bundle.read_real_space_operator_bundle(out)
    for name, op in original["operators"].items():
        assert np.array_equal(again["operators"][name].data, op.data)
    assert ([e.component_reference for e in again["manifest"].entries]
            == [e.component_reference for e in m.entries])
    assert again["manifest"].mathematical_definitions == m.mathematical_definitions


def _model():
    return synthetic_orthogonal_model(6, 1, seed=11, full_position=True)


def test_paired_tb_validation_has_no_source_in_the_current_format(tmp_path):
    """validate_packed_paired_tb: a current-format bundle carries no paired _tb.dat source."""
    from wanniernlqg_b200.model import write_wannier_tb
    model = _model()
    path = bundle.write_model_operator_bundle(str(tmp_path / "m.h5"), model, mp_grid=(4, 4, 4))
    tb = str(tmp_path / "m_tb.dat")
    write_wannier_tb(model, tb)
    with pytest.raises(ValueError, match="MissingPairedTBSource"):
        bundle.validate_packed_paired_tb(path, tb)
    with pytest.raises(ValueError, match="MissingPairedTBSource"):
        bundle.validate_packed_paired_tb(path, str(tmp_path / "absent_tb.dat"))
    with pytest.raises(ValueError, match="operator bundle does not exist"):
        bundle.validate_packed_paired_tb(str(tmp_path / "absent.h5"), tb)


def test_model_round_trip(tmp_path):
    model = _model()
    path = bundle.write_model_operator_bundle(str(tmp_path / "m.h5"), model, mp_grid=(4, 4, 4))
    manifest = bundle.read_real_space_operator_bundle_manifest(path)
    assert manifest.profile == "hamiltonian_position"
    assert manifest.num_orbitals == 6 and manifest.mp_grid == (4, 4, 4)
    back = bundle.model_from_operator_bundle(path)
    assert np.array_equal(back.hamiltonian_r, model.hamiltonian_r)
    assert np.array_equal(back.position_r, model.position_r)
    assert np.array_equal(back.r_vectors, model.r_vectors)
    assert np.array_equal(back.r_degeneracies, model.r_degeneracies)
    assert np.array_equal(back.lattice, model.lattice)
    _, comps = bundle.read_operator_bundle_components(path, {"position": [(2, 0)]})
    assert np.array_equal(comps["position"][(2, 0)], model.position_r[:, :, 1, :])
    with pytest.raises(ValueError, match="absent from bundle profile"):
        bundle.read_operator_bundle_components(path, {"spin": [(1, 0)]})
    with pytest.raises(ValueError, match="refusing to overwrite"):
        bundle.write_model_operator_bundle(path, model)
    with pytest.raises(ValueError, match="publication receipts"):
        bundle.read_real_space_operator_bundle(path, receipt_path="x")
    with pytest.raises(ValueError, match="does not exist"):
        bundle.read_real_space_operator_bundle(str(tmp_path / "missing.h5"))


def _tree():
    model = _model()
    return bundle.bundle_tree(model.lattice, model.r_degeneracies, bundle.model_operators(model),
                              geometry=dict(bundle.DEFAULT_GEOMETRY))


def _index(tree, key):
    return tree.children["index"].children[key]


def _bad(tmp_path, mutate, reader=bundle.read_real_space_operator_bundle_manifest):
    tree = _tree()
    mutate(tree)
    path = str(tmp_path / "bad.h5")
    hdf5lite.write_file(path, tree)
    return lambda: reader(path)


def _set_index(key, fn):
    def mutate(tree):
        tree.children["index"].children[key] = fn(_index(tree, key).copy())
    return mutate


def _payload_nan(tree):
    p = tree.children["payload"].children["complex128"].copy()
    p[3] = np.nan
    tree.children["payload"].children["complex128"] = p


def _append_payload(tree):
    p = tree.children["payload"].children["complex128"]
    tree.children["payload"].children["complex128"] = np.concatenate([p, [0j]])


def _drop_position(tree):
    keep = _index(tree, "operator_kind_id") == 0
    for key in ("operator_kind_id", "component_rank", "component_indices", "offset_elements",
                "length_elements", "logical_shape"):
        tree.children["index"].children[key] = _index(tree, key)[keep]
    n = int(_index(tree, "length_elements")[0])
    p = tree.children["payload"].children["complex128"]
    tree.children["payload"].children["complex128"] = p[:n]


def _attr(path, key, value):
    def mutate(tree):
        node = tree
        for part in path:
            node = node.children[part]
        node.attrs[key] = value
    return mutate


def _duplicate_r(tree):
    r = tree.children["model"].children["r_vectors"].copy()
    r[1] = r[0]
    tree.children["model"].children["r_vectors"] = r


@pytest.mark.parametrize("mutate,message", [
    (_attr((), "schema_version", "1.1"), "MODEL_SCHEMA_UNSUPPORTED"),
    (_attr((), "basis_metric", "overlap"), "unsupported mathematical definition: basis_metric"),
    (_attr((), "fourier_convention", "X(k)=sum_R"), "definition: fourier_convention"),
    (_set_index("offset_elements", lambda a: a + np.uint64(1)), "invalid component shape or extent"),
    (_set_index("logical_shape", lambda a: a[:, ::-1] + np.uint64(1)), "invalid component shape"),
    (_set_index("operator_kind_id", lambda a: np.where(a == 1, 42, a).astype(np.uint8)),
     "unknown operator kind"),
    (_set_index("component_indices", lambda a: a[::-1].copy()),
     "missing or inconsistent Cartesian components"),
    (_set_index("component_rank", lambda a: a[:-1]), "malformed component index"),
    (_append_payload, "unindexed payload elements"),
    (_drop_position, "model lacks H or position"),
    (_duplicate_r, "duplicate R vectors"),
    (_attr(("operators", "position"), "units", "Bohr"), "operator unit definition mismatch"),
    (_attr(("geometry",), "real_space_replica_policy", "minimum_distance"),
     "invalid replica semantics"),
    (_attr(("geometry",), "wannier_center_policy", "average"), "invalid Wannier center policy"),
    (_attr(("geometry",), "wigner_seitz_tolerance", -1.0), "invalid replica controls"),
    (_attr(("definitions",), "position.derivative_frame", "centered"),
     "UNSUPPORTED_MODEL_DERIVATIVE_FRAME"),
])
def test_manifest_rejects_planted_defects(tmp_path, mutate, message):
    with pytest.raises(ValueError, match=message):
        _bad(tmp_path, mutate)()


def test_non_finite_payload_is_rejected_on_load(tmp_path):
    manifest_read = _bad(tmp_path, _payload_nan)
    manifest_read()  # the manifest does not scan the payload
    with pytest.raises(ValueError, match="non-finite"):
        bundle.read_real_space_operator_bundle(str(tmp_path / "bad.h5"))
    with pytest.raises(ValueError, match="non-finite"):
        bundle.model_from_operator_bundle(str(tmp_path / "bad.h5"))


def test_writer_validates_operators(tmp_path):
    model = _model()
    ops = bundle.model_operators(model)
    bad = dict(ops)
    data = ops["hamiltonian"].data.copy()
    data[0, 0, 0] = np.inf
    bad["hamiltonian"] = bundle.RealSpaceOperator(ops["hamiltonian"].spec, ops["hamiltonian"].r_vectors, data)
    with pytest.raises(ValueError, match="nonfinite"):
        bundle.bundle_tree(model.lattice, model.r_degeneracies, bad, geometry=bundle.DEFAULT_GEOMETRY)
    with pytest.raises(ValueError, match="requires Hamiltonian and position"):
        bundle.bundle_tree(model.lattice, model.r_degeneracies, {"hamiltonian": ops["hamiltonian"]},
                           geometry=bundle.DEFAULT_GEOMETRY)
    with pytest.raises(ValueError, match="nonsingular"):
        bundle.bundle_tree(np.zeros((3, 3)), model.r_degeneracies, ops, geometry=bundle.DEFAULT_GEOMETRY)


def test_damaged_metadata_fails_its_checksum(tmp_path):
    path = bundle.write_model_operator_bundle(str(tmp_path / "m.h5"), _model())
    raw = bytearray(open(path, "rb").read())
    at = raw.index(b"OHDR", 64) + 12  # inside the first object header's messages
    raw[at] ^= 0xFF
    damaged = str(tmp_path / "damaged.h5")
    open(damaged, "wb").write(bytes(raw))
    with pytest.raises(ValueError):
        bundle.read_real_space_operator_bundle(damaged)
    with open(str(tmp_path / "not.h5"), "wb") as fh:
        fh.write(b"plain text, not HDF5\n")
    with pytest.raises(hdf5lite.HDF5FormatError, match="not an HDF5 file"):
        hdf5lite.open_file(str(tmp_path / "not.h5"))
