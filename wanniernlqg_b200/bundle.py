"""Packed HDF5 real-space operator bundles: manifest, payload, components, operators, model.

Restates the reader side of the reference's current mathematical model format (schema
``wanniernlqg.real-space-operators`` version 3.0): ``IO/RealSpaceOperatorBundles.jl:1-60, 656-707``
(public entry points, index rows, component references) and
``ext/WannierNLQGOperatorBundleExt/CurrentModelFormat.jl:288-500`` (``_manifest_from_handle``:
the validation of definitions, model arrays, index extents, operator groups and geometry), with
the payload readers of ``WannierNLQGOperatorBundleExt.jl:3928-4187``.  The container is read by
``hdf5lite`` (no HDF5 library is needed).

Layout of a bundle: one contiguous ``payload/complex128`` vector; the ``index`` group lists, per
Cartesian component of every operator, its kind id, Cartesian rank and indices, element offset and
length in the payload and its logical shape (nw, nw, NR); each component is the column-major
(nw, nw, NR) block of that operator.  Julia arrays are written column-major, so every HDF5 array
read here is transposed back to the writer's logical shape.

Errors are ``ValueError`` with the reference's ``ArgumentError`` messages.
"""
from __future__ import annotations

import dataclasses
import json
import os
from typing import Dict, List, Optional, Tuple

import numpy as np

from . import hdf5lite
from .model import TightBindingModel

OPERATOR_BUNDLE_SCHEMA = "wanniernlqg.real-space-operators"
OPERATOR_BUNDLE_SCHEMA_VERSION = "3.0"
LOGICAL_CONVENTION = "R-last"
BLOCH_PHASE_CONVENTION = "R_only"
FOURIER_CONVENTION = "X(k)=sum_R exp(i*2*pi*k.R)*X_stored(R)/degeneracy(R)"

# RealSpaceOperatorKind (Core/RealSpaceOperators.jl:2-43): the kind id is the position here.
REAL_SPACE_OPERATOR_NAMES = (
    "hamiltonian",
    "position",
    "hamiltonian_weighted_connection",
    "hamiltonian_weighted_axial_derivative_overlap",
    "derivative_overlap_tensor",
    "axial_derivative_overlap",
    "symmetric_derivative_overlap",
    "spin",
    "spin_times_hamiltonian",
    "spin_times_position",
    "spin_times_hamiltonian_position",
)

OPERATOR_PROFILE_INVENTORIES = {
    "hamiltonian_position": ("hamiltonian", "position"),
    "hamiltonian_position_spin": ("hamiltonian", "position", "spin"),
    "derivative": REAL_SPACE_OPERATOR_NAMES[:7],
    "full": REAL_SPACE_OPERATOR_NAMES,
}


def _unit_contract(name: str) -> str:
    """``_unit_contract`` (WannierNLQGOperatorBundleExt.jl:1597-1602)."""
    return {"hamiltonian": "eV", "position": "Angstrom",
            "spin": "dimensionless Pauli-spin convention"}.get(
        name, "WannierNLQG native operator convention")


def _component_tuples(rank: int) -> List[Tuple[int, int]]:
    """Stored component order of a Cartesian rank (WannierNLQGOperatorBundleExt.jl:495-500)."""
    if rank == 0:
        return [(0, 0)]
    if rank == 1:
        return [(a, 0) for a in (1, 2, 3)]
    if rank == 2:
        return [(a, b) for a in (1, 2, 3) for b in (1, 2, 3)]
    raise ValueError("Packed HDF5 supports Cartesian ranks zero, one, and two")


def operator_component_reference(kind: int, indices) -> str:
    """``operator_component_reference`` (IO/RealSpaceOperatorBundles.jl:39-50)."""
    if len(indices) != 2:
        raise ValueError("InvalidOperatorComponentReference")
    return "wanniernlqg.operator-component/1:%d:%d:%d" % (int(kind), int(indices[0]),
                                                          int(indices[1]))


@dataclasses.dataclass(frozen=True)
class OperatorBundleIndexEntry:
    """One zero-based row of the packed component index (RealSpaceOperatorBundles.jl:24-32)."""
    kind: int
    component_rank: int
    component_indices: Tuple[int, int]
    offset_elements: int
    length_elements: int
    logical_shape: Tuple[int, int, int]
    component_reference: str

    @property
    def operator(self) -> str:
        return REAL_SPACE_OPERATOR_NAMES[self.kind]


@dataclasses.dataclass(frozen=True)
class RealSpaceOperatorSymmetrySpec:
    """Cartesian rank and parities of one operator (Core/RealSpaceOperators.jl:57-79)."""
    kind: int
    cartesian_rank: int
    inversion_parity: int
    time_reversal_parity: int
    rotate_cartesian: bool = True

    def __post_init__(self):
        if self.cartesian_rank < 0:
            raise ValueError("cartesian_rank must be nonnegative")
        if self.inversion_parity not in (-1, 1):
            raise ValueError("inversion_parity must be +1 or -1")
        if self.time_reversal_parity not in (-1, 1):
            raise ValueError("time_reversal_parity must be +1 or -1")


@dataclasses.dataclass
class RealSpaceOperator:
    """``RealSpaceOperator``: data of shape (nw, nw, 3 x rank, NR), column-major."""
    spec: RealSpaceOperatorSymmetrySpec
    r_vectors: np.ndarray
    data: np.ndarray


@dataclasses.dataclass
class OperatorBundleManifest:
    """Validated metadata needed before loading the payload (RealSpaceOperatorBundles.jl:52-67)."""
    path: str
    profile: str
    inventory: List[str]
    num_orbitals: int
    lattice: np.ndarray                 # (3, 3), rows are lattice vectors
    r_vectors: np.ndarray               # (3, NR) int64
    degeneracies: np.ndarray            # (NR,) int64
    entries: List[OperatorBundleIndexEntry]
    payload_length: int
    schema_version: str
    wannier_centers_cartesian: np.ndarray   # (nw, 3)
    wannier_centers_fractional: np.ndarray  # (nw, 3)
    wannier_center_policy: str
    real_space_replica_policy: str
    minimum_distance_materialized: bool
    mp_grid: Tuple[int, int, int]
    wigner_seitz_tolerance: float
    wigner_seitz_search_size: int
    replica_mapping_reference: str
    mathematical_definitions: dict
    specs: Dict[str, RealSpaceOperatorSymmetrySpec]


def _required_attribute(node, name):
    if name not in node.attrs:
        raise ValueError("operator bundle is missing attribute %s" % name)
    return node.attrs[name]


def _julia_array(dataset) -> np.ndarray:
    """A dataset in the column-major writer's logical shape."""
    value = np.asarray(dataset.read())
    return value.T if value.ndim > 1 else value


def _open(filename: str, receipt_path=None) -> hdf5lite.File:
    """Schema gate of ``_with_operator_bundle_publication`` (WannierNLQGOperatorBundleExt.jl:3928-3945)."""
    if receipt_path is not None:
        raise ValueError("current mathematical model format does not use publication receipts")
    path = os.path.abspath(filename)
    if not os.path.isfile(path):
        raise ValueError("operator bundle does not exist: %s" % path)
    h = hdf5lite.open_file(os.path.realpath(path))
    try:
        if not (str(_required_attribute(h, "schema")) == OPERATOR_BUNDLE_SCHEMA
                and str(_required_attribute(h, "schema_version")) == OPERATOR_BUNDLE_SCHEMA_VERSION):
            raise ValueError("MODEL_SCHEMA_UNSUPPORTED: expected %s version %s"
                             % (OPERATOR_BUNDLE_SCHEMA, OPERATOR_BUNDLE_SCHEMA_VERSION))
    except BaseException:
        h.close()
        raise
    return h


def _cartesian_to_fractional(center, lattice):
    """``real_space_cartesian_to_fractional`` (Core/Coordinates.jl:7-12): lattice^T \\ r."""
    return np.linalg.solve(lattice.T, center)


def _manifest_from_handle(path: str, h) -> OperatorBundleManifest:
    """``_manifest_from_handle`` for the current format (CurrentModelFormat.jl:288-500)."""
    if str(_required_attribute(h, "schema")) != OPERATOR_BUNDLE_SCHEMA:
        raise ValueError("unsupported model schema")
    version = str(_required_attribute(h, "schema_version"))
    if version != OPERATOR_BUNDLE_SCHEMA_VERSION:
        raise ValueError("unsupported mathematical model format; current format 3.0 is required")
    for key, value in (("basis_metric", "orthonormal"),
                       ("logical_convention", LOGICAL_CONVENTION),
                       ("bloch_phase_convention", BLOCH_PHASE_CONVENTION),
                       ("fourier_convention", FOURIER_CONVENTION),
                       ("wannier_center_convention", "Convention_II"),
                       ("energy_unit", "eV"),
                       ("length_unit", "Angstrom")):
        if str(_required_attribute(h, key)) != value:
            raise ValueError("unsupported mathematical definition: %s" % key)
    n = int(h["model/num_orbitals"].read())
    if n <= 0:
        raise ValueError("invalid orbital count")
    lattice = np.asarray(_julia_array(h["model/lattice"]), dtype=np.float64)
    if (lattice.shape != (3, 3) or not np.all(np.isfinite(lattice))
            or abs(np.linalg.det(lattice)) <= np.finfo(np.float64).eps):
        raise ValueError("invalid lattice")
    r = np.asarray(_julia_array(h["model/r_vectors"]), dtype=np.int64).reshape(3, -1) \
        if h["model/r_vectors"].size else np.zeros((3, 0), dtype=np.int64)
    weights = np.asarray(h["model/degeneracies"].read(), dtype=np.int64).reshape(-1)
    if not (r.shape[0] == 3 and r.shape[1] > 0 and weights.size == r.shape[1]
            and np.all(weights > 0)):
        raise ValueError("invalid support or degeneracies")
    if len({tuple(col) for col in r.T}) != r.shape[1]:
        raise ValueError("duplicate R vectors")
    nr = r.shape[1]
    centers = np.asarray(_julia_array(h["model/wannier_centers_cartesian"]), dtype=np.float64)
    if centers.shape != (n, 3) or not np.all(np.isfinite(centers)):
        raise ValueError("invalid centers")
    fractional = np.stack([_cartesian_to_fractional(centers[i], lattice) for i in range(n)])

    ids = np.asarray(h["index/operator_kind_id"].read(), dtype=np.int64).reshape(-1)
    ranks = np.asarray(h["index/component_rank"].read(), dtype=np.int64).reshape(-1)
    components = np.asarray(_julia_array(h["index/component_indices"]), dtype=np.int64)
    offsets = np.asarray(h["index/offset_elements"].read(), dtype=np.uint64).reshape(-1)
    lengths = np.asarray(h["index/length_elements"].read(), dtype=np.uint64).reshape(-1)
    shapes = np.asarray(_julia_array(h["index/logical_shape"]), dtype=np.uint64)
    count = ids.size
    if components.ndim == 1:
        components = components.reshape(2, -1)
    if shapes.ndim == 1:
        shapes = shapes.reshape(3, -1)
    if not (count > 0 and ranks.size == offsets.size == lengths.size == count
            and components.shape == (2, count) and shapes.shape == (3, count)):
        raise ValueError("malformed component index")
    payload_length = h["payload/complex128"].size
    cursor = 0
    entries = []
    for i in range(count):
        kind = int(ids[i])
        if not 0 <= kind < len(REAL_SPACE_OPERATOR_NAMES):
            raise ValueError("unknown operator kind")
        if not (int(offsets[i]) == cursor and int(lengths[i]) == n * n * nr
                and tuple(int(x) for x in shapes[:, i]) == (n, n, nr)):
            raise ValueError("invalid component shape or extent")
        if int(lengths[i]) > payload_length - cursor:
            raise ValueError("component exceeds payload")
        idx = (int(components[0, i]), int(components[1, i]))
        entries.append(OperatorBundleIndexEntry(kind, int(ranks[i]), idx, int(offsets[i]),
                                                int(lengths[i]), (n, n, nr),
                                                operator_component_reference(kind, idx)))
        cursor += int(lengths[i])
    if cursor != payload_length:
        raise ValueError("unindexed payload elements")
    kinds = {e.kind for e in entries}
    inventory = [name for k, name in enumerate(REAL_SPACE_OPERATOR_NAMES) if k in kinds]
    if "hamiltonian" not in inventory or "position" not in inventory:
        raise ValueError("model lacks H or position")
    specs = {}
    for name in inventory:
        group = h["operators/" + name]
        if str(_required_attribute(group, "units")) != _unit_contract(name):
            raise ValueError("operator unit definition mismatch")
        spec = _operator_spec_from_handle(h, name)
        specs[name] = spec
        selected = [e for e in entries if e.operator == name]
        if ([e.component_indices for e in selected] != _component_tuples(spec.cartesian_rank)
                or any(e.component_rank != spec.cartesian_rank for e in selected)):
            raise ValueError("missing or inconsistent Cartesian components")
    geometry = h["geometry"]
    policy = str(_required_attribute(geometry, "wannier_center_policy"))
    if policy not in ("symmetrize", "validate", "keep_input"):
        raise ValueError("invalid Wannier center policy")
    replica = str(_required_attribute(geometry, "real_space_replica_policy"))
    materialized = bool(_required_attribute(geometry, "minimum_distance_materialized"))
    if not (replica in ("input", "minimum_distance")
            and materialized == (replica == "minimum_distance")):
        raise ValueError("invalid replica semantics")
    if materialized and not np.all(weights == 1):
        raise ValueError("materialized replicas require unit degeneracies")
    grid = np.asarray(geometry["mp_grid"].read(), dtype=np.int64).reshape(-1)
    if grid.size != 3 or not np.all(grid > 0):
        raise ValueError("invalid grid")
    tolerance = float(_required_attribute(geometry, "wigner_seitz_tolerance"))
    search = int(_required_attribute(geometry, "wigner_seitz_search_size"))
    if not (np.isfinite(tolerance) and tolerance > 0 and search > 0):
        raise ValueError("invalid replica controls")
    if "replica_mapping_reference" not in geometry.attrs:
        raise ValueError("missing replica mapping reference")
    definitions = {}
    if "definitions" in h:
        for key, value in h["definitions"].attrs.items():
            definitions[key] = value
        for key in [k for k in definitions if k.endswith("__json")]:
            definitions[key[:-6]] = json.loads(definitions.pop(key))
    for key, value in definitions.items():
        if key.split(".")[-1] == "derivative_frame" and value != "uncentered_periodic_wannier":
            raise ValueError("UNSUPPORTED_MODEL_DERIVATIVE_FRAME: %s" % key)
    profile = "custom"
    for name in ("hamiltonian_position", "hamiltonian_position_spin", "derivative", "full"):
        if tuple(inventory) == OPERATOR_PROFILE_INVENTORIES[name]:
            profile = name
            break
    return OperatorBundleManifest(
        path=path, profile=profile, inventory=inventory, num_orbitals=n, lattice=lattice,
        r_vectors=np.asfortranarray(r), degeneracies=weights, entries=entries,
        payload_length=payload_length, schema_version=version,
        wannier_centers_cartesian=centers, wannier_centers_fractional=fractional,
        wannier_center_policy=policy, real_space_replica_policy=replica,
        minimum_distance_materialized=materialized, mp_grid=tuple(int(g) for g in grid),
        wigner_seitz_tolerance=tolerance, wigner_seitz_search_size=search,
        replica_mapping_reference=str(geometry.attrs["replica_mapping_reference"]),
        mathematical_definitions=definitions, specs=specs)


def _operator_spec_from_handle(h, name: str) -> RealSpaceOperatorSymmetrySpec:
    """``_operator_spec_from_handle`` (WannierNLQGOperatorBundleExt.jl:4121-4131)."""
    group = h["operators/" + name]
    return RealSpaceOperatorSymmetrySpec(
        REAL_SPACE_OPERATOR_NAMES.index(name),
        int(_required_attribute(group, "cartesian_rank")),
        int(_required_attribute(group, "inversion_parity")),
        int(_required_attribute(group, "time_reversal_parity")),
        bool(_required_attribute(group, "rotate_cartesian")))


def read_real_space_operator_bundle_manifest(filename: str, receipt_path=None
                                             ) -> OperatorBundleManifest:
    """Validated metadata and index extents, without reading the numerical payload."""
    with _open(filename, receipt_path) as h:
        return _manifest_from_handle(os.path.realpath(os.path.abspath(filename)), h)


def validate_packed_paired_tb(bundle_path: str, filename: str, receipt_path=None) -> None:
    """``validate_packed_paired_tb`` (IO/RealSpaceOperatorBundles.jl:709-720,
    WannierNLQGOperatorBundleExt.jl:4190-4218): the byte-for-byte check of a ``_tb.dat`` against
    the copy a bundle carries.  The current model format (3.0) stores no paired source (its
    manifest's ``paired_tb_source_bytes`` is nothing), so after the schema gate and the manifest
    rules the call reports ``MissingPairedTBSource``, as the reference's does; older formats
    stop at the schema gate (``MODEL_SCHEMA_UNSUPPORTED``)."""
    read_real_space_operator_bundle_manifest(bundle_path, receipt_path)
    # The reference reports the missing source before it opens `filename`.
    raise ValueError("MissingPairedTBSource")


def read_operator_bundle_payload(filename: str, receipt_path=None):
    """The validated manifest and the whole complex128 payload (a host copy)."""
    with _open(filename, receipt_path) as h:
        manifest = _manifest_from_handle(os.path.realpath(os.path.abspath(filename)), h)
        payload = np.array(h["payload/complex128"].read(), dtype=np.complex128, copy=True)
    return manifest, payload.reshape(-1)


def _component(payload, entry: OperatorBundleIndexEntry) -> np.ndarray:
    values = payload[entry.offset_elements:entry.offset_elements + entry.length_elements]
    return values.reshape(entry.logical_shape, order="F")


def read_operator_bundle_components(filename: str, requested_components: dict,
                                    receipt_path=None):
    """Only the requested components: ``{operator name: [(i, j), ...]}`` ->
    ``(manifest, {name: {(i, j): (nw, nw, NR) array}})`` (WannierNLQGOperatorBundleExt.jl:4021-4131)."""
    manifest, payload = read_operator_bundle_payload(filename, receipt_path)
    requested = {}
    for name, comps in requested_components.items():
        if name not in REAL_SPACE_OPERATOR_NAMES:
            raise ValueError("operator demand keys must use RealSpaceOperatorKind")
        if name not in manifest.inventory:
            raise ValueError("required operator %s is absent from bundle profile %s"
                             % (name, manifest.profile))
        requested[name] = {(int(c[0]), int(c[1])) for c in comps}
    selected = [e for e in manifest.entries
                if e.operator in requested and e.component_indices in requested[e.operator]]
    for name, comps in requested.items():
        if {e.component_indices for e in selected if e.operator == name} != comps:
            raise ValueError("required components for %s are absent from the bundle" % name)
    out: Dict[str, Dict[Tuple[int, int], np.ndarray]] = {}
    for e in selected:
        values = _component(payload, e)
        if not np.all(np.isfinite(values)):
            raise ValueError("component contains non-finite values for %s %s"
                             % (e.operator, e.component_indices))
        out.setdefault(e.operator, {})[e.component_indices] = values
    return manifest, out


def read_real_space_operator_bundle(filename: str, receipt_path=None) -> dict:
    """Every operator of the bundle, reconstructed (WannierNLQGOperatorBundleExt.jl:4141-4187).

    Returns ``{"manifest", "lattice", "degeneracies", "operators": {name: RealSpaceOperator}}``.
    """
    manifest, payload = read_operator_bundle_payload(filename, receipt_path)
    n, nr = manifest.num_orbitals, manifest.r_vectors.shape[1]
    operators = {}
    for name in manifest.inventory:
        spec = manifest.specs[name]
        dims = (n, n) + (3,) * spec.cartesian_rank + (nr,)
        data = np.zeros(dims, dtype=np.complex128, order="F")
        for e in manifest.entries:
            if e.operator != name:
                continue
            values = _component(payload, e)
            if spec.cartesian_rank == 0:
                data[:, :, :] = values
            elif spec.cartesian_rank == 1:
                data[:, :, e.component_indices[0] - 1, :] = values
            else:
                data[:, :, e.component_indices[0] - 1, e.component_indices[1] - 1, :] = values
        if not np.all(np.isfinite(data)):
            raise ValueError("operator %s contains non-finite values" % name)
        operators[name] = RealSpaceOperator(spec, manifest.r_vectors, data)
    return {"manifest": manifest, "lattice": manifest.lattice,
            "degeneracies": manifest.degeneracies, "operators": operators}


def model_from_operator_bundle(filename: str, receipt_path=None) -> TightBindingModel:
    """The tight-binding model the runtime builds from a bundle's Hamiltonian and position
    components (``_runtime_component_model``, Runtime/OperatorBundleSetup.jl:338-351).

    The Hamiltonian component is the payload block itself (column-major (nw, nw, NR), the
    layout ``wnlqg_b200_model_create`` takes); the three position components are interleaved
    into (nw, nw, 3, NR)."""
    manifest, comps = read_operator_bundle_components(
        filename, {"hamiltonian": [(0, 0)], "position": [(1, 0), (2, 0), (3, 0)]}, receipt_path)
    n, nr = manifest.num_orbitals, manifest.r_vectors.shape[1]
    position = np.zeros((n, n, 3, nr), dtype=np.complex128, order="F")
    for a in range(3):
        position[:, :, a, :] = comps["position"][(a + 1, 0)]
    return TightBindingModel(manifest.lattice, manifest.r_vectors, manifest.degeneracies,
                             comps["hamiltonian"][(0, 0)], position)


def _bundle_wannier_centers(operators, r_vectors, degeneracies):
    """Re diag A(R = 0) / degeneracy(R = 0) (``_bundle_wannier_centers`` with ``standard``,
    WannierNLQGOperatorBundleExt.jl:1569-1594)."""
    home = [i for i in range(r_vectors.shape[1]) if not np.any(r_vectors[:, i])]
    if len(home) != 1:
        raise ValueError("operator bundle requires exactly one R=(0,0,0) block")
    pos = operators["position"].data
    n = pos.shape[0]
    values = np.stack([pos[np.arange(n), np.arange(n), a, home[0]] for a in range(3)], axis=1)
    values = values / degeneracies[home[0]]
    if not np.all(np.isfinite(values)):
        raise ValueError("operator-bundle Wannier centers contain non-finite values")
    return np.ascontiguousarray(values.real)


def write_real_space_operator_bundle(filename: str, lattice, degeneracies, operators: dict, *,
                                     geometry: dict, definitions: Optional[dict] = None,
                                     overwrite: bool = False) -> str:
    """Write the current model format (``write_real_space_operator_bundle``,
    CurrentModelFormat.jl:97-270): ``operators`` maps operator names to ``RealSpaceOperator``;
    all share one R support; Hamiltonian and position are required.  The file is written to a
    temporary name in the destination directory and renamed into place."""
    path = os.path.abspath(filename)
    if os.path.exists(path) and not overwrite:
        raise ValueError("refusing to overwrite model: %s" % path)
    root = bundle_tree(lattice, degeneracies, operators, geometry=geometry,
                       definitions=definitions)
    directory = os.path.dirname(path) or "."
    os.makedirs(directory, exist_ok=True)
    temporary = os.path.join(directory, ".%s.%d.tmp" % (os.path.basename(path), os.getpid()))
    try:
        hdf5lite.write_file(temporary, root)
        os.replace(temporary, path)
    finally:
        if os.path.exists(temporary):
            os.remove(temporary)
    return path


def bundle_tree(lattice, degeneracies, operators: dict, *, geometry: dict,
                definitions: Optional[dict] = None) -> hdf5lite.WGroup:
    """The validated group tree ``write_real_space_operator_bundle`` writes."""
    lat = np.asarray(lattice, dtype=np.float64)
    if (lat.shape != (3, 3) or not np.all(np.isfinite(lat))
            or abs(np.linalg.det(lat)) <= np.finfo(np.float64).eps):
        raise ValueError("model lattice must be finite and nonsingular")
    unknown = [k for k in operators if k not in REAL_SPACE_OPERATOR_NAMES]
    if unknown:
        raise ValueError("unsupported real-space operator %s" % unknown[0])
    inventory = [k for k in REAL_SPACE_OPERATOR_NAMES if k in operators]
    if "hamiltonian" not in inventory or "position" not in inventory:
        raise ValueError("model requires Hamiltonian and position operators")
    r_vectors = np.asarray(operators["hamiltonian"].r_vectors, dtype=np.int64)
    for name in inventory:
        if not np.array_equal(np.asarray(operators[name].r_vectors), r_vectors):
            raise ValueError("operator bundle operators must share one R support")
    if not (r_vectors.ndim == 2 and r_vectors.shape[0] == 3 and r_vectors.shape[1] > 0):
        raise ValueError("invalid R support")
    if len({tuple(c) for c in r_vectors.T}) != r_vectors.shape[1]:
        raise ValueError("duplicate R vectors")
    weights = np.asarray(degeneracies, dtype=np.int64).reshape(-1)
    if weights.size != r_vectors.shape[1] or not np.all(weights > 0):
        raise ValueError("invalid degeneracies")
    n = operators["hamiltonian"].data.shape[0]
    nr = r_vectors.shape[1]
    centers = _bundle_wannier_centers(operators, r_vectors, weights)
    policy = str(geometry["wannier_center_policy"])
    if policy not in ("symmetrize", "validate", "keep_input"):
        raise ValueError("invalid Wannier center policy")
    replica = str(geometry["real_space_replica_policy"])
    materialized = bool(geometry["minimum_distance_materialized"])
    if materialized != (replica == "minimum_distance"):
        raise ValueError("replica materialization policy mismatch")
    if materialized and not np.all(weights == 1):
        raise ValueError("materialized replicas require unit degeneracies")
    grid = np.asarray(geometry["mp_grid"], dtype=np.int64).reshape(-1)
    if grid.size != 3 or not np.all(grid > 0):
        raise ValueError("invalid generation grid")
    entries, blocks, cursor = [], [], 0
    for name in inventory:
        op = operators[name]
        kind = REAL_SPACE_OPERATOR_NAMES.index(name)
        if op.spec.kind != kind:
            raise ValueError("operator kind mismatch")
        rank = op.spec.cartesian_rank
        if op.data.shape != (n, n) + (3,) * rank + (nr,):
            raise ValueError("operator dimensions disagree for %s" % name)
        for comp in _component_tuples(rank):
            if rank == 0:
                values = op.data[:, :, :]
            elif rank == 1:
                values = op.data[:, :, comp[0] - 1, :]
            else:
                values = op.data[:, :, comp[0] - 1, comp[1] - 1, :]
            values = np.asarray(values, dtype=np.complex128).reshape(-1, order="F")
            if not np.all(np.isfinite(values)):
                raise ValueError("operator contains nonfinite values")
            entries.append((kind, rank, comp, cursor, values.size))
            blocks.append(values)
            cursor += values.size
    root = hdf5lite.WGroup()
    for key, value in (("schema", OPERATOR_BUNDLE_SCHEMA),
                       ("schema_version", OPERATOR_BUNDLE_SCHEMA_VERSION),
                       ("basis_metric", "orthonormal"),
                       ("logical_convention", LOGICAL_CONVENTION),
                       ("bloch_phase_convention", BLOCH_PHASE_CONVENTION),
                       ("fourier_convention", FOURIER_CONVENTION),
                       ("wannier_center_convention", "Convention_II"),
                       ("energy_unit", "eV"), ("length_unit", "Angstrom")):
        root.attrs[key] = value
    # Column-major logical arrays are stored with reversed HDF5 dimensions: write transposes.
    m = root.create_group("model")
    m.children["num_orbitals"] = np.int64(n)
    m.children["lattice"] = np.ascontiguousarray(lat.T)
    m.children["r_vectors"] = np.ascontiguousarray(r_vectors.T)
    m.children["degeneracies"] = weights
    m.children["wannier_centers_cartesian"] = np.ascontiguousarray(centers.T)
    g = root.create_group("geometry")
    g.attrs["real_space_replica_policy"] = replica
    g.attrs["minimum_distance_materialized"] = materialized
    g.attrs["wannier_center_policy"] = policy
    g.attrs["wigner_seitz_tolerance"] = float(geometry["wigner_seitz_tolerance"])
    g.attrs["wigner_seitz_search_size"] = int(geometry["wigner_seitz_search_size"])
    g.attrs["replica_mapping_reference"] = str(geometry["replica_mapping_reference"])
    g.children["mp_grid"] = grid
    root.create_group("payload").children["complex128"] = np.concatenate(blocks)
    idx = root.create_group("index")
    idx.children["operator_kind_id"] = np.array([e[0] for e in entries], dtype=np.uint8)
    idx.children["component_rank"] = np.array([e[1] for e in entries], dtype=np.uint8)
    idx.children["component_indices"] = np.array([e[2] for e in entries], dtype=np.int8)
    idx.children["offset_elements"] = np.array([e[3] for e in entries], dtype=np.uint64)
    idx.children["length_elements"] = np.array([e[4] for e in entries], dtype=np.uint64)
    idx.children["logical_shape"] = np.array([(n, n, nr)] * len(entries), dtype=np.uint64)
    ops = root.create_group("operators")
    for name in inventory:
        spec = operators[name].spec
        a = ops.create_group(name).attrs
        a["cartesian_rank"] = int(spec.cartesian_rank)
        a["inversion_parity"] = int(spec.inversion_parity)
        a["time_reversal_parity"] = int(spec.time_reversal_parity)
        a["rotate_cartesian"] = bool(spec.rotate_cartesian)
        a["units"] = _unit_contract(name)
    d = root.create_group("definitions")
    for key, value in (definitions or {}).items():
        if isinstance(value, (dict, list, tuple)):
            d.attrs[key + "__json"] = json.dumps(value)
        elif isinstance(value, (str, bool, int, float)):
            d.attrs[key] = value
        else:
            raise ValueError("unsupported mathematical definition: %s" % key)
    return root


def model_operators(model: TightBindingModel) -> dict:
    """Hamiltonian and position operators of ``model`` (profile ``hamiltonian_position``)."""
    r = np.asarray(model.r_vectors, dtype=np.int64)
    return {"hamiltonian": RealSpaceOperator(RealSpaceOperatorSymmetrySpec(0, 0, 1, 1), r,
                                             model.hamiltonian_r),
            "position": RealSpaceOperator(RealSpaceOperatorSymmetrySpec(1, 1, 1, 1), r,
                                          model.real_position())}


DEFAULT_GEOMETRY = {"wannier_center_policy": "keep_input", "real_space_replica_policy": "input",
                    "minimum_distance_materialized": False, "mp_grid": [1, 1, 1],
                    "wigner_seitz_tolerance": 1e-5, "wigner_seitz_search_size": 3,
                    "replica_mapping_reference": "wanniernlqg_b200.model-export/1"}


def write_model_operator_bundle(filename: str, model: TightBindingModel, *,
                                mp_grid=(1, 1, 1), overwrite: bool = False) -> str:
    """A Hamiltonian + position bundle of ``model``: input replicas, centres kept as given."""
    geometry = dict(DEFAULT_GEOMETRY, mp_grid=list(mp_grid))
    return write_real_space_operator_bundle(filename, model.lattice, model.r_degeneracies,
                                            model_operators(model), geometry=geometry,
                                            overwrite=overwrite)
