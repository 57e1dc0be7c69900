"""ctypes mirror of the C ABI declared in include/wnlqg_b200.h.

Only structure layouts, enums and array marshalling live here; loading the CUDA library is
the job of :mod:`wanniernlqg_b200._lib`.
"""
from __future__ import annotations

import ctypes
from typing import Sequence

import numpy as np

from .model import TightBindingModel

WNLQG_OK = 0
STATUS_NAMES = {
    0: "OK", 1: "INVALID_ARGUMENT", 2: "DIMENSION_MISMATCH", 3: "NONFINITE", 4: "CUDA",
    5: "OUT_OF_MEMORY", 6: "UNSUPPORTED", 7: "DEVICE_TIMEOUT",
}

SHIFT_CURRENT = 1
INJECTION_CURRENT = 2
BERRY_CURVATURE = 3
QUANTUM_METRIC = 4
INTRINSIC_AHC = 5
BERRY_DIPOLE = 6
SECOND_HARMONIC = 7
JERK_CURRENT = 8
LINEAR_TRANSPORT_BERRY = 9
BERRY_DIPOLE_SEA = 10

GAUSSIAN = 0
LORENTZIAN = 1

PRECISION_FP64 = 0
PRECISION_MIXED = 1

MAX_RESPONSES = 8
MAX_COMPONENTS = 81

# Kinds whose values carry the photon-energy axis.
FREQUENCY_KINDS = (SHIFT_CURRENT, INJECTION_CURRENT, JERK_CURRENT)
FERMI_AXIS_KINDS = (INTRINSIC_AHC, BERRY_DIPOLE, LINEAR_TRANSPORT_BERRY, BERRY_DIPOLE_SEA)


class ModelDesc(ctypes.Structure):
    _fields_ = [
        ("num_orbitals", ctypes.c_int64),
        ("num_r_vectors", ctypes.c_int64),
        ("lattice", ctypes.POINTER(ctypes.c_double)),
        ("r_vectors", ctypes.POINTER(ctypes.c_int64)),
        ("r_degeneracies", ctypes.POINTER(ctypes.c_int64)),
        ("hamiltonian_r", ctypes.POINTER(ctypes.c_double)),
        ("position_r", ctypes.POINTER(ctypes.c_double)),
        ("overlap_r", ctypes.POINTER(ctypes.c_double)),
    ]


class ResponseRequest(ctypes.Structure):
    _fields_ = [
        ("kind", ctypes.c_int32),
        ("num_components", ctypes.c_int32),
        ("components", (ctypes.c_int32 * 4) * MAX_COMPONENTS),
    ]


class AutotuneReport(ctypes.Structure):
    """wnlqg_autotune_report."""
    _fields_ = [
        ("eigh_team", ctypes.c_int32),
        ("energies_per_thread", ctypes.c_int32),
        ("eigh_ms", ctypes.c_double * 3),
        ("response_ms", ctypes.c_double * 3),
        ("from_cache", ctypes.c_int32),
        ("warm_start", ctypes.c_int32),
        ("start_ms", ctypes.c_double * 2),
        ("response_threads", ctypes.c_int32),
        ("width_ms", ctypes.c_double * 2),
        ("metric_shg_grid", ctypes.c_int32),
        ("metric_shg_grid_ms", ctypes.c_double * 3),
        ("shg_grid", ctypes.c_int32),
        ("shg_grid_ms", ctypes.c_double * 3),
        ("response_grid", ctypes.c_int32),
        ("response_grid_ms", ctypes.c_double * 3),
        ("eigh_grid", ctypes.c_int32),
        ("eigh_grid_ms", ctypes.c_double * 3),
    ]


class TaskDesc(ctypes.Structure):
    _fields_ = [
        ("num_responses", ctypes.c_int32),
        ("responses", ResponseRequest * MAX_RESPONSES),
        ("fermi_energy", ctypes.c_double),
        ("temperature", ctypes.c_double),
        ("broadening_type", ctypes.c_int32),
        ("broadening", ctypes.c_double),
        ("transition_window_factor", ctypes.c_double),
        ("denominator_regularization", ctypes.c_double),
        ("degeneracy_threshold", ctypes.c_double),
        ("num_photon_energies", ctypes.c_int64),
        ("photon_energies", ctypes.POINTER(ctypes.c_double)),
        ("num_fermi_energies", ctypes.c_int64),
        ("fermi_energies", ctypes.POINTER(ctypes.c_double)),
        ("precision", ctypes.c_int32),
        ("fermi_surface_broadening", ctypes.c_double),
        ("shg_low_frequency_broadening", ctypes.c_double),
        ("shg_intermediate_regularization", ctypes.c_double),
        ("shg_eta_correction", ctypes.c_int32),
        ("band_window_size", ctypes.c_int32),
        ("use_band_selection", ctypes.c_int32),
        ("valence_bands", ctypes.c_uint32 * 4),
        ("conduction_bands", ctypes.c_uint32 * 4),
        ("wannier_center_convention", ctypes.c_int32),
        ("spectral_gap_tolerance", ctypes.c_double),
        ("linear_transport_gamma_inter", ctypes.c_double),
        ("finite_difference_step", ctypes.c_double),
        ("derivative_backend", ctypes.c_int32),
    ]


def _dptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))


class ModelArrays:
    """Keeps the contiguous arrays behind a :class:`ModelDesc` alive."""

    def __init__(self, model: TightBindingModel):
        self.lattice = np.asfortranarray(model.lattice, dtype=np.float64)
        self.r_vectors = np.asfortranarray(model.r_vectors, dtype=np.int64)
        self.r_degeneracies = np.ascontiguousarray(model.r_degeneracies, dtype=np.int64)
        # Fortran-ordered complex128 memory == interleaved doubles in Julia's column-major layout.
        self.hamiltonian_r = np.asfortranarray(model.hamiltonian_r, dtype=np.complex128)
        self.position_r = None if model.position_r is None else np.asfortranarray(model.position_r, dtype=np.complex128)
        self.overlap_r = None if model.overlap_r is None else np.asfortranarray(model.overlap_r, dtype=np.complex128)
        self.desc = ModelDesc()
        self.desc.num_orbitals = model.num_orbitals
        self.desc.num_r_vectors = model.num_r_vectors
        self.desc.lattice = _dptr(self.lattice)
        self.desc.r_vectors = _iptr(self.r_vectors)
        self.desc.r_degeneracies = _iptr(self.r_degeneracies)
        self.desc.hamiltonian_r = _dptr(self.hamiltonian_r)
        self.desc.position_r = _dptr(self.position_r) if self.position_r is not None else None
        self.desc.overlap_r = _dptr(self.overlap_r) if self.overlap_r is not None else None


def _axes(component) -> list:
    """'xyy' / (0,1,1) -> [0,1,1,0] padded to four 0-based axes."""
    if isinstance(component, str):
        idx = ["xyz".index(ch) for ch in component]
    else:
        idx = [int(v) for v in component]
    if not 1 <= len(idx) <= 4 or any(i < 0 or i > 2 for i in idx):
        raise ValueError(f"invalid Cartesian component {component!r}")
    return idx + [0] * (4 - len(idx))


class TaskArrays:
    """Keeps the arrays behind a :class:`TaskDesc` alive."""

    def __init__(self, responses: Sequence[tuple], *, fermi_energy=0.0, temperature=0.0,
                 broadening_type=GAUSSIAN, broadening=0.040, transition_window_factor=5.0,
                 denominator_regularization=0.001, degeneracy_threshold=2.0e-3,
                 photon_energies=(0.10,), fermi_energies=(), precision=PRECISION_FP64,
                 fermi_surface_broadening=0.0, shg_low_frequency_broadening=0.025,
                 shg_intermediate_regularization=0.0, shg_eta_correction=True, band_window_size=-1,
                 band_selection=None, wannier_center_convention="II", spectral_gap_tolerance=1e-10,
                 linear_transport_gamma_inter=0.0, finite_difference_step=1e-4,
                 derivative_backend="finite_difference"):
        if not 1 <= len(responses) <= MAX_RESPONSES:
            raise ValueError("between 1 and 8 responses are supported per task")
        self.photon_energies = np.ascontiguousarray(np.asarray(photon_energies, dtype=np.float64))
        self.fermi_energies = np.ascontiguousarray(np.asarray(fermi_energies, dtype=np.float64))
        d = TaskDesc()
        d.num_responses = len(responses)
        self.responses = []
        self.components = []   # per response: the 0-based Cartesian axes of each component
        for i, (kind, comps) in enumerate(responses):
            comps = list(comps)
            if not 1 <= len(comps) <= MAX_COMPONENTS:
                raise ValueError("between 1 and 81 components per response")
            d.responses[i].kind = int(kind)
            d.responses[i].num_components = len(comps)
            for c, comp in enumerate(comps):
                ax = _axes(comp)
                for j in range(4):
                    d.responses[i].components[c][j] = ax[j]
            self.responses.append((int(kind), len(comps)))
            self.components.append([tuple(["xyz".index(ch) for ch in comp]) if isinstance(comp, str)
                                    else tuple(int(v) for v in comp) for comp in comps])
        d.fermi_energy = float(fermi_energy)
        d.temperature = float(temperature)
        d.broadening_type = int(broadening_type)
        d.broadening = float(broadening)
        d.transition_window_factor = float(transition_window_factor)
        d.denominator_regularization = float(denominator_regularization)
        d.degeneracy_threshold = float(degeneracy_threshold)
        d.num_photon_energies = self.photon_energies.size
        d.photon_energies = _dptr(self.photon_energies) if self.photon_energies.size else None
        d.num_fermi_energies = self.fermi_energies.size
        d.fermi_energies = _dptr(self.fermi_energies) if self.fermi_energies.size else None
        d.precision = int(precision)
        d.fermi_surface_broadening = float(fermi_surface_broadening)
        d.shg_low_frequency_broadening = float(shg_low_frequency_broadening)
        d.shg_intermediate_regularization = float(shg_intermediate_regularization)
        d.shg_eta_correction = 1 if shg_eta_correction else 0
        d.band_window_size = int(band_window_size)
        if wannier_center_convention not in ("I", "II"):
            raise ValueError("wannier_center_convention must be 'I' or 'II'")
        d.wannier_center_convention = 1 if wannier_center_convention == "I" else 0
        d.spectral_gap_tolerance = float(spectral_gap_tolerance)
        d.linear_transport_gamma_inter = float(linear_transport_gamma_inter)
        d.finite_difference_step = float(finite_difference_step)
        if derivative_backend not in ("finite_difference", "analytic"):
            raise ValueError("derivative_backend must be 'finite_difference' or 'analytic'")
        d.derivative_backend = 1 if derivative_backend == "analytic" else 0
        # band_selection = (conduction bands, valence bands), 1-based as in the reference's
        # cfg.band_selection; pairs (n, m) with n valence and m conduction are kept.
        if band_selection is not None:
            conduction, valence = band_selection
            d.use_band_selection = 1
            for field, bands in (("conduction_bands", conduction), ("valence_bands", valence)):
                words = [0, 0, 0, 0]
                for band in bands:
                    i = int(band) - 1
                    if not 0 <= i < 128:
                        raise ValueError(f"band {band} outside 1..128")
                    words[i // 32] |= 1 << (i % 32)
                arr = getattr(d, field)
                for w in range(4):
                    arr[w] = words[w]
        self.desc = d

    def value_count(self) -> int:
        total = 0
        for kind, nc in self.responses:
            if kind in FREQUENCY_KINDS:
                total += nc * self.photon_energies.size
            elif kind == SECOND_HARMONIC:
                total += nc * self.photon_energies.size * 14
            elif kind in FERMI_AXIS_KINDS:
                total += nc * self.fermi_energies.size
            else:
                total += nc
        return total

    def block_offsets(self) -> list:
        """(offset, length) of each response's block in the concatenated value vector."""
        out = []
        off = 0
        for kind, nc in self.responses:
            if kind == SECOND_HARMONIC:
                n = nc * self.photon_energies.size * 14
            elif kind in FREQUENCY_KINDS:
                n = nc * self.photon_energies.size
            elif kind in FERMI_AXIS_KINDS:
                n = nc * self.fermi_energies.size
            else:
                n = nc
            out.append((off, n))
            off += n
        return out

    def split(self, values: np.ndarray) -> list:
        """Split a concatenated value vector into one (axis, component) array per response;
        second harmonic responses come out as (photon energy, component, term, quantity)."""
        out = []
        off = 0
        for kind, nc in self.responses:
            if kind == SECOND_HARMONIC:
                na = self.photon_energies.size
                block = values[..., off:off + na * nc * 14].reshape(values.shape[:-1] + (2, 7, nc, na))
                out.append(np.moveaxis(block, (-1, -2, -3, -4), (-4, -3, -2, -1)))
                off += na * nc * 14
                continue
            if kind in FREQUENCY_KINDS:
                na = self.photon_energies.size
            elif kind in FERMI_AXIS_KINDS:
                na = self.fermi_energies.size
            else:
                na = 1
            out.append(values[..., off:off + na * nc].reshape(values.shape[:-1] + (nc, na)).swapaxes(-1, -2))
            off += na * nc
        return out
