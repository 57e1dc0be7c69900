"""Python access to the CPU FP64 oracle (oracle/wnlqg_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and bench.py's CPU
baseline leg, as the checker.  The product package never imports this module.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import TightBindingModel

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libwnlqg_oracle.so")
_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (g++ -fopenmp); returns the library path."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        dp = ctypes.POINTER(ctypes.c_double)
        ip = ctypes.POINTER(ctypes.c_int64)
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_value_count.argtypes = [ctypes.POINTER(_abi.TaskDesc)]
        L.oracle_value_count.restype = ctypes.c_int64
        L.oracle_point_values.argtypes = [ctypes.POINTER(_abi.ModelDesc), ctypes.POINTER(_abi.TaskDesc), dp,
                                          ctypes.c_int64, ctypes.c_int, dp]
        L.oracle_integrate_mesh.argtypes = [ctypes.POINTER(_abi.ModelDesc), ctypes.POINTER(_abi.TaskDesc), ip,
                                            ctypes.c_int64, ctypes.c_int64, ctypes.c_int, dp]
        L.oracle_kpoint_spectrum.argtypes = [ctypes.POINTER(_abi.ModelDesc), dp, ctypes.c_int, dp, dp, dp]
        L.oracle_hermitian_eigen.argtypes = [ctypes.c_int64, dp, dp, dp]
        L.oracle_generalized_eigen.argtypes = [ctypes.c_int64, dp, dp, dp, dp]
        L.oracle_generalized_eigen.restype = ctypes.c_int
        L.oracle_jerk_algebra.argtypes = [ctypes.c_int64, dp, dp, dp, dp, ctypes.c_int64, dp, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, ctypes.c_int64, ctypes.POINTER(ctypes.c_int32), dp]
        L.oracle_kpoint_data.argtypes = [ctypes.POINTER(_abi.ModelDesc), dp, dp, dp, dp, dp, dp]
        L.oracle_kpoint_geometry.argtypes = [ctypes.POINTER(_abi.ModelDesc), dp, ctypes.c_double, dp, dp, dp, dp,
                                             dp]
        L.oracle_shg_algebra.argtypes = [ctypes.c_int64, dp, dp, dp, dp, dp, ctypes.c_int64, dp, ctypes.c_int64,
                                         ctypes.POINTER(ctypes.c_int32), ctypes.c_double, ctypes.c_double,
                                         ctypes.c_double, ctypes.c_double, ctypes.c_int, ctypes.c_double,
                                         ctypes.c_int, ctypes.c_double, dp]
        for name in ("oracle_point_values", "oracle_integrate_mesh", "oracle_kpoint_spectrum",
                     "oracle_hermitian_eigen", "oracle_jerk_algebra", "oracle_kpoint_data", "oracle_shg_algebra",
                     "oracle_kpoint_geometry"):
            getattr(L, name).restype = ctypes.c_int
        _lib = L
    return _lib


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _check(rc):
    if rc != 0:
        raise RuntimeError(f"oracle error {rc}: {lib().oracle_last_error().decode()}")


def point_values(model: TightBindingModel, task: _abi.TaskArrays, kpoints, threads: int = 0) -> np.ndarray:
    """Per-point concatenated values, complex array [n, value_count]."""
    k = np.ascontiguousarray(np.asarray(kpoints, dtype=np.float64).reshape(-1, 3))
    m = _abi.ModelArrays(model)
    vc = task.value_count()
    out = np.zeros((k.shape[0], vc), dtype=np.complex128)
    _check(lib().oracle_point_values(ctypes.byref(m.desc), ctypes.byref(task.desc), _dp(k), k.shape[0], threads,
                                     _dp(out)))
    return out


def integrate_mesh(model: TightBindingModel, task: _abi.TaskArrays, mesh, k_begin=0, k_end=None,
                   threads: int = 0) -> np.ndarray:
    """Lane-ordered mesh sum of value/Nk over [k_begin, k_end); complex [value_count]."""
    mesh_a = np.ascontiguousarray(np.asarray(mesh, dtype=np.int64))
    nk = int(np.prod(mesh_a))
    if k_end is None:
        k_end = nk
    m = _abi.ModelArrays(model)
    out = np.zeros(task.value_count(), dtype=np.complex128)
    _check(lib().oracle_integrate_mesh(ctypes.byref(m.desc), ctypes.byref(task.desc),
                                       mesh_a.ctypes.data_as(ctypes.POINTER(ctypes.c_int64)), k_begin, k_end,
                                       threads, _dp(out)))
    return out


def kpoint_spectrum(model: TightBindingModel, k, convention: str = "II"):
    """(energies[nw], canonical U[nw, nw], Hamiltonian-gauge dH[nw, nw, 3]) at one k, in the
    given Wannier-center convention ("II" or "I")."""
    nw = model.num_orbitals
    m = _abi.ModelArrays(model)
    kk = np.ascontiguousarray(np.asarray(k, dtype=np.float64))
    e = np.zeros(nw)
    u = np.zeros((nw, nw), dtype=np.complex128, order="F")
    dh = np.zeros((nw, nw, 3), dtype=np.complex128, order="F")
    _check(lib().oracle_kpoint_spectrum(ctypes.byref(m.desc), _dp(kk), 1 if convention == "I" else 0, _dp(e), _dp(u),
                                        _dp(dh)))
    return e, u, dh


def hermitian_eigen(h: np.ndarray):
    """Oracle eigensolve of one Hermitian matrix (upper triangle), canonicalised columns."""
    h = np.asfortranarray(h, dtype=np.complex128)
    n = h.shape[0]
    e = np.zeros(n)
    u = np.zeros((n, n), dtype=np.complex128, order="F")
    _check(lib().oracle_hermitian_eigen(n, _dp(h), _dp(e), _dp(u)))
    return e, u


def generalized_eigen(h: np.ndarray, s: np.ndarray):
    """Oracle generalised eigensolve (upper triangles): energies and S-orthonormal canonical C."""
    h = np.asfortranarray(h, dtype=np.complex128)
    s_ = np.asfortranarray(s, dtype=np.complex128)
    n = h.shape[0]
    e = np.zeros(n)
    c = np.zeros((n, n), dtype=np.complex128, order="F")
    _check(lib().oracle_generalized_eigen(n, _dp(h), _dp(s_), _dp(e), _dp(c)))
    return e, c


def jerk_algebra(energies, B, A, C, omegas, components, *, mu=0.0, T=0.0, width=0.04, gaussian=True,
                 reg=0.001, window=5.0) -> np.ndarray:
    """Jerk Eq. 9.20 on prepared inputs: complex [n_omega, n_components]."""
    e = np.ascontiguousarray(np.asarray(energies, dtype=np.float64))
    n = e.size
    Bf = np.asfortranarray(B, dtype=np.complex128)
    Af = np.asfortranarray(A, dtype=np.complex128)
    Cf = np.asfortranarray(C, dtype=np.complex128)
    om = np.ascontiguousarray(np.asarray(omegas, dtype=np.float64))
    comps = np.ascontiguousarray(np.array([_abi._axes(c) for c in components], dtype=np.int32))
    out = np.zeros((om.size, len(components)), dtype=np.complex128, order="F")
    _check(lib().oracle_jerk_algebra(n, _dp(e), _dp(Bf), _dp(Af), _dp(Cf), om.size, _dp(om), mu, T, width,
                                     1 if gaussian else 0, reg, window, len(components),
                                     comps.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), _dp(out)))
    return out


def kpoint_data(model: TightBindingModel, k):
    """Hamiltonian-gauge band data at one k: energies[nw], dH[nw,nw,3], A[nw,nw,3],
    dA[nw,nw,3,3] (position axis, derivative axis) and ddH[nw,nw,3,3]."""
    nw = model.num_orbitals
    m = _abi.ModelArrays(model)
    kk = np.ascontiguousarray(np.asarray(k, dtype=np.float64))
    e = np.zeros(nw)
    dh = np.zeros((nw, nw, 3), dtype=np.complex128, order="F")
    a = np.zeros((nw, nw, 3), dtype=np.complex128, order="F")
    da = np.zeros((nw, nw, 3, 3), dtype=np.complex128, order="F")
    ddh = np.zeros((nw, nw, 3, 3), dtype=np.complex128, order="F")
    _check(lib().oracle_kpoint_data(ctypes.byref(m.desc), _dp(kk), _dp(e), _dp(dh), _dp(a), _dp(da), _dp(ddh)))
    return e, dh, a, da, ddh


def kpoint_geometry(model: TightBindingModel, k, eta: float = 0.0):
    """Hamiltonian-gauge geometry at one k (canonical gauge): energies[nw], U[nw, nw],
    r[nw, nw, 3] (A + i D), gder[nw, nw, a, b] = r^a_{nm;b} and F[nw, nw, a, b], at denominator
    regularization ``eta`` (0: bare inverses)."""
    nw = model.num_orbitals
    m = _abi.ModelArrays(model)
    kk = np.ascontiguousarray(np.asarray(k, dtype=np.float64))
    e = np.zeros(nw)
    u = np.zeros((nw, nw), dtype=np.complex128, order="F")
    r = np.zeros((nw, nw, 3), dtype=np.complex128, order="F")
    g = np.zeros((nw, nw, 3, 3), dtype=np.complex128, order="F")
    f = np.zeros((nw, nw, 3, 3), dtype=np.complex128, order="F")
    _check(lib().oracle_kpoint_geometry(ctypes.byref(m.desc), _dp(kk), float(eta), _dp(e), _dp(u), _dp(r), _dp(g),
                                        _dp(f)))
    return e, u, r, g, f


def shg_algebra(energies, V, A, dA, W, omegas, components, *, mu=0.0, T=0.0, broadening=0.025,
                low_frequency_broadening=0.025, gaussian=True, eta=0.04, eta_correction=True,
                degeneracy=0.002) -> np.ndarray:
    """Seven-term SHG on prepared Hamiltonian-gauge inputs: complex [n_omega, n_components, 7, 2]."""
    e = np.ascontiguousarray(np.asarray(energies, dtype=np.float64))
    n = e.size
    arrs = [np.asfortranarray(x, dtype=np.complex128) for x in (V, A, dA, W)]
    om = np.ascontiguousarray(np.asarray(omegas, dtype=np.float64))
    comps = np.ascontiguousarray(np.array([_abi._axes(c) for c in components], dtype=np.int32))
    out = np.zeros((om.size, len(components), 7, 2), dtype=np.complex128, order="F")
    _check(lib().oracle_shg_algebra(n, _dp(e), *[_dp(x) for x in arrs], om.size, _dp(om), len(components),
                                    comps.ctypes.data_as(ctypes.POINTER(ctypes.c_int32)), mu, T, broadening,
                                    low_frequency_broadening, 1 if gaussian else 0, eta,
                                    1 if eta_correction else 0, degeneracy, _dp(out)))
    return out
