"""CPU check of the fixed-point slicing behind the tensor-core Fourier (Ozaki-type split).

Restates the scheme with numpy: phases and channel tiles are cut into S int8 slices
(y = sum_i a_i 2^(-6-7i), |a_i| <= 64, per-row power-of-two scale for the tiles), every pair of
slices with level i + j < S is multiplied with exact integer accumulation, and the levels are
combined in FP64.  The result must reproduce the FP64 Fourier sum X(k) = sum_R f_R(k) T_R to
the stated bound: 2^(-7S) of the row scale times a small multiple of sqrt(K).
"""
import numpy as np
import pytest

from wanniernlqg_b200.model import reference_workload_model


def slices(y, S):
    """int8 slices of |y| <= 1 with units 2^(-6-7i) (round to nearest, exact in FP64)."""
    out = np.zeros((S,) + y.shape, dtype=np.int64)
    unit = 2.0 ** -6
    r = y.copy()
    for i in range(S):
        a = np.rint(r / unit)
        out[i] = a
        r = r - a * unit
        unit *= 2.0 ** -7
    assert np.all(np.abs(out) <= 64)
    return out


def ozaki_fourier(phase, tiles, S):
    """phase [nk, NR] complex, tiles [NR, N] complex -> X [nk, N] via the sliced real GEMM."""
    nk, nr = phase.shape
    N = tiles.shape[1]
    A = np.zeros((nk, 2 * nr))
    A[:, 0::2], A[:, 1::2] = phase.real, phase.imag
    B = np.zeros((2 * N, 2 * nr))
    B[0::2, 0::2], B[0::2, 1::2] = tiles.real.T, -tiles.imag.T
    B[1::2, 0::2], B[1::2, 1::2] = tiles.imag.T, tiles.real.T
    mx = np.max(np.abs(B), axis=1)
    e = np.where(mx > 0, np.frexp(mx)[1], 0)
    Bs = slices(B / np.ldexp(1.0, e)[:, None], S)
    As = slices(A, S)
    D = np.zeros((nk, 2 * N))
    for lv in range(S):
        acc = np.zeros((nk, 2 * N), dtype=np.int64)
        for i in range(lv + 1):
            acc += As[i] @ Bs[lv - i].T
        assert np.max(np.abs(acc)) < 2 ** 31   # int32 TMEM accumulators do not overflow
        D += acc.astype(np.float64) * 2.0 ** (-7 * lv)
    D *= np.ldexp(1.0, e - 12)[None, :]
    return D[:, 0::2] + 1j * D[:, 1::2]


@pytest.mark.parametrize("name,S", [("nw4", 7), ("nw4", 4), ("nw32", 7)])
def test_sliced_fourier_matches_fp64(name, S):
    model = reference_workload_model(name)
    rng = np.random.default_rng(7)
    k = rng.random((6, 3))
    phase = np.exp(2j * np.pi * (k @ model.r_vectors)) / model.r_degeneracies[None, :]
    rc = model.lattice.T @ model.r_vectors
    nw = model.num_orbitals
    H = model.hamiltonian_r.reshape(nw * nw, -1).T                 # [NR, nw^2]
    chans = [H, H * (1j * rc[0])[:, None], H * (-rc[0] * rc[1])[:, None]]
    if model.position_r is not None:
        chans.append(model.position_r[:, :, 1, :].reshape(nw * nw, -1).T)
    tiles = np.concatenate(chans, axis=1)
    if name == "nw32":
        tiles = tiles[:, : 4 * nw * nw]
        k = k[:2]
        phase = phase[:2]
    ref = phase @ tiles
    got = ozaki_fourier(phase, tiles, S)
    scale = np.max(np.abs(tiles), axis=0)          # per-column (row of B) scale
    err = np.max(np.abs(got - ref) / np.maximum(scale, 1e-300)[None, :])
    bound = 16.0 * np.sqrt(2 * model.num_r_vectors) * 2.0 ** (-7 * S)
    assert err < bound
