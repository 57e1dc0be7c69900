"""Model container, _tb.dat reader/writer and the synthetic generators (host logic)."""
import os

import numpy as np

from conftest import GOLDEN
from wanniernlqg_b200.model import (read_wannier_tb, reference_workload_model, synthetic_nonorthogonal_model,
                                    write_wannier_tb)


def test_read_reference_fixture():
    m = read_wannier_tb(os.path.join(GOLDEN, "synthetic_tb.dat"))
    assert m.num_orbitals == 4 and m.num_r_vectors == 2
    assert list(m.r_degeneracies) == [2, 4]
    assert m.hamiltonian_r[0, 0, 0] == -2.5
    assert m.hamiltonian_r[1, 0, 0] == 0.15000000000000002
    np.testing.assert_array_equal(m.r_vectors[:, 1], [1, 0, 0])


def test_write_read_roundtrip(tmp_path):
    m = reference_workload_model("nw4")
    p = tmp_path / "m_tb.dat"
    write_wannier_tb(m, str(p))
    m2 = read_wannier_tb(str(p))
    assert np.array_equal(m.hamiltonian_r, m2.hamiltonian_r)
    assert np.array_equal(m.position_r, m2.position_r)
    assert np.array_equal(m.r_vectors, m2.r_vectors)


def test_generator_hermitian_pairing_and_sizes():
    for name, nw, nr in (("nw4", 4, 125), ("nw32", 32, 729)):
        m = reference_workload_model(name)
        assert m.num_orbitals == nw and m.num_r_vectors == nr
        idx = {tuple(m.r_vectors[:, i]): i for i in range(nr)}
        for i in range(nr):
            j = idx[tuple(-m.r_vectors[:, i])]
            assert np.array_equal(m.hamiltonian_r[:, :, i], m.hamiltonian_r[:, :, j].conj().T)
            for a in range(3):
                assert np.array_equal(m.position_r[:, :, a, i], m.position_r[:, :, a, j].conj().T)


def test_generator_is_seeded():
    a = reference_workload_model("nw4")
    b = reference_workload_model("nw4")
    assert np.array_equal(a.hamiltonian_r, b.hamiltonian_r)


def test_nonorthogonal_overlap_positive():
    m = synthetic_nonorthogonal_model(8, 1, 0)
    rng = np.random.default_rng(0)
    for k in rng.random((5, 3)):
        ph = np.exp(2j * np.pi * (m.r_vectors.T @ k))
        s = np.einsum("ijr,r->ij", m.overlap_r, ph)
        assert np.linalg.eigvalsh(s).min() >= 0.5 - 1e-12
