"""Cell-adaptive integrator logic on CPU (the proposer here is the numpy MLP oracle)."""
import numpy as np

from wanniernlqg_b200.adaptive import integrate_cells


def _bump():
    k0 = np.array([0.31, 0.62, 0.47])
    s = 0.03

    def f(k):
        d = (k - k0 + 0.5) % 1.0 - 0.5
        return np.exp(-np.sum(d * d, axis=1) / (2 * s * s))[:, None].astype(complex)

    return f, (2 * np.pi * s * s) ** 1.5


def test_plain_cells_converge_on_smooth_and_localised_integrands():
    f, exact = _bump()
    r = integrate_cells(f, n0=16, rtol=1e-3, max_level=6)
    assert r.converged and abs(r.value[0] - exact) < 1e-3 * exact
    g = lambda k: (1.0 + 0.3 * np.cos(2 * np.pi * k[:, 0]) * np.sin(2 * np.pi * k[:, 1]))[:, None].astype(complex)
    r2 = integrate_cells(g, n0=8, rtol=1e-3, max_level=3)
    assert r2.converged and abs(r2.value[0] - 1.0) < 1e-3


def test_learned_proposer_saves_evaluations_cpu():
    from oracle.mlp_proposer_cpu import NumpyMlpProposer
    f, exact = _bump()
    spec = lambda k: (np.zeros((k.shape[0], 2)) + np.array([-1.0, 1.0]), None)
    plain = integrate_cells(f, n0=16, rtol=1e-2, max_level=6)
    learned = integrate_cells(f, n0=16, rtol=1e-2, max_level=6,
                              proposer=NumpyMlpProposer(0.0, [1.0], spec, seed=2, train_steps=150))
    assert learned.converged and abs(learned.value[0] - exact) < 1e-2 * exact
    assert learned.evaluations < 0.7 * plain.evaluations
