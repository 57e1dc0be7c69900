"""Adaptive integration on the GPU engine: the HCubature controller against the oracle, and the
cell-adaptive integrator with and without the learned proposer."""
import numpy as np
import pytest

from wanniernlqg_b200 import _abi
from wanniernlqg_b200.model import reference_workload_model, synthetic_orthogonal_model

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def engine_cls():
    from wanniernlqg_b200 import build
    build.build()
    from wanniernlqg_b200.engine import ResponseEngine
    return ResponseEngine


def test_hcubature_controller_with_gpu_nodes_matches_oracle_nodes(engine_cls, oracle_mod):
    from wanniernlqg_b200.integration import HAdaptiveCubature, IntegrationDomain, integrate_response
    model = reference_workload_model("nw4")
    task = _abi.TaskArrays([(_abi.BERRY_CURVATURE, ["xy"]), (_abi.QUANTUM_METRIC, ["xx"])],
                           fermi_energy=0.0, temperature=300.0)
    domain = IntegrationDomain(lower=(0.0, 0.0, 0.0), upper=(1.0, 1.0, 1.0))
    alg = HAdaptiveCubature(atol=1e-9, rtol=1e-4, max_evaluations=40_000)
    with engine_cls(model, task) as eng:
        g = integrate_response(None, domain, alg, batch_evaluator=eng.point_values)
    o = integrate_response(None, domain, alg, batch_evaluator=lambda x: oracle_mod.point_values(model, task, x))
    assert g.evaluations == o.evaluations
    assert np.max(np.abs(g.value - o.value)) <= 1e-9 * np.max(np.abs(o.value))


def _bump():
    k0 = np.array([0.31, 0.62, 0.47])
    s = 0.03

    def f(k):
        d = (k - k0 + 0.5) % 1.0 - 0.5
        return np.exp(-np.sum(d * d, axis=1) / (2 * s * s))[:, None].astype(complex)

    return f, (2 * np.pi * s * s) ** 1.5


def test_gpu_trained_proposer_saves_evaluations_on_a_localised_integrand():
    """What the trained network gains: on a localised integrand the GPU-trained proposer reaches
    the same tolerance as the plain cell-adaptive method with fewer integrand evaluations."""
    from wanniernlqg_b200 import build
    from wanniernlqg_b200.adaptive import MlpProposer, integrate_cells
    build.build()
    f, exact = _bump()
    spec = lambda k: (np.zeros((k.shape[0], 2)) + np.array([-1.0, 1.0]), None)
    plain = integrate_cells(f, n0=16, rtol=1e-2, max_level=6)
    prop = MlpProposer(0.0, [1.0], spec, seed=2, train_steps=300)
    try:
        learned = integrate_cells(f, n0=16, rtol=1e-2, max_level=6, proposer=prop)
    finally:
        prop.close()
    assert plain.converged and learned.converged
    assert abs(plain.value[0] - exact) < 1e-2 * exact
    assert abs(learned.value[0] - exact) < 1e-2 * exact
    assert learned.evaluations < 0.7 * plain.evaluations, (learned, plain)


def test_learned_proposer_on_band_crossing_injection_current():
    """The learned adaptive refinement workload's own integrand: the circular injection current
    eta^xyz of the nw = 16 model whose bands 8 and 9 cross at mu = 0, Gaussian width 2 meV at
    10-20 meV (the Weyl node's resonance shells), cells from 48^3.  With the support guard (every
    cell whose spectrum can reach the broadened window is checked) the learned path's first round
    equals the plain FP64 method's to 1e-3.  At this cell size the guard keeps nearly every cell,
    so the safe learned path saves no evaluations on this integrand: the plain method stays the
    judge."""
    from wanniernlqg_b200 import _abi, build
    from wanniernlqg_b200.adaptive import MlpProposer, integrate_cells
    from wanniernlqg_b200.engine import ResponseEngine
    from wanniernlqg_b200.model import crossing_model
    build.build()
    model = crossing_model(16, 2, 0)
    om = np.array([0.01, 0.015, 0.02])
    eta = 0.002
    cutoff = np.sqrt(200.0) * eta

    def task(prec):
        return _abi.TaskArrays([(_abi.INJECTION_CURRENT, ["xyz"])], broadening_type=_abi.GAUSSIAN, broadening=eta,
                               photon_energies=om, fermi_energy=0.0, precision=prec)

    with ResponseEngine(model, task(_abi.PRECISION_FP64)) as eng:
        plain = integrate_cells(eng.point_values, n0=48, rtol=1e-4, max_level=8, max_rounds=1)
    results = {}
    with ResponseEngine(model, task(_abi.PRECISION_MIXED)) as eng:
        prop = MlpProposer(0.0, om, lambda k: eng.spectrum(k, vectors=False), seed=3, lattice=model.lattice,
                           support=(om.min() - cutoff, om.max() + cutoff))
        try:
            results[True] = integrate_cells(eng.point_values, n0=48, rtol=1e-4, max_level=8, max_rounds=1,
                                            proposer=prop, seed=3)
        finally:
            prop.close()
    ref = np.max(np.abs(plain.value))
    assert ref > 0
    guarded = results[True]
    assert np.max(np.abs(guarded.value - plain.value)) <= 1e-3 * ref
    # At 48^3 almost every cell can hold a resonance: the guard keeps >= 99 % of them.
    assert guarded.checked_cells >= 0.99 * plain.checked_cells
