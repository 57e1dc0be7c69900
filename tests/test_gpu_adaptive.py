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


def test_learned_cells_match_plain_with_fewer_checked_cells(engine_cls):
    from wanniernlqg_b200.adaptive import MlpProposer, integrate_cells
    model = synthetic_orthogonal_model(8, 1, 3, full_position=True)
    omegas = np.linspace(0.5, 2.5, 8)
    task = _abi.TaskArrays([(_abi.INJECTION_CURRENT, ["xyy"])], broadening_type=_abi.LORENTZIAN, broadening=0.02,
                           photon_energies=omegas, precision=_abi.PRECISION_MIXED)
    with engine_cls(model, task) as eng:
        plain = integrate_cells(eng.point_values, n0=12, rtol=2e-3, max_level=5)
        prop = MlpProposer(0.0, omegas, eng.spectrum, seed=3)
        try:
            learned = integrate_cells(eng.point_values, n0=12, rtol=2e-3, max_level=5, proposer=prop)
        finally:
            prop.close()
    assert plain.converged and learned.converged
    scale = np.max(np.abs(plain.value))
    assert np.max(np.abs(learned.value - plain.value)) < 1e-2 * scale
    assert learned.checked_cells < plain.checked_cells
