"""CPU stand-in for the GPU refinement proposer, built on the numpy MLP oracle.

TEST INFRASTRUCTURE ONLY: lets the cell-adaptive controller's logic be exercised without a
GPU (same interface as wanniernlqg_b200.adaptive.MlpProposer; Adam in numpy)."""
import numpy as np

from oracle import mlp_oracle as M
from wanniernlqg_b200.adaptive import MlpProposer


class NumpyMlpProposer(MlpProposer):
    def __init__(self, fermi_energy, omegas, spectrum_fn, *, seed=1, train_steps=200, learning_rate=3e-3):
        self.mu = float(fermi_energy)
        om = np.asarray(omegas, dtype=np.float64)
        self.om_lo, self.om_hi = float(om.min()), float(om.max())
        self.spectrum_fn = spectrum_fn
        self.kscale = 2.0 * np.pi * np.ones(3)
        self.support = None
        self.must_check = None
        self.train_steps = train_steps
        self.lr = learning_rate
        self.X, self.E = [], []
        self.spectrum_evaluations = 0
        rng = np.random.default_rng(seed)
        p = np.zeros(M.COUNT)
        for name, fan_out, fan_in in (("W1", M.H, M.F), ("W2", M.H, M.H), ("W3", M.H, M.H), ("w4", 1, M.H)):
            o, size = M.OFF[name]
            lim = np.sqrt(6.0 / (fan_in + fan_out))
            p[o:o + size] = rng.uniform(-lim, lim, size)
        self.p = p.astype(np.float32)
        self.m = np.zeros(M.COUNT)
        self.v = np.zeros(M.COUNT)
        self.t = 0

    def close(self):
        pass

    def train(self):
        X = np.concatenate(self.X)
        Y = self._targets()
        p = self.p.astype(np.float64)
        for _ in range(self.train_steps):
            _, g = M.loss_grad(p.astype(np.float32), X, Y)
            self.t += 1
            self.m = 0.9 * self.m + 0.1 * g
            self.v = 0.999 * self.v + 0.001 * g * g
            p = p - self.lr * (self.m / (1 - 0.9 ** self.t)) / (np.sqrt(self.v / (1 - 0.999 ** self.t)) + 1e-8)
        self.p = p.astype(np.float32)
        loss, _ = M.loss_grad(self.p, X, Y)
        return loss

    def predict(self, feats):
        y, _ = M.forward(self.p, feats)
        return 10.0 ** (10.0 * y)
