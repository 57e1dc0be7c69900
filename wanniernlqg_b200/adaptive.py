"""Cell-adaptive k-space integration with an optional learned refinement proposer.

Scheme (this engine's own; the reference's adaptive integrator is the HCubature controller in
:mod:`wanniernlqg_b200.integration`):

* The unit cell [0,1)^3 starts as N0^3 cubic cells.  Every leaf cell has a coarse value,
  its volume times the integrand at its centre.
* A cell is *checked* by evaluating the integrand at the centres of its 8 octants; its fine
  value is their mean times the volume and its error estimate is ||fine - coarse|| (maximum
  absolute complex entry, the reference's norm).  A checked cell contributes its fine value.
* Each round splits the checked cells with the largest errors into their octants (whose coarse
  values are the parent's octant values, so no evaluation is repeated) until the error of the
  cells left unsplit fits the tolerance budget, up to `max_level` levels of refinement.  The
  octant rule is second order, so the fine value's error is estimated as |fine - coarse| / 3.
* Stop when sum(errors) <= rtol * ||I||.

The plain method checks every leaf.  The learned method (``MlpProposer``) predicts log10 of each
unchecked leaf's error from cheap features (cell centre and size, the local minimum transition
energy across the Fermi level and that pair's |v_nm| from the spectrum, the parent's error and
the centre value) and
checks only the leaves predicted above the threshold plus a random audit sample.  The audit
estimates the error mass the network missed (audited under-prediction divided by the audit
fraction); if that mass exceeds the tolerance budget, the round falls back to the plain method
and checks every leaf.  Unchecked leaves keep their coarse value (an actual
integrand value) and count their predicted error in the total.  The network never supplies an
integrand value; it only decides which cells are checked first.
"""
from __future__ import annotations

import ctypes
import dataclasses
import time
from typing import Callable, Optional

import numpy as np

from . import _lib

OCTANTS = np.array([[i, j, k] for k in (0, 1) for j in (0, 1) for i in (0, 1)], dtype=np.float64) - 0.5


@dataclasses.dataclass
class AdaptiveResult:
    value: np.ndarray
    error_estimate: float
    evaluations: int
    leaves: int
    checked_cells: int
    rounds: int
    converged: bool
    seconds: float
    fallbacks: int = 0


def _norm(x) -> float:
    return float(np.max(np.abs(x))) if np.size(x) else 0.0


class MlpProposer:
    """Feature builder plus the GPU MLP (wnlqg_b200_mlp_*) trained online on checked cells."""

    def __init__(self, fermi_energy: float, omegas, spectrum_fn: Callable, *, device: int = 0, seed: int = 1,
                 train_steps: int = 200, learning_rate: float = 3e-3, lattice=None, support=None):
        self.L = _lib.load()
        self.m = ctypes.c_void_p()
        _lib.check(self.L.wnlqg_b200_mlp_create(device, seed, ctypes.byref(self.m)))
        self.mu = float(fermi_energy)
        om = np.asarray(omegas, dtype=np.float64)
        self.om_lo, self.om_hi = (float(om.min()), float(om.max())) if om.size else (0.0, 0.0)
        self.spectrum_fn = spectrum_fn
        # Transition energies (eV) where the integrand can be nonzero (for interband responses at
        # T = 0: the photon window widened by the broadening's support; (-inf, inf) for Lorentzian
        # tails).  None: no guard, for integrands that are not band resonances.
        self.support = support
        self.must_check = None
        # Cartesian length (Angstrom^-1) of a unit fractional step along each axis: 2 pi |b_a|.
        lat = np.eye(3) if lattice is None else np.asarray(lattice, dtype=np.float64)
        self.kscale = 2.0 * np.pi * np.linalg.norm(np.linalg.inv(lat), axis=0)
        self.train_steps = train_steps
        self.lr = learning_rate
        self.X = []
        self.E = []
        self.spectrum_evaluations = 0

    def close(self):
        if self.m:
            self.L.wnlqg_b200_mlp_destroy(self.m)
            self.m = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def features(self, centers, sizes, parent_err, coarse_norm) -> np.ndarray:
        """Eight inputs per cell: its centre (sin 2 pi c per axis), its size, the local minimum
        transition energy across mu (the smallest E_m - E_n with n occupied and m empty at the
        centre), |v_nm| of that pair (|grad (E_m - E_n)| by a forward difference of the spectrum,
        eV Angstrom), and the method's own signals: the parent's error and the centre value."""
        n = centers.shape[0]
        h = 1e-4
        pts = np.concatenate([centers] + [centers + h * np.eye(3)[a] for a in range(3)]) % 1.0
        e, _ = self.spectrum_fn(pts)
        self.spectrum_evaluations += pts.shape[0]
        e0 = e[:n]
        occ = e0 <= self.mu
        # Smallest occupied -> empty transition energy and its band pair.
        n_top = np.where(occ, np.arange(e0.shape[1])[None, :], -1).max(axis=1)
        m_bot = np.where(~occ, np.arange(e0.shape[1])[None, :], e0.shape[1]).min(axis=1)
        ok = (n_top >= 0) & (m_bot < e0.shape[1])
        nt, mb = np.clip(n_top, 0, e0.shape[1] - 1), np.clip(m_bot, 0, e0.shape[1] - 1)
        rows = np.arange(n)
        gap = np.where(ok, e0[rows, mb] - e0[rows, nt], 10.0)
        grad = np.zeros((n, 3))
        for a in range(3):
            ea = e[(a + 1) * n:(a + 2) * n]
            grad[:, a] = (ea[rows, mb] - ea[rows, nt] - gap) / (h * self.kscale[a])
        vnm = np.where(ok, np.linalg.norm(grad, axis=1), 0.0)
        # Support guard (not learned): a cell whose smallest transition energy can reach the
        # support anywhere inside it (gap - |v_nm| times the Cartesian half diagonal) must be checked,
        # whatever the network predicts, so that a resonance no training sample has hit is never
        # skipped.  Cells without a pair across mu carry no interband weight.
        if self.support is None:
            self.must_check = None
        else:
            half_diag = 0.5 * np.sqrt(np.sum((np.asarray(sizes)[:, None] * self.kscale[None, :]) ** 2, axis=1))
            lo = gap - vnm * half_diag
            hi = gap + vnm * half_diag
            self.must_check = ok & (hi >= self.support[0]) & (lo <= self.support[1])
        f = np.stack([
            np.sin(2 * np.pi * centers[:, 0]), np.sin(2 * np.pi * centers[:, 1]), np.sin(2 * np.pi * centers[:, 2]),
            np.log2(sizes) / 8.0,
            np.log10(np.maximum(gap, 1e-4)) / 3.0,
            np.log10(np.maximum(vnm, 1e-3)) / 3.0,
            np.log10(np.maximum(parent_err, 1e-30)) / 10.0,
            np.log10(np.maximum(coarse_norm, 1e-30)) / 10.0,
        ], axis=1)
        return np.ascontiguousarray(f, dtype=np.float32)

    def observe(self, feats: np.ndarray, errors: np.ndarray):
        self.X.append(feats)
        self.E.append(np.asarray(errors, dtype=np.float64))

    def _targets(self):
        # Errors far below the largest one never decide a refinement: clip them at 1e-6 of the
        # largest so that the fit spends its capacity on the decisive range.
        e = np.concatenate(self.E)
        floor = max(float(np.max(e)) * 1e-6, 1e-300)
        return (np.log10(np.maximum(e, floor)) / 10.0).astype(np.float32)

    def train(self):
        X = np.ascontiguousarray(np.concatenate(self.X), dtype=np.float32)
        Y = np.ascontiguousarray(self._targets(), dtype=np.float32)
        loss = ctypes.c_float()
        fp = ctypes.POINTER(ctypes.c_float)
        _lib.check(self.L.wnlqg_b200_mlp_train(self.m, X.ctypes.data_as(fp), Y.ctypes.data_as(fp), X.shape[0],
                                               self.train_steps, self.lr, ctypes.byref(loss)))
        return loss.value

    def predict(self, feats: np.ndarray) -> np.ndarray:
        y = np.zeros(feats.shape[0], dtype=np.float32)
        fp = ctypes.POINTER(ctypes.c_float)
        _lib.check(self.L.wnlqg_b200_mlp_forward(self.m, feats.ctypes.data_as(fp), feats.shape[0],
                                                 y.ctypes.data_as(fp)))
        return 10.0 ** (10.0 * y.astype(np.float64))


def integrate_cells(point_values: Callable, *, n0: int = 16, rtol: float = 1e-4, max_level: int = 8,
                    max_evaluations: int = 50_000_000, proposer: Optional[MlpProposer] = None,
                    warmup_fraction: float = 0.15, audit_fraction: float = 0.05,
                    safety: float = 4.0, seed: int = 0, component=None,
                    max_leaves: int = 2_000_000, max_rounds: int = 1_000_000) -> AdaptiveResult:
    """Integrate the domain average of point_values(k[n,3]) -> [n, V] over [0,1)^3.

    `component` (index array) restricts the error norm to those value entries (for example the
    sigma^xyy(omega) block); the integral covers all entries.  Every leaf keeps its coarse, fine
    and 8 octant values (10 V complex numbers), so `max_leaves` bounds the host memory: a round
    that would exceed it ends the run unconverged, like the evaluation budget."""
    t0 = time.perf_counter()
    rng = np.random.default_rng(seed)
    g = (np.arange(n0) + 0.5) / n0
    cz, cy, cx = np.meshgrid(g, g, g, indexing="ij")
    centers = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], axis=1)
    half = np.full(centers.shape[0], 0.5 / n0)
    level = np.zeros(centers.shape[0], dtype=np.int64)
    vol = (2 * half) ** 3
    coarse = point_values(centers) * vol[:, None]
    evaluations = centers.shape[0]
    sel = slice(None) if component is None else component
    nv = coarse.shape[1]
    fine = np.zeros_like(coarse)
    octv = np.zeros((centers.shape[0], 8, nv), dtype=coarse.dtype)
    err = np.full(centers.shape[0], np.nan)
    pred = np.full(centers.shape[0], np.nan)
    checked = np.zeros(centers.shape[0], dtype=bool)
    parent_err = np.full(centers.shape[0], 1e-30)
    rounds = 0
    fallbacks = 0
    checked_total = 0

    def check(idx):
        nonlocal evaluations
        if idx.size == 0:
            return
        # In chunks of at most 131072 cells (about 1M points), so that one device call's host
        # arrays stay small.
        for c0 in range(0, idx.size, 131072):
            sub = idx[c0:c0 + 131072]
            pts = (centers[sub, None, :] + OCTANTS[None, :, :] * half[sub, None, None]).reshape(-1, 3)
            octv[sub] = point_values(pts % 1.0).reshape(sub.size, 8, nv)
            evaluations += pts.shape[0]
        vals = octv[idx]
        fine[idx] = vals.mean(axis=1) * vol[idx, None]
        # Midpoint rules converge as h^2: the fine value's error is |fine - coarse| / 3.
        err[idx] = np.max(np.abs((fine[idx] - coarse[idx])[:, sel]), axis=1) / 3.0
        checked[idx] = True

    while True:
        rounds += 1
        todo = np.where(~checked)[0]
        if proposer is None or todo.size == 0:
            check(todo)
            checked_total += todo.size
        else:
            feats = proposer.features(centers[todo], 2 * half[todo], parent_err[todo],
                                      np.max(np.abs(coarse[todo][:, sel]), axis=1) / vol[todo])
            if not proposer.X:
                # Warm-up labels: a random sample plus the leaves with the largest centre values,
                # so that the first training set contains the cells that matter.
                first = rng.random(todo.size) < warmup_fraction
                mag = np.max(np.abs(coarse[todo][:, sel]), axis=1) / vol[todo]
                first[np.argsort(-mag, kind="stable")[:max(1, int(0.05 * todo.size))]] = True
                check(todo[first])
                checked_total += int(first.sum())
                proposer.observe(feats[first], err[todo[first]])
                proposer.train()
            p = proposer.predict(feats)
            pred[todo] = p * vol[todo] / vol[todo].max()
            value_now = np.where(checked[:, None], fine, coarse).sum(axis=0)
            budget = rtol * _norm(value_now[sel]) / safety
            guard = proposer.must_check
            rest_mask = ~checked[todo]
            rest = todo[rest_mask]
            order = np.argsort(-pred[rest], kind="stable")
            csum = np.cumsum(pred[rest][order][::-1])[::-1]
            must = order[csum > budget * 0.5]
            if guard is not None:
                must = np.union1d(must, np.where(guard[rest_mask])[0])
            audit = rng.random(rest.size) < audit_fraction
            pick = np.zeros(rest.size, dtype=bool)
            pick[must] = True
            pick |= audit
            chosen = rest[pick]
            check(chosen)
            checked_total += chosen.size
            where = np.full(centers.shape[0], -1, dtype=np.int64)
            where[todo] = np.arange(todo.size)
            proposer.observe(feats[where[chosen]], err[chosen])
            aud = rest[audit & ~np.isin(np.arange(rest.size), must)]
            if aud.size:
                # The audit estimates the error mass the network missed among the unchecked leaves
                # (the audited under-prediction scaled by the audit fraction).  If it does not fit
                # the budget, the plain method takes over for the round: every leaf is checked.
                missed = float(np.sum(np.maximum(err[aud] - pred[aud], 0.0))) / audit_fraction
                if missed > 0.5 * budget * safety:
                    fallbacks += 1
                    left = np.where(~checked)[0]
                    check(left)
                    checked_total += left.size
            proposer.train()
        value = np.where(checked[:, None], fine, coarse).sum(axis=0)
        est = np.where(checked, err, np.nan_to_num(pred, nan=0.0))
        total_err = float(est.sum())
        inorm = _norm(value[sel])
        if total_err <= rtol * inorm:
            return AdaptiveResult(value, total_err, evaluations, centers.shape[0], checked_total, rounds, True,
                                  time.perf_counter() - t0, fallbacks)
        splittable = np.where(checked & (level < max_level))[0]
        if splittable.size == 0 or evaluations >= max_evaluations or rounds >= max_rounds:
            return AdaptiveResult(value, total_err, evaluations, centers.shape[0], checked_total, rounds, False,
                                  time.perf_counter() - t0, fallbacks)
        order = splittable[np.argsort(-est[splittable], kind="stable")]
        keep_err = total_err - np.cumsum(est[order])
        nsplit = int(np.searchsorted(-keep_err, -0.5 * rtol * inorm)) + 1
        if centers.shape[0] + 7 * min(nsplit, order.size) > max_leaves:
            return AdaptiveResult(value, total_err, evaluations, centers.shape[0], checked_total, rounds, False,
                                  time.perf_counter() - t0, fallbacks)
        split = order[:min(nsplit, order.size)]
        # Children: octant centres of each split cell, coarse values from the parent's octants.
        ch_c = (centers[split, None, :] + OCTANTS[None, :, :] * half[split, None, None]).reshape(-1, 3)
        ch_h = np.repeat(half[split] / 2, 8)
        ch_l = np.repeat(level[split] + 1, 8)
        ch_v = octv[split].reshape(-1, nv) * ((2 * ch_h) ** 3)[:, None]
        ch_pe = np.repeat(err[split] / 8.0, 8)
        keep = np.ones(centers.shape[0], dtype=bool)
        keep[split] = False
        centers = np.concatenate([centers[keep], ch_c])
        half = np.concatenate([half[keep], ch_h])
        level = np.concatenate([level[keep], ch_l])
        vol = (2 * half) ** 3
        coarse = np.concatenate([coarse[keep], ch_v])
        fine = np.concatenate([fine[keep], np.zeros_like(ch_v)])
        octv = np.concatenate([octv[keep], np.zeros((ch_c.shape[0], 8, nv), dtype=coarse.dtype)])
        err = np.concatenate([err[keep], np.full(ch_c.shape[0], np.nan)])
        pred = np.concatenate([pred[keep], np.full(ch_c.shape[0], np.nan)])
        checked = np.concatenate([checked[keep], np.zeros(ch_c.shape[0], dtype=bool)])
        parent_err = np.concatenate([parent_err[keep], ch_pe])
