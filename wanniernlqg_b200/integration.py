"""Uniform and h-adaptive integration of response integrands over a k-space box.

Public types mirror the reference (src/Runtime/IntegrationAlgorithms.jl:30-114,
src/Runtime/Execution/ResponseIntegration.jl:100-198):

* ``IntegrationDomain(lower, upper, coordinates)``
* ``HAdaptiveCubature(atol, rtol, max_evaluations, initial_divisions)``
* ``UniformIntegration()``
* ``integrate_response(evaluator, domain, algorithm, normalization=..., batch_evaluator=...)``

The adaptive controller follows HCubature 1.8.0 as the reference runs it
(ResponseCubatureTree.jl:24-103): a max-heap of boxes keyed by their error estimate, the
worst box split in half along the rule's ``kdiv`` axis, running sums I and E updated by the two
halves, stop when E <= max(rtol*||I||, atol) or when the evaluation budget is spent, and the
final value re-summed over the heap.  The norm is the maximum absolute complex entry
(ResponseIntegration.jl:57-59).  The box rule is the Genz-Malik degree-7 rule with its
embedded degree-5 estimate in 2D and 3D (A. C. Genz and A. A. Malik, J. Comput. Appl. Math. 6
(1980) 295-302) and the 7/15-point Gauss-Kronrod pair in 1D, written here from the published
rules (HCubature itself is not part of this repository).

``integrate_response_batched`` is the GPU-oriented variant: it splits the ``boxes_per_step``
worst boxes per step so that one device call evaluates 2*K*(rule nodes) points; it converges to
the same tolerance with a different box order.
"""
from __future__ import annotations

import dataclasses
import heapq
import itertools
import math
import warnings
from typing import Callable, Optional, Sequence, Tuple

import numpy as np


@dataclasses.dataclass(frozen=True)
class IntegrationDomain:
    lower: Tuple[float, ...] = (0.0, 0.0)
    upper: Tuple[float, ...] = (1.0, 1.0)
    coordinates: str = "fractional"

    def __post_init__(self):
        lo = tuple(float(x) for x in self.lower)
        hi = tuple(float(x) for x in self.upper)
        if len(lo) != len(hi):
            raise ValueError("matching integration bounds required")  # DimensionMismatch in the reference
        if not 1 <= len(lo) <= 3:
            raise ValueError("integration dimension must be one, two or three")
        if not all(math.isfinite(x) for x in lo + hi) or not all(a < b for a, b in zip(lo, hi)):
            raise ValueError("finite ordered integration bounds required")
        measure = math.prod(b - a for a, b in zip(lo, hi))
        if not (math.isfinite(measure) and measure > 0):
            raise ValueError("integration measure must be positive and representable in Float64")
        if self.coordinates not in ("fractional", "cartesian"):
            raise ValueError("unknown integration coordinates")
        object.__setattr__(self, "lower", lo)
        object.__setattr__(self, "upper", hi)

    @property
    def dimension(self) -> int:
        return len(self.lower)

    @property
    def measure(self) -> float:
        return math.prod(b - a for a, b in zip(self.lower, self.upper))


@dataclasses.dataclass(frozen=True)
class HAdaptiveCubature:
    atol: float = 1e-8
    rtol: float = 1e-5
    max_evaluations: int = 100_000
    initial_divisions: int = 1

    def __post_init__(self):
        for x in (self.atol, self.rtol):
            if not (isinstance(x, (int, float)) and math.isfinite(x) and x >= 0):
                raise ValueError("finite nonnegative atol/rtol with at least one positive value required")
        if not (self.atol > 0 or self.rtol > 0):
            raise ValueError("finite nonnegative atol/rtol with at least one positive value required")
        if not (isinstance(self.initial_divisions, int) and not isinstance(self.initial_divisions, bool)
                and self.initial_divisions > 0):
            raise ValueError("initial_divisions must be positive")
        if not (isinstance(self.max_evaluations, int) and not isinstance(self.max_evaluations, bool)
                and self.max_evaluations > 0):
            raise ValueError("max_evaluations must be positive")


@dataclasses.dataclass(frozen=True)
class UniformIntegration:
    region_quadrature: str = "midpoint"


@dataclasses.dataclass
class ResponseIntegralResult:
    value: np.ndarray
    embedded_estimate: Optional[float]
    evaluations: int
    termination: str
    estimate_converged: Optional[bool]
    domain_measure: float
    normalization: str


def integration_norm(x) -> float:
    """Maximum absolute complex entry (ResponseIntegration.jl:57-59)."""
    a = np.asarray(x)
    return float(np.max(np.abs(a))) if a.size else 0.0


def integration_rule_nodes(dimension: int) -> int:
    """15 (Gauss-Kronrod) in 1D, 1 + 4D + 2D(D-1) + 2^D (Genz-Malik) in 2D/3D."""
    return 15 if dimension == 1 else 1 + 4 * dimension + 2 * dimension * (dimension - 1) + 2 ** dimension


# ---------------------------------------------------------------------------------------------
# Box rules.  A rule maps (a, b) to node coordinates; values at those nodes give (I, E, kdiv).
# ---------------------------------------------------------------------------------------------
class GenzMalikRule:
    """Genz-Malik degree-7 rule with embedded degree-5 estimate for an n-cube, n >= 2.

    Generators (in units of the half-widths): the centre; +-l2 e_i; +-l3 e_i; +-l4 e_i +- l4 e_j
    (i < j); all sign combinations of l5.  l2 = sqrt(9/70), l3 = l4 = sqrt(9/10),
    l5 = sqrt(9/19).  Weights per point, normalised so that the degree-0 sum is 1:
      degree 7: (12824 - 9120n + 400n^2)/19683, 980/6561, (1820 - 400n)/19683, 200/19683, 6859/19683/2^n
      degree 5: (729 - 950n + 50n^2)/729, 245/486, (265 - 100n)/1458, 25/729
    The split axis is the one with the largest fourth divided difference
    |f(+l3)+f(-l3) + 12 f(c) - 7 (f(+l2)+f(-l2))| (7 = (l3/l2)^2).
    """

    def __init__(self, n: int):
        if n < 2:
            raise ValueError("Genz-Malik rule needs n >= 2")
        self.n = n
        l2, l3, l4, l5 = math.sqrt(9 / 70), math.sqrt(9 / 10), math.sqrt(9 / 10), math.sqrt(9 / 19)
        pts = [np.zeros(n)]
        self.idx2 = []
        self.idx3 = []
        for i in range(n):
            e = np.zeros(n)
            e[i] = l2
            self.idx2.append((len(pts), len(pts) + 1))
            pts += [e.copy(), -e]
            e = np.zeros(n)
            e[i] = l3
            self.idx3.append((len(pts), len(pts) + 1))
            pts += [e.copy(), -e]
        start4 = len(pts)
        for i, j in itertools.combinations(range(n), 2):
            for si, sj in itertools.product((1.0, -1.0), repeat=2):
                e = np.zeros(n)
                e[i] = si * l4
                e[j] = sj * l4
                pts.append(e)
        start5 = len(pts)
        for signs in itertools.product((1.0, -1.0), repeat=n):
            pts.append(l5 * np.array(signs))
        self.points = np.array(pts)
        npts = len(pts)
        w7 = np.zeros(npts)
        w5 = np.zeros(npts)
        w7[0] = (12824 - 9120 * n + 400 * n * n) / 19683
        w5[0] = (729 - 950 * n + 50 * n * n) / 729
        for (p, q) in self.idx2:
            w7[[p, q]] = 980 / 6561
            w5[[p, q]] = 245 / 486
        for (p, q) in self.idx3:
            w7[[p, q]] = (1820 - 400 * n) / 19683
            w5[[p, q]] = (265 - 100 * n) / 1458
        w7[start4:start5] = 200 / 19683
        w5[start4:start5] = 25 / 729
        w7[start5:] = 6859 / 19683 / 2 ** n
        self.w7 = w7
        self.w5 = w5

    def nodes(self, a: np.ndarray, b: np.ndarray) -> np.ndarray:
        c = 0.5 * (a + b)
        h = 0.5 * (b - a)
        return c + self.points * h

    def combine(self, a, b, values: np.ndarray):
        """values [npts, ...] -> (I, E, kdiv) (kdiv 0-based)."""
        vol = float(np.prod(b - a))
        flat = values.reshape(values.shape[0], -1)
        I = vol * (self.w7 @ flat)
        I5 = vol * (self.w5 @ flat)
        E = integration_norm(I - I5)
        f1 = flat[0]
        kdiv, best = 0, -1.0
        divs = []
        for i in range(self.n):
            p2, q2 = self.idx2[i]
            p3, q3 = self.idx3[i]
            d = integration_norm(flat[p3] + flat[q3] + 12.0 * f1 - 7.0 * (flat[p2] + flat[q2]))
            divs.append(d)
            if d > best:
                kdiv, best = i, d
        # Equal fourth differences (common for symmetric integrands): split the widest edge.
        if self.n > 1 and all(d == best for d in divs):
            kdiv = int(np.argmax(b - a))
        shape = values.shape[1:]
        return I.reshape(shape), E, kdiv


class GaussKronrod15:
    """7/15-point Gauss-Kronrod pair on [a, b] (published abscissae and weights)."""

    XGK = np.array([0.991455371120812639206854697526329, 0.949107912342758524526189684047851,
                    0.864864423359769072789712788640926, 0.741531185599394439863864773280788,
                    0.586087235467691130294144845693013, 0.405845151377397166906606412076961,
                    0.207784955007898467600689403773245, 0.0])
    WGK = np.array([0.022935322010529224963732008058970, 0.063092092629978553290700663189204,
                    0.104790010322250183839876322541518, 0.140653259715525918745189590510238,
                    0.169004726639267902826583426598550, 0.190350578064785409913256402421014,
                    0.204432940075298892414161999234649, 0.209482141084727828012999174891714])
    WG = np.array([0.129484966168869693270611432679082, 0.279705391489276667901467771423780,
                   0.381830050505118944950369775488975, 0.417959183673469387755102040816327])

    def __init__(self):
        x = np.concatenate([-self.XGK[:-1], self.XGK[::-1]])   # ascending, 15 points
        self.points = x[:, None]
        wk = np.concatenate([self.WGK[:-1], self.WGK[::-1]])
        wg = np.zeros(15)
        # Gauss nodes are the odd-indexed Kronrod nodes (1, 3, 5 of XGK and the centre).
        for j, k in enumerate((1, 3, 5)):
            wg[k] = self.WG[j]
            wg[14 - k] = self.WG[j]
        wg[7] = self.WG[3]
        self.wk = wk
        self.wg = wg
        self.n = 1

    def nodes(self, a, b):
        c = 0.5 * (a + b)
        h = 0.5 * (b - a)
        return c + self.points * h

    def combine(self, a, b, values):
        h = 0.5 * float(b[0] - a[0])
        flat = values.reshape(values.shape[0], -1)
        I = h * (self.wk @ flat)
        Ig = h * (self.wg @ flat)
        return I.reshape(values.shape[1:]), integration_norm(I - Ig), 0


def box_rule(dimension: int):
    return GaussKronrod15() if dimension == 1 else GenzMalikRule(dimension)


# ---------------------------------------------------------------------------------------------
# Controllers.
# ---------------------------------------------------------------------------------------------
def _normalization(domain: IntegrationDomain, normalization: str):
    measure = domain.measure
    if normalization == "domain_average":
        return measure, 1.0 / measure
    if normalization == "integral":
        return measure, 1.0
    raise ValueError("normalization must be 'domain_average' or 'integral'")


def validate_integration_budget(domain: IntegrationDomain, algorithm: HAdaptiveCubature) -> None:
    nodes = integration_rule_nodes(domain.dimension) * algorithm.initial_divisions ** domain.dimension
    if nodes > algorithm.max_evaluations:
        raise ValueError(f"cubature budget cannot cover the initial {domain.dimension}-dimensional divisions: "
                         f"at least {nodes} nodes required")


class _Evaluator:
    """Owns the value shape check, the scale and the evaluation count."""

    def __init__(self, evaluator, batch_evaluator, scale):
        self.evaluator = evaluator
        self.batch = batch_evaluator
        self.scale = scale
        self.shape = None
        self.count = 0

    def __call__(self, nodes: np.ndarray) -> np.ndarray:
        if self.batch is not None:
            vals = np.asarray(self.batch(nodes))
            if vals.shape[0] != nodes.shape[0]:
                raise ValueError("incomplete cubature node batch")
        else:
            vals = np.stack([np.asarray(self.evaluator(tuple(x)), dtype=np.complex128).copy() for x in nodes])
        vals = np.asarray(vals, dtype=np.complex128)
        if self.shape is None:
            self.shape = vals.shape[1:]
        elif vals.shape[1:] != self.shape:
            raise ValueError("DimensionMismatch: evaluator value shape changed")
        if not np.all(np.isfinite(vals)):
            raise ValueError("nonfinite integrand value")
        self.count += nodes.shape[0]
        return self.scale * vals


def _initial_boxes(domain, algorithm):
    a = np.array(domain.lower)
    b = np.array(domain.upper)
    d = domain.dimension
    n0 = algorithm.initial_divisions
    delta = (b - a) / n0
    boxes = []
    for c in itertools.product(range(n0), repeat=d):
        # CartesianIndices order: first index fastest.
        c = tuple(reversed(c))
        lo = np.array([a[i] + c[i] * delta[i] for i in range(d)])
        hi = np.array([b[i] if c[i] == n0 - 1 else a[i] + (c[i] + 1) * delta[i] for i in range(d)])
        boxes.append((lo, hi))
    return boxes


def integrate_response(evaluator, domain: IntegrationDomain, algorithm, *, normalization: str = "domain_average",
                       batch_evaluator=None, k_mesh: Optional[Sequence[int]] = None) -> ResponseIntegralResult:
    """Integrate `evaluator(node) -> array` (or `batch_evaluator(nodes[n, d]) -> [n, ...]`)."""
    measure, scale = _normalization(domain, normalization)
    ev = _Evaluator(evaluator, batch_evaluator, scale)
    if isinstance(algorithm, UniformIntegration):
        d = domain.dimension
        mesh = tuple(k_mesh) if k_mesh is not None else (16,) * d
        if len(mesh) != d or any(int(m) <= 0 for m in mesh):
            raise ValueError("positive midpoint counts matching domain dimension required")
        idx = np.array(list(itertools.product(*[range(m) for m in reversed(mesh)])))[:, ::-1]
        lo = np.array(domain.lower)
        hi = np.array(domain.upper)
        if algorithm.region_quadrature == "left_endpoint":
            nodes = lo + (idx / np.array(mesh)) * (hi - lo)
        else:
            nodes = lo + (idx + 0.5) * (hi - lo) / np.array(mesh)
        vals = ev(nodes) / scale
        value = vals.sum(axis=0) * (measure * scale / math.prod(mesh))
        if not math.isfinite(integration_norm(value)):
            raise ValueError("nonfinite uniform integration result")
        return ResponseIntegralResult(value, None, ev.count, "fixed_rule", None, measure, normalization)
    if not isinstance(algorithm, HAdaptiveCubature):
        raise TypeError("unknown integration algorithm")
    validate_integration_budget(domain, algorithm)
    rule = box_rule(domain.dimension)
    atol = algorithm.atol
    rtol = algorithm.rtol
    maxevals = algorithm.max_evaluations
    per_box = integration_rule_nodes(domain.dimension)

    def apply(lo, hi):
        return rule.combine(lo, hi, ev(rule.nodes(lo, hi)))

    heap = []          # (-E, sequence, lo, hi, I, E, kdiv)
    seq = itertools.count()
    I = None
    E = 0.0
    numevals = 0
    for lo, hi in _initial_boxes(domain, algorithm):
        Ib, Eb, kd = apply(lo, hi)
        I = Ib.copy() if I is None else I + Ib
        E += Eb
        numevals += per_box
        heapq.heappush(heap, (-Eb, next(seq), lo, hi, Ib, Eb, kd))
    if not (E <= max(rtol * integration_norm(I), atol) or numevals >= maxevals):
        while True:
            _, _, lo, hi, Ib, Eb, kd = heapq.heappop(heap)
            w = 0.5 * (hi[kd] - lo[kd])
            a1 = lo.copy()
            a1[kd] += w
            b2 = hi.copy()
            b2[kd] -= w
            I1, E1, k1 = apply(a1, hi)
            I2, E2, k2 = apply(lo, b2)
            heapq.heappush(heap, (-E1, next(seq), a1, hi, I1, E1, k1))
            heapq.heappush(heap, (-E2, next(seq), lo, b2, I2, E2, k2))
            I = I + I1 + I2 - Ib
            E = E + E1 + E2 - Eb
            numevals += 2 * per_box
            inorm = integration_norm(I)
            if E <= max(rtol * inorm, atol) or numevals >= maxevals or not math.isfinite(inorm):
                break
        I = sum(h[4] for h in heap)
        E = sum(h[5] for h in heap)
    return _finish(I, E, ev.count, algorithm, measure, normalization)


def _finish(I, E, count, algorithm, measure, normalization):
    if not (math.isfinite(E) and math.isfinite(integration_norm(I))):
        raise ValueError("nonfinite cubature result")
    converged = E <= max(algorithm.atol, algorithm.rtol * integration_norm(I))
    if not converged:
        warnings.warn("Adaptive integral stopped before its embedded estimate met the requested tolerance; "
                      "result retained")
    return ResponseIntegralResult(np.asarray(I), float(E), count,
                                  "estimated_tolerance" if converged else "evaluation_budget",
                                  converged, measure, normalization)


def integrate_response_batched(batch_evaluator, domain: IntegrationDomain, algorithm: HAdaptiveCubature, *,
                               normalization: str = "domain_average", boxes_per_step: int = 256,
                               select: Optional[Callable] = None) -> ResponseIntegralResult:
    """Batched h-adaptive cubature: each step splits the `boxes_per_step` boxes with the largest
    error estimates (or the boxes `select(boxes)` returns) and evaluates all their children's rule
    nodes in one `batch_evaluator` call.  Same rule, norm and stopping test as the serial
    controller."""
    validate_integration_budget(domain, algorithm)
    measure, scale = _normalization(domain, normalization)
    ev = _Evaluator(None, batch_evaluator, scale)
    rule = box_rule(domain.dimension)
    npts = integration_rule_nodes(domain.dimension)

    def apply_many(boxes):
        nodes = np.concatenate([rule.nodes(lo, hi) for lo, hi in boxes])
        vals = ev(nodes)
        out = []
        for i, (lo, hi) in enumerate(boxes):
            out.append(rule.combine(lo, hi, vals[i * npts:(i + 1) * npts]))
        return out

    boxes = _initial_boxes(domain, algorithm)
    res = apply_many(boxes)
    live = [(lo, hi, I, E, k) for (lo, hi), (I, E, k) in zip(boxes, res)]
    numevals = npts * len(live)
    while True:
        I = sum(b[2] for b in live)
        E = sum(b[3] for b in live)
        inorm = integration_norm(I)
        if E <= max(algorithm.rtol * inorm, algorithm.atol) or numevals >= algorithm.max_evaluations \
                or not math.isfinite(inorm):
            break
        budget_boxes = max(1, (algorithm.max_evaluations - numevals) // (2 * npts))
        kmax = min(boxes_per_step, budget_boxes, len(live))
        if select is not None:
            chosen = select(live, kmax)
        else:
            chosen = list(np.argsort([-b[3] for b in live], kind="stable")[:kmax])
        chosen_set = set(int(c) for c in chosen)
        children = []
        for c in chosen:
            lo, hi, _, _, kd = live[int(c)]
            w = 0.5 * (hi[kd] - lo[kd])
            a1 = lo.copy()
            a1[kd] += w
            b2 = hi.copy()
            b2[kd] -= w
            children += [(a1, hi), (lo, b2)]
        res = apply_many(children)
        live = [b for i, b in enumerate(live) if i not in chosen_set]
        live += [(lo, hi, I_, E_, k_) for (lo, hi), (I_, E_, k_) in zip(children, res)]
        numevals += npts * len(children)
    return _finish(I, E, ev.count, algorithm, measure, normalization)
