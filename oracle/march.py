"""The steppers, restated: exponential Adams and the embedded Runge-Kutta pair.

Test infrastructure (see the package docstring).  The state-sized arithmetic follows
``backends/numpy_ref/adams_kernels.py:404-741`` and ``backends/numpy_ref/engines.py:
97-198``; the coefficient tables ``backends/numpy_ref/adams_tables.py:37-176`` and
``stepper/multistep.py`` (``_basis_rows``); the phi functions
``backends/exponential.py:131-224``; the decisions ``backends/adams_core.py:93-531``,
``backends/numpy_ref/marches/adams.py:318-727``, ``backends/rk_core.py:37-166``,
``backends/numpy_ref/marches/runge_kutta.py:125-250``, ``stepper/schedule.py:959-1090``
and ``stepper/controller.py:162-209,473-676``.  Policies are plain dicts with the
fields of the reference's ``MarchPolicy`` / ``RungeKuttaPolicy``.
"""

from __future__ import annotations

import bisect
import math

import numpy as np

from oracle.source import combine, lab_source, stage_scalars

LANDING_ULPS = 8
START_GROWTH = 100.0
PHI_JOIN = 3.0
_SERIES_TERMS = 24

DOPRI5_NODES = np.array([0.0, 1 / 5, 3 / 10, 4 / 5, 8 / 9, 1.0, 1.0])
DOPRI5_MATRIX = np.array([
    [0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0],
    [1 / 5, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0],
    [3 / 40, 9 / 40, 0.0, 0.0, 0.0, 0.0, 0.0],
    [44 / 45, -56 / 15, 32 / 9, 0.0, 0.0, 0.0, 0.0],
    [19372 / 6561, -25360 / 2187, 64448 / 6561, -212 / 729, 0.0, 0.0, 0.0],
    [9017 / 3168, -355 / 33, 46732 / 5247, 49 / 176, -5103 / 18656, 0.0, 0.0],
    [35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84, 0.0],
])
DOPRI5_SOLUTION = np.array([35 / 384, 0.0, 500 / 1113, 125 / 192, -2187 / 6784, 11 / 84, 0.0])
DOPRI5_EMBEDDED = np.array([5179 / 57600, 0.0, 7571 / 16695, 393 / 640, -92097 / 339200,
                            187 / 2100, 1 / 40])
DOPRI5_ERROR = DOPRI5_SOLUTION - DOPRI5_EMBEDDED


# ---------------------------------------------------------------- coefficient tables
def basis_rows(points, upper: float, integrate: bool):
    """``stepper/multistep.py`` ``_basis_rows``: Lagrange basis from its own roots."""
    points = np.asarray(points, dtype=np.float64)
    n = points.shape[0]
    rows = np.zeros((n, n))
    weights = np.empty(n)
    coefficients = np.empty(n)
    product = np.empty(n)
    for index in range(n):
        node = points[index]
        length = 1
        coefficients[0] = 1.0
        denominator = 1.0
        for other in range(n):
            if other == index:
                continue
            root = points[other]
            product[0] = 0.0
            for power in range(length):
                product[power + 1] = coefficients[power]
            for power in range(length):
                product[power] -= root * coefficients[power]
            length += 1
            for power in range(length):
                coefficients[power] = product[power]
            denominator *= node - root
        if integrate:
            integral = 0.0
            for power in range(length - 1, -1, -1):
                integral = (integral + coefficients[power] / (power + 1)) * upper
            weights[index] = integral / denominator
        else:
            for power in range(length):
                rows[index, power] = coefficients[power] / denominator
    return rows, weights


def lagrange_coefficients(nodes) -> np.ndarray:
    return basis_rows(nodes, 1.0, False)[0]


def integrated_weights(nodes) -> np.ndarray:
    return basis_rows(nodes, 1.0, True)[1]


def exponential_corrector(nodes, order: int, width: int) -> np.ndarray:
    """``adams_tables.py:109-135``."""
    corrector = np.zeros((width, width))
    corrector[: order + 1, : order + 1] = lagrange_coefficients([1.0, *nodes[:order]])
    return corrector


def exponential_rows(nodes, orders, width: int) -> np.ndarray:
    """``adams_tables.py:138-173``: each order's corrector less its predictor."""
    rows = np.zeros((len(orders), width, width))
    for index, order in enumerate(orders):
        stencil = nodes[:order]
        rows[index, : order + 1, : order + 1] = lagrange_coefficients([1.0, *stencil])
        rows[index, 1: order + 1, :order] -= lagrange_coefficients(stencil)
    return rows


# ---------------------------------------------------------------- phi functions
_RECIP_FACT = tuple(1.0 / math.factorial(k) for k in range(16))


def phi_functions(x, order: int) -> np.ndarray:
    """``backends/exponential.py:131-224``: upward recurrence far, scaled series near."""
    values = np.asarray(x, dtype=np.complex128)
    flat = values.reshape(-1)
    out = np.empty((order + 1, flat.size), dtype=np.complex128)
    far = np.abs(flat) > PHI_JOIN
    if np.any(far):
        xf = flat[far]
        o = np.empty((order + 1, xf.size), dtype=np.complex128)
        o[0] = np.exp(xf)
        for k in range(1, order + 1):
            o[k] = (o[k - 1] - _RECIP_FACT[k - 1]) / xf
        out[:, far] = o
    if not np.all(far):
        xn = flat[~far]
        mag = np.abs(xn)
        sq = np.where(mag > 0.5, np.ceil(np.log2(np.maximum(mag, 0.5) / 0.5)), 0.0).astype(np.int64)
        y = xn / np.exp2(sq)
        o = np.empty((order + 1, xn.size), dtype=np.complex128)
        term = np.full(xn.size, _RECIP_FACT[order], dtype=np.complex128)
        total = term.copy()
        for m in range(1, _SERIES_TERMS):
            term = term * y / (m + order)
            total = total + term
        o[order] = total
        for k in range(order - 1, 0, -1):
            o[k] = _RECIP_FACT[k] + y * o[k + 1]
        o[0] = np.exp(y)
        for level in range(int(sq.max(initial=0))):
            active = sq > level
            old = o[:, active]
            doubled = np.empty_like(old)
            doubled[0] = old[0] * old[0]
            for k in range(1, order + 1):
                t = old[0] * old[k]
                for j in range(1, k + 1):
                    t = t + old[j] * _RECIP_FACT[k - j]
                doubled[k] = t / 2.0 ** k
            o[:, active] = doubled
        out[:, ~far] = o
    return out.reshape((order + 1, *values.shape))


def moments(exponent: np.ndarray, count: int) -> np.ndarray:
    """``adams_kernels.py:423-447``: ``M_k = k! phi_{k+1}(x)`` for ``k < count``."""
    phi = phi_functions(exponent, count)
    factors = np.array([math.factorial(k) for k in range(count)], dtype=np.float64)
    return phi[1:] * factors.reshape((count, *([1] * exponent.ndim)))


def apply(mom: np.ndarray, coefficients: np.ndarray, values, dz: float) -> np.ndarray:
    """``adams_kernels.py:555-586``: ``dz sum_k M_k (sum_j c_jk X_j)``."""
    total = np.zeros_like(values[0])
    for k in range(coefficients.shape[1]):
        combined = np.zeros_like(values[0])
        for weight, value in zip(coefficients[:, k], values):
            if weight != 0.0:
                combined = combined + float(weight) * value
        total = total + mom[k] * combined
    return dz * total


# ---------------------------------------------------------------- the workspace
class Workspace:
    """The state, its finish (hard mask) and the norm mask (``workspace.py:425-1070``)."""

    def __init__(self, rec, state=None):
        self.rec = rec
        self.state = np.array(rec.launch_field() if state is None else state, dtype=np.complex128)
        self.state = self.mask(self.state)
        self.evaluations = 0

    def mask(self, state):
        return state * self.rec.active_mask

    def source(self, lab, z):
        self.evaluations += 1
        return lab_source(self.rec, lab, z)

    def delta_phi(self, z0, z1):
        rec = self.rec
        return combine(rec.phi_delta_weights(z0, z1), rec.phi_terms)

    def rate(self, z, before=False):
        rec = self.rec
        return combine(rec.phi_rate_weights(z, before), rec.phi_terms)


# ---------------------------------------------------------------- Adams engine
class AdamsEngine:
    """``multistep.py:806-1070`` (``ExponentialHistory``) on the oracle workspace."""

    def __init__(self, ws: Workspace, policy: dict):
        self.ws = ws
        self.policy = policy
        self.n_slots = policy["order"] + 2
        self.compensated = ws.rec.phi_representation == "expansion"
        shape = ws.state.shape
        self.store = np.zeros((self.n_slots, *shape), dtype=np.complex128)
        self.states = np.zeros_like(self.store) if self.compensated else None
        self.rates = np.zeros_like(self.store) if self.compensated else None
        self.held = None

    def start(self, z):
        state = self.ws.state
        self.store[0] = self.ws.source(state, z)
        if self.compensated:
            self.states[0] = state
            self.rates[0] = self.ws.rate(z)

    def _carried(self, exponent, dz, slots, nodes):
        reference = exponent / dz
        return [np.exp((1.0 - node) * exponent) * ((self.rates[slot] - reference) * self.states[slot])
                for slot, node in zip(slots, nodes)]

    def trial(self, z, dz, nodes, slots, order, orders):
        ws, rec = self.ws, self.ws.rec
        state = ws.state
        width = 1 + max(orders)
        exponent = ws.delta_phi(z, z + dz)
        mom = moments(exponent, width)
        flow = np.exp(exponent)
        rows_read = list(slots[: width - 1])
        values = [self.store[s] for s in rows_read]
        lab = flow * state + apply(mom, lagrange_coefficients(nodes[:order]), values[:order], dz)
        carried = None
        if self.compensated:
            carried = self._carried(exponent, dz, rows_read, nodes[: len(rows_read)])

            def comp_sum(ns, first, count):
                w = integrated_weights(ns)
                total = np.tensordot(w[len(ns) - count:], np.array(carried[:count]), axes=1)
                if first is not None:
                    total = total + w[0] * first
                return dz * total

            lab = lab + comp_sum(list(nodes[:order]), None, order)
        source = ws.source(lab, z + dz)
        corrector = exponential_corrector(nodes, order, width)
        defect_rows = exponential_rows(nodes, orders, width)
        xs = [source, *values]
        advanced = flow * state + apply(mom, corrector, xs, dz)
        extra = None
        endpoint_rate = None
        if self.compensated:
            endpoint_rate = ws.rate(z + dz, before=True)
            endpoint = (endpoint_rate - exponent / dz) * lab

            def corr(k):
                return comp_sum([1.0, *nodes[:k]], endpoint, k)

            def pred(k):
                return comp_sum(list(nodes[:k]), None, k)

            advanced = advanced + corr(order)
            extra = [corr(k) - pred(k) for k in orders]
        mask = rec.norm_mask
        magnitude = float(np.linalg.norm(state[..., mask]))
        scale = self.policy["rtol"] * magnitude + self.policy["atol"]
        norms = np.empty(len(orders))
        for i, row in enumerate(defect_rows):
            defect = apply(mom, row, xs, dz)
            if extra is not None:
                defect = defect + extra[i]
            norms[i] = float(np.linalg.norm(defect[..., mask] / scale))
        self.held = dict(advanced=advanced, source=source, lab=lab, rate=endpoint_rate)
        return norms

    def accept(self, free):
        held, self.held = self.held, None
        self.ws.state = self.ws.mask(held["advanced"])
        self.store[free] = held["source"]
        if self.compensated:
            self.states[free] = held["lab"]
            self.rates[free] = held["rate"]


# ---------------------------------------------------------------- landing rule
def _landing(z, dz, planes, kinks, edges, dz_max, z_end, stretch):
    """``stepper/schedule.py:959-1066``: caps, then the nearest landing."""
    tol = LANDING_ULPS * math.ulp(max(abs(z), abs(z_end)))
    index = min(max(bisect.bisect_right(edges, z) - 1, 0), len(edges) - 2)
    width = edges[index + 1] - edges[index]
    order = {"none": 0, "max_step": 1, "interval_width": 2, "hard_kink": 3, "save_plane": 4, "end": 5}
    caps = [(dz, "none"), (dz_max, "max_step"), (width, "interval_width")]
    landings = []
    for kind, positions in (("hard_kink", kinks), ("save_plane", planes), ("end", (z_end,))):
        found = bisect.bisect_left(positions, z + tol)
        if found < len(positions):
            landings.append((positions[found] - z, kind, positions[found]))
    cap_dz, cap_kind = min(caps, key=lambda b: (b[0], -order[b[1]]))
    gap, kind, ahead = min(landings, key=lambda b: (b[0], -order[b[1]]))
    if gap <= cap_dz:
        return gap, kind, ahead
    if gap <= min(stretch * cap_dz, dz_max):
        return gap, kind, ahead
    return cap_dz, cap_kind, None


def reached(position, target):
    return position >= target - LANDING_ULPS * math.ulp(max(abs(position), abs(target)))


def limit_step(dz, factor, dz_min, dz_max):
    proposed = min(dz * factor, dz_max)
    if proposed < dz_min:
        raise RuntimeError(f"step control asked for {proposed:.3e} m, below dz_min {dz_min:.3e}")
    return proposed


# ---------------------------------------------------------------- Adams march
class AdamsMarch:
    """``marches/adams.py:79-727`` with ``adams_core``'s decisions."""

    def __init__(self, engine: AdamsEngine, policy: dict, proposal: float):
        self.engine = engine
        self.p = policy
        self.z = 0.0
        self.proposal = proposal
        self.history = []  # (z, row), oldest first
        self.rejections = 0
        self.last_rejected = False
        self.order = 1 if policy["variable_order"] else policy["order"]
        self.attempts = 0
        self.rejected = 0
        self.log = []

    def _start(self):
        self.engine.start(self.z)
        self.history = [(self.z, 0)]
        self.order = 1 if self.p["variable_order"] else self.p["order"]

    def _stencil(self, dz):
        p = self.p
        recent = self.history[::-1]
        nodes = [(zz - self.z) / dz for zz, _ in recent]
        slots = [row for _, row in recent]
        held = len(recent)
        order = min(self.order, held)
        rising = not self.last_rejected and held > order
        orders = [order]
        if p["variable_order"]:
            orders += [o for o in (order - 1, order + 1)
                       if 1 <= o <= p["order"] and o <= held and (o < order or rising)]
        return nodes, slots, order, orders

    def _factor(self, norm, order, growth):
        if norm <= 0.0:
            return growth
        raw = self.p["safety"] * norm ** (-1.0 / (order + 1))
        return min(growth, max(self.p["min_factor"], raw))

    def _order_weight(self, norm, order, dz):
        p = self.p
        rate = math.inf if norm <= 0.0 else norm ** (-1.0 / (order + 1))
        allowed = p["safety"] * rate
        stable = math.inf
        if p["collar_rate"] > 0.0:
            stable = p["collar_stability"] * p["real_intervals"][order - 1] / (p["collar_rate"] * dz)
        return min(allowed, stable)

    def _choose_order(self, current, scores, dz):
        p = self.p
        if not p["variable_order"]:
            return p["order"], current, scores[current]
        weights = {o: self._order_weight(n, o, dz) for o, n in scores.items()}
        best = max(scores, key=weights.__getitem__)
        if best != current and weights[best] > p["hysteresis"] * weights[current]:
            return best, best, scores[best]
        return current, current, scores[current]

    def _attempt(self, dz, end, kink, fixed=False):
        p = self.p
        nodes, slots, order, orders = self._stencil(dz)
        norms = self.engine.trial(self.z, dz, nodes, slots, order, orders)
        self.attempts += 1
        norm = float(norms[0])
        self.log.append((self.z, dz, norm, order))
        if not norm <= 1.0 and not (fixed and math.isfinite(norm)):
            self.rejected += 1
            self.last_rejected = True
            count = self.rejections + 1
            restart = count >= p["restart_after"] and len(self.history) > 1
            scale = p["min_factor"] if not math.isfinite(norm) else self._factor(
                norm, order, p["rejection_growth"])
            self.rejections = 0 if restart else count
            if restart:
                self.history = []
            self.proposal = limit_step(dz, scale, p["dz_min"], p["dz_max"])
            return False, norm
        keep = self.history[-p["order"]:] if p["order"] else []
        used = {row for _, row in keep}
        free = next(s for s in range(self.engine.n_slots) if s not in used)
        self.engine.accept(free)
        self.history = [*keep, (self.z + dz, free)]
        self.rejections = 0
        stored, control, cnorm = self._choose_order(order, dict(zip(orders, norms.tolist())), dz)
        self.order = stored
        self.last_rejected = False
        self.z = end
        if kink:
            self.history = []
        self.proposal = limit_step(dz, self._factor(cnorm, control, p["max_growth"]),
                                   p["dz_min"], p["dz_max"])
        return True, norm

    def _approach(self, stop, planes, kinks, target):
        p = self.p
        dz, kind, z_target = stop
        if z_target is None and p["equal_approach"]:
            tol = LANDING_ULPS * math.ulp(max(abs(self.z), abs(target)))
            cands = [target]
            for positions in (planes, kinks):
                i = bisect.bisect_right(positions, self.z + tol)
                if i < len(positions):
                    cands.append(positions[i])
            nearest = min(cands)
            ahead = nearest if nearest > self.z + tol else None
            if ahead is not None and dz < ahead - self.z < 2.0 * dz:
                half = 0.5 * (ahead - self.z)
                return half, self.z + half, False
        end = z_target if z_target is not None else self.z + dz
        tol = LANDING_ULPS * math.ulp(max(abs(end), 1.0))
        interior = end < p["z_end"] - tol
        on_kink = interior and any(abs(k - end) <= tol for k in kinks)
        return dz, end, kind == "hard_kink" or on_kink

    def attempt_towards(self, target):
        """One attempt of :meth:`march_to` (a startup first when the history is empty)."""
        p = self.p
        planes = tuple(float(v) for v in p["save_planes"]) if not p["interpolate"] else ()
        kinks = tuple(float(v) for v in p["hard_kinks"])
        edges = tuple(float(v) for v in p["breakpoints"])
        z_end = p["z_end"] if p["interpolate"] else target
        if not self.history:
            self._start()
        stop = _landing(self.z, self.proposal, planes, kinks, edges, p["dz_max"], z_end, p["stretch"])
        dz, end, kink = self._approach(stop, planes, kinks, target)
        return self._attempt(dz, end, kink)

    def march_to(self, target):
        while not reached(self.z, target):
            self.attempt_towards(target)

    def replay(self, steps, edges):
        for i, dz in enumerate(steps):
            if not self.history:
                self._start()
            self._attempt(float(dz), float(edges[i + 1]), False, fixed=True)


# ---------------------------------------------------------------- Runge-Kutta
class RungeKuttaEngine:
    """``backends/numpy_ref/engines.py:97-198``: the interaction-picture DOPRI5 trial."""

    def __init__(self, ws: Workspace, control: dict):
        self.ws = ws
        self.control = control
        self.trial_state = None

    def trial(self, z, dz):
        ws, rec = self.ws, self.ws.rec
        state = ws.state
        stages = []
        solution = np.zeros_like(state)
        error = np.zeros_like(state)
        for index, node in enumerate(DOPRI5_NODES):
            combination = np.zeros_like(state)
            for prev in range(index):
                combination = combination + float(DOPRI5_MATRIX[index, prev]) * stages[prev]
            z1 = z + float(node) * dz
            exponent = ws.delta_phi(z, z1)
            lab = np.exp(exponent) * (state + dz * combination)
            back = np.exp(-exponent)
            ws.evaluations += 1
            stage = back * lab_source(rec, lab, z1)
            stages.append(stage)
            solution = solution + float(DOPRI5_SOLUTION[index]) * stage
            error = error + float(DOPRI5_ERROR[index]) * stage
        propagator = np.exp(ws.delta_phi(z, z + dz))
        advanced = propagator * (state + dz * solution)
        mask = rec.norm_mask
        c = self.control
        scale = c["rtol"] * max(float(np.linalg.norm(state[..., mask])),
                                float(np.linalg.norm(advanced[..., mask]))) + c["atol"]
        err = propagator * (dz * error)
        norm = float(np.linalg.norm(err[..., mask] / scale))
        self.trial_state = advanced
        return norm

    def accept(self):
        self.ws.state = self.ws.mask(self.trial_state)


class RungeKuttaMarch:
    """``marches/runge_kutta.py:125-250`` with ``rk_core``'s decisions."""

    def __init__(self, engine: RungeKuttaEngine, policy: dict, proposal: float):
        self.engine = engine
        self.p = policy
        self.c = policy["controller"]
        self.z = 0.0
        self.proposal = proposal
        self.norms = []
        self.attempts = 0
        self.rejected = 0

    def _propose_factor(self):
        c = self.c
        index = len(self.norms) - 1 - c["lag"]
        if index < 0:
            return 1.0
        current = self.norms[index]
        if not math.isfinite(current):
            return c["min_factor"]
        if current <= 0.0:
            return c["max_factor"]
        previous = self.norms[index - 1] if index >= 1 else 1.0
        if not math.isfinite(previous) or previous <= 0.0:
            previous = 1.0
        f = c["safety"] * (1.0 / current) ** c["beta1"] * (1.0 / previous) ** c["beta2"]
        return min(max(f, c["min_factor"]), c["max_factor"])

    def _start_up(self, norm):
        """``rk_core.py:67-107`` (``start_up``) with ``controller.py:528-561``
        (``start_factor``): after the first accepted step the deadbeat proposal its norm
        implies, at most ``start_growth`` times the first; the history records the norm
        the first step would have scored at that length, or zero where the cap binds."""
        c, p = self.c, self.p
        growth = float(p.get("start_growth", 100.0))
        q1 = c["estimator_order"] + 1
        if not math.isfinite(norm) or norm <= 0.0:
            factor = growth if norm == 0.0 else c["min_factor"]
        else:
            factor = min(max(c["safety"] * (1.0 / norm) ** (1.0 / q1), c["min_factor"]), growth)
        following = limit_step(self.proposal, factor, p["dz_min"], p["dz_max"])
        recorded = 0.0 if factor >= growth else norm * (following / self.proposal) ** q1
        self.proposal = following
        self.norms[-1] = recorded

    def march_to(self, target):
        p, c = self.p, self.c
        planes = tuple(float(v) for v in p["save_planes"])
        kinks = tuple(float(v) for v in p["hard_kinks"])
        edges = tuple(float(v) for v in p["breakpoints"])
        q1 = c["estimator_order"] + 1
        while not reached(self.z, target):
            dz, kind, z_target = _landing(self.z, self.proposal, planes, kinks, edges,
                                          p["dz_max"], target, p["stretch"])
            norm = self.engine.trial(self.z, dz)
            self.attempts += 1
            equivalent = norm if not math.isfinite(norm) else norm * (self.proposal / dz) ** q1
            accepted = math.isfinite(norm) and (c["reject_free"] or norm <= 1.0)
            end = z_target if z_target is not None else self.z + dz
            if accepted:
                self.engine.accept()
                self.z = end
                self.norms.append(equivalent)
                if p.get("auto_init") and len(self.norms) == 1:
                    self._start_up(equivalent)
                self.proposal = limit_step(self.proposal, self._propose_factor(), p["dz_min"], p["dz_max"])
            else:
                self.rejected += 1
                if not math.isfinite(equivalent):
                    f = c["min_factor"]
                elif equivalent <= 0.0:
                    f = 1.0
                else:
                    f = min(max(c["safety"] * (1.0 / equivalent) ** (1.0 / q1), c["min_factor"]), 1.0)
                self.proposal = limit_step(self.proposal, f, p["dz_min"], p["dz_max"])

    def replay(self, steps, edges):
        for i, dz in enumerate(steps):
            self.engine.trial(self.z, float(dz))
            self.engine.accept()
            self.z = float(edges[i + 1])
