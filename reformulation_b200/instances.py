"""Instance types for the two LPs, and seeded synthetic generators for the
benchmark workloads.

The types mirror the reference's harness records so a caller's instance needs
no conversion:

* `QuboInstance` is ``qubo/harness/instances.py:18-68``: a minimisation QUBO
  ``min x^T W x`` over ``{0,1}^n`` with W symmetric, stored as its diagonal plus
  its strict upper triangle in COO (``rows[e] < cols[e]``).
* `JrpInstance` is ``jrp/harness/instances.py:27-88``: order costs K_i, a joint
  order cost K0 and holding costs H[i, s, t] (upper triangle, s <= t).

The generators produce the benchmark workloads from a seed and a size.  They
draw from ``numpy.random.default_rng(seed)`` in a fixed order, written out in
each function, so a workload is reproducible anywhere:

* `qubo_sparse_bernoulli` -- QUBO n=200, each pair kept with probability 0.05
* `qubo_uniform_edges` -- QUBO n=100,000 with 1,000,000 distinct uniform pairs
* `jrp_demand` -- JRP with demand-driven holding costs H = h_i d_it (t - s)
* `batch_mix` -- 256 QUBO + 128 JRP of log-uniform sizes
* `arrival_stream` -- Poisson arrivals of QUBO/JRP requests (70 % / 30 %)

Weights are uniform integers in [-100, 100] without zero for off-diagonal
pairs (``rng.integers(-100, 100)`` then ``+1`` on the nonnegative half), and
uniform integers in [-100, 100] for the diagonal.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np


@dataclass(frozen=True)
class QuboInstance:
    """A QUBO in minimisation form, ``min_{x in {0,1}^n} x^T W x``.

    :param name: identifier
    :param family: the group it came from
    :param n: number of binary variables
    :param diag: (n,) diagonal of W
    :param rows: (m,) row of each strict-upper-triangle nonzero, i < j
    :param cols: (m,) column of each
    :param vals: (m,) W_ij = W_ji
    """

    name: str
    family: str
    n: int
    diag: np.ndarray
    rows: np.ndarray
    cols: np.ndarray
    vals: np.ndarray

    @property
    def edges(self) -> int:
        return int(self.vals.size)

    def to_dense(self) -> np.ndarray:
        w = np.zeros((self.n, self.n))
        w[np.arange(self.n), np.arange(self.n)] = self.diag
        w[self.rows, self.cols] = self.vals
        w[self.cols, self.rows] = self.vals
        return w

    @classmethod
    def from_dense(cls, matrix, name: str = "dense", family: str = "dense") -> "QuboInstance":
        w = np.asarray(matrix, dtype=float)
        n = w.shape[0]
        rows, cols = np.triu_indices(n, k=1)
        keep = w[rows, cols] != 0.0
        return cls(name, family, n, np.diagonal(w).copy(), rows[keep], cols[keep],
                   w[rows, cols][keep])


@dataclass(frozen=True)
class JrpInstance:
    """A joint replenishment LP.

    :param order_costs: (N,) K_i
    :param joint_order_cost: K0
    :param holding_costs: (N, T, T) H[i, s, t]; only s <= t is read
    """

    name: str
    family: str
    order_costs: np.ndarray
    joint_order_cost: float
    holding_costs: np.ndarray

    @property
    def items(self) -> int:
        return int(self.order_costs.size)

    @property
    def periods(self) -> int:
        return int(self.holding_costs.shape[-1])

    @property
    def entries(self) -> int:
        return self.items * self.periods * (self.periods + 1) // 2


def _pair_weights(rng: np.random.Generator, count: int) -> np.ndarray:
    vals = rng.integers(-100, 100, count)
    vals[vals >= 0] += 1
    return vals.astype(np.float64)


def _decode_pairs(lin: np.ndarray, n: int) -> tuple[np.ndarray, np.ndarray]:
    """Map linear indices of the strict upper triangle (row-major) to (i, j).

    Row i starts at ``i (2n - i - 1) / 2``.  The float estimate of i from the
    quadratic is corrected by one step either way, so the result is exact.
    """
    lin = np.asarray(lin, dtype=np.int64)
    b = 2.0 * n - 1.0
    i = np.floor((b - np.sqrt(b * b - 8.0 * lin.astype(np.float64))) / 2.0).astype(np.int64)
    i = np.clip(i, 0, n - 2)
    start = i * (2 * n - i - 1) // 2
    low = lin < start
    i[low] -= 1
    start = i * (2 * n - i - 1) // 2
    nxt = (i + 1) * (2 * n - i - 2) // 2
    high = lin >= nxt
    i[high] += 1
    start = i * (2 * n - i - 1) // 2
    j = lin - start + i + 1
    return i, j


def qubo_sparse_bernoulli(seed: int = 0, n: int = 200, p: float = 0.05) -> QuboInstance:
    """Each pair i < j kept with probability p.  Draws: keep mask over the
    row-major triangle, pair weights, then the diagonal."""
    rng = np.random.default_rng(seed)
    iu = np.triu_indices(n, 1)
    keep = rng.random(iu[0].size) < p
    vals = _pair_weights(rng, int(keep.sum()))
    diag = rng.integers(-100, 101, n).astype(np.float64)
    return QuboInstance(f"qubo-bern-n{n}-p{p:g}-s{seed}", "qubo-bernoulli", n, diag,
                        iu[0][keep].astype(np.int64), iu[1][keep].astype(np.int64), vals)


def _uniform_pairs(rng: np.random.Generator, n: int, m: int) -> tuple[np.ndarray, np.ndarray]:
    lin = np.sort(rng.choice(n * (n - 1) // 2, m, replace=False))
    return _decode_pairs(lin, n)


def qubo_uniform_edges(seed: int = 1, n: int = 100_000, m: int = 1_000_000) -> QuboInstance:
    """m distinct pairs drawn uniformly without replacement, sorted in
    row-major triangle order.  Draws: the pairs, their weights, the diagonal."""
    rng = np.random.default_rng(seed)
    rows, cols = _uniform_pairs(rng, n, m)
    vals = _pair_weights(rng, m)
    diag = rng.integers(-100, 101, n).astype(np.float64)
    return QuboInstance(f"qubo-unif-n{n}-m{m}-s{seed}", "qubo-uniform", n, diag, rows, cols, vals)


def _jrp_costs(rng: np.random.Generator, items: int, periods: int):
    k0 = float(rng.uniform(50, 150))
    k = rng.uniform(10, 50, items)
    h = rng.uniform(0.1, 1.0, items)
    zero = rng.random((items, periods)) < 0.3
    d = rng.integers(1, 101, (items, periods)).astype(np.float64)
    d[zero] = 0.0
    return k0, k, h, d


def demand_holding(h: np.ndarray, d: np.ndarray) -> np.ndarray:
    """Dense H[i, s, t] = h_i d_it (t - s) for s <= t, 0 below the diagonal."""
    items, periods = d.shape
    lag = np.arange(periods)[None, :] - np.arange(periods)[:, None]
    lag = np.where(lag >= 0, lag, 0).astype(np.float64)
    return (h[:, None, None] * d[:, None, :]) * lag[None, :, :]


def jrp_demand(seed: int = 2, items: int = 100, periods: int = 500) -> JrpInstance:
    """Draws: K0 ~ U[50,150], K_i ~ U[10,50], h_i ~ U[0.1,1.0], the zero-demand
    mask (probability 0.3), demands ~ integers [1,100]."""
    rng = np.random.default_rng(seed)
    k0, k, h, d = _jrp_costs(rng, items, periods)
    return JrpInstance(f"jrp-N{items}-T{periods}-s{seed}", "jrp-demand", k, k0,
                       demand_holding(h, d))


@dataclass(frozen=True)
class JrpSpec:
    """A demand-form JRP, kept compact (H is N T^2 when dense)."""

    name: str
    order_costs: np.ndarray
    joint_order_cost: float
    holding_rate: np.ndarray   # (N,) h_i
    demand: np.ndarray         # (N, T) d_it

    @property
    def items(self) -> int:
        return int(self.order_costs.size)

    @property
    def periods(self) -> int:
        return int(self.demand.shape[1])

    @property
    def entries(self) -> int:
        return self.items * self.periods * (self.periods + 1) // 2

    def build(self) -> JrpInstance:
        return JrpInstance(self.name, "jrp-demand", self.order_costs, self.joint_order_cost,
                           demand_holding(self.holding_rate, self.demand))


def _qubo_log_uniform(rng: np.random.Generator, k: int, seed: int) -> QuboInstance:
    n = int(round(math.exp(rng.uniform(math.log(500), math.log(50_000)))))
    deg = float(rng.uniform(4, 32))
    m = min(int(round(n * deg / 2)), n * (n - 1) // 2)
    rows, cols = _uniform_pairs(rng, n, m)
    vals = _pair_weights(rng, m)
    diag = rng.integers(-100, 101, n).astype(np.float64)
    return QuboInstance(f"mix-qubo{k}-n{n}-s{seed}", "mix-qubo", n, diag, rows, cols, vals)


def _jrp_log_uniform(rng: np.random.Generator, k: int, seed: int) -> JrpSpec:
    items = int(round(math.exp(rng.uniform(math.log(10), math.log(200)))))
    periods = int(round(math.exp(rng.uniform(math.log(50), math.log(1000)))))
    k0, kk, h, d = _jrp_costs(rng, items, periods)
    return JrpSpec(f"mix-jrp{k}-N{items}-T{periods}-s{seed}", kk, k0, h, d)


def batch_mix(seed: int = 3, qubos: int = 256, jrps: int = 128):
    """The mixed batch: `qubos` QUBOs (n log-uniform in [500, 50,000], average
    degree uniform in [4, 32]) then `jrps` JRPs (N log-uniform in [10, 200],
    T log-uniform in [50, 1,000]).  Each QUBO draws n, degree, pairs, weights,
    diagonal; each JRP draws N, T, then its costs as `jrp_demand`."""
    rng = np.random.default_rng(seed)
    q = [_qubo_log_uniform(rng, k, seed) for k in range(qubos)]
    j = [_jrp_log_uniform(rng, k, seed) for k in range(jrps)]
    return q, j


def arrival_stream(seed: int = 4, rate: float = 100.0, seconds: float = 60.0,
                   qubo_share: float = 0.7):
    """Poisson arrivals at `rate` per second for `seconds`.  Each arrival draws
    its gap, its type (QUBO with probability `qubo_share`) and then its
    instance as in `batch_mix`.  Returns a list of (arrival_time, instance)."""
    rng = np.random.default_rng(seed)
    out = []
    now, k = 0.0, 0
    while True:
        now += float(rng.exponential(1.0 / rate))
        if now > seconds:
            break
        if rng.random() < qubo_share:
            out.append((now, _qubo_log_uniform(rng, k, seed)))
        else:
            out.append((now, _jrp_log_uniform(rng, k, seed)))
        k += 1
    return out
