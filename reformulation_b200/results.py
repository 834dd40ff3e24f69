"""Result records and tolerances, mirroring the reference's harness so a
backend here returns what `qubo/harness/results.py:25-83` and
`jrp/harness/results.py` define (same fields, same statuses, same NaN
conventions), and takes the same `Tolerances`
(`qubo/harness/config.py:83-115`).
"""

from __future__ import annotations

import math
from dataclasses import dataclass

STATUSES = ("optimal", "time_limit", "iteration_limit", "error", "unavailable")


@dataclass(frozen=True)
class Tolerances:
    """What a run asks its solvers to stop on.  Only `optimality` reaches
    PRAQ/PRIA, as the relative duality gap; the iterates are feasible by
    construction, so `feasibility` is recorded but never used."""

    optimality: float = 1e-8
    feasibility: float = 1e-9


@dataclass
class QuboResult:
    """One (backend, QUBO instance) measurement; fields of qubo/harness/results.py:25-83."""

    backend: str
    instance: str
    family: str
    n: int
    edges: int
    status: str
    objective: float = math.nan
    lower: float = math.nan
    upper: float = math.nan
    iterations: int = -1
    setup_seconds: float = math.nan
    solve_seconds: float = math.nan
    optimality_tolerance: float = math.nan
    feasibility_tolerance: float = math.nan
    peak_host_bytes: float = math.nan
    peak_device_bytes: float = math.nan
    note: str = ""

    def __post_init__(self):
        if self.status not in STATUSES:
            raise ValueError(f"unknown status {self.status!r}, expected one of {STATUSES}")


@dataclass
class JrpResult:
    """One (backend, JRP instance) measurement; fields of jrp/harness/results.py."""

    backend: str
    instance: str
    family: str
    items: int
    periods: int
    entries: int
    status: str
    objective: float = math.nan
    lower: float = math.nan
    upper: float = math.nan
    iterations: int = -1
    setup_seconds: float = math.nan
    solve_seconds: float = math.nan
    optimality_tolerance: float = math.nan
    feasibility_tolerance: float = math.nan
    peak_host_bytes: float = math.nan
    peak_device_bytes: float = math.nan
    note: str = ""

    def __post_init__(self):
        if self.status not in STATUSES:
            raise ValueError(f"unknown status {self.status!r}, expected one of {STATUSES}")


def relative_gap(lower: float, upper: float) -> float:
    return (upper - lower) / (1.0 + abs(upper) + abs(lower))
