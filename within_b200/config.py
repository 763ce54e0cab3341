"""Advanced preconditioner configuration, mirroring ``within.config``
(python/within/config.py and crates/within-py/src/config.rs).

    from within_b200 import solve
    from within_b200.config import AdditiveSchwarz, LocalSolverConfig, Schur

    schwarz = AdditiveSchwarz(local_solver=LocalSolverConfig(schur=Schur.exact()))
    result = solve(categories, y, preconditioner=schwarz)
"""
from __future__ import annotations

from dataclasses import dataclass, field

__all__ = [
    "AdditiveSchwarz",
    "ApproxCholConfig",
    "ApproxSchurConfig",
    "LocalSolverConfig",
    "ReductionStrategy",
    "ScalingConfig",
    "Schur",
]


class ReductionStrategy:
    """Combination of overlapping subdomain contributions (schwarz/planning.rs).

    Accepted for API compatibility; on the GPU every strategy resolves to the
    same deterministic per-DOF gather, so results do not depend on it.
    """

    __slots__ = ("name",)

    def __init__(self, name: str):
        self.name = name

    def __repr__(self) -> str:
        return f"ReductionStrategy.{self.name}"

    def __eq__(self, other) -> bool:
        return isinstance(other, ReductionStrategy) and other.name == self.name

    def __hash__(self) -> int:
        return hash(self.name)


ReductionStrategy.Auto = ReductionStrategy("Auto")
ReductionStrategy.AtomicScatter = ReductionStrategy("AtomicScatter")
ReductionStrategy.ParallelReduction = ReductionStrategy("ParallelReduction")


@dataclass(frozen=True)
class ApproxCholConfig:
    """ApproxCholConfig (crates/within/src/config.rs:20-26)."""

    seed: int = 0
    split_merge: int | None = None


@dataclass(frozen=True)
class ApproxSchurConfig:
    """ApproxSchurConfig (config.rs:113-131): seed and star-edge split (>= 1)."""

    seed: int = 0
    split: int = 1

    def __post_init__(self):
        if self.split < 1:
            raise ValueError("ApproxSchurConfig.split must be >= 1")


class Schur:
    """SchurMode (config.rs:46-59): approximate (default) or exact."""

    __slots__ = ("exact_mode", "config")

    def __init__(self, exact_mode: bool, config: ApproxSchurConfig | None):
        self.exact_mode = exact_mode
        self.config = config

    @staticmethod
    def approximate(config: ApproxSchurConfig | None = None) -> "Schur":
        return Schur(False, config or ApproxSchurConfig())

    @staticmethod
    def exact() -> "Schur":
        return Schur(True, None)

    def __repr__(self) -> str:
        return "Schur.exact()" if self.exact_mode else f"Schur.approximate({self.config!r})"


@dataclass(frozen=True)
class ScalingConfig:
    """ScalingConfig (config.rs:88-111); on_failure is "warn" or "error"."""

    tolerance: float | None = None
    max_sweeps: int | None = None
    on_failure: str | None = None


@dataclass(frozen=True)
class LocalSolverConfig:
    """LocalSolverConfig (config.rs:61-86)."""

    approx_chol: ApproxCholConfig | None = None
    schur: Schur | None = None
    dense_threshold: int | None = None
    scaling: ScalingConfig | None = None


@dataclass(frozen=True)
class AdditiveSchwarz:
    """PreconditionerConfig::Additive with explicit tuning."""

    local_solver: LocalSolverConfig | None = None
    reduction: ReductionStrategy = field(default_factory=lambda: ReductionStrategy.Auto)
