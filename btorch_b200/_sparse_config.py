"""Sparse connectivity configuration (API of btorch/_sparse_config.py:10-113).

There is one implementation of the sparse product here (hand-written sm_100a
kernels).  The reference's backend names -- "native", "torch_sparse",
"triton" -- and the new name "b200" all select it; they are kept so that
models written against the reference (``config.sparse.backend("triton")``,
``SparseConn(..., sparse_backend="native")``) run unchanged.  The config
objects carry the tunables of the new kernels; the reference's Triton fields
are accepted and validated with the reference's rules but have no effect.
"""

from __future__ import annotations

from copy import deepcopy
from dataclasses import asdict, dataclass, fields, is_dataclass
from typing import Any

DIRECTIONS = ("auto", "gather", "scatter")


@dataclass
class SparseBackendConfig:
    """Tunables of the event-driven sparse product.

    direction: "gather" (pull over in-edges, ordered fmaf chain, deterministic
        and bit-identical to the reference CPU product), "scatter" (push over
        out-edges of the active sources, fp32 reductions in L2, exact only
        when partial sums are), or "auto" (autotuner picks per problem size
        and activity).
    deterministic: force "gather" whatever `direction` says.
    autotune: time both directions on first use of a shape and cache the
        winner (keyed by sizes, nnz, batch and an activity bucket).
    gather_max_nnz_per_step: "auto" without timing data prefers gather when
        nnz is at most this, or when the active fraction is above
        `gather_min_active_fraction`.
    tile: let the autotuner also try the persistent tile engine (networks
        without synaptic delays or receptor channels, batches up to 256).
        Off by default: its push delivery is slow in high-activity bursts.
    """

    direction: str = "auto"
    deterministic: bool = False
    autotune: bool = True
    gather_max_nnz_per_step: int = 1 << 21
    gather_min_active_fraction: float = 0.25
    pull_min_batch: int = 4
    tile: bool = False

    def validate(self) -> None:
        if self.direction not in DIRECTIONS:
            raise ValueError(f"direction must be one of {DIRECTIONS}, got {self.direction!r}.")
        if self.gather_max_nnz_per_step < 0:
            raise ValueError("gather_max_nnz_per_step must be non-negative.")
        if not 0.0 <= self.gather_min_active_fraction <= 1.0:
            raise ValueError("gather_min_active_fraction must lie in [0, 1].")
        if self.pull_min_batch < 1:
            raise ValueError("pull_min_batch must be positive.")


B200SparseConfig = SparseBackendConfig


@dataclass
class TritonSparseConfig(SparseBackendConfig):
    """Accepts the reference's Triton fields (btorch/_sparse_config.py:15-52)
    with the same validation; they do not change the new kernels."""

    reorder: bool = True
    block: bool = True
    hash: bool = True
    block_sources: int = 32
    edge_block: int = 256
    long_fanout_threshold: int = 256
    hash_capacity: int = 512
    hash_max_probe: int = 8
    hash_min_edges: int = 64
    num_warps: int = 4

    def validate(self) -> None:
        super().validate()
        if self.block_sources <= 0:
            raise ValueError("block_sources must be positive.")
        if self.edge_block <= 0 or self.edge_block & (self.edge_block - 1):
            raise ValueError("edge_block must be a positive power of two.")
        if self.long_fanout_threshold <= 0:
            raise ValueError("long_fanout_threshold must be positive.")
        if self.hash_capacity <= 0 or self.hash_capacity & (self.hash_capacity - 1):
            raise ValueError("hash_capacity must be a positive power of two.")
        if self.hash and self.hash_capacity < self.edge_block:
            raise ValueError("hash_capacity must be at least edge_block.")
        if self.hash_max_probe <= 0:
            raise ValueError("hash_max_probe must be positive.")
        if self.hash_min_edges < 0:
            raise ValueError("hash_min_edges must be non-negative.")
        if self.num_warps not in (1, 2, 4, 8):
            raise ValueError("num_warps must be 1, 2, 4, or 8.")


BACKEND_NAMES = ("native", "torch_sparse", "triton", "b200")


class SparseConfigRegistry:
    """Selected backend name plus per-name global config templates
    (btorch/_sparse_config.py:55-113)."""

    def __init__(self, selected: str | None = None):
        self._selected = selected.lower() if selected else None
        self._configs: dict[str, SparseBackendConfig] = {
            "native": SparseBackendConfig(),
            "torch_sparse": SparseBackendConfig(),
            "triton": TritonSparseConfig(),
            "b200": SparseBackendConfig(),
        }

    @property
    def selected(self) -> str | None:
        return self._selected

    def backend(self, name: str | None = None) -> SparseBackendConfig:
        if name is not None:
            normalized = name.lower()
            if normalized not in self._configs:
                choices = ", ".join(sorted(self._configs))
                raise ValueError(f"Unknown sparse backend '{name}'; expected one of {choices}.")
            self._selected = normalized
        if self._selected is None:
            raise RuntimeError("No global sparse backend is selected; call config.sparse.backend('b200') first.")
        return self._configs[self._selected]

    def resolve(self, name: str, override: SparseBackendConfig | dict[str, Any] | None = None) -> SparseBackendConfig:
        resolved = deepcopy(self._configs[name])
        if override is not None:
            values = asdict(override) if is_dataclass(override) else dict(override)
            valid = {f.name for f in fields(resolved)}
            unknown = set(values) - valid
            if unknown:
                raise ValueError(f"Unknown {name} sparse config fields: {', '.join(sorted(unknown))}.")
            for k, v in values.items():
                setattr(resolved, k, v)
        resolved.validate()
        return resolved


__all__ = ["B200SparseConfig", "SparseBackendConfig", "SparseConfigRegistry", "TritonSparseConfig", "BACKEND_NAMES"]
