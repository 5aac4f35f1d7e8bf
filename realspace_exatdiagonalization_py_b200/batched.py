"""Batched multi-sector eigen-solves with resident buffers and captured graphs.

``BatchedSectorSolver`` owns one ``LanczosBatch`` (every sector of the batch
advances in the same kernel launches) plus, for FP32-matvec solves, the FP64
refinement batch.  Both keep their device buffers and their captured CUDA
graphs between calls, so a repeated solve (a new start block, a new flux
point after an in-place phase update) costs only the graph replays.

How a batch is run is a ``SolverConfig``: the block size of every instance,
the one-launch persistent path (one thread-block cluster per instance) or the
per-iteration kernels replayed from a CUDA graph, and whether the matvec
streams the orbit-space projection table.  ``autotune.Autotuner`` picks it by
measurement.
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np
import torch

from .hamiltonian import DeviceModel
from .lanczos import LanczosBatch, LanczosParams, vectors_to_host
from .sector import SectorSet

# rsed_apply_h variants: 0 = automatic (projection table when present),
# 999 = automatic on-the-fly mapping
APPLY_AUTO, APPLY_ON_THE_FLY = 0, 999
# one thread-block cluster per sector only pays while a sector is a few hundred KB
PERSISTENT_MAX_ORBITS = 1 << 16


@dataclass(frozen=True)
class SolverConfig:
    """One way to run a batch.  ``block_sizes`` has one entry per instance;
    ``persistent`` is the cluster size of the one-launch path (0 = graph
    path); ``projection`` streams the projection table in every matvec of
    the graph path and of the FP64 refinement."""

    block_sizes: tuple[int, ...]
    persistent: int = 0
    projection: bool = True
    n_slots: int = 16
    poll: int = 16
    extra: tuple = field(default=(), compare=False)

    def describe(self) -> dict:
        bs = sorted(set(self.block_sizes))
        return {"block_sizes": bs[0] if len(bs) == 1 else list(self.block_sizes),
                "path": f"persistent cluster={self.persistent}" if self.persistent else "graph",
                "matvec": "projection table" if self.projection else "on the fly",
                "n_slots": self.n_slots}


def persistent_ok(block_sizes) -> bool:
    """The one-launch kernel holds uniform blocks of 1, 2 or 4 columns."""
    bs = set(block_sizes)
    return len(bs) == 1 and next(iter(bs)) in (1, 2, 4)


class BatchedSectorSolver:
    """Lowest ``nev`` eigenpairs of several sectors of one catalog."""

    def __init__(self, model: DeviceModel, sset: SectorSet, sectors: list[int], nev: int, *,
                 precision: int = 64, params: LanczosParams | None = None, poll: int = 16,
                 graph: bool = True, persistent: int = 4, config: SolverConfig | None = None):
        p = params or LanczosParams()
        if p.precision != precision:
            p = LanczosParams(**{**p.__dict__, "precision": precision})
        self.model, self.sset, self.sectors, self.nev = model, sset, list(sectors), nev
        self.precision = precision
        if config is None:
            bs = (p.block,) * len(self.sectors)
            small = model.catalog.n_orbits <= PERSISTENT_MAX_ORBITS
            config = SolverConfig(bs, persistent if small and persistent_ok(bs) and persistent in (1, 2, 4, 8)
                                  else 0, projection=model.proj is not None, n_slots=p.n_slots, poll=poll)
        if len(config.block_sizes) != len(self.sectors):
            raise ValueError("config.block_sizes needs one entry per sector")
        if config.persistent and not persistent_ok(config.block_sizes):
            raise ValueError("the persistent path needs uniform blocks of 1, 2 or 4 columns")
        if config.projection and model.proj is None:
            model.build_projection(sset.sqrt_stab, precisions=projection_precisions(model, precision))
        p = LanczosParams(**{**p.__dict__, "n_slots": config.n_slots,
                             "apply_variant": APPLY_AUTO if config.projection else APPLY_ON_THE_FLY})
        self.config = config
        self.params = p
        self.poll = config.poll
        self.graph = graph
        self.persistent = config.persistent
        self.batch = LanczosBatch(model, sset, self.sectors, nev, p, block_sizes=list(config.block_sizes))
        self.last_fp32_vals = None

    def _run(self, b: LanczosBatch, poll: int):
        b.start()
        if self.persistent:
            b.run_persistent(self.persistent)
        elif self.graph:
            b.run_aligned(poll=poll)
        else:
            b.run(poll=poll, graph=False)

    def solve(self, start_blocks=None, *, vectors: bool = True, host: bool = True, seeds=None):
        """Solve every sector; ``start_blocks`` and ``seeds`` (per instance, for
        the seeded blocks drawn where ``start_blocks`` is None) as in
        ``LanczosBatch.load_start``.

        Returns ``(vals, vecs)``: ``vals [n_sectors, nev]`` and a list of
        ``[D_s, nev]`` eigenvector blocks (numpy if ``host`` else CUDA tensors,
        ``None`` when ``vectors`` is false).
        """
        b = self.batch
        b.load_start(start_blocks, seeds)
        self._run(b, self.poll)
        if self.precision == 32:
            self.last_fp32_vals = b.ritz_val[:, : self.nev].clone()
            b.rayleigh_ritz()
        vals = b.ritz_val[:, : self.nev]
        vecs = b.eigenvectors() if vectors else None
        if host:
            vals = vals.cpu().numpy()
            if vecs is not None:
                vecs = vectors_to_host(vecs)
        return vals, vecs

    def fp32_error(self) -> np.ndarray | None:
        """|E(FP32 matvec) - E(after FP64 refinement)| per sector and level."""
        if self.last_fp32_vals is None:
            return None
        return (self.last_fp32_vals - self.batch.ritz_val[:, : self.nev]).abs().cpu().numpy()

    def residuals(self) -> np.ndarray:
        """Residual norms per sector and level: true FP64 norms after the
        refinement, the Lanczos estimates otherwise."""
        return self.batch.residuals()

    def footprint_bytes(self) -> int:
        """Device bytes held by this solver's Lanczos buffers."""
        b = self.batch
        tensors = [b.V, b.W, b.Xf, b.P, b.coef, b.partial, b.ritz_val, b.ritz_vec, b.resid, b.state]
        return int(sum(t.numel() * t.element_size() for t in tensors if t is not None))


def projection_precisions(model: DeviceModel, precision: int, fraction: float = 0.25) -> tuple[int, ...]:
    """Weights to build: an FP32 solve also streams FP64 weights in its
    refinement when both fit in ``fraction`` of the free device memory;
    otherwise the refinement's few FP64 products run on the fly."""
    if precision == 64:
        return (64,)
    free, _ = torch.cuda.mem_get_info(model.hdiag.device)
    return (64, 32) if model.projection_bytes((64, 32)) <= fraction * free else (32,)


def plan_waves(n_orbits: int, block_sizes: list[int], budget: int, n_slots: int = 16,
               precision: int = 32) -> list[list[int]]:
    """Split instances (given by their block sizes, in order) into consecutive
    waves whose Lanczos buffers fit ``budget`` bytes each."""
    waves: list[list[int]] = []
    cur: list[int] = []
    cols = 0
    for i, b in enumerate(block_sizes):
        if cur and lanczos_footprint_bytes(n_orbits, cols + b, n_slots, precision) > budget:
            waves.append(cur)
            cur, cols = [], 0
        if lanczos_footprint_bytes(n_orbits, b, n_slots, precision) > budget:
            raise MemoryError(f"one instance of {b} columns over {n_orbits} orbits needs more than {budget} bytes")
        cur.append(i)
        cols += b
    if cur:
        waves.append(cur)
    return waves


def lanczos_footprint_bytes(n_orbits: int, n_cols: int, n_slots: int = 16, precision: int = 32) -> int:
    """Device bytes a batch of ``n_cols`` total columns needs (the basis slots,
    W, the FP32 block and small buffers), for admission control."""
    ld = n_cols + (n_cols & 1)
    per = n_orbits * ld
    b = (n_slots + 2) * per * 16 + per * 16 + (per * 8 if precision == 32 else 0)
    return int(b * 1.02) + (4 << 20)
