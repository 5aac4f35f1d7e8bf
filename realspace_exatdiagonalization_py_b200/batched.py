"""Batched multi-sector eigen-solves with resident buffers and captured graphs.

``BatchedSectorSolver`` owns one ``LanczosBatch`` (every sector of the batch
advances in the same kernel launches) plus, for FP32-matvec solves, the FP64
refinement batch.  Both keep their device buffers and their captured CUDA
graphs between calls, so a repeated solve (a new start block, a new flux
point after an in-place phase update) costs only the graph replays.
"""

from __future__ import annotations

import numpy as np
import torch

from .hamiltonian import DeviceModel
from .lanczos import LanczosBatch, LanczosParams
from .sector import SectorSet


class BatchedSectorSolver:
    """Lowest ``nev`` eigenpairs of several sectors of one catalog."""

    def __init__(self, model: DeviceModel, sset: SectorSet, sectors: list[int], nev: int, *,
                 precision: int = 64, params: LanczosParams | None = None, poll: int = 16,
                 graph: bool = True, persistent: int = 4):
        p = params or LanczosParams()
        if p.precision != precision:
            p = LanczosParams(**{**p.__dict__, "precision": precision})
        self.model, self.sset, self.sectors, self.nev = model, sset, list(sectors), nev
        self.precision = precision
        self.poll = poll
        self.graph = graph
        # cluster size of the one-launch solve (0 = per-iteration kernels in a CUDA graph)
        self.persistent = persistent if (p.block & (p.block - 1)) == 0 and p.block <= 4 else 0
        self.batch = LanczosBatch(model, sset, self.sectors, nev, p)
        self.refiner = None
        self.last_fp32_vals = None

    def _run(self, b: LanczosBatch, poll: int):
        b.start()
        if self.persistent:
            b.run_persistent(self.persistent)
        else:
            b.run(poll=poll, graph=self.graph)

    def solve(self, start_blocks=None, *, vectors: bool = True, host: bool = True):
        """Solve every sector; ``start_blocks`` as in ``LanczosBatch.load_start``.

        Returns ``(vals, vecs)``: ``vals [n_sectors, nev]`` and a list of
        ``[D_s, nev]`` eigenvector blocks (numpy if ``host`` else CUDA tensors,
        ``None`` when ``vectors`` is false).
        """
        b = self.batch
        b.load_start(start_blocks)
        self._run(b, self.poll)
        if self.precision == 32:
            self.last_fp32_vals = b.ritz_val[:, : self.nev].clone()
            b.rayleigh_ritz()
        vals = b.ritz_val[:, : self.nev]
        vecs = b.eigenvectors() if vectors else None
        if host:
            vals = vals.cpu().numpy()
            if vecs is not None:
                vecs = [v.cpu().numpy() for v in vecs]
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
