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
from . import _lib


def refine_params(nev: int, tol: float = 1e-10) -> LanczosParams:
    """FP64 block Lanczos with block = nev, started from FP32 Ritz vectors."""
    lib = _lib.load()
    n_slots = max(3, min(8, lib.rsed_lanczos_max_projected() // nev))
    keep = max(1, min(lib.rsed_lanczos_max_keep() // nev, n_slots - 2))
    return LanczosParams(block=nev, n_slots=n_slots, keep_blocks=keep, tol=tol, max_restarts=50,
                         check_every=1, precision=64)


class BatchedSectorSolver:
    """Lowest ``nev`` eigenpairs of several sectors of one catalog."""

    def __init__(self, model: DeviceModel, sset: SectorSet, sectors: list[int], nev: int, *,
                 precision: int = 64, params: LanczosParams | None = None, poll: int = 8,
                 graph: bool = True):
        p = params or LanczosParams(block=2 if nev <= 4 else 3, n_slots=16)
        if p.precision != precision:
            p = LanczosParams(**{**p.__dict__, "precision": precision})
        self.model, self.sset, self.sectors, self.nev = model, sset, list(sectors), nev
        self.precision = precision
        self.poll = poll
        self.graph = graph
        self.batch = LanczosBatch(model, sset, self.sectors, nev, p)
        self.refiner = None
        if precision == 32:
            self.refiner = LanczosBatch(model, sset, self.sectors, nev, refine_params(nev, p.tol))
        self.last_fp32_vals = None

    def _run(self, b: LanczosBatch, poll: int):
        b.start()
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
        if self.refiner is not None:
            self.last_fp32_vals = b.ritz_val[:, : self.nev].clone()
            U = b.ritz_vectors_orbit()
            r = self.refiner
            r.W.zero_()
            for i in range(r.n_inst):
                c0 = int(r.col0[i])
                r.W[:, c0 : c0 + self.nev] = U[i].t()
            r.start()
            r.run(poll=max(2, self.poll // 2), graph=self.graph)
            b = r
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
        return (self.last_fp32_vals - self.refiner.ritz_val[:, : self.nev]).abs().cpu().numpy()
