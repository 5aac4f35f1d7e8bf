"""Measured choice of how a batch of sector solves runs.

For one batch shape (catalog size, sector dimensions, nev, precision, device)
the tuner builds every candidate ``SolverConfig`` -- block sizes per
instance, persistent cluster path or graph path, projection-table or
on-the-fly matvec -- runs each one to convergence on the real operator
(seeded start blocks, one untimed solve to capture graphs and warm the
caches, then ``trials`` (at least two) timed solves with CUDA events that
alternate two sets of start blocks, ranked by their mean), discards candidates
that fail or whose eigenvalues disagree with the others beyond the solve
tolerance, and keeps the fastest.  Results are cached per shape in memory and,
optionally, in a JSON file, so a serving process tunes each shape once.

Candidate space:
  * uniform blocks b in {2, 4, 8} that hold ``nev`` in the restart basis, with
    basis lengths 10, 12, 16 and 24 for b = 2 and 12 and 16 for b = 4;
  * for uneven sector sizes, a graded assignment (b = 4 for the larger half of
    the sectors, b = 2 for the rest) -- instances of one batch share launches,
    so a smaller block on the small sectors trades their iteration count
    against the batch's per-iteration cost;
  * the persistent path with clusters of 2, 4 and 8 CTAs (uniform b <= 4,
    bases small enough for one cluster per sector) and the graph path;
  * the projection table (when it fits the memory budget) and the on-the-fly
    apply.
"""

from __future__ import annotations

import json
import os
import time
from dataclasses import asdict

import numpy as np
import torch

from . import _lib
from .batched import PERSISTENT_MAX_ORBITS, BatchedSectorSolver, SolverConfig, persistent_ok
from .hamiltonian import DeviceModel
from .lanczos import LanczosParams, _auto_keep
from .sector import SectorSet

__all__ = ["Autotuner", "candidate_configs", "default_tuner"]


def _nev_fits(nev: int, b: int, n_slots: int) -> bool:
    lib = _lib.load()
    if n_slots * b > lib.rsed_lanczos_max_projected() or b > lib.rsed_lanczos_max_block():
        return False
    try:
        keep = _auto_keep(nev, b, n_slots)
    except ValueError:
        return False
    # the FP64 Rayleigh-Ritz step applies H to the restart basis and its
    # residual block into the slots after them: 2 * keep + 1 <= n_slots
    return keep * b <= lib.rsed_lanczos_max_keep() and 2 * keep + 1 <= n_slots


def candidate_configs(dims: list[int], nev: int, n_orbits: int, *, projection_ok: bool = True,
                      quick: bool = False) -> list[SolverConfig]:
    """The configurations the tuner measures for a batch with sector
    dimensions ``dims`` (``quick`` keeps a short list for large bases)."""
    n = len(dims)
    blocks = [b for b in (2, 4, 8) if _nev_fits(nev, b, 16 if b < 8 else 8)]
    shapes: list[tuple[int, ...]] = [(b,) * n for b in blocks]
    if n > 1 and max(dims) > 1.5 * min(dims) and 2 in blocks and 4 in blocks:
        med = float(np.median(dims))
        shapes.append(tuple(4 if d >= med else 2 for d in dims))
    out: list[SolverConfig] = []
    mats = [True, False] if projection_ok else [False]
    for bs in shapes:
        slots = 16 if max(bs) < 8 else 8
        for proj in mats:
            out.append(SolverConfig(bs, 0, proj, slots))
        # other basis lengths: a longer basis restarts less often, a shorter
        # one reads fewer blocks per Gram-Schmidt step (on the 32-site
        # workload, b = 2: 12 slots 387 ms, 16 slots 410 ms, 24 slots 491 ms)
        for alt in {2: (10, 12, 24), 4: (12,)}.get(max(bs), ()):
            if projection_ok and _nev_fits(nev, max(bs), alt):
                out.append(SolverConfig(bs, 0, True, alt))
        if persistent_ok(bs) and n_orbits <= PERSISTENT_MAX_ORBITS:
            for cs in (2, 4, 8):
                out.append(SolverConfig(bs, cs, False, slots))
    if quick:
        out = [c for c in out if c.persistent == 0 and (c.projection or not projection_ok)
               and len(set(c.block_sizes)) == 1 and c.block_sizes[0] in (2, 4)] or out[:2]
    return out


def _shape_key(dm: DeviceModel, sset: SectorSet, sectors, nev: int, precision: int) -> str:
    dev = torch.cuda.get_device_name(dm.hdiag.device) if dm.hdiag.is_cuda else "cpu"
    dims = tuple(int(sset.dims[s]) for s in sectors)
    cat = dm.catalog
    return json.dumps([dev, cat.n_site, cat.n_filled, int(cat.n_orbits), dm.n_terms, len(dm.density_terms),
                       dims, nev, precision])


class Autotuner:
    """Per-shape measured configuration cache (see module docstring)."""

    def __init__(self, cache_path: str | None = None, trials: int = 2, memory_fraction: float = 0.5):
        self.cache_path = cache_path
        self.trials = trials
        self.memory_fraction = memory_fraction
        self.cache: dict[str, dict] = {}
        if cache_path and os.path.isfile(cache_path):
            with open(cache_path) as f:
                self.cache = json.load(f)

    def _save(self) -> None:
        if self.cache_path:
            tmp = self.cache_path + ".tmp"
            with open(tmp, "w") as f:
                json.dump(self.cache, f, indent=1)
            os.replace(tmp, self.cache_path)

    def _projection_ok(self, dm: DeviceModel, precision: int) -> bool:
        if dm.proj is not None:
            return True
        free, _ = torch.cuda.mem_get_info(dm.hdiag.device)
        need = dm.projection_bytes((64, 32) if precision == 32 else (64,))
        return need <= self.memory_fraction * free

    def tune(self, dm: DeviceModel, sset: SectorSet, sectors: list[int], nev: int, precision: int = 32,
             params: LanczosParams | None = None, candidates: list[SolverConfig] | None = None,
             tol: float = 1e-8) -> tuple[SolverConfig, list[dict]]:
        """Measure every candidate; returns the fastest and the table."""
        sectors = list(sectors)
        dims = [int(sset.dims[s]) for s in sectors]
        if candidates is None:
            quick = dm.catalog.n_orbits * len(sectors) > 4_000_000
            candidates = candidate_configs(dims, nev, dm.catalog.n_orbits,
                                           projection_ok=self._projection_ok(dm, precision), quick=quick)
        base = params or LanczosParams(precision=precision)
        table = []
        ref_vals = None
        for cfg in candidates:
            row = {"config": cfg.describe()}
            try:
                p = LanczosParams(**{**base.__dict__, "precision": precision, "block": max(cfg.block_sizes)})
                sol = BatchedSectorSolver(dm, sset, sectors, nev, precision=precision, params=p, config=cfg)
                sol.solve(None, vectors=False, host=False)  # capture graphs, warm caches
                # two sets of start blocks: convergence is decided at restarts,
                # so a solve's step count is quantised by the restart period and
                # one start set can favour either basis length; the trials
                # alternate one seed for every sector and a seed per sector
                times = []
                for t in range(max(2, self.trials)):
                    seeds = None if t % 2 == 0 else [12345 + s for s in sectors]
                    torch.cuda.synchronize()
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record()
                    vals_t, _ = sol.solve(None, vectors=False, host=False, seeds=seeds)
                    e1.record()
                    torch.cuda.synchronize()
                    times.append(e0.elapsed_time(e1) * 1e-3)
                    if t == 0:
                        vals = vals_t
                vals = vals.cpu().numpy()
                if ref_vals is None:
                    ref_vals = vals
                dev = float(np.max(np.abs(vals - ref_vals)))
                row.update({"time_s": float(np.mean(times)), "max_abs_dE_vs_first": dev,
                            "ok": dev <= tol})
                del sol
            except (_lib.RsedError, ValueError, torch.cuda.OutOfMemoryError) as exc:
                row.update({"time_s": None, "ok": False, "error": str(exc)[:200]})
            table.append(row)
        good = [(r["time_s"], i) for i, r in enumerate(table) if r.get("ok")]
        if not good:
            raise RuntimeError(f"no candidate configuration solved the batch: {table}")
        best = candidates[min(good)[1]]
        return best, table

    def best(self, dm: DeviceModel, sset: SectorSet, sectors: list[int], nev: int, precision: int = 32,
             params: LanczosParams | None = None) -> SolverConfig:
        """Cached configuration for this batch shape, tuning it on a miss."""
        key = _shape_key(dm, sset, sectors, nev, precision)
        hit = self.cache.get(key)
        if hit is not None:
            return SolverConfig(tuple(hit["block_sizes"]), hit["persistent"], hit["projection"],
                                hit["n_slots"], hit.get("poll", 16))
        t0 = time.perf_counter()
        cfg, table = self.tune(dm, sset, sectors, nev, precision, params)
        d = asdict(cfg)
        d.pop("extra", None)
        d["block_sizes"] = list(cfg.block_sizes)
        d["tuned_in_s"] = time.perf_counter() - t0
        d["table"] = table
        self.cache[key] = d
        self._save()
        return cfg

    def last_table(self, dm, sset, sectors, nev, precision=32) -> list[dict] | None:
        hit = self.cache.get(_shape_key(dm, sset, sectors, nev, precision))
        return None if hit is None else hit.get("table")


_DEFAULT: Autotuner | None = None


def default_tuner() -> Autotuner:
    """Process-wide tuner (cache file from ``RSED_TUNE_CACHE`` if set)."""
    global _DEFAULT
    if _DEFAULT is None:
        _DEFAULT = Autotuner(os.environ.get("RSED_TUNE_CACHE"))
    return _DEFAULT
