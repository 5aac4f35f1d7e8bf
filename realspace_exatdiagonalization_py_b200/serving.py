"""Continuous-batching eigen-solve service.

A request is one (lattice model, momentum sector, flux point) eigen-solve.
Per lattice model the server keeps the zero-flux orbit catalog and its
orbit-space projection table; per flux point a ``FluxContext``: a copy of the
catalog whose amplitudes were moved to the flux point by
``update_orbit_stabilizer_phases`` (no rebuild), the twisted device model, the
sector membership and the flux point's projection weights.  The projection
table's structure (row offsets, target orbit and group element of every hop)
does not change under the phase update, so every flux point of a model shares
it and owns only its weights.

Requests run in *lanes*.  A lane is a resident ``LanczosBatch`` (Krylov basis,
projected matrices, state) of 1..``max_width`` instances on its own CUDA
stream, plus the lane's own copy of one flux point's weights and sector
membership.  A lane serves any flux point of its model: taking a request, it
copies that flux point's weights and membership into its buffers (a device
copy of a few hundred MB at most) and replays the Lanczos iterations from
CUDA graphs captured once, with the lane's first solve -- its kernels only
ever see the lane's own buffers.

Scheduling (``step``), one host thread, no blocking waits on the device:
  * admission: pending requests are grouped by (model, flux); a group takes an
    idle lane of its model (or a new one) with as many of its requests as the
    lane is wide.  A new lane or flux context is admitted only while the device
    bytes they need (measured for contexts, computed for lanes) fit the
    budget; idle lanes and flux contexts no running lane uses are evicted
    (least recently used) to make room.  Requests that do not fit wait.
  * progress: every running lane gets the Lanczos steps up to its next thick
    restart (one graph replay; convergence is decided at restarts) on its
    stream, followed by an asynchronous copy of its state
    into pinned host memory and an event; lanes whose event completed and
    whose instances all stopped move on to the FP64 Rayleigh-Ritz refinement
    (FP32 matvec; run against the flux context's own model) and the
    asynchronous copy of their eigenvalues.  Lanes on different streams
    overlap on the device; a request arriving while others run is admitted at
    the next step as soon as a lane and memory are free.

Each request's start block is drawn on the device from a generator seeded with
``12345 + seed`` (the request id by default), so a result does not depend on
which other requests share the device or its lane.
"""

from __future__ import annotations

import copy
import ctypes
import dataclasses
import os
import queue
import threading
import time
from collections import OrderedDict
from dataclasses import dataclass
from fractions import Fraction

import numpy as np
import torch

from . import _lib
from .batched import APPLY_AUTO, lanczos_footprint_bytes
from .catalog import build_symmetry_orbit_catalog, update_orbit_stabilizer_phases
from .hamiltonian import DeviceModel
from .lanczos import S_ACTIVE, S_ITERS, S_STATUS, LanczosBatch, LanczosParams
from .lattice import generate_bilinear_terms
from .sector import SectorSet
from .symmetry import build_irrep_list, build_translation_group, group_order

__all__ = ["ServingModel", "FluxContext", "SolveRequest", "SolveResult", "SolveServer", "ServedCheckpoints",
           "latency_summary", "poisson_requests"]


@dataclass
class SolveRequest:
    rid: int
    sector: int                      # irrep index (0-based, the reference's result key)
    flux: tuple = ()                 # twisted phases over 2 pi, one per lattice dimension
    model: str = "default"
    arrival: float = 0.0             # seconds after the start of the run
    seed: int | None = None          # start-block seed offset (default: rid)
    vectors: bool = False            # also return the eigenvectors (device tensor in the result)


@dataclass
class SolveResult:
    rid: int
    sector: int
    flux: tuple
    model: str
    eigenvalues: np.ndarray
    residuals: np.ndarray
    fp32_error: np.ndarray | None
    iterations: int
    dim: int
    arrival: float
    admitted: float
    finished: float
    lane: int
    lane_width: int
    # [dim, nev] complex128 CUDA tensor in the sector's basis order at the
    # request's flux point, when the request asked for vectors
    eigenvectors: torch.Tensor | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


class ServingModel:
    """One lattice model: its zero-flux catalog, shared by every flux point."""

    def __init__(self, second_quantized_model, n_filled: int, name: str = "default"):
        self.name = name
        self.model = second_quantized_model
        self.n_filled = int(n_filled)
        self.lattice = second_quantized_model.lattice
        self.stats = second_quantized_model.particle_statistics
        self.group0 = build_translation_group(self.lattice)
        self.catalog = build_symmetry_orbit_catalog(
            second_quantized_model=second_quantized_model, n_filled=self.n_filled,
            symmetry_group=self.group0, particle_statistics=self.stats)
        self.n_orbits = self.catalog.n_orbits
        self.n_sectors = len(build_irrep_list(self.group0, self.lattice))
        # sector dimensions at zero flux (flux points differ only for orbits
        # with nontrivial stabilizers): decides dense vs Lanczos admission
        self.dims_hint: list[int] | None = SectorSet(self.catalog, build_irrep_list(self.group0,
                                                                                    self.lattice)).dims
        self.base: FluxContext | None = None  # zero-flux context: owns the shared table structure
        self.ctx_bytes: int | None = None     # measured device bytes of a flux point, once one was built

    def normalize_flux(self, flux) -> tuple:
        f = tuple(float(x) for x in (flux or ()))
        if not f:
            f = (0.0,) * self.lattice.dim
        if len(f) != self.lattice.dim:
            raise ValueError(f"flux needs {self.lattice.dim} components")
        return f

    def base_context(self, precision: int) -> "FluxContext":
        if self.base is None:
            self.base = FluxContext(self, (0.0,) * self.lattice.dim, precision)
        return self.base


class FluxContext:
    """Device state of one flux point of one model."""

    def __init__(self, sm: ServingModel, flux: tuple, precision: int):
        self.sm = sm
        self.flux = flux
        # FP32 serving also keeps FP64 weights: the refinement's FP64 products
        # then stream the table instead of re-deriving every hop
        want = (32, 64) if precision == 32 else (64,)
        zero = not any(flux)
        if zero:
            terms, group, cat = sm.model.bilinear_terms, sm.group0, sm.catalog
        else:
            terms = generate_bilinear_terms(sm.model.tb_model, twisted_phases_over_2π=list(flux))
            group = build_translation_group(sm.lattice, list(flux))
            cat = sm.catalog.clone()
            update_orbit_stabilizer_phases(cat, group, sm.stats)
        self.catalog = cat
        self.irreps = build_irrep_list(group, sm.lattice)
        self.dm = DeviceModel(cat, terms, sm.model.density_density_terms)
        self.sset = SectorSet(cat, self.irreps)
        if zero:
            self.dm.build_projection(self.sset.sqrt_stab, precisions=want)
        else:
            base = sm.base_context(precision)
            if not torch.equal(self.sset.chi, base.sset.chi):
                raise ValueError("the flux point changes the sector characters; lanes cannot share it")
            self.dm.build_projection(self.sset.sqrt_stab, precisions=want, share=base.dm.proj)
        # the device bytes this flux point owns, summed over its own tensors
        # (host-side: no device synchronisation; a flux point shares the
        # zero-flux catalog's masks and stabilizers and the table structure)
        own = [self.dm.hdiag, self.dm.term_begin, self.dm.term_to, self.dm.term_amp, self.dm.term_jw,
               self.sset.member, self.sset.sqrt_stab, self.sset.chi]
        if not zero:
            own += [cat.table, cat.stab_phase]
        skip = ("rowptr", "cg") if self.dm.proj.get("shared") else ()
        own += [t for k, t in self.dm.proj.items() if torch.is_tensor(t) and k not in skip]
        self.bytes = int(sum(t.numel() * t.element_size() for t in own))
        if not zero:
            sm.ctx_bytes = max(sm.ctx_bytes or 0, self.bytes)
        self.users = 0
        self.last_used = time.perf_counter()

    def weights(self, precision: int) -> torch.Tensor:
        return self.dm.proj["w32" if precision == 32 else "w64"]


class _LaneModel:
    """Model view of a lane: the model's shared table structure with the
    lane's own weight buffer (what ``LanczosBatch`` needs of a model)."""

    def __init__(self, base: FluxContext, w: torch.Tensor, precision: int):
        self.catalog = base.catalog
        src = base.dm.c
        self.c = _lib.RsedModel.from_buffer_copy(src)
        self.c.proj_w32 = _lib.ptr(w) if precision == 32 else None
        self.c.proj_w64 = _lib.ptr(w) if precision == 64 else None


class _LaneSectors:
    """Sector view of a lane: the lane's own membership buffer; row lists and
    dimensions come from the flux context of the current request."""

    def __init__(self, base: FluxContext, member: torch.Tensor):
        self.base = base.sset
        self.member = member
        self.sqrt_stab = base.sset.sqrt_stab
        self.chi = base.sset.chi
        self.n_sectors = base.sset.n_sectors
        self.current = base.sset

    @property
    def dims(self):
        return self.current.dims

    def rows(self, s: int, stream=None):
        return self.current.rows(s, stream)

    def sectors_struct(self, col_sector: torch.Tensor, n_cols: int, ld: int) -> _lib.RsedSectors:
        return _lib.RsedSectors(self.n_sectors, n_cols, ld, group_order(self.base.catalog.symmetry_group),
                                _lib.ptr(self.member), _lib.ptr(self.sqrt_stab), _lib.ptr(self.chi),
                                _lib.ptr(col_sector))


class _Lane:
    _ids = 0

    def __init__(self, sm: ServingModel, width: int, nev: int, params: LanczosParams, poll: int):
        _Lane._ids += 1
        self.id = _Lane._ids
        self.sm = sm
        self.width = width
        self.nev = nev
        self.params = params
        self.poll = poll
        self.stream = torch.cuda.Stream()
        base = sm.base_context(params.precision)
        if base.weights(params.precision) is None:
            raise ValueError(f"model {sm.name!r} was first served at another precision")
        wdt = torch.complex64 if params.precision == 32 else torch.complex128
        self.w = torch.empty_like(base.weights(params.precision), dtype=wdt)
        self.member = torch.empty_like(base.sset.member)
        self.model = _LaneModel(base, self.w, params.precision)
        self.sectors = _LaneSectors(base, self.member)
        self.batch: LanczosBatch | None = None
        # restart-aligned graphs ((head, launches), (cycle, launches)),
        # captured with the lane's first solve
        self.graph = None
        self.it = 0          # Lanczos steps of the current solve
        self.aligned = True  # False once a periodic check moved the solve to per-step launches
        self.state = "idle"
        self.ctx: FluxContext | None = None
        self.reqs: list[SolveRequest] = []
        self.admitted = 0.0
        self.last_used = time.perf_counter()
        self.event = torch.cuda.Event()
        self.h_state = self.h_vals = self.h_res = self.h_fp32 = None
        self.vecs: list[torch.Tensor] | None = None
        self.keep_vectors = False  # set by a server that checkpoints its results
        self.bytes = (lanczos_footprint_bytes(sm.n_orbits, width * params.block, params.n_slots, params.precision)
                      + self.w.numel() * self.w.element_size() + self.member.numel() * 8)

    # -- device work (all on the lane's stream) ----------------------------
    def _start_blocks(self):
        out = []
        for r in self.reqs:
            d = self.ctx.sset.dims[r.sector]
            g = torch.Generator(device="cuda")
            g.manual_seed(12345 + (r.rid if r.seed is None else r.seed))
            blk = torch.randn((d, self.params.block), dtype=torch.complex128, device="cuda", generator=g)
            out.append(blk / torch.linalg.vector_norm(blk, dim=0, keepdim=True))
        return out

    def begin(self, reqs: list[SolveRequest], ctx: FluxContext, now: float) -> None:
        assert len(reqs) == self.width and self.state == "idle"
        self.reqs = list(reqs)
        self.ctx = ctx
        ctx.users += 1
        self.admitted = now
        sectors = [r.sector for r in reqs]
        self.sectors.current = ctx.sset
        # the flux context was built on the admitting stream: order the lane after it
        self.stream.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(self.stream):
            # the flux point's weights and membership into the lane's buffers
            self.w.copy_(ctx.weights(self.params.precision), non_blocking=True)
            self.member.copy_(ctx.sset.member, non_blocking=True)
            if self.batch is None:
                self.batch = LanczosBatch(self.model, self.sectors, sectors, self.nev, self.params,
                                          block_sizes=[self.params.block] * self.width)
                self.h_state = torch.empty(self.batch.state.shape, dtype=torch.int32).pin_memory()
                self.h_vals = torch.empty((self.width, self.nev), dtype=torch.float64).pin_memory()
                self.h_res = torch.empty((self.width, self.nev), dtype=torch.float64).pin_memory()
                self.h_fp32 = torch.empty((self.width, self.nev), dtype=torch.float64).pin_memory()
            else:
                b = self.batch
                b.inst_sectors = sectors
                cs = np.concatenate([[s] * self.params.block for s in sectors]).astype(np.int32)
                b.col_sector.copy_(torch.from_numpy(cs), non_blocking=False)
            b = self.batch
            b.load_start(self._start_blocks())
            b.start()
            # head: keep steps, no restart can fall due (see LanczosBatch.run_aligned)
            self.aligned = b.keep >= 1 and b.restart_period >= 1 and not b.periodic_check_in(1, b.keep)
            if not self.aligned:
                b.iterate(self.poll, self.stream)
                self.it = self.poll
            elif self.graph is None:
                b.iterate(b.keep, self.stream)  # the first solve runs every kernel once before the captures
                self.graph = (b.capture_span(b.keep, False, sync=False),
                              b.capture_span(b.restart_period, True, sync=False))
                self.it = b.keep
            else:
                self.graph[0][0].replay()
                self.it = b.keep
            self._advance()
        self.state = "running"

    def _advance(self) -> None:
        """The next cycle of restart_period steps, ending at a restart (or,
        once a periodic check would fall inside a cycle, poll single steps
        for the rest of the solve), then an asynchronous copy of the state."""
        b = self.batch
        if self.aligned and b.periodic_check_in(self.it + 1, self.it + b.restart_period - 1):
            self.aligned = False
        if self.aligned:
            self.graph[1][0].replay()
            self.it += b.restart_period
        else:
            b.iterate(self.poll, self.stream)
            self.it += self.poll
        self.h_state.copy_(b.state, non_blocking=True)
        self.event.record(self.stream)

    def _finish(self) -> None:
        b = self.batch
        if self.params.precision == 32:
            fp32 = b.ritz_val[:, : self.nev].clone()
            # FP64 products against the flux point's own model and membership
            sc = self.ctx.sset.sectors_struct(b.col_sector, b.n_cols, b.ld)
            _lib.check(_lib.lib().rsed_lanczos_rayleigh_ritz(
                ctypes.byref(self.ctx.dm.c), ctypes.byref(sc), ctypes.byref(b.c), APPLY_AUTO,
                _lib.stream_ptr(self.stream)))
            self.h_fp32.copy_((fp32 - b.ritz_val[:, : self.nev]).abs(), non_blocking=True)
        want = self.keep_vectors or any(r.vectors for r in self.reqs)
        self.vecs = b.eigenvectors(stream=self.stream) if want else None
        self.h_vals.copy_(b.ritz_val[:, : self.nev], non_blocking=True)
        self.h_res.copy_(b.resid[:, : self.nev], non_blocking=True)
        self.h_state.copy_(b.state, non_blocking=True)
        self.event.record(self.stream)

    def _release(self) -> None:
        if self.ctx is not None:
            self.ctx.users -= 1
            self.ctx.last_used = time.perf_counter()
        self.ctx = None
        self.reqs = []
        self.state = "idle"
        self.last_used = time.perf_counter()

    def poll_once(self, now: float, max_iter: int) -> list[SolveResult] | None:
        """Advance the lane if its last work completed; results when done."""
        if self.state == "idle" or not self.event.query():
            return None
        st = self.h_state.numpy()
        with torch.cuda.stream(self.stream):
            if self.state == "running":
                if st[:, S_ACTIVE].any() and st[:, S_ITERS].max() < max_iter:
                    self._advance()
                    return None
                bad = [i for i in range(self.width) if st[i, S_STATUS] != 1]
                if bad:
                    code = int(st[bad[0], S_STATUS]) or _lib.RSED_ENOTCONV
                    rids = [self.reqs[i].rid for i in bad]
                    self._release()
                    raise _lib.RsedError(code, f"lane {self.id}: requests {rids} did not converge")
                self._finish()
                self.state = "finishing"
                return None
        # finishing: results are in pinned memory (vectors on the device)
        out = []
        vecs = self.vecs or [None] * self.width
        self.vecs = None
        for i, r in enumerate(self.reqs):
            v = vecs[i] if (r.vectors or self.keep_vectors) else None
            if v is not None:  # the caller reads it on its own stream
                v.record_stream(torch.cuda.current_stream())
            out.append(SolveResult(
                rid=r.rid, sector=r.sector, flux=r.flux, model=r.model,
                eigenvalues=self.h_vals[i].numpy().copy(), residuals=self.h_res[i].numpy().copy(),
                fp32_error=self.h_fp32[i].numpy().copy() if self.params.precision == 32 else None,
                iterations=int(st[i, S_ITERS]), dim=int(self.ctx.sset.dims[r.sector]), arrival=r.arrival,
                admitted=self.admitted, finished=now, lane=self.id, lane_width=self.width, eigenvectors=v))
        self._release()
        return out


class ServedCheckpoints:
    """Served results written as the flux scan's checkpoints: one pickled
    ``Symmetry_Resolved_ED_Data`` per (model, flux point) holding
    ``ed_scan_res[sector] = (eigenvalues, eigenvectors)`` (the reference's
    format, ``symmetry_resolved_ed.py:2530-2600``), so a served run resumes
    from, and leaves behind, what the scan path reads and writes.

    A finished result is copied device -> pinned host on the current stream
    (asynchronous, ordered by an event) and handed to a writer thread, which
    merges all queued results of a file and replaces the file atomically; the
    scheduling loop never waits on the disk or the copy.  ``path_of(sm,
    flux)`` names the file (default: the flux scan's canonical name in
    ``checkpoint_dir``); with ``overwrite`` existing files are neither read
    nor kept.
    """

    def __init__(self, checkpoint_dir: str, *, path_of=None, overwrite: bool = False):
        from .ed import ed_scan_checkpoint_filename

        os.makedirs(checkpoint_dir, exist_ok=True)
        self.dir = checkpoint_dir
        self.overwrite = overwrite
        self.path_of = path_of or (lambda sm, flux: os.path.join(
            checkpoint_dir, ed_scan_checkpoint_filename(sm.model, list(flux), Fraction(sm.n_filled, sm.lattice.n_site))))
        self._data: dict[str, object] = {}      # path -> ED data written (or read) so far
        self._fresh: set[str] = set()           # paths started anew under overwrite
        self._q: queue.Queue = queue.Queue()
        self._lock = threading.Lock()
        self._error: BaseException | None = None
        self._thread = threading.Thread(target=self._loop, name="rsed-checkpoints", daemon=True)
        self._thread.start()
        self.written: set[str] = set()

    # -- reading -------------------------------------------------------------
    def _load(self, path: str):
        with self._lock:
            if path in self._data:
                return self._data[path]
        if self.overwrite or not os.path.isfile(path):
            return None
        from .ed import load_checkpoint

        data = load_checkpoint(path)
        with self._lock:
            self._data.setdefault(path, data)
            return self._data[path]

    def lookup(self, sm: "ServingModel", flux: tuple, sector: int, nev: int):
        """``(eigenvalues, eigenvectors)`` of a finished solve with at least
        ``nev`` levels, or ``None``."""
        data = self._load(self.path_of(sm, flux))
        if data is None:
            return None
        res = data.ed_scan_res.get(sector)
        if res is None or len(res[0]) < nev or res[1] is None:
            return None
        return res

    # -- writing -------------------------------------------------------------
    def put(self, sm: "ServingModel", flux: tuple, sector: int, eigenvalues: np.ndarray,
            eigenvectors: torch.Tensor, dim: int) -> None:
        host = torch.empty(eigenvectors.shape, dtype=eigenvectors.dtype, pin_memory=True)
        host.copy_(eigenvectors, non_blocking=True)
        ev = torch.cuda.Event()
        ev.record()
        self._q.put((self.path_of(sm, flux), sm, tuple(flux), int(sector), np.array(eigenvalues), host, ev, dim))

    def _skeleton(self, sm: "ServingModel", flux: tuple):
        from .ed import Symmetry_Resolved_ED_Data

        lat = copy.copy(sm.lattice)
        lat.twisted_phases_over_2π = list(flux)
        model = dataclasses.replace(sm.model, lattice=lat, bilinear_terms=generate_bilinear_terms(
            sm.model.tb_model, twisted_phases_over_2π=list(flux)))
        group = build_translation_group(lat, list(flux))
        irreps = build_irrep_list(group, lat)
        return Symmetry_Resolved_ED_Data(model, sm.n_filled, Fraction(sm.n_filled, lat.n_site), group, irreps,
                                         None, [0] * len(irreps))

    def _loop(self) -> None:
        from .ed import save_checkpoint

        while True:
            item = self._q.get()
            if item is None:
                self._q.task_done()
                return
            batch = [item]
            while True:  # everything queued meanwhile: one write per file
                try:
                    nxt = self._q.get_nowait()
                except queue.Empty:
                    break
                if nxt is None:
                    self._q.put(None)
                    self._q.task_done()
                    break
                batch.append(nxt)
            try:
                by_path: dict[str, list] = {}
                for it in batch:
                    by_path.setdefault(it[0], []).append(it)
                for path, items in by_path.items():
                    data = self._load(path) if path not in self._fresh else self._data.get(path)
                    if data is None:
                        data = self._skeleton(items[0][1], items[0][2])
                        if self.overwrite:
                            self._fresh.add(path)
                    for _, _, _, sector, vals, host, ev, dim in items:
                        ev.synchronize()
                        data.ed_scan_res[sector] = (vals, host.numpy().copy())
                        data.sector_dims[sector] = dim
                    with self._lock:
                        self._data[path] = data
                    save_checkpoint(data, path)
                    self.written.add(path)
            except BaseException as e:  # reported by flush()
                self._error = e
            finally:
                for _ in batch:
                    self._q.task_done()

    def flush(self) -> None:
        """Wait until every queued result is on disk."""
        self._q.join()
        if self._error is not None:
            err, self._error = self._error, None
            raise RuntimeError("writing a checkpoint failed") from err

    def close(self) -> None:
        self.flush()
        self._q.put(None)
        self._thread.join()


class SolveServer:
    """Continuous-batching server over one or more ``ServingModel``s."""

    def __init__(self, models: dict[str, ServingModel] | ServingModel, *, nev: int = 4, precision: int = 32,
                 block: int = 4, n_slots: int = 16, poll: int = 16, max_width: int = 4,
                 memory_budget: int | None = None, max_iter: int = 4000, creations_per_step: int = 1,
                 dense_max: int = 500, checkpoints: ServedCheckpoints | None = None):
        if isinstance(models, ServingModel):
            models = {models.name: models}
        self.models = dict(models)
        self.nev = nev
        self.precision = precision
        self.params = LanczosParams(block=block, n_slots=n_slots, precision=precision,
                                    apply_variant=APPLY_AUTO)
        self.poll = poll
        self.max_width = max_width
        self.max_iter = max_iter
        # new flux contexts and lanes cost milliseconds of host work; making at
        # most this many per step keeps the running lanes fed in between
        self.creations_per_step = creations_per_step
        # sectors up to this dimension are solved densely at admission (as the
        # reference does below 500), not in a Lanczos lane
        self.dense_max = dense_max
        # finished results also go to per-flux-point checkpoints, and requests
        # already there are answered from them
        self.checkpoints = checkpoints
        self._wants_vectors: dict[int, bool] = {}
        self._ready: list[SolveResult] = []
        if memory_budget is None:
            free, _ = torch.cuda.mem_get_info()
            memory_budget = int(0.8 * free)
        self.budget = memory_budget
        self.contexts: OrderedDict[tuple, FluxContext] = OrderedDict()
        self.lanes: list[_Lane] = []
        self.pending: list[SolveRequest] = []
        self.t0 = time.perf_counter()
        self.peak_running = 0
        self.admissions = 0

    # -- memory ------------------------------------------------------------
    def used_bytes(self) -> int:
        base = sum(sm.base.bytes for sm in self.models.values() if sm.base is not None)
        return base + sum(c.bytes for c in self.contexts.values()) + sum(ln.bytes for ln in self.lanes)

    def _ctx_estimate(self, sm: ServingModel) -> int:
        if sm.ctx_bytes:
            return sm.ctx_bytes
        n = sm.n_orbits
        return int(sm.catalog.n_states * 16 + n * 64 + n * 74 * (16 + (8 if self.precision == 32 else 0)))

    def _lane_bytes(self, sm: ServingModel, width: int) -> int:
        n = sm.n_orbits
        return (lanczos_footprint_bytes(n, width * self.params.block, self.params.n_slots, self.precision)
                + n * 74 * 8 * (self.precision // 32) + n * 8)

    def _evict(self, need: int) -> bool:
        """Drop idle lanes and flux contexts no running lane uses, least
        recently used first, until ``need`` more bytes fit."""
        if self.used_bytes() + need <= self.budget:
            return True
        victims = [("ctx", k, c.last_used) for k, c in self.contexts.items() if c.users == 0]
        victims += [("lane", ln, ln.last_used) for ln in self.lanes if ln.state == "idle"]
        for kind, obj, _ in sorted(victims, key=lambda v: v[2]):
            if kind == "ctx":
                del self.contexts[obj]
            else:
                self.lanes.remove(obj)
            if self.used_bytes() + need <= self.budget:
                break
        torch.cuda.empty_cache()
        return self.used_bytes() + need <= self.budget

    # -- API -----------------------------------------------------------------
    def now(self) -> float:
        return time.perf_counter() - self.t0

    def submit(self, req: SolveRequest) -> None:
        sm = self.models[req.model]
        req.flux = sm.normalize_flux(req.flux)
        if not 0 <= req.sector < sm.n_sectors:
            raise ValueError(f"request {req.rid}: no sector {req.sector}")
        if self.checkpoints is not None:
            hit = self.checkpoints.lookup(sm, req.flux, req.sector, self.nev)
            if hit is not None:
                vals, vecs = hit
                now = self.now()
                v = None
                if req.vectors:
                    v = torch.as_tensor(np.ascontiguousarray(np.asarray(vecs)[:, : self.nev])).to(
                        sm.catalog.table.device, torch.complex128)
                self._ready.append(SolveResult(
                    rid=req.rid, sector=req.sector, flux=req.flux, model=req.model,
                    eigenvalues=np.asarray(vals[: self.nev], dtype=np.float64), residuals=np.zeros(self.nev),
                    fp32_error=None, iterations=0, dim=int(np.asarray(vecs).shape[0]), arrival=req.arrival,
                    admitted=now, finished=now, lane=-1, lane_width=0, eigenvectors=v))
                return
        self._wants_vectors[req.rid] = req.vectors
        self.pending.append(req)

    def _record(self, results: list[SolveResult]) -> list[SolveResult]:
        # checkpoint finished solves; keep vectors only where they were asked for
        if self.checkpoints is None:
            return results
        for r in results:
            if r.lane == -1:
                continue
            sm = self.models[r.model]
            if r.eigenvectors is not None:
                self.checkpoints.put(sm, r.flux, r.sector, r.eigenvalues, r.eigenvectors, r.dim)
            if not self._wants_vectors.pop(r.rid, False):
                r.eigenvectors = None
        return results

    def running(self) -> int:
        return sum(1 for ln in self.lanes if ln.state != "idle")

    def _context(self, sm: ServingModel, flux: tuple) -> FluxContext | None:
        if not any(flux):
            if sm.base is None and not self._evict(self._ctx_estimate(sm)):
                return None
            return sm.base_context(self.precision)
        key = (sm.name, flux)
        ctx = self.contexts.get(key)
        if ctx is None:
            if sm.base is None and not self._evict(2 * self._ctx_estimate(sm)):
                return None
            sm.base_context(self.precision)
            if not self._evict(self._ctx_estimate(sm)):
                return None
            ctx = FluxContext(sm, flux, self.precision)
            self.contexts[key] = ctx
        self.contexts.move_to_end(key)
        return ctx

    def warm(self, n_lanes: int, width: int = 1, model: str | None = None) -> None:
        """Create ``n_lanes`` idle lanes (buffers and captured graphs) ahead of
        the requests, as a server does at start-up."""
        for name, sm in self.models.items():
            if model is not None and name != model:
                continue
            base = sm.base_context(self.precision)
            for _ in range(n_lanes):
                if not self._evict(self._lane_bytes(sm, width)):
                    break
                ln = _Lane(sm, width, self.nev, self.params, self.poll)
                # one throw-away solve on the zero-flux context captures the graph
                ln.begin([SolveRequest(-1, 0, (0.0,) * sm.lattice.dim, name)] * width, base, 0.0)
                self.lanes.append(ln)
            while any(ln.state != "idle" for ln in self.lanes):
                for ln in self.lanes:
                    ln.poll_once(0.0, self.max_iter)

    def _dense(self, req: SolveRequest, ctx: FluxContext, now: float) -> SolveResult:
        from .hamiltonian import MatrixFreeHamiltonian
        from .lanczos import diagonalize_block_matrixfree
        from .sector import Symmetry_Sector_Basis

        basis = Symmetry_Sector_Basis(ctx.irreps[req.sector], ctx.catalog, ctx.sset, req.sector)
        vecs = None
        if basis.dim == 0:
            vals = np.zeros(0)
        else:
            H = MatrixFreeHamiltonian(basis, ctx.dm.bilinear_terms, ctx.dm.density_terms, None, model=ctx.dm)
            vals, vecs = diagonalize_block_matrixfree(H, basis.dim, nev=self.nev)
        k = len(vals)
        keep = req.vectors or self.checkpoints is not None
        if keep:
            vecs = (torch.zeros((0, 0), dtype=torch.complex128, device=ctx.catalog.table.device) if vecs is None
                    else torch.as_tensor(np.asarray(vecs)).to(ctx.catalog.table.device, torch.complex128))
        return SolveResult(rid=req.rid, sector=req.sector, flux=req.flux, model=req.model,
                           eigenvalues=np.asarray(vals, dtype=np.float64), residuals=np.zeros(k), fp32_error=None,
                           iterations=0, dim=basis.dim, arrival=req.arrival, admitted=now, finished=self.now(),
                           lane=0, lane_width=1, eigenvectors=vecs if keep else None)

    def _admit(self, now: float) -> None:
        groups: OrderedDict[tuple, list[SolveRequest]] = OrderedDict()
        for r in self.pending:
            groups.setdefault((r.model, r.flux), []).append(r)
        admitted: set[int] = set()
        created = 0
        for key, reqs in groups.items():
            sm = self.models[key[0]]
            small = [r for r in reqs if sm.dims_hint is not None and sm.dims_hint[r.sector] <= self.dense_max]
            if small:
                have_ctx = (sm.base is not None) if not any(key[1]) else key in self.contexts
                if not have_ctx and created >= self.creations_per_step:
                    continue
                ctx = self._context(sm, key[1])
                if ctx is None:
                    continue
                created += 0 if have_ctx else 1
                for r in small:
                    if ctx.sset.dims[r.sector] <= self.dense_max:
                        self._ready.append(self._dense(r, ctx, now))
                        admitted.add(r.rid)
                reqs = [r for r in reqs if r.rid not in admitted]
            while reqs:
                idle = [ln for ln in self.lanes if ln.sm is sm and ln.state == "idle" and ln.width <= len(reqs)]
                lane = max(idle, key=lambda ln: ln.width) if idle else None
                have_ctx = (sm.base is not None) if not any(key[1]) else key in self.contexts
                cost = (0 if have_ctx else 1) + (0 if lane is not None else 1)
                if cost and created >= self.creations_per_step:
                    break
                created += cost
                if lane is not None:
                    lane.state = "reserved"  # not evictable while the context is made
                ctx = self._context(sm, key[1])
                if lane is not None:
                    lane.state = "idle"
                if ctx is None:
                    break
                if lane is None:
                    width = min(len(reqs), self.max_width)
                    ctx.users += 1  # pinned while the lane is made
                    ok = self._evict(self._lane_bytes(sm, width))
                    ctx.users -= 1
                    if not ok:
                        break
                    lane = _Lane(sm, width, self.nev, self.params, self.poll)
                    self.lanes.append(lane)
                take, reqs[:] = reqs[: lane.width], reqs[lane.width:]
                lane.keep_vectors = self.checkpoints is not None
                lane.begin(take, ctx, now)
                self.admissions += 1
                admitted.update(r.rid for r in take)
        if admitted:
            self.pending = [r for r in self.pending if r.rid not in admitted]

    def step(self) -> list[SolveResult]:
        """One scheduling round; returns the requests that finished in it."""
        now = self.now()
        done: list[SolveResult] = self._ready
        self._ready = []
        for ln in list(self.lanes):
            res = ln.poll_once(now, self.max_iter)
            if res:
                done.extend(res)
        if self.pending:
            self._admit(self.now())
        self.peak_running = max(self.peak_running, self.running())
        return self._record(done)

    def run(self, requests: list[SolveRequest], *, realtime: bool = True, timeout: float = 600.0
            ) -> list[SolveResult]:
        """Serve ``requests``, each submitted at its ``arrival`` time (seconds
        after the start of this call; all at once if ``realtime`` is false)."""
        order = sorted(requests, key=lambda r: r.arrival)
        self.t0 = time.perf_counter()
        results: list[SolveResult] = []
        i = 0
        while len(results) < len(order):
            now = self.now()
            if now > timeout:
                raise TimeoutError(f"{len(order) - len(results)} requests unfinished after {timeout} s")
            while i < len(order) and (not realtime or order[i].arrival <= now):
                self.submit(order[i])
                i += 1
            got = self.step()
            results.extend(got)
            if not got and self.running() == 0 and not self.pending and i < len(order):
                time.sleep(max(0.0, min(0.002, order[i].arrival - self.now())))
        return results


def latency_summary(results: list[SolveResult]) -> dict:
    lat = np.array([r.latency for r in results])
    span = max(r.finished for r in results) - min(r.arrival for r in results)
    return {"requests": len(results), "throughput_per_s": len(results) / span if span > 0 else None,
            "p50_ms": 1e3 * float(np.percentile(lat, 50)), "p99_ms": 1e3 * float(np.percentile(lat, 99)),
            "mean_ms": 1e3 * float(lat.mean()), "max_ms": 1e3 * float(lat.max())}


def poisson_requests(n: int, rate: float, n_sectors: int, flux_grid: int, *, dim: int = 2, seed: int = 0,
                     model: str = "default") -> list[SolveRequest]:
    """``n`` requests with exponential inter-arrival times (rate per second),
    uniform sector and uniform flux point on a ``flux_grid``^dim grid in
    [0, 1)^dim (units of 2 pi), all from ``numpy.random.default_rng(seed)``."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, size=n)) if rate > 0 else np.zeros(n)
    sec = rng.integers(0, n_sectors, size=n)
    fl = rng.integers(0, flux_grid, size=(n, dim))
    return [SolveRequest(rid=i, sector=int(sec[i]), flux=tuple(float(Fraction(int(k), flux_grid)) for k in fl[i]),
                         model=model, arrival=float(t[i])) for i in range(n)]
