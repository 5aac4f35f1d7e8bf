"""Batched thick-restart block Lanczos on the device (K8) and the reference's
``diagonalize_block_*`` API (``symmetry_resolved_ed.py:2180-2299``).

A ``LanczosBatch`` holds any number of sector instances of one catalog; each
instance owns ``b`` columns of the shared ``[n_orbits, ld]`` blocks.  The
Lanczos recurrence, the two-pass block Gram-Schmidt, the projected-matrix
eigen-solve and the restarts are FP64 on the GPU; only the matvec may run in
FP32 (``precision=32``), in which case ``refine`` finishes the solve with an
FP64 block Lanczos started from the FP32 Ritz vectors.
"""

from __future__ import annotations

import ctypes
import math
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from .hamiltonian import DeviceModel
from .sector import SectorSet

S_NB, S_STATUS, S_RESTARTS, S_ITERS, S_ACTIVE, S_RESTART_NB = 0, 1, 2, 3, 4, 5
S_NCONV, S_RR, S_ONEPASS_N, S_RED_BLOCKS, S_PASSES = 7, 9, 11, 12, 13
STATE_INTS = 16

__all__ = [
    "LanczosBatch",
    "LanczosParams",
    "start_block",
    "diagonalize_block_dense",
    "diagonalize_block_arpack",
    "diagonalize_block_matrixfree",
]


@dataclass
class LanczosParams:
    """Thick-restart block Lanczos settings.

    ``tol`` is the FP64 convergence test ``||r_j|| <= tol * max(1, |theta_j|)``
    (the reference's ARPACK tolerance).  With ``precision=32`` the FP32-matvec
    phase stops at ``tol32`` and the eigenpairs are then recomputed by an FP64
    Rayleigh-Ritz step over the thick-restart basis: the eigenvalue error is
    second order in the FP32 residual (on the 32-site workload 3.4e-11 at
    tol32 = 1e-6, 1.0e-11 at 5e-7, 1.2e-12 at 2e-7 for 9 % more time).  Ritz checks run at every restart and
    every ``check_every`` iterations."""

    block: int = 4
    n_slots: int = 16
    keep_blocks: int = 0  # 0 = automatic
    tol: float = 1e-10
    tol32: float = 5e-7  # measured: 1e-6 -> 5e-7 cuts the refined error ~3x at the same speed
    max_restarts: int = 1000  # a cap, not a budget: a 48-site sector with a 3e-4 gap at nev needed 218 (b = 2)
    check_every: int = 1000
    precision: int = 64
    apply_variant: int = 0
    single_pass: bool = True  # skip the second Gram-Schmidt pass when pass 1 lost little norm
    stream: bool = True  # Gram-Schmidt kernels stream whole-row panels by bulk copies (batches with ld <= 64)
    # the update streams too; off by default: on the 32-site workload the
    # row-group update takes 615 us per launch, the streamed one 727 us
    stream_update: bool = False
    row_restart: bool = True  # thick restart over whole rows (all instances per block)


def reserved_bits(p: LanczosParams) -> int:
    """The kernel-form switches of ``rsed_lanczos_t.reserved``: bit 0 adaptive
    single Gram-Schmidt pass, bit 1 per-instance reduction (streaming off),
    bit 2 row-group update after the streamed reduction, bit 3 per-instance
    thick restart."""
    return ((1 if p.single_pass else 0) | (0 if p.stream else 2) | (0 if p.stream_update else 4)
            | (0 if p.row_restart else 8))


def start_block(n: int, b: int, seed: int = 12345) -> np.ndarray:
    """Seeded complex-normal start block ``[n, b]``, each column normalised.

    Column 0 with ``seed=12345`` is the reference's ``v0``
    (``symmetry_resolved_ed.py:2291-2293``)."""
    cols = []
    for j in range(b):
        rng = np.random.default_rng(seed + 7919 * j)
        v = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        cols.append(v / np.linalg.norm(v))
    return np.stack(cols, axis=1)


def _auto_keep(nev: int, b: int, n_slots: int) -> int:
    """Largest restart basis the kernels hold (<= 16 vectors) that leaves room
    for the FP64 Rayleigh-Ritz step (n_slots >= 2*keep + 1)."""
    kmax = _lib.load().rsed_lanczos_max_keep()
    keep = min(kmax // b, (n_slots - 1) // 2)
    keep = max(keep, math.ceil(nev / b))
    if keep * b < nev:
        raise ValueError(f"nev={nev} needs keep_blocks*block >= nev (block={b}, n_slots={n_slots})")
    return keep


class LanczosBatch:
    """Device state of ``len(inst_sectors)`` simultaneous sector solves."""

    def __init__(self, model: DeviceModel, sset: SectorSet, inst_sectors: list[int], nev: int,
                 params: LanczosParams | None = None, block_sizes: list[int] | None = None):
        lib = _lib.lib()
        _lib.check(lib.rsed_lanczos_prepare())
        p = params or LanczosParams()
        self.p = p
        self.model = model
        self.sset = sset
        self.nev = nev
        self.inst_sectors = list(inst_sectors)
        n_inst = len(inst_sectors)
        bs = list(block_sizes) if block_sizes else [p.block] * n_inst
        bmax = max(bs)
        if bmax > lib.rsed_lanczos_max_block():
            raise ValueError("block size too large")
        if p.n_slots * bmax > lib.rsed_lanczos_max_projected():
            raise ValueError("n_slots * block exceeds the projected-matrix limit")
        self.block_sizes = bs
        self.keep = p.keep_blocks or _auto_keep(nev, min(bs), p.n_slots)
        if self.keep * bmax > lib.rsed_lanczos_max_keep():
            self.keep = max(1, lib.rsed_lanczos_max_keep() // bmax)
        if self.keep * min(bs) < nev:
            raise ValueError("nev larger than the restart basis")
        dev = model.catalog.table.device
        self.dev = dev
        n_orb = model.catalog.n_orbits
        self.n_orb = n_orb
        col0 = np.cumsum([0] + bs[:-1]).astype(np.int32)
        self.col0 = col0
        self.n_cols = int(sum(bs))
        self.ld = self.n_cols + (self.n_cols & 1)
        col_sector = np.concatenate([[s] * b for s, b in zip(inst_sectors, bs)]).astype(np.int32)
        self.col_sector = torch.from_numpy(col_sector).to(dev)
        self.inst_col0 = torch.from_numpy(col0).to(dev)
        self.inst_b = torch.tensor(bs, dtype=torch.int32, device=dev)
        S = p.n_slots
        self.pm = (S + 1) * bmax
        # reduction chunks: about 8 blocks per SM over all instances, >= 64
        # rows each and at most 256 per instance (the finalisation sums them)
        n_sm = torch.cuda.get_device_properties(dev).multi_processor_count if dev.type == "cuda" else 148
        target = min(256, max(1, (8 * n_sm) // n_inst))
        self.chunk_rows = max(64, -(-n_orb // target))
        c128 = torch.complex128
        self.V = torch.zeros((S + 2, n_orb, self.ld), dtype=c128, device=dev)
        self.W = torch.zeros((n_orb, self.ld), dtype=c128, device=dev)
        self.Xf = torch.zeros((n_orb, self.ld), dtype=torch.complex64, device=dev) if p.precision == 32 else None
        self.P = torch.zeros((n_inst, self.pm, self.pm), dtype=c128, device=dev)
        self.coef = torch.zeros(int(lib.rsed_lanczos_coef_len(n_inst, S)), dtype=torch.float64, device=dev)
        plen = int(lib.rsed_lanczos_partial_len(n_orb, self.chunk_rows, n_inst, S))
        self.partial = torch.zeros(plen, dtype=torch.float64, device=dev)
        self.ritz_val = torch.zeros((n_inst, self.pm), dtype=torch.float64, device=dev)
        self.ritz_vec = torch.zeros((n_inst, self.pm, self.pm), dtype=c128, device=dev)
        self.resid = torch.zeros((n_inst, self.pm), dtype=torch.float64, device=dev)
        self.state = torch.zeros((n_inst, STATE_INTS), dtype=torch.int32, device=dev)
        self.c = _lib.RsedLanczos(
            n_inst, S, nev, self.keep, p.max_restarts, p.precision, bmax, self.chunk_rows, self.pm,
            reserved_bits(p),
            float(p.tol if p.precision == 64 else max(p.tol, p.tol32)), _lib.ptr(self.inst_col0), _lib.ptr(self.inst_b), _lib.ptr(self.V),
            _lib.ptr(self.W), _lib.ptr(self.Xf), _lib.ptr(self.P), _lib.ptr(self.coef),
            _lib.ptr(self.partial), plen, _lib.ptr(self.ritz_val), _lib.ptr(self.ritz_vec),
            _lib.ptr(self.resid), _lib.ptr(self.state),
        )
        self.sc = sset.sectors_struct(self.col_sector, self.n_cols, self.ld)
        self.replays = 0
        self.replayed_launches = 0  # kernels launched by graph replays
        self.launches_per_graph = None
        self._graph = None
        self._graph_iters = None
        self._spans = None  # restart-aligned graphs: ((head, launches), (cycle, launches))

    @property
    def n_inst(self) -> int:
        return len(self.inst_sectors)

    # -- start ------------------------------------------------------------
    def load_start(self, blocks: list[torch.Tensor | np.ndarray | None], seeds: list[int] | None = None,
                   stream=None) -> None:
        """Place each instance's start block ``[D_s, >= b]`` (compact sector
        rows; the first ``b`` columns are used) into ``W``; ``None`` draws the
        seeded block of :func:`start_block`."""
        self.W.zero_()
        lib = _lib.lib()
        sp = _lib.stream_ptr(stream)
        for i, s in enumerate(self.inst_sectors):
            d = self.sset.dims[s]
            b = self.block_sizes[i]
            blk = blocks[i] if blocks is not None else None
            if blk is None:
                # seeded blocks are deterministic: drawn on the host once per
                # (sector, width, seed) and kept on the device for later solves
                seed = 12345 if seeds is None else seeds[i]
                key = (s, d, b, seed)
                cache = self.__dict__.setdefault("_start_cache", {})
                if key not in cache:
                    cache[key] = torch.from_numpy(start_block(d, b, seed)).to(self.dev)
                blk = cache[key]
            if isinstance(blk, np.ndarray):
                blk = torch.from_numpy(np.ascontiguousarray(blk, dtype=np.complex128))
            blk = blk.to(self.dev, torch.complex128, non_blocking=True).reshape(d, -1).contiguous()
            if blk.shape[1] < b:
                raise ValueError(f"start block of sector {s} has {blk.shape[1]} columns, the instance needs {b}")
            oor, _ = self.sset.rows(s)
            _lib.check(lib.rsed_scatter_block(d, _lib.ptr(oor), _lib.ptr(blk), b, blk.shape[1], _lib.ptr(self.W),
                                              self.ld, int(self.col0[i]), sp))

    def start(self, stream=None) -> None:
        _lib.check(_lib.lib().rsed_lanczos_start(ctypes.byref(self.model.c), ctypes.byref(self.sc),
                                                 ctypes.byref(self.c), _lib.stream_ptr(stream)))

    def iterate(self, n_iter: int = 1, stream=None) -> None:
        _lib.check(_lib.lib().rsed_lanczos_iterate(
            ctypes.byref(self.model.c), ctypes.byref(self.sc), ctypes.byref(self.c), n_iter,
            self.p.check_every, self.p.apply_variant, _lib.stream_ptr(stream)))

    def iterate_span(self, n_iter: int, ritz_last: bool, stream=None) -> None:
        """``n_iter`` steps with the Ritz check and restart after the last step
        only (``ritz_last``) or not at all; see ``restart_period``."""
        _lib.check(_lib.lib().rsed_lanczos_iterate_span(
            ctypes.byref(self.model.c), ctypes.byref(self.sc), ctypes.byref(self.c), n_iter,
            int(bool(ritz_last)), self.p.check_every, self.p.apply_variant, _lib.stream_ptr(stream)))

    def periodic_check_in(self, first: int, last: int) -> bool:
        """Whether a periodic Ritz check (every ``check_every`` iterations)
        can fall due at a step in ``first..last`` (steps counted from 1 after
        ``start()``).  The state's iteration count is 1 after ``start()`` and
        i + 1 after step i; the check of step i runs when (i + 1) is a
        multiple of ``check_every``."""
        ce = self.p.check_every
        return last >= first and (last + 1) // ce > first // ce

    @property
    def restart_period(self) -> int:
        """Steps between two thick restarts.  Every active instance adds one
        block per step, so the first restart falls due ``n_slots`` steps after
        ``start()`` and the next ones every ``n_slots - keep`` steps."""
        return self.p.n_slots - self.keep

    def status(self) -> np.ndarray:
        return self.state.cpu().numpy()

    def rayleigh_ritz(self, stream=None) -> None:
        """FP64 Rayleigh-Ritz over the restart basis of every converged
        instance; afterwards ``residuals()`` are true FP64 residual norms."""
        _lib.check(_lib.lib().rsed_lanczos_rayleigh_ritz(
            ctypes.byref(self.model.c), ctypes.byref(self.sc), ctypes.byref(self.c),
            self.p.apply_variant, _lib.stream_ptr(stream)))

    def restart(self, stream=None) -> None:
        """The thick restart alone for every instance whose ``state[:, 5]``
        (S_RESTART_NB) is nonzero: ``V_j = sum_l V_l S[l, j]`` over the old
        basis with ``S = ritz_vec``, the residual block moved behind the
        ``keep`` new blocks."""
        _lib.check(_lib.lib().rsed_lanczos_restart(ctypes.byref(self.model.c), ctypes.byref(self.sc),
                                                   ctypes.byref(self.c), _lib.stream_ptr(stream)))

    def done(self) -> bool:
        return not bool(self.state[:, S_ACTIVE].any().item())

    def run(self, max_iter: int = 12000, poll: int = 8, graph: bool = False, stream=None) -> np.ndarray:
        """Iterate until every instance converged or failed; returns the state."""
        it = 0
        g = None
        if graph:
            if getattr(self, "_graph", None) is None or self._graph_iters != poll:
                self._graph = self.capture(poll)
                self._graph_iters = poll
                it += 1  # capture() advanced every instance by one warm-up iteration
            g = self._graph
        while it < max_iter:
            if g is not None:
                g.replay()
                self.replays += 1
                self.replayed_launches += self.launches_per_graph or 0
            else:
                self.iterate(poll, stream)
            it += poll
            if self.done():
                break
        return self._final_status()

    def run_aligned(self, max_iter: int = 12000, poll: int = 8) -> np.ndarray:
        """``run(graph=True)`` from a fresh ``start()``, with the graphs cut at
        the restarts: a head graph of ``keep`` steps that launches no Ritz
        check, then a cycle graph of ``restart_period`` steps that checks (and
        restarts) after its last step only, replayed until every instance
        converged.  Convergence is only decided at restarts (unless
        ``check_every`` falls due first), so the host polls once per cycle and
        no step runs past the restart that finished the batch.  The kernels
        and their order are those of ``run`` minus the launches that find no
        check due, so the results are the same.  A periodic check that would
        fall inside a graph hands the rest of the solve to ``run``'s per-step
        path."""
        h, period = self.keep, self.restart_period
        check_inside = self.periodic_check_in
        if h < 1 or period < 1 or check_inside(1, h):
            return self.run(max_iter, poll, graph=True)
        if self._spans is None:
            self.iterate(h)  # first solve: every kernel runs once before the captures
            self._spans = (self.capture_span(h, False), self.capture_span(period, True))
        else:
            g, n = self._spans[0]
            g.replay()
            self.replays += 1
            self.replayed_launches += n
        it = h
        g, n = self._spans[1]
        converged = False
        while it < max_iter and not check_inside(it + 1, it + period - 1):
            g.replay()
            self.replays += 1
            self.replayed_launches += n
            it += period
            if self.done():
                converged = True
                break
        while not converged and it < max_iter:
            self.iterate(poll)
            it += poll
            converged = self.done()
        return self._final_status()

    def _final_status(self) -> np.ndarray:
        st = self.status()
        bad = [i for i in range(self.n_inst) if st[i, S_STATUS] != 1]
        if bad:
            code = int(st[bad[0], S_STATUS])
            if code == 0:
                code = _lib.RSED_ENOTCONV
            raise _lib.RsedError(code, f"instances {bad} did not converge (state {st[bad[0]].tolist()})")
        return st

    def run_persistent(self, cluster_size: int = 4, max_iter: int = 4000, stream=None) -> np.ndarray:
        """Whole solve in one launch (one thread-block cluster per instance);
        raises if an instance did not converge."""
        _lib.check(_lib.lib().rsed_lanczos_persistent(
            ctypes.byref(self.model.c), ctypes.byref(self.sc), ctypes.byref(self.c), int(cluster_size),
            int(max_iter), _lib.stream_ptr(stream)))
        st = self.status()
        bad = [i for i in range(self.n_inst) if st[i, S_STATUS] != 1]
        if bad:
            code = int(st[bad[0], S_STATUS]) or _lib.RSED_ENOTCONV
            raise _lib.RsedError(code, f"instances {bad} did not converge (state {st[bad[0]].tolist()})")
        return st

    def capture(self, n_iter: int, sync: bool = True):
        """CUDA graph of ``n_iter`` iterations (replayed by ``run(graph=True)``).

        Runs one real iteration first, outside the graph, on the live state.
        ``sync=False`` captures without the device-wide synchronisation that
        ``torch.cuda.graph`` performs first (work of other streams keeps
        running; the capture only records this batch's launches)."""
        self.launches_per_graph = None
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.iterate(1, s)  # warm-up outside the graph (kernel attributes, lazy loading)
        torch.cuda.current_stream().wait_stream(s)
        g, self.launches_per_graph = self._capture(lambda st: self.iterate(n_iter, st), sync)
        return g

    def capture_span(self, n_iter: int, ritz_last: bool, sync: bool = True):
        """``(graph, launches)`` of ``iterate_span(n_iter, ritz_last)``.  No
        warm-up: every kernel must have run once before (e.g. an eager first
        span of the same batch)."""
        return self._capture(lambda st: self.iterate_span(n_iter, ritz_last, st), sync)

    def _capture(self, launch, sync: bool):
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        n0 = _lib.load().rsed_launch_count()
        if sync:
            with torch.cuda.graph(g, stream=s):
                launch(s)
        else:
            with torch.cuda.stream(s):
                g.capture_begin(capture_error_mode="thread_local")
                try:
                    launch(s)
                finally:
                    g.capture_end()
        return g, int(_lib.load().rsed_launch_count() - n0)

    # -- results ----------------------------------------------------------
    def eigenvalues(self) -> np.ndarray:
        return self.ritz_val[:, : self.nev].cpu().numpy()

    def residuals(self) -> np.ndarray:
        return self.resid[:, : self.nev].cpu().numpy()

    def ritz_vectors_orbit(self, stream=None) -> torch.Tensor:
        """``U [n_inst, nev, n_orbits]`` in the orbit-row layout."""
        U = torch.zeros((self.n_inst, self.nev, self.n_orb), dtype=torch.complex128, device=self.dev)
        _lib.check(_lib.lib().rsed_lanczos_extract(ctypes.byref(self.model.c), ctypes.byref(self.sc),
                                                   ctypes.byref(self.c), _lib.ptr(U), self.n_orb,
                                                   _lib.stream_ptr(stream)))
        return U

    def eigenvectors(self, U: torch.Tensor | None = None, stream=None) -> list[torch.Tensor]:
        """Per instance ``[D_s, nev]`` eigenvectors in the sector's basis order:
        row-major views, one after the other, of one device buffer (one
        gather launch per instance)."""
        U = self.ritz_vectors_orbit(stream) if U is None else U
        lib = _lib.lib()
        sp = _lib.stream_ptr(stream)
        dims = [self.sset.dims[s] for s in self.inst_sectors]
        flat = torch.empty((sum(dims) * self.nev,), dtype=torch.complex128, device=self.dev)
        out = []
        off = 0
        for i, s in enumerate(self.inst_sectors):
            d = dims[i]
            oor, _ = self.sset.rows(s)
            vec = flat[off: off + d * self.nev].view(d, self.nev)
            _lib.check(lib.rsed_gather_block(d, _lib.ptr(oor), _lib.ptr(U[i]), self.nev, U.stride(1),
                                             _lib.ptr(vec), self.nev, sp))
            out.append(vec)
            off += d * self.nev
        return out


def vectors_to_host(vecs: list[torch.Tensor]) -> list[np.ndarray]:
    """Host copies of ``eigenvectors()``'s blocks in ONE device-to-host copy
    when they are consecutive views of one buffer (as returned), else one
    copy per block.  Device blocks land in page-locked host memory from
    torch's caching host allocator (a full-bandwidth copy with no page faults
    on fresh memory); the returned arrays are views that keep their block
    alive, and a block is reused by a later call only after every array of
    the earlier one is gone."""
    if not vecs:
        return []
    base = vecs[0]
    start = base.storage_offset()
    n = sum(v.numel() for v in vecs)
    consecutive = all(v.is_contiguous() for v in vecs) and all(
        v.untyped_storage().data_ptr() == base.untyped_storage().data_ptr() for v in vecs)
    off = start
    for v in vecs:
        consecutive = consecutive and v.storage_offset() == off
        off += v.numel()
    if not consecutive:
        return [v.cpu().numpy() for v in vecs]
    src = base.as_strided((n,), (1,), start)
    if src.is_cuda:
        pinned = torch.empty(n, dtype=src.dtype, pin_memory=True)
        pinned.copy_(src)
        h = pinned.numpy()
    else:
        h = src.numpy()
    out, off = [], 0
    for v in vecs:
        out.append(h[off: off + v.numel()].reshape(v.shape))
        off += v.numel()
    return out


def refine(batch: LanczosBatch) -> LanczosBatch:
    """FP64 finish of an FP32-matvec solve (in place): Rayleigh-Ritz with the
    FP64 operator over the thick-restart basis; returns the same batch."""
    batch.rayleigh_ritz()
    return batch


# ---------------------------------------------------------------------------
# reference API
# ---------------------------------------------------------------------------


def diagonalize_block_dense(H, *, nev: int = 5):
    """Dense Hermitian solve of a small block on its UPPER triangle
    (``symmetry_resolved_ed.py:2180-2211``); runs ``zheevd`` on the GPU."""
    n = H.shape[0]
    if n == 0:
        return np.zeros(0, dtype=np.float64), np.zeros((0, 0), dtype=np.complex128)
    dense = H.toarray() if hasattr(H, "toarray") else np.asarray(H)
    A = torch.from_numpy(np.ascontiguousarray(dense, dtype=np.complex128)).to(
        torch.device("cuda", torch.cuda.current_device()))
    vals, vecs = torch.linalg.eigh(A, UPLO="U")
    k = min(nev, n)
    return vals[:k].cpu().numpy().real, vecs[:, :k].cpu().numpy()


def _solve_sector(model: DeviceModel, sset: SectorSet, s: int, nev: int, params: LanczosParams):
    b = LanczosBatch(model, sset, [s], nev, params)
    b.load_start(None)
    b.start()
    b.run()
    if params.precision == 32:
        refine(b)
    vals = b.eigenvalues()[0]
    vecs = b.eigenvectors()[0]
    return vals, vecs


def _csr_lanczos(csr, nev: int, *, tol: float = 1e-10, m: int | None = None, max_restarts: int = 500,
                 seed: int = 12345):
    """Lowest ``nev`` eigenpairs of a device CSR block (``DeviceCSR``) by
    thick-restart Lanczos with full FP64 reorthogonalisation (classical
    Gram-Schmidt applied twice), all on the GPU; the start vector is the
    reference's ``v0`` (``default_rng(12345)`` complex normal).  The Ritz
    problem is the Hermitian part of the projected matrix, as in the batched
    solver; convergence is ``||r_j|| <= tol * max(1, |theta_j|)``."""
    n = csr.n
    dev = csr.val.device
    m = min(n - 1, m or max(2 * nev + 16, 40))
    keep = max(nev, min(m - 2, nev + (m - nev) // 2))
    V = torch.zeros((m + 1, n), dtype=torch.complex128, device=dev)
    T = torch.zeros((m + 1, m), dtype=torch.complex128, device=dev)
    V[0] = torch.from_numpy(start_block(n, 1, seed)[:, 0]).to(dev)
    j0 = 0
    for _ in range(max_restarts):
        for j in range(j0, m):
            w = csr.matvec(V[j])
            Vj = V[: j + 1]
            c = Vj.conj() @ w
            w = w - Vj.T @ c
            c2 = Vj.conj() @ w
            w = w - Vj.T @ c2
            T[: j + 1, j] = c + c2
            beta = torch.linalg.vector_norm(w)
            T[j + 1, j] = beta
            if float(beta) <= 1e-14 * max(1.0, float(torch.linalg.vector_norm(c + c2))):
                # invariant subspace: continue from a random vector orthogonal to V
                g = torch.Generator(device=dev).manual_seed(seed + j)
                w = torch.randn(n, dtype=torch.complex128, device=dev, generator=g)
                for _ in range(2):
                    w = w - Vj.T @ (Vj.conj() @ w)
                T[j + 1, j] = 0
                beta = torch.linalg.vector_norm(w)
            V[j + 1] = w / beta
        A = T[:m, :m]
        A = 0.5 * (A + A.conj().T)
        theta, Y = torch.linalg.eigh(A)
        bm = T[m, m - 1]
        resid = (bm.abs() * Y[m - 1, :].abs()).cpu().numpy()
        th = theta.cpu().numpy()
        if np.all(resid[:nev] <= tol * np.maximum(1.0, np.abs(th[:nev]))):
            U = Y[:, :nev].T @ V[:m]
            return th[:nev].copy(), U.T.contiguous().cpu().numpy()
        # thick restart: the lowest `keep` Ritz vectors plus the residual vector
        Vk = Y[:, :keep].T @ V[:m]
        V[:keep] = Vk
        V[keep] = V[m]
        coupling = bm * Y[m - 1, :keep]
        T.zero_()
        T[torch.arange(keep), torch.arange(keep)] = theta[:keep].to(torch.complex128)
        T[keep, :keep] = coupling
        T[:keep, keep] = coupling.conj()
        j0 = keep
    raise _lib.RsedError(_lib.RSED_ENOTCONV, f"CSR Lanczos did not converge in {max_restarts} restarts")


def diagonalize_block_arpack(H, *, nev: int = 5, params: LanczosParams | None = None,
                             basis=None, model: DeviceModel | None = None):
    """Lowest ``nev`` eigenpairs of a sector block, ascending: dense for
    ``n <= 500`` (``diagonalize_block_dense``), else a device Lanczos
    (``symmetry_resolved_ed.py:2214-2245``).  With the block's ``basis`` and
    device ``model`` the batched block Lanczos streams the projection table;
    a bare CSR block (scipy or ``DeviceCSR``) is solved by a thick-restart
    Lanczos on the device CSR."""
    n = H.shape[0] if hasattr(H, "shape") else H.n
    if n == 0:
        return np.zeros(0, dtype=np.float64), np.zeros((0, 0), dtype=np.complex128)
    if n <= 500:
        return diagonalize_block_dense(H.to_dense().cpu().numpy() if hasattr(H, "to_dense") else H, nev=nev)
    if basis is not None and model is not None:
        vals, vecs = _solve_sector(model, basis.sector_set, basis.sector_index, nev, params or LanczosParams())
        return vals, vecs.cpu().numpy()
    from .hamiltonian import DeviceCSR

    csr = H if isinstance(H, DeviceCSR) else _scipy_to_device_csr(H)
    return _csr_lanczos(csr, min(nev, n - 1), tol=(params or LanczosParams()).tol)


def _scipy_to_device_csr(H):
    from .hamiltonian import DeviceCSR

    c = H.tocoo()
    dev = torch.device("cuda", torch.cuda.current_device())
    return DeviceCSR(torch.from_numpy(c.row.astype(np.int64)).to(dev), torch.from_numpy(c.col.astype(np.int64)).to(dev),
                     torch.from_numpy(np.ascontiguousarray(c.data, dtype=np.complex128)).to(dev), H.shape[0])


def diagonalize_block_matrixfree(H_op, n: int, *, nev: int = 5, params: LanczosParams | None = None):
    """Lowest ``nev`` eigenpairs of a matrix-free sector operator
    (``symmetry_resolved_ed.py:2248-2299``).  ``n <= 500``: the dense block
    (the operator's exact CSR, which is what the reference obtains by applying
    ``H_op`` to the unit vectors) solved on its upper triangle like the
    reference's ``eigh(UPLO="U")``; larger sectors use the device block
    Lanczos over the projection table."""
    if n == 0:
        return np.zeros(0, dtype=np.float64), np.zeros((0, 0), dtype=np.complex128)
    if n <= 500:
        A = H_op.csr().to_dense()
        vals, vecs = torch.linalg.eigh(A, UPLO="U")
        k = min(nev, n)
        return vals[:k].cpu().numpy().real, vecs[:, :k].cpu().numpy()
    params = params or LanczosParams()
    vals, vecs = _solve_sector(H_op.model, H_op.basis.sector_set, H_op.basis.sector_index, nev, params)
    return vals, vecs.cpu().numpy()
