"""Matrix-free and matrix-mode Hamiltonians on the device.

* ``DeviceModel``: bilinear terms grouped by annihilated site (the hop loop
  of the apply kernel visits only occupied sites), density diagonal per orbit.
* ``MatrixFreeHamiltonian`` / ``hamiltonian_linear_operator`` /
  ``apply_hamiltonian``: the reference's operator API
  (``symmetry_resolved_ed.py:1884-2094``), ``y = H x`` from the sector's
  exact CSR block; the eigen-solvers stream the K6b projection table instead.
* ``build_ed_Hamiltonian_symmetry_block``: matrix mode (``:2102-2174``), with
  the triplets produced by the K7 kernel.

Term semantics follow the reference's code: ``(i, j, t)`` annihilates at
``i`` and creates at ``j`` (gate ``symmetry_resolved_ed.py:656``, XOR ``:660``).
"""

from __future__ import annotations

import ctypes

import numpy as np
import scipy.sparse as sp
import torch

from . import _lib
from .catalog import Symmetry_Orbit_Catalog
from .sector import SectorSet, Symmetry_Sector_Basis
from .symmetry import Particle_Statistics, group_order, hopping_phase_for_stats

__all__ = [
    "DeviceModel",
    "MatrixFreeHamiltonian",
    "hamiltonian_linear_operator",
    "apply_hamiltonian",
    "apply_hamiltonian_with_threads",
    "build_ed_Hamiltonian_symmetry_block",
    "build_matrixfree_projection_table",
    "hopping_phase_for_stats",
]


def _merge_terms(bilinear_terms, n_site, merge: bool = True):
    """Group directed terms by source site.  ``merge``: duplicate (i, j)
    amplitudes add (one hop per site pair, what the solvers stream);
    otherwise every term stays its own entry, in input order within a site
    pair (one triplet per term, as the reference's per-term builder emits)."""
    acc: dict[tuple[int, ...], complex] = {}
    order: list[tuple[int, ...]] = []
    for n_in, (i, j, t) in enumerate(bilinear_terms):
        i, j = int(i), int(j)
        if not (1 <= i <= n_site and 1 <= j <= n_site):
            raise ValueError(f"bilinear term ({i}, {j}) outside sites 1..{n_site}")
        if i == j:
            raise ValueError(
                f"bilinear term ({i}, {i}) is on-site; put on-site energies in the density terms"
            )
        key = (i - 1, j - 1) if merge else (i - 1, j - 1, n_in)
        if key not in acc:
            acc[key] = 0j
            order.append(key)
        acc[key] += complex(t)
    keys = sorted(order)  # by source site, then target (then input order)
    begin = np.zeros(n_site + 1, dtype=np.int32)
    for k in keys:
        begin[k[0] + 1] += 1
    begin = np.cumsum(begin).astype(np.int32)
    to = np.array([k[1] for k in keys], dtype=np.uint8)
    amp = np.array([acc[k] for k in keys], dtype=np.complex128)
    jw = np.zeros(len(keys), dtype=np.uint64)
    for n, (i, j, *_) in enumerate(keys):
        lo, hi = min(i, j), max(i, j)
        jw[n] = np.uint64(((1 << (hi - lo - 1)) - 1) << (lo + 1)) if hi - lo > 1 else np.uint64(0)
    return begin, to, amp, jw


class DeviceModel:
    """Hamiltonian terms of one model on one catalog (``rsed_model_t``)."""

    def __init__(self, catalog: Symmetry_Orbit_Catalog, bilinear_terms, density_terms, stream=None,
                 merge_terms: bool = True):
        lib = _lib.lib()
        dev = catalog.table.device
        n_site = catalog.n_site
        self.catalog = catalog
        self.bilinear_terms = [(int(i), int(j), complex(t)) for (i, j, t) in bilinear_terms]
        self.density_terms = [(int(i), int(j), complex(v)) for (i, j, v) in density_terms]
        begin, to, amp, jw = _merge_terms(self.bilinear_terms, n_site, merge_terms)
        self.n_terms = int(len(to))
        self.term_begin = torch.from_numpy(begin).to(dev)
        self.term_to = torch.from_numpy(to if len(to) else np.zeros(1, np.uint8)).to(dev)
        self.term_amp = torch.from_numpy(amp if len(amp) else np.zeros(1, np.complex128)).to(dev)
        self.term_jw = torch.from_numpy(jw.view(np.int64) if len(jw) else np.zeros(1, np.int64)).to(dev)
        nd = len(self.density_terms)
        di = np.array([t[0] - 1 for t in self.density_terms] or [0], dtype=np.uint8)
        dj = np.array([t[1] - 1 for t in self.density_terms] or [0], dtype=np.uint8)
        dv = np.array([t[2] for t in self.density_terms] or [0j], dtype=np.complex128)
        if nd and (di.max() >= n_site or dj.max() >= n_site):
            raise ValueError("density term outside the lattice")
        self._di, self._dj, self._dv = (torch.from_numpy(a).to(dev) for a in (di, dj, dv))
        self.hdiag = torch.empty(catalog.n_orbits, dtype=torch.complex128, device=dev)
        _lib.check(lib.rsed_density_diag(catalog.n_orbits, _lib.ptr(catalog.repr_masks), nd,
                                         _lib.ptr(self._di), _lib.ptr(self._dj), _lib.ptr(self._dv),
                                         _lib.ptr(self.hdiag), _lib.stream_ptr(stream)))
        self.proj = None
        self.refresh()

    def refresh(self) -> None:
        """Rebuild the C descriptor (after an in-place catalog update, which
        also drops the projection table built from the old amplitudes)."""
        cat = self.catalog
        dg = cat.dgroup
        if self.proj is not None and self.proj["table_version"] != cat.version:
            self.proj = None
        pj = self.proj or {}
        self.c = _lib.RsedModel(
            dg.n_site, dg.n_filled, dg.n_group, int(dg.fermionic), dg.n_states, cat.n_orbits,
            _lib.ptr(dg.binom), _lib.ptr(cat.table), _lib.ptr(cat.repr_masks), self.n_terms,
            _lib.ptr(self.term_begin), _lib.ptr(self.term_to), _lib.ptr(self.term_amp),
            _lib.ptr(self.term_jw), _lib.ptr(self.hdiag),
            _lib.ptr(pj.get("rowptr")), _lib.ptr(pj.get("cg")), _lib.ptr(pj.get("w64")),
            _lib.ptr(pj.get("w32")), int(dg.species_b), int(dg.n_filled_b), 0,
        )

    def projection_bytes(self, precisions=(64, 32)) -> int:
        """Device bytes of the projection table (exact hop count; one pass)."""
        if self.proj is not None:
            skip = ("rowptr", "cg") if self.proj.get("shared") else ()
            return sum(int(t.numel() * t.element_size()) for k, t in self.proj.items()
                       if torch.is_tensor(t) and k not in skip)
        n = self.count_hops()
        return 8 * (self.catalog.n_orbits + 1) + n * (4 + (16 if 64 in precisions else 0)
                                                      + (8 if 32 in precisions else 0))

    def count_hops(self, stream=None) -> int:
        """Hops over all orbit rows (the projection table's entry count)."""
        lib = _lib.lib()
        n_orb = self.catalog.n_orbits
        dev = self.hdiag.device
        rowptr = torch.empty(n_orb + 1, dtype=torch.int64, device=dev)
        scratch = torch.empty(lib.rsed_proj_scratch_bytes(n_orb), dtype=torch.uint8, device=dev)
        n = ctypes.c_int64()
        _lib.check(lib.rsed_proj_count(ctypes.byref(self.c), _lib.ptr(rowptr), ctypes.byref(n),
                                       _lib.ptr(scratch), scratch.numel(), _lib.stream_ptr(stream)))
        self._rowptr_cache = rowptr
        return int(n.value)

    def build_projection(self, sqrt_stab: torch.Tensor, precisions=(64, 32), stream=None,
                         share: dict | None = None) -> None:
        """Build the orbit-space projection table (K6b) for the current
        catalog amplitudes; afterwards ``rsed_apply_h`` variant 0 streams it.

        ``share``: the table of another amplitude state of the same catalog
        (a copy moved to another flux point by ``update_orbit_stabilizer_phases``
        keeps every target orbit and group element); its ``rowptr`` and ``cg``
        are reused and only the weights are computed."""
        lib = _lib.lib()
        want = tuple(sorted(set(precisions)))
        if self.proj is not None and self.proj["table_version"] == self.catalog.version and \
                set(want) <= set(self.proj["precisions"]):
            return
        if share is not None:
            rowptr, cg, n = share["rowptr"], share["cg"], share["n_hops"]
            dev = rowptr.device
            w64 = torch.empty(max(n, 1), dtype=torch.complex128, device=dev) if 64 in want else None
            w32 = torch.empty(max(n, 1), dtype=torch.complex64, device=dev) if 32 in want else None
            _lib.check(lib.rsed_proj_fill(ctypes.byref(self.c), _lib.ptr(sqrt_stab), _lib.ptr(rowptr), None,
                                          _lib.ptr(w64), _lib.ptr(w32), _lib.stream_ptr(stream)))
            self.proj = {"rowptr": rowptr, "cg": cg, "w64": w64, "w32": w32, "n_hops": n, "precisions": want,
                         "table_version": self.catalog.version, "shared": True}
            self.refresh()
            return
        n = self.count_hops(stream)
        rowptr = self._rowptr_cache
        dev = rowptr.device
        cg = torch.empty(max(n, 1), dtype=torch.int32, device=dev)
        w64 = torch.empty(max(n, 1), dtype=torch.complex128, device=dev) if 64 in want else None
        w32 = torch.empty(max(n, 1), dtype=torch.complex64, device=dev) if 32 in want else None
        _lib.check(lib.rsed_proj_fill(ctypes.byref(self.c), _lib.ptr(sqrt_stab), _lib.ptr(rowptr),
                                      _lib.ptr(cg), _lib.ptr(w64), _lib.ptr(w32), _lib.stream_ptr(stream)))
        self.proj = {"rowptr": rowptr, "cg": cg, "w64": w64, "w32": w32, "n_hops": n,
                     "precisions": want, "table_version": self.catalog.version}
        self.refresh()

    def drop_projection(self) -> None:
        self.proj = None
        self.refresh()

    def apply_block(self, sset: SectorSet, col_sector: torch.Tensor, X: torch.Tensor,
                    Y: torch.Tensor, precision: int = 64, variant: int = 0, stream=None) -> None:
        """``Y = H^dagger X`` for a row-major block ``[n_orbits, ld]`` (K6)."""
        n_cols = int(col_sector.numel())
        ld = int(X.shape[1])
        sc = sset.sectors_struct(col_sector, n_cols, ld)
        _lib.check(_lib.lib().rsed_apply_h(ctypes.byref(self.c), ctypes.byref(sc), _lib.ptr(X),
                                           _lib.ptr(Y), precision, variant, _lib.stream_ptr(stream)))


class MatrixFreeHamiltonian:
    """``H_op(x) -> y = H x`` for one sector (``symmetry_resolved_ed.py:1884-1976``).

    Same constructor and call contract as the reference: ``x`` and the result
    are complex128 of length ``sector_dim`` (or ``[sector_dim, k]`` blocks);
    numpy arrays stay numpy, CUDA tensors stay on the device.  Like the
    reference, the operator is the sector block in CSR form, assembled from
    the exact projected hops and the density diagonal (K7 triplets, the
    reference's element formula and product order) and applied by
    ``rsed_csr_spmv``; the CSR is built on the first call.

    The eigen-solvers do not go through ``__call__``: they stream the
    sector-independent orbit-space projection table (``DeviceModel``,
    ``rsed_apply_h``), whose pull form yields ``H^dagger x`` -- equal to
    ``H x`` for the reference's zero-flux blocks and, for flux blocks
    (Hermitian only to the complex64 rounding of the amplitude table), with
    the same real spectrum.  ``precision=32`` makes ``__call__`` that FP32
    streaming apply (``H^dagger x`` in FP32 arithmetic).
    """

    def __init__(self, basis: Symmetry_Sector_Basis, bilinear_terms, density_terms, cmap,
                 *, precision: int = 64, model: DeviceModel | None = None):
        self.basis = basis
        self.bilinear_terms = [(i, j, complex(t)) for (i, j, t) in bilinear_terms]
        self.density_terms = [(i, j, complex(v)) for (i, j, v) in density_terms]
        self.cmap = cmap
        self.n = basis.dim
        self.precision = precision
        self.model = model or DeviceModel(basis.catalog, self.bilinear_terms, self.density_terms)
        dev = basis.catalog.table.device
        self._col_sector = torch.tensor([basis.sector_index], dtype=torch.int32, device=dev)
        self._orbit_of_row = basis.orbit_of_row if self.n else None
        self._csr: DeviceCSR | None = None

    def csr(self) -> "DeviceCSR":
        """The sector block as a device CSR matrix (built once)."""
        if self._csr is None:
            rows, cols, vals = _sector_triplets(self.basis, self.model)
            self._csr = DeviceCSR(rows, cols, vals, self.n)
        return self._csr

    def matvec_device(self, x: torch.Tensor, ncols: int = 1) -> torch.Tensor:
        """``H x`` for ``ncols`` compact column vectors ``x [n, ncols]`` on the device."""
        if self.precision == 32:
            return self.adjoint_device(x, ncols, precision=32)
        xt = x.reshape(self.n, ncols).to(torch.complex128).T.contiguous()
        return self.csr().matvec(xt).T.reshape(self.n, ncols)

    def adjoint_device(self, x: torch.Tensor, ncols: int = 1, precision: int = 64) -> torch.Tensor:
        """``H^dagger x`` through the streaming orbit-layout apply of the
        eigensolver (``rsed_apply_h``) for ``x [n, ncols]`` on the device."""
        dev = x.device
        n_orb = self.basis.catalog.n_orbits
        ld = ncols + (ncols & 1)
        X = torch.zeros((n_orb, ld), dtype=torch.complex128, device=dev)
        X[self._orbit_of_row.long(), :ncols] = x.reshape(self.n, ncols).to(torch.complex128)
        col_sector = self._col_sector.repeat(ncols)
        Y = torch.empty_like(X)
        if precision == 32:
            self.model.apply_block(self.basis.sector_set, col_sector, X.to(torch.complex64), Y, 32)
        else:
            self.model.apply_block(self.basis.sector_set, col_sector, X, Y, 64)
        return Y[self._orbit_of_row.long(), :ncols]

    def __call__(self, x):
        if self.n == 0:
            if isinstance(x, torch.Tensor):
                return torch.zeros_like(x, dtype=torch.complex128)
            return np.zeros(np.shape(x), dtype=np.complex128)
        if isinstance(x, torch.Tensor) and x.is_cuda:
            k = x.numel() // self.n
            return self.matvec_device(x, k).reshape(x.shape)
        xa = np.ascontiguousarray(x, dtype=np.complex128)
        k = xa.size // self.n
        xt = torch.from_numpy(xa.reshape(self.n, k)).to(self.basis.catalog.table.device)
        y = self.matvec_device(xt, k)
        return y.cpu().numpy().reshape(xa.shape)


def hamiltonian_linear_operator(basis, bilinear_terms, density_terms, cmap):
    """``(H_op, n)`` with ``H_op(x) = H x`` (``symmetry_resolved_ed.py:2072-2094``)."""
    return MatrixFreeHamiltonian(basis, bilinear_terms, density_terms, cmap), basis.dim


def _cached_operator(basis, bilinear_terms, density_terms, cmap) -> MatrixFreeHamiltonian:
    """The sector's operator for these terms, kept on the basis object so
    that repeated ``apply_hamiltonian`` calls build the device model and the
    CSR once (the reference re-derives its lookup arrays on every call)."""
    key = (tuple((int(i), int(j), complex(t)) for (i, j, t) in bilinear_terms),
           tuple((int(i), int(j), complex(v)) for (i, j, v) in density_terms),
           basis.catalog.version)
    cache = basis.__dict__.setdefault("_operators", {})
    op = cache.get(key)
    if op is None:
        cache.clear()
        op = MatrixFreeHamiltonian(basis, bilinear_terms, density_terms, cmap)
        cache[key] = op
    return op


def apply_hamiltonian_with_threads(y, x, basis, bilinear_terms, density_terms, cmap, y_threads=None):
    """``y[:] = H x``, written into the caller's ``y`` and returned
    (``symmetry_resolved_ed.py:2011-2069``); ``y_threads`` (the reference's
    per-thread buffers) is accepted for API parity and unused."""
    n = len(x)
    assert len(y) == n, "apply_hamiltonian: y and x must have the same length"
    op = _cached_operator(basis, bilinear_terms, density_terms, cmap)
    y[:] = op(x)
    return y


def apply_hamiltonian(y, x, basis, bilinear_terms, density_terms, cmap):
    """``y[:] = H x`` (``symmetry_resolved_ed.py:1979-2008``)."""
    return apply_hamiltonian_with_threads(y, x, basis, bilinear_terms, density_terms, cmap)


def _sector_triplets(basis: Symmetry_Sector_Basis, model: DeviceModel, stream=None):
    """Device triplets (rows, cols, vals) of one sector block, diagonal included."""
    lib = _lib.lib()
    dev = basis.catalog.table.device
    n = basis.dim
    oor, roo = basis.device_rows()
    chi = torch.from_numpy(np.asarray(basis.irrep.values, dtype=np.complex128)).to(dev)
    col_off = torch.empty(n + 1, dtype=torch.int64, device=dev)
    nbytes = lib.rsed_triplet_scratch_bytes(n)
    scratch = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)
    nnz = ctypes.c_int64(0)
    sp_ = _lib.stream_ptr(stream)
    _lib.check(lib.rsed_triplets_count(ctypes.byref(model.c), n, _lib.ptr(oor), _lib.ptr(roo),
                                       _lib.ptr(chi), _lib.ptr(basis.catalog.stab_mask),
                                       _lib.ptr(col_off), ctypes.byref(nnz), _lib.ptr(scratch),
                                       scratch.numel(), sp_))
    nnz = int(nnz.value)
    rows = torch.empty(nnz, dtype=torch.int64, device=dev)
    cols = torch.empty(nnz, dtype=torch.int64, device=dev)
    vals = torch.empty(nnz, dtype=torch.complex128, device=dev)
    _lib.check(lib.rsed_triplets_fill(ctypes.byref(model.c), n, _lib.ptr(oor), _lib.ptr(roo),
                                      _lib.ptr(chi), _lib.ptr(basis.catalog.stab_mask),
                                      _lib.ptr(col_off), _lib.ptr(rows), _lib.ptr(cols), _lib.ptr(vals),
                                      sp_))
    return rows, cols, vals


class DeviceCSR:
    """Sector block in CSR form on the device, applied by ``rsed_csr_spmv``."""

    def __init__(self, rows, cols, vals, n):
        order = torch.argsort(rows * n + cols, stable=True)
        r = rows[order]
        self.n = n
        self.col = cols[order].to(torch.int32)
        self.val = vals[order].contiguous()
        counts = torch.bincount(r, minlength=n)
        self.row_ptr = torch.zeros(n + 1, dtype=torch.int64, device=rows.device)
        self.row_ptr[1:] = torch.cumsum(counts, 0)

    def to_dense(self) -> torch.Tensor:
        """The matrix as a dense device tensor (duplicates summed)."""
        A = torch.zeros((self.n, self.n), dtype=torch.complex128, device=self.val.device)
        rows = torch.repeat_interleave(torch.arange(self.n, device=self.val.device),
                                       self.row_ptr[1:] - self.row_ptr[:-1])
        A.index_put_((rows, self.col.long()), self.val, accumulate=True)
        return A

    def matvec(self, x: torch.Tensor) -> torch.Tensor:
        """``A x_v`` for ``x [n]`` or ``x [n_vec, n]`` (vectors contiguous)."""
        x = x.to(torch.complex128).contiguous()
        nvec = 1 if x.dim() == 1 else x.shape[0]
        y = torch.empty_like(x)
        _lib.check(_lib.lib().rsed_csr_spmv(self.n, _lib.ptr(self.row_ptr), _lib.ptr(self.col),
                                            _lib.ptr(self.val), nvec, _lib.ptr(x), _lib.ptr(y),
                                            _lib.stream_ptr()))
        return y


def build_ed_Hamiltonian_symmetry_block(basis, bilinear_terms, density_terms, cmap,
                                        *, model: DeviceModel | None = None) -> sp.csr_matrix:
    """Sector block as a scipy CSR matrix, entries computed on the GPU
    (``symmetry_resolved_ed.py:2102-2174``)."""
    n = basis.dim
    if n == 0:
        return sp.csr_matrix((0, 0), dtype=np.complex128)
    model = model or DeviceModel(basis.catalog, bilinear_terms, density_terms)
    rows, cols, vals = _sector_triplets(basis, model)
    H = sp.coo_matrix((vals.cpu().numpy(), (rows.cpu().numpy(), cols.cpu().numpy())),
                      shape=(n, n)).tocsr()
    H.eliminate_zeros()
    return H


def build_matrixfree_projection_table(basis, bilinear_terms, density_terms, cmap):
    """``(row_ind, col_ind, vals, h_diag)`` of the off-diagonal projected
    hops and the diagonal (``symmetry_resolved_ed.py:1719-1769``): one
    triplet per term and valid hop, as the reference's per-term builder
    (duplicate site pairs, e.g. bonds that meet across both periodic
    boundaries of a small lattice, stay separate triplets)."""
    model = DeviceModel(basis.catalog, bilinear_terms, density_terms, merge_terms=False)
    rows, cols, vals = _sector_triplets(basis, model)
    n = basis.dim
    h_diag = model.hdiag[basis.orbit_of_row.long()]
    # the K7 triplets come column by column, each column led by its density
    # diagonal entry (rsed_triplets_fill): drop exactly that leading entry
    counts = torch.bincount(cols, minlength=n)
    starts = torch.zeros(n, dtype=torch.int64, device=rows.device)
    starts[1:] = torch.cumsum(counts, 0)[:-1]
    keep = torch.ones(rows.numel(), dtype=torch.bool, device=rows.device)
    keep[starts] = False
    return (rows[keep].cpu().numpy(), cols[keep].cpu().numpy(), vals[keep].cpu().numpy(),
            h_diag.cpu().numpy())
