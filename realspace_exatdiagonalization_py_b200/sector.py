"""Symmetry sectors on the device.

``SectorSet`` runs the compatibility filter (``_is_orbit_compatible``,
``symmetry_resolved_ed.py:1484-1512``) for up to 64 irreps in one launch and
keeps the per-orbit membership bitmask that the batched matrix-free apply and
Lanczos use.  ``Symmetry_Sector_Basis`` / ``build_symmetry_sector_basis`` keep
the reference's single-sector API (``:1444-1546``) with device-side row maps;
``CanonicalMap`` / ``get_canonical`` / ``project_to_sector`` keep the scalar
lookup API (``:1554-1716``).
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .catalog import Symmetry_Orbit_Catalog
from .symmetry import (
    COMPLEX_ONE,
    OneDim_Irrep,
    Particle_Statistics,
    get_canonical_representative,
    group_order,
    rank_combination,
)

__all__ = [
    "SectorSet",
    "Symmetry_Sector_Basis",
    "build_symmetry_sector_basis",
    "CanonicalMap",
    "get_canonical",
    "populate_canonical_map",
    "project_to_sector",
    "project_to_unnormalized_sector",
]


class SectorSet:
    """Membership of every orbit in each of ``len(irreps) <= 64`` sectors."""

    def __init__(self, catalog: Symmetry_Orbit_Catalog, irreps: list[OneDim_Irrep], *,
                 atol: float = 1e-12, stream=None):
        if not 1 <= len(irreps) <= 64:
            raise ValueError("SectorSet holds between 1 and 64 irreps")
        lib = _lib.lib()
        dev = catalog.table.device
        self.catalog = catalog
        self.irreps = list(irreps)
        self.atol = atol
        n_g = group_order(catalog.symmetry_group)
        chi = np.stack([np.asarray(ir.values, dtype=np.complex128) for ir in irreps])
        if chi.shape[1] != n_g:
            raise ValueError("irrep values must have one entry per group element")
        self.chi = torch.from_numpy(chi).to(dev)
        n_orb = catalog.n_orbits
        self.member = torch.empty(n_orb, dtype=torch.int64, device=dev)
        self.sqrt_stab = torch.empty(n_orb, dtype=torch.float64, device=dev)
        dims = torch.empty(len(irreps), dtype=torch.int64, device=dev)
        _lib.check(lib.rsed_sector_members(
            n_orb, n_g, len(irreps), _lib.ptr(catalog.stab_mask), _lib.ptr(catalog.stab_off),
            _lib.ptr(catalog.stab_phase), _lib.ptr(self.chi), float(atol), _lib.ptr(self.member),
            _lib.ptr(self.sqrt_stab), _lib.ptr(dims), _lib.stream_ptr(stream)))
        self.dims = [int(v) for v in dims.cpu().tolist()]
        self._rows: dict[int, tuple[torch.Tensor, torch.Tensor]] = {}

    @property
    def n_sectors(self) -> int:
        return len(self.irreps)

    def rows(self, s: int, stream=None) -> tuple[torch.Tensor, torch.Tensor]:
        """(orbit_of_row int32 [D_s], row_of_orbit int32 [n_orb]) of sector ``s``."""
        if s not in self._rows:
            lib = _lib.lib()
            dev = self.member.device
            n_orb = self.catalog.n_orbits
            d = self.dims[s]
            oor = torch.empty(max(d, 1), dtype=torch.int32, device=dev)
            roo = torch.empty(n_orb, dtype=torch.int32, device=dev)
            nbytes = lib.rsed_sector_scratch_bytes(n_orb, 1)
            scratch = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)
            _lib.check(lib.rsed_sector_rows(n_orb, _lib.ptr(self.member), s, _lib.ptr(oor),
                                            _lib.ptr(roo), _lib.ptr(scratch), scratch.numel(),
                                            _lib.stream_ptr(stream)))
            self._rows[s] = (oor[:d], roo)
        return self._rows[s]

    def sectors_struct(self, col_sector: torch.Tensor, n_cols: int, ld: int) -> _lib.RsedSectors:
        return _lib.RsedSectors(self.n_sectors, n_cols, ld, group_order(self.catalog.symmetry_group),
                                _lib.ptr(self.member), _lib.ptr(self.sqrt_stab), _lib.ptr(self.chi),
                                _lib.ptr(col_sector))


class Symmetry_Sector_Basis:
    """Sector basis of one irrep (reference fields as lazy host views)."""

    def __init__(self, irrep: OneDim_Irrep, catalog: Symmetry_Orbit_Catalog, sset: SectorSet,
                 index: int = 0):
        self.irrep = irrep
        self.symmetry_group = catalog.symmetry_group
        self.catalog = catalog
        self.sector_set = sset
        self.sector_index = index
        self.dim = sset.dims[index]
        self._host: dict = {}

    def device_rows(self):
        return self.sector_set.rows(self.sector_index)

    @property
    def orbit_of_row(self) -> torch.Tensor:
        return self.device_rows()[0]

    @property
    def representative_mask_list(self) -> list[int]:
        if "reprs" not in self._host:
            if self.dim == 0:
                self._host["reprs"] = []
            else:
                o = self.orbit_of_row.long()
                m = self.catalog.repr_masks[o].cpu().numpy().astype(np.uint64)
                self._host["reprs"] = [int(v) for v in m]
        return self._host["reprs"]

    @property
    def stabilizer_order_list(self) -> list[int]:
        if "stab" not in self._host:
            if self.dim == 0:
                self._host["stab"] = []
            else:
                o = self.orbit_of_row.long()
                s = self.catalog.stab_mask[o].cpu().numpy().astype(np.uint64)
                self._host["stab"] = [int(v).bit_count() for v in s]
        return self._host["stab"]

    @property
    def representative_mask_to_mask_idx_map(self) -> dict[int, int]:
        if "map" not in self._host:
            self._host["map"] = {m: i for i, m in enumerate(self.representative_mask_list)}
        return self._host["map"]

    def __len__(self) -> int:
        return self.dim


def build_symmetry_sector_basis(catalog: Symmetry_Orbit_Catalog, irrep: OneDim_Irrep, *,
                                atol: float = 1e-12) -> Symmetry_Sector_Basis:
    """Orbits compatible with ``irrep`` (``|chi(h) - alpha_h| <= atol`` on the
    stabilizer), in catalog order (``symmetry_resolved_ed.py:1515-1546``)."""
    sset = SectorSet(catalog, [irrep], atol=atol)
    return Symmetry_Sector_Basis(irrep, catalog, sset, 0)


def _basis_index(basis: Symmetry_Sector_Basis, repr_mask: int):
    return basis.representative_mask_to_mask_idx_map.get(repr_mask)


class CanonicalMap:
    """O(1) canonical lookup backed by the device catalog (``:1554-1592``)."""

    def __init__(self, symmetry_group, particle_statistics: Particle_Statistics,
                 catalog: Symmetry_Orbit_Catalog):
        self.symmetry_group = symmetry_group
        self.particle_statistics = particle_statistics
        self.catalog = catalog
        self._stats_flag = particle_statistics is Particle_Statistics.FERMIONIC

    def __len__(self) -> int:
        return self.catalog.n_states


def get_canonical(cmap: CanonicalMap, m: int) -> tuple[int, int, complex]:
    """``(repr, g, alpha)`` of a fixed-filling mask: rank + one table read
    (``symmetry_resolved_ed.py:1595-1632``); other masks fall back to the
    O(|G|) scan as in the reference."""
    cat = cmap.catalog
    if not cat.in_basis(m):
        return get_canonical_representative(m, cmap.symmetry_group, cmap.particle_statistics)
    idx = cat.rank_of(m)
    e = cat.table[idx].cpu().numpy()
    rep = int(e[0])
    if rep < 0:
        return get_canonical_representative(m, cmap.symmetry_group, cmap.particle_statistics)
    amp = np.ascontiguousarray(e[2:4]).view(np.float32)
    return int(cat.repr_masks[rep].item()) & ((1 << 64) - 1), int(e[1]), complex(
        np.complex64(complex(float(amp[0]), float(amp[1])))
    )


def populate_canonical_map(cmap: CanonicalMap, basis, bilinear_terms) -> CanonicalMap:
    """No-op kept for API compatibility (tables are prebuilt, ``:1635-1654``)."""
    return cmap


def project_to_sector(m: int, basis: Symmetry_Sector_Basis, cmap: CanonicalMap):
    """``(row, alpha * conj(chi(g)))`` or ``None`` (``:1662-1690``)."""
    rep, g, alpha = get_canonical(cmap, m)
    idx = _basis_index(basis, rep)
    if idx is None:
        return None
    return idx, alpha * np.conj(basis.irrep.values[g])


def project_to_unnormalized_sector(m: int, basis: Symmetry_Sector_Basis,
                                   stats: Particle_Statistics = Particle_Statistics.BOSONIC):
    """Uncached projection (``:1693-1716``)."""
    rep, g, alpha = get_canonical_representative(m, basis.symmetry_group, stats)
    idx = _basis_index(basis, rep)
    if idx is None:
        return None
    return idx, alpha * np.conj(basis.irrep.values[g])
