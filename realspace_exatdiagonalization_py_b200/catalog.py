"""Orbit-stabilizer catalog, resident in HBM.

Replaces ``build_symmetry_orbit_catalog`` / ``Symmetry_Orbit_Catalog`` /
``update_orbit_stabilizer_phases`` (``symmetry_resolved_ed.py:1151-1404``).
The tables are built and updated by the K1-K4 kernels of ``librsed.so``; the
reference's list/array fields are exposed as lazily materialised host
copies, so code that reads ``catalog.rep_rank_table`` or
``catalog.representative_mask_list`` keeps working.
"""

from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _lib
from .symmetry import (
    LIN_TABLE_MAX_N_SITE,
    MAX_N_SITE_UINT64,
    Finite_Symmetry_Group,
    Particle_Statistics,
    _binom_table,
    _lin_table,
    group_arrays,
    group_order,
    rank_combination,
    rank_two_species,
)

__all__ = [
    "Symmetry_Orbit_Catalog",
    "build_symmetry_orbit_catalog",
    "update_orbit_stabilizer_phases",
]


def _device():
    _lib.lib()
    return torch.device("cuda", torch.cuda.current_device())


class DeviceGroup:
    """Group tables uploaded for the kernels (``rsed_group_t``)."""

    def __init__(self, G: Finite_Symmetry_Group, n_filled: int, stats: Particle_Statistics,
                 binom_dev: torch.Tensor | None = None, species: tuple[int, int] | None = None):
        dev = _device()
        self.group = G
        self.n_site = G.n_site
        self.n_filled = n_filled
        self.n_group = group_order(G)
        self.fermionic = stats is Particle_Statistics.FERMIONIC
        # species = (mask of species-B sites, particles on them) or None
        self.species_b, self.n_filled_b = species if species else (0, 0)
        if self.species_b:
            nb = int(self.species_b).bit_count()
            self.c_b = math.comb(nb, self.n_filled_b)
            self.n_states = math.comb(self.n_site - nb, n_filled - self.n_filled_b) * self.c_b
        else:
            self.c_b = 1
            self.n_states = math.comb(self.n_site, n_filled)
        perm0, eta, angle = group_arrays(G)
        self.binom_host = _binom_table(self.n_site, n_filled)
        self.binom = binom_dev if binom_dev is not None else torch.from_numpy(self.binom_host).to(dev)
        self.perm = torch.from_numpy(perm0).to(dev)
        self.eta = torch.from_numpy(eta).to(dev)
        self.angle = torch.from_numpy(angle).to(dev)
        self.c = _lib.RsedGroup(
            self.n_site, n_filled, self.n_group, int(self.fermionic), self.n_states,
            _lib.ptr(self.binom), _lib.ptr(self.perm), _lib.ptr(self.angle), _lib.ptr(self.eta),
            int(self.species_b), int(self.n_filled_b), 0,
        )


class Symmetry_Orbit_Catalog:
    """Catalog of symmetry orbits at fixed particle number, in device memory.

    Device tensors: ``table`` (int32 ``[C, 4]``: rep, g, re/im bits of the
    complex64 amplitude), ``repr_masks`` (int64 ``[n_orb]``), ``stab_mask``,
    ``stab_off`` and ``stab_phase`` (complex128).  Reference fields are
    properties computed from them on first access.
    """

    def __init__(self, symmetry_group, particle_statistics, n_filled, dgroup, table, repr_masks,
                 stab_mask, stab_off, stab_phase):
        self.symmetry_group = symmetry_group
        self.particle_statistics = particle_statistics
        self.n_filled = n_filled
        self.dgroup = dgroup
        self.table = table
        self.repr_masks = repr_masks
        self.stab_mask = stab_mask
        self.stab_off = stab_off
        self.stab_phase = stab_phase
        self.binom_table = dgroup.binom_host
        self.n_site = dgroup.n_site
        self.n_states = dgroup.n_states
        self.n_orbits = int(repr_masks.shape[0])
        self._host: dict = {}
        self._lin = None
        # bumped by every in-place amplitude update; device-side derived
        # tables (the projection table) record the version they were built at
        self.version = 0

    # -- host views --------------------------------------------------------
    def invalidate_host(self) -> None:
        self._host.clear()

    def _table_host(self) -> np.ndarray:
        if "table" not in self._host:
            self._host["table"] = self.table.cpu().numpy()
        return self._host["table"]

    @property
    def rep_rank_table(self) -> np.ndarray:
        return self._table_host()[:, 0].copy()

    @property
    def rep_sym_table(self) -> np.ndarray:
        return self._table_host()[:, 1].copy()

    @property
    def rep_amp_table(self) -> np.ndarray:
        t = self._table_host()
        return np.ascontiguousarray(t[:, 2:4]).view(np.float32).view(np.complex64).reshape(-1)

    @property
    def representative_mask_list(self) -> list[int]:
        if "reprs" not in self._host:
            self._host["reprs"] = [int(m) for m in self.repr_masks.cpu().numpy().astype(np.uint64)]
        return self._host["reprs"]

    def _stab_host(self):
        if "stab" not in self._host:
            sm = self.stab_mask.cpu().numpy().astype(np.uint64)
            off = self.stab_off.cpu().numpy()
            ph = self.stab_phase.cpu().numpy()
            gl, pl = [], []
            for o in range(self.n_orbits):
                s = int(sm[o])
                gs = [g for g in range(64) if (s >> g) & 1]
                gl.append(gs)
                pl.append([complex(v) for v in ph[off[o] : off[o + 1]]])
            self._host["stab"] = (gl, pl)
        return self._host["stab"]

    @property
    def stabilizer_order_list(self) -> list[int]:
        return [len(g) for g in self._stab_host()[0]]

    @property
    def stabilizer_g_indices_list(self) -> list[list[int]]:
        return self._stab_host()[0]

    @property
    def stabilizer_phases_list(self) -> list[list[complex]]:
        return self._stab_host()[1]

    def _lin_tables(self):
        if self._lin is None:
            if self.n_site <= LIN_TABLE_MAX_N_SITE:
                self._lin = _lin_table(self.n_site, self.n_filled)
            else:
                self._lin = (np.zeros(1, np.int64), np.zeros(1, np.int64), -1)
        return self._lin

    @property
    def lin_left(self):
        return self._lin_tables()[0]

    @property
    def lin_right(self):
        return self._lin_tables()[1]

    @property
    def lin_n_right(self):
        return self._lin_tables()[2]

    def footprint_bytes(self) -> int:
        return int(
            self.table.numel() * 4 + self.repr_masks.numel() * 8 + self.stab_mask.numel() * 8
            + self.stab_off.numel() * 8 + self.stab_phase.numel() * 16
        )

    @property
    def species(self) -> tuple[int, int] | None:
        """(species-B site mask, particles on species B) of a two-species
        basis, ``None`` for one species."""
        dg = self.dgroup
        return (dg.species_b, dg.n_filled_b) if dg.species_b else None

    def rank_of(self, m: int) -> int:
        """Table index of a basis mask."""
        dg = self.dgroup
        if dg.species_b:
            return rank_two_species(int(m), dg.species_b, self.binom_table, dg.c_b)
        return rank_combination(int(m), self.binom_table)

    def in_basis(self, m: int) -> bool:
        m = int(m)
        if m.bit_count() != self.n_filled or m >> self.n_site:
            return False
        dg = self.dgroup
        return not dg.species_b or (m & dg.species_b).bit_count() == dg.n_filled_b

    def clone(self) -> "Symmetry_Orbit_Catalog":
        """Independent copy of the flux-dependent parts (table, stabilizer
        phases); the representative list and stabilizer masks are shared."""
        return Symmetry_Orbit_Catalog(
            self.symmetry_group, self.particle_statistics, self.n_filled, self.dgroup,
            self.table.clone(), self.repr_masks, self.stab_mask, self.stab_off,
            self.stab_phase.clone(),
        )

    def __repr__(self) -> str:  # pragma: no cover - cosmetic
        return (f"Symmetry_Orbit_Catalog(n_site={self.n_site}, n_filled={self.n_filled}, "
                f"|G|={self.dgroup.n_group}, n_orbits={self.n_orbits})")


def build_symmetry_orbit_catalog(
    *,
    second_quantized_model,
    n_filled: int,
    symmetry_group: Finite_Symmetry_Group,
    particle_statistics: Particle_Statistics,
    stream=None,
    species: tuple[list[int], int] | None = None,
) -> Symmetry_Orbit_Catalog:
    """Partition the fixed-filling Hilbert space into orbits on the GPU.

    Same contract as the reference (``symmetry_resolved_ed.py:1298-1404``):
    asserts ``symmetry_group.n_site == lattice.n_site``, ``ValueError`` above
    63 sites; the tables equal the reference's bit for bit (integer tables
    exactly, complex64 amplitudes to the last bit of ``sincos``).

    ``species = (sites_b, n_filled_b)`` (1-based sites) fixes the particle
    number on those sites as well (e.g. spin-down orbitals at fixed N_down):
    the basis is then the product of two fixed-filling spaces, ranked
    ``rank_A * C(|B|, n_filled_b) + rank_B``.  Every group element must map
    the species-B sites onto themselves.
    """
    n_site = symmetry_group.n_site
    assert n_site == second_quantized_model.lattice.n_site, (
        "build_symmetry_orbit_catalog: symmetry_group.n_site must equal lattice.n_site."
    )
    if n_site > MAX_N_SITE_UINT64:
        raise ValueError(
            f"n_site = {n_site} exceeds the 64-bit kernel limit ({MAX_N_SITE_UINT64}); "
            "use a smaller system."
        )
    assert 0 <= n_filled <= n_site
    lib = _lib.lib()
    dev = _device()
    sp_mask = _species_mask(species, symmetry_group, n_site, n_filled)
    dg = DeviceGroup(symmetry_group, n_filled, particle_statistics, species=sp_mask)
    sp = _lib.stream_ptr(stream)
    nbytes = lib.rsed_catalog_scratch_bytes(ctypes.byref(dg.c))
    scratch = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=dev)
    n_orb = ctypes.c_int64(0)
    _lib.check(lib.rsed_catalog_count(ctypes.byref(dg.c), _lib.ptr(scratch), scratch.numel(),
                                      ctypes.byref(n_orb), sp))
    n_orb = int(n_orb.value)
    repr_masks = torch.empty(n_orb, dtype=torch.int64, device=dev)
    table = torch.empty((dg.n_states, 4), dtype=torch.int32, device=dev)
    stab_mask = torch.empty(n_orb, dtype=torch.int64, device=dev)
    _lib.check(lib.rsed_catalog_fill(ctypes.byref(dg.c), _lib.ptr(scratch), scratch.numel(), n_orb,
                                     _lib.ptr(repr_masks), _lib.ptr(table), _lib.ptr(stab_mask), sp))
    del scratch
    sbytes = lib.rsed_stab_scratch_bytes(n_orb)
    scratch = torch.empty(max(int(sbytes), 256), dtype=torch.uint8, device=dev)
    stab_off = torch.empty(n_orb + 1, dtype=torch.int64, device=dev)
    n_stab = ctypes.c_int64(0)
    _lib.check(lib.rsed_catalog_stab_count(n_orb, _lib.ptr(stab_mask), _lib.ptr(stab_off),
                                           ctypes.byref(n_stab), _lib.ptr(scratch), scratch.numel(), sp))
    stab_phase = torch.empty(int(n_stab.value), dtype=torch.complex128, device=dev)
    _lib.check(lib.rsed_catalog_stab(ctypes.byref(dg.c), n_orb, _lib.ptr(repr_masks),
                                     _lib.ptr(stab_mask), _lib.ptr(stab_off), _lib.ptr(stab_phase), sp))
    return Symmetry_Orbit_Catalog(symmetry_group, particle_statistics, n_filled, dg, table,
                                  repr_masks, stab_mask, stab_off, stab_phase)


def _species_mask(species, G: Finite_Symmetry_Group, n_site: int, n_filled: int):
    if not species:
        return None
    sites, kb = species
    sb = 0
    for i in sites:
        if not 1 <= int(i) <= n_site:
            raise ValueError(f"species site {i} outside 1..{n_site}")
        sb |= 1 << (int(i) - 1)
    nb = sb.bit_count()
    if not (0 < nb < n_site and 0 <= kb <= nb and 0 <= n_filled - kb <= n_site - nb):
        raise ValueError("species: particle numbers do not fit the two site sets")
    for op in G.operations:
        img = 0
        for i in range(n_site):
            if (sb >> i) & 1:
                img |= 1 << (int(op.perm[i]) - 1)
        if img != sb:
            raise ValueError(f"symmetry operation {op.label!r} mixes the two species")
    return sb, int(kb)


def update_orbit_stabilizer_phases(
    catalog: Symmetry_Orbit_Catalog,
    new_group: Finite_Symmetry_Group,
    particle_statistics: Particle_Statistics,
    stream=None,
) -> Symmetry_Orbit_Catalog:
    """In-place phase update for a group with the same permutations
    (``symmetry_resolved_ed.py:1220-1269``); no-op for the same group object."""
    if catalog.symmetry_group is new_group:
        return catalog
    old = catalog.symmetry_group
    if group_order(new_group) != group_order(old) or any(
        a.perm != b.perm for a, b in zip(old.operations, new_group.operations)
    ):
        raise ValueError("update_orbit_stabilizer_phases: the new group must have the same permutations.")
    lib = _lib.lib()
    dg = DeviceGroup(new_group, catalog.n_filled, particle_statistics, binom_dev=catalog.dgroup.binom,
                     species=catalog.species)
    err = torch.zeros(1, dtype=torch.int32, device=catalog.table.device)
    sp = _lib.stream_ptr(stream)
    _lib.check(lib.rsed_phase_update(
        ctypes.byref(dg.c), catalog.n_orbits, _lib.ptr(catalog.repr_masks), _lib.ptr(catalog.stab_mask),
        _lib.ptr(catalog.stab_off), _lib.ptr(catalog.stab_phase), _lib.ptr(catalog.table),
        _lib.ptr(err), sp))
    if int(err.item()) != 0:
        raise ValueError("update_orbit_stabilizer_phases: catalog does not match the group.")
    catalog.symmetry_group = new_group
    catalog.dgroup = dg
    catalog.version += 1
    catalog.invalidate_host()
    return catalog
