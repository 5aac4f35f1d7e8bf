"""Flux-grid drivers on top of the device solvers.

``flux_spectrum_flow`` keeps the contract of the reference's driver
(``observables/spectrum_flow.py:25-169``): the lowest ``nev`` energies of the
given sectors at every flux value of a scan along one lattice direction,
returned as a ``SimpleNamespace`` with the reference's fields.  Two engines:

* ``engine="scan"`` (the reference's route): one ``ed_scan`` flux scan with a
  canonical checkpoint per flux value (reused unless ``overwrite``), every
  sector of a flux point solved in one batched launch sequence;
* ``engine="served"``: every (flux value, sector) solve is a request to a
  ``SolveServer`` -- the zero-flux catalog is built once and moved to each flux
  point by ``update_orbit_stabilizer_phases``, solves of different flux points
  overlap on the device; the results are written (and, unless ``overwrite``,
  read back) as the same per-flux-point checkpoints the scan engine uses
  (``ServedCheckpoints``: asynchronous device-to-host copies, a writer
  thread).

``many_body_chern_number`` keeps the contract of the reference's driver
(``observables/many_body_chern_number.py:341-458``): the Chern number of the
manifold spanned by the lowest ``nev_per_sector`` states of the given sectors
on an ``nx x ny`` twisted-boundary flux torus, from U(1) links (phases of the
determinants of overlap matrices between neighbouring flux points) and
plaquette phases summed over 2 pi.  Each flux point is solved like the
reference's (one ED scan of the listed sectors with a checkpoint per point,
reused unless ``overwrite``), on a phase-updated copy of the zero-flux
catalog; its manifold states are expanded into dense rank-indexed Fock
vectors on the device, and the overlap matrices of each row of links are one
device launch (``rsed_fock_overlaps``).  Only the zero-flux row and the two
most recent rows stay resident, so device memory is
``3 * ny * n_manifold * n_states * 16`` bytes, not the whole grid.  With
``engine="served"`` every (flux point, sector) solve of the grid is instead a
request to a ``SolveServer`` that returns its eigenvectors; solves of
different flux points overlap on the device, and the sector eigenvectors
(not the Fock states) of the whole grid wait on the device for the links.

``flux_charge_pump`` keeps the contract of the reference's driver
(``observables/charge_pump.py:325-558``): along a flux scan (the flux-scan
checkpoints shared with ``flux_spectrum_flow``) Resta's periodic position
operator in the transverse direction is projected into the manifold of
(sector, level) states, one device launch per pair of sectors
(``rsed_position_overlaps``: the orbit-diagonal element and the products with
every pair of levels in one stream over the orbit-layout vectors); its
eigenvalue phases are tracked branch by branch into pumped charges.
"""

from __future__ import annotations

import os
from fractions import Fraction
from types import SimpleNamespace

import numpy as np

__all__ = ["flux_spectrum_flow", "many_body_chern_number", "flux_charge_pump", "many_body_position_phases"]


def _no_figure(fig_path) -> None:
    """The drivers accept the reference's ``fig_path`` and return it in their
    results, but draw no figure: plotting is presentation, outside this
    package (the reference draws with matplotlib)."""
    if fig_path is not None:
        import warnings

        warnings.warn(f"fig_path={fig_path!r}: figures are not drawn by this package; the results carry the data",
                      stacklevel=3)


def _labels(sector_labels):
    if isinstance(sector_labels, str):
        ident = sector_labels == "identity"
        return ident, ["identity"] if ident else [sector_labels]
    if isinstance(sector_labels, tuple):
        return False, [tuple(int(x) for x in sector_labels)]
    return False, [tuple(int(x) for x in lab) for lab in sector_labels]


def flux_spectrum_flow(model, sector_labels, *, filling_fraction, flux_direction: int = 1,
                       twisted_phases_over_2π_list=None, checkpoint_dir: str = "checkpoints", nev: int = 3,
                       fig_path: str | None = None, overwrite: bool = False, engine: str = "scan",
                       precision: int = 32):
    from .ed import build_ed_data, ed_scan, load_checkpoint
    from .second_quantized_model import update_second_quantized_model_with_twisted_phases
    from .symmetry import build_irrep_list, build_translation_group

    if twisted_phases_over_2π_list is None:
        twisted_phases_over_2π_list = list(np.linspace(0.0, 1.0, 9))
    thetas = [float(t) for t in twisted_phases_over_2π_list]
    is_identity, labels = _labels(sector_labels)
    dim = model.lattice.dim
    if not 1 <= flux_direction <= dim:
        raise ValueError(f"flux_direction must be in 1..{dim}")
    flux0 = [0.0] * dim
    update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=flux0)
    if not isinstance(filling_fraction, Fraction):
        filling_fraction = Fraction(filling_fraction)
    energies = np.full((len(thetas), len(labels), nev), np.nan)
    checkpoint_paths = None
    if engine == "scan":
        if is_identity:
            raise ValueError("the identity sector is served by full_ed, not by a translation flux scan")
        init = build_ed_data(model, filling_fraction=filling_fraction,
                             symmetry_group=build_translation_group(model.lattice, flux0))
        checkpoint_paths = ed_scan(init, nev=nev, mode="matrixfree", twisted_phases_over_2π_list=thetas,
                                   flux_direction=flux_direction, checkpoint_dir=checkpoint_dir,
                                   overwrite=overwrite, scanned_sectors=labels)
        for it, path in enumerate(checkpoint_paths):
            data = load_checkpoint(path)
            for isec, lab in enumerate(labels):
                idx = next((i for i, ir in enumerate(data.irrep_list) if ir.label == lab), None)
                if idx is not None and idx in data.ed_scan_res:
                    vals = data.ed_scan_res[idx][0]
                    nv = min(len(vals), nev)
                    energies[it, isec, :nv] = vals[:nv]
    elif engine == "served":
        from .serving import ServedCheckpoints, ServingModel, SolveRequest, SolveServer

        n_filled = int(filling_fraction * model.lattice.n_site)
        sm = ServingModel(model, n_filled, name="flow")
        irr = [ir.label for ir in build_irrep_list(sm.group0, model.lattice)]
        reqs, where = [], {}
        for it, th in enumerate(thetas):
            flux = [0.0] * dim
            flux[flux_direction - 1] = th
            for isec, lab in enumerate(labels):
                if lab not in irr:
                    raise ValueError(f"No irrep with label {lab!r} in irrep_list.")
                rid = len(reqs)
                reqs.append(SolveRequest(rid, irr.index(lab), tuple(flux), "flow"))
                where[rid] = (it, isec)
        ck = ServedCheckpoints(checkpoint_dir, overwrite=overwrite)
        server = SolveServer(sm, nev=nev, precision=precision, block=2, checkpoints=ck)
        for res in server.run(reqs, realtime=False):
            it, isec = where[res.rid]
            nv = min(len(res.eigenvalues), nev)
            energies[it, isec, :nv] = res.eigenvalues[:nv]
        ck.close()
        checkpoint_paths = []
        for th in thetas:
            flux = [0.0] * dim
            flux[flux_direction - 1] = th
            checkpoint_paths.append(ck.path_of(sm, tuple(flux)))
    else:
        raise ValueError(f"unknown engine {engine!r}")
    _no_figure(fig_path)
    return SimpleNamespace(twisted_phases_over_2π_list=thetas, energies=energies, sector_labels=labels,
                           flux_direction=flux_direction, nev=nev, is_identity=is_identity, fig_path=fig_path,
                           checkpoint_paths=checkpoint_paths)


# ---- many-body Chern number ----------------------------------------------------


def _normalize_flux_grid_size(flux_grid_size) -> tuple[int, int]:
    """``(nx, ny)`` from an int (square grid) or a pair; each at least 2
    (``many_body_chern_number.py:37-56``)."""
    if isinstance(flux_grid_size, int):
        nx = ny = int(flux_grid_size)
    else:
        nx, ny = int(flux_grid_size[0]), int(flux_grid_size[1])
    if min(nx, ny) < 2:
        raise ValueError("flux_grid_size must be at least 2 in both directions.")
    return nx, ny


def _chern_sector_labels(sector_labels) -> list:
    """``["identity"]`` or the momentum labels as int tuples (``:59-72``)."""
    if isinstance(sector_labels, str) and sector_labels == "identity":
        return ["identity"]
    return [tuple(int(x) for x in lab) for lab in sector_labels]


def _chern_params_digest(params: dict) -> str:
    """64-bit FNV-1a of the UTF-8 ``repr`` of the parameter pairs sorted by key
    name, in hex: the checkpoint-name tag of the reference (``:75-94``), kept
    byte-compatible so checkpoints of either implementation are found."""
    data = repr(sorted(params.items(), key=lambda kv: str(kv[0]))).encode("utf-8")
    h = 0xCBF29CE484222325
    for byte in data:
        h = ((h ^ byte) * 0x100000001B3) % (1 << 64)
    return f"{h:x}"


def _chern_flux_tag(flux) -> str:
    """``0.250000_0.500000`` style tag with ``.`` -> ``p`` and ``-`` -> ``m`` (``:97-108``)."""
    return "_".join(f"{float(t):.6f}".replace(".", "p").replace("-", "m") for t in flux)


def _chern_checkpoint_path(model, filling_fraction: Fraction, flux, checkpoint_dir: str) -> str:
    """Checkpoint file of one flux point of the Chern scan, named as the
    reference names it (``:111-138``)."""
    sample = "x".join(str(n) for n in model.lattice.sample_size)
    name = (f"many_body_chern_{model.tb_model.model_name}_{sample}_nu={filling_fraction.numerator}_"
            f"{filling_fraction.denominator}_theta={_chern_flux_tag(flux)}_p={_chern_params_digest(model.params)}.pkl")
    return os.path.join(checkpoint_dir, name)


def _unit_det_link(M: np.ndarray, *, det_atol: float = 1e-10):
    """``(z / |z|, |z|)`` for ``z = det(M)``; a near-singular ``|z| <= det_atol``
    gives the link 1 and a warning (``:185-207``)."""
    import warnings

    z = complex(np.linalg.det(M))
    if abs(z) <= det_atol:
        warnings.warn("Near-singular Berry link; selected manifold may not be isolated.", stacklevel=2)
        return 1.0 + 0.0j, abs(z)
    return z / abs(z), abs(z)


def _chern_point(model, labels, base, filling_fraction, flux, nev_per_sector, mode, checkpoint_dir, overwrite,
                 out):
    """Solve one flux point and expand its manifold states into ``out``
    (``[n_manifold, n_states]`` device rows) -- the reference's
    ``_flux_point_states_for_chern`` (``:210-307``) with dense device states."""
    from .catalog import update_orbit_stabilizer_phases
    from .ed import Symmetry_Resolved_ED_Data, _ed_scan_sectors
    from .fock import expand_sector_state_to_fock_dense
    from .second_quantized_model import update_second_quantized_model_with_twisted_phases
    from .sector import Symmetry_Sector_Basis, build_symmetry_sector_basis
    from .symmetry import build_irrep_list, build_translation_group

    update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=list(flux))
    identity = labels == ["identity"]
    if identity:
        group, cat = base.symmetry_group, base.orbit_catalog
    else:
        group = build_translation_group(model.lattice, list(flux))
        cat = base.orbit_catalog.clone()
        update_orbit_stabilizer_phases(cat, group, model.particle_statistics)
    irreps = build_irrep_list(group, model.lattice)
    data = Symmetry_Resolved_ED_Data(model, base.n_filled, filling_fraction, group, irreps, cat, [0] * len(irreps))
    path = _chern_checkpoint_path(model, filling_fraction, flux, checkpoint_dir)
    _ed_scan_sectors(data, nev=nev_per_sector, mode=mode, scanned_sectors=None if identity else list(labels),
                     checkpoint_path=path, overwrite=overwrite)
    _, sset = data._device()
    energies, level_labels = [], []
    row = 0
    for label in labels:
        if identity:
            idx = 0
        else:
            idx = next((i for i, ir in enumerate(irreps) if ir.label == label), None)
            if idx is None:
                raise ValueError(f"Sector {label!r} not found at flux {list(flux)}.")
        if idx not in data.ed_scan_res:
            raise ValueError(f"Sector {label!r} was not scanned at flux {list(flux)}.")
        vals, vecs = data.ed_scan_res[idx]
        n_take = min(nev_per_sector, vecs.shape[1])
        if n_take != nev_per_sector:
            raise ValueError(f"Requested {nev_per_sector} states in sector {label!r}, only found {n_take}.")
        basis = (Symmetry_Sector_Basis(irreps[idx], cat, sset, idx) if sset is not None
                 else build_symmetry_sector_basis(cat, irreps[idx]))
        for level in range(n_take):
            expand_sector_state_to_fock_dense(vecs[:, level], basis, out=out[row])
            energies.append(float(vals[level]))
            level_labels.append((label, level + 1))
            row += 1
    return energies, level_labels, path


def _chern_served(model, labels, n_filled, flux_x, flux_y, nev_per_sector, checkpoint_dir, overwrite):
    """Every (flux point, sector) solve of the grid as one request to a
    ``SolveServer`` (FP64, eigenvectors kept on the device, results written
    to -- and, unless ``overwrite``, answered from -- the Chern scan's
    per-point checkpoints); returns the catalog, a function that expands one
    flux point's manifold into dense Fock rows, and the checkpoint path of a
    flux point."""
    from .catalog import update_orbit_stabilizer_phases
    from .fock import expand_sector_state_to_fock_dense
    from .sector import SectorSet, Symmetry_Sector_Basis
    from .serving import ServedCheckpoints, ServingModel, SolveRequest, SolveServer
    from .symmetry import build_irrep_list, build_translation_group

    sm = ServingModel(model, n_filled, name="chern")
    ff = Fraction(n_filled, model.lattice.n_site)
    ck = ServedCheckpoints(checkpoint_dir, overwrite=overwrite,
                           path_of=lambda sm_, flux: _chern_checkpoint_path(model, ff, list(flux), checkpoint_dir))
    irr = [ir.label for ir in build_irrep_list(sm.group0, model.lattice)]
    for lab in labels:
        if lab not in irr:
            raise ValueError(f"Sector {lab!r} not found at flux [0.0, 0.0].")
    reqs, where = [], {}
    for ix, fx in enumerate(flux_x):
        for iy, fy in enumerate(flux_y):
            for lab in labels:
                where[len(reqs)] = (ix, iy, lab)
                reqs.append(SolveRequest(len(reqs), irr.index(lab), (float(fx), float(fy)), "chern", vectors=True))
    server = SolveServer(sm, nev=nev_per_sector, precision=64, block=2, checkpoints=ck)
    solved = {where[r.rid]: r for r in server.run(reqs, realtime=False, timeout=24 * 3600.0)}
    del server
    ck.close()

    def fill(ix, iy, out):
        flux = [float(flux_x[ix]), float(flux_y[iy])]
        group = build_translation_group(model.lattice, flux)
        cat = sm.catalog.clone()
        update_orbit_stabilizer_phases(cat, group, sm.stats)
        irreps = build_irrep_list(group, model.lattice)
        sset = SectorSet(cat, irreps)
        energies, row = [], 0
        for lab in labels:
            res = solved.pop((ix, iy, lab))
            idx = irr.index(lab)
            if len(res.eigenvalues) < nev_per_sector:
                raise ValueError(f"Requested {nev_per_sector} states in sector {lab!r}, "
                                 f"only found {len(res.eigenvalues)}.")
            basis = Symmetry_Sector_Basis(irreps[idx], cat, sset, idx)
            for level in range(nev_per_sector):
                expand_sector_state_to_fock_dense(res.eigenvectors[:, level], basis, out=out[row])
                energies.append(float(res.eigenvalues[level]))
                row += 1
        return energies, ck.path_of(sm, tuple(flux))

    return sm.catalog, fill


def many_body_chern_number(model, sector_labels, *, filling_fraction, flux_grid_size=(5, 5), nev_per_sector: int = 1,
                           mode: str = "matrix", checkpoint_dir: str = "checkpoints", overwrite: bool = False,
                           fig_path: str | None = None, det_atol: float = 1e-10, engine: str = "scan"):
    """Chern number of the many-body manifold on the flux torus; returns the
    reference's fields (``chern_number``, ``rounded_chern``,
    ``berry_curvature[ix, iy]``, ``flux_x``, ``flux_y``, ``sector_labels``,
    ``nev_per_sector``, ``flux_grid_size``, ``energies[ix][iy]``,
    ``min_link_det``, ``link_det_abs_x``, ``link_det_abs_y``,
    ``checkpoint_paths[ix][iy]``, ``fig_path``).

    ``engine="scan"`` solves flux point after flux point with the
    reference's per-point checkpoints; ``engine="served"`` submits every
    (flux point, sector) solve to a ``SolveServer`` at once (FP64, solves of
    different flux points overlapping on the device; momentum sectors only)
    and keeps the same per-point checkpoints through ``ServedCheckpoints``."""
    import torch

    from .ed import build_ed_data
    from .fock import fock_overlaps
    from .second_quantized_model import update_second_quantized_model_with_twisted_phases
    from .symmetry import build_identity_group, build_translation_group

    filling_fraction = Fraction(filling_fraction)
    if model.lattice.dim != 2:
        raise ValueError("many_body_chern_number currently expects a 2D lattice.")
    nx, ny = _normalize_flux_grid_size(flux_grid_size)
    labels = _chern_sector_labels(sector_labels)
    if mode not in ("matrix", "matrixfree"):
        raise ValueError(f"Unknown ED scan mode: {mode}. Use 'matrix' or 'matrixfree'.")
    if engine not in ("scan", "served"):
        raise ValueError(f"unknown engine {engine!r}")
    flux_x = np.arange(nx) / nx
    flux_y = np.arange(ny) / ny

    # the zero-flux catalog, moved to every flux point by a phase update
    update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=[0.0, 0.0])
    if engine == "scan":
        os.makedirs(checkpoint_dir, exist_ok=True)
        group0 = (build_identity_group(model.lattice.n_site) if labels == ["identity"]
                  else build_translation_group(model.lattice, [0.0, 0.0]))
        base = build_ed_data(model, filling_fraction=filling_fraction, symmetry_group=group0)
        cat = base.orbit_catalog

        def fill(ix, iy, out):
            e, _, path = _chern_point(model, labels, base, filling_fraction, (float(flux_x[ix]), float(flux_y[iy])),
                                      nev_per_sector, mode, checkpoint_dir, overwrite, out)
            return e, path
    else:
        if labels == ["identity"]:
            raise ValueError("the served engine solves momentum sectors; use engine='scan' for 'identity'")
        n_filled = filling_fraction * model.lattice.n_site
        if n_filled.denominator != 1:
            raise ValueError("filling_fraction * n_site must be an integer (particle number).")
        os.makedirs(checkpoint_dir, exist_ok=True)
        cat, fill = _chern_served(model, labels, int(n_filled), flux_x, flux_y, int(nev_per_sector), checkpoint_dir,
                                  overwrite)
    n_m = len(labels) * int(nev_per_sector)
    rows_kept = min(nx, 3)
    states = torch.zeros((rows_kept * ny, n_m, cat.n_states), dtype=torch.complex128, device=cat.table.device)

    def slot(ix, iy):  # row 0 stays; later rows alternate between two row buffers
        return iy if ix == 0 else ny * (1 + (ix - 1) % 2) + iy

    Ux = np.empty((nx, ny), dtype=np.complex128)
    Uy = np.empty((nx, ny), dtype=np.complex128)
    det_abs_x = np.empty((nx, ny))
    det_abs_y = np.empty((nx, ny))

    def row_links(ix, ixp):
        pairs = [(slot(ix, iy), slot(ixp, iy)) for iy in range(ny)]
        pairs += [(slot(ix, iy), slot(ix, (iy + 1) % ny)) for iy in range(ny)]
        M = fock_overlaps(states, pairs)
        for iy in range(ny):
            Ux[ix, iy], det_abs_x[ix, iy] = _unit_det_link(M[iy], det_atol=det_atol)
            Uy[ix, iy], det_abs_y[ix, iy] = _unit_det_link(M[ny + iy], det_atol=det_atol)

    energies = [[None] * ny for _ in range(nx)]
    checkpoint_paths = [[None] * ny for _ in range(nx)]
    for ix in range(nx):
        for iy in range(ny):
            energies[ix][iy], checkpoint_paths[ix][iy] = fill(ix, iy, states[slot(ix, iy)])
        if ix >= 1:
            row_links(ix - 1, ix)
    row_links(nx - 1, 0)

    ixp = (np.arange(nx) + 1) % nx
    iyp = (np.arange(ny) + 1) % ny
    plaquette = Ux * Uy[ixp, :] * np.conj(Ux[:, iyp]) * np.conj(Uy)
    berry_curvature = np.angle(plaquette).astype(np.float64)
    chern_number = float(np.sum(berry_curvature)) / (2 * np.pi)
    res = SimpleNamespace(chern_number=chern_number, rounded_chern=round(chern_number),
                          berry_curvature=berry_curvature, flux_x=flux_x, flux_y=flux_y, sector_labels=labels,
                          nev_per_sector=nev_per_sector, flux_grid_size=(nx, ny), energies=energies,
                          min_link_det=min(float(det_abs_x.min()), float(det_abs_y.min())),
                          link_det_abs_x=det_abs_x, link_det_abs_y=det_abs_y, checkpoint_paths=checkpoint_paths,
                          fig_path=fig_path)
    _no_figure(fig_path)
    return res


# ---- charge pump -----------------------------------------------------------------


def many_body_position_phases(lattice, direction: int, *, include_sublattice: bool = True) -> np.ndarray:
    """``exp(2 pi i x_j / L)`` per site (0-based), ``x_j`` the crystal
    coordinate of site ``j`` along the 1-based ``direction`` (cell index plus,
    optionally, the sub-lattice offset) and ``L`` the sample size there
    (``charge_pump.py:41-78``)."""
    import cmath
    import math

    if not 1 <= direction <= lattice.dim:
        raise ValueError(f"direction must be in 1..{lattice.dim}.")
    L = float(lattice.sample_size[direction - 1])
    out = np.zeros(lattice.n_site, dtype=np.complex128)
    for i, (cell, sub) in enumerate(lattice.site_list):
        x = float(cell[direction - 1])
        if include_sublattice:
            x += float(lattice.sub_crys_list[sub - 1][direction - 1])
        out[i] = cmath.exp(2j * math.pi * x / L)
    return out


def _default_polarization_direction(dim: int, flux_direction: int) -> int:
    """The next direction after the flux direction (1-based, cyclic); the flux
    direction itself in 1-D (``charge_pump.py:164-177``)."""
    return flux_direction if dim == 1 else flux_direction % dim + 1


def _best_phase_permutation(raw: np.ndarray, prev: np.ndarray) -> np.ndarray:
    """The assignment of current branches to previous ones with the least
    sum of squared wrapped phase jumps; among equal costs the lexicographically
    first, each cost summed in branch order (``charge_pump.py:180-216``)."""
    import itertools

    n = len(prev)
    best, best_cost = tuple(range(n)), float("inf")
    for perm in itertools.permutations(range(n)):
        cost = 0.0
        for depth, j in enumerate(perm):
            d = raw[j] - prev[depth]
            d -= round(d)
            cost = cost + d ** 2
            if cost >= best_cost:
                break
        else:
            best, best_cost = perm, cost
    return np.asarray(best, dtype=np.int64)


def _tracked_phase_branches(raw_phases: np.ndarray) -> np.ndarray:
    """Branches sorted at the first flux value, then matched step by step
    (``_best_phase_permutation``) and shifted by whole windings to stay
    continuous (``charge_pump.py:219-240``)."""
    n_t, _ = raw_phases.shape
    tracked = np.empty_like(raw_phases)
    tracked[0] = raw_phases[0, np.argsort(raw_phases[0])]
    for it in range(1, n_t):
        perm = _best_phase_permutation(raw_phases[it], tracked[it - 1])
        for b, j in enumerate(perm):
            phi = raw_phases[it, j]
            tracked[it, b] = phi + round(tracked[it - 1, b] - phi)
    return tracked


class _ManifoldState:
    """One manifold state: a sector label and a 1-based level."""

    __slots__ = ("sector", "level")

    def __init__(self, sector, level):
        self.sector, self.level = sector, level

    def __eq__(self, other):
        return isinstance(other, _ManifoldState) and (self.sector, self.level) == (other.sector, other.level)

    def __repr__(self):
        return f"_ManifoldState(sector={self.sector!r}, level={self.level})"


def _normalize_manifold_state_specs(sector_labels, nev_per_sector: int, manifold_states):
    """``(labels, specs, required_levels, is_identity)`` from the legacy
    ``nev_per_sector`` form or explicit ``(sector, level)`` states, with the
    reference's validation (``charge_pump.py:256-322``)."""
    if nev_per_sector <= 0:
        raise ValueError("nev_per_sector must be positive.")
    is_identity = isinstance(sector_labels, str) and sector_labels == "identity"
    if is_identity:
        base = ["identity"]
    elif isinstance(sector_labels, tuple):
        base = [tuple(int(x) for x in sector_labels)]
    else:
        base = [tuple(int(x) for x in lab) for lab in sector_labels]
    if manifold_states is None:
        specs = [_ManifoldState(lab, lev) for lab in base for lev in range(1, nev_per_sector + 1)]
    else:
        if is_identity:
            raise ValueError("Explicit manifold_states are only supported for symmetry-sector ED.")
        specs = []
        for st in manifold_states:
            if hasattr(st, "sector"):
                sec, lev = st.sector, st.level
            elif isinstance(st, dict):
                sec, lev = st["sector"], st["level"]
            else:
                sec, lev = st[0], st[1]
            sec, lev = tuple(int(x) for x in sec), int(lev)
            if lev <= 0:
                raise ValueError(f"Manifold levels must be positive; got {lev} in sector {sec}.")
            if sec not in base:
                raise ValueError(f"Manifold state ({sec}, level {lev}) is absent from sector_labels={base}.")
            specs.append(_ManifoldState(sec, lev))
        if not specs:
            raise ValueError("manifold_states must not be empty.")
        if len({(x.sector, x.level) for x in specs}) != len(specs):
            raise ValueError("manifold_states contains duplicate (sector, level) entries.")
    labels = list(dict.fromkeys(x.sector for x in specs))
    required: dict = {}
    for x in specs:
        required[x.sector] = max(required.get(x.sector, 0), x.level)
    return labels, specs, required, is_identity


def _position_block(cat, chi_to, chi_from, x_to, x_from, site_phase, stream=None) -> np.ndarray:
    """``[k_to, k_from]`` position-operator products of orbit-layout vectors
    ``x_to [k_to, n_orbits]`` and ``x_from [k_from, n_orbits]`` on the device."""
    import ctypes

    import torch

    from . import _lib

    lib = _lib.lib()
    k_to, k_from = int(x_to.shape[0]), int(x_from.shape[0])
    n_orb = cat.n_orbits
    out = torch.empty((k_to, k_from), dtype=torch.complex128, device=x_to.device)
    scratch = torch.empty(int(lib.rsed_position_scratch_bytes(n_orb, k_to, k_from)), dtype=torch.uint8,
                          device=x_to.device)
    _lib.check(lib.rsed_position_overlaps(ctypes.byref(cat.dgroup.c), n_orb, _lib.ptr(cat.repr_masks),
                                          _lib.ptr(chi_to), _lib.ptr(chi_from), _lib.ptr(site_phase), _lib.ptr(x_to),
                                          k_to, _lib.ptr(x_from), k_from, _lib.ptr(out), _lib.ptr(scratch),
                                          scratch.numel(), _lib.stream_ptr(stream)))
    return out.cpu().numpy()


def flux_charge_pump(model, sector_labels, *, filling_fraction, flux_direction: int = 1,
                     polarization_direction: int | None = None, twisted_phases_over_2π_list=None,
                     nev_per_sector: int = 1, manifold_states=None, include_sublattice: bool = True,
                     checkpoint_dir: str = "checkpoints", fig_path: str | None = None, overwrite: bool = False):
    """Many-body charge pump under flux insertion; returns the reference's
    fields (``twisted_phases_over_2π_list``, ``energies[θ, sector, level]``,
    ``sector_labels``, ``flux_direction``, ``polarization_direction``,
    ``nev_per_sector``, ``manifold_states``, ``polarization_eigenvalues``,
    ``polarizations``, ``pumped_charge_trajectories``, ``pumped_charges``,
    ``include_sublattice``, ``is_identity``, ``fig_path``,
    ``checkpoint_paths``).  The identity sector is rejected: the flux scan
    holds translation sectors only."""
    import math

    import torch

    from .catalog import update_orbit_stabilizer_phases
    from .ed import build_ed_data, ed_scan, load_checkpoint
    from .second_quantized_model import update_second_quantized_model_with_twisted_phases
    from .sector import SectorSet
    from .symmetry import build_translation_group

    if twisted_phases_over_2π_list is None:
        twisted_phases_over_2π_list = list(np.linspace(0.0, 1.0, 9))
    labels, specs, required, is_identity = _normalize_manifold_state_specs(sector_labels, nev_per_sector,
                                                                            manifold_states)
    if is_identity:
        raise ValueError("flux_charge_pump reads translation-sector flux-scan checkpoints; "
                         "the 'identity' sector is not among them.")
    dim = model.lattice.dim
    if not 1 <= flux_direction <= dim:
        raise ValueError(f"flux_direction must be in 1..{dim}.")
    if polarization_direction is None:
        polarization_direction = _default_polarization_direction(dim, flux_direction)
    if not 1 <= polarization_direction <= dim:
        raise ValueError(f"polarization_direction must be in 1..{dim}.")
    thetas = list(twisted_phases_over_2π_list)
    n_states = len(specs)
    max_level = max(required.values())
    energies = np.full((len(thetas), len(labels), max_level), np.nan)
    pol_ev = np.zeros((len(thetas), n_states), dtype=np.complex128)

    flux0 = [0.0] * dim
    update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=flux0)
    init = build_ed_data(model, filling_fraction=filling_fraction,
                         symmetry_group=build_translation_group(model.lattice, flux0))
    paths = ed_scan(init, nev=max(max_level, 2), mode="matrix", twisted_phases_over_2π_list=thetas,
                    flux_direction=flux_direction, checkpoint_dir=checkpoint_dir, overwrite=overwrite,
                    scanned_sectors=labels)
    base = init.orbit_catalog
    dev = base.table.device
    site_phase = torch.as_tensor(many_body_position_phases(model.lattice, polarization_direction,
                                                           include_sublattice=include_sublattice)).to(dev)
    for it, path in enumerate(paths):
        data = load_checkpoint(path)
        cat = base.clone()
        update_orbit_stabilizer_phases(cat, data.symmetry_group, model.particle_statistics)
        sset = SectorSet(cat, data.irrep_list)
        X, chi = {}, {}
        for il, lab in enumerate(labels):
            idx = next((i for i, ir in enumerate(data.irrep_list) if ir.label == lab), None)
            if idx is None or idx not in data.ed_scan_res:
                raise ValueError(f"sector {lab} not found in checkpoint {path}")
            vals, vecs = data.ed_scan_res[idx]
            nv = required[lab]
            if vecs.shape[1] < nv:
                raise ValueError(f"Sector {lab} in {path} has {vecs.shape[1]} eigenvectors; need {nv}.")
            if len(vals) < nv:
                raise ValueError(f"Sector {lab} in {path} has {len(vals)} eigenvalues; need {nv}.")
            energies[it, il, :nv] = vals[:nv]
            rows = sset.rows(idx)[0].long()
            x = torch.zeros((nv, cat.n_orbits), dtype=torch.complex128, device=dev)
            x[:, rows] = torch.as_tensor(np.ascontiguousarray(np.asarray(vecs)[:, :nv].T)).to(dev)
            X[lab], chi[lab] = x, sset.chi[idx].contiguous()
        blocks: dict = {}
        P = np.zeros((n_states, n_states), dtype=np.complex128)
        for r, st in enumerate(specs):
            for c, sf in enumerate(specs):
                key = (st.sector, sf.sector)
                if key not in blocks:
                    blocks[key] = _position_block(cat, chi[st.sector], chi[sf.sector], X[st.sector], X[sf.sector],
                                                  site_phase)
                P[r, c] = blocks[key][st.level - 1, sf.level - 1]
        ev = np.linalg.eigvals(P)
        pol_ev[it] = ev[np.argsort(np.angle(ev))]
    raw = np.angle(pol_ev) / (2 * math.pi)
    polarizations = _tracked_phase_branches(raw)
    trajectories = polarizations - polarizations[0:1, :]
    pumped = trajectories[-1, :]
    _no_figure(fig_path)
    return SimpleNamespace(twisted_phases_over_2π_list=thetas, energies=energies, sector_labels=labels,
                           flux_direction=flux_direction, polarization_direction=polarization_direction,
                           nev_per_sector=max_level, manifold_states=specs, polarization_eigenvalues=pol_ev,
                           polarizations=polarizations, pumped_charge_trajectories=trajectories,
                           pumped_charges=pumped, include_sublattice=include_sublattice, is_identity=is_identity,
                           fig_path=fig_path, checkpoint_paths=paths)
