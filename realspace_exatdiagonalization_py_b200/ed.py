"""ED data structure, sector scans, flux scans and checkpoints.

Mirrors ``Symmetry_Resolved_ED_Data`` / ``build_ed_data`` / ``ed_scan`` /
``ed_scan_at_irrep_*`` / ``full_ed`` / checkpoint I/O
(``symmetry_resolved_ed.py:2307-2703, 2906-2992``).  Differences in how, not
what: a scan solves every pending sector of one catalog in a single batched
device Lanczos (one apply per iteration serves all sectors), and the flux scan
reuses the catalog through ``update_orbit_stabilizer_phases`` instead of
rebuilding it at every flux point.
"""

from __future__ import annotations

import math
import os
import pickle
from dataclasses import dataclass, field
from fractions import Fraction

import numpy as np
import torch

from .catalog import Symmetry_Orbit_Catalog, build_symmetry_orbit_catalog, update_orbit_stabilizer_phases
from .hamiltonian import DeviceModel, MatrixFreeHamiltonian, build_ed_Hamiltonian_symmetry_block
from .lanczos import (
    LanczosBatch,
    LanczosParams,
    diagonalize_block_arpack,
    diagonalize_block_dense,
    diagonalize_block_matrixfree,
    refine,
)
from .sector import CanonicalMap, SectorSet, Symmetry_Sector_Basis
from .symmetry import (
    Finite_Symmetry_Group,
    OneDim_Irrep,
    build_identity_group,
    build_irrep_list,
    build_translation_group,
)

__all__ = [
    "Symmetry_Resolved_ED_Data",
    "build_ed_data",
    "ed_scan",
    "ed_scan_at_irrep_matrix",
    "ed_scan_at_irrep_matrixfree",
    "full_ed",
    "save_checkpoint",
    "load_checkpoint",
    "ed_scan_checkpoint_filename",
    "print_spectrum",
]


@dataclass
class Symmetry_Resolved_ED_Data:
    second_quantized_model: object
    n_filled: int
    filling_fraction: Fraction
    symmetry_group: Finite_Symmetry_Group
    irrep_list: list[OneDim_Irrep]
    orbit_catalog: Symmetry_Orbit_Catalog
    sector_dims: list[int]
    ed_scan_res: dict = field(default_factory=dict)

    def __getstate__(self):
        # device tables are rebuilt, not pickled: keep model, labels and results
        st = dict(self.__dict__)
        st["orbit_catalog"] = None
        st.pop("_dev", None)
        st.pop("_solvers", None)
        return st

    def __setstate__(self, st):
        self.__dict__.update(st)

    # device-side helpers cached per catalog/model
    def _device(self):
        dv = self.__dict__.get("_dev")
        cat = self.orbit_catalog
        model = self.second_quantized_model
        key = (id(cat), id(model.bilinear_terms), id(model.density_density_terms),
               id(cat.symmetry_group), cat.version)
        if dv is None or dv[0] != key:
            dm = DeviceModel(cat, model.bilinear_terms, model.density_density_terms)
            sset = SectorSet(cat, self.irrep_list[:64]) if len(self.irrep_list) <= 64 else None
            dv = (key, dm, sset)
            self.__dict__["_dev"] = dv
        return dv[1], dv[2]


def build_ed_data(second_quantized_model, *, filling_fraction=Fraction(1, 2),
                  symmetry_group: Finite_Symmetry_Group,
                  species: tuple[list[int], int] | None = None) -> Symmetry_Resolved_ED_Data:
    """``n_filled = filling * n_site`` (exact), irreps and the device catalog
    (``symmetry_resolved_ed.py:2906-2963``).  ``species = (sites_b, n_b)``
    additionally fixes ``n_b`` particles on the 1-based sites ``sites_b``
    (e.g. the spin-down orbitals: fixed N_up and N_down)."""
    n_site = second_quantized_model.lattice.n_site
    if not isinstance(filling_fraction, Fraction):
        filling_fraction = Fraction(filling_fraction)
    n_filled = int(filling_fraction * n_site)
    assert filling_fraction.denominator * n_filled == filling_fraction.numerator * n_site, (
        "build_ed_data: filling_fraction * n_site must be an integer (particle number)."
    )
    irreps = build_irrep_list(symmetry_group, second_quantized_model.lattice)
    catalog = build_symmetry_orbit_catalog(
        second_quantized_model=second_quantized_model,
        n_filled=n_filled,
        symmetry_group=symmetry_group,
        particle_statistics=second_quantized_model.particle_statistics,
        species=species,
    )
    return Symmetry_Resolved_ED_Data(second_quantized_model, n_filled, filling_fraction,
                                     symmetry_group, irreps, catalog, [0] * len(irreps))


def _find_irrep_idx(ed_data, irrep_label) -> int:
    for idx, irrep in enumerate(ed_data.irrep_list):
        if irrep.label == irrep_label:
            return idx
    raise ValueError(f"No irrep with label {irrep_label!r} in irrep_list.")


def _empty():
    return np.zeros(0, dtype=np.float64), np.zeros((0, 0), dtype=np.complex128)


def _default_params(nev: int, precision: int = 64) -> LanczosParams:
    return LanczosParams(precision=precision)


def ed_scan_at_irrep_matrixfree(irrep_label, ed_data, *, nev: int = 5,
                                params: LanczosParams | None = None):
    """One sector, matrix-free (``symmetry_resolved_ed.py:2402-2459``)."""
    idx = _find_irrep_idx(ed_data, irrep_label)
    dm, sset = ed_data._device()
    basis = Symmetry_Sector_Basis(ed_data.irrep_list[idx], ed_data.orbit_catalog, sset, idx)
    n = basis.dim
    ed_data.sector_dims[idx] = n
    if n == 0:
        ed_data.ed_scan_res[idx] = _empty()
        return _empty()
    cmap = CanonicalMap(ed_data.symmetry_group, ed_data.second_quantized_model.particle_statistics,
                        ed_data.orbit_catalog)
    H_op = MatrixFreeHamiltonian(basis, ed_data.second_quantized_model.bilinear_terms,
                                 ed_data.second_quantized_model.density_density_terms, cmap, model=dm)
    vals, vecs = diagonalize_block_matrixfree(H_op, n, nev=nev, params=params or _default_params(nev))
    ed_data.ed_scan_res[idx] = (vals, vecs)
    return vals, vecs


def ed_scan_at_irrep_matrix(irrep_label, ed_data, *, nev: int = 5,
                            params: LanczosParams | None = None):
    """One sector, matrix mode (``symmetry_resolved_ed.py:2367-2399``): the
    block is assembled on the GPU; ``n <= 500`` is solved densely on the
    block's upper triangle, larger blocks with the device block Lanczos."""
    idx = _find_irrep_idx(ed_data, irrep_label)
    dm, sset = ed_data._device()
    basis = Symmetry_Sector_Basis(ed_data.irrep_list[idx], ed_data.orbit_catalog, sset, idx)
    n = basis.dim
    ed_data.sector_dims[idx] = n
    if n == 0:
        ed_data.ed_scan_res[idx] = _empty()
        return _empty()
    cmap = CanonicalMap(ed_data.symmetry_group, ed_data.second_quantized_model.particle_statistics,
                        ed_data.orbit_catalog)
    H = build_ed_Hamiltonian_symmetry_block(basis, ed_data.second_quantized_model.bilinear_terms,
                                            ed_data.second_quantized_model.density_density_terms,
                                            cmap, model=dm)
    vals, vecs = diagonalize_block_arpack(H, nev=nev, basis=basis, model=dm,
                                          params=params or _default_params(nev))
    ed_data.ed_scan_res[idx] = (vals, vecs)
    return vals, vecs


def solve_sectors_batched(ed_data, sector_ids: list[int], *, nev: int = 5, precision: int = 64,
                          params: LanczosParams | None = None, graph: bool = True,
                          return_vectors: bool = True, start_blocks=None, config=None,
                          autotune: bool = False):
    """Solve many sectors of one catalog in one batched block Lanczos.

    Sectors with ``dim <= 500`` take the dense path (as the reference does);
    the rest run together: every iteration is one apply launch for all of
    them.  ``precision=32`` runs the matvec in FP32 and finishes each sector
    with an FP64 refinement.  The batched solver (buffers, captured graphs)
    is kept on ``ed_data`` and reused by later calls with the same sectors.
    ``config`` (a ``SolverConfig``) fixes how the batch runs; ``autotune``
    picks it by measurement (``autotune.default_tuner``, cached per shape).
    Returns ``{sector: (vals, vecs)}``.
    """
    from .batched import BatchedSectorSolver

    dm, sset = ed_data._device()
    out = {}
    big = []
    for s in sector_ids:
        n = sset.dims[s]
        ed_data.sector_dims[s] = n
        if n == 0:
            out[s] = _empty()
        elif n <= 500:
            basis = Symmetry_Sector_Basis(ed_data.irrep_list[s], ed_data.orbit_catalog, sset, s)
            H_op = MatrixFreeHamiltonian(basis, ed_data.second_quantized_model.bilinear_terms,
                                         ed_data.second_quantized_model.density_density_terms, None,
                                         model=dm)
            out[s] = diagonalize_block_matrixfree(H_op, n, nev=nev)
        else:
            big.append(s)
    if big:
        from .batched import lanczos_footprint_bytes, plan_waves, projection_precisions

        p = params or LanczosParams(precision=precision)
        if dm.proj is None and (config is None or config.projection):
            # the streaming matvec, when its table fits half the free memory
            free, _ = torch.cuda.mem_get_info()
            if dm.projection_bytes((precision,)) <= 0.5 * free:
                dm.build_projection(sset.sqrt_stab, precisions=projection_precisions(dm, precision))
        cache = ed_data.__dict__.setdefault("_solvers", {})
        resident = None
        if not (config is None and autotune):
            resident = cache.get((tuple(big), nev, precision,
                                  None if params is None else tuple(params.__dict__.items()), graph, config))
        if resident is not None and resident.model is dm:
            # the solver of an earlier call with the same sectors holds all its
            # buffers: no wave plan, and no free-memory query (cudaMemGetInfo
            # takes about 0.4 ms per call and at times stalls for ~100 ms)
            waves = [list(range(len(big)))]
        else:
            free, _ = torch.cuda.mem_get_info()
            n_orb = ed_data.orbit_catalog.n_orbits
            bs = list(config.block_sizes) if config is not None else [p.block] * len(big)
            budget = int(0.7 * free)
            if lanczos_footprint_bytes(n_orb, sum(bs), p.n_slots, precision) <= budget:
                waves = [list(range(len(big)))]
            else:
                waves = plan_waves(n_orb, bs, budget, p.n_slots, precision)
            if config is None and autotune and len(waves) == 1:
                from .autotune import default_tuner

                config = default_tuner().best(dm, sset, big, nev, precision, params)
        for wave in waves:
            secs = [big[i] for i in wave]
            cfg = config if len(waves) == 1 else (None if config is None else type(config)(
                tuple(config.block_sizes[i] for i in wave), config.persistent, config.projection,
                config.n_slots, config.poll))
            key = (tuple(secs), nev, precision, None if params is None else tuple(params.__dict__.items()),
                   graph, cfg)
            solver = cache.get(key)
            if solver is None or solver.model is not dm:
                solver = BatchedSectorSolver(dm, sset, secs, nev, precision=precision, params=params,
                                             graph=graph, config=cfg)
                if len(waves) == 1:
                    cache[key] = solver
            blocks = None if start_blocks is None else [start_blocks[big.index(s)] for s in secs]
            vals, vecs = solver.solve(blocks, vectors=return_vectors)
            for i, s in enumerate(secs):
                out[s] = (vals[i].copy(), vecs[i] if vecs is not None else None)
            if len(waves) > 1:
                del solver
                torch.cuda.empty_cache()
    return out


def _ed_scan_sectors(ed_data, *, nev=5, mode="matrix", checkpoint_path=None, scanned_sectors=None,
                     overwrite=False, batched=True):
    if checkpoint_path is not None and os.path.isfile(checkpoint_path) and not overwrite:
        ed_data.ed_scan_res = load_checkpoint(checkpoint_path).ed_scan_res
        return checkpoint_path
    todo = [i for i, ir in enumerate(ed_data.irrep_list)
            if i not in ed_data.ed_scan_res
            and (scanned_sectors is None or ir.label in scanned_sectors)]
    if mode not in ("matrix", "matrixfree"):
        raise ValueError(f"Unknown ED scan mode: {mode}. Use 'matrix' or 'matrixfree'.")
    if mode == "matrixfree" and batched and len(ed_data.irrep_list) <= 64 and todo:
        res = solve_sectors_batched(ed_data, todo, nev=nev)
        for s in todo:
            ed_data.ed_scan_res[s] = res[s]
        if checkpoint_path is not None:
            save_checkpoint(ed_data, checkpoint_path)
        return checkpoint_path
    for idx in todo:
        label = ed_data.irrep_list[idx].label
        if mode == "matrixfree":
            ed_scan_at_irrep_matrixfree(label, ed_data, nev=nev)
        else:
            ed_scan_at_irrep_matrix(label, ed_data, nev=nev)
        if checkpoint_path is not None:
            save_checkpoint(ed_data, checkpoint_path)
    return checkpoint_path


def save_checkpoint(ed_data, path: str) -> None:
    """Atomic pickle (temporary file + ``os.replace``) of the results
    (``symmetry_resolved_ed.py:2530-2549``); device tables are not stored."""
    os.makedirs(os.path.dirname(os.path.abspath(path)) or ".", exist_ok=True)
    tmp = path + ".tmp"
    try:
        with open(tmp, "wb") as f:
            pickle.dump(ed_data, f, protocol=pickle.HIGHEST_PROTOCOL)
        os.replace(tmp, path)
    finally:
        if os.path.isfile(tmp):
            os.remove(tmp)


def load_checkpoint(path: str):
    with open(path, "rb") as f:
        return pickle.load(f)


def ed_scan_checkpoint_filename(model, twisted_phases_over_2π, filling_fraction) -> str:
    """Checkpoint name of one flux point (``symmetry_resolved_ed.py:2571-2600``)."""
    params_short = {k: round(v, 3) if isinstance(v, (int, float)) else v
                    for k, v in model.params.items()}
    return (
        f"{model.tb_model.model_name}_{model.lattice.sample_size}_ν_graph="
        f"{filling_fraction.numerator}_{filling_fraction.denominator}_"
        f"twisted_phases_over_2π={twisted_phases_over_2π}_params={params_short}.pkl"
    )


def ed_scan(ed_data, *, nev: int = 5, mode: str = "matrix", scanned_sectors=None,
            checkpoint_path: str | None = None, checkpoint_dir: str = "checkpoints",
            overwrite: bool = False, flux_direction: int = 1,
            twisted_phases_over_2π_list: list[float] | None = None):
    """Sector scan, or flux scan along ``flux_direction`` (1-based)
    (``symmetry_resolved_ed.py:2608-2703``).  Each flux point gets its own
    ``Symmetry_Resolved_ED_Data`` checkpoint, as in the reference; its catalog
    is a phase-updated copy of the zero-flux one."""
    from .second_quantized_model import update_second_quantized_model_with_twisted_phases

    if mode not in ("matrix", "matrixfree"):
        raise ValueError(f"Unknown ED scan mode: {mode}.")
    if twisted_phases_over_2π_list is None:
        p = _ed_scan_sectors(ed_data, nev=nev, mode=mode, checkpoint_path=checkpoint_path,
                             scanned_sectors=scanned_sectors, overwrite=overwrite)
        return None if p is None else [p]
    model = ed_data.second_quantized_model
    os.makedirs(checkpoint_dir, exist_ok=True)
    dim = model.lattice.dim
    paths = []
    base = ed_data.orbit_catalog
    for th in twisted_phases_over_2π_list:
        flux = [0.0] * dim
        flux[flux_direction - 1] = float(th)
        name = ed_scan_checkpoint_filename(model, flux, ed_data.filling_fraction)
        path = os.path.join(checkpoint_dir, name)
        if os.path.isfile(path) and not overwrite:
            paths.append(path)
            continue
        update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=flux)
        group = build_translation_group(model.lattice, flux)
        cat = base.clone()
        update_orbit_stabilizer_phases(cat, group, model.particle_statistics)
        th_data = Symmetry_Resolved_ED_Data(model, ed_data.n_filled, ed_data.filling_fraction, group,
                                            build_irrep_list(group, model.lattice), cat,
                                            [0] * len(ed_data.irrep_list))
        _ed_scan_sectors(th_data, nev=nev, mode=mode, scanned_sectors=scanned_sectors,
                         overwrite=overwrite)
        save_checkpoint(th_data, path)
        paths.append(path)
    return paths


def full_ed(second_quantized_model, n_filled: int, *, nev: int = 5):
    """Identity-group ED (``symmetry_resolved_ed.py:2966-2992``)."""
    G = build_identity_group(second_quantized_model.lattice.n_site)
    data = build_ed_data(second_quantized_model,
                         filling_fraction=Fraction(n_filled, second_quantized_model.lattice.n_site),
                         symmetry_group=G)
    ed_scan(data, nev=nev)
    return data.ed_scan_res[0]


def _spectrum_matrix(ed_data, shift_to_zero=True):
    scanned = sorted(ed_data.ed_scan_res.keys())
    if not scanned:
        return np.zeros((0, 0))
    nev = max(len(ed_data.ed_scan_res[i][0]) for i in scanned)
    spec = np.full((len(ed_data.irrep_list), nev), np.nan)
    for i in scanned:
        v = ed_data.ed_scan_res[i][0]
        spec[i, : len(v)] = v
    if shift_to_zero:
        fin = spec[~np.isnan(spec)]
        if fin.size:
            spec = spec - np.min(fin)
    return spec


def print_spectrum(ed_data, *, shift_to_zero: bool = True):
    """Print rows = irreps, cols = eigenvalue index (``:3029-3056``)."""
    spec = _spectrum_matrix(ed_data, shift_to_zero)
    if spec.size == 0:
        return spec
    print("ED Spectrum (rows = irrep, cols = eigenvalue #):")
    for i in range(spec.shape[0]):
        s = "  ".join("  NaN" if math.isnan(x) else f"{x:.8f}" for x in spec[i])
        print(f"  [{i}] {ed_data.irrep_list[i].label!r}: {s}")
    return spec
