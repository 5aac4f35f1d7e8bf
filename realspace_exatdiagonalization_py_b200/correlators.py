"""Correlators of one sector eigenstate on the device.

Keeps the contracts of the reference's ``off_diagonal_long_range_order`` /
``compute_odlro_map`` (``observables/off_diagonal_long_range_order.py:43-197``)
and ``static_structure_factor`` / ``compute_structure_factor_map``
(``observables/static_structure_factor.py:54-208, 380-527, 789-905``): the same
arguments, ED bootstrap, return values and layouts.  The reductions over the
sector's orbits run on the GPU:

* ``rsed_one_body_density`` -- <a_i^dagger a_j> for all (i, j) in one pass
  over the (orbit, group element) kets, every hop projected back into the
  sector through the catalog table;
* ``rsed_density_pairs`` -- sum over the representatives of |c|^2 n_a n_b;
  the group sum that turns it into <n_i n_j> and the densities is a |G| x N^2
  scatter on the host, followed by the flavour filters and the Fourier sums.

Manifold averages (an incoherent mixture of (sector, level) states) combine
the per-state correlation matrices with normalised weights before the
connected part is taken; the allowed-momenta variants fold the mesh into the
first Brillouin zone (the nearest of the 25 shifts by n_1 b_1 + n_2 b_2).

The momentum mesh of ``static_structure_factor`` comes from
``lattice.initialize_uniform_grids_from_lattice`` (the q = sum_d (n_d/L_d) b_d
grid of the ``tightbinding_py`` dependency, which the reference imports).
"""

from __future__ import annotations

import ctypes
from fractions import Fraction
from typing import Callable

import numpy as np
import torch

from . import _lib

__all__ = ["off_diagonal_long_range_order", "compute_odlro_map", "static_structure_factor",
           "compute_structure_factor_map", "static_structure_factor_manifold_average",
           "compute_structure_factor_manifold_average_map", "structure_factor_allowed_momenta",
           "structure_factor_manifold_allowed_momenta"]


def _bootstrap_ed_sector(model, sector_label, filling_fraction, target_eigval_idx: int, ed_mode: str, ed_data):
    """``(ed_data, basis, c)``: the sector's ``target_eigval_idx``-th (1-based)
    eigenvector, scanning the zero-flux model first when no ``ed_data`` is
    given (``static_structure_factor.py:380-459``)."""
    from .ed import build_ed_data, ed_scan
    from .second_quantized_model import update_second_quantized_model_with_twisted_phases
    from .sector import Symmetry_Sector_Basis, build_symmetry_sector_basis
    from .symmetry import build_identity_group, build_translation_group

    lattice = model.lattice
    if ed_data is None:
        flux0 = [0.0] * lattice.dim
        update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=flux0)
        G = (build_identity_group(lattice.n_site) if sector_label == "identity"
             else build_translation_group(lattice, flux0))
        ed_data = build_ed_data(model, filling_fraction=Fraction(filling_fraction), symmetry_group=G)
        ed_scan(ed_data, nev=max(target_eigval_idx, 2), mode=ed_mode,
                scanned_sectors=None if sector_label == "identity" else [sector_label])
    idx = next((i for i, ir in enumerate(ed_data.irrep_list) if ir.label == sector_label), None)
    if idx is None:
        raise ValueError(f"Sector {sector_label!r} not found in ed_data.irrep_list.")
    if idx not in ed_data.ed_scan_res:
        raise ValueError(f"Sector {sector_label!r} was not scanned.")
    _, vecs = ed_data.ed_scan_res[idx]
    if target_eigval_idx > vecs.shape[1]:
        raise ValueError(f"target_eigval_idx={target_eigval_idx} exceeds {vecs.shape[1]} eigenvectors.")
    _, sset = ed_data._device()
    basis = (Symmetry_Sector_Basis(ed_data.irrep_list[idx], ed_data.orbit_catalog, sset, idx) if sset is not None
             else build_symmetry_sector_basis(ed_data.orbit_catalog, ed_data.irrep_list[idx]))
    return ed_data, basis, vecs[:, target_eigval_idx - 1]


def _orbit_vector(basis, c) -> torch.Tensor:
    cat = basis.catalog
    dev = cat.table.device
    x = torch.zeros(cat.n_orbits, dtype=torch.complex128, device=dev)
    rows = basis.device_rows()[0].long()
    x[rows] = torch.as_tensor(np.asarray(c) if not torch.is_tensor(c) else c).to(dev, torch.complex128).reshape(-1)
    return x


def one_body_density_matrix(basis, c, *, stream=None) -> np.ndarray:
    """``rho[i, j] = <psi| a_{i+1}^dagger a_{j+1} |psi>`` (0-based) of the
    sector state ``c`` (basis order of ``basis``), from the device."""
    lib = _lib.lib()
    cat = basis.catalog
    n = cat.symmetry_group.n_site
    x = _orbit_vector(basis, c)
    sset = basis.sector_set
    rho = torch.empty((n, n), dtype=torch.complex128, device=x.device)
    scratch = torch.empty(int(lib.rsed_obdm_scratch_bytes(n)), dtype=torch.uint8, device=x.device)
    _lib.check(lib.rsed_one_body_density(ctypes.byref(cat.dgroup.c), _lib.ptr(cat.table), cat.n_orbits,
                                         _lib.ptr(cat.repr_masks), _lib.ptr(cat.stab_mask), _lib.ptr(sset.member),
                                         int(basis.sector_index), _lib.ptr(sset.chi[basis.sector_index].contiguous()),
                                         _lib.ptr(x), _lib.ptr(rho), _lib.ptr(scratch), scratch.numel(),
                                         _lib.stream_ptr(stream)))
    if stream is not None:
        stream.synchronize()
    return rho.cpu().numpy()


def density_pairs(basis, c, *, stream=None) -> np.ndarray:
    """``D[a, b] = sum over the sector's representatives of |c|^2 n_a n_b``."""
    lib = _lib.lib()
    cat = basis.catalog
    n = cat.symmetry_group.n_site
    x = _orbit_vector(basis, c)
    D = torch.empty((n, n), dtype=torch.float64, device=x.device)
    scratch = torch.empty(int(lib.rsed_density_pairs_scratch_bytes(n)), dtype=torch.uint8, device=x.device)
    _lib.check(lib.rsed_density_pairs(n, cat.n_orbits, _lib.ptr(cat.repr_masks), _lib.ptr(x), _lib.ptr(D),
                                      _lib.ptr(scratch), scratch.numel(), _lib.stream_ptr(stream)))
    if stream is not None:
        stream.synchronize()
    return D.cpu().numpy()


def _build_density_correlation_matrix(C, density_a, density_b, c, basis, n_site: int, flavor_a, flavor_b,
                                      particle_statistics=None, *, subtract_disconnected: bool = True):
    """Fill ``C`` (connected <n_i n_j>), ``density_a`` and ``density_b`` in place
    from the device pair sums (``static_structure_factor.py:54-149``):
    <n_i n_j> = (1/|G|) sum_g D[a, b] at i = g(a), j = g(b)."""
    D = density_pairs(basis, c)
    perm0 = np.array([[p - 1 for p in op.perm] for op in basis.symmetry_group.operations], dtype=np.int64)
    ng = perm0.shape[0]
    full = np.zeros((n_site, n_site))
    for g in range(ng):
        pg = perm0[g]
        full[np.ix_(pg, pg)] += D
    full /= ng
    dens = np.diag(full).copy()
    fa = np.array([bool(flavor_a(i + 1)) for i in range(n_site)])
    fb = np.array([bool(flavor_b(i + 1)) for i in range(n_site)])
    density_a[:] = np.where(fa, dens, 0.0)
    density_b[:] = np.where(fb, dens, 0.0)
    C[:] = np.where(fa[:, None] & fb[None, :], full, 0.0)
    if subtract_disconnected:
        C -= np.outer(density_a, density_b)
    return C


def _precompute_phases(q_points, positions) -> np.ndarray:
    """``phases[q, i] = exp(-i q . r_i)`` (``static_structure_factor.py:152-177``)."""
    pos = np.asarray([np.asarray(p, dtype=np.float64) for p in positions]).reshape(len(positions), -1)
    out = np.empty((len(q_points), len(positions)), dtype=np.complex128)
    for k, q in enumerate(q_points):
        out[k] = np.exp(-1j * (pos @ np.asarray(q, dtype=np.float64)))
    return out


def _fourier_transform(S_q: np.ndarray, phases: np.ndarray, C: np.ndarray, n_site: int) -> np.ndarray:
    """``S_q[k] = Re(ph_k^T C conj(ph_k)) / N`` in place (``:180-207``)."""
    for k in range(phases.shape[0]):
        ph = phases[k]
        S_q[k] = float(np.real(np.dot(np.dot(ph, C), np.conj(ph)))) / n_site
    return S_q


def _dense_grid(k_resolution: int):
    span = 3 * np.pi
    kx = np.linspace(-span / 2, span / 2, num=k_resolution)
    ky = np.linspace(-span / 2, span / 2, num=k_resolution)
    return kx, ky, [[x, y] for y in ky for x in kx]


def off_diagonal_long_range_order(model, sector_label, *, target_eigval_idx: int = 1, filling_fraction,
                                  ed_mode: str = "matrix", ed_data=None) -> np.ndarray:
    """One-body density matrix ``odlro[i, j] = <a_{i+1}^dagger a_{j+1}>``
    (complex ``(n_site, n_site)``) of the sector's ``target_eigval_idx``-th
    state (``off_diagonal_long_range_order.py:43-140``)."""
    _, basis, c = _bootstrap_ed_sector(model, sector_label, filling_fraction, target_eigval_idx, ed_mode, ed_data)
    return one_body_density_matrix(basis, c)


def compute_odlro_map(model, sector_label, *, target_eigval_idx: int = 1, filling_fraction, k_resolution: int = 61,
                      ed_mode: str = "matrix", ed_data=None):
    """``(kx, ky, rho_map)`` with ``rho_map[i, j] = rho(kx[i], ky[j])`` =
    Re(conj(ph)^T odlro ph) / N over ``[-1.5 pi, 1.5 pi]^2`` (``:143-197``)."""
    lattice = model.lattice
    odlro = off_diagonal_long_range_order(model, sector_label, target_eigval_idx=target_eigval_idx,
                                          filling_fraction=filling_fraction, ed_mode=ed_mode, ed_data=ed_data)
    kx, ky, q = _dense_grid(k_resolution)
    phases = _precompute_phases(q, lattice.site_cart_list)
    flat = np.zeros(len(q))
    for k in range(len(q)):
        ph = phases[k]
        flat[k] = float(np.real(np.dot(np.dot(np.conj(ph), odlro), ph))) / lattice.n_site
    return kx, ky, flat.reshape(k_resolution, k_resolution, order="F")


def _structure_factor_C(model, sector_label, target_eigval_idx, filling_fraction, flavor_a, flavor_b, ed_mode,
                        ed_data):
    n = model.lattice.n_site
    flavor_a = flavor_a or (lambda i: True)
    flavor_b = flavor_b or (lambda i: True)
    _, basis, c = _bootstrap_ed_sector(model, sector_label, filling_fraction, target_eigval_idx, ed_mode, ed_data)
    C = np.zeros((n, n))
    _build_density_correlation_matrix(C, np.zeros(n), np.zeros(n), c, basis, n, flavor_a, flavor_b,
                                      model.particle_statistics)
    return C


def static_structure_factor(model, sector_label, *, target_eigval_idx: int = 1, filling_fraction,
                            flavor_a: Callable[[int], bool] | None = None,
                            flavor_b: Callable[[int], bool] | None = None, ed_mode: str = "matrix", ed_data=None):
    """``(q_points, S_q)``: the connected structure factor on the lattice's
    momentum mesh (``static_structure_factor.py:462-527``)."""
    from .lattice import initialize_uniform_grids_from_lattice

    lattice = model.lattice
    C = _structure_factor_C(model, sector_label, target_eigval_idx, filling_fraction, flavor_a, flavor_b, ed_mode,
                            ed_data)
    kgrid = initialize_uniform_grids_from_lattice(lattice)
    phases = _precompute_phases(kgrid.site_cart_list, lattice.site_cart_list)
    S_q = np.zeros(kgrid.nsite)
    _fourier_transform(S_q, phases, C, lattice.n_site)
    return list(kgrid.site_cart_list), S_q


def compute_structure_factor_map(model, sector_label, *, target_eigval_idx: int = 1, filling_fraction,
                                 flavor_a: Callable[[int], bool] | None = None,
                                 flavor_b: Callable[[int], bool] | None = None, k_resolution: int = 61,
                                 ed_data=None):
    """``(kx, ky, S_map)`` over ``[-1.5 pi, 1.5 pi]^2``, ``S_map[i, j] =
    S(kx[i], ky[j])`` (``static_structure_factor.py:789-850``; matrix-mode ED)."""
    lattice = model.lattice
    C = _structure_factor_C(model, sector_label, target_eigval_idx, filling_fraction, flavor_a, flavor_b, "matrix",
                            ed_data)
    kx, ky, q = _dense_grid(k_resolution)
    phases = _precompute_phases(q, lattice.site_cart_list)
    flat = np.zeros(len(q))
    _fourier_transform(flat, phases, C, lattice.n_site)
    return kx, ky, flat.reshape(k_resolution, k_resolution, order="F")


# ---- manifold averages and the first Brillouin zone ----------------------------


def _manifold_state_components(state):
    """``(sector, level)`` of a manifold state given as an object with
    ``sector``/``level``, a dict, or a pair (``static_structure_factor.py:530-550``)."""
    if hasattr(state, "sector") and hasattr(state, "level"):
        return tuple(int(x) for x in state.sector), int(state.level)
    if isinstance(state, dict) and "sector" in state and "level" in state:
        return tuple(int(x) for x in state["sector"]), int(state["level"])
    if isinstance(state, tuple) and len(state) == 2:
        return tuple(int(x) for x in state[0]), int(state[1])
    raise ValueError(f"A manifold state must provide `(sector, level)`; got {state!r}.")


def _manifold_connected_density_correlation(model, manifold_states, *, weights=None, filling_fraction,
                                            flavor_a=None, flavor_b=None, ed_mode: str = "matrix",
                                            ed_data=None) -> np.ndarray:
    """Connected <n_i n_j> of rho = sum_a w_a |psi_a><psi_a| (weights
    normalised to one; uniform by default): the weighted per-state
    correlations and densities, then the disconnected part of the mixture
    (``static_structure_factor.py:551-632``)."""
    if not manifold_states:
        raise ValueError("The manifold-state list must not be empty.")
    if weights is None:
        w = [1.0 / len(manifold_states)] * len(manifold_states)
    else:
        if len(weights) != len(manifold_states):
            raise ValueError(f"Received {len(weights)} weights for {len(manifold_states)} states.")
        if any(x < 0 for x in weights):
            raise ValueError("Manifold weights must be nonnegative.")
        total = sum(weights)
        if total <= 0:
            raise ValueError("At least one manifold weight must be positive.")
        w = [float(x) / total for x in weights]
    flavor_a = flavor_a or (lambda i: True)
    flavor_b = flavor_b or (lambda i: True)
    n = model.lattice.n_site
    C = np.zeros((n, n))
    da = np.zeros(n)
    db = np.zeros(n)
    for state, wt in zip(manifold_states, w):
        sector, level = _manifold_state_components(state)
        _, basis, vec = _bootstrap_ed_sector(model, sector, filling_fraction, level, ed_mode, ed_data)
        Cs, das, dbs = np.zeros((n, n)), np.zeros(n), np.zeros(n)
        _build_density_correlation_matrix(Cs, das, dbs, vec, basis, n, flavor_a, flavor_b,
                                          model.particle_statistics, subtract_disconnected=False)
        C += wt * Cs
        da += wt * das
        db += wt * dbs
    C -= np.outer(da, db)
    return C


def static_structure_factor_manifold_average(model, manifold_states, *, weights=None, filling_fraction,
                                             flavor_a=None, flavor_b=None, ed_mode: str = "matrix", ed_data=None):
    """``(q_points, S_q)`` of the manifold mixture on the lattice's momentum
    mesh (``static_structure_factor.py:635-683``)."""
    from .lattice import initialize_uniform_grids_from_lattice

    C = _manifold_connected_density_correlation(model, manifold_states, weights=weights,
                                                filling_fraction=filling_fraction, flavor_a=flavor_a,
                                                flavor_b=flavor_b, ed_mode=ed_mode, ed_data=ed_data)
    kgrid = initialize_uniform_grids_from_lattice(model.lattice)
    phases = _precompute_phases(kgrid.site_cart_list, model.lattice.site_cart_list)
    S_q = np.zeros(kgrid.nsite)
    _fourier_transform(S_q, phases, C, model.lattice.n_site)
    return list(kgrid.site_cart_list), S_q


def compute_structure_factor_manifold_average_map(model, manifold_states, *, weights=None, filling_fraction,
                                                  flavor_a=None, flavor_b=None, k_resolution: int = 61,
                                                  ed_mode: str = "matrix", ed_data=None):
    """``(kx, ky, S_map)`` of the manifold mixture over ``[-1.5 pi, 1.5 pi]^2``
    (``static_structure_factor.py:853-905``)."""
    C = _manifold_connected_density_correlation(model, manifold_states, weights=weights,
                                                filling_fraction=filling_fraction, flavor_a=flavor_a,
                                                flavor_b=flavor_b, ed_mode=ed_mode, ed_data=ed_data)
    kx, ky, q = _dense_grid(k_resolution)
    phases = _precompute_phases(q, model.lattice.site_cart_list)
    flat = np.zeros(len(q))
    _fourier_transform(flat, phases, C, model.lattice.n_site)
    return kx, ky, flat.reshape(k_resolution, k_resolution, order="F")


def _reciprocal_basis_vectors(lattice):
    """``[b1, b2]`` with a_i . b_j = 2 pi delta_ij (2-D lattices)."""
    if lattice.dim != 2:
        raise ValueError("BZ boundary plotting is implemented only for 2D lattices.")
    A = np.array([[lattice.brav_vec_list[0][0], lattice.brav_vec_list[1][0]],
                  [lattice.brav_vec_list[0][1], lattice.brav_vec_list[1][1]]], dtype=np.float64)
    B = 2 * np.pi * np.linalg.inv(A).T
    return [B[:, 0], B[:, 1]]


def _clip_polygon_by_halfplane(poly, normal, offset, *, atol: float = 1e-12):
    """The part of polygon ``poly`` with normal . p <= offset (Sutherland-Hodgman
    step against one half-plane)."""
    if not poly:
        return poly
    normal = np.asarray(normal, dtype=np.float64)
    out = []
    for idx in range(len(poly)):
        p = np.asarray(poly[idx], dtype=np.float64)
        q = np.asarray(poly[(idx + 1) % len(poly)], dtype=np.float64)
        fp, fq = float(np.dot(normal, p) - offset), float(np.dot(normal, q) - offset)
        if fp <= atol and fq <= atol:
            out.append(q)
        elif fp <= atol or fq <= atol:
            t = fp / (fp - fq)
            out.append(p + t * (q - p))
            if fq <= atol:
                out.append(q)
    return out


def _first_bz_polygon(lattice):
    """First Brillouin zone: a large square clipped by the bisecting
    half-planes of the reciprocal vectors n1 b1 + n2 b2 (|n| <= 2), shortest
    first."""
    b1, b2 = _reciprocal_basis_vectors(lattice)
    ext = 2.5 * max(float(np.linalg.norm(b1)), float(np.linalg.norm(b2)))
    poly = [np.array([-ext, -ext]), np.array([ext, -ext]), np.array([ext, ext]), np.array([-ext, ext])]
    Gs = [n1 * b1 + n2 * b2 for n1 in range(-2, 3) for n2 in range(-2, 3) if (n1, n2) != (0, 0)]
    Gs.sort(key=lambda g: float(np.linalg.norm(g)))
    for G in Gs:
        poly = _clip_polygon_by_halfplane(poly, G, float(np.dot(G, G)) / 2)
        if not poly:
            break
    return poly


def _fold_momentum_to_first_bz(q, lattice):
    """The shortest of q - n1 b1 - n2 b2, n1, n2 in -2..2 (the first strictly
    shorter one in that order); q itself for lattices that are not 2-D."""
    q = np.asarray(q, dtype=np.float64)
    if lattice.dim != 2:
        return q.copy()
    b1, b2 = _reciprocal_basis_vectors(lattice)
    best, best_n = q.copy(), float(np.dot(q, q))
    for n1 in range(-2, 3):
        for n2 in range(-2, 3):
            f = q - n1 * b1 - n2 * b2
            fn = float(np.dot(f, f))
            if fn < best_n:
                best, best_n = f, fn
    return best


def _fold_momenta_to_first_bz(q_points, lattice):
    return [_fold_momentum_to_first_bz(np.asarray(q, dtype=np.float64), lattice) for q in q_points]


def structure_factor_allowed_momenta(model, sector_label, *, target_eigval_idx: int = 1, filling_fraction,
                                     flavor_a=None, flavor_b=None, ed_mode: str = "matrix", ed_data=None,
                                     fold_to_first_bz: bool = True):
    """``(qx, qy, S_q)`` on the mesh, momenta folded into the first Brillouin
    zone (``static_structure_factor.py:734-780``)."""
    q, S = static_structure_factor(model, sector_label, target_eigval_idx=target_eigval_idx,
                                   filling_fraction=filling_fraction, flavor_a=flavor_a, flavor_b=flavor_b,
                                   ed_mode=ed_mode, ed_data=ed_data)
    pts = _fold_momenta_to_first_bz(q, model.lattice) if fold_to_first_bz else q
    return [p[0] for p in pts], [p[1] for p in pts], S


def structure_factor_manifold_allowed_momenta(model, manifold_states, *, weights=None, filling_fraction,
                                              flavor_a=None, flavor_b=None, ed_mode: str = "matrix", ed_data=None,
                                              fold_to_first_bz: bool = True):
    """``(qx, qy, S_q)`` of the manifold mixture, folded as above
    (``static_structure_factor.py:686-731``)."""
    q, S = static_structure_factor_manifold_average(model, manifold_states, weights=weights,
                                                    filling_fraction=filling_fraction, flavor_a=flavor_a,
                                                    flavor_b=flavor_b, ed_mode=ed_mode, ed_data=ed_data)
    pts = _fold_momenta_to_first_bz(q, model.lattice) if fold_to_first_bz else q
    return [p[0] for p in pts], [p[1] for p in pts], S
