"""Lattice models used by the benchmarks and the parity tests.

The four model families of the reference (``models/heisenberg.py``,
``models/hubbard.py``, ``models/bosonic_fci.py``, ``models/fermionic_fci.py``)
written against this package's lattice module.  Each builder produces the
same Hamiltonian (same bonds, amplitudes and density terms) as its reference
counterpart; the test-suite checks the term multisets against the reference
builders and the energies against the reference's golden values.
"""

from __future__ import annotations

import cmath
import math
from fractions import Fraction
from typing import Any

from .lattice import (
    add_hopping_term,
    generate_bilinear_terms,
    initialize_real_space_lattice,
    initialize_real_space_tightbinding_model,
)
from .second_quantized_model import Real_Space_Second_Quantized_Model
from .symmetry import Particle_Statistics

__all__ = [
    "params_DNSheng",
    "params_Sun_Gu_Katsura_Sarma",
    "my_optimal_param",
    "build_heisenberg_second_quantized_model",
    "build_spinful_hubbard_second_quantized_model",
    "build_zero_flux_bosonic_fci_second_quantized_model",
    "build_zero_flux_fermionic_fci_second_quantized_model",
    "build_phase_explore_fermionic_checkerboard_model",
    "build_fermionic_checkerboard_tb_model",
    "CHECKERBOARD_TPP_DENOMINATOR",
    "default_fci_sectors",
    "default_fci_sectors_fermionic",
    "build_heisenberg_ed_data",
    "build_spinful_hubbard_ed_data",
    "build_bosonic_fci_ed_data",
    "build_fermionic_fci_ed_data",
    "config_model",
]

# t'' = 1 / CHECKERBOARD_TPP_DENOMINATOR in the Sun-Gu-Katsura-Das Sarma
# couplings (models/fermionic_fci.py:55)
CHECKERBOARD_TPP_DENOMINATOR = 2 + 2 * math.sqrt(2)

# Parameter sets of the reference's model modules (models/bosonic_fci.py:33-40,
# models/fermionic_fci.py:42-51, :759-772).
params_DNSheng: dict[str, float] = {
    "t": 1.0, "t'": 0.60, "t''": -0.58, "phi_over_2pi": 0.2, "V1": 0.0, "V2": 0.0,
}
params_Sun_Gu_Katsura_Sarma: dict[str, float] = {
    "t": 1.0,
    "t'_1": 1 / (2 + math.sqrt(2)),
    "t'_2": -1 / (2 + math.sqrt(2)),
    "t''": 1 / (2 + 2 * math.sqrt(2)),
    "phi_over_2pi": 1 / 8,
    "V1": 2.0,
    "V2": 1.0,
    "V3": 0.0,
}
my_optimal_param: dict[str, float] = {
    "t": -1.0,
    "t'_1": -1.4 / (2 + math.sqrt(2)),
    "t'_2": 1.4 / (2 + math.sqrt(2)),
    "t''": -1.0 / (2 + 2 * math.sqrt(2)),
    "phi_over_2pi": 1 / 8,
    "V1": 2.0,
    "V2": 0.45,
    "V3": 0.2,
    "λ": 2.8,
}


def _wrap(cell, shift, L):
    return tuple((c + s) % n for c, s, n in zip(cell, shift, L))


# ---------------------------------------------------------------------------
# Heisenberg chain (hard-core bosons; models/heisenberg.py:39-100)
# ---------------------------------------------------------------------------


def build_heisenberg_second_quantized_model(N: int, J: float = 1.0):
    """S_i.S_j on a ring: hopping J/2 on each bond, J n_i n_j on bonds and
    -J/2 n_i on sites (the constant of the spin mapping absorbed)."""
    lat = initialize_real_space_lattice(
        sample_size=[N, 1], brav_vec_list=[[1.0, 0.0], [0.0, 1.0]], sub_crys_list=[[0.0, 0.0]],
        lattice_name="1D_Chain", pbc_indicator=[True, False],
    )
    tb = initialize_real_space_tightbinding_model(lat, model_name="Heisenberg_Chain")
    add_hopping_term(tb, ((((0, 0), 1), ((1, 0), 1)), J / 2))
    site = lat.site_to_index_map
    dens = [(site[((x, 0), 1)], site[(((x + 1) % N, 0), 1)], complex(J)) for x in range(N)]
    dens += [(site[((x, 0), 1)], site[((x, 0), 1)], complex(-J / 2)) for x in range(N)]
    return Real_Space_Second_Quantized_Model(
        params={"J": J, "N_site": N}, lattice=lat, tb_model=tb,
        particle_statistics=Particle_Statistics.BOSONIC,
        bilinear_terms=generate_bilinear_terms(tb, twisted_phases_over_2π=[0.0] * lat.dim),
        density_density_terms=dens,
    )


# ---------------------------------------------------------------------------
# Spinful Hubbard on the square lattice, spin flattened into two sublattices
# (models/hubbard.py:30-100)
# ---------------------------------------------------------------------------


def build_spinful_hubbard_second_quantized_model(sample_size: list[int], t: float = 1.0,
                                                 U: float = 8.0):
    Lx, Ly = sample_size
    spatial = initialize_real_space_lattice(
        sample_size=sample_size, brav_vec_list=[[1.0, 0.0], [0.0, 1.0]], sub_crys_list=[[0.0, 0.0]],
        lattice_name="Square_Hubbard", pbc_indicator=[True, True],
    )
    tb0 = initialize_real_space_tightbinding_model(spatial, model_name="hubbard_spinless")
    add_hopping_term(tb0, ((((0, 0), 1), ((1, 0), 1)), complex(-t)))
    add_hopping_term(tb0, ((((0, 0), 1), ((0, 1), 1)), complex(-t)))
    lat = initialize_real_space_lattice(
        sample_size=sample_size, brav_vec_list=[[1.0, 0.0], [0.0, 1.0]],
        sub_crys_list=[[0.0, 0.0], [0.0, 0.0]], lattice_name="Square_Hubbard_Spinful",
        pbc_indicator=[True, True],
    )
    idx = lat.site_to_index_map
    bil = []
    for ((a, b), amp) in tb0.full_hopping_map.items():
        for spin in (1, 2):
            bil.append((idx[(a[0], spin)], idx[(b[0], spin)], complex(amp)))
    dens = [(idx[((x, y), 1)], idx[((x, y), 2)], complex(U)) for y in range(Ly) for x in range(Lx)]
    return Real_Space_Second_Quantized_Model(
        params={"t": t, "U": U}, lattice=lat,
        tb_model=initialize_real_space_tightbinding_model(lat, model_name="Hubbard"),
        particle_statistics=Particle_Statistics.FERMIONIC, bilinear_terms=bil,
        density_density_terms=dens,
    )


# ---------------------------------------------------------------------------
# Hard-core bosons on the Haldane honeycomb (models/bosonic_fci.py:44-167)
# ---------------------------------------------------------------------------

_HALDANE_NN = [((0, 0), (0, 0)), ((0, 0), (0, -1)), ((0, 0), (-1, 0))]  # sub 1 -> sub 2
_HALDANE_NNN = [((1, 0), +1), ((0, 1), -1), ((-1, 1), +1)]  # direction, flux sign on sub 1


def build_zero_flux_bosonic_fci_second_quantized_model(*, sample_size=None, params=None):
    sample_size = [3, 4] if sample_size is None else sample_size
    p = dict(params_DNSheng if params is None else params)
    t, t1, t2 = p["t"], p["t'"], p["t''"]
    phi = 2 * math.pi * p["phi_over_2pi"]
    lat = initialize_real_space_lattice(
        sample_size=sample_size, brav_vec_list=[[1.0, 0.0], [1 / 2, math.sqrt(3) / 2]],
        sub_crys_list=[[0.0, 0.0], [1 / 3, 1 / 3]], lattice_name="Haldane_Honeycomb",
        pbc_indicator=[True, True],
    )
    tb = initialize_real_space_tightbinding_model(lat, model_name="haldane_boson_FCI")
    for (c1, c2) in _HALDANE_NN:
        add_hopping_term(tb, (((c1, 1), (c2, 2)), -t))
    for sub, sgn in ((1, 1), (2, -1)):
        for d, s in _HALDANE_NNN:
            add_hopping_term(tb, ((((0, 0), sub), (d, sub)), -t1 * cmath.exp(1j * phi * s * sgn)))
    add_hopping_term(tb, ((((0, 0), 2), ((1, 1), 1)), -t2))
    add_hopping_term(tb, ((((1, 0), 1), ((0, 1), 2)), -t2))
    add_hopping_term(tb, ((((1, 0), 2), ((0, 1), 1)), -t2))
    L = lat.sample_size
    idx = lat.site_to_index_map
    dens, seen = [], set()

    def pair(i, j, V):
        if i == j:
            return
        key = (min(i, j), max(i, j))
        if key not in seen:
            seen.add(key)
            dens.append((key[0], key[1], complex(V)))

    if p["V1"] != 0.0:
        for (cell, sub) in lat.site_list:
            if sub == 1:
                for shift in ((0, 0), (0, -1), (-1, 0)):
                    pair(idx[(cell, 1)], idx[(_wrap(cell, shift, L), 2)], p["V1"])
    if p["V2"] != 0.0:
        for (cell, sub) in lat.site_list:
            for shift in ((1, 0), (0, 1), (-1, 1)):
                pair(idx[(cell, sub)], idx[(_wrap(cell, shift, L), sub)], p["V2"])
    return Real_Space_Second_Quantized_Model(
        params=p, lattice=lat, tb_model=tb, particle_statistics=Particle_Statistics.BOSONIC,
        bilinear_terms=generate_bilinear_terms(tb, twisted_phases_over_2π=[0.0] * lat.dim),
        density_density_terms=dens,
    )


# ---------------------------------------------------------------------------
# Spinless fermions on the checkerboard (models/fermionic_fci.py:62-220, 596-756)
# ---------------------------------------------------------------------------


def _checkerboard_tb(sample_size, t, t1_1, t1_2, t2, phi):
    lat = initialize_real_space_lattice(
        lattice_name="checkerboard", sample_size=sample_size, brav_vec_list=[[1.0, 0.0], [0.0, 1.0]],
        sub_crys_list=[[0.5, 0], [0.0, 0.5]], pbc_indicator=[True, True],
    )
    tb = initialize_real_space_tightbinding_model(lat, model_name="checkerboard")
    e_m, e_p = cmath.exp(-1j * phi), cmath.exp(1j * phi)
    nn = [(((0, 0), 1), ((0, 0), 2), e_m), (((0, 0), 1), ((1, 0), 2), e_p),
          (((0, 0), 2), ((0, 1), 1), e_m), (((1, 0), 2), ((0, 1), 1), e_p)]
    for a, b, e in nn:
        add_hopping_term(tb, ((a, b), -t * e))
    for (a, b, amp) in [(((0, 0), 1), ((1, 0), 1), t1_1), (((0, 0), 1), ((0, 1), 1), t1_2),
                        (((0, 0), 2), ((1, 0), 2), t1_2), (((0, 0), 2), ((0, 1), 2), t1_1)]:
        add_hopping_term(tb, ((a, b), -amp))
    for (a, b) in [(((0, 0), 1), ((1, 1), 1)), (((0, 0), 2), ((1, 1), 2)),
                   (((1, 0), 2), ((0, 1), 2)), (((0, 1), 1), ((1, 0), 1))]:
        add_hopping_term(tb, ((a, b), -t2))
    return tb


def _checkerboard_density(lat, V1, V2, V3):
    """Ordered site pairs (i, j), i != j, by sublattice and cell offset
    (models/fermionic_fci.py:175-212)."""
    L1, L2 = lat.sample_size
    out = []
    sites = list(enumerate(lat.site_list, start=1))
    for (i, (ci, si)) in sites:
        for (j, (cj, sj)) in sites:
            if i == j:
                continue
            d = tuple((b - a) % n for a, b, n in zip(ci, cj, lat.sample_size))
            if V1 != 0.0 and si == 1 and sj == 2 and d in ((0, 0), (1, 0), (0, L2 - 1), (1, L2 - 1)):
                out.append((i, j, complex(V1)))
            if V2 != 0.0 and si == sj and d in ((1, 0), (0, 1)):
                out.append((i, j, complex(V2)))
            if V3 != 0.0 and si == sj and d in ((1, 1), (1, L2 - 1)):
                out.append((i, j, complex(V3)))
    return out


def build_fermionic_checkerboard_tb_model(*, sample_size=None, params=None, flip_bands: bool = True):
    """Checkerboard tight-binding model with staggered flux
    (``models/fermionic_fci.py:58-131``): NN ``-t e^{-+i phi}``, NNN
    ``-t'_1 / -t'_2``, NNNN ``-t''``; ``flip_bands`` negates t, t'_1, t'_2 and
    t'' first (the flat band becomes the lower one)."""
    sample_size = [3, 4] if sample_size is None else sample_size
    q = dict(params_Sun_Gu_Katsura_Sarma if params is None else params)
    if flip_bands:
        for k in ("t", "t'_1", "t'_2", "t''"):
            q[k] = -q[k]
    return _checkerboard_tb(sample_size, q["t"], q["t'_1"], q["t'_2"], q["t''"], 2 * math.pi * q["phi_over_2pi"])


def build_zero_flux_fermionic_fci_second_quantized_model(*, sample_size=None, params=None,
                                                         flip_bands: bool = True):
    sample_size = [3, 4] if sample_size is None else sample_size
    p = dict(params_Sun_Gu_Katsura_Sarma if params is None else params)
    tb = build_fermionic_checkerboard_tb_model(sample_size=sample_size, params=p, flip_bands=flip_bands)
    lat = tb.lattice
    return Real_Space_Second_Quantized_Model(
        params=p, lattice=lat, tb_model=tb, particle_statistics=Particle_Statistics.FERMIONIC,
        bilinear_terms=generate_bilinear_terms(tb, twisted_phases_over_2π=[0.0] * lat.dim),
        density_density_terms=_checkerboard_density(lat, p["V1"], p["V2"], p["V3"]),
    )


def build_phase_explore_fermionic_checkerboard_model(params, sample_size, filling_fraction_per_band):
    """Pre-flipped hoppings, interactions scaled by ``params["λ"]``
    (``models/fermionic_fci.py:599-757``); returns ``(model, ed_data,
    n_filled, filling_fraction)`` with the translation-group ED data built on
    the device."""
    p = dict(params)
    tb = _checkerboard_tb(sample_size, p["t"], p["t'_1"], p["t'_2"], p["t''"],
                          2 * math.pi * p["phi_over_2pi"])
    lat = tb.lattice
    lam = p["λ"]
    model = Real_Space_Second_Quantized_Model(
        params=p, lattice=lat, tb_model=tb, particle_statistics=Particle_Statistics.FERMIONIC,
        bilinear_terms=generate_bilinear_terms(tb, twisted_phases_over_2π=[0.0] * lat.dim),
        density_density_terms=_checkerboard_density(lat, p["V1"] * lam, p["V2"] * lam, p["V3"] * lam),
    )
    ff = Fraction(filling_fraction_per_band) / lat.n_sub
    return model, _translation_ed_data(model, ff), int(lat.n_site * ff), ff


# ---------------------------------------------------------------------------
# ED data of the model families (the reference's convenience builders)
# ---------------------------------------------------------------------------


def _translation_ed_data(model, filling_fraction):
    from .ed import build_ed_data
    from .symmetry import build_translation_group

    return build_ed_data(model, filling_fraction=Fraction(filling_fraction),
                         symmetry_group=build_translation_group(model.lattice))


def default_fci_sectors(sample_size: list[int]) -> list[tuple[int, int]]:
    """Momentum labels of the two bosonic semion FCI ground states
    (``models/bosonic_fci.py:171-196``); unknown sizes warn and give [(0, 0)]."""
    known = {(2, 3): [(0, 0), (1, 0)], (3, 2): [(0, 0), (0, 1)],
             (3, 4): [(0, 0), (0, 2)], (4, 3): [(0, 0), (2, 0)]}
    key = tuple(sample_size)
    if key in known:
        return list(known[key])
    print(f"WARNING: Unknown `sample_size={sample_size}` — defaulting sector labels to [(0,0)]. "
          "The user should manually specify the FCI ground-state sectors.")
    return [(0, 0)]


def default_fci_sectors_fermionic(sample_size: list[int]) -> list[tuple[int, int]]:
    """Momentum labels of the three fermionic checkerboard FCI ground states
    (``models/fermionic_fci.py:222-255``); unknown sizes raise ValueError."""
    known = {(2, 3): [(0, 0), (0, 1), (0, 2)], (3, 2): [(0, 0), (1, 0), (2, 0)],
             (3, 4): [(0, 0), (1, 0), (2, 0)], (4, 3): [(0, 0), (0, 1), (0, 2)]}
    key = tuple(sample_size)
    if key in known:
        return list(known[key])
    raise ValueError(f"Unknown sample_size={sample_size} — run a full ED scan to identify the FCI sectors.")


def build_heisenberg_ed_data(N: int, J: float = 1.0):
    """Heisenberg ring at S^z = 0 (N/2 up spins) with the translation group
    (``models/heisenberg.py:97-118``)."""
    model = build_heisenberg_second_quantized_model(N, J)
    return _translation_ed_data(model, Fraction(N // 2, model.lattice.n_site))


def build_spinful_hubbard_ed_data(sample_size: list[int], t: float = 1.0, U: float = 8.0):
    """Spinful Hubbard at half filling (Lx * Ly particles on 2 Lx Ly
    spin-orbitals, total particle number) with the translation group
    (``models/hubbard.py:102-127``)."""
    model = build_spinful_hubbard_second_quantized_model(sample_size, t, U)
    return _translation_ed_data(model, Fraction(sample_size[0] * sample_size[1], model.lattice.n_site))


def build_bosonic_fci_ed_data(*, sample_size=None, params=None, filling_fraction_per_band=Fraction(1, 2)):
    """Haldane-boson FCI ED data (``models/bosonic_fci.py:394-424``): filling
    per flat band over the number of sublattices."""
    model = build_zero_flux_bosonic_fci_second_quantized_model(
        sample_size=[3, 4] if sample_size is None else sample_size,
        params=dict(params_DNSheng) if params is None else params)
    return _translation_ed_data(model, Fraction(filling_fraction_per_band) / model.lattice.n_sub)


def build_fermionic_fci_ed_data(*, sample_size=None, params=None, filling_fraction_per_band=Fraction(1, 3)):
    """Checkerboard-fermion FCI ED data (``models/fermionic_fci.py:548-581``)."""
    model = build_zero_flux_fermionic_fci_second_quantized_model(
        sample_size=[3, 4] if sample_size is None else sample_size,
        params=dict(params_Sun_Gu_Katsura_Sarma) if params is None else params)
    return _translation_ed_data(model, Fraction(filling_fraction_per_band) / model.lattice.n_sub)


# ---------------------------------------------------------------------------
# The benchmark workloads
# ---------------------------------------------------------------------------


def config_model(name: str) -> tuple[Any, int]:
    """``(model, n_filled)`` of a named workload.

    * ``heisenberg16``: Heisenberg ring N=16, J=1, 8 up spins.
    * ``checkerboard24``: checkerboard 3x4x2, 4 fermions, Sun-Gu-Katsura-Das Sarma
      hoppings (band-flipped), V1=1, V2=V3=0.
    * ``haldane32``: Haldane honeycomb 4x4x2, 8 hard-core bosons, t=1,
      t'=0.6 exp(+-0.4 pi i), t''=0, V1=1.
    * ``haldane24``: the same couplings on 3x4x2, 6 bosons (also nu = 1/2).
    * ``checkerboard48``: checkerboard 4x6x2, 8 fermions, couplings of
      ``checkerboard24``.
    * ``hubbard32``: spinful Fermi-Hubbard 4x4 (32 spin-orbitals), t=1, U=4,
      10 electrons; with ``hubbard_spin_species`` the basis fixes
      N_up = N_down = 5.
    """
    if name == "heisenberg16":
        return build_heisenberg_second_quantized_model(16, 1.0), 8
    if name in ("checkerboard24", "checkerboard48"):
        p = dict(params_Sun_Gu_Katsura_Sarma)
        p.update({"V1": 1.0, "V2": 0.0, "V3": 0.0})
        ss, nf = ([3, 4], 4) if name == "checkerboard24" else ([4, 6], 8)
        return build_zero_flux_fermionic_fci_second_quantized_model(sample_size=ss, params=p), nf
    if name == "hubbard32":
        return build_spinful_hubbard_second_quantized_model([4, 4], 1.0, 4.0), 10
    if name in ("haldane32", "haldane24"):
        p = {"t": 1.0, "t'": 0.6, "t''": 0.0, "phi_over_2pi": 0.2, "V1": 1.0, "V2": 0.0}
        ss, nf = ([4, 4], 8) if name == "haldane32" else ([3, 4], 6)
        return build_zero_flux_bosonic_fci_second_quantized_model(sample_size=ss, params=p), nf
    raise ValueError(f"unknown workload {name!r}")


def hubbard_spin_species(model, n_down: int) -> tuple[list[int], int]:
    """``species`` argument fixing ``n_down`` electrons on the spin-down
    orbitals of a model from :func:`build_spinful_hubbard_second_quantized_model`
    (sublattice 2 of every cell)."""
    idx = model.lattice.site_to_index_map
    sites = sorted(i for (cell_sub, i) in idx.items() if cell_sub[1] == 2)
    return sites, int(n_down)
