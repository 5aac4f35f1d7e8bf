"""Symmetry groups, irreps and the scalar bitmask API (host side, exact integers).

These are the reference's data classes and scalar helpers
(``symmetry_resolved_ed.py:94-339, 930-1143, 1193-1217, 1412-1436,
2706-2898``), kept with the same names, argument meaning and errors so user
code ports unchanged.  They operate on one mask at a time with Python
integers; the bulk work (all C(N,k) states) runs in the CUDA kernels of
``librsed.so``.
"""

from __future__ import annotations

import cmath
import itertools
import math
from dataclasses import dataclass
from enum import Enum
from typing import Any

import numpy as np

Mask = int
COMPLEX_ONE = 1.0 + 0.0j
MAX_N_SITE_UINT64 = 63


class Particle_Statistics(Enum):
    """Hard-core bosons or spinless fermions (``second_quantized_model.py:29-45``)."""

    BOSONIC = "Bosonic"
    FERMIONIC = "Fermionic"

    def __repr__(self) -> str:  # pragma: no cover - cosmetic
        return f"Particle_Statistics.{self.name}"


@dataclass(init=False)
class Symmetry_Operation:
    """One group element: a site permutation (1-based) and per-site U(1)
    phases ``eta_g(i)`` (``symmetry_resolved_ed.py:930-974``)."""

    label: Any
    perm: list[int]
    perm_phases: np.ndarray

    def __init__(self, label: Any, perm: list[int], *, perm_phases=None):
        n_site = len(perm)
        if perm_phases is None:
            phases = np.full(n_site, COMPLEX_ONE, dtype=np.complex128)
        else:
            phases = np.asarray(perm_phases, dtype=np.complex128)
        assert phases.shape[0] == n_site, (
            "Symmetry_Operation: perm_phases must have length n_site."
        )
        self.label = label
        self.perm = [int(p) for p in perm]
        self.perm_phases = phases

    def __repr__(self) -> str:  # pragma: no cover - cosmetic
        return f"Symmetry_Operation(label={self.label!r}, perm={self.perm})"


@dataclass(init=False)
class Finite_Symmetry_Group:
    """Ordered list of operations; ``identity_idx`` is 0-based
    (``symmetry_resolved_ed.py:1016-1067``)."""

    name: str
    n_site: int
    operations: list[Symmetry_Operation]
    identity_idx: int

    def __init__(self, name: str, ops: list[Symmetry_Operation], *, identity_idx: int = 0):
        if len(ops) == 0:
            raise ValueError("Finite_Symmetry_Group: ops must not be empty.")
        n_site = len(ops[0].perm)
        for op in ops:
            if len(op.perm) != n_site or op.perm_phases.shape[0] != n_site:
                raise ValueError(
                    "Finite_Symmetry_Group: all operations must have "
                    "perm/perm_phases of length n_site."
                )
        if ops[identity_idx].perm != list(range(1, n_site + 1)):
            raise ValueError(
                "Finite_Symmetry_Group: the identity operation must have the trivial permutation."
            )
        self.name = name
        self.n_site = n_site
        self.operations = ops
        self.identity_idx = identity_idx

    def __repr__(self) -> str:  # pragma: no cover - cosmetic
        return (
            f"Finite_Symmetry_Group(name={self.name!r}, n_site={self.n_site}, "
            f"|G|={len(self.operations)})"
        )


def group_order(G: Finite_Symmetry_Group) -> int:
    return len(G.operations)


@dataclass(init=False)
class OneDim_Irrep:
    """A 1-D irrep: label and character of each group element (``:1412-1436``)."""

    label: Any
    values: np.ndarray

    def __init__(self, label: Any, values):
        self.label = label
        self.values = np.asarray(values, dtype=np.complex128)

    def __repr__(self) -> str:  # pragma: no cover - cosmetic
        return f"OneDim_Irrep(label={self.label!r}, |values|={len(self.values)})"


# ---------------------------------------------------------------------------
# scalar mask API
# ---------------------------------------------------------------------------


def apply_operation_to_mask(
    m: Mask, op: Symmetry_Operation, particle_statistics: Particle_Statistics
) -> tuple[Mask, complex]:
    """``U_g |m> = phase |g m>``; phase = prod of eta over occupied sites in
    ascending order, times the fermionic permutation parity counted as
    ``popcount(placed >> pi(i))`` (``symmetry_resolved_ed.py:977-1008``)."""
    tmp = m
    new_mask = 0
    phase = COMPLEX_ONE
    parity = 1
    fermion = particle_statistics is Particle_Statistics.FERMIONIC
    while tmp:
        low = tmp & -tmp
        site = low.bit_length()  # 1-based
        p = op.perm[site - 1]
        if fermion and (new_mask >> p).bit_count() & 1:
            parity = -parity
        new_mask |= 1 << (p - 1)
        phase *= op.perm_phases[site - 1]
        tmp ^= low
    return new_mask, phase * parity


def get_canonical_representative(
    m: Mask, G: Finite_Symmetry_Group, stats: Particle_Statistics
) -> tuple[Mask, int, complex]:
    """Smallest image of ``m`` over the group; ties keep the earlier ``g``
    (``symmetry_resolved_ed.py:1087-1114``)."""
    best = m
    best_g = G.identity_idx
    best_amp = COMPLEX_ONE
    for g_idx, g in enumerate(G.operations):
        img, alpha = apply_operation_to_mask(m, g, stats)
        if img < best:
            best, best_g, best_amp = img, g_idx, alpha
    return best, best_g, best_amp


def _binom_table(n_site: int, n_filled: int) -> np.ndarray:
    """``C(b, j)`` for ``b <= n_site``, ``j <= n_filled`` (``:143-158``)."""
    t = np.zeros((n_site + 1, n_filled + 1), dtype=np.int64)
    for b in range(n_site + 1):
        for j in range(min(b, n_filled) + 1):
            t[b, j] = math.comb(b, j)
    return t


def rank_combination(m: Mask, binom_table: np.ndarray) -> int:
    """Colexicographic rank ``sum_j C(b_j, j+1)`` (``:1193-1217``)."""
    r = 0
    j = 1
    while m:
        low = m & -m
        r += int(binom_table[low.bit_length() - 1, j])
        j += 1
        m ^= low
    return r


def rank_two_species(m: Mask, species_b: int, binom_table: np.ndarray, c_b: int) -> int:
    """Rank in a two-species basis: ``rank_A * C(|B|, k_B) + rank_B``, each
    species ranked in colex order over its own sites (ascending)."""
    ra = rb = 0
    ja = jb = 1
    while m:
        low = m & -m
        b = low.bit_length() - 1
        below = (species_b & (low - 1)).bit_count()
        if (species_b >> b) & 1:
            rb += int(binom_table[below, jb])
            jb += 1
        else:
            ra += int(binom_table[b - below, ja])
            ja += 1
        m ^= low
    return ra * c_b + rb


def unrank_combination(r: int, n_site: int, n_filled: int, binom_table: np.ndarray) -> Mask:
    """Inverse of :func:`rank_combination` (``:377-394`` for one rank)."""
    m = 0
    b = n_site - 1
    for j in range(n_filled, 0, -1):
        while int(binom_table[b, j]) > r:
            b -= 1
        m |= 1 << b
        r -= int(binom_table[b, j])
        b -= 1
    return m


def _gosper_next(x: Mask) -> Mask:
    """Next mask with the same popcount (``:1117-1129``)."""
    c = x & -x
    r = x + c
    return (((r ^ x) >> 2) // c) | r


def _first_combination_mask(n_filled: int) -> Mask:
    return 0 if n_filled == 0 else (1 << n_filled) - 1


def hopping_phase_for_stats(
    particle_statistics: Particle_Statistics, m: Mask, i_from: int, i_to: int
) -> complex:
    """Jordan-Wigner sign of the hop ``i_from -> i_to`` (1-based sites):
    ``(-1)^{#occupied sites strictly between}`` for fermions (``:1777-1810``)."""
    if particle_statistics is not Particle_Statistics.FERMIONIC or i_from == i_to:
        return COMPLEX_ONE
    lo, hi = min(i_from, i_to), max(i_from, i_to)
    between = ((1 << (hi - lo - 1)) - 1) << lo if hi - lo > 1 else 0
    return -COMPLEX_ONE if (m & between).bit_count() & 1 else COMPLEX_ONE


def _lin_table(n_site: int, n_filled: int) -> tuple[np.ndarray, np.ndarray, int]:
    """Split-table rank ``L[hi] + R[lo]`` (Lin 1990), for API parity with the
    reference catalog fields ``lin_left/lin_right/lin_n_right`` (``:161-211``)."""
    n_right = n_site // 2
    n_left = n_site - n_right
    right = np.zeros(1 << n_right, dtype=np.int64)
    for v in range(1 << n_right):
        r, j, t = 0, 1, v
        while t:
            low = t & -t
            r += math.comb(low.bit_length() - 1, j)
            j += 1
            t ^= low
        right[v] = r
    left = np.zeros(1 << n_left, dtype=np.int64)
    acc = 0
    for u in range(1 << n_left):
        left[u] = acc
        rem = n_filled - u.bit_count()
        if 0 <= rem <= n_right:
            acc += math.comb(n_right, rem)
    return left, right, n_right


LIN_TABLE_MAX_N_SITE = 42

# ---------------------------------------------------------------------------
# pre-built groups and irreps
# ---------------------------------------------------------------------------


def build_identity_group(n_site: int) -> Finite_Symmetry_Group:
    op = Symmetry_Operation("identity", list(range(1, n_site + 1)))
    return Finite_Symmetry_Group("identity", [op], identity_idx=0)


def _translation_phase(theta, cell, shifted, Lf) -> complex:
    # The same floating-point expression as symmetry_resolved_ed.py:2781-2788,
    # so the per-site phases (and every amplitude derived from them) agree
    # bit for bit with the reference's group.
    return cmath.exp(
        2j * math.pi * sum(th * (c - sc) / L for th, c, sc, L in zip(theta, cell, shifted, Lf))
    )


def build_translation_group(lattice, θ=None) -> Finite_Symmetry_Group:
    """Translations of the sample, with twisted-boundary phases
    ``exp(2*pi*i * sum_d theta_d (c_d - c'_d)/L_d)`` on every site
    (``symmetry_resolved_ed.py:2724-2790``).  Operation labels are the shift
    tuples in ``itertools.product`` order."""
    n_site = lattice.n_site
    L = lattice.sample_size
    if θ is None or len(θ) == 0:
        tw = getattr(lattice, "twisted_phases_over_2π", [])
        theta = [float(x) for x in tw] if tw else [0.0] * lattice.dim
    else:
        if len(θ) != lattice.dim:
            raise ValueError(f"θ must have length {lattice.dim}.")
        theta = [float(x) for x in θ]
    Lf = [float(x) for x in L]
    ops = []
    for shift in itertools.product(*[range(n) for n in L]):
        perm = [0] * n_site
        phases = np.zeros(n_site, dtype=np.complex128)
        for i, (cell, sub) in enumerate(lattice.site_list):
            shifted = tuple((c + s) % n for c, s, n in zip(cell, shift, L))
            perm[i] = lattice.site_to_index_map[(shifted, sub)]
            phases[i] = _translation_phase(theta, cell, shifted, Lf)
        ops.append(Symmetry_Operation(tuple(shift), perm, perm_phases=phases))
    return Finite_Symmetry_Group("translations", ops, identity_idx=0)


def build_identity_irrep_list() -> list[OneDim_Irrep]:
    return [OneDim_Irrep("identity", [1.0 + 0.0j])]


def build_translation_irrep_list(G: Finite_Symmetry_Group, lattice) -> list[OneDim_Irrep]:
    """Momentum irreps ``chi_(k1,k2)(d1,d2) = exp(2*pi*i (k1 d1/L1 + k2 d2/L2))``,
    ``k1``-major (``symmetry_resolved_ed.py:2824-2860``)."""
    assert G.name == "translations" and group_order(G) == math.prod(lattice.sample_size)
    L1, L2 = lattice.sample_size
    out = []
    for k1 in range(L1):
        for k2 in range(L2):
            chi = []
            for op in G.operations:
                dx, dy = op.label
                chi.append(cmath.exp(2j * math.pi * (k1 * dx / L1 + k2 * dy / L2)))
            out.append(OneDim_Irrep((k1, k2), chi))
    return out


def build_irrep_list(G: Finite_Symmetry_Group, lattice) -> list[OneDim_Irrep]:
    if G.name == "identity":
        return build_identity_irrep_list()
    if G.name == "translations":
        return build_translation_irrep_list(G, lattice)
    raise ValueError(f"Irrep construction for group {G.name!r} is not yet implemented.")


def group_arrays(G: Finite_Symmetry_Group):
    """``(perm0 uint8 [|G|, N] 0-based, eta complex128 [|G|, N], angle float64)``
    — the kernel inputs (reference ``_group_kernel_arrays``, ``:1272-1295``, and
    ``np.angle`` of the phases as in ``:346-374``)."""
    perm0 = np.array([[p - 1 for p in op.perm] for op in G.operations], dtype=np.uint8)
    eta = np.array([op.perm_phases for op in G.operations], dtype=np.complex128)
    return perm0, eta, np.angle(eta)
