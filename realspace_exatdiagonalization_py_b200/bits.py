"""Scalar occupation-mask helpers of the reference's L0 layer
(``utils/bitwise_operations.py:37-214``), same names and semantics.

A mask is a Python ``int`` whose bit ``i - 1`` tells whether the 1-based site
``i`` is occupied.  These are the one-mask conveniences of the public API;
the bulk paths work on uint64 masks inside the CUDA kernels.
"""

from __future__ import annotations

from collections.abc import Iterable, Iterator

import numpy as np

from .symmetry import COMPLEX_ONE, MAX_N_SITE_UINT64, Mask

__all__ = [
    "Mask",
    "COMPLEX_ONE",
    "MAX_N_SITE_UINT64",
    "bitmask_of_site",
    "occupy_site_for_mask",
    "empty_site_for_mask",
    "is_site_occupied",
    "is_site_empty",
    "n_occupied_for_mask",
    "filled_site_iter_for_mask",
    "empty_site_iter_for_mask",
    "encode_configuration_to_bit_mask",
    "decode_bit_mask_to_configuration",
    "decode_bit_mask_to_configuration_inplace",
    "as_uint64_array",
]


def bitmask_of_site(i: int) -> Mask:
    """The mask with only site ``i`` (1-based) set."""
    return 1 << (i - 1)


def occupy_site_for_mask(m: Mask, i: int) -> Mask:
    """``m`` with site ``i`` (1-based) occupied."""
    return m | (1 << (i - 1))


def empty_site_for_mask(m: Mask, i: int) -> Mask:
    """``m`` with site ``i`` (1-based) emptied."""
    return m & ~(1 << (i - 1))


def is_site_occupied(m: Mask, i: int) -> bool:
    """Whether site ``i`` (1-based) is occupied in ``m``."""
    return (m >> (i - 1)) & 1 == 1


def is_site_empty(m: Mask, i: int) -> bool:
    """Whether site ``i`` (1-based) is empty in ``m``."""
    return (m >> (i - 1)) & 1 == 0


def n_occupied_for_mask(m: Mask) -> int:
    """Number of occupied sites (population count)."""
    return m.bit_count()


def filled_site_iter_for_mask(m: Mask, n_site: int) -> Iterator[int]:
    """Occupied 1-based sites of ``m`` among ``1..n_site``, ascending
    (``0b10110``, 5 sites -> 2, 3, 5)."""
    return (i for i in range(1, n_site + 1) if (m >> (i - 1)) & 1)


def empty_site_iter_for_mask(m: Mask, n_site: int) -> Iterator[int]:
    """Empty 1-based sites of ``m`` among ``1..n_site``, ascending
    (``0b10110``, 5 sites -> 1, 4)."""
    return (i for i in range(1, n_site + 1) if not (m >> (i - 1)) & 1)


def encode_configuration_to_bit_mask(occ: Iterable[int]) -> Mask:
    """Mask of a list of occupied 1-based sites."""
    m = 0
    for i in occ:
        m |= 1 << (int(i) - 1)
    return m


def decode_bit_mask_to_configuration(m: Mask, n_site: int) -> list[int]:
    """Occupied 1-based sites of ``m``, ascending (inverse of
    :func:`encode_configuration_to_bit_mask`)."""
    return list(filled_site_iter_for_mask(m, n_site))


def decode_bit_mask_to_configuration_inplace(occ: list[int], m: Mask, n_site: int) -> list[int]:
    """Overwrite ``occ`` (length = popcount of ``m``, asserted) with the
    occupied 1-based sites of ``m``; returns ``occ``."""
    assert len(occ) == m.bit_count(), (
        "decode_bit_mask_to_configuration_inplace: length(occ) must equal "
        "the number of occupied sites in the mask."
    )
    for k, i in enumerate(filled_site_iter_for_mask(m, n_site)):
        occ[k] = i
    return occ


def as_uint64_array(mask_list: list[Mask]) -> np.ndarray:
    """Masks as a 1-D uint64 array."""
    return np.asarray(mask_list, dtype=np.uint64)
