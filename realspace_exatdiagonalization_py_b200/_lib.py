"""ctypes binding of ``librsed.so`` (the C ABI declared in ``include/rsed.h``).

The product path has no CPU fallback: importing a compute entry point without
the built library or without a CUDA device raises immediately.
"""

from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_int64, c_size_t, c_void_p

_PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_PKG_DIR, "librsed.so")

RSED_OK = 0
RSED_EINVAL = -1
RSED_ECUDA = -2
RSED_ENOTCONV = -3
RSED_ERANGE = -4
RSED_EBREAKDOWN = -5
RSED_ESCRATCH = -6
RSED_ETIMEOUT = -7

_ERR_NAMES = {
    RSED_EINVAL: "RSED_EINVAL",
    RSED_ECUDA: "RSED_ECUDA",
    RSED_ENOTCONV: "RSED_ENOTCONV",
    RSED_ERANGE: "RSED_ERANGE",
    RSED_EBREAKDOWN: "RSED_EBREAKDOWN",
    RSED_ESCRATCH: "RSED_ESCRATCH",
    RSED_ETIMEOUT: "RSED_ETIMEOUT",
}


class RsedError(RuntimeError):
    """A librsed call failed with a CUDA or solver error."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{_ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


class RsedGroup(ctypes.Structure):
    _fields_ = [
        ("n_site", c_int32),
        ("n_filled", c_int32),
        ("n_group", c_int32),
        ("fermionic", c_int32),
        ("n_states", c_int64),
        ("binom", c_void_p),
        ("perm", c_void_p),
        ("angle", c_void_p),
        ("eta", c_void_p),
        ("species_b", ctypes.c_uint64),
        ("n_filled_b", c_int32),
        ("reserved_b", c_int32),
    ]


class RsedModel(ctypes.Structure):
    _fields_ = [
        ("n_site", c_int32),
        ("n_filled", c_int32),
        ("n_group", c_int32),
        ("fermionic", c_int32),
        ("n_states", c_int64),
        ("n_orbits", c_int64),
        ("binom", c_void_p),
        ("table", c_void_p),
        ("repr_masks", c_void_p),
        ("n_terms", c_int32),
        ("term_begin", c_void_p),
        ("term_to", c_void_p),
        ("term_amp", c_void_p),
        ("term_jw", c_void_p),
        ("hdiag", c_void_p),
        ("proj_rowptr", c_void_p),
        ("proj_cg", c_void_p),
        ("proj_w64", c_void_p),
        ("proj_w32", c_void_p),
        ("species_b", ctypes.c_uint64),
        ("n_filled_b", c_int32),
        ("reserved_b", c_int32),
    ]


class RsedSectors(ctypes.Structure):
    _fields_ = [
        ("n_sectors", c_int32),
        ("n_cols", c_int32),
        ("ld", c_int32),
        ("n_group", c_int32),
        ("member", c_void_p),
        ("sqrt_stab", c_void_p),
        ("chi", c_void_p),
        ("col_sector", c_void_p),
    ]


class RsedLanczos(ctypes.Structure):
    _fields_ = [
        ("n_inst", c_int32),
        ("n_slots", c_int32),
        ("nev", c_int32),
        ("keep_blocks", c_int32),
        ("max_restarts", c_int32),
        ("precision", c_int32),
        ("bmax", c_int32),
        ("chunk_rows", c_int32),
        ("pm", c_int32),
        ("reserved", c_int32),
        ("tol", c_double),
        ("inst_col0", c_void_p),
        ("inst_b", c_void_p),
        ("V", c_void_p),
        ("W", c_void_p),
        ("Xf", c_void_p),
        ("P", c_void_p),
        ("coef", c_void_p),
        ("partial", c_void_p),
        ("partial_len", c_int64),
        ("ritz_val", c_void_p),
        ("ritz_vec", c_void_p),
        ("resid", c_void_p),
        ("state", c_void_p),
    ]


# name -> (restype, argtypes); every symbol include/rsed.h declares.
SIGNATURES = {
    "rsed_version": (c_char_p, []),
    "rsed_last_error": (c_char_p, []),
    "rsed_catalog_scratch_bytes": (c_size_t, [POINTER(RsedGroup)]),
    "rsed_catalog_count": (c_int, [POINTER(RsedGroup), c_void_p, c_size_t, POINTER(c_int64), c_void_p]),
    "rsed_catalog_fill": (
        c_int,
        [POINTER(RsedGroup), c_void_p, c_size_t, c_int64, c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "rsed_stab_scratch_bytes": (c_size_t, [c_int64]),
    "rsed_catalog_stab_count": (
        c_int,
        [c_int64, c_void_p, c_void_p, POINTER(c_int64), c_void_p, c_size_t, c_void_p],
    ),
    "rsed_catalog_stab": (
        c_int,
        [POINTER(RsedGroup), c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "rsed_phase_update": (
        c_int,
        [POINTER(RsedGroup), c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "rsed_sector_members": (
        c_int,
        [c_int64, c_int32, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_double, c_void_p, c_void_p,
         c_void_p, c_void_p],
    ),
    "rsed_sector_scratch_bytes": (c_size_t, [c_int64, c_int32]),
    "rsed_sector_rows": (
        c_int,
        [c_int64, c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p],
    ),
    "rsed_sector_rows_noalloc": (c_int, [c_int64, c_void_p, c_int32, c_void_p, c_void_p, c_void_p]),
    "rsed_sector_rows_noalloc_max_orbits": (c_int64, []),
    "rsed_density_diag": (
        c_int,
        [c_int64, c_void_p, c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p],
    ),
    "rsed_apply_h": (
        c_int,
        [POINTER(RsedModel), POINTER(RsedSectors), c_void_p, c_void_p, c_int32, c_int32, c_void_p],
    ),
    "rsed_fock_scratch_bytes": (c_size_t, [c_int64]),
    "rsed_fock_expand": (c_int, [POINTER(RsedGroup), c_void_p, c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                                 c_double, c_void_p, c_void_p, POINTER(c_double), c_void_p, c_size_t, c_void_p]),
    "rsed_fock_overlap_scratch_bytes": (c_size_t, [c_int64, c_int32, c_int32]),
    "rsed_fock_overlaps": (c_int, [c_void_p, c_int64, c_int32, c_int32, c_void_p, c_int32, c_void_p, c_void_p,
                                   c_size_t, c_void_p]),
    "rsed_position_scratch_bytes": (c_size_t, [c_int64, c_int32, c_int32]),
    "rsed_position_overlaps": (c_int, [POINTER(RsedGroup), c_int64, c_void_p, c_void_p, c_void_p, c_void_p,
                                       c_void_p, c_int32, c_void_p, c_int32, c_void_p, c_void_p, c_size_t,
                                       c_void_p]),
    "rsed_obdm_scratch_bytes": (c_size_t, [c_int32]),
    "rsed_one_body_density": (c_int, [POINTER(RsedGroup), c_void_p, c_int64, c_void_p, c_void_p, c_void_p,
                                      c_int32, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t, c_void_p]),
    "rsed_density_pairs_scratch_bytes": (c_size_t, [c_int32]),
    "rsed_density_pairs": (c_int, [c_int32, c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_size_t,
                                   c_void_p]),
    "rsed_proj_scratch_bytes": (c_size_t, [c_int64]),
    "rsed_proj_count": (c_int, [POINTER(RsedModel), c_void_p, POINTER(c_int64), c_void_p, c_size_t, c_void_p]),
    "rsed_proj_fill": (c_int, [POINTER(RsedModel), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p]),
    "rsed_triplet_scratch_bytes": (c_size_t, [c_int64]),
    "rsed_triplets_count": (
        c_int,
        [POINTER(RsedModel), c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, POINTER(c_int64),
         c_void_p, c_size_t, c_void_p],
    ),
    "rsed_triplets_fill": (
        c_int,
        [POINTER(RsedModel), c_int64, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
         c_void_p, c_void_p],
    ),
    "rsed_csr_spmv": (
        c_int,
        [c_int64, c_void_p, c_void_p, c_void_p, c_int32, c_void_p, c_void_p, c_void_p],
    ),
    "rsed_lanczos_partial_len": (c_int64, [c_int64, c_int32, c_int32, c_int32]),
    "rsed_lanczos_coef_len": (c_int64, [c_int32, c_int32]),
    "rsed_lanczos_max_block": (c_int, []),
    "rsed_lanczos_max_keep": (c_int, []),
    "rsed_lanczos_max_projected": (c_int, []),
    "rsed_lanczos_prepare": (c_int, []),
    "rsed_lanczos_start": (
        c_int,
        [POINTER(RsedModel), POINTER(RsedSectors), POINTER(RsedLanczos), c_void_p],
    ),
    "rsed_lanczos_iterate": (
        c_int,
        [POINTER(RsedModel), POINTER(RsedSectors), POINTER(RsedLanczos), c_int32, c_int32, c_int32,
         c_void_p],
    ),
    "rsed_lanczos_iterate_span": (
        c_int,
        [POINTER(RsedModel), POINTER(RsedSectors), POINTER(RsedLanczos), c_int32, c_int32, c_int32,
         c_int32, c_void_p],
    ),
    "rsed_lanczos_rayleigh_ritz": (
        c_int,
        [POINTER(RsedModel), POINTER(RsedSectors), POINTER(RsedLanczos), c_int32, c_void_p],
    ),
    "rsed_lanczos_restart": (
        c_int,
        [POINTER(RsedModel), POINTER(RsedSectors), POINTER(RsedLanczos), c_void_p],
    ),
    "rsed_lanczos_persistent": (
        c_int,
        [POINTER(RsedModel), POINTER(RsedSectors), POINTER(RsedLanczos), c_int32, c_int32, c_void_p],
    ),
    "rsed_lanczos_extract": (
        c_int,
        [POINTER(RsedModel), POINTER(RsedSectors), POINTER(RsedLanczos), c_void_p, c_int64, c_void_p],
    ),
    "rsed_gather_rows": (
        c_int,
        [c_int64, c_void_p, c_void_p, c_int64, c_int32, c_void_p, c_int64, c_void_p],
    ),
    "rsed_scatter_rows": (
        c_int,
        [c_int64, c_void_p, c_void_p, c_int64, c_void_p, c_int64, c_int32, c_void_p],
    ),
    "rsed_gather_block": (
        c_int,
        [c_int64, c_void_p, c_void_p, c_int32, c_int64, c_void_p, c_int64, c_void_p],
    ),
    "rsed_scatter_block": (
        c_int,
        [c_int64, c_void_p, c_void_p, c_int32, c_int64, c_void_p, c_int64, c_int32, c_void_p],
    ),
    "rsed_device_sync": (c_int, [c_void_p]),
    "rsed_launch_count": (ctypes.c_longlong, []),
}

_lib = None


def load(path: str | None = None):
    """Load ``librsed.so`` and bind every declared symbol (no GPU needed)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise RuntimeError(
            f"librsed.so not found at {p}; build it with "
            "`python -m realspace_exatdiagonalization_py_b200.build`"
        )
    lib = ctypes.CDLL(p)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def lib():
    """The loaded library, requiring a CUDA device (compute entry points)."""
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError(
            "realspace_exatdiagonalization_py_b200 needs a CUDA device (B200, sm_100a); "
            "there is no CPU fallback"
        )
    return load()


def check(rc: int) -> None:
    """Raise the Python exception that matches a librsed status code."""
    if rc == RSED_OK:
        return
    msg = load().rsed_last_error().decode(errors="replace")
    if rc in (RSED_EINVAL, RSED_ERANGE):
        raise ValueError(msg)
    raise RsedError(rc, msg)


def stream_ptr(stream=None) -> int:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def ptr(t) -> int | None:
    return None if t is None else int(t.data_ptr())
