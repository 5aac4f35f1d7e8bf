"""Sector state -> Fock amplitudes (the first consumer of sector eigenvectors:
entanglement spectra and Chern-number links of the reference's observables).

``expand_sector_state_to_fock_amplitudes`` keeps the contract of the
reference's ``_expand_sector_state_to_fock_amplitudes``
(``observables/entanglement_spectrum.py:82-145``): a sector vector in the
basis order of ``Symmetry_Sector_Basis`` in, a ``{mask: amplitude}`` dictionary
of unit norm out, amplitudes at or below ``atol`` dropped, ``ValueError`` for a
near-zero norm.  The expansion itself is one pass of ``rsed_fock_expand`` over
the catalog's table on the GPU; ``as_dict=False`` returns the nonzero masks and
amplitudes as device tensors instead.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .sector import Symmetry_Sector_Basis

__all__ = ["expand_sector_state_to_fock_amplitudes", "_expand_sector_state_to_fock_amplitudes"]


def expand_sector_state_to_fock_amplitudes(c, basis: Symmetry_Sector_Basis, particle_statistics=None, *,
                                           atol: float = 1e-12, as_dict: bool = True, stream=None):
    lib = _lib.lib()
    cat = basis.catalog
    dev = cat.table.device
    n_orb = cat.n_orbits
    if basis.dim == 0:
        raise ValueError("Expanded state has near-zero norm.")
    cvec = torch.as_tensor(np.asarray(c) if not torch.is_tensor(c) else c).to(dev, torch.complex128).reshape(-1)
    if cvec.numel() != basis.dim:
        raise ValueError(f"sector vector has {cvec.numel()} entries, the basis {basis.dim}")
    oor, _ = basis.device_rows()
    xo = torch.zeros(n_orb, dtype=torch.complex128, device=dev)
    xo[oor.long()] = cvec
    chi = basis.sector_set.chi[basis.sector_index].contiguous()
    n_states = cat.n_states
    amp = torch.empty(n_states, dtype=torch.complex128, device=dev)
    masks = torch.empty(n_states, dtype=torch.int64, device=dev)
    scratch = torch.empty(int(lib.rsed_fock_scratch_bytes(n_states)), dtype=torch.uint8, device=dev)
    norm2 = ctypes.c_double(0.0)
    _lib.check(lib.rsed_fock_expand(ctypes.byref(cat.dgroup.c), _lib.ptr(cat.table), n_orb,
                                    _lib.ptr(cat.repr_masks), _lib.ptr(cat.stab_mask), _lib.ptr(xo), _lib.ptr(chi),
                                    float(atol), _lib.ptr(amp), _lib.ptr(masks), ctypes.byref(norm2),
                                    _lib.ptr(scratch), scratch.numel(), _lib.stream_ptr(stream)))
    nz = torch.nonzero(amp != 0).reshape(-1)
    m_nz, a_nz = masks[nz], amp[nz]
    if not as_dict:
        return m_nz, a_nz
    keys = (m_nz.cpu().numpy().view(np.uint64)).tolist()
    vals = a_nz.cpu().numpy().tolist()
    return dict(zip(keys, vals))


# the reference's (private) name
_expand_sector_state_to_fock_amplitudes = expand_sector_state_to_fock_amplitudes
