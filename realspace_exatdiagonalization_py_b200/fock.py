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

``expand_sector_state_to_fock_dense`` writes the same amplitudes as one dense
vector indexed by the catalog's table rank (the combinadic rank of the mask,
the same for every flux point of a catalog), and ``fock_overlaps`` takes the
overlap matrices of such vectors on the device (``rsed_fock_overlaps``): the
Berry links of ``many_body_chern_number`` without host dictionaries.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib
from .sector import Symmetry_Sector_Basis

__all__ = ["expand_sector_state_to_fock_amplitudes", "_expand_sector_state_to_fock_amplitudes",
           "expand_sector_state_to_fock_dense", "fock_overlaps"]


def _expand(c, basis, atol, amp, masks, stream):
    lib = _lib.lib()
    cat = basis.catalog
    dev = cat.table.device
    n_orb = cat.n_orbits
    if basis.dim == 0:
        raise ValueError("Expanded state has near-zero norm.")
    cvec = torch.as_tensor(np.asarray(c) if not torch.is_tensor(c) else c).to(dev, torch.complex128).reshape(-1)
    if cvec.numel() != basis.dim:
        raise ValueError(f"sector vector has {cvec.numel()} entries, the basis {basis.dim}")
    if amp.numel() != cat.n_states or amp.dtype != torch.complex128 or not amp.is_contiguous():
        raise ValueError("amplitude buffer must be a contiguous complex128 vector of n_states entries")
    oor, _ = basis.device_rows()
    xo = torch.zeros(n_orb, dtype=torch.complex128, device=dev)
    xo[oor.long()] = cvec
    chi = basis.sector_set.chi[basis.sector_index].contiguous()
    scratch = torch.empty(int(lib.rsed_fock_scratch_bytes(cat.n_states)), dtype=torch.uint8, device=dev)
    norm2 = ctypes.c_double(0.0)
    _lib.check(lib.rsed_fock_expand(ctypes.byref(cat.dgroup.c), _lib.ptr(cat.table), n_orb,
                                    _lib.ptr(cat.repr_masks), _lib.ptr(cat.stab_mask), _lib.ptr(xo), _lib.ptr(chi),
                                    float(atol), _lib.ptr(amp), _lib.ptr(masks),
                                    ctypes.byref(norm2), _lib.ptr(scratch), scratch.numel(),
                                    _lib.stream_ptr(stream)))
    return amp


def expand_sector_state_to_fock_amplitudes(c, basis: Symmetry_Sector_Basis, particle_statistics=None, *,
                                           atol: float = 1e-12, as_dict: bool = True, stream=None):
    cat = basis.catalog
    dev = cat.table.device
    amp = torch.empty(cat.n_states, dtype=torch.complex128, device=dev)
    masks = torch.empty(cat.n_states, dtype=torch.int64, device=dev)
    _expand(c, basis, atol, amp, masks, stream)
    nz = torch.nonzero(amp != 0).reshape(-1)
    m_nz, a_nz = masks[nz], amp[nz]
    if not as_dict:
        return m_nz, a_nz
    keys = (m_nz.cpu().numpy().view(np.uint64)).tolist()
    vals = a_nz.cpu().numpy().tolist()
    return dict(zip(keys, vals))


def expand_sector_state_to_fock_dense(c, basis: Symmetry_Sector_Basis, *, out: torch.Tensor | None = None,
                                      atol: float = 1e-12, stream=None) -> torch.Tensor:
    """The unit-norm Fock amplitudes of sector vector ``c`` as a dense device
    vector (complex128, ``catalog.n_states`` entries, entry ``r`` = the state
    of table rank ``r``), amplitudes at or below ``atol`` zero; written into
    ``out`` when given.  ``ValueError`` for a near-zero norm."""
    cat = basis.catalog
    if out is None:
        out = torch.empty(cat.n_states, dtype=torch.complex128, device=cat.table.device)
    return _expand(c, basis, atol, out, None, stream)


def fock_overlaps(states: torch.Tensor, pairs, *, stream=None) -> np.ndarray:
    """Overlap matrices ``M[p][i][j] = <states[a_p][i] | states[b_p][j]>`` of
    dense Fock-amplitude vectors ``states`` (device complex128
    ``[n_slots, n_m, n_states]``) for the slot pairs ``pairs`` (``[(a, b), ...]``),
    computed on the device and returned as a host array ``[n_pairs, n_m, n_m]``."""
    lib = _lib.lib()
    if states.dim() != 3 or states.dtype != torch.complex128 or not states.is_contiguous() or not states.is_cuda:
        raise ValueError("states must be a contiguous complex128 CUDA tensor [n_slots, n_m, n_states]")
    n_slots, n_m, n_states = (int(x) for x in states.shape)
    pr = np.ascontiguousarray(np.asarray(pairs, dtype=np.int32).reshape(-1, 2))
    n_pairs = pr.shape[0]
    out = torch.empty((n_pairs, n_m, n_m), dtype=torch.complex128, device=states.device)
    if n_pairs == 0:
        return out.cpu().numpy()
    scratch = torch.empty(int(lib.rsed_fock_overlap_scratch_bytes(n_states, n_m, n_pairs)), dtype=torch.uint8,
                          device=states.device)
    _lib.check(lib.rsed_fock_overlaps(_lib.ptr(states), n_states, n_m, n_slots,
                                      pr.ctypes.data_as(ctypes.c_void_p), n_pairs, _lib.ptr(out), _lib.ptr(scratch),
                                      scratch.numel(), _lib.stream_ptr(stream)))
    if stream is not None:
        stream.synchronize()
    return out.cpu().numpy()


# the reference's (private) name
_expand_sector_state_to_fock_amplitudes = expand_sector_state_to_fock_amplitudes
