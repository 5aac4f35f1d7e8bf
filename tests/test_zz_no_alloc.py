"""The allocation-free sector-rows entry point against the regular one.

``rsed_sector_rows_noalloc`` exists for callers that cannot allocate device
memory (a service that hands all of HBM to its own pool up front, or a hot
loop that must avoid the device-wide synchronisation of cudaFree): its scan
scratch is a fixed device array inside the library.  This file is collected
last so that a failure here cannot hide failures elsewhere, and it must pass
both alone in a fresh process and after the rest of the suite.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _member_bits(n, seed):
    rng = np.random.default_rng(seed)
    return torch.from_numpy(rng.integers(0, 2**62, size=n, dtype=np.int64)).cuda()


def _rows(lib, fn_name, n, member, sector, with_scratch):
    from realspace_exatdiagonalization_py_b200 import _lib

    oor = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    roo = torch.full((n,), -7, dtype=torch.int32, device="cuda")
    sp = torch.cuda.current_stream().cuda_stream
    if with_scratch:
        nbytes = lib.rsed_sector_scratch_bytes(n, 1)
        scratch = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device="cuda")
        rc = lib.rsed_sector_rows(n, member.data_ptr(), sector, oor.data_ptr(), roo.data_ptr(),
                                  scratch.data_ptr(), scratch.numel(), sp)
    else:
        rc = getattr(lib, fn_name)(n, member.data_ptr(), sector, oor.data_ptr(), roo.data_ptr(), sp)
    _lib.check(rc)
    torch.cuda.synchronize()
    d = int(((member >> sector) & 1).sum().item())
    return oor[:d].cpu().numpy(), roo.cpu().numpy()


@pytest.mark.parametrize("n", [1, 1000, 8192, 8193, 300_000])
def test_noalloc_matches_allocating_entry_point(n):
    from realspace_exatdiagonalization_py_b200 import _lib

    lib = _lib.lib()
    member = _member_bits(n, n)
    for sector in (0, 17, 61):
        ref = _rows(lib, "rsed_sector_rows", n, member, sector, True)
        # two calls in a row: the shared device array keeps the first call's
        # contents, which must not leak into the second result
        for _ in range(2):
            got = _rows(lib, "rsed_sector_rows_noalloc", n, member, sector, False)
            np.testing.assert_array_equal(got[0], ref[0])
            np.testing.assert_array_equal(got[1], ref[1])


def test_noalloc_on_a_catalog():
    """Sector bases of a real catalog, both entry points."""
    import realspace_exatdiagonalization_py_b200 as ed
    from fractions import Fraction
    from realspace_exatdiagonalization_py_b200 import _lib, models

    lib = _lib.lib()
    m, nf = models.config_model("checkerboard24")
    G = ed.build_translation_group(m.lattice)
    data = ed.build_ed_data(m, filling_fraction=Fraction(nf, m.lattice.n_site), symmetry_group=G)
    _, sset = data._device()
    n = data.orbit_catalog.n_orbits
    for s in range(sset.n_sectors):
        ref_oor, ref_roo = sset.rows(s)
        for _ in range(2):
            oor, roo = _rows(lib, "rsed_sector_rows_noalloc", n, sset.member, s, False)
            np.testing.assert_array_equal(oor, ref_oor.cpu().numpy())
            np.testing.assert_array_equal(roo, ref_roo.cpu().numpy())


def test_noalloc_rejects_oversize_input():
    from realspace_exatdiagonalization_py_b200 import _lib

    lib = _lib.lib()
    limit = lib.rsed_sector_rows_noalloc_max_orbits()
    assert limit == 2**27
    member = torch.zeros(1, dtype=torch.int64, device="cuda")
    out = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.rsed_sector_rows_noalloc(limit + 1, member.data_ptr(), 0, out.data_ptr(), None,
                                      torch.cuda.current_stream().cuda_stream)
    assert rc == _lib.RSED_ERANGE
    assert b"at most" in lib.rsed_last_error()
