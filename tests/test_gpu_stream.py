"""The streamed Gram-Schmidt kernels (whole-row panels moved by bulk copies:
k_lz_gram_stream, k_lz_finalize, k_lz_update_stream) against the
per-instance kernels (``LanczosParams(stream=False)``) and the reference's
golden energies.

Covered: one and two columns per lane (ld <= 32 and 33..64), uniform and mixed
block sizes (the kernel's block bound rounded up to 2, 4 and 8), the adaptive
single pass and the always-two-pass form, FP64 and FP32 matvecs, and a batch
too wide for streaming (ld > 64), which keeps the per-instance kernels.
Tolerances: eigenvalues 1e-10 absolute against the reference; the two kernel
forms 1e-10 against each other (their sums run in different orders, so
Lanczos may take a step more or less).
"""

import numpy as np
import pytest

from _cases import ed_data_for

pytestmark = pytest.mark.gpu


def _solve(data, sectors, nev, block_sizes, *, stream, precision=64, single=True, n_slots=16, stream_update=True):
    import realspace_exatdiagonalization_py_b200 as ed

    dm, sset = data._device()
    if dm.proj is None:
        from realspace_exatdiagonalization_py_b200.batched import projection_precisions

        dm.build_projection(sset.sqrt_stab, precisions=projection_precisions(dm, 32))
    p = ed.LanczosParams(block=max(block_sizes), n_slots=n_slots, precision=precision, single_pass=single,
                         stream=stream, stream_update=stream_update)
    sol = ed.BatchedSectorSolver(dm, sset, sectors, nev, precision=precision, params=p,
                                 config=ed.SolverConfig(tuple(block_sizes), 0, True, n_slots))
    vals, _ = sol.solve(None, vectors=False)
    return vals, sol.batch.status()


CASES = [
    # (case, block size per sector (cycled), precision, single pass)
    ("heisenberg16", [2], 64, True),          # ld 32, one column per lane
    ("heisenberg16", [3], 64, True),          # ld 48, two columns per lane, block bound 4
    ("heisenberg16", [1, 2, 3, 4], 64, True),  # mixed blocks
    ("heisenberg16", [2], 64, False),         # two passes
    ("checkerboard24", [4], 32, True),        # ld 48, FP32 matvec + FP64 refinement
    ("haldane24_flux", [2], 32, True),        # flux block, FP32
    ("haldane24_flux", [4], 64, False),       # flux block, two passes
    ("heisenberg16", [8], 64, True),          # block bound 8, 8 sectors: ld 64
]


@pytest.mark.parametrize("case,bs,precision,single", CASES)
def test_streamed_gram_schmidt_matches_reference_and_per_instance_kernels(golden, case, bs, precision, single):
    g = golden(case)
    data = ed_data_for(case, g)
    nev = int(g["nev"])
    sectors = [int(s) for s in g["eig_sectors"]]
    ref = {s: v for s, v in zip(sectors, g["eig_vals"])}
    dims = data._device()[1].dims
    sectors = [s for s in sectors if dims[s] > 500]
    if bs == [8]:
        sectors = sectors[:8]
    block_sizes = [bs[i % len(bs)] for i in range(len(sectors))]
    n_slots = 8 if max(block_sizes) == 8 else 16
    v_str, st_str = _solve(data, sectors, nev, block_sizes, stream=True, precision=precision, single=single,
                           n_slots=n_slots)
    v_per, st_per = _solve(data, sectors, nev, block_sizes, stream=False, precision=precision, single=single,
                           n_slots=n_slots)
    for i, s in enumerate(sectors):
        k = min(nev, len(ref[s]))
        np.testing.assert_allclose(v_str[i, :k], ref[s][:k], atol=1e-10, rtol=0)
        np.testing.assert_allclose(v_per[i, :k], ref[s][:k], atol=1e-10, rtol=0)
    np.testing.assert_allclose(v_str, v_per, atol=1e-10, rtol=0)
    # status 1 = converged; iteration counts within a restart of each other
    assert (st_str[:, 1] == 1).all() and (st_per[:, 1] == 1).all()
    assert np.abs(st_str[:, 3] - st_per[:, 3]).max() <= 16
    if not single:
        assert st_str[:, 11].sum() == 0


@pytest.mark.parametrize("single", [True, False])
def test_streamed_reduction_with_row_group_update(golden, single):
    """The streamed reduction followed by the row-group update
    (``stream_update=False``) gives the same eigenvalues."""
    g = golden("heisenberg16")
    data = ed_data_for("heisenberg16", g)
    nev = int(g["nev"])
    sectors = [int(s) for s in g["eig_sectors"]]
    v1, st1 = _solve(data, sectors, nev, [2] * len(sectors), stream=True, single=single, stream_update=False)
    v2, _ = _solve(data, sectors, nev, [2] * len(sectors), stream=False, single=single)
    np.testing.assert_allclose(v1, v2, atol=1e-10, rtol=0)
    for i, ref in enumerate(g["eig_vals"]):
        k = min(nev, len(ref))
        np.testing.assert_allclose(v1[i, :k], ref[:k], atol=1e-10, rtol=0)
    assert (st1[:, 1] == 1).all()


def test_batch_wider_than_the_stream_limit(golden):
    """16 sectors x 5 columns (ld 80): the per-instance kernels run, with or
    without the stream flag, and give the reference's energies."""
    g = golden("heisenberg16")
    data = ed_data_for("heisenberg16", g)
    nev = int(g["nev"])
    sectors = [int(s) for s in g["eig_sectors"]]
    v1, _ = _solve(data, sectors, nev, [5] * len(sectors), stream=True, n_slots=12)
    v2, _ = _solve(data, sectors, nev, [5] * len(sectors), stream=False, n_slots=12)
    np.testing.assert_array_equal(v1, v2)
    for i, ref in enumerate(g["eig_vals"]):
        k = min(nev, len(ref))
        np.testing.assert_allclose(v1[i, :k], ref[:k], atol=1e-10, rtol=0)
