"""48 sites -- beyond the reference's 42-site limit, where its rank fallback
returns 0 for every mask (symmetry_resolved_ed.py:665, 896 -> 404-418) --
on the device against the C++ restatement (oracle/cpu_ref.cpp, pinned to the
numpy oracle and through it to the reference by tests/test_oracle_cpp.py):
the 4x6x2 checkerboard of the 48-site workload with 4 fermions (194,580
states, about 8,100 orbits per sector, so every sector takes the Lanczos
path): catalog tables bit for bit, sector dimensions, the streaming apply,
the reference-signature operator and batched eigenvalues (FP64 and FP32 +
refinement) of three sectors, 1e-10."""

import math
from fractions import Fraction

import numpy as np
import pytest
import torch

from oracle import cpu, port

pytestmark = pytest.mark.gpu

N, K = 48, 4


@pytest.fixture(scope="module")
def cb48():
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models

    model, _ = models.config_model("checkerboard48")
    G = ed.build_translation_group(model.lattice)
    data = ed.build_ed_data(model, filling_fraction=Fraction(K, N), symmetry_group=G)
    perm0, eta = port.group_arrays(G)
    ref = cpu.catalog(N, K, perm0, eta, True)
    return ed, model, data, ref


def test_catalog_beyond_42_sites(cb48):
    ed, model, data, ref = cb48
    cat = data.orbit_catalog
    assert cat.n_states == math.comb(N, K)
    np.testing.assert_array_equal(np.array(cat.representative_mask_list, dtype=np.uint64), ref["reprs"])
    np.testing.assert_array_equal(cat.rep_rank_table, ref["rep_rank"])
    np.testing.assert_array_equal(cat.rep_sym_table, ref["rep_sym"])
    a = cat.rep_amp_table.view(np.float32).copy()
    b = ref["rep_amp"].view(np.float32).copy()
    a[np.abs(a) < 1e-15] = 0
    b[np.abs(b) < 1e-15] = 0
    np.testing.assert_array_equal(a, b)
    _, sset = data._device()
    chi = np.array([ir.values for ir in data.irrep_list], dtype=np.complex128)
    mem = cpu.members(ref, chi)
    dims = [int(((mem >> np.uint64(s)) & np.uint64(1)).sum()) for s in range(len(chi))]
    assert sset.dims == dims and min(dims) > 500


def test_apply_and_eigenpairs_beyond_42_sites(cb48):
    """FP64 batched block Lanczos: every eigenpair verified with the C++
    operator (residual and orthonormality: this sector's pairs are exactly
    degenerate, which a block Lanczos resolves and the single-vector ARPACK
    of the oracle returns once), its distinct values equal to the oracle's
    ARPACK eigenvalues; the streaming apply and the reference-signature
    operator equal the C++ apply."""
    ed, model, data, ref = cb48
    secs = [0, 7, 13]
    res = ed.solve_sectors_batched(data, secs, nev=4, precision=64)
    dm, sset = data._device()
    for s in secs:
        chi = np.asarray(data.irrep_list[s].values, dtype=np.complex128)
        op = cpu.SectorOperator(ref, chi, model.bilinear_terms, model.density_density_terms)
        vals, vecs = res[s]
        for j in range(4):
            r = np.linalg.norm(op(vecs[:, j]) - vals[j] * vecs[:, j])
            assert r < 1e-8, (s, j, r)
        np.testing.assert_allclose(vecs.conj().T @ vecs, np.eye(4), atol=1e-10)
        arp, _ = cpu.solve(op, 6)
        distinct = [v for k, v in enumerate(vals) if k == 0 or v - vals[k - 1] > 1e-8]
        for v in distinct:
            assert np.min(np.abs(arp - v)) < 1e-10, (s, v, arp)
        assert abs(vals[0] - arp[0]) < 1e-10
        basis = ed.Symmetry_Sector_Basis(data.irrep_list[s], data.orbit_catalog, sset, s)
        H = ed.MatrixFreeHamiltonian(basis, model.bilinear_terms, model.density_density_terms, None, model=dm)
        rng = np.random.default_rng(s)
        x = rng.standard_normal(op.n) + 1j * rng.standard_normal(op.n)
        y = H.adjoint_device(torch.from_numpy(x).cuda()).cpu().numpy()[:, 0]
        np.testing.assert_allclose(y, op(x), rtol=0, atol=1e-12 * np.abs(x).sum())
        np.testing.assert_allclose(H(x), op(x), rtol=0, atol=1e-12 * np.abs(x).sum())


def test_fp32_matvec_with_refinement_beyond_42_sites(cb48):
    """FP32 matvec + FP64 refinement against the FP64 solve of the same
    sectors, 1e-10."""
    ed, model, data, ref = cb48
    secs = [0, 7, 13]
    r64 = ed.solve_sectors_batched(data, secs, nev=4, precision=64, return_vectors=False)
    r32 = ed.solve_sectors_batched(data, secs, nev=4, precision=32, return_vectors=False)
    for s in secs:
        np.testing.assert_allclose(r32[s][0], r64[s][0], atol=1e-10, rtol=0)


def test_single_and_two_pass_agree(cb48):
    """The adaptive single Gram-Schmidt pass gives the eigenvalues of the
    always-two-pass solve, and takes the single pass on most steps."""
    ed, model, data, ref = cb48
    dm, sset = data._device()
    out = {}
    for single in (True, False):
        p = ed.LanczosParams(block=2, precision=64, single_pass=single)
        sol = ed.BatchedSectorSolver(dm, sset, [2, 9], 4, precision=64, params=p,
                                     config=ed.SolverConfig((2, 2), 0, True, 16))
        vals, _ = sol.solve(None, vectors=False)
        st = sol.batch.status()
        out[single] = (vals, st)
    np.testing.assert_allclose(out[True][0], out[False][0], atol=1e-10, rtol=0)
    st1, st2 = out[True][1], out[False][1]
    assert st2[:, 11].sum() == 0
    assert st1[:, 11].sum() >= 0.5 * (st1[:, 3] - 1).sum()
    assert st1[:, 13].sum() < st2[:, 13].sum()
