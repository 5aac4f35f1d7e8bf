"""Many-body Chern number (observables/many_body_chern_number.py:341-458) on
the device against the reference's own driver (tests/golden/make_chern_golden.py),
and the device overlap kernel behind its links against numpy."""

import os
import warnings
from fractions import Fraction

import numpy as np
import pytest
import torch

from _cases import CHERN_CASES, chern_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_m,n_states,n_slots", [(1, 1, 2), (1, 70001, 3), (3, 4099, 4), (5, 20000, 3),
                                                  (9, 3001, 2)])
def test_fock_overlaps_match_numpy(n_m, n_states, n_slots):
    import realspace_exatdiagonalization_py_b200 as ed

    g = torch.Generator().manual_seed(n_m * 7 + n_slots)
    s = torch.complex(torch.randn(n_slots, n_m, n_states, generator=g, dtype=torch.float64),
                      torch.randn(n_slots, n_m, n_states, generator=g, dtype=torch.float64))
    pairs = [(a, b) for a in range(n_slots) for b in range(n_slots)]
    M = ed.fock_overlaps(s.cuda().contiguous(), pairs)
    host = s.numpy()
    for p, (a, b) in enumerate(pairs):
        ref = host[a].conj() @ host[b].T
        np.testing.assert_allclose(M[p], ref, rtol=0, atol=1e-11 * max(1.0, np.abs(ref).max()))
    again = ed.fock_overlaps(s.cuda().contiguous(), pairs)
    assert np.array_equal(M.view(np.float64), again.view(np.float64))  # fixed summation order


def test_fock_overlaps_reject_bad_pairs():
    import realspace_exatdiagonalization_py_b200 as ed

    s = torch.zeros((2, 1, 16), dtype=torch.complex128, device="cuda")
    with pytest.raises(Exception):
        ed.fock_overlaps(s, [(0, 2)])
    with pytest.raises(Exception):
        ed.fock_overlaps(s, [(-1, 0)])


def _run(case, tmp, mode="matrix", overwrite=False):
    import realspace_exatdiagonalization_py_b200 as ed

    model, n_part, labels, nev, grid, f = chern_case(case)
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        res = ed.many_body_chern_number(model, labels, filling_fraction=Fraction(n_part, model.lattice.n_site),
                                        flux_grid_size=grid, nev_per_sector=nev, mode=mode,
                                        checkpoint_dir=str(tmp), overwrite=overwrite)
    n_warn = sum("Near-singular Berry link" in str(w.message) for w in caught)
    return res, n_warn, f


def _check(res, n_warn, f):
    nx, ny = res.flux_grid_size
    assert (nx, ny) == tuple(int(x) for x in f["grid"])
    E = np.array([[res.energies[ix][iy] for iy in range(ny)] for ix in range(nx)])
    np.testing.assert_allclose(E, f["energies"], atol=1e-9, rtol=0)
    np.testing.assert_allclose(res.berry_curvature, f["berry_curvature"], atol=1e-8, rtol=0)
    assert abs(res.chern_number - float(f["chern_number"])) < 1e-8
    assert res.rounded_chern == int(f["rounded_chern"])
    for k in ("link_det_abs_x", "link_det_abs_y"):
        got, want = getattr(res, k), f[k]
        big = want > 1e-8
        np.testing.assert_allclose(got[big], want[big], atol=1e-8, rtol=0)
        assert np.all(got[~big] <= 1e-10)
    if float(f["min_link_det"]) > 1e-8:
        assert abs(res.min_link_det - float(f["min_link_det"])) < 1e-8
    assert n_warn == int(f["n_singular_warnings"])
    np.testing.assert_array_equal(res.flux_x, np.arange(nx) / nx)
    np.testing.assert_array_equal(res.flux_y, np.arange(ny) / ny)


@pytest.mark.parametrize("case", CHERN_CASES)
def test_chern_matches_reference(tmp_path, case):
    res, n_warn, f = _run(case, tmp_path)
    _check(res, n_warn, f)
    assert os.path.basename(res.checkpoint_paths[0][0]) == str(f["checkpoint_00"])
    assert os.path.basename(res.checkpoint_paths[1][1]) == str(f["checkpoint_11"])


def test_chern_checkpoints_reused_and_matrixfree(tmp_path):
    res, n_warn, f = _run("haldane16", tmp_path, mode="matrixfree")
    _check(res, n_warn, f)
    paths = [p for row in res.checkpoint_paths for p in row]
    assert all(os.path.isfile(p) for p in paths)
    stamp = [os.path.getmtime(p) for p in paths]
    again, n2, _ = _run("haldane16", tmp_path, mode="matrixfree")
    assert [os.path.getmtime(p) for p in paths] == stamp  # loaded, not recomputed
    np.testing.assert_array_equal(again.berry_curvature, res.berry_curvature)
    fresh, n3, _ = _run("haldane16", tmp_path, mode="matrixfree", overwrite=True)
    _check(fresh, n3, f)


@pytest.mark.parametrize("case", ["haldane12", "haldane16", "checkerboard12"])
def test_chern_served_engine_matches_reference(tmp_path, case):
    import realspace_exatdiagonalization_py_b200 as ed

    model, n_part, labels, nev, grid, f = chern_case(case)
    kw = dict(filling_fraction=Fraction(n_part, model.lattice.n_site), flux_grid_size=grid, nev_per_sector=nev,
              engine="served", checkpoint_dir=str(tmp_path))
    with warnings.catch_warnings(record=True) as caught:
        warnings.simplefilter("always")
        res = ed.many_body_chern_number(model, labels, **kw)
    _check(res, sum("Near-singular Berry link" in str(w.message) for w in caught), f)
    # the served engine leaves the scan engine's per-point checkpoints behind
    assert os.path.basename(res.checkpoint_paths[0][0]) == str(f["checkpoint_00"])
    paths = [p for row in res.checkpoint_paths for p in row]
    assert all(os.path.isfile(p) for p in paths)
    stamp = [os.path.getmtime(p) for p in paths]
    with warnings.catch_warnings():
        warnings.simplefilter("ignore")
        scan = ed.many_body_chern_number(model, labels, filling_fraction=kw["filling_fraction"], flux_grid_size=grid,
                                         nev_per_sector=nev, checkpoint_dir=str(tmp_path))
        again = ed.many_body_chern_number(model, labels, **kw)
    assert [os.path.getmtime(p) for p in paths] == stamp  # both read them back, neither recomputed
    np.testing.assert_allclose(scan.berry_curvature, res.berry_curvature, atol=1e-12, rtol=0)
    np.testing.assert_allclose(again.berry_curvature, res.berry_curvature, atol=1e-12, rtol=0)


def test_chern_served_lanes_match_scan():
    """Sectors above the dense limit (24-site Haldane bosons, ~11k orbits per
    sector): eigenvectors out of the server's Lanczos lanes give the scan
    engine's links and curvature."""
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models

    model, nf = models.config_model("haldane24")
    ff = Fraction(nf, model.lattice.n_site)
    labels = [(0, 0), (0, 1)]
    kw = dict(filling_fraction=ff, flux_grid_size=(2, 3), nev_per_sector=1)
    import tempfile

    with tempfile.TemporaryDirectory() as d:
        served = ed.many_body_chern_number(model, labels, engine="served", checkpoint_dir=d, **kw)
    with tempfile.TemporaryDirectory() as d:
        scan = ed.many_body_chern_number(model, labels, mode="matrixfree", checkpoint_dir=d, **kw)
    np.testing.assert_allclose(np.array(served.energies), np.array(scan.energies), atol=1e-9, rtol=0)
    np.testing.assert_allclose(served.berry_curvature, scan.berry_curvature, atol=1e-8, rtol=0)
    np.testing.assert_allclose(served.link_det_abs_x, scan.link_det_abs_x, atol=1e-8, rtol=0)
    np.testing.assert_allclose(served.link_det_abs_y, scan.link_det_abs_y, atol=1e-8, rtol=0)
    assert abs(served.chern_number - scan.chern_number) < 1e-8


def test_served_request_vectors_are_eigenvectors():
    """A request with ``vectors=True`` gets unit eigenvectors in its sector's
    basis order at its flux point: H v = E v through the device operator."""
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models

    model, nf = models.config_model("haldane24")
    sm = ed.ServingModel(model, nf, name="h24")
    srv = ed.SolveServer(sm, nev=2, precision=64, block=2)
    reqs = [ed.SolveRequest(i, s, (0.25, 0.5), "h24", vectors=True) for i, s in enumerate((0, 3))]
    reqs.append(ed.SolveRequest(2, 1, (0.25, 0.5), "h24"))
    res = {r.rid: r for r in srv.run(reqs, realtime=False)}
    assert res[2].eigenvectors is None
    ctx = ed.FluxContext(sm, (0.25, 0.5), 64)
    for rid, s in ((0, 0), (1, 3)):
        v = res[rid].eigenvectors
        assert v.shape == (res[rid].dim, 2) and v.is_cuda
        basis = ed.Symmetry_Sector_Basis(ctx.irreps[s], ctx.catalog, ctx.sset, s)
        H = ed.MatrixFreeHamiltonian(basis, ctx.dm.bilinear_terms, ctx.dm.density_terms, None, model=ctx.dm)
        Hv = H.matvec_device(v.contiguous(), 2)
        # the operator applies H
        for j in range(2):
            r = torch.linalg.vector_norm(Hv[:, j] - res[rid].eigenvalues[j] * v[:, j]).item()
            assert r < 1e-8, r
            assert abs(torch.linalg.vector_norm(v[:, j]).item() - 1.0) < 1e-12
