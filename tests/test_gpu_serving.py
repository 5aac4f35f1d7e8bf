"""Continuous-batching server: every result is the same alone and in the mix
(|dE| <= 1e-10), and equals the reference energies where the goldens hold
them; requests of one flux point share a lane, lanes overlap."""

from fractions import Fraction

import numpy as np
import pytest

from _cases import model_for

pytestmark = pytest.mark.gpu


def _models(golden):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden("haldane24_flux")
    hal = ed.ServingModel(model_for("haldane24_flux"), int(g["n_filled"]), name="haldane24")
    gh = golden("heisenberg16")
    heis = ed.ServingModel(model_for("heisenberg16"), int(gh["n_filled"]), name="heisenberg16")
    return {"haldane24": hal, "heisenberg16": heis}, g, gh


def _requests(g):
    import realspace_exatdiagonalization_py_b200 as ed

    theta = tuple(float(x) for x in g["theta"])
    reqs = []
    rid = 0
    for s in (0, 6):                       # golden flux point, golden sectors
        reqs.append(ed.SolveRequest(rid, s, theta, "haldane24")); rid += 1
    for s in (1, 2, 3):                    # same flux point, other sectors
        reqs.append(ed.SolveRequest(rid, s, theta, "haldane24")); rid += 1
    for s, f in ((0, (0.25, 0.5)), (4, (0.25, 0.5)), (2, (0.0, 0.0)), (5, (0.75, 0.125))):
        reqs.append(ed.SolveRequest(rid, s, f, "haldane24")); rid += 1
    for s in (0, 5, 9):
        reqs.append(ed.SolveRequest(rid, s, (0.0, 0.0), "heisenberg16")); rid += 1
    return reqs


def test_results_same_alone_and_in_the_mix(golden):
    import realspace_exatdiagonalization_py_b200 as ed

    models, g, gh = _models(golden)
    reqs = _requests(g)
    nev = 4
    alone = {}
    server = ed.SolveServer(models, nev=nev, precision=32, max_width=1)
    for r in reqs:
        res = server.run([ed.SolveRequest(r.rid, r.sector, r.flux, r.model)], realtime=False)
        alone[r.rid] = res[0]
    mix_server = ed.SolveServer(models, nev=nev, precision=32, max_width=4)
    mixed = {r.rid: r for r in mix_server.run(
        [ed.SolveRequest(r.rid, r.sector, r.flux, r.model) for r in reqs], realtime=False)}
    assert set(mixed) == set(alone)
    for rid, a in alone.items():
        np.testing.assert_allclose(mixed[rid].eigenvalues, a.eigenvalues, atol=1e-10, rtol=0)
    # batching and overlap happened in the mix
    assert max(r.lane_width for r in mixed.values()) > 1
    assert mix_server.peak_running > 1
    # reference energies: haldane24 at the golden flux, heisenberg16 at zero flux
    for r in reqs:
        if r.model == "haldane24" and r.sector in (0, 6) and r.rid < 2:
            ref = g["eig_vals"][list(g["eig_sectors"]).index(r.sector)][:nev]
            np.testing.assert_allclose(mixed[r.rid].eigenvalues, ref, atol=1e-10, rtol=0)
        if r.model == "heisenberg16":
            np.testing.assert_allclose(mixed[r.rid].eigenvalues, gh["eig_vals"][r.sector][:nev], atol=1e-10,
                                       rtol=0)
        # FP32 phase stops at residual 1e-6 relative; the FP64 Rayleigh-Ritz
        # pairs keep residuals of that order (eigenvalue error is second order)
        assert mixed[r.rid].fp32_error is not None and mixed[r.rid].residuals.max() < 1e-5


def test_admission_respects_memory_budget(golden):
    """With room for one lane at a time, requests wait and still finish."""
    import realspace_exatdiagonalization_py_b200 as ed

    models, g, _ = _models(golden)
    sm = models["haldane24"]
    theta = tuple(float(x) for x in g["theta"])
    probe = ed.SolveServer({"haldane24": sm}, nev=4, precision=32, max_width=1)
    probe.run([ed.SolveRequest(99, 0, (0.5, 0.5), "haldane24")], realtime=False)  # measures a flux point
    ctx_bytes = probe._ctx_estimate(sm)
    assert ctx_bytes == sm.ctx_bytes > 0 and sm.base is not None
    lane_bytes = probe._lane_bytes(sm, 1)
    del probe
    # room for the shared zero-flux table, one flux point and its lane, not for a second flux point
    server = ed.SolveServer({"haldane24": sm}, nev=4, precision=32, max_width=1,
                            memory_budget=int(sm.base.bytes + ctx_bytes + 1.5 * lane_bytes))
    # four flux points: a second one never fits next to a running first one
    reqs = [ed.SolveRequest(i, s, f, "haldane24") for i, (s, f) in
            enumerate([(0, theta), (1, (0.5, 0.0)), (2, (0.25, 0.75)), (3, (0.0, 0.25))])]
    res = server.run(reqs, realtime=False)
    assert len(res) == 4
    assert server.peak_running == 1
    assert server.used_bytes() <= server.budget


def test_poisson_stream_latency_summary(golden):
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200.serving import poisson_requests

    models, g, _ = _models(golden)
    reqs = poisson_requests(12, rate=200.0, n_sectors=models["haldane24"].n_sectors, flux_grid=4,
                            model="haldane24", seed=0)
    server = ed.SolveServer(models, nev=4, precision=32)
    res = server.run(reqs, realtime=True)
    summ = ed.latency_summary(res)
    assert summ["requests"] == 12 and summ["p99_ms"] >= summ["p50_ms"] > 0
    assert all(r.finished >= r.admitted >= r.arrival - 1e-3 for r in res)


def test_checkpointed_server_writes_and_resumes(golden, tmp_path):
    """Served results land in the flux scan's per-flux-point checkpoint files
    (loadable by ``load_checkpoint``, eigenvectors included); a second server
    over the same directory answers those requests from disk, with the same
    eigenvalues and vectors; ``overwrite`` solves again."""
    import os

    import torch

    import realspace_exatdiagonalization_py_b200 as ed

    models, g, gh = _models(golden)
    sm = models["haldane24"]
    reqs = [ed.SolveRequest(0, 0, (0.25, 0.5), "haldane24", vectors=True),
            ed.SolveRequest(1, 4, (0.25, 0.5), "haldane24"),
            ed.SolveRequest(2, 2, (0.0, 0.0), "haldane24", vectors=True)]
    ck = ed.ServedCheckpoints(str(tmp_path))
    first = {r.rid: r for r in ed.SolveServer(sm, nev=3, precision=64, block=2, checkpoints=ck).run(
        [ed.SolveRequest(r.rid, r.sector, r.flux, r.model, vectors=r.vectors) for r in reqs], realtime=False)}
    ck.close()
    assert first[1].eigenvectors is None and first[0].eigenvectors is not None
    paths = sorted(ck.written)
    assert len(paths) == 2 and all(os.path.isfile(p) for p in paths)
    assert ck.path_of(sm, (0.25, 0.5)) == os.path.join(str(tmp_path), ed.ed_scan_checkpoint_filename(
        sm.model, [0.25, 0.5], Fraction(sm.n_filled, sm.lattice.n_site)))
    data = ed.load_checkpoint(ck.path_of(sm, (0.25, 0.5)))
    assert sorted(data.ed_scan_res) == [0, 4] and data.symmetry_group.name == "translations"
    vals, vecs = data.ed_scan_res[0]
    np.testing.assert_array_equal(vals, first[0].eigenvalues)
    np.testing.assert_array_equal(vecs, first[0].eigenvectors.cpu().numpy())
    assert data.sector_dims[0] == first[0].dim
    # resume: answered from disk
    ck2 = ed.ServedCheckpoints(str(tmp_path))
    stamp = [os.path.getmtime(p) for p in paths]
    second = {r.rid: r for r in ed.SolveServer(sm, nev=3, precision=64, block=2, checkpoints=ck2).run(
        [ed.SolveRequest(r.rid, r.sector, r.flux, r.model, vectors=r.vectors) for r in reqs], realtime=False)}
    ck2.close()
    assert all(r.lane == -1 and r.iterations == 0 for r in second.values())
    assert [os.path.getmtime(p) for p in paths] == stamp
    for rid in first:
        np.testing.assert_array_equal(second[rid].eigenvalues, first[rid].eigenvalues)
    assert torch.equal(second[2].eigenvectors, first[2].eigenvectors)
    # overwrite: solved again, files rewritten
    ck3 = ed.ServedCheckpoints(str(tmp_path), overwrite=True)
    third = ed.SolveServer(sm, nev=3, precision=64, block=2, checkpoints=ck3).run(
        [ed.SolveRequest(0, 0, (0.25, 0.5), "haldane24")], realtime=False)
    ck3.close()
    assert third[0].lane != -1
    np.testing.assert_allclose(third[0].eigenvalues, first[0].eigenvalues, atol=1e-10, rtol=0)
    assert sorted(ed.load_checkpoint(ck.path_of(sm, (0.25, 0.5))).ed_scan_res) == [0]
