"""The measured configuration choice: every candidate the tuner accepts
solves the batch to the oracle's energies, and the cache returns the choice."""

import numpy as np
import pytest

from _cases import ed_data_for

pytestmark = pytest.mark.gpu


def test_autotuner_candidates_agree_and_cache(golden, tmp_path):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden("checkerboard24")
    data = ed_data_for("checkerboard24", g)
    dm, sset = data._device()
    sectors = [0, 1, 2, 3]
    nev = 6
    tuner = ed.Autotuner(str(tmp_path / "tune.json"), trials=1)
    best, table = tuner.tune(dm, sset, sectors, nev, precision=32)
    assert best in ed.candidate_configs([sset.dims[s] for s in sectors], nev, dm.catalog.n_orbits)
    ok = [r for r in table if r["ok"]]
    assert len(ok) >= 6
    paths = {r["config"]["path"] for r in ok}
    assert "graph" in paths and any(p.startswith("persistent") for p in paths)
    # every accepted candidate reproduced the first one's energies
    assert max(r["max_abs_dE_vs_first"] for r in ok) <= 1e-8
    sol = ed.BatchedSectorSolver(dm, sset, sectors, nev, precision=32, config=best)
    vals, _ = sol.solve(None, vectors=False)
    for i, s in enumerate(sectors):
        np.testing.assert_allclose(vals[i], g["eig_vals"][s][:nev], atol=1e-10, rtol=0)
    cfg = tuner.best(dm, sset, sectors, nev, precision=32)
    tuner2 = ed.Autotuner(str(tmp_path / "tune.json"))
    assert tuner2.best(dm, sset, sectors, nev, precision=32) == cfg


def test_solve_sectors_batched_autotune(golden):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden("heisenberg16")
    data = ed_data_for("heisenberg16", g)
    sectors = [0, 5, 9]
    res = ed.solve_sectors_batched(data, sectors, nev=4, precision=32, autotune=True)
    for s in sectors:
        np.testing.assert_allclose(res[s][0], g["eig_vals"][s][:4], atol=1e-10, rtol=0)
