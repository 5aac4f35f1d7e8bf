"""Candidate space of the autotuner (host logic, no GPU)."""

from realspace_exatdiagonalization_py_b200.autotune import PERSISTENT_MAX_ORBITS, candidate_configs
from realspace_exatdiagonalization_py_b200.batched import SolverConfig, lanczos_footprint_bytes, persistent_ok


def test_candidates_small_even_batch():
    cands = candidate_configs([890, 880, 892], nev=6, n_orbits=892)
    shapes = {c.block_sizes for c in cands}
    assert shapes == {(2, 2, 2), (4, 4, 4), (8, 8, 8)}
    # persistent clusters only for uniform blocks <= 4
    pers = [c for c in cands if c.persistent]
    assert pers and all(persistent_ok(c.block_sizes) and c.persistent in (2, 4, 8) for c in pers)
    assert all(max(c.block_sizes) <= 4 for c in pers)
    # every block size has a graph path with and without the projection table
    for b in (2, 4, 8):
        assert SolverConfig((b,) * 3, 0, True, 16 if b < 8 else 8) in cands
        assert SolverConfig((b,) * 3, 0, False, 16 if b < 8 else 8) in cands


def test_candidates_uneven_batch_gets_graded_blocks():
    dims = [1000, 4000, 1200, 3900]
    cands = candidate_configs(dims, nev=4, n_orbits=5000)
    assert (2, 4, 2, 4) in {c.block_sizes for c in cands}


def test_candidates_large_basis_has_no_persistent_path():
    cands = candidate_configs([600000] * 4, nev=4, n_orbits=PERSISTENT_MAX_ORBITS + 1)
    assert cands and all(c.persistent == 0 for c in cands)
    quick = candidate_configs([600000] * 4, nev=4, n_orbits=PERSISTENT_MAX_ORBITS + 1, quick=True)
    assert 0 < len(quick) < len(cands)
    assert all(c.projection for c in quick)
    # shorter and longer basis lengths for blocks of 2 (measured: 12 slots fastest on the 32-site workload)
    for n_slots in (10, 12, 16, 24):
        assert SolverConfig((2,) * 4, 0, True, n_slots) in quick


def test_candidates_without_projection_memory():
    cands = candidate_configs([900] * 2, nev=4, n_orbits=900, projection_ok=False)
    assert all(not c.projection for c in cands)


def test_nev_limits_block_choice():
    # the restart basis holds at most 16 vectors and must leave room for the
    # Rayleigh-Ritz step: blocks of 2 keep at most 7 of them (n_slots 16)
    cands = candidate_configs([5000] * 2, nev=16, n_orbits=5000)
    assert {max(c.block_sizes) for c in cands} == {4, 8}
    assert candidate_configs([5000] * 2, nev=20, n_orbits=5000) == []


def test_footprint_grows_with_columns():
    a = lanczos_footprint_bytes(10000, 8)
    b = lanczos_footprint_bytes(10000, 16)
    assert b > a > 10000 * 8 * 16 * 18


def test_plan_waves_splits_by_footprint():
    import pytest

    from realspace_exatdiagonalization_py_b200.batched import plan_waves

    n = 1_000_000
    one = lanczos_footprint_bytes(n, 4)
    waves = plan_waves(n, [4] * 10, budget=int(3.5 * one))
    assert [i for w in waves for i in w] == list(range(10))
    assert all(lanczos_footprint_bytes(n, 4 * len(w)) <= 3.5 * one for w in waves)
    assert len(waves) == 4
    assert plan_waves(n, [4] * 3, budget=10 * one) == [[0, 1, 2]]
    with pytest.raises(MemoryError):
        plan_waves(n, [8], budget=one)
