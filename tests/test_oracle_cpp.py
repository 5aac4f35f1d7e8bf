"""The C++ restatement (oracle/cpu_ref.cpp via oracle/cpu.py) against the numpy
oracle (oracle/port.py, itself pinned to the reference engine by
tests/test_oracle_golden.py): catalog tables bit for bit (complex64
amplitudes exact except components below 1e-15), sector membership, the
sector apply (y = H^dagger x of the reference's block) and eigenvalues, on
the golden cases and on 48 sites (beyond the reference's 42-site limit)."""

import math

import numpy as np
import pytest

from oracle import cpu, port

CASES = ["heisenberg16", "haldane12_flux", "checkerboard12_flux", "checkerboard24", "haldane24_flux"]


def _cat_pair(g):
    n, k, fer = int(g["n_site"]), int(g["n_filled"]), bool(g["fermionic"])
    perm0 = (g["perm"] - 1).astype(np.uint8)
    return n, k, fer, perm0, cpu.catalog(n, k, perm0, g["eta"], fer), port.catalog(n, k, perm0, g["eta"], fer)


def _amp_equal(a, b):
    a = a.view(np.float32).copy()
    b = b.view(np.float32).copy()
    a[np.abs(a) < 1e-15] = 0
    b[np.abs(b) < 1e-15] = 0
    np.testing.assert_array_equal(a, b)


@pytest.mark.parametrize("case", CASES)
def test_cpp_catalog_matches_oracle(golden, case):
    g = golden(case)
    n, k, fer, perm0, c, p = _cat_pair(g)
    np.testing.assert_array_equal(c["reprs"], p["reprs"])
    np.testing.assert_array_equal(c["rep_rank"], p["rep_rank"])
    np.testing.assert_array_equal(c["rep_sym"], p["rep_sym"])
    _amp_equal(c["rep_amp"], p["rep_amp"])
    sm = np.array([sum(1 << int(x) for x in gs) for gs in p["stab_g"]], dtype=np.uint64)
    np.testing.assert_array_equal(c["stab_mask"], sm)
    # and against the reference's own tables
    np.testing.assert_array_equal(c["rep_rank"], g["rep_rank"])
    np.testing.assert_array_equal(c["rep_sym"], g["rep_sym"])


@pytest.mark.parametrize("case", CASES)
def test_cpp_members_apply_and_eigs(golden, case):
    g = golden(case)
    n, k, fer, perm0, c, p = _cat_pair(g)
    chi = g["chi"]
    mem = cpu.members(c, chi)
    bil = [(int(i), int(j), t) for (i, j), t in zip(g["bil_ij"], g["bil_t"])]
    den = [(int(i), int(j), v) for (i, j), v in zip(g["den_ij"], g["den_v"])]
    for s in range(len(chi)):
        orbits = port.sector_orbits(p, chi[s])
        np.testing.assert_array_equal(np.nonzero((mem >> np.uint64(s)) & np.uint64(1))[0], orbits)
    rng = np.random.default_rng(9)
    for s in sorted({0, len(chi) // 2}):
        orbits = port.sector_orbits(p, chi[s])
        if len(orbits) == 0:
            continue
        H = port.csr_block(p, n, orbits, bil, den, chi[s], fer)
        op = cpu.SectorOperator(c, chi[s], bil, den)
        assert op.n == H.shape[0]
        x = rng.standard_normal(op.n) + 1j * rng.standard_normal(op.n)
        scale = abs(H).max() * np.abs(x).sum()
        np.testing.assert_allclose(op(x), H.conj().T @ x, rtol=0, atol=1e-12 * scale)
    if "eig_sectors" in g and case in ("checkerboard24", "haldane24_flux"):
        s = int(g["eig_sectors"][0])
        op = cpu.SectorOperator(c, chi[s], bil, den)
        vals, _ = cpu.solve(op, int(g["nev"]))
        np.testing.assert_allclose(vals, g["eig_vals"][0][: len(vals)], rtol=0, atol=1e-10)


def test_cpp_matches_oracle_beyond_42_sites():
    """48-site checkerboard with 3 fermions (17,296 states): the reference's
    rank returns 0 there; the C++ restatement and the numpy oracle rank
    exactly and agree table for table and eigenvalue for eigenvalue."""
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models

    model, _ = models.config_model("checkerboard48")
    G = ed.build_translation_group(model.lattice)
    irreps = ed.build_irrep_list(G, model.lattice)
    perm0, eta = port.group_arrays(G)
    n, k = 48, 3
    c = cpu.catalog(n, k, perm0, eta, True)
    p = port.catalog(n, k, perm0, eta, True)
    assert len(c["rep_rank"]) == math.comb(48, 3)
    np.testing.assert_array_equal(c["reprs"], p["reprs"])
    np.testing.assert_array_equal(c["rep_rank"], p["rep_rank"])
    np.testing.assert_array_equal(c["rep_sym"], p["rep_sym"])
    _amp_equal(c["rep_amp"], p["rep_amp"])
    # the rank is a bijection onto 0..C-1 (what the reference's fallback loses)
    idx = port.rank(port.unrank(np.arange(len(c["rep_rank"])), n, k, p["binom"]), n, p["binom"])
    np.testing.assert_array_equal(idx, np.arange(len(c["rep_rank"])))
    chi = np.asarray(irreps[5].values, dtype=np.complex128)
    orbits = port.sector_orbits(p, chi)
    H = port.csr_block(p, n, orbits, model.bilinear_terms, model.density_density_terms, chi, True)
    op = cpu.SectorOperator(c, chi, model.bilinear_terms, model.density_density_terms)
    x = np.random.default_rng(4).standard_normal(op.n) + 0.5j
    np.testing.assert_allclose(op(x), H.conj().T @ x, rtol=0, atol=1e-12 * abs(H).max() * np.abs(x).sum())
    w_port, _ = port.solve(H, 4)
    w_cpp, _ = cpu.solve(op, 4)
    np.testing.assert_allclose(w_cpp, w_port, rtol=0, atol=1e-10)
