"""Orbit-space projection table (K6b) and its streaming apply, against the
oracle's sector blocks and against the on-the-fly apply.

Tolerances: FP64 matvec 1e-12 relative to ||H|| ||x|| (oracle) and 1e-13
absolute against the on-the-fly kernel (same hop order, same weights);
FP32 2e-6 relative; eigenvalues 1e-10 absolute.
"""

import numpy as np
import pytest
import torch

from _cases import ed_data_for, oracle_block

pytestmark = pytest.mark.gpu

CASES = ["heisenberg16", "checkerboard24", "haldane12", "hubbard12", "haldane12_flux",
         "checkerboard12_flux", "haldane24_flux"]


def _block(data, rng, ns):
    dm, sset = data._device()
    n_orb = data.orbit_catalog.n_orbits
    ld = ns + (ns & 1)
    X = torch.zeros((n_orb, ld), dtype=torch.complex128, device="cuda")
    for s in range(ns):
        oor, _ = sset.rows(s)
        d = sset.dims[s]
        x = rng.standard_normal(d) + 1j * rng.standard_normal(d)
        X[oor.long(), s] = torch.from_numpy(x).cuda()
    return dm, sset, X, torch.arange(ns, dtype=torch.int32, device="cuda")


@pytest.mark.parametrize("case", CASES)
def test_projection_apply_matches_oracle(golden, case):
    g = golden(case)
    data = ed_data_for(case, g)
    ns = len(g["chi"])
    dm, sset, X, cs = _block(data, np.random.default_rng(21), ns)
    dm.build_projection(sset.sqrt_stab)
    try:
        Y = torch.empty_like(X)
        dm.apply_block(sset, cs, X, Y)  # variant 0 streams the table
        for s in sorted({0, ns // 2, ns - 1}):
            H, _ = oracle_block(g, s)
            if H.shape[0] == 0:
                continue
            oor, _ = sset.rows(s)
            x = X[oor.long(), s].cpu().numpy()
            y = Y[oor.long(), s].cpu().numpy()
            scale = abs(H).max() * np.abs(x).sum()
            np.testing.assert_allclose(y, H.conj().T @ x, atol=1e-12 * scale, rtol=0)
        # rows outside a column's sector are written as zero
        for s in range(ns):
            mask = torch.ones(X.shape[0], dtype=torch.bool, device="cuda")
            oor, _ = sset.rows(s)
            mask[oor.long()] = False
            assert torch.count_nonzero(Y[mask, s]) == 0
    finally:
        dm.drop_projection()


@pytest.mark.parametrize("case", ["checkerboard24", "haldane24_flux", "hubbard12"])
def test_projection_variants_match_on_the_fly(golden, case):
    g = golden(case)
    data = ed_data_for(case, g)
    ns = len(g["chi"])
    dm, sset, X, cs = _block(data, np.random.default_rng(22), ns)
    Yref = torch.empty_like(X)
    dm.apply_block(sset, cs, X, Yref, variant=0)
    Xf = X.to(torch.complex64)
    Yref32 = torch.empty_like(X)
    dm.apply_block(sset, cs, Xf, Yref32, precision=32, variant=0)
    dm.build_projection(sset.sqrt_stab)
    try:
        for v in (302, 304, 308, 316, 332, 402, 404, 408, 416, 432, 504, 508, 516, 532, 564, 604, 608, 616,
                  632, 664):
            Y = torch.full_like(X, complex("nan"))
            dm.apply_block(sset, cs, X, Y, variant=v)
            assert (Y[:, :ns] - Yref[:, :ns]).abs().max().item() < 1e-13, v
        nrm = Yref32[:, :ns].abs().max().item()
        for v in (304, 308, 316, 332, 364, 404, 408, 416, 432, 464, 508, 516, 532, 564, 528, 608, 616, 632,
                  664, 628):
            Y = torch.full_like(X, complex("nan"))
            dm.apply_block(sset, cs, Xf, Y, precision=32, variant=v)
            assert (Y[:, :ns] - Yref32[:, :ns]).abs().max().item() < 2e-6 * nrm, v
    finally:
        dm.drop_projection()


def test_projection_rejects_bad_variant(golden):
    from realspace_exatdiagonalization_py_b200 import _lib

    g = golden("checkerboard24")
    data = ed_data_for("checkerboard24", g)
    dm, sset, X, cs = _block(data, np.random.default_rng(1), 2)
    Y = torch.empty_like(X)
    with pytest.raises(ValueError):
        dm.apply_block(sset, cs, X, Y, variant=304)  # no table built
    dm.build_projection(sset.sqrt_stab, precisions=(64,))
    try:
        with pytest.raises(ValueError):
            dm.apply_block(sset, cs, X.to(torch.complex64), Y, precision=32, variant=308)  # no FP32 weights
        for bad in (303, 502, 700):
            with pytest.raises(ValueError):
                dm.apply_block(sset, cs, X, Y, variant=bad)
    finally:
        dm.drop_projection()
    assert _lib.lib() is not None


def test_projection_dropped_after_phase_update(golden):
    """An in-place amplitude update invalidates a table built before it."""
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden("checkerboard24")
    data = ed_data_for("checkerboard24", g)
    cat = data.orbit_catalog.clone()
    model = data.second_quantized_model
    dm = ed.DeviceModel(cat, model.bilinear_terms, model.density_density_terms)
    sset = ed.SectorSet(cat, data.irrep_list)
    dm.build_projection(sset.sqrt_stab)
    assert dm.proj is not None
    G2 = ed.build_translation_group(model.lattice, [0.25, 0.0])
    ed.update_orbit_stabilizer_phases(cat, G2, model.particle_statistics)
    dm.refresh()
    assert dm.proj is None and dm.c.proj_rowptr is None


@pytest.mark.parametrize("case", ["checkerboard24", "haldane24_flux", "heisenberg16"])
@pytest.mark.parametrize("precision", [64, 32])
def test_projection_solve_energies(golden, case, precision):
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200.batched import BatchedSectorSolver

    g = golden(case)
    data = ed_data_for(case, g)
    dm, sset = data._device()
    sectors = [int(s) for s in g["eig_sectors"] if g["sector_dims"][int(s)] > 0]
    nev = int(g["nev"])
    dm.build_projection(sset.sqrt_stab)
    try:
        sol = BatchedSectorSolver(dm, sset, sectors, nev, precision=precision,
                                  params=ed.LanczosParams(precision=precision), persistent=0)
        vals, _ = sol.solve(None, vectors=False)
        for i, s in enumerate(sectors):
            ref = g["eig_vals"][list(g["eig_sectors"]).index(s)]
            k = min(nev, len(ref), sset.dims[s])
            np.testing.assert_allclose(vals[i][:k], ref[:k], atol=1e-10, rtol=0)
    finally:
        dm.drop_projection()
