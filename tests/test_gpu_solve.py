"""GPU matvec (K6), matrix mode (K7) and eigen-solves (K8) against the oracle
and the reference's golden energies.

Tolerances: matvec FP64 1e-12 relative to ||H|| ||x||; eigenvalues 1e-10
absolute (the target of the path); FP32 matvec 2e-6 relative.
"""

import numpy as np
import pytest
import torch

from _cases import ed_data_for, oracle_block

pytestmark = pytest.mark.gpu

ZERO_FLUX = ["heisenberg16", "checkerboard24", "haldane12", "hubbard12"]
FLUX = ["haldane12_flux", "checkerboard12_flux", "haldane24_flux"]
ALL = ZERO_FLUX + FLUX


def _op(data, s, precision=64):
    import realspace_exatdiagonalization_py_b200 as ed

    dm, sset = data._device()
    basis = ed.Symmetry_Sector_Basis(data.irrep_list[s], data.orbit_catalog, sset, s)
    return ed.MatrixFreeHamiltonian(basis, data.second_quantized_model.bilinear_terms,
                                    data.second_quantized_model.density_density_terms, None,
                                    precision=precision, model=dm)


@pytest.mark.parametrize("case", ALL)
def test_matvec_matches_reference_block(golden, case):
    g = golden(case)
    data = ed_data_for(case, g)
    rng = np.random.default_rng(3)
    nsec = len(g["chi"])
    for s in sorted({0, nsec // 2, nsec - 1}):
        H, orbits = oracle_block(g, s)
        n = H.shape[0]
        if n == 0:
            continue
        x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
        op = _op(data, s)
        y = op(x)
        scale = abs(H).max() * np.abs(x).sum()
        # the operator is the reference's y = H x, flux blocks included
        np.testing.assert_allclose(y, H @ x, atol=1e-12 * scale, rtol=0)
        # the eigensolver's streaming pull-form apply computes H^dagger x
        ya = op.adjoint_device(torch.from_numpy(x).cuda()).cpu().numpy()[:, 0]
        np.testing.assert_allclose(ya, H.conj().T @ x, atol=1e-12 * scale, rtol=0)
        herm = abs(H - H.conj().T).max()
        if case in ZERO_FLUX:
            assert herm < 1e-13
        else:
            # the reference's flux blocks are Hermitian only to complex64 rounding
            assert herm < 1e-6


@pytest.mark.parametrize("case", ["checkerboard24", "haldane24_flux"])
def test_matvec_fp32(golden, case):
    g = golden(case)
    data = ed_data_for(case, g)
    H, _ = oracle_block(g, 0)
    n = H.shape[0]
    x = np.random.default_rng(5).standard_normal(n) + 0j
    y64 = _op(data, 0)(x)
    y32 = _op(data, 0, precision=32)(x)
    assert np.linalg.norm(y32 - y64) <= 2e-6 * np.linalg.norm(y64)


@pytest.mark.parametrize("case", ["checkerboard24", "haldane24_flux"])
def test_batched_apply_equals_single_sector(golden, case):
    """One launch over all sectors (columns) equals the per-sector operator."""
    g = golden(case)
    data = ed_data_for(case, g)
    dm, sset = data._device()
    n_orb = data.orbit_catalog.n_orbits
    ns = len(data.irrep_list)
    ld = ns + (ns & 1)
    rng = np.random.default_rng(11)
    X = torch.zeros((n_orb, ld), dtype=torch.complex128, device="cuda")
    xs = []
    for s in range(ns):
        oor, _ = sset.rows(s)
        x = rng.standard_normal(sset.dims[s]) + 1j * rng.standard_normal(sset.dims[s])
        xs.append(x)
        X[oor.long(), s] = torch.from_numpy(x).cuda()
    Y = torch.empty_like(X)
    cs = torch.arange(ns, dtype=torch.int32, device="cuda")
    dm.apply_block(sset, cs, X, Y)
    for s in range(ns):
        oor, _ = sset.rows(s)
        # the single-sector form of the same streaming apply (H^dagger x)
        ys = _op(data, s).adjoint_device(torch.from_numpy(xs[s]).cuda()).cpu().numpy()[:, 0]
        np.testing.assert_allclose(Y[oor.long(), s].cpu().numpy(), ys, atol=1e-13, rtol=0)


@pytest.mark.parametrize("case", ALL)
def test_batched_sector_energies(golden, case):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden(case)
    data = ed_data_for(case, g)
    sectors = [int(s) for s in g["eig_sectors"]]
    nev = int(g["nev"])
    res = ed.solve_sectors_batched(data, sectors, nev=nev)
    for s, ref in zip(sectors, g["eig_vals"]):
        vals, vecs = res[s]
        k = min(nev, len(vals))
        np.testing.assert_allclose(vals[:k], ref[:k], atol=1e-10, rtol=0)
        assert data.sector_dims[s] == g["sector_dims"][s]


@pytest.mark.parametrize("case", ["heisenberg16", "checkerboard24", "haldane24_flux"])
def test_fp32_matvec_with_fp64_refinement(golden, case):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden(case)
    data = ed_data_for(case, g)
    sectors = [int(s) for s in g["eig_sectors"]]
    nev = int(g["nev"])
    res = ed.solve_sectors_batched(data, sectors, nev=nev, precision=32)
    for s, ref in zip(sectors, g["eig_vals"]):
        vals, _ = res[s]
        k = min(nev, len(vals))
        np.testing.assert_allclose(vals[:k], ref[:k], atol=1e-10, rtol=0)


def test_eigenvectors_are_eigenvectors(golden):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden("checkerboard24")
    data = ed_data_for("checkerboard24", g)
    res = ed.solve_sectors_batched(data, [0, 5], nev=6)
    for s in (0, 5):
        H, _ = oracle_block(g, s)
        vals, vecs = res[s]
        for j in range(6):
            r = H @ vecs[:, j] - vals[j] * vecs[:, j]
            assert np.linalg.norm(r) < 1e-8
        np.testing.assert_allclose(vecs.conj().T @ vecs, np.eye(6), atol=1e-10)


def test_plain_single_sector_path(golden):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden("heisenberg16")
    data = ed_data_for("heisenberg16", g)
    p = ed.LanczosParams(block=1, n_slots=48, precision=64)
    vals, _ = ed.ed_scan_at_irrep_matrixfree(data.irrep_list[0].label, data, nev=4, params=p)
    np.testing.assert_allclose(vals, g["eig_vals"][0][:4], atol=1e-10, rtol=0)
    np.testing.assert_allclose(vals, [-7.14229636, -6.12231527, -5.74759572, -5.59129049], atol=1e-8)


@pytest.mark.parametrize("case", ["checkerboard24", "haldane12_flux"])
def test_matrix_mode_triplets(golden, case):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden(case)
    data = ed_data_for(case, g)
    dm, sset = data._device()
    for s in (0, len(g["chi"]) - 1):
        Href, _ = oracle_block(g, s)
        basis = ed.Symmetry_Sector_Basis(data.irrep_list[s], data.orbit_catalog, sset, s)
        H = ed.build_ed_Hamiltonian_symmetry_block(basis, data.second_quantized_model.bilinear_terms,
                                                   data.second_quantized_model.density_density_terms,
                                                   None, model=dm)
        assert abs(H - Href).max() < 1e-14


def test_reference_regression_haldane_2x3():
    """test/test_core.py:162-198 of the reference."""
    import realspace_exatdiagonalization_py_b200 as ed
    from fractions import Fraction
    from realspace_exatdiagonalization_py_b200 import models

    m = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[2, 3],
                                                                  params=models.params_DNSheng)
    G = ed.build_translation_group(m.lattice)
    data = ed.build_ed_data(m, filling_fraction=Fraction(3, 12), symmetry_group=G)
    ed.ed_scan_at_irrep_matrix((0, 0), data, nev=3)
    vm = data.ed_scan_res[0][0]
    assert abs(vm[0] - (-7.163805363423441)) < 1e-9
    data2 = ed.build_ed_data(m, filling_fraction=Fraction(3, 12), symmetry_group=G)
    ed.ed_scan_at_irrep_matrixfree((0, 0), data2, nev=3)
    np.testing.assert_allclose(vm, data2.ed_scan_res[0][0], atol=1e-8)


JULIA_REF_BOSON_34 = {
    (0, 0): [-14.301456146831018, -13.722130823772558, -13.646661890699379, -13.640042308564075,
             -13.550170758301450],
    (0, 2): [-14.299362590626847, -13.743011957063569, -13.717272063933615, -13.586585123115862,
             -13.554354573641792],
    (1, 0): [-13.766743604919926, -13.699026453227097, -13.584647328593840, -13.513897654278470,
             -13.431386726887309],
}
JULIA_REF_FERMION_34 = {
    (0, 0): [-6.536696664020559, -6.377168957543855, -6.339387043488890, -6.192010626043237,
             -5.495381320129844],
    (0, 2): [-6.832285968463585, -6.488761638231560, -5.835575203799947, -5.713457341901553,
             -5.572292581119391],
    (1, 0): [-6.533812748546839, -6.512852966567995, -6.266923917001573, -6.084898163737772,
             -5.557311700956236],
}


def _sector_vals(data, label):
    for i, ir in enumerate(data.irrep_list):
        if ir.label == label:
            return data.ed_scan_res[i][0]
    raise KeyError(label)


def test_reference_energy_alignment():
    """test/test_energy_alignment.py of the reference (atol 1e-9), through
    the full scan API in both modes."""
    import realspace_exatdiagonalization_py_b200 as ed
    from fractions import Fraction
    from realspace_exatdiagonalization_py_b200 import models

    m = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[3, 4],
                                                                  params=models.params_DNSheng)
    G = ed.build_translation_group(m.lattice)
    data = ed.build_ed_data(m, filling_fraction=Fraction(6, 24), symmetry_group=G)
    ed.ed_scan(data, nev=5, mode="matrixfree")
    for k, ref in JULIA_REF_BOSON_34.items():
        np.testing.assert_allclose(_sector_vals(data, k)[:5], ref, atol=1e-9)
    p = dict(models.my_optimal_param)
    p["t''"] = -0.2
    mf, data, nf, ff = models.build_phase_explore_fermionic_checkerboard_model(p, [3, 4], Fraction(1, 3))
    assert nf == 4 and ff == Fraction(1, 6) and data.n_filled == 4
    ed.ed_scan(data, nev=5, mode="matrix", scanned_sectors=list(JULIA_REF_FERMION_34))
    for k, ref in JULIA_REF_FERMION_34.items():
        np.testing.assert_allclose(_sector_vals(data, k)[:5], ref, atol=1e-9)


@pytest.mark.parametrize("cluster", [1, 2, 8])
def test_persistent_cluster_solve(golden, cluster):
    """The one-launch solve (one thread-block cluster per sector) agrees with
    the oracle for every cluster size, and is deterministic."""
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200.batched import BatchedSectorSolver

    g = golden("checkerboard24")
    data = ed_data_for("checkerboard24", g)
    dm, sset = data._device()
    sectors = [int(s) for s in g["eig_sectors"]]
    for prec in (64, 32):
        sol = BatchedSectorSolver(dm, sset, sectors, 6, precision=prec,
                                  params=ed.LanczosParams(precision=prec), persistent=cluster)
        v1, _ = sol.solve(None, vectors=False)
        v2, _ = sol.solve(None, vectors=False)
        np.testing.assert_array_equal(v1, v2)
        for i, s in enumerate(sectors):
            np.testing.assert_allclose(v1[i], g["eig_vals"][list(g["eig_sectors"]).index(s)][:6], atol=1e-10,
                                       rtol=0)
