"""The reference-signature single-sector API on the GPU, called exactly as the
reference's callers call it, against the reference's own outputs
(tests/golden/api_*.npz, written by tests/golden/make_api_golden.py from the
reference engine):

* ``hamiltonian_linear_operator`` -> ``H_op(x)`` and ``apply_hamiltonian``
  return the reference's ``y = H x`` (flux blocks included, whose ``H`` is
  Hermitian only to the complex64 rounding of the amplitude table);
* ``build_matrixfree_projection_table`` returns the reference's triplets and
  diagonal;
* ``CanonicalMap`` / ``get_canonical`` / ``project_to_sector`` /
  ``project_to_unnormalized_sector`` agree mask by mask;
* ``diagonalize_block_dense`` / ``_arpack`` / ``_matrixfree`` agree with the
  reference's eigenvalues, including a bare 11,240-row CSR block solved on
  the device (the reference's ARPACK ``eigs`` path);
* ``full_ed`` equals the lowest levels of the union of the sector spectra.

Tolerances: matvec 1e-12 relative to max|H_ij| * ||x||_1; amplitudes exact
except components below 1e-15; eigenvalues 1e-10 absolute.
"""

import numpy as np
import pytest
import scipy.sparse as sp
import torch

from _cases import ed_data_for

pytestmark = pytest.mark.gpu

CASES = ["heisenberg16", "haldane12_flux", "checkerboard12_flux"]


def _setup(golden, case):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden(case)
    a = golden("api_" + case)
    data = ed_data_for(case, g)
    model = data.second_quantized_model
    cmap = ed.CanonicalMap(data.symmetry_group, model.particle_statistics, data.orbit_catalog)
    return ed, a, data, model, cmap


def _sectors(a):
    return [int(s) for s in a["sectors"]]


@pytest.mark.parametrize("case", CASES)
def test_operator_and_apply_return_h_times_x(golden, case):
    ed, a, data, model, cmap = _setup(golden, case)
    bil, den = model.bilinear_terms, model.density_density_terms
    for s in _sectors(a):
        p = f"s{s}_"
        basis = ed.build_symmetry_sector_basis(data.orbit_catalog, data.irrep_list[s])
        assert basis.dim == int(a[p + "dim"])
        x = a[p + "x"]
        H_op, n = ed.hamiltonian_linear_operator(basis, bil, den, cmap)
        assert n == len(x)
        scale = float(H_op.csr().val.abs().max()) * np.abs(x).sum()
        y = H_op(x)
        assert isinstance(y, np.ndarray) and y.dtype == np.complex128
        np.testing.assert_allclose(y, a[p + "y_op"], rtol=0, atol=1e-12 * scale)
        # CUDA input stays on the device; [n, k] blocks apply column by column
        xd = torch.from_numpy(np.stack([x, 2j * x], axis=1)).cuda()
        yd = H_op(xd)
        assert yd.is_cuda and yd.shape == (n, 2)
        np.testing.assert_allclose(yd[:, 1].cpu().numpy(), 2j * a[p + "y_op"], rtol=0, atol=2e-12 * scale)
        # apply_hamiltonian writes into the caller's y and returns it
        yy = np.zeros(n, dtype=np.complex128)
        out = ed.apply_hamiltonian(yy, x, basis, bil, den, cmap)
        assert out is yy
        np.testing.assert_allclose(yy, a[p + "y_apply"], rtol=0, atol=1e-12 * scale)
        yy2 = np.zeros(n, dtype=np.complex128)
        ed.apply_hamiltonian_with_threads(yy2, x, basis, bil, den, cmap, None)
        np.testing.assert_array_equal(yy2, yy)
        with pytest.raises(AssertionError):
            ed.apply_hamiltonian(np.zeros(n + 1, dtype=np.complex128), x, basis, bil, den, cmap)


@pytest.mark.parametrize("case", CASES)
def test_projection_table_matches_reference(golden, case):
    ed, a, data, model, cmap = _setup(golden, case)
    for s in _sectors(a):
        p = f"s{s}_"
        basis = ed.build_symmetry_sector_basis(data.orbit_catalog, data.irrep_list[s])
        row, col, vals, hdiag = ed.build_matrixfree_projection_table(
            basis, model.bilinear_terms, model.density_density_terms, cmap)
        n = basis.dim
        np.testing.assert_allclose(hdiag, a[p + "pt_hdiag"], rtol=0, atol=1e-14)
        assert len(row) == len(a[p + "pt_row"])

        def canon(r, c, v):
            o = np.lexsort((np.round(v.imag, 11), np.round(v.real, 11), r, c))
            return r[o], c[o], v[o]

        r0, c0, v0 = canon(np.asarray(row), np.asarray(col), np.asarray(vals))
        r1, c1, v1 = canon(a[p + "pt_row"], a[p + "pt_col"], a[p + "pt_vals"])
        np.testing.assert_array_equal(r0, r1)
        np.testing.assert_array_equal(c0, c1)
        np.testing.assert_allclose(v0, v1, rtol=0, atol=1e-14)
        A = sp.coo_matrix((vals, (row, col)), shape=(n, n)).toarray()
        B = sp.coo_matrix((a[p + "pt_vals"], (a[p + "pt_row"], a[p + "pt_col"])), shape=(n, n)).toarray()
        np.testing.assert_allclose(A, B, rtol=0, atol=1e-14)


@pytest.mark.parametrize("case", CASES)
def test_canonical_lookups_match_reference(golden, case):
    ed, a, data, model, cmap = _setup(golden, case)
    masks = [int(m) for m in a["masks"]]
    got = [ed.get_canonical(cmap, m) for m in masks]
    assert [r for r, _, _ in got] == [int(m) for m in a["canon_repr"]]
    assert [g for _, g, _ in got] == [int(x) for x in a["canon_g"]]
    np.testing.assert_allclose(np.array([al for _, _, al in got]), a["canon_alpha"], rtol=0, atol=1e-15)
    assert ed.populate_canonical_map(cmap, None, model.bilinear_terms) is cmap
    for s in _sectors(a):
        p = f"s{s}_"
        basis = ed.build_symmetry_sector_basis(data.orbit_catalog, data.irrep_list[s])
        for name, fn in (("proj", lambda m: ed.project_to_sector(m, basis, cmap)),
                         ("uproj", lambda m: ed.project_to_unnormalized_sector(m, basis, model.particle_statistics))):
            res = [fn(m) for m in masks]
            idx = np.array([-1 if r is None else r[0] for r in res])
            coef = np.array([0j if r is None else r[1] for r in res])
            np.testing.assert_array_equal(idx, a[p + name + "_idx"])
            np.testing.assert_allclose(coef, a[p + name + "_coef"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("case", CASES)
def test_diagonalize_block_functions_match_reference(golden, case):
    ed, a, data, model, cmap = _setup(golden, case)
    bil, den = model.bilinear_terms, model.density_density_terms
    for s in _sectors(a):
        p = f"s{s}_"
        basis = ed.build_symmetry_sector_basis(data.orbit_catalog, data.irrep_list[s])
        H = ed.build_ed_Hamiltonian_symmetry_block(basis, bil, den, cmap)
        assert isinstance(H, sp.csr_matrix)
        vd, Ud = ed.diagonalize_block_dense(H, nev=3)
        np.testing.assert_allclose(vd, a[p + "dense_vals"], rtol=0, atol=1e-10)
        va, Ua = ed.diagonalize_block_arpack(H, nev=3)  # bare CSR: dense <= 500 rows, device Lanczos above
        np.testing.assert_allclose(va, a[p + "arpack_vals"], rtol=0, atol=1e-10)
        for vals, U in ((vd, Ud), (va, Ua)):
            assert U.shape == (H.shape[0], 3)
            for j in range(3):
                assert np.linalg.norm(H @ U[:, j] - vals[j] * U[:, j]) < 1e-7
        H_op, n = ed.hamiltonian_linear_operator(basis, bil, den, cmap)
        vm, _ = ed.diagonalize_block_matrixfree(H_op, n, nev=3)
        np.testing.assert_allclose(vm, a[p + "mf_vals"], rtol=0, atol=1e-10)


def test_diagonalize_block_arpack_on_a_large_bare_csr(golden):
    """An 11,240-row flux block handed over as a scipy CSR without its basis:
    the reference solves it with ARPACK ``eigs``; here the device Lanczos."""
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden("haldane24_flux")
    a = golden("api_haldane24_flux_arpack")
    data = ed_data_for("haldane24_flux", g)
    model = data.second_quantized_model
    cmap = ed.CanonicalMap(data.symmetry_group, model.particle_statistics, data.orbit_catalog)
    basis = ed.build_symmetry_sector_basis(data.orbit_catalog, data.irrep_list[int(a["sector"])])
    H = ed.build_ed_Hamiltonian_symmetry_block(basis, model.bilinear_terms, model.density_density_terms, cmap)
    assert H.shape[0] == int(a["dim"]) and H.nnz == int(a["nnz"])
    vals, vecs = ed.diagonalize_block_arpack(H, nev=4)
    np.testing.assert_allclose(vals, a["vals"], rtol=0, atol=1e-10)
    for j in range(4):
        assert np.linalg.norm(H @ vecs[:, j] - vals[j] * vecs[:, j]) < 1e-6


def test_full_ed_is_the_union_of_the_sectors(golden):
    import realspace_exatdiagonalization_py_b200 as ed
    from _cases import model_for

    g = golden("heisenberg16")
    vals, vecs = ed.full_ed(model_for("heisenberg16"), 8, nev=4)
    union = np.sort(g["eig_vals"].ravel())[:4]
    np.testing.assert_allclose(vals, union, rtol=0, atol=1e-10)
    assert vecs.shape == (12870, 4)


def test_print_spectrum_rows(golden, capsys):
    ed, a, data, model, cmap = _setup(golden, "heisenberg16")
    ed.ed_scan(data, nev=2, mode="matrixfree", scanned_sectors=[data.irrep_list[0].label, data.irrep_list[8].label])
    spec = ed.print_spectrum(data)
    out = capsys.readouterr().out.splitlines()
    assert out[0] == "ED Spectrum (rows = irrep, cols = eigenvalue #):"
    assert len(out) == 1 + len(data.irrep_list)
    assert np.nanmin(spec) == 0.0 and spec.shape == (len(data.irrep_list), 2)
    assert "NaN" in out[2] and "NaN" not in out[1]
