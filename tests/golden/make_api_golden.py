"""Generate tests/golden/api_<case>.npz: outputs of the reference's
single-sector API functions, called with the reference's own signatures.

For the cases heisenberg16, haldane12_flux and checkerboard12_flux (the
models of tests/golden/make_golden.py) and two sectors each, the reference
engine (loaded through oracle/ref_shim.py) gives

* ``hamiltonian_linear_operator(basis, bilinear, density, cmap)`` -> ``H_op(x)``
  and ``apply_hamiltonian(y, x, basis, bilinear, density, cmap)`` on a seeded
  complex vector;
* ``build_matrixfree_projection_table(basis, bilinear, density, cmap)`` ->
  ``(row_ind, col_ind, vals, h_diag)``;
* ``get_canonical(cmap, m)``, ``project_to_sector(m, basis, cmap)`` and
  ``project_to_unnormalized_sector(m, basis, stats)`` for 300 seeded masks of
  the fixed-filling basis;
* ``diagonalize_block_dense`` / ``diagonalize_block_arpack`` of the sector
  block from ``build_ed_Hamiltonian_symmetry_block`` and
  ``diagonalize_block_matrixfree(H_op, n)`` eigenvalues (nev 3).

A large-block case (haldane24_flux, sector (0, 0), 11k rows, where
``diagonalize_block_arpack`` takes the ARPACK ``eigs`` path on the bare CSR)
stores the reference's eigenvalues of that call.

    python tests/golden/make_api_golden.py
"""

from __future__ import annotations

import os
import sys
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
sys.path.insert(0, HERE)

from make_golden import quiet  # noqa: E402

from oracle import ref_shim  # noqa: E402

N_MASKS = 300
NEV = 3


def build_case(R, case):
    sre = R.sre
    theta = None
    if case == "heisenberg16":
        model, nf = quiet(R.heisenberg.build_heisenberg_second_quantized_model, 16, 1.0), 8
    elif case == "haldane12_flux":
        model, nf = R.bosonic.build_zero_flux_bosonic_fci_second_quantized_model(
            sample_size=[2, 3], params=R.bosonic.params_DNSheng), 3
        theta = [0.3, 0.1]
    elif case == "checkerboard12_flux":
        model, nf = quiet(R.fermionic.build_zero_flux_fermionic_fci_second_quantized_model,
                          sample_size=[2, 3], params=dict(R.fermionic.params_Sun_Gu_Katsura_Sarma)), 4
        theta = [0.25, 0.4]
    elif case == "haldane24_flux":
        pb = {"t": 1.0, "t'": 0.6, "t''": 0.0, "phi_over_2pi": 0.2, "V1": 1.0, "V2": 0.0}
        model, nf = R.bosonic.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[3, 4], params=pb), 6
        theta = [0.125, 0.375]
    else:
        raise ValueError(case)
    if theta is not None:
        R.sqm.update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=theta)
    G = sre.build_translation_group(model.lattice, theta)
    data = quiet(sre.build_ed_data, model, filling_fraction=Fraction(nf, model.lattice.n_site), symmetry_group=G)
    return model, nf, G, data


def none_pair(r):
    return (-1, 0j) if r is None else (int(r[0]), complex(r[1]))


def make(R, case):
    sre = R.sre
    model, nf, G, data = build_case(R, case)
    n_site = model.lattice.n_site
    stats = model.particle_statistics
    cat = data.orbit_catalog
    cmap = sre.CanonicalMap(G, stats, cat)
    bil, den = model.bilinear_terms, model.density_density_terms
    rng = np.random.default_rng(77)
    masks = []
    for _ in range(N_MASKS):
        sites = rng.choice(n_site, size=nf, replace=False)
        masks.append(int(sum(1 << int(i) for i in sites)))
    out = {"masks": np.array(masks, dtype=np.uint64)}
    canon = [sre.get_canonical(cmap, m) for m in masks]
    out["canon_repr"] = np.array([c[0] for c in canon], dtype=np.uint64)
    out["canon_g"] = np.array([c[1] for c in canon], dtype=np.int64)
    out["canon_alpha"] = np.array([c[2] for c in canon], dtype=np.complex128)
    nsec = len(data.irrep_list)
    secs = sorted({0, nsec // 2})
    out["sectors"] = np.array(secs, dtype=np.int64)
    for s in secs:
        irrep = data.irrep_list[s]
        basis = sre.build_symmetry_sector_basis(cat, irrep)
        n = len(basis.representative_mask_list)
        p = f"s{s}_"
        out[p + "dim"] = np.int64(n)
        x = np.random.default_rng(100 + s).standard_normal(n) + 1j * np.random.default_rng(200 + s).standard_normal(n)
        out[p + "x"] = x
        H_op, n2 = quiet(sre.hamiltonian_linear_operator, basis, bil, den, cmap)
        assert n2 == n
        out[p + "y_op"] = H_op(x)
        y = np.zeros(n, dtype=np.complex128)
        out[p + "y_apply"] = quiet(sre.apply_hamiltonian, y, x, basis, bil, den, cmap)
        row, col, vals, hdiag = quiet(sre.build_matrixfree_projection_table, basis, bil, den, cmap)
        out[p + "pt_row"], out[p + "pt_col"] = np.asarray(row, np.int64), np.asarray(col, np.int64)
        out[p + "pt_vals"], out[p + "pt_hdiag"] = np.asarray(vals, np.complex128), np.asarray(hdiag, np.complex128)
        ps = [none_pair(sre.project_to_sector(m, basis, cmap)) for m in masks]
        out[p + "proj_idx"] = np.array([a for a, _ in ps], dtype=np.int64)
        out[p + "proj_coef"] = np.array([b for _, b in ps], dtype=np.complex128)
        pu = [none_pair(sre.project_to_unnormalized_sector(m, basis, stats)) for m in masks]
        out[p + "uproj_idx"] = np.array([a for a, _ in pu], dtype=np.int64)
        out[p + "uproj_coef"] = np.array([b for _, b in pu], dtype=np.complex128)
        H = quiet(sre.build_ed_Hamiltonian_symmetry_block, basis, bil, den, cmap)
        out[p + "dense_vals"] = quiet(sre.diagonalize_block_dense, H, nev=NEV)[0]
        out[p + "arpack_vals"] = quiet(sre.diagonalize_block_arpack, H, nev=NEV)[0]
        out[p + "mf_vals"] = quiet(sre.diagonalize_block_matrixfree, H_op, n, nev=NEV)[0]
    path = os.path.join(HERE, f"api_{case}.npz")
    np.savez_compressed(path, **out)
    print(f"api_{case}: sectors {secs} -> {os.path.getsize(path)} B")


def make_large(R):
    sre = R.sre
    model, nf, G, data = build_case(R, "haldane24_flux")
    cmap = sre.CanonicalMap(G, model.particle_statistics, data.orbit_catalog)
    basis = sre.build_symmetry_sector_basis(data.orbit_catalog, data.irrep_list[0])
    H = quiet(sre.build_ed_Hamiltonian_symmetry_block, basis, model.bilinear_terms, model.density_density_terms, cmap)
    vals, _ = quiet(sre.diagonalize_block_arpack, H, nev=4)
    path = os.path.join(HERE, "api_haldane24_flux_arpack.npz")
    np.savez_compressed(path, sector=np.int64(0), dim=np.int64(H.shape[0]), nnz=np.int64(H.nnz), vals=vals)
    print(f"api_haldane24_flux_arpack: n={H.shape[0]} nnz={H.nnz} -> {vals}")


def main():
    R = ref_shim.load()
    for case in ("heisenberg16", "haldane12_flux", "checkerboard12_flux"):
        make(R, case)
    make_large(R)


if __name__ == "__main__":
    main()
