"""Correlators of one sector eigenstate on the device -- the one-body density
matrix and the connected density correlations behind the static structure
factor -- against the reference's own functions
(tests/golden/make_corr_golden.py)."""

from fractions import Fraction

import numpy as np
import pytest

from _cases import CORR_CASES, corr_case

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", CORR_CASES)
def test_correlators_match_reference(case):
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import correlators as cr

    model, label, level, fa, f = corr_case(case)
    ff = Fraction(int(f["n_particles"]), model.lattice.n_site)
    n = model.lattice.n_site
    ed_data, basis, c = cr._bootstrap_ed_sector(model, label, ff, level, "matrix", None)
    rho = ed.off_diagonal_long_range_order(model, label, target_eigval_idx=level, filling_fraction=ff,
                                           ed_data=ed_data)
    np.testing.assert_allclose(rho, f["odlro"], atol=1e-10, rtol=0)
    C, da, db = np.zeros((n, n)), np.zeros(n), np.zeros(n)
    cr._build_density_correlation_matrix(C, da, db, c, basis, n, fa, lambda i: True)
    np.testing.assert_allclose(C, f["C"], atol=1e-11, rtol=0)
    np.testing.assert_allclose(da, f["density_a"], atol=1e-11, rtol=0)
    np.testing.assert_allclose(db, f["density_b"], atol=1e-11, rtol=0)
    q, S = ed.static_structure_factor(model, label, target_eigval_idx=level, filling_fraction=ff, flavor_a=fa,
                                      ed_data=ed_data)
    np.testing.assert_allclose(np.array(q), f["q_points"], atol=1e-14, rtol=0)
    np.testing.assert_allclose(S, f["S_q"], atol=1e-11, rtol=0)
    _, _, Smap = ed.compute_structure_factor_map(model, label, target_eigval_idx=level, filling_fraction=ff,
                                                 flavor_a=fa, k_resolution=5, ed_data=ed_data)
    np.testing.assert_allclose(Smap, f["S_map"], atol=1e-11, rtol=0)
    _, _, rmap = ed.compute_odlro_map(model, label, target_eigval_idx=level, filling_fraction=ff, k_resolution=5,
                                      ed_data=ed_data)
    np.testing.assert_allclose(rmap, f["odlro_map"], atol=1e-10, rtol=0)


def test_correlators_bootstrap_without_ed_data():
    """The drivers scan the zero-flux model themselves when no ED data is
    passed (the reference's bootstrap), with the same results."""
    import realspace_exatdiagonalization_py_b200 as ed

    model, label, level, fa, f = corr_case("haldane12")
    ff = Fraction(int(f["n_particles"]), model.lattice.n_site)
    rho = ed.off_diagonal_long_range_order(model, label, target_eigval_idx=level, filling_fraction=ff)
    np.testing.assert_allclose(rho, f["odlro"], atol=1e-10, rtol=0)
    with pytest.raises(ValueError):
        ed.off_diagonal_long_range_order(model, (7, 7), filling_fraction=ff)


def test_one_body_density_two_species_blocks():
    """Two-species basis (Hubbard, fixed N_up and N_down): hops between the
    species are zero, the trace is the particle number and the matrix is
    Hermitian."""
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import correlators as cr
    from realspace_exatdiagonalization_py_b200 import models

    m = models.build_spinful_hubbard_second_quantized_model([2, 3], 1.0, 4.0)
    G = ed.build_translation_group(m.lattice)
    sites_b, nb = models.hubbard_spin_species(m, 3)
    data = ed.build_ed_data(m, filling_fraction=Fraction(6, 12), symmetry_group=G, species=(sites_b, nb))
    ed.ed_scan(data, nev=2, scanned_sectors=[data.irrep_list[0].label])
    _, basis, c = cr._bootstrap_ed_sector(m, data.irrep_list[0].label, Fraction(6, 12), 1, "matrix", data)
    rho = cr.one_body_density_matrix(basis, c)
    assert abs(np.trace(rho) - 6) < 1e-10
    np.testing.assert_allclose(rho, rho.conj().T, atol=1e-12)
    b = np.zeros(12, dtype=bool)
    b[[s - 1 for s in sites_b]] = True
    assert np.abs(rho[np.ix_(b, ~b)]).max() == 0 and np.abs(rho[np.ix_(~b, b)]).max() == 0
    assert abs(np.trace(rho[np.ix_(b, b)]) - nb) < 1e-10


def test_manifold_structure_factor_matches_reference():
    """Manifold averages (uniform and 2:1 weights), their allowed-momenta and
    map forms, and the single-state allowed momenta against the reference
    (tests/golden/make_corr_golden.py)."""
    import os

    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models

    f = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "corr_manifold_haldane12.npz")))
    m = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[2, 3], params=models.params_DNSheng)
    ff = Fraction(3, 12)
    states = [((0, 0), 1), ((1, 0), 1)]
    q, S = ed.static_structure_factor_manifold_average(m, states, filling_fraction=ff)
    np.testing.assert_allclose(np.array(q), f["q_points"], atol=1e-14, rtol=0)
    np.testing.assert_allclose(S, f["S_uniform"], atol=1e-11, rtol=0)
    _, Sw = ed.static_structure_factor_manifold_average(m, states, weights=[2.0, 1.0], filling_fraction=ff)
    np.testing.assert_allclose(Sw, f["S_weighted"], atol=1e-11, rtol=0)
    mx, my, mS = ed.structure_factor_manifold_allowed_momenta(m, states, filling_fraction=ff)
    np.testing.assert_allclose(mx, f["manifold_qx"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(my, f["manifold_qy"], atol=1e-12, rtol=0)
    np.testing.assert_allclose(mS, f["manifold_S"], atol=1e-11, rtol=0)
    _, _, mmap = ed.compute_structure_factor_manifold_average_map(m, states, filling_fraction=ff, k_resolution=5)
    np.testing.assert_allclose(mmap, f["manifold_map"], atol=1e-11, rtol=0)
    ax, ay, aS = ed.structure_factor_allowed_momenta(m, (0, 0), filling_fraction=ff)
    np.testing.assert_allclose(aS, f["allowed_S"], atol=1e-11, rtol=0)
    np.testing.assert_allclose(ax, f["allowed_qx"], atol=1e-12, rtol=0)
    with pytest.raises(ValueError):
        ed.static_structure_factor_manifold_average(m, states, weights=[1.0], filling_fraction=ff)
    with pytest.raises(ValueError):
        ed.static_structure_factor_manifold_average(m, [], filling_fraction=ff)
