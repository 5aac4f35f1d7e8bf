"""The CPU oracle (oracle/port.py) against the reference's golden fixtures.

Pins the oracle before it is trusted as the checker of the GPU kernels:
catalog tables bit for bit, stabilizers, the flux phase update, sector
dimensions and sector eigenvalues (ARPACK / dense, |dE| < 1e-10).
"""

import numpy as np
import pytest

from oracle import port

CASES = ["heisenberg16", "checkerboard24", "haldane12", "haldane12_flux", "checkerboard12_flux",
         "haldane24_flux", "hubbard12"]


def _oracle_catalog(g, eta=None):
    perm0 = (g["perm"] - 1).astype(np.uint8)
    return port.catalog(int(g["n_site"]), int(g["n_filled"]), perm0,
                        g["eta"] if eta is None else eta, bool(g["fermionic"]))


def _check_catalog(cat, g, prefix=""):
    np.testing.assert_array_equal(cat["reprs"], g[prefix + "reprs"])
    np.testing.assert_array_equal(cat["rep_rank"], g[prefix + "rep_rank"])
    np.testing.assert_array_equal(cat["rep_sym"], g[prefix + "rep_sym"])
    np.testing.assert_array_equal(cat["rep_amp"], g[prefix + "rep_amp"])
    off = g[prefix + "stab_off"]
    for o in range(len(cat["reprs"])):
        np.testing.assert_array_equal(cat["stab_g"][o], g[prefix + "stab_g"][off[o]:off[o + 1]])
        np.testing.assert_array_equal(cat["stab_phase"][o], g[prefix + "stab_phase"][off[o]:off[o + 1]])


@pytest.mark.parametrize("case", CASES)
def test_catalog_matches_reference(golden, case):
    g = golden(case)
    _check_catalog(_oracle_catalog(g), g)


@pytest.mark.parametrize("case", ["haldane12_flux", "checkerboard12_flux", "haldane24_flux"])
def test_phase_update_matches_reference(golden, case):
    g = golden(case)
    eta0 = np.ones_like(g["eta"])
    cat = _oracle_catalog(g, eta0)
    port.update_phases(cat, int(g["n_site"]), (g["perm"] - 1).astype(np.uint8), g["eta"],
                       bool(g["fermionic"]))
    _check_catalog(cat, g, "upd_")


@pytest.mark.parametrize("case", CASES)
def test_sector_dims_and_energies(golden, case):
    g = golden(case)
    cat = _oracle_catalog(g)
    bil = [(int(i), int(j), t) for (i, j), t in zip(g["bil_ij"], g["bil_t"])]
    den = [(int(i), int(j), v) for (i, j), v in zip(g["den_ij"], g["den_v"])]
    dims = [len(port.sector_orbits(cat, chi)) for chi in g["chi"]]
    np.testing.assert_array_equal(dims, g["sector_dims"])
    nev = int(g["nev"])
    for s, ref in zip(g["eig_sectors"], g["eig_vals"]):
        chi = g["chi"][s]
        orbits = port.sector_orbits(cat, chi)
        H = port.csr_block(cat, int(g["n_site"]), orbits, bil, den, chi, bool(g["fermionic"]))
        w, _ = port.solve(H, nev)
        k = min(nev, len(w))
        np.testing.assert_allclose(w[:k], ref[:k], atol=1e-10, rtol=0)


def test_rank_unrank_roundtrip():
    n, k = 20, 7
    bt = port.binom_table(n, k)
    r = np.arange(0, 77520, 37, dtype=np.int64)
    m = port.unrank(r, n, k, bt)
    np.testing.assert_array_equal(port.rank(m, n, bt), r)
    assert np.all(np.bitwise_count(m) == k)


def test_rank_beyond_42_sites():
    # the reference's >42-site fallback returns 0; the oracle's rank is exact
    n, k = 48, 3
    bt = port.binom_table(n, k)
    r = np.array([0, 1, 17295, 17296 - 1], dtype=np.int64)
    m = port.unrank(r, n, k, bt)
    np.testing.assert_array_equal(port.rank(m, n, bt), r)


def _spin_down_mask(n_site):
    # spin-orbital index = 2 * cell + spin (1-based sites 2, 4, ... are spin down)
    return sum(1 << i for i in range(1, n_site, 2))


def test_two_species_spectra_union_is_total_n(golden):
    """Per-spin (N_up, N_down) bases: the union of their sector spectra over
    all N_down equals the reference's total-N sector spectrum (Hubbard 2x3,
    6 electrons), and the lowest levels equal the reference's energies."""
    g = golden("hubbard12")
    n, k = int(g["n_site"]), int(g["n_filled"])
    perm0 = (g["perm"] - 1).astype(np.uint8)
    bil = [(int(i), int(j), t) for (i, j), t in zip(g["bil_ij"], g["bil_t"])]
    den = [(int(i), int(j), v) for (i, j), v in zip(g["den_ij"], g["den_v"])]
    sb = _spin_down_mask(n)
    total = port.catalog(n, k, perm0, g["eta"], True)
    per = {kb: port.catalog(n, k, perm0, g["eta"], True, species=(sb, kb))
           for kb in range(0, k + 1) if k - kb <= n // 2 and kb <= n // 2}
    assert sum(len(c["rep_rank"]) for c in per.values()) == len(total["rep_rank"])
    for s in range(len(g["chi"])):
        chi = g["chi"][s]
        full = np.linalg.eigvalsh(port.csr_block(total, n, port.sector_orbits(total, chi), bil, den, chi,
                                                 True).toarray())
        parts = []
        for c in per.values():
            orb = port.sector_orbits(c, chi)
            if len(orb):
                parts.append(np.linalg.eigvalsh(port.csr_block(c, n, orb, bil, den, chi, True).toarray()))
        union = np.sort(np.concatenate(parts))
        np.testing.assert_allclose(union, full, atol=1e-10, rtol=0)
        np.testing.assert_allclose(full[:4], g["eig_vals"][s][:4], atol=1e-9, rtol=0)


def test_two_species_rank_roundtrip():
    bt = port.binom_table(12, 6)
    for kb in range(0, 7):
        C, rk, ur = port.species_basis(12, 6, (_spin_down_mask(12), kb), bt)
        r = np.arange(C)
        m = ur(r)
        assert np.array_equal(rk(m), r)
        assert np.all(np.diff(r) > 0) and len(np.unique(m)) == C


@pytest.mark.parametrize("case", ["haldane12_flux", "checkerboard12_flux", "hubbard12"])
def test_fock_expansion_matches_reference(golden, case):
    """The oracle's sector -> Fock expansion against the reference's own
    function (tests/golden/make_fock_golden.py)."""
    import os

    g = golden(case)
    f = np.load(os.path.join(os.path.dirname(__file__), "golden", f"fock_{case}.npz"))
    n, k = int(g["n_site"]), int(g["n_filled"])
    perm0 = (g["perm"] - 1).astype(np.uint8)
    cat = port.catalog(n, k, perm0, g["eta"], bool(g["fermionic"]))
    for s in f["sectors"]:
        orbits = port.sector_orbits(cat, g["chi"][s])
        amps = port.fock_expand(cat, orbits, f[f"c_{s}"], g["chi"][s], perm0, g["eta"], bool(g["fermionic"]))
        keys = np.array(sorted(amps), dtype=np.uint64)
        np.testing.assert_array_equal(keys, f[f"masks_{s}"])
        np.testing.assert_allclose(np.array([amps[int(x)] for x in keys]), f[f"amps_{s}"], atol=1e-14, rtol=0)


@pytest.mark.parametrize("case", ["haldane12", "haldane16", "haldane16_singular", "checkerboard12",
                                  "haldane12_identity"])
def test_chern_oracle_matches_reference(case):
    """The oracle's flux-torus Chern number against the reference's driver
    (tests/golden/make_chern_golden.py): gauge-invariant plaquette phases,
    |det| of every link, energies and the near-singular count."""
    from _cases import chern_case

    import realspace_exatdiagonalization_py_b200 as ed

    model, n_part, labels, nev, grid, f = chern_case(case)
    ident = labels == "identity"

    def flux_setup(flux):
        ed.update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=flux)
        G = ed.build_identity_group(model.lattice.n_site) if ident else ed.build_translation_group(model.lattice, flux)
        return G, ed.build_irrep_list(G, model.lattice)

    r = port.chern(model, n_part, ["identity"] if ident else labels, grid, nev, flux_setup)
    np.testing.assert_allclose(r["energies"], f["energies"], atol=1e-10, rtol=0)
    np.testing.assert_allclose(r["berry_curvature"], f["berry_curvature"], atol=1e-9, rtol=0)
    assert abs(r["chern_number"] - float(f["chern_number"])) < 1e-9
    for k in ("link_det_abs_x", "link_det_abs_y"):
        big = f[k] > 1e-8
        np.testing.assert_allclose(r[k][big], f[k][big], atol=1e-9, rtol=0)
        assert np.all(r[k][~big] <= 1e-10)
    assert r["n_singular"] == int(f["n_singular_warnings"])


def test_chern_checkpoint_names():
    """Checkpoint file names of the Chern scan, including the FNV-1a digest of
    the parameters, are the reference's (many_body_chern_number.py:75-138)."""
    from fractions import Fraction

    from _cases import chern_case

    from realspace_exatdiagonalization_py_b200 import observables as obs

    for case in ("haldane12", "checkerboard12", "haldane16"):
        model, n_part, labels, nev, grid, f = chern_case(case)
        ff = Fraction(n_part, model.lattice.n_site)
        nx, ny = grid
        assert obs._chern_checkpoint_path(model, ff, [0.0, 0.0], "d") == "d/" + str(f["checkpoint_00"])
        assert obs._chern_checkpoint_path(model, ff, [1 / nx, 1 / ny], "d") == "d/" + str(f["checkpoint_11"])
    assert obs._normalize_flux_grid_size(4) == (4, 4) and obs._normalize_flux_grid_size([3, 2]) == (3, 2)
    with pytest.raises(ValueError):
        obs._normalize_flux_grid_size((1, 3))
    assert obs._chern_sector_labels("identity") == ["identity"]
    assert obs._chern_sector_labels([[1, 0]]) == [(1, 0)]
    assert obs._chern_flux_tag([0.25, -0.5]) == "0p250000_m0p500000"


@pytest.mark.parametrize("case", ["haldane12", "checkerboard12", "haldane16"])
def test_charge_pump_oracle_matches_reference(case):
    """The oracle's charge pump against the reference's driver
    (tests/golden/make_pump_golden.py): polarization eigenvalues (invariant
    under the gauge of the manifold states), tracked polarizations, pumped
    charges and energies."""
    from _cases import pump_case, pump_specs

    import realspace_exatdiagonalization_py_b200 as ed

    model, f = pump_case(case)

    def flux_setup(flux):
        ed.update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=flux)
        G = ed.build_translation_group(model.lattice, flux)
        return G, ed.build_irrep_list(G, model.lattice)

    phases = ed.many_body_position_phases(model.lattice, int(f["polarization_direction"]),
                                          include_sublattice=bool(f["include_sublattice"]))
    ev, pol, pumped, E = port.charge_pump(model, int(f["n_particles"]), pump_specs(f), list(f["thetas"]),
                                          int(f["flux_direction"]), phases, flux_setup)
    np.testing.assert_allclose(E, f["energies"], atol=1e-10, rtol=0)
    np.testing.assert_allclose(ev, f["polarization_eigenvalues"], atol=1e-9, rtol=0)
    np.testing.assert_allclose(pol, f["polarizations"], atol=1e-9, rtol=0)
    np.testing.assert_allclose(pumped, f["pumped_charges"], atol=1e-9, rtol=0)


def test_charge_pump_host_helpers():
    """Position phases, default direction, manifold specs and branch tracking
    (charge_pump.py:41-322) on fixed inputs."""
    from realspace_exatdiagonalization_py_b200 import models
    from realspace_exatdiagonalization_py_b200 import observables as obs

    m = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[2, 3], params=models.params_DNSheng)
    ph = obs.many_body_position_phases(m.lattice, 2)
    for i, (cell, sub) in enumerate(m.lattice.site_list):
        x = cell[1] + m.lattice.sub_crys_list[sub - 1][1]
        assert abs(ph[i] - np.exp(2j * np.pi * x / 3)) < 1e-15
    with pytest.raises(ValueError):
        obs.many_body_position_phases(m.lattice, 3)
    assert obs._default_polarization_direction(2, 1) == 2 and obs._default_polarization_direction(2, 2) == 1
    assert obs._default_polarization_direction(1, 1) == 1
    labels, specs, req, ident = obs._normalize_manifold_state_specs([(0, 0), (1, 0)], 2, None)
    assert labels == [(0, 0), (1, 0)] and len(specs) == 4 and req == {(0, 0): 2, (1, 0): 2} and not ident
    labels, specs, req, _ = obs._normalize_manifold_state_specs([(0, 0)], 1, [((0, 0), 2), {"sector": (0, 0),
                                                                                             "level": 1}])
    assert [(s.sector, s.level) for s in specs] == [((0, 0), 2), ((0, 0), 1)] and req == {(0, 0): 2}
    for bad in ([((1, 1), 1)], [((0, 0), 0)], [((0, 0), 1), ((0, 0), 1)], []):
        with pytest.raises(ValueError):
            obs._normalize_manifold_state_specs([(0, 0)], 1, bad)
    with pytest.raises(ValueError):
        obs._normalize_manifold_state_specs([(0, 0)], 0, None)
    raw = np.array([[0.1, -0.2, 0.4], [0.45, 0.15, -0.1], [-0.45, 0.2, -0.05]])
    np.testing.assert_array_equal(obs._tracked_phase_branches(raw), port._track(raw))


def test_charge_pump_rejects_identity_before_any_work():
    from fractions import Fraction

    from realspace_exatdiagonalization_py_b200 import models
    from realspace_exatdiagonalization_py_b200 import observables as obs

    m = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[2, 3], params=models.params_DNSheng)
    with pytest.raises(ValueError, match="identity"):
        obs.flux_charge_pump(m, "identity", filling_fraction=Fraction(3, 12))
    with pytest.raises(ValueError, match="flux_direction"):
        obs.flux_charge_pump(m, [(0, 0)], filling_fraction=Fraction(3, 12), flux_direction=3)


@pytest.mark.parametrize("case", ["haldane12", "checkerboard12", "haldane12_identity", "haldane16"])
def test_correlators_oracle_matches_reference(case):
    """The oracle's one-body density matrix (the reference's orbit-by-orbit
    accumulation) and connected <n_i n_j> (exact sums over the state's Fock
    amplitudes) against the reference's functions
    (tests/golden/make_corr_golden.py)."""
    from _cases import corr_case

    import realspace_exatdiagonalization_py_b200 as ed

    model, label, level, fa, f = corr_case(case)
    n = model.lattice.n_site
    nf = int(f["n_particles"])
    G = ed.build_identity_group(n) if label == "identity" else ed.build_translation_group(model.lattice)
    irreps = ed.build_irrep_list(G, model.lattice)
    s = 0 if label == "identity" else next(i for i, ir in enumerate(irreps) if ir.label == label)
    perm0, eta = port.group_arrays(G)
    fermion = model.particle_statistics.name == "FERMIONIC"
    cat = port.catalog(n, nf, perm0, eta, fermion)
    chi = np.asarray(irreps[s].values, dtype=np.complex128)
    orbits = port.sector_orbits(cat, chi)
    H = port.csr_block(cat, n, orbits, model.bilinear_terms, model.density_density_terms, chi, fermion)
    _, v = port.solve(H, max(level, 2), seeded_v0=False)
    rho = port.obdm_orbitwise(cat, orbits, v[:, level - 1], chi, perm0, eta, fermion, n, nf)
    np.testing.assert_allclose(rho, f["odlro"], atol=1e-11, rtol=0)
    amps = port.fock_expand(cat, orbits, v[:, level - 1], chi, perm0, eta, fermion)
    rho_fock, nn = port.fock_correlators(amps, n, fermion)
    if case in ("haldane12", "haldane12_identity"):
        # real projection coefficients (zero flux, real characters): the
        # reference's matrix is the exact <a_i^dagger a_j>
        np.testing.assert_allclose(rho_fock, f["odlro"], atol=1e-11, rtol=0)
    a = np.array([fa(i + 1) for i in range(n)])
    dens = np.diag(nn)
    da = np.where(a, dens, 0.0)
    C = np.where(a[:, None], nn, 0.0) - np.outer(da, dens)
    np.testing.assert_allclose(da, f["density_a"], atol=1e-11, rtol=0)
    np.testing.assert_allclose(dens, f["density_b"], atol=1e-11, rtol=0)
    np.testing.assert_allclose(C, f["C"], atol=1e-11, rtol=0)


def test_uniform_grid_and_positions():
    """The momentum mesh q = sum_d (n_d / L_d) b_d and the site positions of
    the lattice restatement: a_d . b_e = 2 pi delta_de, L_1 L_2 points, and
    exp(i q . R) = 1 for q on the mesh and R a torus period."""
    from realspace_exatdiagonalization_py_b200 import lattice as tb
    from realspace_exatdiagonalization_py_b200 import models

    m = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[2, 3], params=models.params_DNSheng)
    lat = m.lattice
    grid = tb.initialize_uniform_grids_from_lattice(lat)
    assert grid.nsite == 6 and len(grid.site_cart_list) == 6
    a = np.array(lat.brav_vec_list)
    for q in grid.site_cart_list:
        for d, L in enumerate(lat.sample_size):
            assert abs(np.exp(1j * np.dot(q, L * a[d])) - 1) < 1e-12
    pos = np.array(lat.site_cart_list)
    cell, sub = lat.site_list[5]
    want = sum((cell[d] + lat.sub_crys_list[sub - 1][d]) * a[d] for d in range(2))
    np.testing.assert_allclose(pos[5], want, atol=1e-15)


@pytest.mark.parametrize("model,label", [("Heisenberg", "N=18"), ("Haldane_Boson", "2×3"), ("Haldane_Boson", "2×4"),
                                         ("Haldane_Boson", "2×5"), ("Hubbard_Fermion", "2×2"),
                                         ("Hubbard_Fermion", "2×3"), ("Hubbard_Fermion", "2×4")])
def test_oracle_matches_reference_benchmark(model, label):
    """The oracle's sector-0 dimension and lowest energy against the
    reference's own benchmark results (tests/golden/make_benchmark_golden.py)
    on the sizes the CPU restatement finishes in seconds."""
    import os
    from fractions import Fraction

    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models

    f = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "reference_benchmark.npz")))
    i = next(k for k in range(len(f["model"])) if str(f["model"][k]) == model and str(f["label"][k]) == label)
    n_site, n_filled = int(f["n_site"][i]), int(f["n_filled"][i])
    if model == "Heisenberg":
        m = models.build_heisenberg_second_quantized_model(n_site, 1.0)
    elif model == "Haldane_Boson":
        m = models.build_zero_flux_bosonic_fci_second_quantized_model(
            sample_size=[int(x) for x in label.split("×")], params=models.params_DNSheng)
    else:
        m = models.build_spinful_hubbard_second_quantized_model([int(x) for x in label.split("×")], 1.0, 8.0)
    G = ed.build_translation_group(m.lattice)
    irreps = ed.build_irrep_list(G, m.lattice)
    out = port.scan(m, n_filled, G, irreps, 1, sectors=[0])
    vals, dim = out[0]
    assert dim == int(f["sector_dim"][i])
    assert abs(float(vals[0]) - float(f["energy"][i])) < 1e-9


def test_brillouin_zone_helpers_match_reference():
    """First-Brillouin-zone polygon and folded mesh momenta of the 2x3
    honeycomb lattice against the reference (static_structure_factor.py:210-377,
    tests/golden/make_corr_golden.py)."""
    import os

    from realspace_exatdiagonalization_py_b200 import correlators as cr
    from realspace_exatdiagonalization_py_b200 import models

    f = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", "corr_manifold_haldane12.npz")))
    m = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[2, 3], params=models.params_DNSheng)
    poly = np.array([np.asarray(p) for p in cr._first_bz_polygon(m.lattice)])
    np.testing.assert_allclose(poly, f["bz_polygon"], atol=1e-12, rtol=0)
    folded = cr._fold_momenta_to_first_bz(list(f["q_points"]), m.lattice)
    np.testing.assert_allclose([p[0] for p in folded], f["allowed_qx"], atol=1e-12, rtol=0)
    np.testing.assert_allclose([p[1] for p in folded], f["allowed_qy"], atol=1e-12, rtol=0)
