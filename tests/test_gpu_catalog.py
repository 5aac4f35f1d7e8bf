"""GPU catalog kernels (K1-K5) against the reference's golden tables."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CASES = ["heisenberg16", "checkerboard24", "haldane12", "haldane12_flux", "checkerboard12_flux",
         "haldane24_flux", "hubbard12"]


def _group(g, eta=None):
    import realspace_exatdiagonalization_py_b200 as ed

    eta = g["eta"] if eta is None else eta
    ops = [ed.Symmetry_Operation(i, list(map(int, p)), perm_phases=e) for i, (p, e) in
           enumerate(zip(g["perm"], eta))]
    return ed.Finite_Symmetry_Group("translations", ops, identity_idx=0)


class _Lat:
    def __init__(self, n):
        self.n_site = n


class _Model:
    def __init__(self, n):
        self.lattice = _Lat(n)


def _stats(g):
    import realspace_exatdiagonalization_py_b200 as ed

    return ed.Particle_Statistics.FERMIONIC if int(g["fermionic"]) else ed.Particle_Statistics.BOSONIC


def build(g, eta=None):
    import realspace_exatdiagonalization_py_b200 as ed

    return ed.build_symmetry_orbit_catalog(second_quantized_model=_Model(int(g["n_site"])),
                                           n_filled=int(g["n_filled"]), symmetry_group=_group(g, eta),
                                           particle_statistics=_stats(g))


def assert_amplitudes(got, ref):
    """complex64 amplitudes bit for bit, except components below 1e-15 in
    magnitude (sin/cos of multiples of pi/2 land on different tiny values in
    different libm implementations)."""
    got = np.asarray(got, dtype=np.complex64)
    ref = np.asarray(ref, dtype=np.complex64)
    for part in (np.real, np.imag):
        a, b = part(got), part(ref)
        exact = a == b
        tiny = (np.abs(a) < 1e-15) & (np.abs(b) < 1e-15)
        bad = ~(exact | tiny)
        assert not bad.any(), (np.nonzero(bad)[0][:10], a[bad][:5], b[bad][:5])


def check_tables(cat, g, prefix=""):
    np.testing.assert_array_equal(np.array(cat.representative_mask_list, dtype=np.uint64), g[prefix + "reprs"])
    np.testing.assert_array_equal(cat.rep_rank_table, g[prefix + "rep_rank"])
    np.testing.assert_array_equal(cat.rep_sym_table, g[prefix + "rep_sym"])
    assert_amplitudes(cat.rep_amp_table, g[prefix + "rep_amp"])
    off = g[prefix + "stab_off"]
    np.testing.assert_array_equal(cat.stabilizer_order_list, np.diff(off))
    flat_g = [x for gs in cat.stabilizer_g_indices_list for x in gs]
    np.testing.assert_array_equal(flat_g, g[prefix + "stab_g"])
    flat_p = np.array([x for ps in cat.stabilizer_phases_list for x in ps], dtype=np.complex128)
    np.testing.assert_allclose(flat_p, g[prefix + "stab_phase"], atol=1e-15, rtol=0)


@pytest.mark.parametrize("case", CASES)
def test_catalog_bit_exact(golden, case):
    g = golden(case)
    check_tables(build(g), g)


@pytest.mark.parametrize("case", ["haldane12_flux", "checkerboard12_flux", "haldane24_flux"])
def test_phase_update_bit_exact(golden, case):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden(case)
    cat = build(g, np.ones_like(g["eta"]))
    new = _group(g)
    ed.update_orbit_stabilizer_phases(cat, new, _stats(g))
    check_tables(cat, g, "upd_")
    # same permutations, the update of the fresh flux catalog leaves integers intact
    np.testing.assert_array_equal(cat.rep_rank_table, g["rep_rank"])
    np.testing.assert_array_equal(cat.rep_sym_table, g["rep_sym"])


@pytest.mark.parametrize("case", CASES)
def test_sector_dims(golden, case):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden(case)
    cat = build(g)
    irreps = [ed.OneDim_Irrep(i, chi) for i, chi in enumerate(g["chi"])]
    ss = ed.SectorSet(cat, irreps)
    np.testing.assert_array_equal(ss.dims, g["sector_dims"])
    # the single-sector API agrees with the batched membership
    for s in range(len(irreps)):
        b = ed.build_symmetry_sector_basis(cat, irreps[s])
        assert len(b.representative_mask_list) == g["sector_dims"][s]
        oor, roo = ss.rows(s)
        oor = oor.cpu().numpy()
        assert np.all(np.diff(oor) > 0)
        roo = roo.cpu().numpy()
        np.testing.assert_array_equal(roo[oor], np.arange(len(oor)))


def test_edge_fillings():
    """n_filled in {0, n_site}: single state, product-form amplitudes."""
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models
    from oracle import port

    m = models.build_zero_flux_fermionic_fci_second_quantized_model(
        sample_size=[2, 3], params=models.params_Sun_Gu_Katsura_Sarma)
    ed.update_second_quantized_model_with_twisted_phases(m, twisted_phases_over_2π=[0.3, 0.2])
    G = ed.build_translation_group(m.lattice, [0.3, 0.2])
    perm0 = np.array([[p - 1 for p in op.perm] for op in G.operations], dtype=np.uint8)
    eta = np.array([op.perm_phases for op in G.operations])
    for k in (0, 12):
        cat = ed.build_symmetry_orbit_catalog(second_quantized_model=m, n_filled=k, symmetry_group=G,
                                              particle_statistics=m.particle_statistics)
        ref = port.catalog(12, k, perm0, eta, True)
        assert cat.representative_mask_list == [int(x) for x in ref["reprs"]]
        np.testing.assert_array_equal(cat.rep_rank_table, ref["rep_rank"])
        np.testing.assert_array_equal(cat.rep_sym_table, ref["rep_sym"])
        assert_amplitudes(cat.rep_amp_table, ref["rep_amp"])


def test_oracle_cross_check_random_groups():
    """Random permutation groups (not translations) and random phases: the
    kernels and the oracle agree on every table entry."""
    import realspace_exatdiagonalization_py_b200 as ed
    from oracle import port

    rng = np.random.default_rng(7)
    for n, k, fermion in [(10, 4, False), (11, 5, True), (14, 6, True), (13, 3, False)]:
        # cyclic group generated by a random permutation (orbits must be disjoint)
        while True:
            gen = rng.permutation(n)
            perms0 = [np.arange(n)]
            while True:
                nxt = gen[perms0[-1]]
                if np.array_equal(nxt, perms0[0]):
                    break
                perms0.append(nxt)
            if 2 <= len(perms0) <= 24:
                break
        ng = len(perms0)
        perms = [list(p + 1) for p in perms0]
        phases = [np.ones(n)] + [np.exp(2j * np.pi * rng.random(n)) for _ in range(ng - 1)]
        ops = [ed.Symmetry_Operation(i, p, perm_phases=e) for i, (p, e) in enumerate(zip(perms, phases))]
        G = ed.Finite_Symmetry_Group("custom", ops)
        stats = ed.Particle_Statistics.FERMIONIC if fermion else ed.Particle_Statistics.BOSONIC
        cat = ed.build_symmetry_orbit_catalog(second_quantized_model=_Model(n), n_filled=k,
                                              symmetry_group=G, particle_statistics=stats)
        perm0 = np.array([[p - 1 for p in q] for q in perms], dtype=np.uint8)
        ref = port.catalog(n, k, perm0, np.array(phases, dtype=np.complex128), fermion)
        np.testing.assert_array_equal(np.array(cat.representative_mask_list, dtype=np.uint64), ref["reprs"])
        np.testing.assert_array_equal(cat.rep_rank_table, ref["rep_rank"])
        np.testing.assert_array_equal(cat.rep_sym_table, ref["rep_sym"])
        assert_amplitudes(cat.rep_amp_table, ref["rep_amp"])


def test_large_site_count_rank():
    """48 sites (beyond the reference's 42-site rank limit): the catalog is a
    partition of all C(48, 2) states under the 24-element translation group."""
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models

    p = dict(models.params_Sun_Gu_Katsura_Sarma)
    m = models.build_zero_flux_fermionic_fci_second_quantized_model(sample_size=[4, 6], params=p)
    G = ed.build_translation_group(m.lattice)
    cat = ed.build_symmetry_orbit_catalog(second_quantized_model=m, n_filled=2, symmetry_group=G,
                                          particle_statistics=m.particle_statistics)
    rr = cat.rep_rank_table
    assert rr.min() == 0 and rr.max() == cat.n_orbits - 1
    counts = np.bincount(rr, minlength=cat.n_orbits)
    np.testing.assert_array_equal(counts, 24 // np.array(cat.stabilizer_order_list))


def test_maximum_site_count():
    """63 sites, the most a 64-bit mask holds (the reference's limit is the
    same, n_site <= 63): fillings 2 and 61 under the cyclic group of order 7
    generated by a shift of 9 sites, with random phases, for both statistics.
    Every table entry equals the oracle's."""
    import realspace_exatdiagonalization_py_b200 as ed
    from oracle import port

    n = 63
    gen = (np.arange(n) + 9) % n
    perms0 = [np.arange(n)]
    while not np.array_equal(gen[perms0[-1]], perms0[0]):
        perms0.append(gen[perms0[-1]])
    assert len(perms0) == 7
    rng = np.random.default_rng(3)
    phases = [np.ones(n)] + [np.exp(2j * np.pi * rng.random(n)) for _ in range(len(perms0) - 1)]
    ops = [ed.Symmetry_Operation(i, list(p + 1), perm_phases=e) for i, (p, e) in enumerate(zip(perms0, phases))]
    G = ed.Finite_Symmetry_Group("shift9", ops)
    perm0 = np.array(perms0, dtype=np.uint8)
    for k, fermion in [(2, True), (61, False), (61, True)]:
        stats = ed.Particle_Statistics.FERMIONIC if fermion else ed.Particle_Statistics.BOSONIC
        cat = ed.build_symmetry_orbit_catalog(second_quantized_model=_Model(n), n_filled=k,
                                              symmetry_group=G, particle_statistics=stats)
        ref = port.catalog(n, k, perm0, np.array(phases, dtype=np.complex128), fermion)
        assert cat.n_orbits == len(ref["reprs"]) == 279
        np.testing.assert_array_equal(np.array(cat.representative_mask_list, dtype=np.uint64), ref["reprs"])
        np.testing.assert_array_equal(cat.rep_rank_table, ref["rep_rank"])
        np.testing.assert_array_equal(cat.rep_sym_table, ref["rep_sym"])
        assert_amplitudes(cat.rep_amp_table, ref["rep_amp"])
