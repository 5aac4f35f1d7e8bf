"""Two-species (fixed N_up, N_down) bases on the device against the oracle's
two-species restatement, which the CPU suite pins to the reference's total-N
spectra (union over N_down = total-N spectrum)."""

from fractions import Fraction

import numpy as np
import pytest

from oracle import port
from test_gpu_catalog import _group, _stats, assert_amplitudes

pytestmark = pytest.mark.gpu


def _down_mask(n):
    return sum(1 << i for i in range(1, n, 2))


class _Lat:
    def __init__(self, n):
        self.n_site = n


class _Model:
    def __init__(self, n):
        self.lattice = _Lat(n)


@pytest.mark.parametrize("kb", [0, 2, 3])
def test_two_species_catalog_tables(golden, kb):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden("hubbard12")
    n, k = int(g["n_site"]), int(g["n_filled"])
    sites_b = [i + 1 for i in range(1, n, 2)]
    cat = ed.build_symmetry_orbit_catalog(second_quantized_model=_Model(n), n_filled=k,
                                          symmetry_group=_group(g), particle_statistics=_stats(g),
                                          species=(sites_b, kb))
    ref = port.catalog(n, k, (g["perm"] - 1).astype(np.uint8), g["eta"], True, species=(_down_mask(n), kb))
    assert cat.n_states == len(ref["rep_rank"])
    np.testing.assert_array_equal(np.array(cat.representative_mask_list, dtype=np.uint64), ref["reprs"])
    np.testing.assert_array_equal(cat.rep_rank_table, ref["rep_rank"])
    np.testing.assert_array_equal(cat.rep_sym_table, ref["rep_sym"])
    assert_amplitudes(cat.rep_amp_table, ref["rep_amp"])
    # host rank of every basis mask addresses its own table entry
    masks = port.species_basis(n, k, (_down_mask(n), kb), ref["binom"])[2](np.arange(cat.n_states))
    for r in range(0, cat.n_states, max(1, cat.n_states // 50)):
        assert cat.rank_of(int(masks[r])) == r and cat.in_basis(int(masks[r]))


def test_two_species_rejects_mixing_group(golden):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden("hubbard12")
    n = int(g["n_site"])
    with pytest.raises(ValueError):
        ed.build_symmetry_orbit_catalog(second_quantized_model=_Model(n), n_filled=6, symmetry_group=_group(g),
                                        particle_statistics=_stats(g), species=([1, 2, 3, 4, 5, 6], 3))


def test_two_species_energies_hubbard_2x3(golden):
    """N_up = N_down = 3 sector energies through the scan API, against the
    oracle's dense per-spin spectra; the reference's total-N ground state of
    each momentum sector lies in the per-spin spectrum."""
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models

    g = golden("hubbard12")
    m = models.build_spinful_hubbard_second_quantized_model([2, 3], 1.0, 4.0)
    G = ed.build_translation_group(m.lattice)
    data = ed.build_ed_data(m, filling_fraction=Fraction(6, 12), symmetry_group=G,
                            species=models.hubbard_spin_species(m, 3))
    ed.ed_scan(data, nev=4, mode="matrixfree")
    n = int(g["n_site"])
    ref = port.catalog(n, 6, (g["perm"] - 1).astype(np.uint8), g["eta"], True, species=(_down_mask(n), 3))
    bil = [(int(i), int(j), t) for (i, j), t in zip(g["bil_ij"], g["bil_t"])]
    den = [(int(i), int(j), v) for (i, j), v in zip(g["den_ij"], g["den_v"])]
    for s in range(len(g["chi"])):
        orb = port.sector_orbits(ref, g["chi"][s])
        ev = np.linalg.eigvalsh(port.csr_block(ref, n, orb, bil, den, g["chi"][s], True).toarray())
        vals = data.ed_scan_res[s][0]
        np.testing.assert_allclose(vals, ev[:4], atol=1e-10, rtol=0)
        assert np.min(np.abs(ev - g["eig_vals"][s][0])) < 1e-9


def test_two_species_lanczos_and_projection(golden):
    """A per-spin basis large enough for the batched Lanczos path (Hubbard
    2x4, N_up = N_down = 4): batched FP32 + refinement, projection table and
    on-the-fly apply agree with the oracle."""
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models

    m = models.build_spinful_hubbard_second_quantized_model([2, 4], 1.0, 4.0)
    G = ed.build_translation_group(m.lattice)
    data = ed.build_ed_data(m, filling_fraction=Fraction(8, 16), symmetry_group=G,
                            species=models.hubbard_spin_species(m, 4))
    n = m.lattice.n_site
    perm0 = np.array([[p - 1 for p in op.perm] for op in G.operations], dtype=np.uint8)
    eta = np.array([op.perm_phases for op in G.operations], dtype=np.complex128)
    ref = port.catalog(n, 8, perm0, eta, True, species=(_down_mask(n), 4))
    np.testing.assert_array_equal(data.orbit_catalog.rep_rank_table, ref["rep_rank"])
    sectors = [s for s in range(len(data.irrep_list))]
    dims = [len(port.sector_orbits(ref, np.asarray(data.irrep_list[s].values))) for s in sectors]
    big = [s for s, d in zip(sectors, dims) if d > 500]
    assert big, dims
    res = ed.solve_sectors_batched(data, big, nev=4, precision=32)
    bil = [(int(i), int(j), complex(t)) for (i, j, t) in m.bilinear_terms]
    den = [(int(i), int(j), complex(v)) for (i, j, v) in m.density_density_terms]
    for s in big[:3]:
        chi = np.asarray(data.irrep_list[s].values)
        orb = port.sector_orbits(ref, chi)
        H = port.csr_block(ref, n, orb, bil, den, chi, True)
        ev = np.linalg.eigvalsh(H.toarray())
        np.testing.assert_allclose(res[s][0], ev[:4], atol=1e-10, rtol=0)


def test_config3_per_spin_union_is_total_n_at_gamma():
    """Hubbard 4x4 (32 spin-orbitals), U = 4, 10 electrons, momentum Gamma:
    the lowest levels of the reference's total-N sector (about 4.03M orbits)
    equal the lowest levels of the union over N_down of the per-spin sectors
    (N_up = N_down = 5: 19,079,424 states; the multiplets' other S_z
    components in N_down = 4, 6), each solved on the device, 1e-9."""
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models

    m, nf = models.config_model("hubbard32")
    G = ed.build_translation_group(m.lattice)
    total = ed.build_ed_data(m, filling_fraction=Fraction(nf, 32), symmetry_group=G)
    cfg = ed.SolverConfig((4,), 0, True, 12)
    e_total = ed.solve_sectors_batched(total, [0], nev=4, precision=64, config=cfg, return_vectors=False)[0][0]
    del total
    union = []
    for kb in (4, 5, 6):
        d = ed.build_ed_data(m, filling_fraction=Fraction(nf, 32), symmetry_group=G,
                             species=models.hubbard_spin_species(m, kb))
        if kb == 5:
            assert d.orbit_catalog.n_states == 19_079_424
        union.extend(ed.solve_sectors_batched(d, [0], nev=4, precision=64, config=cfg,
                                              return_vectors=False)[0][0].tolist())
        del d
    np.testing.assert_allclose(np.sort(union)[:4], e_total, atol=1e-9, rtol=0)
