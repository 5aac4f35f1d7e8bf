"""CPU tests: model builders, groups/irreps, the scalar mask API, the C ABI
symbol table.  No GPU needed."""

import math
import os
import re
from collections import Counter
from fractions import Fraction

import numpy as np
import pytest

import realspace_exatdiagonalization_py_b200 as ed
from realspace_exatdiagonalization_py_b200 import _lib, lattice, models
from realspace_exatdiagonalization_py_b200.symmetry import (
    _binom_table,
    _gosper_next,
    rank_combination,
    unrank_combination,
)

from oracle import ref_shim

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


def _multiset(terms, digits=14):
    return Counter((int(i), int(j), round(complex(t).real, digits), round(complex(t).imag, digits))
                   for (i, j, t) in terms)


def _golden_terms(g, key):
    return [(int(i), int(j), t) for (i, j), t in zip(g[key + "_ij"], g[key + "_t" if key == "bil" else key + "_v"])]


# ---- model builders reproduce the reference's term lists --------------------

def _model_for(case):
    if case == "heisenberg16":
        return models.build_heisenberg_second_quantized_model(16, 1.0)
    if case == "checkerboard24":
        p = dict(models.params_Sun_Gu_Katsura_Sarma)
        p.update({"V1": 1.0, "V2": 0.0, "V3": 0.0})
        return models.build_zero_flux_fermionic_fci_second_quantized_model(sample_size=[3, 4], params=p)
    if case.startswith("haldane12"):
        return models.build_zero_flux_bosonic_fci_second_quantized_model(
            sample_size=[2, 3], params=models.params_DNSheng)
    if case == "checkerboard12_flux":
        return models.build_zero_flux_fermionic_fci_second_quantized_model(
            sample_size=[2, 3], params=models.params_Sun_Gu_Katsura_Sarma)
    if case == "haldane24_flux":
        p = {"t": 1.0, "t'": 0.6, "t''": 0.0, "phi_over_2pi": 0.2, "V1": 1.0, "V2": 0.0}
        return models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[3, 4], params=p)
    if case == "hubbard12":
        return models.build_spinful_hubbard_second_quantized_model([2, 3], 1.0, 4.0)
    raise KeyError(case)


@pytest.mark.parametrize("case", ["heisenberg16", "checkerboard24", "haldane12", "haldane12_flux",
                                  "checkerboard12_flux", "haldane24_flux", "hubbard12"])
def test_model_terms_match_reference(golden, case):
    g = golden(case)
    m = _model_for(case)
    theta = list(g["theta"])
    if any(theta):
        ed.update_second_quantized_model_with_twisted_phases(m, twisted_phases_over_2π=theta)
    assert _multiset(m.bilinear_terms) == _multiset(_golden_terms(g, "bil"))
    assert _multiset(m.density_density_terms) == _multiset(_golden_terms(g, "den"))
    # group arrays and characters bit for bit
    G = ed.build_translation_group(m.lattice, theta if any(theta) else None)
    np.testing.assert_array_equal(np.array([op.perm for op in G.operations]), g["perm"])
    np.testing.assert_array_equal(np.array([op.perm_phases for op in G.operations]), g["eta"])
    irreps = ed.build_irrep_list(G, m.lattice)
    np.testing.assert_array_equal(np.array([ir.values for ir in irreps]), g["chi"])


def test_term_counts_of_reference_tests():
    # test/test_core.py:106-140 of the reference
    m = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[2, 3],
                                                                  params=models.params_DNSheng)
    assert m.lattice.n_site == 12 and len(m.bilinear_terms) == 144
    summed = {}
    for (i, j, t) in m.bilinear_terms:
        summed[(i, j)] = summed.get((i, j), 0j) + t
    for (i, j), t in summed.items():
        assert abs(t - np.conj(summed.get((j, i), 0j))) < 1e-12
    c = models.build_zero_flux_fermionic_fci_second_quantized_model(
        sample_size=[3, 4], params=models.params_Sun_Gu_Katsura_Sarma)
    assert c.lattice.n_site == 24 and len(c.density_density_terms) == 96
    assert c.particle_statistics is ed.Particle_Statistics.FERMIONIC
    h = models.build_spinful_hubbard_second_quantized_model([2, 2])
    assert h.lattice.n_site == 8 and len(h.density_density_terms) == 4
    s = models.build_heisenberg_second_quantized_model(8, J=1.0)
    assert s.lattice.n_site == 8 and s.particle_statistics is ed.Particle_Statistics.BOSONIC


# ---- scalar API known answers (reference test/test_core.py:54-87) ----------

def test_boson_permutation_action():
    op = ed.Symmetry_Operation("t", [2, 3, 1])
    m, ph = ed.apply_operation_to_mask(0b101, op, ed.Particle_Statistics.BOSONIC)
    assert m == 0b011 and abs(ph - 1.0) == 0.0


def test_fermion_permutation_sign():
    op = ed.Symmetry_Operation("id", [1, 2, 3])
    _, ph = ed.apply_operation_to_mask(0b001, op, ed.Particle_Statistics.FERMIONIC)
    assert ph == 1.0 + 0.0j
    swap = ed.Symmetry_Operation("swap", [2, 1, 3])
    _, ph = ed.apply_operation_to_mask(0b011, swap, ed.Particle_Statistics.FERMIONIC)
    assert ph == -1.0 + 0.0j


def test_canonical_representative():
    ops = [ed.Symmetry_Operation("id", [1, 2, 3, 4]), ed.Symmetry_Operation("T", [4, 1, 2, 3])]
    G = ed.Finite_Symmetry_Group("cyclic", ops, identity_idx=0)
    rep, g, _ = ed.get_canonical_representative(0b1000, G, ed.Particle_Statistics.BOSONIC)
    assert rep == 0b0100 and g == 1


def test_translation_group_structure():
    lat = lattice.initialize_real_space_lattice(sample_size=[2, 3], lattice_name="honeycomb",
                                                pbc_indicator=[True, True])
    G = ed.build_translation_group(lat)
    assert len(G.operations) == 6 and G.operations[0].label == (0, 0)
    irreps = ed.build_translation_irrep_list(G, lat)
    assert len(irreps) == 6 and irreps[0].label == (0, 0)


def test_group_validation_errors():
    with pytest.raises(ValueError):
        ed.Finite_Symmetry_Group("empty", [])
    with pytest.raises(ValueError):
        ed.Finite_Symmetry_Group("bad", [ed.Symmetry_Operation("x", [2, 1])])
    lat = lattice.initialize_real_space_lattice(sample_size=[2, 3])
    with pytest.raises(ValueError):
        ed.build_translation_group(lat, [0.1])
    G = ed.build_translation_group(lat)
    G.name = "other"
    with pytest.raises(ValueError):
        ed.build_irrep_list(G, lat)


def test_rank_unrank_gosper():
    n, k = 12, 5
    bt = _binom_table(n, k)
    m = (1 << k) - 1
    for r in range(math.comb(n, k)):
        assert rank_combination(m, bt) == r
        assert unrank_combination(r, n, k, bt) == m
        m = _gosper_next(m)


def test_hopping_phase():
    F = ed.Particle_Statistics.FERMIONIC
    assert ed.hopping_phase_for_stats(F, 0b0100, 1, 4) == -1
    assert ed.hopping_phase_for_stats(F, 0b0110, 1, 4) == 1
    assert ed.hopping_phase_for_stats(ed.Particle_Statistics.BOSONIC, 0b0100, 1, 4) == 1


def test_filling_assertion_without_gpu():
    m = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[2, 3],
                                                                  params=models.params_DNSheng)
    G = ed.build_translation_group(m.lattice)
    with pytest.raises(AssertionError):
        ed.build_ed_data(m, filling_fraction=Fraction(1, 5), symmetry_group=G)


def test_term_merging_and_on_site_rejection():
    from realspace_exatdiagonalization_py_b200.hamiltonian import _merge_terms

    begin, to, amp, jw = _merge_terms([(1, 3, 1.0), (1, 3, 0.5j), (3, 1, 2.0), (2, 1, 1.0)], 4)
    assert list(begin) == [0, 1, 2, 3, 3]
    assert list(to) == [2, 0, 0] and amp[0] == 1.0 + 0.5j
    assert int(jw[0]) == 0b10  # site 2 lies between sites 1 and 3
    with pytest.raises(ValueError):
        _merge_terms([(2, 2, 1.0)], 4)


# ---- the C ABI --------------------------------------------------------------

def _declared_symbols():
    text = open(os.path.join(ROOT, "include", "rsed.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(rsed_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    names = _declared_symbols()
    assert len(names) >= 25
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)
    assert lib.rsed_version().startswith(b"rsed-b200")


def test_library_rejects_bad_arguments_without_gpu():
    lib = _lib.load()
    # descriptor checks run before any CUDA call
    grp = _lib.RsedGroup(70, 3, 4, 0, 10, None, None, None, None)
    import ctypes

    n = ctypes.c_int64(0)
    rc = lib.rsed_catalog_count(ctypes.byref(grp), None, 0, ctypes.byref(n), None)
    assert rc == _lib.RSED_ERANGE
    assert b"n_site" in lib.rsed_last_error()
    with pytest.raises(ValueError):
        _lib.check(rc)
    # block gather and scatter validate their shapes before any CUDA call
    assert lib.rsed_gather_block(4, None, None, 2, 8, None, 2, None) == _lib.RSED_EINVAL
    assert lib.rsed_scatter_block(4, None, None, 3, 2, None, 8, 0, None) == _lib.RSED_EINVAL


def test_vectors_to_host_single_copy_layout():
    """Consecutive row-major views of one buffer come back as one host copy,
    split in order; any other list is copied block by block."""
    import torch

    from realspace_exatdiagonalization_py_b200.lanczos import vectors_to_host

    flat = torch.arange(30, dtype=torch.float64).to(torch.complex128)
    for vs in ([flat[0:12].view(4, 3), flat[12:30].view(6, 3)],
               [flat[12:30].view(6, 3), flat[0:12].view(4, 3)],
               [torch.ones(3, 2, dtype=torch.complex128).t(), torch.zeros(2, 2, dtype=torch.complex128)]):
        hs = vectors_to_host(vs)
        assert [h.shape for h in hs] == [tuple(v.shape) for v in vs]
        for h, v in zip(hs, vs):
            np.testing.assert_array_equal(h, v.numpy())
    assert vectors_to_host([]) == []


def test_periodic_check_schedule():
    """The O(1) test for a periodic Ritz check inside a span of steps agrees
    with stepping through the span (the state's count is i + 1 after step i)."""
    from types import SimpleNamespace

    from realspace_exatdiagonalization_py_b200.lanczos import LanczosBatch

    for ce in range(1, 25):
        stub = SimpleNamespace(p=SimpleNamespace(check_every=ce))
        for first in range(0, 50):
            for last in range(first - 2, first + 30):
                want = any((i + 1) % ce == 0 for i in range(first, last + 1))
                assert LanczosBatch.periodic_check_in(stub, first, last) == want


# Names of the reference's top-level API that this package does not provide,
# each outside the hot path: plotting (matplotlib figures), entanglement
# spectra and the full-ED density distribution (post-processing observables),
# and the model modules' figure-writing example drivers.
OUT_OF_SCOPE_EXPORTS = {
    "plot_ed_scan_res", "plot_spectrum", "plot_entanglement_spectrum", "plot_odlro_map", "plot_odlro_map_panels",
    "plot_particle_entanglement_spectrum", "plot_structure_factor_allowed_momenta",
    "plot_structure_factor_allowed_momenta_panels", "plot_structure_factor_map", "plot_structure_factor_map_panels",
    "entanglement_spectrum", "particle_entanglement_spectrum", "vertices_occupation_distribution_full_ed",
    "test_bosonic_fci_charge_pump", "test_bosonic_fci_spectrum_flow", "test_fermionic_fci_charge_pump",
    "test_fermionic_fci_full_ed", "test_fermionic_fci_spectrum_flow",
}


def test_package_exports_the_reference_api():
    """Every name the reference re-exports at top level is importable from
    this package, except the explicit out-of-scope list above."""
    import json

    import realspace_exatdiagonalization_py_b200 as pkg

    names = json.load(open(os.path.join(GOLDEN, "reference_exports.json")))["names"]
    missing = sorted(n for n in names if n not in OUT_OF_SCOPE_EXPORTS and not hasattr(pkg, n))
    assert not missing, missing
    assert OUT_OF_SCOPE_EXPORTS <= set(names)


def test_bit_utilities_known_answers():
    from realspace_exatdiagonalization_py_b200 import bits

    m = 0b10110
    assert list(bits.filled_site_iter_for_mask(m, 5)) == [2, 3, 5]
    assert list(bits.empty_site_iter_for_mask(m, 5)) == [1, 4]
    assert bits.decode_bit_mask_to_configuration(m, 5) == [2, 3, 5]
    assert bits.encode_configuration_to_bit_mask([2, 3, 5]) == m
    occ = [0, 0, 0]
    assert bits.decode_bit_mask_to_configuration_inplace(occ, m, 5) is occ and occ == [2, 3, 5]
    with pytest.raises(AssertionError):
        bits.decode_bit_mask_to_configuration_inplace([0, 0], m, 5)
    assert bits.bitmask_of_site(1) == 1 and bits.bitmask_of_site(63) == 1 << 62
    assert bits.occupy_site_for_mask(m, 1) == 0b10111 and bits.empty_site_for_mask(m, 2) == 0b10100
    assert bits.is_site_occupied(m, 2) and bits.is_site_empty(m, 1) and bits.n_occupied_for_mask(m) == 3
    assert bits.as_uint64_array([m, 1 << 62]).dtype == np.uint64


@pytest.mark.skipif(not ref_shim.available(), reason="reference package not present")
def test_bit_utilities_match_reference():
    import importlib

    from realspace_exatdiagonalization_py_b200 import bits

    ref_shim.load()
    rb = importlib.import_module(ref_shim.PKG + ".utils.bitwise_operations")
    rng = np.random.default_rng(5)
    for _ in range(200):
        n = int(rng.integers(1, 64))
        m = int(rng.integers(0, 1 << n, dtype=np.uint64))
        i = int(rng.integers(1, n + 1))
        for f in ("occupy_site_for_mask", "empty_site_for_mask", "is_site_occupied", "is_site_empty"):
            assert getattr(bits, f)(m, i) == getattr(rb, f)(m, i), f
        assert bits.n_occupied_for_mask(m) == rb.n_occupied_for_mask(m)
        assert list(bits.filled_site_iter_for_mask(m, n)) == list(rb.filled_site_iter_for_mask(m, n))
        assert list(bits.empty_site_iter_for_mask(m, n)) == list(rb.empty_site_iter_for_mask(m, n))
        occ = rb.decode_bit_mask_to_configuration(m, n)
        assert bits.decode_bit_mask_to_configuration(m, n) == occ
        assert bits.encode_configuration_to_bit_mask(occ) == rb.encode_configuration_to_bit_mask(occ)


def test_default_fci_sectors():
    from realspace_exatdiagonalization_py_b200 import models

    assert models.default_fci_sectors([3, 4]) == [(0, 0), (0, 2)]
    assert models.default_fci_sectors([9, 9]) == [(0, 0)]
    assert models.default_fci_sectors_fermionic([2, 3]) == [(0, 0), (0, 1), (0, 2)]
    with pytest.raises(ValueError):
        models.default_fci_sectors_fermionic([9, 9])
    tb = models.build_fermionic_checkerboard_tb_model(sample_size=[2, 3])
    assert tb.lattice.n_site == 12
    assert models.CHECKERBOARD_TPP_DENOMINATOR == pytest.approx(2 + 2 * np.sqrt(2))


@pytest.mark.skipif(not ref_shim.available(), reason="reference package not present")
def test_scalar_api_matches_reference():
    """Jordan-Wigner sign, colex rank and single-mask group actions against
    the reference's own scalar functions on random masks."""
    R = ref_shim.load()
    sre = R.sre
    rng = np.random.default_rng(11)
    for stats in (ed.Particle_Statistics.BOSONIC, ed.Particle_Statistics.FERMIONIC):
        rstats = getattr(sre.Particle_Statistics, stats.name)
        for _ in range(300):
            n = int(rng.integers(2, 40))
            m = int(rng.integers(0, 1 << n, dtype=np.uint64))
            i, j = (int(x) for x in rng.integers(1, n + 1, size=2))
            assert ed.hopping_phase_for_stats(stats, m, i, j) == sre.hopping_phase_for_stats(rstats, m, i, j)
    for _ in range(200):
        n = int(rng.integers(2, 42))
        k = int(rng.integers(1, n))
        m = sum(1 << int(s) for s in rng.choice(n, size=k, replace=False))
        bt = sre._binom_table(n, k)
        assert ed.rank_combination(m, bt) == sre.rank_combination(m, bt)


def test_lanczos_kernel_form_bits():
    """LanczosParams switches -> rsed_lanczos_t.reserved bits (the C side reads
    bit 0 single pass, bit 1 no streaming, bit 2 row-group update, bit 3
    per-instance restart)."""
    from realspace_exatdiagonalization_py_b200.lanczos import LanczosParams, reserved_bits

    assert reserved_bits(LanczosParams()) == 1 | 4  # defaults: single pass, streamed reduction, row-group update
    assert reserved_bits(LanczosParams(single_pass=False)) == 4
    assert reserved_bits(LanczosParams(stream=False)) == 1 | 2 | 4
    assert reserved_bits(LanczosParams(stream_update=True)) == 1
    assert reserved_bits(LanczosParams(row_restart=False)) == 1 | 4 | 8
