"""Sector state -> Fock amplitudes on the device against the reference's own
function (golden vectors of tests/golden/make_fock_golden.py) and, for a
two-species basis the reference does not have, against the oracle."""

import os

import numpy as np
import pytest

from _cases import ed_data_for
from oracle import port

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)


@pytest.mark.parametrize("case", ["haldane12_flux", "checkerboard12_flux", "hubbard12"])
def test_fock_expansion_matches_reference(golden, case):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden(case)
    f = np.load(os.path.join(HERE, "golden", f"fock_{case}.npz"))
    data = ed_data_for(case, g)
    dm, sset = data._device()
    stats = data.second_quantized_model.particle_statistics
    for s in f["sectors"]:
        basis = ed.Symmetry_Sector_Basis(data.irrep_list[s], data.orbit_catalog, sset, int(s))
        amps = ed.expand_sector_state_to_fock_amplitudes(f[f"c_{s}"], basis, stats)
        keys = np.array(sorted(amps), dtype=np.uint64)
        np.testing.assert_array_equal(keys, f[f"masks_{s}"])
        np.testing.assert_allclose(np.array([amps[int(k)] for k in keys]), f[f"amps_{s}"], atol=1e-13, rtol=0)
        # device-tensor form: same content
        m, a = ed.expand_sector_state_to_fock_amplitudes(f[f"c_{s}"], basis, stats, as_dict=False)
        order = np.argsort(m.cpu().numpy().view(np.uint64))
        np.testing.assert_array_equal(m.cpu().numpy().view(np.uint64)[order], f[f"masks_{s}"])
        assert abs(np.linalg.norm(a.cpu().numpy()) - 1.0) < 1e-14


def test_fock_expansion_two_species_matches_oracle(golden):
    import realspace_exatdiagonalization_py_b200 as ed
    from fractions import Fraction

    from realspace_exatdiagonalization_py_b200 import models

    g = golden("hubbard12")
    m = models.build_spinful_hubbard_second_quantized_model([2, 3], 1.0, 4.0)
    G = ed.build_translation_group(m.lattice)
    data = ed.build_ed_data(m, filling_fraction=Fraction(6, 12), symmetry_group=G,
                            species=models.hubbard_spin_species(m, 3))
    dm, sset = data._device()
    n = m.lattice.n_site
    perm0 = (g["perm"] - 1).astype(np.uint8)
    ref = port.catalog(n, 6, perm0, g["eta"], True, species=(sum(1 << i for i in range(1, n, 2)), 3))
    for s in (0, 2):
        basis = ed.Symmetry_Sector_Basis(data.irrep_list[s], data.orbit_catalog, sset, s)
        rng = np.random.default_rng(s)
        c = rng.standard_normal(basis.dim) + 1j * rng.standard_normal(basis.dim)
        amps = ed.expand_sector_state_to_fock_amplitudes(c, basis, m.particle_statistics)
        orbits = port.sector_orbits(ref, g["chi"][s])
        want = port.fock_expand(ref, orbits, c, g["chi"][s], perm0, g["eta"], True)
        assert set(amps) == set(want)
        np.testing.assert_allclose(np.array([amps[k] for k in want]), np.array(list(want.values())), atol=1e-13,
                                   rtol=0)


def test_fock_expansion_rejects_zero_state(golden):
    import realspace_exatdiagonalization_py_b200 as ed

    g = golden("haldane12_flux")
    data = ed_data_for("haldane12_flux", g)
    dm, sset = data._device()
    basis = ed.Symmetry_Sector_Basis(data.irrep_list[0], data.orbit_catalog, sset, 0)
    with pytest.raises(ValueError):
        ed.expand_sector_state_to_fock_amplitudes(np.zeros(basis.dim), basis, None)
