"""Known answers at full size from the reference's own benchmark results
(tests/golden/make_benchmark_golden.py): for Heisenberg chains N = 18..28,
Haldane bosons 2x3..4x4 (the 32-site, 657,756-orbit lattice of the flux-grid
workload) and spinful Hubbard 2x2..2x7 (up to 2,865,228 rows), the full
dimension, orbit count, group order, sector-0 dimension and the lowest
sector-0 energy of the device solver equal the reference's."""

import os
from fractions import Fraction

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)
F = dict(np.load(os.path.join(HERE, "golden", "reference_benchmark.npz")))


def build_model(model: str, label: str, n_site: int):
    from realspace_exatdiagonalization_py_b200 import models

    if model == "Heisenberg":
        return models.build_heisenberg_second_quantized_model(n_site, 1.0)
    ss = [int(x) for x in label.split("×")]
    if model == "Haldane_Boson":
        return models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=ss, params=models.params_DNSheng)
    return models.build_spinful_hubbard_second_quantized_model(ss, 1.0, 8.0)


@pytest.mark.parametrize("i", range(len(F["model"])), ids=[f"{m}-{l}" for m, l in zip(F["model"], F["label"])])
def test_reference_benchmark_known_answer(i):
    import realspace_exatdiagonalization_py_b200 as ed

    model, label = str(F["model"][i]), str(F["label"][i])
    n_site, n_filled = int(F["n_site"][i]), int(F["n_filled"][i])
    m = build_model(model, label, n_site)
    assert m.lattice.n_site == n_site
    G = ed.build_translation_group(m.lattice)
    assert len(G.operations) == int(F["n_group"][i])
    data = ed.build_ed_data(m, filling_fraction=Fraction(n_filled, n_site), symmetry_group=G)
    assert data.orbit_catalog.n_states == int(F["full_dim"][i])
    assert data.orbit_catalog.n_orbits == int(F["n_orbits"][i])
    res = ed.solve_sectors_batched(data, [0], nev=1, precision=64, return_vectors=False)
    assert data.sector_dims[0] == int(F["sector_dim"][i])
    assert abs(float(res[0][0][0]) - float(F["energy"][i])) < 1e-9
