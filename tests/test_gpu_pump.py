"""Flux charge pump (observables/charge_pump.py:325-558) on the device against
the reference's own driver (tests/golden/make_pump_golden.py), and the device
position-operator products against the oracle's element formula."""

import os
from fractions import Fraction

import numpy as np
import pytest

from _cases import PUMP_CASES, pump_case, pump_specs
from oracle import port

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("case", PUMP_CASES)
def test_charge_pump_matches_reference(tmp_path, case):
    import realspace_exatdiagonalization_py_b200 as ed

    model, f = pump_case(case)
    labels = [tuple(int(x) for x in lab) for lab in f["labels"]]
    states = [((int(a), int(b)), int(lev)) for a, b, lev in f["states"]] or None
    kw = dict(filling_fraction=Fraction(int(f["n_particles"]), model.lattice.n_site),
              flux_direction=int(f["flux_direction"]), twisted_phases_over_2π_list=[float(t) for t in f["thetas"]],
              nev_per_sector=int(f["nev"]), manifold_states=states,
              include_sublattice=bool(f["include_sublattice"]), checkpoint_dir=str(tmp_path))
    res = ed.flux_charge_pump(model, labels, **kw)
    assert res.polarization_direction == int(f["polarization_direction"])
    np.testing.assert_allclose(res.energies, f["energies"], atol=1e-9, rtol=0)
    np.testing.assert_allclose(res.polarization_eigenvalues, f["polarization_eigenvalues"], atol=1e-8, rtol=0)
    np.testing.assert_allclose(res.polarizations, f["polarizations"], atol=1e-8, rtol=0)
    np.testing.assert_allclose(res.pumped_charges, f["pumped_charges"], atol=1e-8, rtol=0)
    assert [(s.sector, s.level) for s in res.manifold_states] == pump_specs(f)
    assert all(os.path.isfile(p) for p in res.checkpoint_paths)
    # the flux-scan checkpoints are reused (shared with flux_spectrum_flow)
    stamp = [os.path.getmtime(p) for p in res.checkpoint_paths]
    again = ed.flux_charge_pump(model, labels, **kw)
    assert [os.path.getmtime(p) for p in res.checkpoint_paths] == stamp
    np.testing.assert_array_equal(again.polarization_eigenvalues, res.polarization_eigenvalues)


@pytest.mark.parametrize("k_to,k_from", [(1, 1), (2, 3), (5, 2)])
def test_position_block_matches_oracle(golden, k_to, k_from):
    """Random orbit-layout vectors of two sectors of the 24-site checkerboard
    catalog: the device products equal the oracle's element formula summed on
    the host."""
    import torch

    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models
    from realspace_exatdiagonalization_py_b200.observables import _position_block

    model, nf = models.config_model("checkerboard24")
    G = ed.build_translation_group(model.lattice, [0.2, 0.0])
    data = ed.build_ed_data(model, filling_fraction=Fraction(nf, model.lattice.n_site), symmetry_group=G)
    dm, sset = data._device()
    cat = data.orbit_catalog
    n_orb = cat.n_orbits
    phases = ed.many_body_position_phases(model.lattice, 2)
    rng = np.random.default_rng(k_to * 10 + k_from)
    s_to, s_from = 0, 4
    X = []
    for s, k in ((s_to, k_to), (s_from, k_from)):
        rows = sset.rows(s)[0].long().cpu().numpy()
        x = np.zeros((k, n_orb), dtype=np.complex128)
        x[:, rows] = rng.standard_normal((k, len(rows))) + 1j * rng.standard_normal((k, len(rows)))
        X.append(x)
    chi_to, chi_from = sset.chi[s_to].contiguous(), sset.chi[s_from].contiguous()
    got = _position_block(cat, chi_to, chi_from, torch.as_tensor(X[0]).cuda(), torch.as_tensor(X[1]).cuda(),
                          torch.as_tensor(phases).cuda())
    perm0 = np.array([[p - 1 for p in op.perm] for op in G.operations], dtype=np.uint8)
    w = chi_to.cpu().numpy() * np.conj(chi_from.cpu().numpy())
    reprs = cat.repr_masks.cpu().numpy().view(np.uint64)
    both = np.nonzero((np.abs(X[0]).sum(0) > 0) & (np.abs(X[1]).sum(0) > 0))[0]
    e = np.array([port.position_element(int(reprs[o]), perm0, w, phases) for o in both])
    want = np.conj(X[0][:, both]) @ (e[:, None] * X[1][:, both].T)
    np.testing.assert_allclose(got, want, atol=1e-10 * max(1.0, np.abs(want).max()), rtol=0)
