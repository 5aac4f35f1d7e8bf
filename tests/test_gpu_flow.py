"""Flux spectrum flow (observables/spectrum_flow.py:25-169) against the
reference's own driver (tests/golden/make_flow_golden.py), through the
checkpointed flux scan and through the request server."""

import os
from fractions import Fraction

import numpy as np
import pytest

from _cases import model_for

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(__file__)


@pytest.mark.parametrize("engine", ["scan", "served"])
def test_flux_spectrum_flow_matches_reference(tmp_path, engine):
    import realspace_exatdiagonalization_py_b200 as ed

    f = np.load(os.path.join(HERE, "golden", "flow_haldane12.npz"))
    labels = [tuple(int(x) for x in lab) for lab in f["labels"]]
    thetas = [float(t) for t in f["thetas"]]
    model = model_for("haldane12")
    res = ed.flux_spectrum_flow(model, labels, filling_fraction=Fraction(3, 12), flux_direction=1,
                                twisted_phases_over_2π_list=thetas, checkpoint_dir=str(tmp_path), nev=3,
                                engine=engine)
    assert res.energies.shape == f["energies"].shape and res.sector_labels == labels
    np.testing.assert_allclose(res.energies, f["energies"], atol=1e-9, rtol=0)
    if engine == "scan":
        assert len(res.checkpoint_paths) == len(thetas) and all(os.path.isfile(p) for p in res.checkpoint_paths)
        stamp = [os.path.getmtime(p) for p in res.checkpoint_paths]
        again = ed.flux_spectrum_flow(model, labels, filling_fraction=Fraction(3, 12), flux_direction=1,
                                      twisted_phases_over_2π_list=thetas, checkpoint_dir=str(tmp_path), nev=3)
        assert [os.path.getmtime(p) for p in again.checkpoint_paths] == stamp  # reused, not recomputed
        np.testing.assert_array_equal(again.energies, res.energies)
    else:
        # the served results are the scan engine's checkpoints: a scan run reads them, recomputes nothing
        assert len(res.checkpoint_paths) == len(thetas) and all(os.path.isfile(p) for p in res.checkpoint_paths)
        stamp = [os.path.getmtime(p) for p in res.checkpoint_paths]
        scan = ed.flux_spectrum_flow(model, labels, filling_fraction=Fraction(3, 12), flux_direction=1,
                                     twisted_phases_over_2π_list=thetas, checkpoint_dir=str(tmp_path), nev=3)
        assert scan.checkpoint_paths == res.checkpoint_paths
        assert [os.path.getmtime(p) for p in res.checkpoint_paths] == stamp
        np.testing.assert_array_equal(scan.energies, res.energies)
