"""Generate tests/golden/pump_*.npz: the reference's ``flux_charge_pump``
(observables/charge_pump.py:325-558) on small models, run through
``oracle/ref_shim.py`` with its flux-scan checkpoints in a temporary
directory.  Runs only where the reference checkout is present:

    python tests/golden/make_pump_golden.py

Cases:

* haldane12: 2x3 Haldane bosons, 3 bosons, sectors (0,0),(1,0), one level
  each, flux along 1, five flux values
* checkerboard12: 2x3 checkerboard fermions, 2 fermions, sectors (0,0),
  (0,2), (0,1) (the position operator along 2 moves k2 by 2, so it couples
  the three), one level each, flux along 1 (polarization along 2, length 3),
  no sub-lattice offset
* haldane16: 2x4 Haldane bosons, 4 bosons, explicit manifold states
  ((0,0), 1) and ((0,0), 2), flux along 1, four flux values

Stored per case: the inputs, ``polarization_eigenvalues``, ``polarizations``,
``pumped_charges`` and ``energies``.
"""

from __future__ import annotations

import contextlib
import importlib
import io
import os
import sys
import tempfile
import types
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref_shim  # noqa: E402

CASES = {
    "haldane12": dict(kind="bosonic", sample=[2, 3], n=3, labels=[(0, 0), (1, 0)], nev=1, flux_direction=1,
                      thetas=[0.0, 0.25, 0.5, 0.75, 1.0], include_sublattice=True, states=None),
    "checkerboard12": dict(kind="fermionic", sample=[2, 3], n=2, labels=[(0, 0), (0, 2), (0, 1)], nev=1, flux_direction=1,
                           thetas=[0.0, 1 / 3, 2 / 3, 1.0], include_sublattice=False, states=None),
    "haldane16": dict(kind="bosonic", sample=[2, 4], n=4, labels=[(0, 0)], nev=1, flux_direction=1,
                      thetas=[0.0, 0.3, 0.6, 1.0], include_sublattice=True, states=[((0, 0), 1), ((0, 0), 2)]),
}


def build_model(R, kind, sample):
    if kind == "bosonic":
        return R.bosonic.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=sample,
                                                                            params=R.bosonic.params_DNSheng)
    return R.fermionic.build_zero_flux_fermionic_fci_second_quantized_model(
        sample_size=sample, params=dict(R.fermionic.params_Sun_Gu_Katsura_Sarma))


def main():
    R = ref_shim.load()
    pkg = ref_shim.PKG
    if pkg + ".observables" not in sys.modules:
        obs = types.ModuleType(pkg + ".observables")
        obs.__path__ = [os.path.join(ref_shim.package_dir(), "observables")]
        sys.modules[pkg + ".observables"] = obs
    cp = importlib.import_module(pkg + ".observables.charge_pump")
    for name, c in CASES.items():
        with contextlib.redirect_stdout(io.StringIO()):
            model = build_model(R, c["kind"], c["sample"])
        ff = Fraction(c["n"], model.lattice.n_site)
        with tempfile.TemporaryDirectory() as d, contextlib.redirect_stdout(io.StringIO()):
            res = cp.flux_charge_pump(model, c["labels"], filling_fraction=ff, flux_direction=c["flux_direction"],
                                      twisted_phases_over_2π_list=c["thetas"], nev_per_sector=c["nev"],
                                      manifold_states=c["states"], include_sublattice=c["include_sublattice"],
                                      checkpoint_dir=d)
        out = dict(kind=np.array(c["kind"]), sample=np.array(c["sample"]), n_particles=np.int64(c["n"]),
                   labels=np.array(c["labels"], dtype=np.int64), nev=np.int64(c["nev"]),
                   flux_direction=np.int64(c["flux_direction"]), thetas=np.array(c["thetas"]),
                   include_sublattice=np.bool_(c["include_sublattice"]),
                   states=np.array([[*s, lev] for s, lev in c["states"]], dtype=np.int64) if c["states"] else
                   np.zeros((0, 3), dtype=np.int64),
                   polarization_direction=np.int64(res.polarization_direction),
                   polarization_eigenvalues=res.polarization_eigenvalues, polarizations=res.polarizations,
                   pumped_charges=res.pumped_charges, energies=res.energies)
        path = os.path.join(HERE, f"pump_{name}.npz")
        np.savez_compressed(path, **out)
        print(f"pump_{name}: pumped {np.round(res.pumped_charges, 6)} -> {os.path.getsize(path)} B")


if __name__ == "__main__":
    main()
