"""Generate tests/golden/flow_haldane12.npz: the reference's
``flux_spectrum_flow`` (observables/spectrum_flow.py:25-169) on the 2x3
Haldane boson model (3 bosons), two sectors, three flux values along
direction 1, nev 3, run through ``oracle/ref_shim.py`` with its checkpoints in
a temporary directory.  Runs only where the reference checkout is present:

    python tests/golden/make_flow_golden.py
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


def main():
    R = ref_shim.load()
    pkg = ref_shim.PKG
    if pkg + ".observables" not in sys.modules:
        obs = types.ModuleType(pkg + ".observables")
        obs.__path__ = [os.path.join(ref_shim.package_dir(), "observables")]
        sys.modules[pkg + ".observables"] = obs
    sf = importlib.import_module(pkg + ".observables.spectrum_flow")
    model = R.bosonic.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[2, 3],
                                                                         params=R.bosonic.params_DNSheng)
    thetas = [0.0, 0.25, 0.5]
    labels = [(0, 0), (1, 1)]
    with tempfile.TemporaryDirectory() as d, contextlib.redirect_stdout(io.StringIO()):
        res = sf.flux_spectrum_flow(model, labels, filling_fraction=Fraction(3, 12), flux_direction=1,
                                    twisted_phases_over_2π_list=thetas, checkpoint_dir=d, nev=3)
    path = os.path.join(HERE, "flow_haldane12.npz")
    np.savez_compressed(path, thetas=np.array(thetas), labels=np.array(labels), energies=res.energies,
                        flux_direction=np.int64(1), nev=np.int64(3))
    print("flow_haldane12:", res.energies.shape, os.path.getsize(path), "B")


if __name__ == "__main__":
    main()
