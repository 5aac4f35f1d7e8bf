"""Generate tests/golden/chern_*.npz: the reference's ``many_body_chern_number``
(observables/many_body_chern_number.py:341-458) on small models, run through
``oracle/ref_shim.py`` with its checkpoints in a temporary directory.  Runs
only where the reference checkout is present:

    python tests/golden/make_chern_golden.py

Cases (model, particles, sector labels, levels per sector, flux grid):

* haldane12: 2x3 Haldane bosons, 3 bosons, sectors (0,0),(1,0), 1, 3x3
* haldane16: 2x4 Haldane bosons, 4 bosons, sector (0,0), 2, 4x4
* haldane16_singular: the same on a 2x3 grid, where two links are
  near-singular (the reference's warning path, link replaced by 1)
* checkerboard12: 2x3 checkerboard fermions, 2 fermions, sector (1,1), 1, 3x3
* haldane12_identity: 2x3 Haldane bosons, 3 bosons, "identity", 2, 4x3

Stored per case: the inputs, ``chern_number``, ``berry_curvature``,
``link_det_abs_x/y``, ``min_link_det``, the energies as ``[nx, ny, n]`` and the
checkpoint file names of two flux points.
"""

from __future__ import annotations

import contextlib
import importlib
import io
import os
import sys
import tempfile
import types
import warnings
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref_shim  # noqa: E402

CASES = {
    "haldane12": ("bosonic", [2, 3], 3, [(0, 0), (1, 0)], 1, (3, 3)),
    "haldane16": ("bosonic", [2, 4], 4, [(0, 0)], 2, (4, 4)),
    "haldane16_singular": ("bosonic", [2, 4], 4, [(0, 0)], 2, (2, 3)),
    "checkerboard12": ("fermionic", [2, 3], 2, [(1, 1)], 1, (3, 3)),
    "haldane12_identity": ("bosonic", [2, 3], 3, "identity", 2, (4, 3)),
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
    mbc = importlib.import_module(pkg + ".observables.many_body_chern_number")
    for name, (kind, sample, n_part, labels, nev, grid) in CASES.items():
        with contextlib.redirect_stdout(io.StringIO()):
            model = build_model(R, kind, sample)
        ff = Fraction(n_part, model.lattice.n_site)
        with tempfile.TemporaryDirectory() as d, contextlib.redirect_stdout(io.StringIO()), \
                warnings.catch_warnings(record=True) as caught:
            warnings.simplefilter("always")
            res = mbc.many_body_chern_number(model, labels, filling_fraction=ff, flux_grid_size=grid,
                                             nev_per_sector=nev, checkpoint_dir=d)
        n_warn = sum("Near-singular Berry link" in str(w.message) for w in caught)
        nx, ny = res.flux_grid_size
        energies = np.array([[res.energies[ix][iy] for iy in range(ny)] for ix in range(nx)])
        out = dict(kind=np.array(kind), sample=np.array(sample), n_particles=np.int64(n_part),
                   labels=np.array("identity") if labels == "identity" else np.array(labels, dtype=np.int64),
                   nev=np.int64(nev), grid=np.array(grid, dtype=np.int64), chern_number=np.float64(res.chern_number),
                   rounded_chern=np.int64(res.rounded_chern), berry_curvature=res.berry_curvature,
                   link_det_abs_x=res.link_det_abs_x, link_det_abs_y=res.link_det_abs_y,
                   min_link_det=np.float64(res.min_link_det), energies=energies, n_singular_warnings=np.int64(n_warn),
                   checkpoint_00=np.array(os.path.basename(res.checkpoint_paths[0][0])),
                   checkpoint_11=np.array(os.path.basename(res.checkpoint_paths[1][1])))
        path = os.path.join(HERE, f"chern_{name}.npz")
        np.savez_compressed(path, **out)
        print(f"chern_{name}: C={res.chern_number:.10f} min|det|={res.min_link_det:.3e} "
              f"warnings={n_warn} -> {os.path.getsize(path)} B")


if __name__ == "__main__":
    main()
