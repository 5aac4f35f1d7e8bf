"""Generate tests/golden/fock_*.npz: the reference's sector-state -> Fock
amplitude expansion on seeded sector vectors.

Runs only where the reference checkout is present (the build container):

    python tests/golden/make_fock_golden.py

It loads the reference engine through ``oracle/ref_shim.py``, registers the
reference's ``observables`` package the same way (its ``__init__`` is not
executed) and calls ``_expand_sector_state_to_fock_amplitudes``
(``observables/entanglement_spectrum.py:82-145``) for two sectors of three of
the cases of ``make_golden.py``, with a complex-normal sector vector from
``numpy.random.default_rng(7 + sector)``.  Stored per case: the sectors, the
input vectors (in the reference's basis order) and the resulting masks and
amplitudes.
"""

from __future__ import annotations

import contextlib
import importlib
import io
import os
import sys
import types
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref_shim  # noqa: E402


def quiet(f, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return f(*a, **k)


def load_expand():
    R = ref_shim.load()
    pkg = ref_shim.PKG
    if pkg + ".observables" not in sys.modules:
        obs = types.ModuleType(pkg + ".observables")
        obs.__path__ = [os.path.join(ref_shim.package_dir(), "observables")]
        sys.modules[pkg + ".observables"] = obs
    es = importlib.import_module(pkg + ".observables.entanglement_spectrum")
    return R, es._expand_sector_state_to_fock_amplitudes


def make(R, expand, name, model, n_filled, theta, sectors):
    sre = R.sre
    if theta is not None:
        R.sqm.update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=theta)
    G = sre.build_translation_group(model.lattice, theta)
    data = quiet(sre.build_ed_data, model, filling_fraction=Fraction(n_filled, model.lattice.n_site),
                 symmetry_group=G)
    out = {"sectors": np.array(sectors, dtype=np.int64)}
    for s in sectors:
        basis = sre.build_symmetry_sector_basis(data.orbit_catalog, data.irrep_list[s])
        d = len(basis.representative_mask_list)
        rng = np.random.default_rng(7 + s)
        c = rng.standard_normal(d) + 1j * rng.standard_normal(d)
        c /= np.linalg.norm(c)
        amps = expand(c, basis, model.particle_statistics, atol=1e-12)
        keys = np.array(sorted(amps), dtype=np.uint64)
        out[f"c_{s}"] = c
        out[f"masks_{s}"] = keys
        out[f"amps_{s}"] = np.array([amps[int(k)] for k in keys], dtype=np.complex128)
    path = os.path.join(HERE, f"fock_{name}.npz")
    np.savez_compressed(path, **out)
    print(f"fock_{name}: sectors {sectors} -> {os.path.getsize(path)} B")


def main():
    R, expand = load_expand()
    make(R, expand, "haldane12_flux",
         R.bosonic.build_zero_flux_bosonic_fci_second_quantized_model(
             sample_size=[2, 3], params=R.bosonic.params_DNSheng), 3, [0.3, 0.1], [0, 4])
    pf = dict(R.fermionic.params_Sun_Gu_Katsura_Sarma)
    make(R, expand, "checkerboard12_flux",
         quiet(R.fermionic.build_zero_flux_fermionic_fci_second_quantized_model, sample_size=[2, 3], params=pf),
         4, [0.25, 0.4], [1, 5])
    make(R, expand, "hubbard12",
         quiet(R.hubbard.build_spinful_hubbard_second_quantized_model, [2, 3], 1.0, 4.0), 6, None, [0, 3])


if __name__ == "__main__":
    main()
