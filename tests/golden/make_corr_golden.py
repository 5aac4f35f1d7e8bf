"""Generate tests/golden/corr_*.npz: the reference's correlators of one
sector eigenstate -- ``off_diagonal_long_range_order`` and
``compute_odlro_map`` (observables/off_diagonal_long_range_order.py:43-197),
``_build_density_correlation_matrix``, ``static_structure_factor`` and
``compute_structure_factor_map`` (observables/static_structure_factor.py) --
run through ``oracle/ref_shim.py``.  The reference imports the momentum mesh
from its ``tightbinding_py`` dependency, which the shim supplies from this
repository's restatement (``lattice.initialize_uniform_grids_from_lattice``).
Runs only where the reference checkout is present:

    python tests/golden/make_corr_golden.py

Cases (model, particles, sector, 1-based level, flavour filter a):

* haldane12: 2x3 Haldane bosons, 3 bosons, (0,0), 1, all sites
* checkerboard12: 2x3 checkerboard fermions, 2 fermions, (1,1), 2, odd sites
* haldane12_identity: 2x3 Haldane bosons, 3 bosons, "identity", 1, all sites
* haldane16: 2x4 Haldane bosons, 4 bosons, (0,1), 1, all sites

Stored per case: the ODLRO matrix, the connected correlation matrix C and the
densities, S(q) on the mesh and both 5 x 5 maps.

corr_manifold_haldane12.npz: the manifold functions on the 2x3 Haldane bosons
for the states ((0,0), 1), ((1,0), 1) -- static_structure_factor_manifold_average
(uniform and 2:1 weights), structure_factor_manifold_allowed_momenta,
compute_structure_factor_manifold_average_map (5 x 5),
structure_factor_allowed_momenta of ((0,0), 1) and the first-Brillouin-zone
polygon.
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

CASES = {
    "haldane12": ("bosonic", [2, 3], 3, (0, 0), 1, "all"),
    "checkerboard12": ("fermionic", [2, 3], 2, (1, 1), 2, "odd"),
    "haldane12_identity": ("bosonic", [2, 3], 3, "identity", 1, "all"),
    "haldane16": ("bosonic", [2, 4], 4, (0, 1), 1, "all"),
}


def flavor(name):
    return (lambda i: True) if name == "all" else (lambda i: i % 2 == 1)


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
    ssf = importlib.import_module(pkg + ".observables.static_structure_factor")
    odl = importlib.import_module(pkg + ".observables.off_diagonal_long_range_order")
    for name, (kind, sample, npart, label, level, fl) in CASES.items():
        with contextlib.redirect_stdout(io.StringIO()):
            model = build_model(R, kind, sample)
            ff = Fraction(npart, model.lattice.n_site)
            n = model.lattice.n_site
            ed_data, basis, c = ssf._bootstrap_ed_sector(model, label, ff, level, "matrix", None)
            rho = odl.off_diagonal_long_range_order(model, label, target_eigval_idx=level, filling_fraction=ff,
                                                    ed_data=ed_data)
            C = np.zeros((n, n))
            da, db = np.zeros(n), np.zeros(n)
            ssf._build_density_correlation_matrix(C, da, db, c, basis, n, flavor(fl), lambda i: True,
                                                  model.particle_statistics)
            q, S = ssf.static_structure_factor(model, label, target_eigval_idx=level, filling_fraction=ff,
                                               flavor_a=flavor(fl), ed_data=ed_data)
            kx, ky, Smap = ssf.compute_structure_factor_map(model, label, target_eigval_idx=level,
                                                            filling_fraction=ff, flavor_a=flavor(fl),
                                                            k_resolution=5, ed_data=ed_data)
            _, _, rmap = odl.compute_odlro_map(model, label, target_eigval_idx=level, filling_fraction=ff,
                                               k_resolution=5, ed_data=ed_data)
        out = dict(kind=np.array(kind), sample=np.array(sample), n_particles=np.int64(npart),
                   label=np.array("identity") if label == "identity" else np.array(label, dtype=np.int64),
                   level=np.int64(level), flavor_a=np.array(fl), odlro=rho, C=C, density_a=da, density_b=db,
                   q_points=np.array(q), S_q=S, S_map=Smap, odlro_map=rmap)
        path = os.path.join(HERE, f"corr_{name}.npz")
        np.savez_compressed(path, **out)
        print(f"corr_{name}: trace rho = {np.trace(rho).real:.6f}, max S = {S.max():.6f} -> {os.path.getsize(path)} B")


def manifold_case(R, ssf):
    with contextlib.redirect_stdout(io.StringIO()):
        model = build_model(R, "bosonic", [2, 3])
        ff = Fraction(3, 12)
        states = [((0, 0), 1), ((1, 0), 1)]
        q, S_u = ssf.static_structure_factor_manifold_average(model, states, filling_fraction=ff)
        _, S_w = ssf.static_structure_factor_manifold_average(model, states, weights=[2.0, 1.0], filling_fraction=ff)
        mx, my, mS = ssf.structure_factor_manifold_allowed_momenta(model, states, filling_fraction=ff)
        _, _, mmap = ssf.compute_structure_factor_manifold_average_map(model, states, filling_fraction=ff,
                                                                      k_resolution=5)
        ax, ay, aS = ssf.structure_factor_allowed_momenta(model, (0, 0), filling_fraction=ff)
        poly = ssf._first_bz_polygon(model.lattice)
    out = dict(q_points=np.array(q), S_uniform=S_u, S_weighted=S_w, manifold_qx=np.array(mx),
               manifold_qy=np.array(my), manifold_S=mS, manifold_map=mmap, allowed_qx=np.array(ax),
               allowed_qy=np.array(ay), allowed_S=aS, bz_polygon=np.array([np.asarray(p) for p in poly]))
    path = os.path.join(HERE, "corr_manifold_haldane12.npz")
    np.savez_compressed(path, **out)
    print(f"corr_manifold_haldane12: {len(poly)}-gon zone -> {os.path.getsize(path)} B")


if __name__ == "__main__":
    main()
    _R = ref_shim.load()
    manifold_case(_R, importlib.import_module(ref_shim.PKG + ".observables.static_structure_factor"))
