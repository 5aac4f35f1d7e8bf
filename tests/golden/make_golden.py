"""Generate the golden fixtures of tests/golden/ from the reference engine.

Runs only where the reference checkout is present (the build container):

    python tests/golden/make_golden.py

It loads the reference's own ``symmetry_resolved_ed.py`` and model builders
through ``oracle/ref_shim.py`` and stores, per case, the reference's group
arrays, term lists, orbit catalog (integer tables, complex64 amplitudes,
stabilizers), the result of ``update_orbit_stabilizer_phases``, sector
dimensions and sector eigenvalues as compressed ``.npz`` files.  The fixtures
travel with the repository; the GPU tests read them, never the reference.
"""

from __future__ import annotations

import contextlib
import io
import os
import sys
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref_shim  # noqa: E402


def quiet(f, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return f(*a, **k)


def terms_array(terms):
    return np.array([(i, j) for (i, j, _) in terms], dtype=np.int64).reshape(-1, 2), np.array(
        [complex(t) for (_, _, t) in terms], dtype=np.complex128
    )


def catalog_arrays(cat, prefix=""):
    stab_g = cat.stabilizer_g_indices_list
    off = np.cumsum([0] + [len(g) for g in stab_g]).astype(np.int64)
    return {
        prefix + "reprs": np.array(cat.representative_mask_list, dtype=np.uint64),
        prefix + "stab_off": off,
        prefix + "stab_g": np.array([g for gs in stab_g for g in gs], dtype=np.int64),
        prefix + "stab_phase": np.array(
            [p for ps in cat.stabilizer_phases_list for p in ps], dtype=np.complex128
        ),
        prefix + "rep_rank": np.asarray(cat.rep_rank_table, dtype=np.int32),
        prefix + "rep_sym": np.asarray(cat.rep_sym_table, dtype=np.int32),
        prefix + "rep_amp": np.asarray(cat.rep_amp_table, dtype=np.complex64),
    }


def group_arrays(G):
    return (
        np.array([op.perm for op in G.operations], dtype=np.int64),
        np.array([op.perm_phases for op in G.operations], dtype=np.complex128),
    )


def make_case(R, name, model, n_filled, theta=None, nev=4, sectors="all", mode="matrixfree"):
    sre = R.sre
    if theta is not None:
        R.sqm.update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=theta)
    G = sre.build_translation_group(model.lattice, theta)
    data = quiet(sre.build_ed_data, model, filling_fraction=Fraction(n_filled, model.lattice.n_site),
                 symmetry_group=G)
    out = {}
    perm, eta = group_arrays(G)
    out["perm"], out["eta"] = perm, eta
    out["n_site"] = np.int64(model.lattice.n_site)
    out["n_filled"] = np.int64(n_filled)
    out["fermionic"] = np.int64(model.particle_statistics.name == "FERMIONIC")
    out["theta"] = np.array(theta if theta is not None else [0.0] * model.lattice.dim)
    out["bil_ij"], out["bil_t"] = terms_array(model.bilinear_terms)
    out["den_ij"], out["den_v"] = terms_array(model.density_density_terms)
    out.update(catalog_arrays(data.orbit_catalog))
    out["chi"] = np.array([ir.values for ir in data.irrep_list], dtype=np.complex128)
    labels = [ir.label for ir in data.irrep_list]
    idxs = range(len(labels)) if sectors == "all" else [labels.index(s) for s in sectors]
    dims, vals = [], []
    for i in range(len(labels)):
        b = sre.build_symmetry_sector_basis(data.orbit_catalog, data.irrep_list[i])
        dims.append(len(b.representative_mask_list))
    for i in idxs:
        f = sre.ed_scan_at_irrep_matrixfree if mode == "matrixfree" else sre.ed_scan_at_irrep_matrix
        v, _ = quiet(f, labels[i], data, nev=nev)
        row = np.full(nev, np.nan)
        row[: len(v)] = v
        vals.append(row)
    out["sector_dims"] = np.array(dims, dtype=np.int64)
    out["eig_sectors"] = np.array(list(idxs), dtype=np.int64)
    out["eig_vals"] = np.array(vals)
    out["nev"] = np.int64(nev)
    # flux update of the zero-flux catalog, as the reference function does it
    if theta is not None:
        G0 = sre.build_translation_group(model.lattice, [0.0] * model.lattice.dim)
        cat0 = quiet(sre.build_symmetry_orbit_catalog, second_quantized_model=model, n_filled=n_filled,
                     symmetry_group=G0, particle_statistics=model.particle_statistics)
        sre.update_orbit_stabilizer_phases(cat0, G, model.particle_statistics)
        out.update(catalog_arrays(cat0, prefix="upd_"))
    path = os.path.join(HERE, f"{name}.npz")
    np.savez_compressed(path, **out)
    print(f"{name}: C={len(out['rep_rank'])} orbits={len(out['reprs'])} -> {os.path.getsize(path)} B")


def main():
    R = ref_shim.load()
    # Heisenberg ring N=16 (8 up spins), all 16 momentum sectors
    make_case(R, "heisenberg16", quiet(R.heisenberg.build_heisenberg_second_quantized_model, 16, 1.0),
              8, nev=4)
    # checkerboard 3x4x2, 4 fermions, V1=1
    p = dict(R.fermionic.params_Sun_Gu_Katsura_Sarma)
    p.update({"V1": 1.0, "V2": 0.0, "V3": 0.0})
    make_case(R, "checkerboard24",
              quiet(R.fermionic.build_zero_flux_fermionic_fci_second_quantized_model,
                    sample_size=[3, 4], params=p), 4, nev=6)
    # Haldane 2x3, 3 bosons (test_core regression lattice), zero flux and flux
    make_case(R, "haldane12",
              R.bosonic.build_zero_flux_bosonic_fci_second_quantized_model(
                  sample_size=[2, 3], params=R.bosonic.params_DNSheng), 3, nev=3)
    make_case(R, "haldane12_flux",
              R.bosonic.build_zero_flux_bosonic_fci_second_quantized_model(
                  sample_size=[2, 3], params=R.bosonic.params_DNSheng), 3, theta=[0.3, 0.1], nev=3)
    # checkerboard 2x3, 4 fermions with flux (fermionic signs + phases)
    pf = dict(R.fermionic.params_Sun_Gu_Katsura_Sarma)
    make_case(R, "checkerboard12_flux",
              quiet(R.fermionic.build_zero_flux_fermionic_fci_second_quantized_model,
                    sample_size=[2, 3], params=pf), 4, theta=[0.25, 0.4], nev=3)
    # Haldane 3x4 bosons with flux: sectors of dim > 500 (Lanczos path of the reference)
    pb = {"t": 1.0, "t'": 0.6, "t''": 0.0, "phi_over_2pi": 0.2, "V1": 1.0, "V2": 0.0}
    make_case(R, "haldane24_flux",
              R.bosonic.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[3, 4], params=pb),
              6, theta=[0.125, 0.375], nev=4, sectors=[(0, 0), (1, 2)])
    # spinful Hubbard 2x3 (total particle number, 12 spin-orbitals, 6 fermions)
    make_case(R, "hubbard12", quiet(R.hubbard.build_spinful_hubbard_second_quantized_model, [2, 3], 1.0, 4.0),
              6, nev=4)


if __name__ == "__main__":
    main()
