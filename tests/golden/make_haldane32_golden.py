"""Generate tests/golden/haldane32.npz from the reference engine: the
32-site Haldane-boson workload at full size.

Model: honeycomb 4 x 4 cells x 2 sublattices = 32 sites, 8 hard-core bosons
(C(32, 8) = 10,518,300 states), t = 1, t' = 0.6 exp(+-0.4 pi i), t'' = 0,
V1 = 1, translation group of order 16 (657,756 orbits).  Built with the
reference's own ``build_zero_flux_bosonic_fci_second_quantized_model`` and
engine, loaded through ``oracle/ref_shim.py``:

* zero flux: checksums of the orbit catalog (representatives, the three
  representative tables, stabilizers), the 16 sector dimensions and the
  lowest 4 eigenvalues of every sector (``ed_scan_at_irrep_matrixfree``,
  ARPACK ``eigs(which="SR", tol=1e-10)``);
* flux (theta_x, theta_y) = (0.25, 0.5) (point (4, 8) of a 16 x 16 grid): the
  catalog the reference's flux drivers build (a fresh catalog with the flux
  group), its checksums and sector dimensions, the lowest 4 eigenvalues of
  sectors (0, 0) and (1, 2), and the reference's matrix-free operator
  ``H_op(x)`` of sector (1, 2) on a seeded vector, sampled at 4096 rows plus
  its norm and <x, H x>.

The tables are 168 MB per catalog, so they are stored as SHA-256 digests; in
the complex64 amplitude table, components below 1e-15 in magnitude are set to
+0 before hashing (the device's sincos and the host libm differ only there).
Takes about 15 minutes on 8 host cores:

    python tests/golden/make_haldane32_golden.py
"""

from __future__ import annotations

import contextlib
import hashlib
import io
import os
import sys
import time
from fractions import Fraction

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref_shim  # noqa: E402

PARAMS = {"t": 1.0, "t'": 0.6, "t''": 0.0, "phi_over_2pi": 0.2, "V1": 1.0, "V2": 0.0}
FLUX = [0.25, 0.5]
FLUX_SECTORS = [(0, 0), (1, 2)]
MATVEC_SECTOR = (1, 2)
MATVEC_SEED = 2024
N_SAMPLE = 4096
NEV = 4


def quiet(f, *a, **k):
    with contextlib.redirect_stdout(io.StringIO()):
        return f(*a, **k)


def amp_digest(amp: np.ndarray) -> str:
    """SHA-256 of a complex64 table with components |x| < 1e-15 set to +0."""
    a = np.ascontiguousarray(amp, dtype=np.complex64).view(np.float32).copy()
    a[np.abs(a) < 1e-15] = 0.0
    return hashlib.sha256(a.tobytes()).hexdigest()


def catalog_digests(cat) -> dict:
    stab_g = cat.stabilizer_g_indices_list
    flat_g = np.array([g for gs in stab_g for g in gs], dtype=np.int64)
    flat_p = np.array([p for ps in cat.stabilizer_phases_list for p in ps], dtype=np.complex128)
    return {
        "n_orbits": np.int64(len(cat.representative_mask_list)),
        "reprs_sha": hashlib.sha256(np.array(cat.representative_mask_list, dtype=np.uint64).tobytes()).hexdigest(),
        "rep_rank_sha": hashlib.sha256(np.ascontiguousarray(cat.rep_rank_table, dtype=np.int32).tobytes()).hexdigest(),
        "rep_sym_sha": hashlib.sha256(np.ascontiguousarray(cat.rep_sym_table, dtype=np.int32).tobytes()).hexdigest(),
        "rep_amp_sha": amp_digest(cat.rep_amp_table),
        "stab_sizes": np.bincount(np.array([len(g) for g in stab_g]), minlength=17).astype(np.int64),
        "stab_g_sha": hashlib.sha256(flat_g.tobytes()).hexdigest(),
        "stab_phase_sum": np.complex128(flat_p.sum()),
    }


def spectra(sre, data, labels):
    out = []
    for lab in labels:
        t0 = time.perf_counter()
        v, _ = quiet(sre.ed_scan_at_irrep_matrixfree, lab, data, nev=NEV)
        print(f"  sector {lab}: {time.perf_counter() - t0:.1f} s  {v}", flush=True)
        out.append(np.asarray(v, dtype=np.float64))
    return np.array(out)


def main():
    R = ref_shim.load()
    sre = R.sre
    model = R.bosonic.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[4, 4], params=PARAMS)
    out = {"params_keys": np.array(list(PARAMS)), "params_vals": np.array(list(PARAMS.values())),
           "n_site": np.int64(32), "n_filled": np.int64(8), "nev": np.int64(NEV)}

    # ---- zero flux ---------------------------------------------------------
    G0 = sre.build_translation_group(model.lattice, None)
    t0 = time.perf_counter()
    d0 = quiet(sre.build_ed_data, model, filling_fraction=Fraction(8, 32), symmetry_group=G0)
    print(f"zero-flux catalog {time.perf_counter() - t0:.1f} s", flush=True)
    for k, v in catalog_digests(d0.orbit_catalog).items():
        out["zf_" + k] = v
    labels = [ir.label for ir in d0.irrep_list]
    out["labels"] = np.array(labels, dtype=np.int64)
    out["zf_sector_dims"] = np.array(
        [len(sre.build_symmetry_sector_basis(d0.orbit_catalog, ir).representative_mask_list)
         for ir in d0.irrep_list], dtype=np.int64)
    out["zf_eig"] = spectra(sre, d0, labels)
    del d0

    # ---- one flux point ----------------------------------------------------
    R.sqm.update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=FLUX)
    G = sre.build_translation_group(model.lattice, FLUX)
    t0 = time.perf_counter()
    d1 = quiet(sre.build_ed_data, model, filling_fraction=Fraction(8, 32), symmetry_group=G)
    print(f"flux catalog {time.perf_counter() - t0:.1f} s", flush=True)
    out["flux"] = np.array(FLUX)
    for k, v in catalog_digests(d1.orbit_catalog).items():
        out["fx_" + k] = v
    out["fx_sector_dims"] = np.array(
        [len(sre.build_symmetry_sector_basis(d1.orbit_catalog, ir).representative_mask_list)
         for ir in d1.irrep_list], dtype=np.int64)
    out["fx_sectors"] = np.array(FLUX_SECTORS, dtype=np.int64)
    out["fx_eig"] = spectra(sre, d1, FLUX_SECTORS)
    # the reference's matrix-free operator on a seeded vector
    irrep = d1.irrep_list[labels.index(MATVEC_SECTOR)]
    basis = sre.build_symmetry_sector_basis(d1.orbit_catalog, irrep)
    cmap = sre.CanonicalMap(G, model.particle_statistics, d1.orbit_catalog)
    H_op, n = quiet(sre.hamiltonian_linear_operator, basis, model.bilinear_terms,
                    model.density_density_terms, cmap)
    rng = np.random.default_rng(MATVEC_SEED)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y = H_op(x)
    idx = np.sort(np.random.default_rng(MATVEC_SEED + 1).choice(n, size=N_SAMPLE, replace=False))
    out.update({"mv_sector": np.array(MATVEC_SECTOR, dtype=np.int64), "mv_seed": np.int64(MATVEC_SEED),
                "mv_n": np.int64(n), "mv_idx": idx.astype(np.int64), "mv_y": y[idx],
                "mv_norm": np.float64(np.linalg.norm(y)), "mv_xhy": np.complex128(np.vdot(x, y))})
    path = os.path.join(HERE, "haldane32.npz")
    np.savez_compressed(path, **out)
    print(f"-> {path} ({os.path.getsize(path)} B)")


if __name__ == "__main__":
    main()
