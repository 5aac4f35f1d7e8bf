"""The 32-site Haldane-boson workload at full size (10,518,300 states,
657,756 orbits, |G| = 16) against the reference's own results
(tests/golden/haldane32.npz, written by tests/golden/make_haldane32_golden.py):

* the orbit catalog at zero flux and at flux (0.25, 0.5): SHA-256 digests of
  the representatives, of the rep / g / complex64 amplitude tables (amplitude
  components below 1e-15 set to +0 on both sides) and of the stabilizers;
  the flux catalog both built fresh (the reference's route) and moved there
  from the zero-flux catalog by ``update_orbit_stabilizer_phases`` (integer
  tables and stabilizers identical);
* all 16 sector dimensions and spectra at zero flux (batched FP32 matvec +
  FP64 refinement) and two flux sectors (batched FP64, and served through
  ``SolveServer`` on the phase-updated catalog), 1e-10 absolute;
* the reference's ``H_op(x)`` of sector (1, 2) at the flux point, sampled at
  4096 rows, with its norm and <x, H x>.
"""

import hashlib
from fractions import Fraction

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _digests(cat):
    t = cat.table.cpu().numpy()
    amp = np.ascontiguousarray(t[:, 2:4]).view(np.float32).reshape(-1).copy()
    amp[np.abs(amp) < 1e-15] = 0.0
    sm = cat.stab_mask.cpu().numpy().view(np.uint64)
    n_g = cat.dgroup.n_group
    bits = ((sm[:, None] >> np.arange(n_g, dtype=np.uint64)) & np.uint64(1)).astype(bool)
    sizes = bits.sum(axis=1)
    return {
        "n_orbits": cat.n_orbits,
        "reprs_sha": hashlib.sha256(cat.repr_masks.cpu().numpy().view(np.uint64).tobytes()).hexdigest(),
        "rep_rank_sha": hashlib.sha256(np.ascontiguousarray(t[:, 0]).tobytes()).hexdigest(),
        "rep_sym_sha": hashlib.sha256(np.ascontiguousarray(t[:, 1]).tobytes()).hexdigest(),
        "rep_amp_sha": hashlib.sha256(amp.tobytes()).hexdigest(),
        "stab_sizes": np.bincount(sizes, minlength=17),
        "stab_g_sha": hashlib.sha256(np.nonzero(bits)[1].astype(np.int64).tobytes()).hexdigest(),
        "stab_phase_sum": cat.stab_phase.cpu().numpy().sum(),
    }


def _check_digests(d, g, prefix, amplitudes=True):
    assert d["n_orbits"] == int(g[prefix + "n_orbits"])
    for k in ("reprs_sha", "rep_rank_sha", "rep_sym_sha", "stab_g_sha") + (("rep_amp_sha",) if amplitudes else ()):
        assert d[k] == str(g[prefix + k]), k
    np.testing.assert_array_equal(d["stab_sizes"], g[prefix + "stab_sizes"])
    np.testing.assert_allclose(d["stab_phase_sum"], g[prefix + "stab_phase_sum"], rtol=1e-12)


@pytest.fixture(scope="module")
def h32(golden):
    import realspace_exatdiagonalization_py_b200 as ed
    from realspace_exatdiagonalization_py_b200 import models

    g = golden("haldane32")
    model, nf = models.config_model("haldane32")
    G = ed.build_translation_group(model.lattice)
    data = ed.build_ed_data(model, filling_fraction=Fraction(nf, 32), symmetry_group=G)
    return ed, models, g, data


def test_zero_flux_catalog_and_dims(h32):
    ed, _, g, data = h32
    _check_digests(_digests(data.orbit_catalog), g, "zf_")
    _, sset = data._device()
    np.testing.assert_array_equal(sset.dims, g["zf_sector_dims"])
    assert [tuple(ir.label) for ir in data.irrep_list] == [tuple(x) for x in g["labels"]]


def test_zero_flux_spectra_batched_fp32(h32):
    ed, _, g, data = h32
    secs = list(range(16))
    cfg = ed.SolverConfig((2,) * 16, 0, True, 16)
    res = ed.solve_sectors_batched(data, secs, nev=4, precision=32, config=cfg, return_vectors=False)
    for s in secs:
        np.testing.assert_allclose(res[s][0], g["zf_eig"][s], atol=1e-10, rtol=0)
    data.__dict__.pop("_solvers", None)


def _flux_model(models, g):
    import realspace_exatdiagonalization_py_b200 as ed

    model, nf = models.config_model("haldane32")
    flux = [float(x) for x in g["flux"]]
    ed.update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=flux)
    return model, nf, flux, ed.build_translation_group(model.lattice, flux)


def test_flux_catalog_both_routes(h32):
    ed, models, g, data0 = h32
    model, nf, flux, G = _flux_model(models, g)
    fresh = ed.build_ed_data(model, filling_fraction=Fraction(nf, 32), symmetry_group=G)
    _check_digests(_digests(fresh.orbit_catalog), g, "fx_")
    _, sset = fresh._device()
    np.testing.assert_array_equal(sset.dims, g["fx_sector_dims"])
    moved = data0.orbit_catalog.clone()
    ed.update_orbit_stabilizer_phases(moved, G, model.particle_statistics)
    # the reference's update keeps every integer table of a fresh build;
    # its product-form amplitudes differ from the fresh exp(i sum) form only
    # in near-zero components, so they are compared through the spectra below
    _check_digests(_digests(moved), g, "fx_", amplitudes=False)


def test_flux_spectra_batched_and_served(h32):
    ed, models, g, _ = h32
    model, nf, flux, G = _flux_model(models, g)
    data = ed.build_ed_data(model, filling_fraction=Fraction(nf, 32), symmetry_group=G)
    labels = [tuple(ir.label) for ir in data.irrep_list]
    secs = [labels.index(tuple(x)) for x in g["fx_sectors"]]
    res = ed.solve_sectors_batched(data, secs, nev=4, precision=64)
    for k, s in enumerate(secs):
        np.testing.assert_allclose(res[s][0], g["fx_eig"][k], atol=1e-10, rtol=0)
    del data
    m0, _ = models.config_model("haldane32")
    sm = ed.ServingModel(m0, nf, name="haldane32")
    srv = ed.SolveServer(sm, nev=4, precision=32, block=2)
    reqs = [ed.SolveRequest(k, s, tuple(flux), "haldane32") for k, s in enumerate(secs)]
    reqs += [ed.SolveRequest(10 + s, s, (0.0, 0.0), "haldane32") for s in (0, 7)]
    out = {r.rid: r for r in srv.run(reqs, realtime=False)}
    for k in range(len(secs)):
        np.testing.assert_allclose(out[k].eigenvalues, g["fx_eig"][k], atol=1e-10, rtol=0)
    for s in (0, 7):
        np.testing.assert_allclose(out[10 + s].eigenvalues, g["zf_eig"][s], atol=1e-10, rtol=0)


def test_reference_operator_at_scale(h32):
    ed, models, g, _ = h32
    model, nf, flux, G = _flux_model(models, g)
    data = ed.build_ed_data(model, filling_fraction=Fraction(nf, 32), symmetry_group=G)
    labels = [tuple(ir.label) for ir in data.irrep_list]
    s = labels.index(tuple(int(x) for x in g["mv_sector"]))
    basis = ed.build_symmetry_sector_basis(data.orbit_catalog, data.irrep_list[s])
    cmap = ed.CanonicalMap(G, model.particle_statistics, data.orbit_catalog)
    H_op, n = ed.hamiltonian_linear_operator(basis, model.bilinear_terms, model.density_density_terms, cmap)
    assert n == int(g["mv_n"])
    rng = np.random.default_rng(int(g["mv_seed"]))
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    y = H_op(x)
    np.testing.assert_allclose(y[g["mv_idx"]], g["mv_y"], rtol=0, atol=1e-11)
    assert abs(np.linalg.norm(y) - float(g["mv_norm"])) <= 1e-12 * float(g["mv_norm"])
    assert abs(np.vdot(x, y) - complex(g["mv_xhy"])) <= 1e-12 * abs(complex(g["mv_xhy"]))
