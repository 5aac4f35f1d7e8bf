"""Shared builders of the golden cases (models from this package's builders,
which the CPU tests pin to the reference's term lists)."""

from fractions import Fraction

import numpy as np


def model_for(case):
    from realspace_exatdiagonalization_py_b200 import models

    if case == "heisenberg16":
        return models.build_heisenberg_second_quantized_model(16, 1.0)
    if case == "checkerboard24":
        p = dict(models.params_Sun_Gu_Katsura_Sarma)
        p.update({"V1": 1.0, "V2": 0.0, "V3": 0.0})
        return models.build_zero_flux_fermionic_fci_second_quantized_model(sample_size=[3, 4], params=p)
    if case.startswith("haldane12"):
        return models.build_zero_flux_bosonic_fci_second_quantized_model(
            sample_size=[2, 3], params=models.params_DNSheng)
    if case == "checkerboard12_flux":
        return models.build_zero_flux_fermionic_fci_second_quantized_model(
            sample_size=[2, 3], params=models.params_Sun_Gu_Katsura_Sarma)
    if case == "haldane24_flux":
        p = {"t": 1.0, "t'": 0.6, "t''": 0.0, "phi_over_2pi": 0.2, "V1": 1.0, "V2": 0.0}
        return models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=[3, 4], params=p)
    if case == "hubbard12":
        return models.build_spinful_hubbard_second_quantized_model([2, 3], 1.0, 4.0)
    raise KeyError(case)


def ed_data_for(case, g):
    import realspace_exatdiagonalization_py_b200 as ed

    m = model_for(case)
    theta = [float(x) for x in g["theta"]]
    if any(theta):
        ed.update_second_quantized_model_with_twisted_phases(m, twisted_phases_over_2π=theta)
        G = ed.build_translation_group(m.lattice, theta)
    else:
        G = ed.build_translation_group(m.lattice)
    return ed.build_ed_data(m, filling_fraction=Fraction(int(g["n_filled"]), m.lattice.n_site),
                            symmetry_group=G)


def oracle_block(g, s):
    """The reference's sector block (CSR) rebuilt by the oracle from the
    golden catalog tables."""
    from oracle import port

    cat = port.catalog(int(g["n_site"]), int(g["n_filled"]), (g["perm"] - 1).astype(np.uint8), g["eta"],
                       bool(g["fermionic"]))
    bil = [(int(i), int(j), t) for (i, j), t in zip(g["bil_ij"], g["bil_t"])]
    den = [(int(i), int(j), v) for (i, j), v in zip(g["den_ij"], g["den_v"])]
    chi = g["chi"][s]
    orbits = port.sector_orbits(cat, chi)
    return port.csr_block(cat, int(g["n_site"]), orbits, bil, den, chi, bool(g["fermionic"])), orbits


CHERN_CASES = ["haldane12", "haldane16", "haldane16_singular", "checkerboard12", "haldane12_identity"]


def chern_case(name):
    """(model at zero flux, n_particles, labels, nev, grid, fixture) of one
    chern_*.npz fixture (tests/golden/make_chern_golden.py)."""
    import os

    import numpy as np

    from realspace_exatdiagonalization_py_b200 import models

    f = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", f"chern_{name}.npz")))
    sample = [int(x) for x in f["sample"]]
    if str(f["kind"]) == "bosonic":
        m = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=sample, params=models.params_DNSheng)
    else:
        m = models.build_zero_flux_fermionic_fci_second_quantized_model(
            sample_size=sample, params=dict(models.params_Sun_Gu_Katsura_Sarma))
    labels = "identity" if f["labels"].dtype.kind == "U" else [tuple(int(x) for x in lab) for lab in f["labels"]]
    return m, int(f["n_particles"]), labels, int(f["nev"]), tuple(int(x) for x in f["grid"]), f


PUMP_CASES = ["haldane12", "checkerboard12", "haldane16"]


def pump_case(name):
    """(model at zero flux, fixture) of one pump_*.npz fixture
    (tests/golden/make_pump_golden.py)."""
    import os

    import numpy as np

    from realspace_exatdiagonalization_py_b200 import models

    f = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", f"pump_{name}.npz")))
    sample = [int(x) for x in f["sample"]]
    if str(f["kind"]) == "bosonic":
        m = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=sample, params=models.params_DNSheng)
    else:
        m = models.build_zero_flux_fermionic_fci_second_quantized_model(
            sample_size=sample, params=dict(models.params_Sun_Gu_Katsura_Sarma))
    return m, f


def pump_specs(f):
    """The (sector, level) manifold of a pump fixture."""
    labels = [tuple(int(x) for x in lab) for lab in f["labels"]]
    if len(f["states"]):
        return [((int(a), int(b)), int(lev)) for a, b, lev in f["states"]]
    return [(lab, lev) for lab in labels for lev in range(1, int(f["nev"]) + 1)]


CORR_CASES = ["haldane12", "checkerboard12", "haldane12_identity", "haldane16"]


def corr_case(name):
    """(model at zero flux, sector label, level, flavour_a filter, fixture) of
    one corr_*.npz fixture (tests/golden/make_corr_golden.py)."""
    import os

    import numpy as np

    from realspace_exatdiagonalization_py_b200 import models

    f = dict(np.load(os.path.join(os.path.dirname(__file__), "golden", f"corr_{name}.npz")))
    sample = [int(x) for x in f["sample"]]
    if str(f["kind"]) == "bosonic":
        m = models.build_zero_flux_bosonic_fci_second_quantized_model(sample_size=sample, params=models.params_DNSheng)
    else:
        m = models.build_zero_flux_fermionic_fci_second_quantized_model(
            sample_size=sample, params=dict(models.params_Sun_Gu_Katsura_Sarma))
    label = "identity" if f["label"].dtype.kind == "U" else tuple(int(x) for x in f["label"])
    fa = (lambda i: True) if str(f["flavor_a"]) == "all" else (lambda i: i % 2 == 1)
    return m, label, int(f["level"]), fa, f
