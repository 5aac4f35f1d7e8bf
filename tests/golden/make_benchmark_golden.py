"""Extract tests/golden/reference_benchmark.npz from the reference's own
benchmark results (benchmark/benchmark_data/benchmark_raw_latest_py.csv):
for every (model, size) the orbit count, the dimension of sector 0 and the
lowest energy of sector 0 found by its matrix-free mode, and the published
single-sector times of both modes (seconds on the reference's 12-core CPU).  The reference's
benchmark builds the models with build_heisenberg_ed_data(N) (J = 1, half
filling), build_bosonic_fci_ed_data(sample_size=...) (params_DNSheng, a
quarter of the vertices filled) and build_spinful_hubbard_ed_data(sample_size)
(t = 1, U = 8, half filling, total particle number).  Runs where a
reference checkout is present (its root in RSED_REFERENCE_ROOT):

    RSED_REFERENCE_ROOT=<checkout> python tests/golden/make_benchmark_golden.py
"""

import csv
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
CSV_REL = os.path.join("benchmark", "benchmark_data", "benchmark_raw_latest_py.csv")


def main():
    root = os.environ.get("RSED_REFERENCE_ROOT")
    if not root:
        raise SystemExit("set RSED_REFERENCE_ROOT to the reference checkout")
    CSV = os.path.join(root, CSV_REL)
    allrows = list(csv.DictReader(open(CSV)))
    rows = [r for r in allrows if r["mode"] == "matrixfree"]
    t_matrix = {(r["model"], r["label"]): float(r["elapsed_s"]) for r in allrows if r["mode"] == "matrix"}
    out = {
        "model": np.array([r["model"] for r in rows]),
        "label": np.array([r["label"] for r in rows]),
        "n_site": np.array([int(r["n_site"]) for r in rows]),
        "n_filled": np.array([int(r["n_filled"]) for r in rows]),
        "full_dim": np.array([int(r["full_dim"]) for r in rows]),
        "n_orbits": np.array([int(r["n_orbits"]) for r in rows]),
        "n_group": np.array([int(r["n_group"]) for r in rows]),
        "sector_dim": np.array([int(r["sector_dim"]) for r in rows]),
        "energy": np.array([float(r["energy"]) for r in rows]),
        "elapsed_matrixfree_s": np.array([float(r["elapsed_s"]) for r in rows]),
        "elapsed_matrix_s": np.array([t_matrix[(r["model"], r["label"])] for r in rows]),
    }
    path = os.path.join(HERE, "reference_benchmark.npz")
    np.savez_compressed(path, **out)
    print(len(rows), "rows ->", path)


if __name__ == "__main__":
    main()
