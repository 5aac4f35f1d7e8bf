"""Flux-grid drivers on top of the device solvers.

``flux_spectrum_flow`` keeps the contract of the reference's driver
(``observables/spectrum_flow.py:25-169``): the lowest ``nev`` energies of the
given sectors at every flux value of a scan along one lattice direction,
returned as a ``SimpleNamespace`` with the reference's fields.  Two engines:

* ``engine="scan"`` (the reference's route): one ``ed_scan`` flux scan with a
  canonical checkpoint per flux value (reused unless ``overwrite``), every
  sector of a flux point solved in one batched launch sequence;
* ``engine="served"``: every (flux value, sector) solve is a request to a
  ``SolveServer`` -- the zero-flux catalog is built once and moved to each flux
  point by ``update_orbit_stabilizer_phases``, solves of different flux points
  overlap on the device; no checkpoints (``checkpoint_paths`` is ``None``).
"""

from __future__ import annotations

import os
from fractions import Fraction
from types import SimpleNamespace

import numpy as np

__all__ = ["flux_spectrum_flow"]


def _labels(sector_labels):
    if isinstance(sector_labels, str):
        ident = sector_labels == "identity"
        return ident, ["identity"] if ident else [sector_labels]
    if isinstance(sector_labels, tuple):
        return False, [tuple(int(x) for x in sector_labels)]
    return False, [tuple(int(x) for x in lab) for lab in sector_labels]


def flux_spectrum_flow(model, sector_labels, *, filling_fraction, flux_direction: int = 1,
                       twisted_phases_over_2π_list=None, checkpoint_dir: str = "checkpoints", nev: int = 3,
                       fig_path: str | None = None, overwrite: bool = False, engine: str = "scan",
                       precision: int = 32):
    from .ed import build_ed_data, ed_scan, load_checkpoint
    from .second_quantized_model import update_second_quantized_model_with_twisted_phases
    from .symmetry import build_irrep_list, build_translation_group

    if twisted_phases_over_2π_list is None:
        twisted_phases_over_2π_list = list(np.linspace(0.0, 1.0, 9))
    thetas = [float(t) for t in twisted_phases_over_2π_list]
    is_identity, labels = _labels(sector_labels)
    dim = model.lattice.dim
    if not 1 <= flux_direction <= dim:
        raise ValueError(f"flux_direction must be in 1..{dim}")
    flux0 = [0.0] * dim
    update_second_quantized_model_with_twisted_phases(model, twisted_phases_over_2π=flux0)
    if not isinstance(filling_fraction, Fraction):
        filling_fraction = Fraction(filling_fraction)
    energies = np.full((len(thetas), len(labels), nev), np.nan)
    checkpoint_paths = None
    if engine == "scan":
        if is_identity:
            raise ValueError("the identity sector is served by full_ed, not by a translation flux scan")
        init = build_ed_data(model, filling_fraction=filling_fraction,
                             symmetry_group=build_translation_group(model.lattice, flux0))
        checkpoint_paths = ed_scan(init, nev=nev, mode="matrixfree", twisted_phases_over_2π_list=thetas,
                                   flux_direction=flux_direction, checkpoint_dir=checkpoint_dir,
                                   overwrite=overwrite, scanned_sectors=labels)
        for it, path in enumerate(checkpoint_paths):
            data = load_checkpoint(path)
            for isec, lab in enumerate(labels):
                idx = next((i for i, ir in enumerate(data.irrep_list) if ir.label == lab), None)
                if idx is not None and idx in data.ed_scan_res:
                    vals = data.ed_scan_res[idx][0]
                    nv = min(len(vals), nev)
                    energies[it, isec, :nv] = vals[:nv]
    elif engine == "served":
        from .serving import ServingModel, SolveRequest, SolveServer

        n_filled = int(filling_fraction * model.lattice.n_site)
        sm = ServingModel(model, n_filled, name="flow")
        irr = [ir.label for ir in build_irrep_list(sm.group0, model.lattice)]
        reqs, where = [], {}
        for it, th in enumerate(thetas):
            flux = [0.0] * dim
            flux[flux_direction - 1] = th
            for isec, lab in enumerate(labels):
                if lab not in irr:
                    raise ValueError(f"No irrep with label {lab!r} in irrep_list.")
                rid = len(reqs)
                reqs.append(SolveRequest(rid, irr.index(lab), tuple(flux), "flow"))
                where[rid] = (it, isec)
        server = SolveServer(sm, nev=nev, precision=precision, block=2)
        for res in server.run(reqs, realtime=False):
            it, isec = where[res.rid]
            nv = min(len(res.eigenvalues), nev)
            energies[it, isec, :nv] = res.eigenvalues[:nv]
    else:
        raise ValueError(f"unknown engine {engine!r}")
    if fig_path is not None:
        import matplotlib.pyplot as plt  # optional, as in the reference

        os.makedirs(os.path.dirname(os.path.abspath(fig_path)), exist_ok=True)
        fig, ax = plt.subplots(figsize=(8.0, 6.0))
        ax.set_xlabel(f"Inserted Flux [2π] along Direction-{flux_direction}")
        ax.set_ylabel("E")
        for isec in range(len(labels)):
            for level in range(nev):
                ax.plot(thetas, energies[:, isec, level], alpha=1 - level / nev, linewidth=2,
                        label=f"sector {labels[isec]!r}" if level == 0 else None)
        ax.legend(loc="best")
        fig.tight_layout()
        fig.savefig(fig_path)
    return SimpleNamespace(twisted_phases_over_2π_list=thetas, energies=energies, sector_labels=labels,
                           flux_direction=flux_direction, nev=nev, is_identity=is_identity, fig_path=fig_path,
                           checkpoint_paths=checkpoint_paths)
