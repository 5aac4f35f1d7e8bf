"""Loader for the reference's own Python engine (golden-vector generation only).

TEST INFRASTRUCTURE.  Nothing in the product imports this module.  It is used
by ``tests/golden/make_*.py`` to produce the committed fixtures, by the
CPU-only tests that pin the oracle against the reference when the reference
is present, and by ``bench.py``'s reference arm (the reference's own
numpy/scipy path timed on the host cores).

The reference package ``realspace_exactdiagonalization_py`` cannot be imported
normally here: its ``__init__`` pulls in ``models/`` which imports the absent
``tightbinding_py`` dependency.  This shim

1. registers a synthetic top-level package whose ``__path__`` is the
   reference's source directory (its ``__init__`` is not executed);
2. registers this repository's restatement of ``tightbinding_py``
   (``realspace_exatdiagonalization_py_b200.lattice``) under that name, so the
   reference's own model builders (``models/*.py``) run unmodified on it;
3. imports the engine (``symmetry_resolved_ed``) and the model modules.
"""

from __future__ import annotations

import importlib
import os
import sys
import types

PKG = "realspace_exactdiagonalization_py"
_REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
# the reference as installed by oracle/install_reference.py (travels with the
# working tree), else a checkout named by RSED_REFERENCE_ROOT
INSTALLED = os.path.join(_REPO, "baseline", "_ref", PKG)


def package_dir() -> str | None:
    """Directory of the reference package's sources, or None."""
    cands = []
    root = os.environ.get("RSED_REFERENCE_ROOT")
    if root:
        cands.append(os.path.join(root, "src", PKG))
    cands.append(INSTALLED)
    for d in cands:
        if os.path.isfile(os.path.join(d, "symmetry_resolved_ed.py")):
            return d
    return None


def available() -> bool:
    return package_dir() is not None


def load():
    """Return a namespace with the reference engine and model modules."""
    src = package_dir()
    if src is None:
        raise RuntimeError("reference package not present (run oracle/install_reference.py)")
    if PKG in sys.modules and hasattr(sys.modules[PKG], "_rsed_shim"):
        return sys.modules[PKG]._rsed_shim

    from realspace_exatdiagonalization_py_b200 import lattice as tb

    tb_pkg = types.ModuleType("tightbinding_py")
    for name in tb.__all__:
        setattr(tb_pkg, name, getattr(tb, name))
    tb_pkg.__path__ = []  # mark as package
    tb_utils = types.ModuleType("tightbinding_py.utils")
    tb_utils.generate_bilinear_terms = tb.generate_bilinear_terms
    tb_lat = types.ModuleType("tightbinding_py.lattice")
    tb_lat.Real_Space_Lattice = tb.Real_Space_Lattice
    tb_mod = types.ModuleType("tightbinding_py.tb_model")
    tb_mod.Real_Space_TightBinding_Model = tb.Real_Space_TightBinding_Model
    tb_pkg.utils, tb_pkg.lattice, tb_pkg.tb_model = tb_utils, tb_lat, tb_mod
    sys.modules.update(
        {
            "tightbinding_py": tb_pkg,
            "tightbinding_py.utils": tb_utils,
            "tightbinding_py.lattice": tb_lat,
            "tightbinding_py.tb_model": tb_mod,
        }
    )

    pkg = types.ModuleType(PKG)
    pkg.__path__ = [src]
    sys.modules[PKG] = pkg
    sre = importlib.import_module(PKG + ".symmetry_resolved_ed")
    sqm = importlib.import_module(PKG + ".second_quantized_model")
    models_pkg = types.ModuleType(PKG + ".models")
    models_pkg.__path__ = [os.path.join(src, "models")]
    sys.modules[PKG + ".models"] = models_pkg
    heis = importlib.import_module(PKG + ".models.heisenberg")
    hub = importlib.import_module(PKG + ".models.hubbard")
    bos = importlib.import_module(PKG + ".models.bosonic_fci")
    fer = importlib.import_module(PKG + ".models.fermionic_fci")
    ns = types.SimpleNamespace(
        sre=sre, sqm=sqm, heisenberg=heis, hubbard=hub, bosonic=bos, fermionic=fer
    )
    pkg._rsed_shim = ns
    return ns
