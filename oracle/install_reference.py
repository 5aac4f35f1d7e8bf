"""Install the reference package into ``baseline/_ref`` (bench reference arm).

TEST INFRASTRUCTURE.  The reference ``realspace_exactdiagonalization_py``
declares ``uv_build`` as its build backend, which is not in the offline
wheelhouse.  This recipe copies the reference checkout to a temporary
directory, replaces only the ``[build-system]`` table of the copy's
``pyproject.toml`` with setuptools (package sources under ``src/``, no code
touched), and runs

    pip install --no-index --no-build-isolation --no-deps --target baseline/_ref <copy>

``--no-deps``: the ``tightbinding-py`` path dependency is not vendored with
the reference (``oracle/ref_shim.py`` supplies this repository's restatement
of it at import time) and matplotlib / ipykernel are only used for plots and
notebooks.  ``baseline/_ref`` is git-ignored; it travels with the working
tree so that ``bench.py --impl reference`` runs the reference's own numpy /
scipy code path on the GPU box's host cores.

    python oracle/install_reference.py [--reference DIR]
"""

from __future__ import annotations

import argparse
import os
import re
import shutil
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
TARGET = os.path.join(ROOT, "baseline", "_ref")
PKG = "realspace_exactdiagonalization_py"

_SETUPTOOLS_BACKEND = """[build-system]
requires = ["setuptools"]
build-backend = "setuptools.build_meta"

[tool.setuptools.packages.find]
where = ["src"]
"""


def installed() -> bool:
    return os.path.isfile(os.path.join(TARGET, PKG, "symmetry_resolved_ed.py"))


def install(reference: str, quiet: bool = True) -> str:
    """Install (or reinstall) the reference into ``baseline/_ref``; returns the
    installed package directory."""
    src = os.path.join(reference, "src", PKG, "symmetry_resolved_ed.py")
    if not os.path.isfile(src):
        raise FileNotFoundError(f"no reference checkout at {reference}")
    with tempfile.TemporaryDirectory(prefix="rsed_ref_") as tmp:
        copy = os.path.join(tmp, "ref")
        shutil.copytree(reference, copy, ignore=shutil.ignore_patterns(
            ".git", "doc", "figures", "benchmark", "examples", "*.ipynb"))
        py = os.path.join(copy, "pyproject.toml")
        text = open(py).read()
        text = re.sub(r"\[build-system\].*?(?=\n\[|\Z)", "", text, flags=re.S)
        text = re.sub(r"\[tool\.uv\.sources\].*?(?=\n\[|\Z)", "", text, flags=re.S)
        with open(py, "w") as f:
            f.write(text.rstrip() + "\n\n" + _SETUPTOOLS_BACKEND)
        if os.path.isdir(TARGET):
            shutil.rmtree(TARGET)
        cmd = [sys.executable, "-m", "pip", "install", "--no-index", "--no-build-isolation", "--no-deps",
               "--find-links", "/opt/wheelhouse", "--target", TARGET, copy]
        subprocess.run(cmd, check=True, stdout=subprocess.DEVNULL if quiet else None)
    if not installed():
        raise RuntimeError("reference install finished without the engine module")
    return os.path.join(TARGET, PKG)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("RSED_REFERENCE_ROOT", "/root/reference"))
    args = ap.parse_args()
    print(install(args.reference, quiet=False))


if __name__ == "__main__":
    main()
