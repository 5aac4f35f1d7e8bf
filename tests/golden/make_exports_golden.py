"""Write tests/golden/reference_exports.json: the names the reference package
re-exports at top level (``realspace_exactdiagonalization_py/__init__.py``),
read from its source with ``ast`` (nothing is imported).

    python tests/golden/make_exports_golden.py
"""

import ast
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

from oracle import ref_shim  # noqa: E402


def main():
    src = os.path.join(ref_shim.package_dir(), "__init__.py")
    tree = ast.parse(open(src).read())
    names = sorted({a.asname or a.name for n in tree.body if isinstance(n, ast.ImportFrom) for a in n.names})
    path = os.path.join(HERE, "reference_exports.json")
    with open(path, "w") as f:
        json.dump({"source": "realspace_exactdiagonalization_py/__init__.py", "names": names}, f, indent=1)
    print(f"{len(names)} names -> {path}")


if __name__ == "__main__":
    main()
