"""Import helper for the ``dft-zig_b200`` package (its directory name is not a Python identifier).

``load()`` registers it as the module ``dftzig_b200`` and returns it.
"""
from __future__ import annotations

import importlib.util
import os
import sys

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "dft-zig_b200")


def load():
    if "dftzig_b200" in sys.modules:
        return sys.modules["dftzig_b200"]
    spec = importlib.util.spec_from_file_location("dftzig_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dftzig_b200"] = mod
    spec.loader.exec_module(mod)
    return mod
