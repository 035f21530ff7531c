"""Registers the package directory `proliferatingcellcollectives-idp_b200/`
(not a valid Python identifier) under the import name `pcc_b200`."""
from __future__ import annotations

import importlib.util
import sys
from pathlib import Path

PKG_DIR = Path(__file__).resolve().parent / "proliferatingcellcollectives-idp_b200"


def load_package():
    if "pcc_b200" in sys.modules:
        return sys.modules["pcc_b200"]
    spec = importlib.util.spec_from_file_location("pcc_b200", PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["pcc_b200"] = mod
    spec.loader.exec_module(mod)
    return mod
