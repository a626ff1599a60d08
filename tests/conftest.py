"""Shared pytest set-up: registers the `gpu` marker, makes the package importable as
`misa_b200` (its directory name has hyphens) and builds the CUDA library and the
oracle in-tree when they are missing or stale."""
from __future__ import annotations

import importlib.util
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))
if str(ROOT / "tests") not in sys.path:
    sys.path.insert(0, str(ROOT / "tests"))


def load_package():
    if "misa_b200" in sys.modules:
        return sys.modules["misa_b200"]
    pkg_dir = ROOT / "misa-md-hip_b200"
    spec = importlib.util.spec_from_file_location("misa_b200", pkg_dir / "__init__.py",
                                                  submodule_search_locations=[str(pkg_dir)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["misa_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


mb = load_package()


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs on the B200 box)")
    from misa_b200 import builder
    builder.build()
    from oracle import oracle
    oracle.build()
