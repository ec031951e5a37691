"""Imports the `gpu-fem-project_b200/` package (its directory name is not a
Python identifier) under the module name `gpu_fem_project_b200`."""
from __future__ import annotations

import importlib.util
import pathlib
import sys

ROOT = pathlib.Path(__file__).resolve().parent
PKG_DIR = ROOT / "gpu-fem-project_b200"
NAME = "gpu_fem_project_b200"


def load():
    if NAME in sys.modules:
        return sys.modules[NAME]
    spec = importlib.util.spec_from_file_location(NAME, PKG_DIR / "__init__.py",
                                                  submodule_search_locations=[str(PKG_DIR)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[NAME] = mod
    try:
        spec.loader.exec_module(mod)
    except BaseException:
        del sys.modules[NAME]
        raise
    return mod


def load_builder():
    """The build recipe module (gpu-fem-project_b200/build.py), importable without the .so."""
    spec = importlib.util.spec_from_file_location(NAME + "_build", PKG_DIR / "build.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def load_module(name: str):
    """A single module of the package directory that needs no compiled library
    (e.g. `replicas`), importable on machines without the built .so."""
    full = f"{NAME}_{name}"
    if full in sys.modules:
        return sys.modules[full]
    spec = importlib.util.spec_from_file_location(full, PKG_DIR / f"{name}.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules[full] = mod
    spec.loader.exec_module(mod)
    return mod
