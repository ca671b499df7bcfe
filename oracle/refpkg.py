"""Imports the reference's own Python depth-map module (``orthomosaic.densify``) in place, for
the golden-fixture script only - TEST INFRASTRUCTURE, never used by the product.

A virtual ``orthomosaic`` package is created whose ``__path__`` is the reference source
directory, so ``densify.py`` and its pure-Python dependencies load from where they lie; the
compiled kernels it needs (``_dense``, ``_fast``, ``_mvs``) are the reference's own sources
compiled into oracle/_ref by ``make -C oracle ref``. The package ``__init__`` (which pulls in the
whole pipeline) is not executed. Works only where the reference tree exists.
"""
from __future__ import annotations

import importlib
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
# the reference's package sources: $MVS_REFERENCE_SRC, else the `reference` tree beside this
# repository's root
REF_SRC = os.environ.get("MVS_REFERENCE_SRC",
                         os.path.join(os.path.dirname(os.path.dirname(HERE)), "reference", "orthomosaic"))


def load_densify():
    """Returns the reference's ``densify`` module, or None if the reference is not present."""
    if not os.path.isdir(REF_SRC):
        return None
    from . import oracle as O
    ref = O.reference()
    if ref is None:
        return None
    if "orthomosaic" not in sys.modules:
        pkg = types.ModuleType("orthomosaic")
        pkg.__path__ = [REF_SRC]
        pkg.__package__ = "orthomosaic"
        sys.modules["orthomosaic"] = pkg
        import _mvs  # noqa: F401  (oracle/_ref is on sys.path after O.reference())
        sys.modules["orthomosaic._dense"] = ref._dense
        sys.modules["orthomosaic._fast"] = ref._fast
        sys.modules["orthomosaic._mvs"] = sys.modules["_mvs"]
        try:
            import _core  # noqa: F401  (the backend module imports it; built by make -C oracle ref)
            sys.modules["orthomosaic._core"] = sys.modules["_core"]
        except ImportError:
            pass
    return importlib.import_module("orthomosaic.densify")


def load_module(name: str):
    """Another module of the reference package (e.g. "mvs", "backend"), or None."""
    if load_densify() is None:
        return None
    return importlib.import_module(f"orthomosaic.{name}")
