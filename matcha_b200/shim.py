"""Route the reference's hot-path imports to matcha_b200.

    import matcha_b200.shim
    matcha_b200.shim.install()
    # from here on, ``from matcha.core.Matcha import Matcha`` (and the other hot-path
    # modules) resolve to the B200 implementations

Only the modules of the alignment hot path are replaced:

    matcha.core.Matcha                  -> matcha_b200.core.Matcha
    matcha.core.SOFFT                   -> matcha_b200.core.SOFFT
    matcha.core.FLEBasis3D              -> matcha_b200.core.FLEBasis3D
    matcha.core.CrossCorrelationMatcher -> matcha_b200.core.CrossCorrelationMatcher
    matcha.core.ShiftMatcher            -> matcha_b200.core.ShiftMatcher

The reference's orchestration, I/O, CLI and RELION glue (matcha.run, matcha.utils.*,
matcha.align_subtomograms) keep running unchanged on top of them.  Call ``install``
before those modules are first imported.
"""
from __future__ import annotations

import importlib
import sys

ALIASES = {
    "matcha.core.Matcha": "matcha_b200.core.Matcha",
    "matcha.core.SOFFT": "matcha_b200.core.SOFFT",
    "matcha.core.FLEBasis3D": "matcha_b200.core.FLEBasis3D",
    "matcha.core.CrossCorrelationMatcher": "matcha_b200.core.CrossCorrelationMatcher",
    "matcha.core.ShiftMatcher": "matcha_b200.core.ShiftMatcher",
}


def install(force: bool = False) -> dict:
    """Register the aliases in sys.modules; returns {reference name: module}."""
    done = {}
    for ref_name, ours in ALIASES.items():
        if ref_name in sys.modules and not force:
            mod = sys.modules[ref_name]
            if getattr(mod, "__name__", "") != ours:
                raise RuntimeError(f"{ref_name} was imported before matcha_b200.shim.install(); call it earlier")
        mod = importlib.import_module(ours)
        sys.modules[ref_name] = mod
        done[ref_name] = mod
    return done


def uninstall() -> None:
    for ref_name, ours in ALIASES.items():
        mod = sys.modules.get(ref_name)
        if mod is not None and getattr(mod, "__name__", "") == ours:
            del sys.modules[ref_name]
