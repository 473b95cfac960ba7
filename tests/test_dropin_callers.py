"""The drop-in classes accept every call the reference's own callers make.

The reference's alignment driver and benchmark (src/matcha/align_subtomograms.py,
src/matcha/example.py, src/matcha/utils/run_utils.py) construct the hot-path classes and call
their methods; after ``matcha_b200.shim.install()`` those calls land on this package.  This
test reads the callers' source (a checkout named by MATCHA_REFERENCE_ROOT; skipped without
one), finds every constructor and method call of the replaced classes, and binds its
positional count and keyword names against the signatures here, so a caller's argument the
drop-in does not take fails here and not in an alignment run.  It needs no GPU: binding a
signature runs nothing.
"""
import ast
import inspect
import os

import pytest

REF = os.environ.get("MATCHA_REFERENCE_ROOT")
CALLERS = ["src/matcha/align_subtomograms.py", "src/matcha/example.py", "src/matcha/utils/run_utils.py"]


def _classes():
    from matcha_b200.core.CrossCorrelationMatcher import CrossCorrelationMatcher
    from matcha_b200.core.FLEBasis3D import FLEBasis3D
    from matcha_b200.core.Matcha import Matcha
    from matcha_b200.core.ShiftMatcher import ShiftMatcher
    from matcha_b200.core.SOFFT import SOFFT

    return {c.__name__: c for c in (CrossCorrelationMatcher, FLEBasis3D, Matcha, ShiftMatcher, SOFFT)}


# methods of the replaced classes the callers use, by name
METHODS = {"get_sigma": "CrossCorrelationMatcher", "set_template": "CrossCorrelationMatcher",
           "search_orientations": "Matcha", "set_reference": "ShiftMatcher", "search_shifts": "ShiftMatcher",
           "get_base_shifts": "ShiftMatcher", "evaluate_t": "FLEBasis3D"}


def _calls(tree):
    for node in ast.walk(tree):
        if isinstance(node, ast.Call):
            f = node.func
            name = f.id if isinstance(f, ast.Name) else f.attr if isinstance(f, ast.Attribute) else None
            if name:
                yield name, node


def _bind(fn, node, skip_self=False):
    n_pos = len(node.args)
    if any(isinstance(a, ast.Starred) for a in node.args) or any(k.arg is None for k in node.keywords):
        return  # *args / **kwargs forwarding: nothing static to check
    sig = inspect.signature(fn)
    params = list(sig.parameters.values())
    if skip_self:
        params = params[1:]
    sig = sig.replace(parameters=params)
    sig.bind_partial(*([None] * n_pos), **{k.arg: None for k in node.keywords})


@pytest.mark.skipif(not REF, reason="MATCHA_REFERENCE_ROOT names no checkout of the reference")
def test_reference_callers_bind_to_the_drop_in_signatures():
    classes = _classes()
    seen = set()
    for rel in CALLERS:
        path = os.path.join(REF, rel)
        tree = ast.parse(open(path, encoding="utf-8").read(), path)
        for name, node in _calls(tree):
            where = f"{rel}:{node.lineno}"
            if name in classes:
                _bind(classes[name].__init__, node, skip_self=True)
                seen.add(name)
            elif name in METHODS and isinstance(node.func, ast.Attribute):
                _bind(getattr(classes[METHODS[name]], name), node, skip_self=True)
                seen.add(name)
            del where
    # the alignment driver builds all three matchers and calls the search and the shift match
    assert {"CrossCorrelationMatcher", "Matcha", "ShiftMatcher", "get_sigma", "search_orientations",
            "search_shifts", "set_reference", "set_template"} <= seen, seen


def test_recorded_driver_calls_bind_to_the_drop_in_signatures():
    """The calls of the reference's driver recorded in caller_trace.npz (make_caller_trace.py)
    bind to the drop-in signatures by keyword, as the driver made them; the GPU replay of the
    same trace is tests/test_caller_trace_gpu.py."""
    import json

    from tests.helpers import golden

    classes = _classes()
    z = golden("caller_trace.npz")
    events = json.loads(str(z["events"]))
    calls = [e["call"] for e in events]
    assert calls[:6] == ["Matcha", "ShiftMatcher", "CrossCorrelationMatcher", "CrossCorrelationMatcher.set_template",
                         "ShiftMatcher.set_reference", "ShiftMatcher.get_base_shifts"], calls
    assert calls[6:] == ["CrossCorrelationMatcher.get_sigma", "Matcha.search_orientations",
                         "ShiftMatcher.search_shifts"] * 2, calls
    for e in events:
        cls, _, meth = e["call"].partition(".")
        fn = getattr(classes[cls], meth) if meth else classes[cls].__init__
        sig = inspect.signature(fn)
        sig = sig.replace(parameters=list(sig.parameters.values())[1:])
        sig.bind(**{k: None for k in e["args"]})
