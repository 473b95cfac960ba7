"""The reference's hot-path imports resolve to matcha_b200 after shim.install()."""
import sys
import types

from matcha_b200 import shim


def test_install_routes_reference_modules(monkeypatch):
    # parents as the installed reference would provide them
    for name in ("matcha", "matcha.core"):
        if name not in sys.modules:
            mod = types.ModuleType(name)
            mod.__path__ = []
            monkeypatch.setitem(sys.modules, name, mod)
    for name in shim.ALIASES:
        monkeypatch.delitem(sys.modules, name, raising=False)
    done = shim.install()
    try:
        from matcha.core.CrossCorrelationMatcher import CrossCorrelationMatcher
        from matcha.core.Matcha import Matcha
        from matcha.core.ShiftMatcher import ShiftMatcher

        import matcha_b200.core.CrossCorrelationMatcher as C
        import matcha_b200.core.Matcha as M
        import matcha_b200.core.ShiftMatcher as S

        assert Matcha is M.Matcha and CrossCorrelationMatcher is C.CrossCorrelationMatcher
        assert ShiftMatcher is S.ShiftMatcher
        assert set(done) == set(shim.ALIASES)
    finally:
        shim.uninstall()
    assert "matcha.core.Matcha" not in sys.modules


def test_bench_cases_need_a_device(monkeypatch):
    import torch

    import bench_cases as profile_cases

    monkeypatch.setattr(torch.cuda, "is_available", lambda: False)
    assert profile_cases.main(["shift", "2"]) == 2
    assert set(profile_cases.CASES) == {"shift", "search", "fle", "prepare", "reader", "graph", "fftbound"}
