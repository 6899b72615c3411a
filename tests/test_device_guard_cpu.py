"""Every C entry point that launches work runs with the wrapper's device current.

The library launches on the calling thread's current CUDA device; the Python
wrappers pass buffers and a stream of their own device.  These CPU tests
check the guard itself with a fake library and a fake device context, and
check by reading the package source that no device-launching entry point is
called without it.
"""

from __future__ import annotations

import ast
import contextlib
from pathlib import Path

import pytest

from critmc_b200 import _lib

PKG = Path(_lib.__file__).resolve().parent


def test_call_on_makes_the_device_current(monkeypatch):
    import torch

    current = {"dev": 0}
    seen = []

    @contextlib.contextmanager
    def fake_device(dev):
        prev = current["dev"]
        current["dev"] = torch.device(dev).index
        try:
            yield
        finally:
            current["dev"] = prev

    class FakeLib:
        def __getattr__(self, name):
            def fn(*args):
                seen.append((name, current["dev"], args))
                return 0
            return fn

    monkeypatch.setattr(torch.cuda, "device", fake_device)
    monkeypatch.setattr(_lib, "lib", lambda: FakeLib())
    _lib.call_on(torch.device("cuda", 3), "critmc_ising_msc_run", 1, 2)
    _lib.call_on(torch.device("cuda", 1), "critmc_on_run", 5)
    assert seen == [("critmc_ising_msc_run", 3, (1, 2)), ("critmc_on_run", 1, (5,))]
    assert current["dev"] == 0, "the previous device is restored after the call"


def test_call_on_restores_the_device_when_the_call_fails(monkeypatch):
    import torch

    current = {"dev": 0}

    @contextlib.contextmanager
    def fake_device(dev):
        prev = current["dev"]
        current["dev"] = torch.device(dev).index
        try:
            yield
        finally:
            current["dev"] = prev

    class FailingLib:
        def __getattr__(self, name):
            if name == "critmc_last_error":
                return lambda buf, n: 0
            return lambda *a: -1

    monkeypatch.setattr(torch.cuda, "device", fake_device)
    monkeypatch.setattr(_lib, "lib", lambda: FailingLib())
    with pytest.raises(_lib.CritmcError):
        _lib.call_on(torch.device("cuda", 2), "critmc_potts_run")
    assert current["dev"] == 0


def _lib_calls(tree):
    for node in ast.walk(tree):
        if not isinstance(node, ast.Call) or not isinstance(node.func, ast.Attribute):
            continue
        f = node.func
        if isinstance(f.value, ast.Name) and f.value.id == "_lib" and f.attr in ("call", "call_on"):
            yield node


def test_every_device_launching_entry_point_is_called_through_the_guard():
    unguarded, unknown = [], []
    for path in sorted(PKG.glob("*.py")):
        if path.name == "_lib.py":
            continue
        tree = ast.parse(path.read_text())
        for node in _lib_calls(tree):
            args = node.args if node.func.attr == "call" else node.args[1:]
            if not args or not isinstance(args[0], ast.Constant):
                unknown.append(f"{path.name}:{node.lineno}")
                continue
            name = args[0].value
            if name not in _lib.SIGNATURES:
                unknown.append(f"{path.name}:{node.lineno} {name}")
            if node.func.attr == "call" and name not in _lib.HOST_ONLY:
                unguarded.append(f"{path.name}:{node.lineno} {name}")
    assert not unknown, f"calls whose entry point is not in the ABI table: {unknown}"
    assert not unguarded, f"device-launching entry points called without call_on: {unguarded}"


def test_host_only_entry_points_are_in_the_abi_table():
    assert _lib.HOST_ONLY <= set(_lib.SIGNATURES)
