"""
register_with_reference() against a stand-in of the reference's registry
module (aimd/backends/registry.py:21-39: register_backend keys a class by
its lower-cased ``name``; get_backend looks it up and raises ValueError for
unknown names). The reference itself is not importable where the tests run;
the stand-in has the same interface, which is all the hook uses.
"""

import sys
import types

import pytest

from aimd_b200.backend import ForceBackend, HFGPUBackend, register_with_reference


def _stub_registry():
    reg = types.ModuleType("aimd.backends.registry")
    reg._REGISTRY = {}

    def register_backend(cls):
        key = str(cls.name).strip().lower()
        if not key:
            raise ValueError("backend classes need a name")
        reg._REGISTRY[key] = cls
        return cls

    def get_backend(name):
        key = str(name).strip().lower()
        if key not in reg._REGISTRY:
            raise ValueError(f"Unknown backend '{name}'")
        return reg._REGISTRY[key]

    reg.register_backend = register_backend
    reg.get_backend = get_backend
    pkg = types.ModuleType("aimd")
    pkg.__path__ = []
    sub = types.ModuleType("aimd.backends")
    sub.__path__ = []
    sub.registry = reg
    pkg.backends = sub
    return {"aimd": pkg, "aimd.backends": sub, "aimd.backends.registry": reg}


def test_registers_hf_gpu_in_the_reference_registry(monkeypatch):
    mods = _stub_registry()
    for name, mod in mods.items():
        monkeypatch.setitem(sys.modules, name, mod)
    assert register_with_reference() is True
    reg = mods["aimd.backends.registry"]
    cls = reg.get_backend("HF-GPU")
    assert cls is HFGPUBackend
    # the protocol the reference's integrators and checkpoints rely on
    assert issubclass(cls, ForceBackend)
    assert cls.name == "hf-gpu" and cls.supports_density_guess is True
    for meth in ("compute", "set_density_guess", "close"):
        assert callable(getattr(cls, meth))
    with pytest.raises(ValueError):
        reg.get_backend("no-such-backend")


def test_without_the_reference_nothing_is_registered(monkeypatch):
    for name in ("aimd", "aimd.backends", "aimd.backends.registry"):
        monkeypatch.setitem(sys.modules, name, None)      # import of these names fails
    assert register_with_reference() is False
