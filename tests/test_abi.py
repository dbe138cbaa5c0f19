"""The C ABI library loads without a GPU and exports every function the
public header declares; without a device the product path fails loudly."""
import ctypes as C
import glob
import os
import re
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        names.update(re.findall(r"\b(hp_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_declares_entry_points():
    names = declared_functions()
    for must in ("hp_init", "hp_ppmsolver", "hp_ppm_lxlylz", "hp_speed", "hp_timedet", "hp_evolve",
                 "hp_attach_state", "hp_sync_to_host", "hp_finalize", "hp_strerror"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from hydropad_b200.build import LIB_PATH
    assert os.path.exists(LIB_PATH), "build the library first (python -m hydropad_b200.build)"
    out = subprocess.run(["nm", "-D", "--defined-only", LIB_PATH], capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r"\bT (hp_[a-z0-9_]+)\b", out))
    missing = [n for n in declared_functions() if n not in exported]
    assert not missing, missing


def test_library_loads_and_binds():
    from hydropad_b200 import _lib
    L = _lib.lib()
    for name in _lib.EXPORTS:
        assert hasattr(L, name)
    assert L.hp_strerror(-4).decode().startswith("Riemann Newton")


def test_no_device_is_an_error_not_a_fallback():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from hydropad_b200._lib import HydroError
    from hydropad_b200.api import Hydro
    from hydropad_b200.params import HydroParams
    with pytest.raises(HydroError, match="NO_DEVICE"):
        Hydro(HydroParams(shape=(16, 16, 16)))
