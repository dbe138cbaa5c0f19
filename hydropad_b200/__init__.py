"""hydropad_b200 -- Hydropad's PPM hydro step on NVIDIA B200 (sm_100a).

The compute path is the CUDA library ``libhydropad_b200.so`` built from
``csrc/`` (see :mod:`hydropad_b200.build`); there is no CPU fallback.
"""
import importlib

from . import ics  # noqa: F401
from .params import HydroParams  # noqa: F401

__all__ = ["HydroParams", "Hydro", "ics"]


def __getattr__(name):
    if name == "Hydro":
        return importlib.import_module(".api", __name__).Hydro
    raise AttributeError(name)
