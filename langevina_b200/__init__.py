"""B200-native (sm_100a) Model A / Model G stepper and measurer for langevinA.

The compute lives in liblgv.so (include/lgv.h); this package is its Python
host mirror.  Importing it loads the library and raises if it is missing.
"""
from . import _lib
from ._lib import LgvError, Measurement, load, make_params  # noqa: F401
from .model import (EulerLangevinHB, IdealEulerMaruyama, IdealPV2, Measurer, ModelA, ModelAData,  # noqa: F401
                    ModelAEulerMaruyama, ModelGChargeHB, PV2HBSplit, Stepper, make_stepper)

lib = load()
