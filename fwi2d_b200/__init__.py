"""fwi2d_b200 — B200-native (sm_100a) wave-propagation engine with the
capabilities of phbastosa/FWI2D's modeling / migration / inversion path.

The product is ``libfwi2d.so`` (C ABI in include/fwi2d.h) and the three
drop-in executables under ``bin/``; this package binds the ABI for Python.
"""
from .api import (  # noqa: F401
    MODE_INVERSION, MODE_MIGRATION, MODE_MODELING, Context, FwiError, Inversion, Migration, Modeling, lib,
    load_library, LIB_PATH, SIGNATURES,
)
