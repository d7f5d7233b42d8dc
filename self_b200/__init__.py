"""self_b200: a B200-native (sm_100a) engine for SELF's 2-D DGSEM tendency path.

The compute lives in ``libselfgpu.so`` (CUDA, built in-tree by
``self_b200.build``); this package is the host-side mirror of SELF's
Lagrange / Mesh2D / SEMQuad / Model2D API over that library's C ABI.
"""
from ._lib import SelfGpuError, check, exported_symbols, lib  # noqa: F401
from .api import (BC_NONORMALFLOW, BC_PRESCRIBED, BC_RADIATION, CLOSURE_INDICATOR, CLOSURE_MLP,  # noqa: F401
                  CLOSURE_OFF, FP32_BULK, FP64, FP64_REF, GAUSS, GAUSS_LOBATTO, MODEL_CIG, MODEL_LSW, MODEL_SW, UNIFORM, CompressibleIdealGas2D, Lagrange,
                  LinearShallowWater, Mesh2D, Model2D, SEMQuad, ShallowWater, to_device, to_host)
from .fields import MappedScalar2D, MappedVector2D, Scalar2D, Vector2D  # noqa: F401,E402
