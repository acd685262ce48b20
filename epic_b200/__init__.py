"""B200-native EPIC 3-D parcel step.

The compute path is the CUDA library ``libepic_b200.so`` (hand-written
sm_100a kernels behind the C ABI of include/epic_gpu.h).  There is no CPU
fallback: ``load()`` fails loudly when the library is missing.
"""
from __future__ import annotations

import os

from .abi import EpicContext, EpicError, EpicLib  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libepic_b200.so")

_LIB = None


def load() -> EpicLib:
    """The CUDA library bound through ctypes (prefix epic_gpu_)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build the CUDA library with "
                "`python -m epic_b200.build` (no CPU fallback exists)")
        _LIB = EpicLib(LIB_PATH, "epic_gpu_")
    return _LIB


def make_context(setup, lib: EpicLib | None = None, **overrides) -> EpicContext:
    """Create a context for a Setup (epic_b200.initial) and load its parcels."""
    lib = lib or load()
    opts = dict(setup.options)
    opts.update(overrides)
    cfg = lib.default_config(setup.nx, setup.ny, setup.nz, setup.lower, setup.extent, **opts)
    ctx = EpicContext(lib, cfg)
    ctx.set_parcels(*setup.arrays())
    ctx.init_correction()
    return ctx


def make_context_device(spec, lib: EpicLib | None = None, **overrides) -> EpicContext:
    """Create a context for an initial.DeviceSpec: the parcels are generated on
    the device (epic_gpu_init_state), then init_correction."""
    lib = lib or load()
    opts = dict(spec.options)
    opts.update(overrides)
    cfg = lib.default_config(spec.nx, spec.ny, spec.nz, spec.lower, spec.extent, **opts)
    ctx = EpicContext(lib, cfg)
    ctx.init_state(spec.init_spec())
    ctx.init_correction()
    return ctx
