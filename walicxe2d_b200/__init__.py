"""walicxe2d_b200 -- B200 (sm_100a) block-update path of Walicxe-2D.

The per-timestep work of the reference's ``tstep``/``timestep`` (Hancock
half and full steps, Riemann fluxes, slope limiters, viscosity, the CFL
reduction, the intra-grid ghost fills, refine/coarse data motion and the
cooling source terms) runs as hand-written CUDA kernels behind the C-ABI of
``include/w2d.h``; this package is its Python binding.
"""
from .params import (W2dError, W2dInit, W2dParams, base_params, config, sedov,  # noqa: F401
                     scalings)

__all__ = ["W2dParams", "W2dInit", "W2dError", "base_params", "config", "sedov", "scalings",
           "Context", "Simulation", "load"]


def load():
    """Loads the native library (raises if it is missing)."""
    from . import _lib
    return _lib.load()


def __getattr__(name):
    if name in ("Context", "Simulation"):
        from . import api
        return getattr(api, name)
    raise AttributeError(name)
