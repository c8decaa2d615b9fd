"""hpcg_b200: the HPCG 3.1 preconditioned-CG path on NVIDIA B200 (sm_100a).

The product is the C-ABI library ``libhpcg_b200.so`` (declared in
``include/hpcg_b200.h``) and the C++ drop-in translation unit
``dropin/hpcg_dropin.cpp`` that binds the reference's entry points to it.
This package adds a Python binding of the same C ABI (``binding``).
"""
from .binding import (  # noqa: F401
    ComputeDotProduct, ComputeResidual, ComputeWAXPBY, HpcgError, Problem, lib, last_error,
    SYMGS_COLOUR, SYMGS_NATURAL,
)

__all__ = ["Problem", "ComputeDotProduct", "ComputeWAXPBY", "ComputeResidual", "HpcgError", "lib",
           "last_error", "SYMGS_COLOUR", "SYMGS_NATURAL"]
