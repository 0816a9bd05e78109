"""effplast2d_b200 -- B200-native (sm_100a) pseudo-transient elastoplastic RVE solver.

A from-scratch implementation of the GPU calculation of beacon1143/EffPlast2D behind
its own entry points: the C ABI of include/ep2d.h (libep2d.so), the drop-in C++
`EffPlast2D` class and CLI (csrc/dropin), and this Python binding.
"""
from ._abi import FIELDS, FP64, KERNEL_AUTO, KERNEL_STREAM, KERNEL_TILE, MIXED, field_dims  # noqa: F401
from .solver import (EP2DError, Solver, device_count, lib, make_pa, read_pa,  # noqa: F401
                     write_pa)

__version__ = "0.1.0"
