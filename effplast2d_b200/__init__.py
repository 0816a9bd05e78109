"""effplast2d_b200 -- B200-native (sm_100a) pseudo-transient elastoplastic RVE solver.

A from-scratch implementation of the GPU calculation of beacon1143/EffPlast2D behind
its own entry points: the C ABI of include/ep2d.h (libep2d.so), the drop-in C++
`EffPlast2D` class and CLI (csrc/dropin), and this Python binding.
"""
from ._abi import (ERR_ARG, ERR_CUDA, ERR_IO, ERR_NODEV, ERR_NOMEM, ERR_RANGE, ERR_STATE, F32_BULK, FIELDS, FP64,  # noqa: F401
                   KERNEL_AUTO, KERNEL_RESIDENT, KERNEL_STREAM, KERNEL_TILE, MIXED, field_dims)
from .solver import (EP2DError, Solver, check_grid_barrier, device_count, lib, make_pa,  # noqa: F401
                     read_pa, write_pa)

__version__ = "0.1.0"
