"""The scratch-free averaging entry point (ep2d_average_fields_noalloc).

It serves callers that must not call cudaMalloc because their device memory belongs to
their own allocator: the caller passes device arrays it already owns -- here allocated
by torch, as such a framework would -- and the reduction's scratch lives in a fixed
device array inside the library.  Its output must equal what the library's ordinary
path records for the same state (ep2d_solve_step's sigma, sigma_per and eps_per), within
the 1e-9 the chain tests use, on two calls in a row (the second call reuses the scratch
the first left behind), and a grid beyond the array's capacity must be refused before
anything reaches the GPU.  This file is collected last so that a failure here cannot
hide the results of the other GPU tests.
"""
import ctypes
import math

import numpy as np
import pytest

import effplast2d_b200 as ep
from effplast2d_b200 import _abi

pytestmark = pytest.mark.gpu

FIELDS = ("P", "tauXX", "tauYY", "tauXY", "Ux", "Uy")


def _close(a, b, scale):
    return abs(a - b) <= 1e-9 * abs(b) + 1e-9 * scale


# square, and rectangular both ways: a swap of nx and ny in the reference-layout strides
# (tauXY nx-1, Ux nx+1, Uy nx per row) shows on a rectangle
@pytest.mark.parametrize("nx,ny", [(96, 96), (96, 64), (64, 96)])
def test_noalloc_average_matches_recorded_averages(nx, ny):
    import torch

    pa = ep.make_pa(20.0, 20.0, nx, ny, g0=0.5, yield_stress=1e-5, porosity=0.02, n_pores=3)
    s = ep.Solver(nx, ny, pa, nl=2, niter=3000, eiter=1e-9, check_every=1000)
    s.compute_eff_moduli(-6e-5, [1.0, 0.8, 0.3], 1)
    rec = s.record(1, 0)  # the state the fields hold now: end of the last load step
    dev = {f: torch.from_numpy(np.ascontiguousarray(s.get(f))).to("cuda") for f in FIELDS}
    out = torch.full((11,), float("nan"), dtype=torch.float64, device="cuda")
    pa_c = (ctypes.c_double * 11)(*pa)
    expect = list(rec["sigma"]) + list(rec["sigma_per"]) + list(rec["eps_per"])
    stress_scale = max(abs(v) for v in rec["sigma"] + rec["sigma_per"])
    strain_scale = max(abs(v) for v in rec["macro_strain"])
    L = ep.lib()
    for call in range(2):
        rc = L.ep2d_average_fields_noalloc(nx, ny, pa_c, *[ctypes.c_void_p(dev[f].data_ptr()) for f in FIELDS],
                                           ctypes.c_void_p(out.data_ptr()), None)
        assert rc == 0, L.ep2d_last_error()
        torch.cuda.synchronize()
        got = out.cpu().tolist()
        for k, (a, b) in enumerate(zip(got, expect)):
            scale = strain_scale if k >= 8 else stress_scale
            assert math.isfinite(a) and _close(a, b, scale), (call, k, a, b)
        out.fill_(float("nan"))


def test_noalloc_average_rejects_grids_beyond_its_scratch():
    L = ep.lib()
    pa = ep.make_pa(20.0, 20.0, 64, 9000)
    pa_c = (ctypes.c_double * 11)(*pa)
    fake = ctypes.c_void_p(1)  # never dereferenced: the size check comes first
    rc = L.ep2d_average_fields_noalloc(64, 9000, pa_c, *([fake] * 6), fake, None)
    assert rc == _abi.ERR_ARG
    assert b"8194" in L.ep2d_last_error()


def test_noalloc_average_rejects_bad_parameters():
    L = ep.lib()
    fake = ctypes.c_void_p(1)  # never dereferenced: the checks come first
    for k, v in ((0, 0.0), (1, -1.0), (10, 65.0), (10, 0.5)):
        pa = ep.make_pa(20.0, 20.0, 64, 64)
        pa[k] = v
        pa_c = (ctypes.c_double * 11)(*pa)
        assert L.ep2d_average_fields_noalloc(64, 64, pa_c, *([fake] * 6), fake, None) == _abi.ERR_ARG, (k, v)
