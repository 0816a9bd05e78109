"""CPU-only checks of the C ABI boundary (no compute calls): the library loads, exports
every symbol include/ep2d.h declares, its struct layouts match the ctypes mirrors, and
the host-side helpers (pa.dat derivation and reading) behave like the reference."""
import ctypes
import math
import os
import re

import numpy as np
import pytest

import effplast2d_b200 as ep
from effplast2d_b200 import _abi
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions():
    src = open(os.path.join(ROOT, "include", "ep2d.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ep2d_[a-z0-9_]+)\s*\(", src)))


def test_library_exports_every_declared_symbol():
    L = ep.lib()
    names = header_functions()
    assert len(names) >= 18
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert set(names) == set(ep.solver.EXPORTS)


def test_struct_layouts_match():
    out = (ctypes.c_int64 * 7)()
    n = ep.lib().ep2d_abi_sizes(out, 7)
    assert n == 7
    sizes = [ctypes.sizeof(s) for s in (_abi.Params, _abi.StepRecord, _abi.Moduli, _abi.Result, _abi.RveSpec,
                                        _abi.BatchConfig, _abi.BatchStats)]
    assert list(out) == sizes


def test_version_and_device_count():
    assert b"sm_100a" in ep.lib().ep2d_version()
    assert ep.device_count() >= 0


@pytest.mark.parametrize("n,npores,phi,g0,Y", [(128, 1, 0.005, 0.5, 1.0), (1024, 3, 0.01, 0.5, 1e-5),
                                              (2048, 4, 0.02, 0.5, 1e-5), (96, 2, 0.03, 0.01, 1e-5)])
def test_make_pa_matches_get_sigma_restatement(n, npores, phi, g0, Y):
    a = ep.make_pa(20.0, 20.0, n, n, g0=g0, yield_stress=Y, porosity=phi, n_pores=npores)
    b = oracle.make_pa(20.0, 20.0, n, n, g0=g0, yield_stress=Y, porosity=phi, n_pores=npores)
    assert a == b  # bit-identical
    # get_sigma_2D.m:27-29 relations
    dx = 20.0 / (n - 1)
    assert a[0] == dx and a[2] == 0.5 * dx / math.sqrt((1.0 + 4 * g0 / 3) / 1.0)
    assert a[6] == 4.0 / a[2] / n


def test_read_pa_roundtrip_and_errors(tmp_path):
    pa = ep.make_pa(20.0, 20.0, 64, 64, n_pores=2)
    p = tmp_path / "pa.dat"
    ep.write_pa(str(p), pa)
    assert p.stat().st_size == 88
    assert ep.read_pa(str(p)) == pa
    with pytest.raises(ep.EP2DError) as e1:
        ep.read_pa(str(tmp_path / "missing.dat"))
    assert e1.value.status == 3 and "Cannot open file" in str(e1.value)
    short = tmp_path / "short.dat"
    np.zeros(5).tofile(str(short))
    with pytest.raises(ep.EP2DError) as e2:
        ep.read_pa(str(short))
    assert e2.value.status == 3


def test_field_dims_match_reference_arrays():
    L = ep.lib()
    w, h = ctypes.c_int32(), ctypes.c_int32()
    for name, fid in _abi.FIELD_ID.items():
        assert L.ep2d_field_dims(64, 48, fid, ctypes.byref(w), ctypes.byref(h)) == 0
        assert (w.value, h.value) == _abi.field_dims(64, 48, name)
    assert L.ep2d_field_dims(64, 48, 99, ctypes.byref(w), ctypes.byref(h)) == _abi.ERR_ARG


def test_solver_without_device_fails_loudly():
    if ep.device_count() > 0:
        pytest.skip("a CUDA device is present")
    pa = ep.make_pa(20.0, 20.0, 32, 32)
    with pytest.raises(ep.EP2DError) as e:
        ep.Solver(32, 32, pa)
    assert e.value.status == _abi.ERR_NODEV


@pytest.mark.parametrize("bad", ["nan_dx", "nl65", "nl0", "tiny", "side65537", "field_2e31", "zero_pores", "kernel4",
                                 "tile_rows12", "stream_rows2", "stream_rows2048", "resident_rows64", "precision3"])
def test_invalid_params_rejected_before_device(bad):
    # argument validation runs before any device call, so it is testable without a GPU
    pa = ep.make_pa(20.0, 20.0, 32, 32)
    nx, nl = 32, 1
    kw = {"kernel4": dict(kernel=4), "tile_rows12": dict(kernel=ep.KERNEL_TILE, rows=12),
          "resident_rows64": dict(kernel=ep.KERNEL_RESIDENT, rows=64),
          "stream_rows2": dict(kernel=ep.KERNEL_STREAM, rows=2),
          "stream_rows2048": dict(kernel=ep.KERNEL_STREAM, rows=2048),
          "precision3": dict(precision=3)}.get(bad, {})
    if bad == "nan_dx":
        pa[0] = float("nan")
    elif bad == "nl65":  # beyond EP2D_MAX_STEPS (nl 4..64 is the damping mode)
        nl = 65
    elif bad == "nl0":
        nl = 0
    elif bad == "tiny":
        nx = 4
    elif bad == "side65537":  # more than 65536 nodes per side
        nx = 65537
    elif bad == "field_2e31":  # pitch 46,368 x 46,342 rows per field: over the 2^31 index range
        nx = 46341
    elif bad == "zero_pores":
        pa[10] = 0.0
    with pytest.raises(ep.EP2DError) as e:
        ep.Solver(nx, nx, pa, nl=nl, **kw)
    assert e.value.status == _abi.ERR_ARG


def test_batch_and_server_argument_errors():
    # configuration checks happen before any device call
    from effplast2d_b200 import batch as B

    pa = ep.make_pa(20.0, 20.0, 64, 64)
    s = B.spec(64, pa, 2, 1, -6e-5, (1.0, 1.0, 0.0))
    assert B.footprint(s) > 64 * 65 * 8 * 13
    assert B.footprint(s, ep.MIXED) == B.footprint(s)  # same allocation, half of V unused
    with pytest.raises(ep.EP2DError) as e:  # niter not a multiple of check_every
        B.batch_solve([s], niter=1500, check_every=1000)
    assert e.value.status in (_abi.ERR_ARG, _abi.ERR_NODEV)
    with pytest.raises(ep.EP2DError) as e:
        B.batch_solve([s], niter=2000, check_every=1000, rows=12)
    assert e.value.status in (_abi.ERR_ARG, _abi.ERR_NODEV)
    with pytest.raises(ep.EP2DError) as e:  # the resident form is single-RVE only
        B.batch_solve([s], niter=2000, check_every=1000, kernel=ep.KERNEL_RESIDENT)
    assert e.value.status == _abi.ERR_ARG


def test_precisions_accepted_by_validation():
    # FP64, mixed and the FP32 bulk pass argument validation: without a device the
    # failure is the missing device, not the argument
    if ep.device_count() > 0:
        pytest.skip("a CUDA device is present")
    pa = ep.make_pa(20.0, 20.0, 32, 32)
    for prec in (ep.FP64, ep.MIXED, ep.F32_BULK):
        with pytest.raises(ep.EP2DError) as e:
            ep.Solver(32, 32, pa, precision=prec)
        assert e.value.status == _abi.ERR_NODEV, prec
    for rows in (0, 8, 16, 32):  # so does the resident form with a tile height
        with pytest.raises(ep.EP2DError) as e:
            ep.Solver(32, 32, pa, kernel=ep.KERNEL_RESIDENT, rows=rows)
        assert e.value.status == _abi.ERR_NODEV, rows


def test_f32_bulk_footprint_adds_the_perturbation_arrays():
    from effplast2d_b200 import batch as B

    pa = ep.make_pa(20.0, 20.0, 64, 64)
    s = B.spec(64, pa, 2, 1, -6e-5, (1.0, 1.0, 0.0))
    # four float arrays of the common pitch (96 for nx = 64) x 65 rows, 256-byte aligned
    extra = 4 * (((96 * 65 * 4) + 255) // 256 * 256)
    assert B.footprint(s, ep.F32_BULK) == B.footprint(s) + extra


def test_grid_barrier_check_arguments_before_device():
    # the barrier check validates its arguments before any device call
    for kw in (dict(blocks=0), dict(blocks=4, missing=5), dict(blocks=4, rounds=-1),
               dict(blocks=4, rounds=2_000_000), dict(blocks=4, timeout_ns=20_000_000_000)):
        with pytest.raises(ep.EP2DError) as e:
            ep.check_grid_barrier(**kw)
        assert e.value.status == _abi.ERR_ARG, kw
