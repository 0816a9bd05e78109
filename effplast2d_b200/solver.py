"""ctypes binding of libep2d.so (include/ep2d.h).

The library is built in-tree by effplast2d_b200.build (or __graft_entry__.build()).
There is no fallback: without libep2d.so, or without a CUDA device, every solver call
raises.
"""
import ctypes
import os

import numpy as np

from . import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libep2d.so")

_lib = None

# every symbol include/ep2d.h declares
EXPORTS = (
    "ep2d_version", "ep2d_last_error", "ep2d_device_count", "ep2d_read_pa", "ep2d_make_pa",
    "ep2d_field_dims", "ep2d_create", "ep2d_destroy", "ep2d_reset", "ep2d_iterate", "ep2d_get_field",
    "ep2d_set_field", "ep2d_solve_step", "ep2d_get_record", "ep2d_get_check_errors",
    "ep2d_compute_eff_moduli", "ep2d_static_fields", "ep2d_analytic_fields", "ep2d_abi_sizes", "ep2d_get_stats",
    "ep2d_batch_solve", "ep2d_rve_footprint", "ep2d_server_create", "ep2d_server_submit", "ep2d_server_wait",
    "ep2d_server_stats", "ep2d_server_destroy", "ep2d_average_fields_noalloc", "ep2d_get_kernel_shape",
    "ep2d_compute_eff_damping", "ep2d_polar_fields", "ep2d_get_f32_iterations",
    "ep2d_iterate_f32", "ep2d_track_plastic_zone", "ep2d_check_grid_barrier",
)


class EP2DError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("ep2d status %d: %s" % (status, message))
        self.status = status


def lib():
    """Load libep2d.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libep2d.so is not built; run effplast2d_b200.build.build_lib() "
                               "or __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        vp, d, i32, i64 = ctypes.c_void_p, ctypes.c_double, ctypes.c_int32, ctypes.c_int64
        L.ep2d_version.restype = ctypes.c_char_p
        L.ep2d_last_error.restype = ctypes.c_char_p
        L.ep2d_read_pa.argtypes = [ctypes.c_char_p, P(d)]
        L.ep2d_make_pa.argtypes = [d, d, i32, i32, d, d, d, d, d, d, d, P(d)]
        L.ep2d_field_dims.argtypes = [i32, i32, i32, P(i32), P(i32)]
        L.ep2d_create.argtypes = [P(_abi.Params), P(vp)]
        L.ep2d_destroy.argtypes = [vp]
        L.ep2d_reset.argtypes = [vp]
        L.ep2d_iterate.argtypes = [vp, i64]
        L.ep2d_get_field.argtypes = [vp, i32, P(d)]
        L.ep2d_set_field.argtypes = [vp, i32, P(d)]
        L.ep2d_solve_step.argtypes = [vp, i32, d, P(d), i32, P(_abi.StepRecord)]
        L.ep2d_get_record.argtypes = [vp, i32, i32, P(_abi.StepRecord)]
        L.ep2d_get_check_errors.argtypes = [vp, i32, i32, P(d), i32, P(i32)]
        L.ep2d_compute_eff_moduli.argtypes = [vp, d, P(d), i32, P(_abi.Result)]
        L.ep2d_static_fields.argtypes = [vp, P(d), P(d), P(d)]
        L.ep2d_analytic_fields.argtypes = [vp, d, d] + [P(d)] * 7
        L.ep2d_abi_sizes.argtypes = [P(i64), i32]
        L.ep2d_get_stats.argtypes = [vp, P(d), P(i64), P(i64), P(i64)]
        L.ep2d_get_f32_iterations.argtypes = [vp, P(i64)]
        L.ep2d_iterate_f32.argtypes = [vp, i64]
        L.ep2d_track_plastic_zone.argtypes = [vp, i32]
        L.ep2d_batch_solve.argtypes = [P(_abi.BatchConfig), P(_abi.RveSpec), i32, P(_abi.Result),
                                       P(_abi.BatchStats)]
        L.ep2d_rve_footprint.argtypes = [P(_abi.RveSpec), i32]
        L.ep2d_rve_footprint.restype = i64
        L.ep2d_server_create.argtypes = [P(_abi.BatchConfig), i64, i32, P(vp)]
        L.ep2d_server_submit.argtypes = [vp, P(_abi.RveSpec), P(ctypes.c_uint64)]
        L.ep2d_server_wait.argtypes = [vp, ctypes.c_uint64, i32, P(i32), P(_abi.Result), P(d), P(d)]
        L.ep2d_server_stats.argtypes = [vp, P(i64), P(i64), P(i64), P(i64), P(_abi.BatchStats)]
        L.ep2d_server_destroy.argtypes = [vp]
        L.ep2d_average_fields_noalloc.argtypes = [i32, i32, P(d)] + [vp] * 8
        L.ep2d_get_kernel_shape.argtypes = [vp, P(i32), P(i32)]
        L.ep2d_compute_eff_damping.argtypes = [vp, d, P(d), i32, d, P(i64)]
        L.ep2d_polar_fields.argtypes = [vp, d] + [P(d)] * 4 + [P(ctypes.c_uint8)]
        L.ep2d_check_grid_barrier.argtypes = [i32, i32, i32, i32, i64, P(i32), P(i32)]
        _lib = L
    return _lib


def _check(rc):
    if rc != 0:
        raise EP2DError(rc, lib().ep2d_last_error().decode(errors="replace"))


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def device_count():
    return int(lib().ep2d_device_count())


def check_grid_barrier(blocks, missing=0, rounds=4, timeout_ns=1_000_000, device=0):
    """The resident form's grid barrier alone (ep2d_check_grid_barrier): `blocks` CTAs
    meet `rounds` times, `missing` of them never arrive.  Returns (CTAs that passed every
    round, error flag)."""
    passed, flag = ctypes.c_int32(), ctypes.c_int32()
    _check(lib().ep2d_check_grid_barrier(int(device), int(blocks), int(missing), int(rounds), int(timeout_ns),
                                         ctypes.byref(passed), ctypes.byref(flag)))
    return passed.value, flag.value


def make_pa(lx, ly, nx, ny, k0=1.0, g0=0.5, rho0=1.0, cfl=0.5, yield_stress=1.0, porosity=0.005,
            n_pores=1):
    """pa.dat values (get_sigma_2D.m:3-32) computed by the library."""
    out = np.zeros(_abi.NPARS)
    _check(lib().ep2d_make_pa(lx, ly, nx, ny, k0, g0, rho0, cfl, yield_stress, porosity,
                              float(n_pores), _dptr(out)))
    return out.tolist()


def read_pa(path):
    out = np.zeros(_abi.NPARS)
    _check(lib().ep2d_read_pa(os.fsencode(path), _dptr(out)))
    return out.tolist()


def write_pa(path, pa):
    np.asarray(pa, dtype="<f8").tofile(path)


class Solver:
    """One RVE on the GPU (an ep2d_handle): the reference's EffPlast2D object."""

    def __init__(self, nx, ny, pa, nl=1, niter=100000, eiter=1e-9, check_every=10000, device=0,
                 precision=_abi.FP64, kernel=_abi.KERNEL_AUTO, rows=0):
        self.nx, self.ny = int(nx), int(ny)
        self.params = _abi.make_params(nx, ny, pa, nl=nl, niter=niter, eiter=eiter,
                                       check_every=check_every, precision=precision, device=device,
                                       kernel=kernel, rows=rows)
        h = ctypes.c_void_p()
        _check(lib().ep2d_create(ctypes.byref(self.params), ctypes.byref(h)))
        self._h = h

    def close(self):
        if getattr(self, "_h", None):
            lib().ep2d_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def dims(self, field):
        return _abi.field_dims(self.nx, self.ny, field)

    def get(self, field):
        w, h = self.dims(field)
        a = np.empty((h, w), dtype=np.float64)
        _check(lib().ep2d_get_field(self._h, _abi.FIELD_ID[field], _dptr(a)))
        return a

    def set(self, field, arr):
        w, h = self.dims(field)
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(h, w)
        _check(lib().ep2d_set_field(self._h, _abi.FIELD_ID[field], _dptr(a)))

    def reset(self):
        _check(lib().ep2d_reset(self._h))

    def iterate(self, n):
        _check(lib().ep2d_iterate(self._h, int(n)))

    def track_plastic_zone(self, on=True):
        """get_sigma_2D.m's plastic zone: mark every node / corner that yields at any
        iteration from now on (on=True clears the marks); polar_fields then uses them"""
        _check(lib().ep2d_track_plastic_zone(self._h, 1 if on else 0))

    def iterate_f32(self, n):
        """n iterations of the FP32 bulk's FP32 form (precision=F32_BULK handles)"""
        _check(lib().ep2d_iterate_f32(self._h, int(n)))

    def solve_step(self, step, load_step_value, load_type, n_time_steps=1):
        lt = np.asarray(load_type, dtype=np.float64)
        recs = (_abi.StepRecord * n_time_steps)()
        _check(lib().ep2d_solve_step(self._h, int(step), float(load_step_value), _dptr(lt),
                                     int(n_time_steps), recs))
        return [r.as_dict() for r in recs]

    def record(self, step, time_step):
        r = _abi.StepRecord()
        _check(lib().ep2d_get_record(self._h, int(step), int(time_step), ctypes.byref(r)))
        return r.as_dict()

    def check_errors(self, step, time_step):
        n = ctypes.c_int32()
        _check(lib().ep2d_get_check_errors(self._h, int(step), int(time_step), None, 0, ctypes.byref(n)))
        buf = np.zeros(max(n.value, 1))
        _check(lib().ep2d_get_check_errors(self._h, int(step), int(time_step), _dptr(buf), n.value,
                                           ctypes.byref(n)))
        return buf[: n.value].tolist()

    def compute_eff_moduli(self, init_load_value, load_type, n_time_steps=1):
        lt = np.asarray(load_type, dtype=np.float64)
        res = _abi.Result()
        _check(lib().ep2d_compute_eff_moduli(self._h, float(init_load_value), _dptr(lt),
                                             int(n_time_steps), ctypes.byref(res)))
        return res.as_dict()

    def compute_eff_damping(self, init_load_value, load_type, n_time_steps, load_value):
        """ComputeEffDamping (nl >= 4): returns the total iteration count; the strain and
        stress tensors are the records of (0, n_time_steps-1) and (i, 0)."""
        lt = np.asarray(load_type, dtype=np.float64)
        tot = ctypes.c_int64()
        _check(lib().ep2d_compute_eff_damping(self._h, float(init_load_value), _dptr(lt), int(n_time_steps),
                                              float(load_value), ctypes.byref(tot)))
        return tot.value

    def static_fields(self):
        nx, ny = self.nx, self.ny
        unu = np.zeros((ny, nx))
        j1 = np.zeros((ny - 1, nx - 1))
        j2 = np.zeros((ny - 1, nx - 1))
        _check(lib().ep2d_static_fields(self._h, _dptr(unu), _dptr(j1), _dptr(j2)))
        return {"UnuAbs": unu, "J1nu": j1, "J2nu": j2}

    def polar_fields(self, load_value):
        """get_sigma_2D.m:170-194 on the recorded state: dict of Snurr, Snuff, Sanrr, Sanff
        ((ny, nx) doubles) and Plast ((ny, nx) uint8 counts)."""
        nx, ny = self.nx, self.ny
        out = {k: np.zeros((ny, nx)) for k in ("Snurr", "Snuff", "Sanrr", "Sanff")}
        pl = np.zeros((ny, nx), dtype=np.uint8)
        _check(lib().ep2d_polar_fields(self._h, float(load_value), *[_dptr(out[k]) for k in
                                                                     ("Snurr", "Snuff", "Sanrr", "Sanff")],
                                       pl.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        out["Plast"] = pl
        return out

    def analytic_fields(self, delta_p, tau_infty):
        nx, ny = self.nx, self.ny
        out = {k: np.zeros((ny, nx)) for k in ("UanAbs", "errorUabs")}
        out.update({k: np.zeros((ny - 1, nx - 1)) for k in ("J1an", "J2an", "errorJ1", "errorJ2")})
        st = np.zeros(6)
        _check(lib().ep2d_analytic_fields(self._h, float(delta_p), float(tau_infty),
                                          *[_dptr(out[k]) for k in ("UanAbs", "errorUabs", "J1an", "J2an",
                                                                     "errorJ1", "errorJ2")], _dptr(st)))
        out["stats"] = st
        return out

    def stats(self):
        ms = ctypes.c_double()
        la, cu, al = ctypes.c_int64(), ctypes.c_int64(), ctypes.c_int64()
        _check(lib().ep2d_get_stats(self._h, ctypes.byref(ms), ctypes.byref(la), ctypes.byref(cu),
                                    ctypes.byref(al)))
        f32 = ctypes.c_int64()
        _check(lib().ep2d_get_f32_iterations(self._h, ctypes.byref(f32)))
        return {"kernel_ms": ms.value, "launches": la.value, "cell_updates": cu.value,
                "all_launches": al.value, "f32_iterations": f32.value}

    def kernel_shape(self):
        """(kernel form, rows) of the iteration kernel this solver launches"""
        k, r = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().ep2d_get_kernel_shape(self._h, ctypes.byref(k), ctypes.byref(r)))
        return k.value, r.value
