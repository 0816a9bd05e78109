"""CPU oracle for the EffPlast2D solver -- TEST INFRASTRUCTURE ONLY.

Python access to liboracle.so (ep2d_oracle.c, the plain-C FP64 restatement of the
reference's EffPlast2D.cu) and to the reference's own binaries under oracle/_ref.
Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this module,
and only to check results or time the CPU baseline.  The product package never imports it.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

from effplast2d_b200 import _abi

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_lib = None


def build():
    """Build liboracle.so (gcc) with the committed Makefile."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = ctypes.CDLL(LIB_PATH)
        P = ctypes.POINTER
        vp = ctypes.c_void_p
        d = ctypes.c_double
        i32 = ctypes.c_int32
        L.orc_create.argtypes = [P(_abi.Params), P(vp)]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_iterate.argtypes = [vp, ctypes.c_int64]
        L.orc_get_field.argtypes = [vp, i32, P(d)]
        L.orc_set_field.argtypes = [vp, i32, P(d)]
        L.orc_solve_step.argtypes = [vp, i32, d, P(d), i32, P(_abi.StepRecord)]
        L.orc_get_record.argtypes = [vp, i32, i32, P(_abi.StepRecord)]
        L.orc_get_check_errors.argtypes = [vp, i32, i32, P(d), i32, P(i32)]
        L.orc_compute_eff_moduli.argtypes = [vp, d, P(d), i32, P(_abi.Result)]
        L.orc_compute_eff_damping.argtypes = [vp, d, P(d), i32, d, P(ctypes.c_int64)]
        L.orc_static_fields.argtypes = [vp, d, d] + [P(d)] * 9 + [P(d)]
        L.orc_get_masks.argtypes = [vp, P(ctypes.c_uint8), P(ctypes.c_uint8)]
        L.orc_track_plastic_zone.argtypes = [vp, i32]
        L.orc_polar_fields.argtypes = [vp, d, P(d), P(d), P(d), P(d), P(ctypes.c_uint8)]
        _lib = L
    return _lib


def set_threads(n):
    return lib().orc_set_threads(int(n))


def make_pa(lx, ly, nx, ny, k0=1.0, g0=0.5, rho0=1.0, cfl=0.5, yield_stress=1.0,
            porosity=0.005, n_pores=1):
    """pa.dat values as get_sigma_2D.m:3-32 derives them, operation by operation:
    coh = Y*sqrt(2) (:6), rad = sqrt(porosity*Lx*Ly/(pi*N*N)) (:9),
    dX = Lx/(Nx-1) (:17), dt = CFL*min(dX,dY)/sqrt((K0+4*G0/3)/rho0) (:27),
    damp = 4/dt/Nx (:28-29), pa order of :32."""
    coh = yield_stress * math.sqrt(2.0)
    rad = math.sqrt(porosity * lx * ly / (math.pi * n_pores * n_pores))
    dx = lx / (nx - 1)
    dy = ly / (ny - 1)
    dt = cfl * min(dx, dy) / math.sqrt((k0 + 4 * g0 / 3) / rho0)
    dampx = 4.0 / dt / nx
    dampy = 4.0 / dt / ny
    return [dx, dy, dt, k0, g0, rho0, dampx, dampy, coh, rad, float(n_pores)]


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class Oracle:
    """One RVE on the CPU; methods mirror effplast2d_b200.Solver."""

    def __init__(self, nx, ny, pa, nl=1, niter=100000, eiter=1e-9, check_every=10000):
        self.nx, self.ny = int(nx), int(ny)
        self.params = _abi.make_params(nx, ny, pa, nl=nl, niter=niter, eiter=eiter,
                                       check_every=check_every)
        h = ctypes.c_void_p()
        rc = lib().orc_create(ctypes.byref(self.params), ctypes.byref(h))
        if rc != 0:
            raise ValueError("orc_create failed with status %d" % rc)
        self._h = h

    def close(self):
        if self._h:
            lib().orc_destroy(self._h)
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
        rc = lib().orc_get_field(self._h, _abi.FIELD_ID[field], _dptr(a))
        assert rc == 0
        return a

    def set(self, field, arr):
        w, h = self.dims(field)
        a = np.ascontiguousarray(arr, dtype=np.float64).reshape(h, w)
        rc = lib().orc_set_field(self._h, _abi.FIELD_ID[field], _dptr(a))
        assert rc == 0

    def iterate(self, n):
        rc = lib().orc_iterate(self._h, int(n))
        assert rc == 0

    def solve_step(self, step, load_step_value, load_type, n_time_steps=1):
        lt = np.asarray(load_type, dtype=np.float64)
        recs = (_abi.StepRecord * n_time_steps)()
        rc = lib().orc_solve_step(self._h, int(step), float(load_step_value), _dptr(lt),
                                  int(n_time_steps), recs)
        if rc != 0:
            raise ValueError("orc_solve_step failed with status %d" % rc)
        return [r.as_dict() for r in recs]

    def record(self, step, time_step):
        r = _abi.StepRecord()
        rc = lib().orc_get_record(self._h, int(step), int(time_step), ctypes.byref(r))
        assert rc == 0
        return r.as_dict()

    def check_errors(self, step, time_step):
        buf = np.zeros(4096)
        n = ctypes.c_int32()
        rc = lib().orc_get_check_errors(self._h, int(step), int(time_step), _dptr(buf), 4096,
                                        ctypes.byref(n))
        assert rc == 0
        return buf[: n.value].tolist()

    def compute_eff_moduli(self, init_load_value, load_type, n_time_steps=1):
        lt = np.asarray(load_type, dtype=np.float64)
        res = _abi.Result()
        rc = lib().orc_compute_eff_moduli(self._h, float(init_load_value), _dptr(lt),
                                          int(n_time_steps), ctypes.byref(res))
        if rc != 0:
            raise ValueError("orc_compute_eff_moduli failed with status %d" % rc)
        return res.as_dict()

    def compute_eff_damping(self, init_load_value, load_type, n_time_steps, load_value):
        lt = np.asarray(load_type, dtype=np.float64)
        tot = ctypes.c_int64()
        rc = lib().orc_compute_eff_damping(self._h, float(init_load_value), _dptr(lt), int(n_time_steps),
                                           float(load_value), ctypes.byref(tot))
        if rc != 0:
            raise ValueError("orc_compute_eff_damping failed with status %d" % rc)
        return tot.value

    def masks(self):
        node = np.zeros((self.ny, self.nx), dtype=np.uint8)
        corner = np.zeros((self.ny - 1, self.nx - 1), dtype=np.uint8)
        u8 = ctypes.POINTER(ctypes.c_uint8)
        rc = lib().orc_get_masks(self._h, node.ctypes.data_as(u8), corner.ctypes.data_as(u8))
        assert rc == 0
        return node, corner

    def track_plastic_zone(self, on=True):
        assert lib().orc_track_plastic_zone(self._h, 1 if on else 0) == 0

    def polar_fields(self, load_value):
        """get_sigma_2D.m:170-194 with the zone tracked since track_plastic_zone(True):
        dict of Snurr, Snuff, Sanrr, Sanff (ny x nx) and Plast (counts)"""
        out = {k: np.zeros((self.ny, self.nx)) for k in ("Snurr", "Snuff", "Sanrr", "Sanff")}
        plast = np.zeros((self.ny, self.nx), dtype=np.uint8)
        rc = lib().orc_polar_fields(self._h, float(load_value), *[_dptr(out[k]) for k in
                                                                  ("Snurr", "Snuff", "Sanrr", "Sanff")],
                                    plast.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)))
        assert rc == 0
        out["Plast"] = plast
        return out

    def static_fields(self, delta_p, tau_infty):
        nx, ny = self.nx, self.ny
        node = lambda: np.zeros((ny, nx))  # noqa: E731
        corner = lambda: np.zeros((ny - 1, nx - 1))  # noqa: E731
        out = {"UnuAbs": node(), "J1nu": corner(), "J2nu": corner(), "UanAbs": node(),
               "errorUabs": node(), "J1an": corner(), "J2an": corner(),
               "errorJ1": corner(), "errorJ2": corner()}
        stats = np.zeros(6)
        order = ["UnuAbs", "J1nu", "J2nu", "UanAbs", "errorUabs", "J1an", "J2an", "errorJ1", "errorJ2"]
        rc = lib().orc_static_fields(self._h, float(delta_p), float(tau_infty),
                                     *[_dptr(out[k]) for k in order], _dptr(stats))
        assert rc == 0
        out["stats"] = stats
        return out
