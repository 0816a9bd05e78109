"""ctypes mirrors of the C ABI declared in include/ep2d.h.

Pure declarations: no library is loaded here.  `effplast2d_b200.solver` binds these
to libep2d.so; the test-only oracle wrapper binds the same declarations to its own
library.  `abi_sizes()` in both C libraries reports sizeof() of every struct so the
tests can check these mirrors against the compiler's layout.
"""
import ctypes
from ctypes import c_double, c_int32, c_int64

NPARS = 11
MAX_NL = 3
MAX_STEPS = 64  # load steps of the damping mode (nl >= 4)

OK = 0
ERR_ARG = 1
ERR_CUDA = 2
ERR_IO = 3
ERR_STATE = 4
ERR_NOMEM = 5
ERR_RANGE = 6
ERR_NODEV = 7

FP64 = 0
MIXED = 1
F32_BULK = 2

KERNEL_AUTO = 0
KERNEL_TILE = 1
KERNEL_STREAM = 2
KERNEL_RESIDENT = 3

# field identifiers (include/ep2d.h), in the reference's array order
FIELDS = ("P", "tauXX", "tauYY", "tauXY", "tauXYav", "J2", "J2XY",
          "Ux", "Uy", "Vx", "Vy", "K", "G")
FIELD_ID = {name: i for i, name in enumerate(FIELDS)}

PA_NAMES = ("dX", "dY", "dt", "K0", "G0", "rho0", "dampX", "dampY", "coh", "rad", "N")


def field_dims(nx, ny, field):
    """(width, height) of a field for an nx x ny grid (EffPlast2D.cu:1577-1604)."""
    f = FIELD_ID[field] if isinstance(field, str) else int(field)
    name = FIELDS[f]
    if name in ("tauXY", "J2XY"):
        return nx - 1, ny - 1
    if name in ("Ux", "Vx"):
        return nx + 1, ny
    if name in ("Uy", "Vy"):
        return nx, ny + 1
    return nx, ny


class Params(ctypes.Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32),
        ("pa", c_double * NPARS),
        ("nl", c_int32), ("check_every", c_int32),
        ("niter", c_int64),
        ("eiter", c_double),
        ("precision", c_int32), ("device", c_int32),
        ("kernel", c_int32), ("rows", c_int32),
    ]


class StepRecord(ctypes.Structure):
    _fields_ = [
        ("step", c_int32), ("time_step", c_int32),
        ("iterations", c_int64),
        ("converged", c_int32), ("n_checks", c_int32),
        ("error", c_double),
        ("macro_strain", c_double * 3),
        ("sigma", c_double * 4),
        ("sigma_per", c_double * 4),
        ("eps_per", c_double * 3),
        ("delta_p", c_double), ("delta_p_per", c_double), ("tau_infty", c_double),
        ("hole_area_pi", c_double), ("internal_hole_area_pi", c_double),
        ("phi0", c_double), ("phi", c_double), ("phi_per", c_double),
        ("dphi", c_double), ("dphi_per", c_double),
        ("kphi_exact_elast", c_double), ("kd_exact_elast", c_double),
        ("kphi_exact_plast", c_double), ("kd_exact_plast", c_double),
        ("kphi_exact_plast_per", c_double), ("kd_exact_plast_per", c_double),
        ("g_exact_elast", c_double), ("g_exact_plast", c_double), ("g_exact_plast_per", c_double),
    ]

    def as_dict(self):
        out = {}
        for name, ctype in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if hasattr(ctype, "_length_") else v
        return out


class Moduli(ctypes.Structure):
    _fields_ = [("kphi", c_double), ("kd", c_double), ("g", c_double)]

    def as_dict(self):
        return {"kphi": self.kphi, "kd": self.kd, "g": self.g}


class Result(ctypes.Structure):
    _fields_ = [
        ("an", Moduli), ("an_per", Moduli), ("num", Moduli), ("num_per", Moduli),
        ("nl", c_int32), ("n_time_steps", c_int32),
        ("total_iterations", c_int64),
        ("all_converged", c_int32), ("reserved", c_int32),
    ]

    def as_dict(self):
        return {
            "an": self.an.as_dict(), "an_per": self.an_per.as_dict(),
            "num": self.num.as_dict(), "num_per": self.num_per.as_dict(),
            "nl": self.nl, "n_time_steps": self.n_time_steps,
            "total_iterations": self.total_iterations, "all_converged": self.all_converged,
        }


class RveSpec(ctypes.Structure):
    _fields_ = [
        ("nx", c_int32), ("ny", c_int32),
        ("pa", c_double * NPARS),
        ("nl", c_int32), ("n_time_steps", c_int32),
        ("init_load_value", c_double),
        ("load_type", c_double * 3),
    ]


class BatchConfig(ctypes.Structure):
    _fields_ = [
        ("niter", c_int64), ("eiter", c_double),
        ("check_every", c_int32), ("precision", c_int32), ("device", c_int32),
        ("rows", c_int32), ("graph_len", c_int32), ("kernel", c_int32),
    ]


class BatchStats(ctypes.Structure):
    _fields_ = [
        ("kernel_ms", c_double), ("wall_ms", c_double),
        ("launches", c_int64), ("all_launches", c_int64), ("cell_updates", c_int64),
        ("rows", c_int32), ("blocks", c_int32),
        ("kernel", c_int32), ("n_tuned", c_int32),
        ("tune_us", c_double * 7),
        ("n_tunes", c_int32), ("solo_intervals", c_int32),
    ]

    def as_dict(self):
        return {"kernel_ms": self.kernel_ms, "wall_ms": self.wall_ms, "launches": self.launches,
                "all_launches": self.all_launches, "cell_updates": self.cell_updates,
                "rows": self.rows, "blocks": self.blocks, "kernel": self.kernel,
                "n_tuned": self.n_tuned, "tune_us": list(self.tune_us), "n_tunes": self.n_tunes,
                "solo_intervals": self.solo_intervals}


def make_spec(nx, ny, pa, nl, n_time_steps, init_load_value, load_type):
    s = RveSpec()
    s.nx, s.ny = int(nx), int(ny)
    for i, v in enumerate(pa):
        s.pa[i] = float(v)
    s.nl = int(nl)
    s.n_time_steps = int(n_time_steps)
    s.init_load_value = float(init_load_value)
    for i in range(3):
        s.load_type[i] = float(load_type[i])
    return s


def make_batch_config(niter=100000, eiter=1e-9, check_every=10000, precision=FP64, device=0, rows=0,
                      graph_len=0, kernel=0):
    c = BatchConfig()
    c.niter = int(niter)
    c.eiter = float(eiter)
    c.check_every = int(check_every)
    c.precision = int(precision)
    c.device = int(device)
    c.rows = int(rows)
    c.graph_len = int(graph_len)
    c.kernel = int(kernel)
    return c


STRUCTS = {"ep2d_params": Params, "ep2d_step_record": StepRecord,
           "ep2d_moduli": Moduli, "ep2d_result": Result, "ep2d_rve_spec": RveSpec,
           "ep2d_batch_config": BatchConfig, "ep2d_batch_stats": BatchStats}


def make_params(nx, ny, pa, nl=1, niter=100000, eiter=1e-9, check_every=10000,
                precision=FP64, device=0, kernel=0, rows=0):
    p = Params()
    p.nx, p.ny = int(nx), int(ny)
    if len(pa) != NPARS:
        raise ValueError("pa must hold %d values" % NPARS)
    for i, v in enumerate(pa):
        p.pa[i] = float(v)
    p.nl = int(nl)
    p.check_every = int(check_every)
    p.niter = int(niter)
    p.eiter = float(eiter)
    p.precision = int(precision)
    p.device = int(device)
    p.kernel = int(kernel)
    p.rows = int(rows)
    return p
