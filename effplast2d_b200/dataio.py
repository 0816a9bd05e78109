"""The reference's file formats: the field .dat files, pa.dat and EffPlast2D.log / stdout.

* `<var>_<n>_.dat` -- one field as raw little-endian FP64, element (i, j) (x index i,
  y index j) at position j*width + i: what SaveMatrix writes (EffPlast2D.cu:795-799) and
  read_data_2D.m:1-12 reads.  MATLAB reshapes the values column-major to (width, height),
  so its field(i+1, j+1) is element (i, j); `read_data_2d(..., matlab=True)` returns that
  orientation, the default a row-major (height, width) array indexed [j, i] like the
  library's fields.  A missing file is an error message and a zero field, as in
  read_data_2D.m:10-11.
* `pa.dat` -- the 11 parameters dX, dY, dt, K0, G0, rho0, dampX, dampY, coh, rad, N as
  little-endian FP64 (get_sigma_2D.m:32, read at EffPlast2D.cu:700-707).
* EffPlast2D.log / stdout -- `parse_log` turns the text the reference writes
  (EffPlast2D.cu:311-698, :1295-1409, :1412-1454) into per-step records.
"""
import os
import re

import numpy as np

PA_NAMES = ("dX", "dY", "dt", "K0", "G0", "rho0", "dampX", "dampY", "coh", "rad", "N")


def dat_name(var_name, size):
    """read_data_2D.m:2: strcat(var_name, '_', int2str(size), '_.dat')"""
    return "%s_%d_.dat" % (var_name, int(size))


def write_data_2d(var_name, size, field):
    """Write `field` ((height, width) row-major, element [j, i]) as SaveMatrix does."""
    a = np.ascontiguousarray(np.asarray(field, dtype="<f8"))
    path = dat_name(var_name, size)
    a.tofile(path)
    return path


def read_data_2d(var_name, size, nx, ny, matlab=False, quiet=False):
    """read_data_2D.m: the field of `<var_name>_<size>_.dat` with width nx, height ny.
    Returns (ny, nx) indexed [j, i]; with matlab=True the (nx, ny) array MATLAB's
    reshape gives, indexed [i, j].  A missing file prints the reference's message and
    returns zeros; a file of the wrong length raises ValueError."""
    path = dat_name(var_name, size)
    if not os.path.isfile(path):
        if not quiet:
            print(" ".join(["Error! File", path, "does not exist!"]))
        return np.zeros((nx, ny) if matlab else (ny, nx))
    v = np.fromfile(path, dtype="<f8")
    if v.size != nx * ny:
        raise ValueError("%s holds %d values, not %d x %d" % (path, v.size, nx, ny))
    return v.reshape(nx, ny, order="F") if matlab else v.reshape(ny, nx)


def read_pa(path):
    """pa.dat as a dict of the 11 named parameters."""
    v = np.fromfile(path, dtype="<f8")
    if v.size < len(PA_NAMES):
        raise ValueError("%s holds %d values, expected %d" % (path, v.size, len(PA_NAMES)))
    return dict(zip(PA_NAMES, (float(x) for x in v[: len(PA_NAMES)])))


def write_pa(path, pa):
    """pa: the 11 values in pa.dat order, or a dict keyed by PA_NAMES."""
    if isinstance(pa, dict):
        pa = [pa[k] for k in PA_NAMES]
    np.asarray(pa, dtype="<f8").tofile(path)


_NUM = r"([-+]?(?:\d+\.?\d*(?:[eE][-+]?\d+)?|inf|nan))"


def _num(s):
    return float(s)


def parse_log(text):
    """Parse EffPlast2D.log (or the binary's stdout) into
    {"calculation": str, "load_steps": [step, ...], "moduli": {...}, "warnings": [...],
     "time": str}; each step = {"index", "of", "kind", "porosity_pct", "grid",
    "time_steps": [...]}, each time step = {"macro_strain", "checks": [(iteration,
    error)], "converged", "iterations", "values": {name: value}}; "values" holds the
    per-step lines (dPhi, P / Y, tau / Y, analytic moduli) and "calc" of a step the
    calc* block after it (Kphi, KphiPer, Kd, KdPer, G, Gper).  moduli =
    {"non_periodic"|"periodic": {"analytical"|"numerical": {Kphi, Kd[, G]}}}."""
    out = {"calculation": "", "load_steps": [], "moduli": {}, "warnings": [], "time": None}
    lines = text.splitlines()
    step = ts = None
    section = sub = None
    in_moduli = False
    for k, line in enumerate(lines):
        s = line.strip()
        m = re.match(r"LOAD STEP (\d+) FROM (\d+): ?(.*)", line)
        if m:
            step = {"index": int(m.group(1)), "of": int(m.group(2)), "kind": "", "porosity_pct": None,
                    "grid": None, "time_steps": [], "calc": {}}
            rest = m.group(3)
            pm = re.match(r"Porosity is " + _NUM + "%", rest)
            if pm:  # damping mode: no kind, the porosity follows on the same line
                step["porosity_pct"] = _num(pm.group(1))
            else:
                step["kind"] = rest.strip()
            out["load_steps"].append(step)
            ts = None
            in_moduli = False
            continue
        if not out["calculation"] and s.endswith("CALCULATION") and k + 1 < len(lines):
            out["calculation"] = s + " / " + lines[k + 1].strip()
            continue
        m = re.match(r"Porosity is " + _NUM + "%", s)
        if m and step is not None:
            step["porosity_pct"] = _num(m.group(1))
            continue
        m = re.match(r"Grid resolution is (\d+)x(\d+)", s)
        if m and step is not None:
            step["grid"] = (int(m.group(1)), int(m.group(2)))
            continue
        m = re.match(r"Time step (\d+) from (\d+)", s)
        if m and step is not None:
            ts = {"index": int(m.group(1)), "of": int(m.group(2)), "macro_strain": None, "checks": [],
                  "converged": False, "iterations": None, "values": {}}
            step["time_steps"].append(ts)
            continue
        m = re.match(r"Macro strain: \(" + _NUM + ", " + _NUM + ", " + _NUM + r"\)", s)
        if m and ts is not None:
            ts["macro_strain"] = [_num(m.group(a)) for a in (1, 2, 3)]
            continue
        m = re.match(r"Iteration (\d+): Error is " + _NUM, s)
        if m and ts is not None:
            ts["checks"].append((int(m.group(1)), _num(m.group(2))))
            continue
        m = re.match(r"Number of iterations is (\d+)", s)
        if m and ts is not None:
            ts["converged"] = True
            ts["iterations"] = int(m.group(1))
            continue
        if s.startswith("WARNING: Maximum number of iterations") and ts is not None:
            ts["iterations"] = ts["checks"][-1][0] if ts["checks"] else None
            continue
        if s == "EFFECTIVE MODULI ESTIMATED":
            in_moduli = True
            continue
        if in_moduli:
            if s in ("NON-PERIODIC", "PERIODIC"):
                section = out["moduli"].setdefault(s.lower().replace("-", "_"), {})
                continue
            if s in ("Analytical:", "Numerical:"):
                sub = section.setdefault(s[:-1].lower(), {}) if section is not None else None
                continue
            m = re.match(r"(\w+) = " + _NUM + "$", s)
            if m and sub is not None:
                sub[m.group(1)] = _num(m.group(2))
                continue
        if s.startswith("WARNING:"):
            out["warnings"].append(s)
            continue
        m = re.match(r"Calculation time is (.*)", s)
        if m:
            out["time"] = m.group(1)
            continue
        m = re.match(r"([A-Za-z][\w /]*?) = " + _NUM + "$", s)
        if m and step is not None and not in_moduli:
            name = m.group(1).strip()
            if name in ("Kphi", "KphiPer", "Kd", "KdPer", "G", "Gper"):
                step["calc"][name] = _num(m.group(2))
            elif ts is not None:
                ts["values"][name] = _num(m.group(2))
    return out


def total_iterations(log):
    """Iterations of a whole run from a parsed log: the converged checkpoint of every time
    step, or its last checkpoint where the iteration cap ended it (NITER itself when NITER
    is a multiple of the 10,000-iteration checkpoint interval)."""
    return sum(t["iterations"] or 0 for s in log["load_steps"] for t in s["time_steps"])
