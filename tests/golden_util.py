"""Helpers for the golden fixtures in tests/golden (made by tests/golden/make_golden.py
from runs of the unmodified reference on a B200)."""
import json
import math
import os
import re

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

KERNEL_CASES = ["k32_nl1_it1", "k32_nl3_it1", "k64x32_nl2_it1", "k64_nl3_it100", "k32x64_nl1_it100"]
CHAIN_CASES = ["c32_nl1", "c64_nl2", "c64_nl3", "c96_nl3", "cfg1", "c64_nl5"]  # c64_nl5: damping mode (NL=5)

FIELDS = ["P", "tauXX", "tauYY", "tauXY", "tauXYav", "J2", "J2XY", "Ux", "Uy", "Vx", "Vy"]

# record keys of the reference (records.txt) -> ep2d_step_record keys
REC_KEYS = {"deltaP": "delta_p", "deltaPper": "delta_p_per", "tauInfty": "tau_infty", "dPhi": "dphi",
            "dPhiPer": "dphi_per", "epsilon": "macro_strain", "epsilonPer": "eps_per", "sigma": "sigma",
            "sigmaPer": "sigma_per"}


def load(name):
    meta = json.load(open(os.path.join(GOLDEN, name + ".json")))
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    return meta, z


def field_rel_err(a, b):
    scale = float(np.max(np.abs(b)))
    d = float(np.max(np.abs(np.asarray(a) - np.asarray(b))))
    return d if scale == 0.0 else d / scale


def close(a, b, rtol, atol=0.0):
    if a == b:
        return True
    if math.isnan(a) or math.isnan(b):
        return math.isnan(a) and math.isnan(b)
    if math.isinf(a) or math.isinf(b):
        return a == b
    return abs(a - b) <= rtol * abs(b) + atol


def record_scale(rec):
    """stress scale of a time step, for absolute floors on near-zero stress values"""
    return max(abs(v) for v in rec["sigma"] + [rec["deltaP"][0]]) or 1.0


def compare_record(mine, ref, rtol=1e-9):
    """mine: ep2d_step_record dict; ref: the reference's records.txt entry"""
    s = record_scale(ref)
    bad = []
    for rk, mk in REC_KEYS.items():
        rv = ref[rk]
        mv = mine[mk] if isinstance(mine[mk], list) else [mine[mk]]
        for a, b in zip(mv, rv):
            floor = 1e-9 * s if rk in ("deltaP", "deltaPper", "tauInfty", "sigma", "sigmaPer") else 0.0
            if rk in ("epsilonPer",):
                floor = 1e-9 * max(abs(v) for v in ref["epsilon"])
            if not close(a, b, rtol, floor):
                bad.append((rk, a, b))
    return bad


def parse_steps(text):
    """split reference/drop-in output into per-(load step, time step) checkpoint data:
    list of dicts {iterations: [...], errors: [...], converged: bool, warned: bool}"""
    out = []
    cur = None
    for line in text.splitlines():
        if line.startswith("Time step "):
            cur = {"iterations": [], "errors": [], "converged": False, "warned": False}
            out.append(cur)
        m = re.match(r"\s+Iteration (\d+): Error is (\S+)", line)
        if m and cur is not None:
            cur["iterations"].append(int(m.group(1)))
            cur["errors"].append(float(m.group(2)))
        if line.startswith("Number of iterations is") and cur is not None:
            cur["converged"] = True
        if line.startswith("WARNING: Maximum number of iterations") and cur is not None:
            cur["warned"] = True
    return out


NUM = re.compile(r"[-+]?(?:\d+\.?\d*(?:[eE][-+]?\d+)?|inf|nan)")


def same_printed(x, y, rtol, noise=1e-12):
    """Printed numbers agree: within rtol; or both below `noise` in magnitude (rounding
    noise, e.g. tau/Y under a hydrostatic load, ~1e-16); or both non-finite (G when the
    deviatoric increment has no xx - yy part: the reference divides by exactly zero and
    prints +-inf or nan depending on the sign of a rounding-noise numerator)."""
    if not math.isfinite(x) or not math.isfinite(y):
        return not math.isfinite(x) and not math.isfinite(y)
    if abs(x) < noise and abs(y) < noise:
        return True
    return close(x, y, rtol, 1e-300)


def tensor_tables(text):
    """The strain / stress tensor tables ComputeEffDamping prints (EffPlast2D.cu:245-297):
    {title: [[values of step 0], [step 1], ...]}"""
    out, cur = {}, None
    for line in text.splitlines():
        if line.endswith("tensors:") or line.endswith("tensors periodic:"):
            cur = out.setdefault(line, [])
        elif cur is not None and re.match(r"\d+\) ", line):
            cur.append([float(v) for v in line.split()[1:]])
        elif cur is not None and not line.strip():
            cur = None
    return out


def compare_text(mine, ref, rtol=2e-6, skip=("Calculation time",)):
    """line-by-line comparison: identical text, numbers equal within rtol (6-digit output)"""
    a = [l for l in mine.splitlines() if not l.startswith(skip)]
    b = [l for l in ref.splitlines() if not l.startswith(skip)]
    diffs = []
    if len(a) != len(b):
        return ["line count %d != %d" % (len(a), len(b))]
    for la, lb in zip(a, b):
        if la == lb:
            continue
        if NUM.sub("#", la) != NUM.sub("#", lb):
            diffs.append((la, lb))
            continue
        # a checkpoint error below 1e-10 is max|V| of a converged state, i.e. rounding
        # noise of the velocities: its leading digits agree, the sixth need not
        tol = 1e-3 if ("Error is" in lb and abs(float(NUM.findall(lb)[-1])) < 1e-10) else rtol
        for x, y in zip(NUM.findall(la), NUM.findall(lb)):
            if not same_printed(float(x), float(y), tol):
                diffs.append((la, lb))
                break
    return diffs
