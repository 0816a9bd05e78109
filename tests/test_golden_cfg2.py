"""The headline configuration at full size against the reference's own run.

1024 x 1024 grid, 3 x 3 pores, porosity 0.01, G0 = 0.5, Y = 1e-5, preload -6e-5*[1,1,0]
over two time steps, then the bulk increment (NL = 2), EITER = 1e-9, NITER = 5e6.  The
reference needs 110,000 + 5,000,000 (capped, not converged) + 1,940,000 iterations.  The
fixture keeps the reference's records and moduli at 17 digits and every 8th row and
column of its final fields (tests/golden/make_golden.py reduce_fixture).  Bars: 1e-6
on fields and 1e-5 on the moduli; identical iteration counts.
"""
import json
import math
import os

import numpy as np
import pytest

import effplast2d_b200 as ep
from golden_util import GOLDEN, compare_record, parse_steps

pytestmark = pytest.mark.gpu


def test_config2_full_size_vs_reference():
    meta = json.load(open(os.path.join(GOLDEN, "cfg2.json")))
    z = np.load(os.path.join(GOLDEN, "cfg2_reduced.npz"))
    n, mac = meta["n"], meta["macros"]
    s = ep.Solver(n, n, list(z["pa"]), nl=mac["NL"], niter=mac["NITER"], eiter=mac["EITER"], check_every=10000)
    res = s.compute_eff_moduli(meta["load"], meta["load_type"], meta["n_time_steps"])
    assert res["total_iterations"] == meta["total_iterations"] == 7_050_000
    steps = parse_steps(meta["cli_stdout"])
    k = 0
    for st in range(mac["NL"]):
        for t in range(meta["n_time_steps"] if st == 0 else 1):
            mine = s.record(st, t)
            assert not compare_record(mine, meta["records"]["%d_%d" % (st, t)], rtol=1e-6), (st, t)
            assert bool(mine["converged"]) == steps[k]["converged"]
            assert mine["n_checks"] == len(steps[k]["iterations"])
            k += 1
    for i, key in enumerate(("kphi", "kd")):
        for kind in ("num", "num_per", "an", "an_per"):
            a, b = res[kind][key], meta["moduli"][kind][i]
            assert math.isfinite(a) and abs(a - b) <= 1e-5 * abs(b), (kind, key, a, b)
    stride = int(z["stride"])
    for f in ("P", "tauXX", "tauXY", "Ux", "Uy"):
        mine = s.get(f)
        ref_sub = z["f_%s__sub" % f]
        scale = np.max(np.abs(ref_sub))
        assert np.max(np.abs(mine[::stride, ::stride] - ref_sub)) <= 1e-6 * scale, f
        assert np.max(np.abs(mine[mine.shape[0] // 2, :] - z["f_%s__midrow" % f])) <= 1e-6 * scale, f
