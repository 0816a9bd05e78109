"""Pin the CPU oracle against the reference's own output (CPU only).

The fixtures come from the unmodified reference (EffPlast2D.cu) run on a B200 through
oracle/_ref (tests/golden/make_golden.py).  The reference contracts multiply-adds on the
GPU, the oracle does not: fields and records agree to rounding (1e-12 after one
iteration, 1e-9 over full load steps).  Iteration counts and convergence decisions
agree exactly.
"""
import math

import numpy as np
import pytest

import oracle
from golden_util import CHAIN_CASES, FIELDS, KERNEL_CASES, compare_record, field_rel_err, load, parse_steps


@pytest.fixture(scope="module", autouse=True)
def _threads():
    oracle.set_threads(4)


@pytest.mark.parametrize("name", KERNEL_CASES)
def test_oracle_kernels_vs_reference(name):
    meta, z = load(name)
    nx, ny, nl, iters = meta["nx"], meta["ny"], meta["nl"], meta["iterations"]
    with oracle.Oracle(nx, ny, list(z["pa"]), nl=nl) as o:
        assert np.array_equal(o.get("K"), z["K"]) and np.array_equal(o.get("G"), z["G"])
        for f in ("Ux", "Uy", "Vx", "Vy"):
            o.set(f, z["in_" + f])
        o.iterate(iters)
        tol = 1e-12 if iters == 1 else 1e-10
        for f in FIELDS:
            assert field_rel_err(o.get(f), z["out_" + f]) <= tol, f
        node, corner = o.masks()
        assert np.array_equal(z["out_P"] == 0.0, node.astype(bool))
        assert np.array_equal(z["out_tauXY"] == 0.0, corner.astype(bool))


def run_chain(name):
    meta, z = load(name)
    n, mac = meta["n"], meta["macros"]
    o = oracle.Oracle(n, n, list(z["pa"]), nl=mac["NL"], niter=mac["NITER"], eiter=mac["EITER"], check_every=10000)
    if mac["NL"] >= 4:  # ComputeEffDamping; the load value is the CLI's sixth argument
        res = {"total_iterations": o.compute_eff_damping(meta["load"], meta["load_type"], meta["n_time_steps"],
                                                         float(meta["argv"][5]))}
    else:
        res = o.compute_eff_moduli(meta["load"], meta["load_type"], meta["n_time_steps"])
    return meta, z, o, res


def check_chain(meta, z, solver, res, rtol_rec=1e-9, rtol_fields=1e-9):
    nl = meta["macros"]["NL"]
    nts = meta["n_time_steps"]
    steps = parse_steps(meta["cli_stdout"])
    k = 0
    for s in range(nl):
        for t in range(nts if s == 0 else 1):
            mine = solver.record(s, t)
            ref = meta["records"]["%d_%d" % (s, t)]
            bad = compare_record(mine, ref, rtol_rec)
            assert not bad, (s, t, bad)
            st = steps[k]
            k += 1
            assert mine["n_checks"] == len(st["iterations"])
            assert bool(mine["converged"]) == st["converged"]
            if st["converged"]:
                assert mine["iterations"] == st["iterations"][-1]
            errs = solver.check_errors(s, t)
            for a, b in zip(errs, st["errors"]):
                assert abs(a - b) <= 1e-5 * abs(b) + 1e-13, (s, t, a, b)
    if nl >= 4:  # damping mode: no moduli, no Pc / tauXXc files (EffPlast2D.cu:230-310)
        for f in ("P", "tauXX", "tauYY", "tauXY", "Ux", "Uy"):
            assert field_rel_err(solver.get(f), z["f_" + f]) <= rtol_fields, f
        return
    mod = meta["moduli"]
    keys = ["kphi", "kd"] + (["g"] if nl == 3 else [])
    kinds = ["num", "an"] + (["num_per", "an_per"] if (nl > 1 and meta["n_pores"] > 2) else [])
    if nl == 1:
        kinds = ["num", "an", "num_per"]
        keys = ["kphi", "kd"]
    for kind in kinds:
        for i, key in enumerate(keys):
            a, b = res[kind][key], mod[kind][i]
            if math.isnan(b) or math.isinf(b):
                # undefined in the reference (a division by an exact zero): ours must be too
                assert not math.isfinite(a), (kind, key, a, b)
            else:
                assert abs(a - b) <= 1e-8 * abs(b) + 1e-300, (kind, key, a, b)
    for f in ("P", "tauXX", "tauYY", "tauXY", "Ux", "Uy"):
        assert field_rel_err(solver.get(f), z["f_" + f]) <= rtol_fields, f
    # the reference's own output files
    n = meta["n"]
    assert field_rel_err(solver.get("P"), z["dat_Pc_%d_.dat" % n].reshape(n, n)) <= rtol_fields
    assert field_rel_err(solver.get("tauXX"), z["dat_tauXXc_%d_.dat" % n].reshape(n, n)) <= rtol_fields


@pytest.mark.parametrize("name", CHAIN_CASES)
def test_oracle_chain_vs_reference(name):
    meta, z, o, res = run_chain(name)
    check_chain(meta, z, o, res)
    o.close()


def test_oracle_static_fields_vs_reference_files():
    # UnuAbs / J1nu / J2nu written by the reference's SaveAnStatic2D (NL > 1)
    meta, z, o, res = run_chain("c96_nl3")
    r0 = o.record(0, meta["n_time_steps"] - 1)
    sf = o.static_fields(r0["delta_p"], r0["tau_infty"])
    n = meta["n"]
    assert field_rel_err(sf["UnuAbs"], z["dat_UnuAbs_%d_.dat" % n].reshape(n, n)) <= 1e-9
    assert field_rel_err(sf["J1nu"], z["dat_J1nu_%d_.dat" % n].reshape(n - 1, n - 1)) <= 1e-9
    assert field_rel_err(sf["J2nu"], z["dat_J2nu_%d_.dat" % n].reshape(n - 1, n - 1)) <= 1e-8
