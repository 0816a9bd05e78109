"""The B200 path and the drop-in CLI against the reference's own output.

Fixtures: tests/golden (runs of the unmodified reference on a B200).  Kernel-level
cases must agree to 1e-12 (one iteration) / 1e-10 (100 iterations) -- the fraction of
bit-identical values is reported; load-step chains to 1e-9 on records and fields and
1e-8 on moduli with identical iteration counts; the drop-in CLI (csrc/dropin, built
with the same compile-time macros) must write the same EffPlast2D.log lines (6 digits)
and the same data/*.dat files.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

import effplast2d_b200 as ep
from effplast2d_b200 import build as epbuild
from golden_util import (CHAIN_CASES, FIELDS, KERNEL_CASES, compare_text, field_rel_err, load, same_printed,
                         tensor_tables)
from test_golden_oracle import check_chain

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", KERNEL_CASES)
def test_kernels_vs_reference(name):
    meta, z = load(name)
    nx, ny, nl, iters = meta["nx"], meta["ny"], meta["nl"], meta["iterations"]
    s = ep.Solver(nx, ny, list(z["pa"]), nl=nl)
    assert np.array_equal(s.get("K"), z["K"]) and np.array_equal(s.get("G"), z["G"])
    for f in ("Ux", "Uy", "Vx", "Vy"):
        s.set(f, z["in_" + f])
    s.iterate(iters)
    tol = 1e-12 if iters == 1 else 1e-10
    same = total = 0
    for f in FIELDS:
        a, b = s.get(f), z["out_" + f]
        assert field_rel_err(a, b) <= tol, f
        same += int(np.sum(a == b))
        total += a.size
    print("%s: %.4f of values bit-identical to the reference" % (name, same / total))


@pytest.mark.parametrize("name", CHAIN_CASES)
def test_chain_vs_reference(name):
    meta, z = load(name)
    n, mac = meta["n"], meta["macros"]
    s = ep.Solver(n, n, list(z["pa"]), nl=mac["NL"], niter=mac["NITER"], eiter=mac["EITER"], check_every=10000)
    if mac["NL"] >= 4:  # ComputeEffDamping; the load value is the CLI's sixth argument
        res = {"total_iterations": s.compute_eff_damping(meta["load"], meta["load_type"], meta["n_time_steps"],
                                                         float(meta["argv"][5]))}
        assert res["total_iterations"] == meta["total_iterations"]
    else:
        res = s.compute_eff_moduli(meta["load"], meta["load_type"], meta["n_time_steps"])
    check_chain(meta, z, s, res)
    if mac["NL"] > 1:
        sf = s.static_fields()
        assert field_rel_err(sf["UnuAbs"], z["dat_UnuAbs_%d_.dat" % n].reshape(n, n)) <= 1e-9
        assert field_rel_err(sf["J1nu"], z["dat_J1nu_%d_.dat" % n].reshape(n - 1, n - 1)) <= 1e-9
        assert field_rel_err(sf["J2nu"], z["dat_J2nu_%d_.dat" % n].reshape(n - 1, n - 1)) <= 1e-8


def cli_for(name):
    meta, _ = load(name)
    path = os.path.join(epbuild.BUILD, "cli_" + name)
    epbuild.build_cli(macros=meta["macros"] | {"NPARS": 11, "DEVICE_IDX": 0}, out=path,
                      force=not os.path.exists(path))
    return path


@pytest.mark.parametrize("name", CHAIN_CASES)
def test_dropin_cli_vs_reference(name):
    meta, z = load(name)
    exe = cli_for(name)
    work = tempfile.mkdtemp()
    os.makedirs(os.path.join(work, "data"))
    np.asarray(z["pa"], dtype="<f8").tofile(os.path.join(work, "data", "pa.dat"))
    r = subprocess.run([exe] + meta["argv"], cwd=work, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    log = open(os.path.join(work, "EffPlast2D.log")).read()
    diffs = compare_text(log, meta["cli_log"])
    assert not diffs, diffs[:5]
    if meta["macros"]["NL"] >= 4:
        # the damping tables go to stdout only: ours at the default 6 digits, the
        # reference's captured at 17
        mine_t, ref_t = tensor_tables(r.stdout), tensor_tables(meta["cli_stdout"])
        assert sorted(mine_t) == sorted(ref_t) and len(ref_t) == 4
        for title, rows in ref_t.items():
            assert len(mine_t[title]) == len(rows) == meta["macros"]["NL"], title
            for a_row, b_row in zip(mine_t[title], rows):
                assert len(a_row) == len(b_row)
                for a, b in zip(a_row, b_row):
                    assert same_printed(a, b, 1e-5, noise=1e-15), (title, a_row, b_row)
    assert sorted(os.listdir(os.path.join(work, "data"))) == meta["cli_dat_files"]
    n = meta["n"]
    for f in meta["cli_dat_files"]:
        if f == "pa.dat":
            continue
        mine = np.fromfile(os.path.join(work, "data", f), dtype="<f8")
        ref = z["dat_" + f]
        assert mine.shape == ref.shape, f
        tol = 1e-8 if f.startswith(("J2", "error")) else 1e-9
        if f.startswith("error"):
            assert np.max(np.abs(mine - ref)) <= 1e-6, f
        else:
            assert field_rel_err(mine, ref) <= tol, f


def test_dropin_unity_build_vs_reference():
    # the self-contained build (library sources compiled into the drop-in binary with
    # -DEP2D_UNITY, no separate libep2d.so): same log and .dat files as the reference's
    name = "c64_nl2"
    meta, z = load(name)
    exe = epbuild.build_cli_unity(meta["macros"] | {"NPARS": 11, "DEVICE_IDX": 0},
                                  os.path.join(epbuild.BUILD, "cli_unity_" + name))
    work = tempfile.mkdtemp()
    os.makedirs(os.path.join(work, "data"))
    np.asarray(z["pa"], dtype="<f8").tofile(os.path.join(work, "data", "pa.dat"))
    r = subprocess.run([exe] + meta["argv"], cwd=work, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    diffs = compare_text(open(os.path.join(work, "EffPlast2D.log")).read(), meta["cli_log"])
    assert not diffs, diffs[:5]
    assert sorted(os.listdir(os.path.join(work, "data"))) == meta["cli_dat_files"]
    n = meta["n"]
    mine = np.fromfile(os.path.join(work, "data", "Pc_%d_.dat" % n), dtype="<f8")
    assert field_rel_err(mine, z["dat_Pc_%d_.dat" % n]) <= 1e-9


def test_dropin_cli_error_paths():
    exe = cli_for("c32_nl1")
    work = tempfile.mkdtemp()
    r = subprocess.run([exe, "-4e-5", "1", "1", "0", "1", "0"], cwd=work, capture_output=True, text=True)
    assert r.returncode == 1 and "Cannot open file data/pa.dat" in r.stderr
    r = subprocess.run([exe, "-4e-5", "1", "1", "0", "1"], cwd=work, capture_output=True, text=True)
    assert r.returncode == 1 and "missing arguments" in r.stderr
