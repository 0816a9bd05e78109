"""The file-format library (effplast2d_b200.dataio) against the reference's own outputs:
the .dat files, pa.dat and EffPlast2D.log of the golden runs (tests/golden), read the way
read_data_2D.m and eff_props_2D.m read them.  CPU only."""
import math
import os

import numpy as np
import pytest

from effplast2d_b200 import dataio
from golden_util import CHAIN_CASES, load


@pytest.fixture
def in_tmp(tmp_path, monkeypatch):
    monkeypatch.chdir(tmp_path)
    return tmp_path


def test_dat_round_trip_and_matlab_orientation(in_tmp):
    rng = np.random.default_rng(3)
    f = rng.standard_normal((5, 7))  # height 5, width 7: [j, i]
    path = dataio.write_data_2d("data_Pc", 7, f)
    assert path == "data_Pc_7_.dat" and os.path.getsize(path) == 8 * 35
    assert np.array_equal(dataio.read_data_2d("data_Pc", 7, 7, 5), f)
    m = dataio.read_data_2d("data_Pc", 7, 7, 5, matlab=True)  # MATLAB's field(i+1, j+1)
    assert m.shape == (7, 5) and np.array_equal(m, f.T)
    with pytest.raises(ValueError):
        dataio.read_data_2d("data_Pc", 7, 6, 5)


def test_missing_file_is_a_zero_field(in_tmp, capsys):
    z = dataio.read_data_2d("nothing", 32, 32, 31)
    assert z.shape == (31, 32) and not z.any()
    assert "Error! File nothing_32_.dat does not exist!" in capsys.readouterr().out


def test_pa_round_trip(in_tmp):
    import oracle

    pa = oracle.make_pa(20.0, 20.0, 64, 64, g0=0.5, yield_stress=1e-5, porosity=0.02, n_pores=2)
    dataio.write_pa("pa.dat", pa)
    d = dataio.read_pa("pa.dat")
    assert list(d) == list(dataio.PA_NAMES) and [d[k] for k in dataio.PA_NAMES] == list(pa)
    dataio.write_pa("pa2.dat", d)
    assert open("pa.dat", "rb").read() == open("pa2.dat", "rb").read()


@pytest.mark.parametrize("name", [c for c in CHAIN_CASES])
def test_reference_dat_files_read_as_its_fields(name, in_tmp):
    # the reference's own output files, read back with the reader, equal the device
    # fields the harness dumped from the same run
    meta, z = load(name)
    n = meta["n"]
    for key in z.files:
        if not key.startswith("dat_"):
            continue
        fname = key[len("dat_"):]
        var = fname[: -len("_%d_.dat" % n)]
        nodes = var in ("Pc", "tauXXc", "UnuAbs", "UanAbs", "errorUabs")
        w = n if nodes else n - 1
        z[key].astype("<f8").tofile(fname)
        a = dataio.read_data_2d(var, n, w, w)
        assert a.shape == (w, w)
        if var == "Pc":
            assert np.array_equal(a, z["f_P"])
        if var == "tauXXc":
            assert np.array_equal(a, z["f_tauXX"])


@pytest.mark.parametrize("name", CHAIN_CASES)
def test_parse_reference_log(name):
    meta, _ = load(name)
    log = dataio.parse_log(meta["cli_log"])
    nl, nts = meta["macros"]["NL"], meta["n_time_steps"]
    assert [s["index"] for s in log["load_steps"]] == list(range(1, nl + 1))
    assert all(s["of"] == nl and s["grid"] == (meta["n"], meta["n"]) for s in log["load_steps"])
    assert abs(log["load_steps"][0]["porosity_pct"] - 100 * meta["porosity"]) < 1e-3
    assert dataio.total_iterations(log) == meta["total_iterations"]
    for s, step in enumerate(log["load_steps"]):
        assert len(step["time_steps"]) == (nts if s == 0 else 1)
        for t, ts in enumerate(step["time_steps"]):
            rec = meta["records"]["%d_%d" % (s, t)]
            for a, b in zip(ts["macro_strain"], rec["epsilon"]):
                assert abs(a - b) <= 1e-5 * abs(b) + 1e-15
            assert ts["checks"] and all(it % 10000 == 0 for it, _ in ts["checks"])
            y = float(meta["Y"])
            assert abs(ts["values"]["P / Y"] - rec["deltaP"][0] / y) <= 1e-5 * abs(rec["deltaP"][0] / y) + 1e-12
    if nl <= 3:  # ComputeEffModuli prints the moduli block
        names = ["Kphi", "Kd"] + (["G"] if nl == 3 else [])
        for kind, key in (("numerical", "num"), ("analytical", "an")):
            for i, nm in enumerate(names):
                a, b = log["moduli"]["non_periodic"][kind][nm], meta["moduli"][key][i]
                if math.isfinite(b) and abs(b) > 1e-12:
                    assert abs(a - b) <= 1e-5 * abs(b), (kind, nm, a, b)
    else:
        assert log["moduli"] == {} and "DAMPING" in log["calculation"]
