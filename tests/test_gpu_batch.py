"""Batched persistent solver and continuous-batching server.

Each RVE of a batch must give exactly what the single-RVE path gives for the same
inputs (every kernel form, batched or not, evaluates the same explicitly rounded
per-cell formulas, so neither the form, the rows nor the batch changes a bit), the
mixed-precision batch must stay within the parity bar of 1e-5 relative on K_phi, K_d
and G, and the server must return the same result for a request alone and in a mix.
"""
import math

import pytest

import effplast2d_b200 as ep
from effplast2d_b200 import batch as B

pytestmark = pytest.mark.gpu

NITER, CE = 6000, 500


def mk(n, n_pores, phi, Y, nl, load, lt, nts):
    pa = ep.make_pa(20.0, 20.0, n, n, g0=0.5, yield_stress=Y, porosity=phi, n_pores=n_pores)
    return B.spec(n, pa, nl, nts, load, lt)


SPECS = [
    (64, 1, 0.005, 1.0, 1, -4e-5, (1.0, 1.0, 0.0), 1),
    (96, 3, 0.02, 1e-5, 3, -6e-5, (1.0, 0.8, 0.3), 2),
    (64, 2, 0.02, 1e-5, 2, -6e-5, (1.0, 1.0, 0.0), 2),
    (128, 1, 0.01, 2e-5, 3, -5e-5, (0.9, 1.0, 0.2), 1),
    (80, 2, 0.03, 1e-5, 2, -3e-5, (1.0, 1.0, 0.1), 1),
    (100, 4, 0.02, 5e-6, 3, -7e-5, (1.0, 0.6, 0.4), 1),
]


def single(sp, kernel=ep.KERNEL_AUTO, rows=0):
    n, npo, phi, Y, nl, load, lt, nts = sp
    pa = ep.make_pa(20.0, 20.0, n, n, g0=0.5, yield_stress=Y, porosity=phi, n_pores=npo)
    s = ep.Solver(n, n, pa, nl=nl, niter=NITER, eiter=1e-9, check_every=CE, kernel=kernel, rows=rows)
    return s.compute_eff_moduli(load, list(lt), nts)


def same(a, b, rtol):
    if a == b or (math.isnan(a) and math.isnan(b)):
        return True
    return abs(a - b) <= rtol * abs(b)


def check_result(r, ref, rtol, nl):
    assert r["total_iterations"] == ref["total_iterations"]
    keys = ["kphi", "kd"] + (["g"] if nl == 3 else [])
    for kind in ("num", "num_per", "an", "an_per"):
        for k in keys:
            assert same(r[kind][k], ref[kind][k], rtol), (kind, k, r[kind][k], ref[kind][k])


SHAPES = [(ep.KERNEL_AUTO, 0), (ep.KERNEL_TILE, 8), (ep.KERNEL_TILE, 32), (ep.KERNEL_STREAM, 32),
          (ep.KERNEL_STREAM, 128)]


@pytest.mark.parametrize("kernel,rows", SHAPES, ids=["auto", "tile8", "tile32", "stream32", "stream128"])
def test_batch_matches_single_fp64(kernel, rows):
    specs = [mk(*s) for s in SPECS]
    res, st = B.batch_solve(specs, niter=NITER, eiter=1e-9, check_every=CE, rows=rows, kernel=kernel)
    assert st["launches"] > 0 and st["kernel"] in (ep.KERNEL_TILE, ep.KERNEL_STREAM)
    if rows:
        assert st["rows"] == rows and st["kernel"] == (kernel or ep.KERNEL_STREAM)
    else:
        assert st["n_tuned"] == 7 and all(u > 0 for u in st["tune_us"])
    # with rows = 0 the first 168 launches time seven kernel shapes on the live solution;
    # the shapes round alike, so the result is still exact
    for sp, r in zip(SPECS, res):
        check_result(r, single(sp), 0.0, sp[4])


def test_batch_mixed_precision_moduli_error():
    # FP32 velocity storage: moduli within 1e-5 of the FP64 path (measured ~1e-10)
    specs = [mk(*s) for s in SPECS]
    res, st = B.batch_solve(specs, niter=NITER, eiter=1e-9, check_every=CE, precision=ep.MIXED)
    for sp, r in zip(SPECS, res):
        ref = single(sp, st["kernel"], st["rows"])
        keys = ["kphi", "kd"] + (["g"] if sp[4] == 3 else [])
        for k in keys:
            a, b = r["num"][k], ref["num"][k]
            if math.isfinite(b):
                assert abs(a - b) <= 1e-5 * abs(b), (sp, k, a, b)


def test_server_result_same_alone_and_in_mix():
    target = mk(*SPECS[1])
    others = [mk(*s) for s in SPECS]
    shape = dict(kernel=ep.KERNEL_STREAM, rows=64)  # one form for both runs
    with B.Server(mem_budget_bytes=1 << 34, niter=NITER, eiter=1e-9, check_every=CE, **shape) as srv:
        t_alone = srv.submit(target)
        alone, lat_alone, _ = srv.wait(t_alone)
    with B.Server(mem_budget_bytes=1 << 34, niter=NITER, eiter=1e-9, check_every=CE, **shape) as srv:
        tickets = [srv.submit(s) for s in others[:3]]
        t_mix = srv.submit(target)
        tickets += [srv.submit(s) for s in others[3:]]
        mix, lat_mix, _ = srv.wait(t_mix)
        for t in tickets:
            assert srv.wait(t, timeout_ms=600000) is not None
        st = srv.stats()
    assert st["finished"] == len(others) + 1
    check_result(mix, alone, 0.0, SPECS[1][4])
    assert lat_alone > 0 and lat_mix > 0


def test_server_admission_by_memory_budget():
    # a budget that fits about one RVE at a time: requests queue, all complete in order
    specs = [mk(*s) for s in SPECS[:4]]
    biggest = max(B.footprint(s) for s in specs)
    with B.Server(mem_budget_bytes=biggest + 1, niter=NITER, eiter=1e-9, check_every=CE, kernel=ep.KERNEL_STREAM,
                  rows=64) as srv:
        tickets = [srv.submit(s) for s in specs]
        outs = [srv.wait(t, timeout_ms=600000) for t in tickets]
        st = srv.stats()
    assert all(o is not None for o in outs)
    assert st["admitted"] == len(specs)
    # queueing happened: later requests waited in the queue
    assert max(o[2] for o in outs) > 0.0
    for sp, o in zip(SPECS[:4], outs):
        check_result(o[0], single(sp), 0.0, sp[4])


def test_server_ticket_results_are_collected_once():
    # the wait that reports a result releases it; waits on that ticket again, or on a
    # ticket the server never issued, are argument errors (they do not block)
    with B.Server(mem_budget_bytes=1 << 34, niter=NITER, eiter=1e-9, check_every=CE, kernel=ep.KERNEL_STREAM,
                  rows=64) as srv:
        t = srv.submit(mk(*SPECS[0]))
        assert srv.wait(t, timeout_ms=600000) is not None
        for bad in (t, t + 1000):
            with pytest.raises(ep.EP2DError) as ei:
                srv.wait(bad)
            assert ei.value.status == ep.ERR_ARG


def test_server_fails_every_request_after_an_engine_error(monkeypatch):
    # host-side fault injection: the worker treats its second checkpoint interval as a
    # failed CUDA call; every admitted and queued request ends with that status (with
    # EITER 1e-30 none converges first), waits return at once, and submissions are refused
    monkeypatch.setenv("EP2D_SERVER_FAIL_AFTER", "2")
    specs = [mk(*s) for s in SPECS]
    with B.Server(mem_budget_bytes=2 * B.footprint(specs[1]), niter=NITER, eiter=1e-30, check_every=CE,
                  kernel=ep.KERNEL_STREAM, rows=64) as srv:
        tickets = [srv.submit(s) for s in specs]
        for t in tickets:
            with pytest.raises(ep.EP2DError) as ei:
                srv.wait(t, timeout_ms=600000)
            assert ei.value.status == ep.ERR_CUDA and "injected" in str(ei.value), str(ei.value)
        st = srv.stats()
        assert st["finished"] == len(specs) and st["bytes_in_use"] == 0
        with pytest.raises(ep.EP2DError) as ei:
            srv.submit(specs[0])
        assert ei.value.status == ep.ERR_STATE


# Batched-workload-sized RVEs (grid sides 256..1024, pores 1..4, parameters inside the
# batched workload's ranges: porosity U(0.005, 0.05), Y in [5e-6, 5e-5], preload
# magnitude in [2e-5, 8e-5]), every time step solved to convergence: the mixed-precision
# batch against the plain FP64 single-RVE path, RVE by RVE, at the 1e-5 bar.
LARGE = [
    # n, pores, porosity, Y, nl, load, load type, time steps
    (256, 1, 0.01, 5e-5, 3, -2e-5, (0.9, 1.0, 0.3), 1),
    (512, 2, 0.02, 4e-5, 2, -3e-5, (1.0, 0.8, 0.0), 1),
    (768, 3, 0.01, 5e-5, 2, -2e-5, (1.0, 1.0, 0.0), 1),
    (1024, 4, 0.005, 5e-5, 3, -2e-5, (1.0, 0.9, 0.2), 1),
]


def test_batch_mixed_matches_fp64_at_batched_workload_sizes():
    niter, ce = 2_000_000, 10_000
    specs = [mk(*s) for s in LARGE]
    res, st = B.batch_solve(specs, niter=niter, eiter=1e-9, check_every=ce, precision=ep.MIXED)
    for sp, r in zip(LARGE, res):
        n, npo, phi, Y, nl, load, lt, nts = sp
        pa = ep.make_pa(20.0, 20.0, n, n, g0=0.5, yield_stress=Y, porosity=phi, n_pores=npo)
        s = ep.Solver(n, n, pa, nl=nl, niter=niter, eiter=1e-9, check_every=ce)
        ref = s.compute_eff_moduli(load, list(lt), nts)
        s.close()
        assert ref["all_converged"] and r["all_converged"], (sp, ref["total_iterations"], r["total_iterations"])
        assert r["total_iterations"] == ref["total_iterations"], sp
        for kind in ("num", "num_per"):
            for k in ["kphi", "kd"] + (["g"] if nl == 3 else []):
                a, b = r[kind][k], ref[kind][k]
                if math.isfinite(b) and b != 0.0:
                    print("n=%d %s %s: mixed batch %.12g FP64 %.12g rel %.2e" % (n, kind, k, a, b,
                                                                               abs(a - b) / abs(b)))
                    assert abs(a - b) <= 1e-5 * abs(b), (sp, kind, k, a, b)


def test_batch_with_gpu_filling_rve_matches_single_bit_for_bit():
    # a 1024^2 RVE fills the GPU alone, so the batch runs it through the single-RVE path
    # while the small ones share batched launches; every path rounds alike, so each RVE
    # must equal its single-RVE run exactly (iteration-capped steps: NITER 20000)
    niter, ce = 20000, 10000
    specs_p = [(1024, 3, 0.01, 1e-5, 2, -6e-5, (1.0, 1.0, 0.0), 1),
               (96, 3, 0.02, 1e-5, 3, -6e-5, (1.0, 0.8, 0.3), 1),
               (128, 1, 0.01, 2e-5, 2, -5e-5, (0.9, 1.0, 0.2), 1)]
    specs = [mk(*s) for s in specs_p]
    res, st = B.batch_solve(specs, niter=niter, eiter=1e-9, check_every=ce)
    assert st["solo_intervals"] > 0
    for sp, r in zip(specs_p, res):
        n, npo, phi, Y, nl, load, lt, nts = sp
        pa = ep.make_pa(20.0, 20.0, n, n, g0=0.5, yield_stress=Y, porosity=phi, n_pores=npo)
        s = ep.Solver(n, n, pa, nl=nl, niter=niter, eiter=1e-9, check_every=ce)
        ref = s.compute_eff_moduli(load, list(lt), nts)
        s.close()
        check_result(r, ref, 0.0, nl)
