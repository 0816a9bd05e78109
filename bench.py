#!/usr/bin/env python
"""bench.py -- converged RVE solves/s of the EffPlast2D pseudo-transient solver on B200.

The headline workload is the 1024^2 elastoplastic RVE (3x3 pores): one converged solve
is the reference's ComputeEffModuli chain (preload over 2 time steps, then the bulk
increment, each iterated to EITER with the reference's checkpoint cadence), 7,050,000
pseudo-time iterations in the reference's own run and in this implementation.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME] [--impl ours|reference]

value: one step = one checkpoint interval (10,000 pseudo-time iterations, the last
recording max|V| and the stresses as the convergence check does) of the preloaded RVE,
device-timed with CUDA events; solves/s = iterations/s / iterations per solve.
e2e: complete converged solves (--e2e-solves, default 1) through the C ABI from host
inputs: create, the whole chain, the output fields back to host memory, destroy.

Multi-GPU (torchrun, one rank per GPU): every rank iterates / solves its own RVE
(independent replicas, no collective on the data path), timed between barriers; the
time is the max over ranks; value = work of all ranks / that time ("scaling": "weak").

--impl reference times the reference algorithm on the host cores (the CPU restatement
of EffPlast2D.cu's four kernels, all threads): each step is the same 10,000-iteration
step of the same preloaded RVE, host-timed, and solves/s uses the same iteration count.
Rank 0 only.  Both cpu_baseline objects add a single-thread sample of the same
restatement.  Both arms print the same `config` object.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

# ---- workloads (synthetic by construction: the reference has no dataset) -----------
WORKLOADS = {
    # the configuration the metric is quoted on (1024^2, 3x3 pores, elastoplastic)
    "cfg2": dict(n=1024, n_pores=3, porosity=0.01, g0=0.5, yield_stress=1e-5, load=-6e-5, load_type=(1.0, 1.0, 0.0),
                 n_time_steps=2, nl=2, niter=5_000_000, eiter=1e-9, check_every=10_000,
                 label="1024x1024 grid, 3x3 pores, porosity 0.01, K0=1 G0=0.5 Y=1e-5, preload -6e-5*[1,1,0] "
                       "over 2 time steps + bulk increment (NL=2), eIter 1e-9"),
    # config 3 geometry (2048^2, 4x4 pores, shear load, NL=3), larger than L2 in FP64
    "cfg3": dict(n=2048, n_pores=4, porosity=0.02, g0=0.5, yield_stress=1e-5, load=-6e-5, load_type=(1.0, 1.0, 0.5),
                 n_time_steps=1, nl=3, niter=5_000_000, eiter=1e-9, check_every=10_000,
                 label="2048x2048 grid, 4x4 pores, porosity 0.02, K0=1 G0=0.5 Y=1e-5, preload -6e-5*[1,1,0.5] "
                       "+ bulk and shear increments (NL=3), eIter 1e-9"),
    # single small RVEs of the batched workload's kind (sides 256 and 512): too small to
    # fill the GPU, where one iteration is a few microseconds and the launch boundary counts
    "rve256": dict(n=256, n_pores=2, porosity=0.02, g0=0.5, yield_stress=1e-5, load=-6e-5, load_type=(1.0, 1.0, 0.5),
                   n_time_steps=1, nl=3, niter=2_000_000, eiter=1e-9, check_every=10_000,
                   label="256x256 grid, 2x2 pores, porosity 0.02, K0=1 G0=0.5 Y=1e-5, preload -6e-5*[1,1,0.5] "
                         "+ bulk and shear increments (NL=3), eIter 1e-9"),
    "rve512": dict(n=512, n_pores=2, porosity=0.02, g0=0.5, yield_stress=1e-5, load=-6e-5, load_type=(1.0, 1.0, 0.5),
                   n_time_steps=1, nl=3, niter=2_000_000, eiter=1e-9, check_every=10_000,
                   label="512x512 grid, 2x2 pores, porosity 0.02, K0=1 G0=0.5 Y=1e-5, preload -6e-5*[1,1,0.5] "
                         "+ bulk and shear increments (NL=3), eIter 1e-9"),
    # the reference's CPU-runnable case (elastic, one pore)
    "cfg1": dict(n=128, n_pores=1, porosity=0.005, g0=0.5, yield_stress=1.0, load=-4e-5, load_type=(1.0, 1.0, 0.0),
                 n_time_steps=1, nl=1, niter=100_000, eiter=1e-9, check_every=10_000,
                 label="128x128 grid, 1 pore, porosity 0.005, K0=1 G0=0.5 Y=1, preload -4e-5*[1,1,0] (NL=1), "
                       "eIter 1e-9"),
}
L2_FLUSH_BYTES = 256 << 20  # > 126 MB L2


def make_pa(w):
    from effplast2d_b200 import make_pa as lib_make_pa

    n = w["n"]
    return lib_make_pa(20.0, 20.0, n, n, g0=w["g0"], yield_stress=w["yield_stress"], porosity=w["porosity"],
                       n_pores=w["n_pores"])


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload):
    """DRAM bytes per launch of the iteration kernel from the committed ncu summary."""
    p = os.path.join(ROOT, "profiles", "iter_stream_%s.json" % workload)
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("dram_bytes_per_launch")
    return None


class ClockSampler:
    """nvidia-smi samples every 200 ms while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = str(device_index)
        self.rows = []
        self.proc = None
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                                          "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
        except OSError:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()
        # nvidia-smi's start-up (NVML initialisation) must not fall inside the timed
        # region: wait for its first sample
        t = time.time()
        while not self.rows and time.time() - t < 5.0 and self.proc.poll() is None:
            time.sleep(0.05)

    def _read(self):
        for line in self.proc.stdout:
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9 and p[0] == self.dev:
                self.rows.append(p)

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        if self.thread is not None:
            self.thread.join(timeout=2)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in self.rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def shard(n_items, rank, world):
    """RVE indices this rank solves: independent units, round-robin, no overlap."""
    return list(range(rank, n_items, world))


def reduce_over_ranks(values, op, device=None):
    """max / sum of a list of floats over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(values, dtype=torch.float64, device=device)
    if dist.is_available() and dist.is_initialized() and dist.get_world_size() > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return [float(v) for v in t.cpu()]


def cpu_sample(w, seconds=12.0, threads=None):
    """The CPU restatement of the reference on `threads` host threads, iterating the
    workload's preloaded state: returns (cell updates per second, threads, description)."""
    import oracle

    threads = threads or host_threads()
    oracle.set_threads(threads)
    n = w["n"]
    pa = make_pa_oracle(w)
    o = oracle.Oracle(n, n, pa, nl=w["nl"], niter=1, eiter=w["eiter"], check_every=w["check_every"])
    ux, uy = preloaded_state(w)
    o.set("Ux", ux)
    o.set("Uy", uy)
    o.iterate(2)
    t = time.perf_counter()
    o.iterate(10)
    dt = time.perf_counter() - t
    iters = max(10, int(seconds / max(dt / 10, 1e-9)))
    t = time.perf_counter()
    o.iterate(iters)
    dt = time.perf_counter() - t
    o.close()
    rate = iters * n * n / dt
    return rate, threads, "%d pseudo-time iterations of the %dx%d preloaded state (%.1f s)" % (iters, n, n, dt)


def make_pa_oracle(w):
    import oracle

    n = w["n"]
    return oracle.make_pa(20.0, 20.0, n, n, g0=w["g0"], yield_stress=w["yield_stress"], porosity=w["porosity"],
                          n_pores=w["n_pores"])


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def bench_config(w, workload, world, ips):
    """The `config` object both arms print: it names the workload and the step, nothing
    about the implementation that runs it, so the two arms' objects are equal."""
    return {"workload": workload, "description": w["label"],
            "step": "%d pseudo-time iterations (one checkpoint interval) of the preloaded RVE" % w["check_every"],
            "iterations_per_solve": ips,
            "value_from": "solves/s = iterations/s / iterations_per_solve (recorded from the reference's own run of "
                          "this workload and reproduced exactly by this implementation)",
            "global_batch": world,
            "l2": "device arm: a 256 MB buffer is written between timed steps (the %d^2 state, %.0f MB, is "
                  "L2-resident within a step); host arm: no device" % (w["n"], 13 * 8 * w["n"] ** 2 / 1e6),
            "parallelism": "replicas x%d" % world}


def run_reference(args, w):
    """The reference algorithm on the host cores: the CPU restatement of EffPlast2D.cu's
    four kernels (oracle, OpenMP over all host threads), one step = the same
    check_every-iteration step of the same preloaded RVE as the device arm, timed with
    the host clock.  Warm-up steps are shorter (200 iterations): they only warm the
    caches and the thread pool."""
    world, rank, _ = dist_setup()
    if rank != 0:
        return 0
    ips = iterations_per_solve(args.workload)
    if not ips:
        print(json.dumps({"impl": "reference", "unavailable": "no recorded reference run of workload %s" % args.workload}))
        return 0
    import oracle

    n = w["n"]
    step_iters = int(os.environ.get("EP2D_REF_STEP_ITERS", str(w["check_every"])))
    threads = host_threads()
    oracle.set_threads(threads)
    o = oracle.Oracle(n, n, make_pa_oracle(w), nl=w["nl"], niter=1, eiter=w["eiter"], check_every=w["check_every"])
    ux, uy = preloaded_state(w)
    o.set("Ux", ux)
    o.set("Uy", uy)
    for _ in range(args.warmup):
        o.iterate(200)
    times = []
    for _ in range(args.steps):
        t = time.perf_counter()
        o.iterate(step_iters)
        times.append(time.perf_counter() - t)
    o.close()
    total = sum(times)
    iters_per_s = args.steps * step_iters / total
    v = iters_per_s / ips
    rate1, _, desc1 = cpu_sample(w, seconds=float(os.environ.get("EP2D_CPU_SAMPLE_1T_S", "4")), threads=1)
    desc = ("%d steps of %d pseudo-time iterations of the %dx%d preloaded state on %d host threads (%.1f s); "
            "solves/s = iterations/s / %d iterations per solve (the reference's own run)"
            % (args.steps, step_iters, n, n, threads, total, ips))
    line = {
        "impl": "reference", "metric": "converged RVE solves/s", "value": v, "unit": "RVE solves/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": bench_config(w, args.workload, world, ips),
        "implementation": "CPU restatement of EffPlast2D.cu's four kernels (ComputeStress, ComputeJ2, "
                          "ComputePlasticity, ComputeDisp), unfused as the reference runs them, FP64",
        "cpu_baseline": {"value": v, "unit": "RVE solves/s", "cores": threads, "kind": "port", "sample": desc,
                         "single_thread": {"value": rate1 / (n * n * ips), "cores": 1, "sample": desc1}},
        # the host arm has no host<->device traffic: its end-to-end rate is its rate
        "e2e": {"value": v, "unit": "RVE solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "step": "the same host step as value (no device, nothing to copy)"},
        "cell_updates_per_s": iters_per_s * n * n,
    }
    print(json.dumps(line))
    return 0


def preloaded_state(w):
    """Ux, Uy of the workload's first preload increment (an affine strain field), the
    state both the device step and the CPU sample iterate from."""
    import numpy as np

    n = w["n"]
    dx = 20.0 / (n - 1)
    e = w["load"] / w["n_time_steps"]
    xi = -0.5 * dx * n + dx * np.arange(n + 1)
    yj = -0.5 * dx * n + dx * np.arange(n + 1)
    ux = np.ascontiguousarray(np.broadcast_to(e * w["load_type"][0] * xi[None, :], (n, n + 1)))
    uy = np.ascontiguousarray(np.broadcast_to(e * w["load_type"][1] * yj[:, None], (n + 1, n)))
    return ux, uy


def iterations_per_solve(workload):
    """Pseudo-time iterations of one converged solve of the workload, recorded from the
    reference's own run (tests/golden/<workload>.json); this implementation reproduces
    the count exactly (tests/test_golden_cfg2.py)."""
    p = os.path.join(ROOT, "tests", "golden", workload + ".json")
    if os.path.exists(p):
        return json.load(open(p)).get("total_iterations")
    return None


def run_ours(args, w):
    import torch

    import effplast2d_b200 as ep

    world, rank, local = dist_setup()
    dev = local if world > 1 else 0
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600), device_id=torch.device("cuda", dev))
    n = w["n"]
    pa = make_pa(w)
    lt = list(w["load_type"])
    step_iters = w["check_every"]
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if world > 1:
            import torch.distributed as dist

            dist.barrier()
        torch.cuda.synchronize()

    # value: every rank iterates its own RVE (replicas, no collective); one step = one
    # checkpoint interval (check_every pseudo-time iterations, the last one recording
    # the stresses and max|V| as the convergence check does) of the preloaded state
    s = ep.Solver(n, n, pa, nl=w["nl"], niter=w["niter"], eiter=w["eiter"], check_every=w["check_every"], device=dev,
                  kernel=args.kernel, rows=args.rows)
    ux, uy = preloaded_state(w)
    s.set("Ux", ux)
    s.set("Uy", uy)
    for _ in range(args.warmup):
        s.iterate(step_iters)
    st0 = s.stats()
    clocks = ClockSampler(dev)
    clocks.start()
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record()
    for _ in range(args.steps):
        flush.zero_()
        s.iterate(step_iters)
    ev1.record()
    ev1.synchronize()
    barrier()
    clocks.stop()
    ms = ev0.elapsed_time(ev1)
    st1 = s.stats()
    shape = s.kernel_shape()
    s.close()

    # e2e: complete converged solves through the C ABI from host inputs: create (pa.dat
    # values and the pore-edge sample list to the device, mask set-up), the reference's
    # whole ComputeEffModuli chain, the output fields it writes (Pc, tauXXc) back to
    # host memory, destroy
    h2d = 8 * (len(pa) + 20 * int(w["n_pores"]) ** 2)
    d2h = 2 * n * n * 8
    res = None
    e2e_ms = None
    if args.e2e_solves > 0:
        barrier()
        t0 = time.perf_counter()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(args.e2e_solves):
            flush.zero_()
            s2 = ep.Solver(n, n, pa, nl=w["nl"], niter=w["niter"], eiter=w["eiter"], check_every=w["check_every"],
                           device=dev, kernel=args.kernel, rows=args.rows)
            res = s2.compute_eff_moduli(w["load"], lt, w["n_time_steps"])
            s2.get("P")
            s2.get("tauXX")
            s2.close()
        e1.record()
        e1.synchronize()
        barrier()
        e2e_ms = max(e0.elapsed_time(e1), 1000.0 * (time.perf_counter() - t0))

    # device time: max over ranks; kernel launches: summed over ranks
    ms, e2e_max = reduce_over_ranks([ms, e2e_ms or 0.0], "max", device="cuda")
    launches = int(reduce_over_ranks([float(st1["all_launches"] - st0["all_launches"])], "sum", device="cuda")[0])

    # roofline of the fused iteration kernel over the timed region
    it_launches = st1["launches"] - st0["launches"]
    it_ms = st1["kernel_ms"] - st0["kernel_ms"]
    avg_launch_s = it_ms / 1000.0 / max(it_launches, 1)
    bytes_alg = 64 * n * n  # Ux, Uy, Vx, Vy read once and written once, FP64
    achieved = bytes_alg / avg_launch_s / 1e9
    peak, peak_kind = measured_peaks()
    ips = iterations_per_solve(args.workload) or (res["total_iterations"] if res else None)

    line = None
    if rank == 0:
        iters_per_s = world * args.steps * step_iters / (ms / 1000.0)
        value = iters_per_s / ips
        line = {
            "metric": "converged RVE solves/s", "value": value, "unit": "RVE solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": bench_config(w, args.workload, world, ips),
            "kernel": {"form": KERNEL_NAMES[shape[0]], "rows": shape[1]},
            "e2e": None,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": ncu_traffic(args.workload),
                         "kernel": "k_iter_stream (fused stress, J2 return, momentum update)",
                         "algorithmic_bytes_per_launch": bytes_alg, "avg_launch_us": avg_launch_s * 1e6,
                         "peak_source": peak_kind,
                         "note": "the %d^2 state (%.0f MB) is L2-resident within a step, so this fraction "
                                 "measures throughput against a bound the kernel does not meet here; the "
                                 "HBM-resident case of the same kernel is roofline_hbm" % (n, 13 * 8 * n * n / 1e6)},
            "gpu_launches": launches,
            "clocks": clocks.summary(),
            "cell_updates_per_s": iters_per_s * n * n,
        }
        if e2e_ms:
            line["e2e"] = {"value": world * args.e2e_solves / (e2e_max / 1000.0), "unit": "RVE solves/s",
                           "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                           "steps": args.e2e_solves, "step": "one complete converged solve (create, "
                           "ComputeEffModuli chain, Pc and tauXXc to host, destroy)",
                           "iterations_per_solve": res["total_iterations"],
                           "moduli": {"kd": res["num"]["kd"], "kphi": res["num"]["kphi"], "g": res["num"]["g"]}}
        if world == 1 and not args.no_cpu_baseline:
            rate, threads, desc = cpu_sample(w, seconds=float(os.environ.get("EP2D_CPU_SAMPLE_S", "12")))
            rate1, _, desc1 = cpu_sample(w, seconds=float(os.environ.get("EP2D_CPU_SAMPLE_1T_S", "4")), threads=1)
            v = rate / (n * n * ips)
            line["cpu_baseline"] = {"value": v, "unit": "RVE solves/s", "cores": threads, "kind": "port",
                                    "sample": desc + "; converted with %d iterations per solve" % ips,
                                    "single_thread": {"value": rate1 / (n * n * ips), "cores": 1, "sample": desc1}}
        if world == 1 and not args.no_extras:
            # the HBM-bound case of the same kernel (the 1024^2 state above is L2-resident)
            line["roofline_hbm"] = dict(kernel_timing("cfg3", args.hbm_iters),
                                        note="2048x2048 grid, FP64: 13 fields of 34 MB (0.45 GB) > 126 MB L2; "
                                             "achieved = 64 B x 2048^2 per launch / CUDA-event time per launch; "
                                             "traffic from the committed ncu capture of this kernel and grid")
            # the metric's batched and served headline, sized to fit this run
            sides = tuple(int(x) for x in args.extra_sides.split(","))
            line["batched"] = batch_object(args.extra_batch, args.seed, args.extra_niter, sides=sides)
            line["served"] = serve_object(args.extra_requests, args.seed, args.extra_rate, args.extra_niter,
                                          sides=sides)
    if world > 1:
        import torch.distributed as dist

        dist.barrier()
        dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line))
    return 0


def kernel_timing(workload, iters, kernel=0, rows=0, precision="fp64", w=None):
    """Exactly `iters` pseudo-time iterations of the workload's preload step (no
    convergence test), after one untimed pass of the same length: CUDA-event time per
    launch of the fused iteration kernel on its own stream, and its HBM roofline.
    precision "f32": the FP32 bulk's FP32 form (32 B per cell-update: u' and V in FP32)."""
    import torch

    import effplast2d_b200 as ep

    w = w or WORKLOADS[workload]
    n = w["n"]
    prec = {"fp64": ep.FP64, "mixed": ep.MIXED, "f32": ep.F32_BULK}[precision]
    s = ep.Solver(n, n, make_pa(w), nl=w["nl"], niter=iters, eiter=0.0, check_every=iters, device=0,
                  kernel=kernel, rows=rows, precision=prec)
    s.solve_step(0, w["load"], list(w["load_type"]), 1)  # warm-up and preload
    if precision == "f32":
        s.iterate_f32(iters)
    st0 = s.stats()
    torch.cuda.synchronize()
    t = time.perf_counter()
    if precision == "f32":
        s.iterate_f32(iters)
    else:
        s.solve_step(0, w["load"], list(w["load_type"]), 1)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t
    st1 = s.stats()
    shape = s.kernel_shape()
    s.close()
    # per iteration (a resident-form launch runs many)
    iters_run = (st1["cell_updates"] - st0["cell_updates"]) // (n * n)
    per = (st1["kernel_ms"] - st0["kernel_ms"]) / max(iters_run, 1)
    bytes_alg = {"fp64": 64, "mixed": 48, "f32": 32}[precision] * n * n
    peak, kind = measured_peaks()
    achieved = bytes_alg / (per / 1e3) / 1e9
    return {"workload": workload, "grid": "%dx%d" % (n, n), "iterations": iters, "precision": precision,
            "kernel": {"form": KERNEL_NAMES[shape[0]], "rows": shape[1]},
            "iteration_launches": st1["launches"] - st0["launches"],
            "avg_launch_us": per * 1e3, "algorithmic_bytes_per_launch": bytes_alg, "achieved": achieved,
            "peak": peak, "unit": "GB/s", "peak_source": kind, "frac": achieved / peak,
            "traffic": ncu_traffic(workload), "wall_s": wall, "cell_updates_per_s": n * n / (per / 1e3)}


KERNEL_NAMES = {0: "auto", 1: "tile", 2: "stream", 3: "resident"}


def run_solve_only(args, w):
    """One complete ComputeEffModuli solve of the workload with the chosen kernel form:
    device time, iterations, time per iteration and the moduli."""
    import effplast2d_b200 as ep

    n = w["n"]
    s = ep.Solver(n, n, make_pa(w), nl=w["nl"], niter=w["niter"], eiter=w["eiter"], check_every=w["check_every"],
                  device=0, kernel=args.kernel, rows=args.rows)
    shape = s.kernel_shape()
    t = time.perf_counter()
    r = s.compute_eff_moduli(w["load"], list(w["load_type"]), w["n_time_steps"])
    wall = time.perf_counter() - t
    st = s.stats()
    s.close()
    iters = st["cell_updates"] // (n * n)
    print(json.dumps({"workload": args.workload, "kernel": {"form": KERNEL_NAMES[shape[0]], "rows": shape[1]},
                      "wall_s": wall, "kernel_ms": st["kernel_ms"], "iterations": iters,
                      "iteration_launches": st["launches"], "us_per_iteration": st["kernel_ms"] * 1e3 / max(iters, 1),
                      "all_converged": bool(r["all_converged"]), "num": r["num"]}))
    return 0


def run_kernel_only(args, w):
    """The fixed, short launch sequence used for ncu captures and for timing the fused
    iteration kernel alone."""
    print(json.dumps(kernel_timing(args.workload, args.kernel_only, args.kernel, args.rows, args.precision, w)))
    return 0


def sample_requests(count, seed, sides=(256, 512, 768, 1024)):
    """Seeded RVEs with the batched/served workload's distributions: grid side uniform in
    `sides`, nPores uniform in 1..4, porosity U(0.005, 0.05), Y log-uniform in
    [5e-6, 5e-5], preload magnitude U(2e-5, 8e-5) along a random unit load type with
    |xy| <= 0.5 (compressive xx, yy), NL uniform in {2, 3}, one time step."""
    import math

    import numpy as np

    from effplast2d_b200 import batch as B

    rng = np.random.default_rng(seed)
    out = []
    for _ in range(count):
        n = int(rng.choice(sides))
        npores = int(rng.integers(1, 5))
        phi = float(rng.uniform(0.005, 0.05))
        yld = float(math.exp(rng.uniform(math.log(5e-6), math.log(5e-5))))
        mag = float(rng.uniform(2e-5, 8e-5))
        th = float(rng.uniform(math.pi / 8, 3 * math.pi / 8))
        lt = np.array([math.cos(th), math.sin(th), float(rng.uniform(-0.5, 0.5))])
        lt /= np.linalg.norm(lt)
        nl = int(rng.integers(2, 4))
        pa = make_pa({"n": n, "g0": 0.5, "yield_stress": yld, "porosity": phi, "n_pores": npores})
        out.append({"spec": B.spec(n, pa, nl, 1, -mag, tuple(lt)), "n": n, "nl": nl, "pa": pa, "load": -mag,
                    "lt": list(lt)})
    return out


def batch_object(count, seed, niter, sides=(256, 512, 768, 1024)):
    """Batched mixed-precision solve of `count` seeded RVEs of the batched workload's
    distribution against the plain FP64 single-RVE path solving the same RVEs one at a
    time (host wall clock around each leg, device work included)."""
    import numpy as np
    import torch

    import effplast2d_b200 as ep
    from effplast2d_b200 import batch as B

    reqs = sample_requests(count, seed, sides=sides)
    torch.cuda.synchronize()
    t = time.perf_counter()
    res_b, st = B.batch_solve([r["spec"] for r in reqs], niter=niter, eiter=1e-9, check_every=10_000,
                              precision=ep.MIXED)
    torch.cuda.synchronize()
    t_batch = time.perf_counter() - t
    t = time.perf_counter()
    res_s = []
    for r in reqs:
        s = ep.Solver(r["n"], r["n"], r["pa"], nl=r["nl"], niter=niter, eiter=1e-9, check_every=10_000)
        res_s.append(s.compute_eff_moduli(r["load"], r["lt"], 1))
        s.close()
    t_single = time.perf_counter() - t
    # The moduli error is a property of converged solves: an RVE whose time step stops at
    # NITER in either run compares two unconverged states, whose difference is set by the
    # residual left, not by the precision.  Both are reported, separately.
    errs = {k: [] for k in ("kphi", "kd", "g")}
    errs_capped = {k: [] for k in ("kphi", "kd", "g")}
    n_conv = 0
    same_iters = True
    for rb, rs, r in zip(res_b, res_s, reqs):
        both = bool(rb["all_converged"]) and bool(rs["all_converged"])
        n_conv += both
        same_iters &= rb["total_iterations"] == rs["total_iterations"]
        for k in errs:
            if k == "g" and r["nl"] < 3:
                continue
            a, b = rb["num"][k], rs["num"][k]
            if np.isfinite(b) and b != 0:
                (errs if both else errs_capped)[k].append(abs(a - b) / abs(b))
    cells = sum(r["n"] ** 2 * rs["total_iterations"] for r, rs in zip(reqs, res_s))
    return {
        "rves": len(reqs), "seed": seed, "sides": sorted({r["n"] for r in reqs}),
        "distribution": "grid side uniform in %s, nPores U{1..4}, porosity U(0.005, 0.05), Y log-uniform "
                        "[5e-6, 5e-5], preload U(2e-5, 8e-5) along a random unit load type (|xy| <= 0.5), "
                        "NL U{2, 3}, one time step" % (list(sides),),
        "niter": niter, "precision": "mixed (FP32 velocities, FP64 stencil arithmetic and reductions)",
        "batched_solves_per_s": len(reqs) / t_batch, "single_fp64_solves_per_s": len(reqs) / t_single,
        "speedup": t_single / t_batch, "batched_s": t_batch, "single_fp64_s": t_single,
        "batched_cell_updates_per_s": cells / t_batch, "single_cell_updates_per_s": cells / t_single,
        "converged_rves": n_conv, "same_iteration_counts": bool(same_iters),
        "max_rel_moduli_error": {k: (max(v) if v else None) for k, v in errs.items()},
        "max_rel_moduli_error_capped": {k: (max(v) if v else None) for k, v in errs_capped.items()},
        "kernel": st["kernel"], "rows": st["rows"], "tunes": st["n_tunes"], "solo_intervals": st["solo_intervals"],
        "blocks": st["blocks"],
        "per_rve": [{"n": r["n"], "nl": r["nl"], "iterations": rs["total_iterations"],
                     "converged": bool(rb["all_converged"] and rs["all_converged"])}
                    for r, rb, rs in zip(reqs, res_b, res_s)]}


def run_residency(args):
    """Does keeping an RVE's state on chip pay?  The same batched kernel (stream form,
    32-row segments, FP64) on batches of 256^2 RVEs whose combined state fits in the
    126 MB L2 and on batches that do not: cell-update rate and device time per
    iteration, for fixed iteration counts (no convergence test)."""
    import effplast2d_b200 as ep
    from effplast2d_b200 import batch as B

    out = []
    n = 256
    pa = make_pa({"n": n, "g0": 0.5, "yield_stress": 1e-5, "porosity": 0.02, "n_pores": 3})
    for count in (8, 32, 128, 512):
        specs = [B.spec(n, pa, 2, 1, -6e-5, (1.0, 1.0, 0.0)) for _ in range(count)]
        iters = 20_000
        _, st = B.batch_solve(specs, niter=iters, eiter=0.0, check_every=10_000, kernel=ep.KERNEL_STREAM, rows=32)
        state = count * 13 * 8 * (n + 1) * (n + 1)
        out.append({"rves": count, "state_mb": state / 1e6, "l2_resident": state < 126e6,
                    "us_per_iteration": 1000.0 * st["kernel_ms"] / st["launches"],
                    "cell_updates_per_s": st["cell_updates"] / (st["kernel_ms"] / 1000.0)})
    print(json.dumps({"workload": "residency", "grid": "%dx%d" % (n, n), "kernel": "stream, 32-row segments, FP64",
                      "runs": out}))
    return 0


def run_batch(args):
    sides = tuple(int(x) for x in args.sides.split(",")) if args.sides else (256, 512, 768, 1024)
    print(json.dumps(dict(workload="batch", **batch_object(args.batch_size, args.seed, args.niter, sides=sides))))
    return 0


def run_precision(args):
    """The mixed path (FP32 velocity storage) and the FP32 bulk (FP32 stencil until its
    residual stalls, then FP64) against the plain FP64 path on one workload, each solved to
    convergence through the whole ComputeEffModuli chain: the relative error of every
    modulus, iteration counts (FP32 ones included), solve times."""
    import math

    import effplast2d_b200 as ep

    w = WORKLOADS[args.precision_workload]
    n = w["n"]
    pa = make_pa(w)
    out = {}
    runs = (("fp64", ep.FP64), ("mixed", ep.MIXED), ("f32_bulk", ep.F32_BULK))
    wanted = args.precisions.split(",")
    for name, prec in runs:
        if name not in wanted and name != "fp64":
            continue
        s = ep.Solver(n, n, pa, nl=w["nl"], niter=w["niter"], eiter=w["eiter"], check_every=w["check_every"],
                      precision=prec)
        t = time.perf_counter()
        res = s.compute_eff_moduli(w["load"], list(w["load_type"]), w["n_time_steps"])
        st = s.stats()
        out[name] = {"seconds": time.perf_counter() - t, "total_iterations": res["total_iterations"],
                     "f32_iterations": st["f32_iterations"],
                     "all_converged": bool(res["all_converged"]), "num": res["num"], "num_per": res["num_per"],
                     "kernel_us": 1000 * st["kernel_ms"] / max(st["launches"], 1),
                     "checks": [s.check_errors(k, t_) for k in range(w["nl"])
                                for t_ in range(w["n_time_steps"] if k == 0 else 1)]}
        s.close()
    err = {}
    for name in out:
        if name == "fp64":
            continue
        e = {}
        for kind in ("num", "num_per"):
            for k in ("kphi", "kd", "g"):
                a, b = out[name][kind][k], out["fp64"][kind][k]
                if math.isfinite(a) and math.isfinite(b) and b != 0.0:
                    e["%s_%s" % (kind, k)] = abs(a - b) / abs(b)
                else:
                    e["%s_%s" % (kind, k)] = None  # undefined in both (e.g. G without shear)
        err[name] = e
    print(json.dumps({"workload": "precision", "config": args.precision_workload, "description": w["label"],
                      "relative_error_vs_fp64": err, "runs": out}))
    return 0


def serve_object(count, seed, rate, niter, sides=(256, 512, 768, 1024, 2048)):
    """Poisson stream of `count` requests at `rate`/s into the continuous-batching server
    (mixed precision, 180 GB admission budget): p50/p99 latency, queue time, solves/s."""
    import numpy as np

    import effplast2d_b200 as ep
    from effplast2d_b200 import batch as B

    reqs = sample_requests(count, seed, sides=sides)
    rng = np.random.default_rng(seed + 1)
    gaps = rng.exponential(1.0 / rate, size=len(reqs))
    with B.Server(mem_budget_bytes=int(180e9), niter=niter, eiter=1e-9, check_every=10_000,
                  precision=ep.MIXED) as srv:
        t0 = time.perf_counter()
        tickets = []
        for r, gap in zip(reqs, gaps):
            time.sleep(gap)
            tickets.append(srv.submit(r["spec"]))
        outs = [srv.wait(t) for t in tickets]
        wall = time.perf_counter() - t0
        st = srv.stats()
    lat = np.array([o[1] for o in outs])
    return {
        "requests": len(reqs), "rate_per_s": rate, "seed": seed, "sides": sorted({r["n"] for r in reqs}),
        "niter": niter, "admission_budget_bytes": int(180e9),
        "precision": "mixed (FP32 velocities, FP64 stencil arithmetic and reductions)",
        "solves_per_s": len(reqs) / wall, "wall_s": wall,
        "latency_p50_s": float(np.percentile(lat, 50)), "latency_p99_s": float(np.percentile(lat, 99)),
        "queue_p50_s": float(np.percentile([o[2] for o in outs], 50)),
        "converged_requests": sum(1 for o in outs if o[0]["all_converged"]), "engine": st["engine"]}


def run_serve(args):
    sides = tuple(int(x) for x in args.sides.split(",")) if args.sides else (256, 512, 768, 1024, 2048)
    print(json.dumps(dict(workload="serve", **serve_object(args.batch_size, args.seed, args.rate, args.niter,
                                                           sides=sides))))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--batch-size", type=int, default=32, help="RVEs of the batch / serve workloads")
    ap.add_argument("--sides", default="", help="grid sides of the batch / serve workloads, comma-separated "
                                                "(default 256..1024; serve: up to 2048)")
    ap.add_argument("--seed", type=int, default=2026)
    ap.add_argument("--rate", type=float, default=1.0, help="request rate of the serve workload (1/s)")
    ap.add_argument("--niter", type=int, default=2_000_000, help="NITER of the batch / serve workloads")
    ap.add_argument("--kernel-only", type=int, default=0, metavar="N",
                    help="run N iterations of the workload's preload step and report the kernel timing")
    ap.add_argument("--kernel", type=int, default=0, choices=[0, 1, 2, 3],
                    help="iteration kernel form: 0 library's choice, 1 tile, 2 stream, 3 resident")
    ap.add_argument("--solve-only", action="store_true",
                    help="one complete solve of the workload with --kernel/--rows: time per iteration, moduli")
    ap.add_argument("--rows", type=int, default=0, help="rows per tile / strip segment (0: library's choice)")
    ap.add_argument("--side", type=int, default=0,
                    help="grid side of --kernel-only / --solve-only (0: the workload's own)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--workload", default="cfg2", choices=sorted(WORKLOADS) + ["batch", "serve", "precision", "residency"])
    ap.add_argument("--precisions", default="mixed,f32_bulk",
                    help="paths --workload precision compares with FP64 (mixed, f32_bulk)")
    ap.add_argument("--precision-workload", default="cfg3", choices=sorted(WORKLOADS),
                    help="workload of --workload precision (mixed vs FP64 moduli)")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed", "f32"],
                    help="arithmetic of --kernel-only (f32: the FP32 bulk's FP32 form)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="leave the batched, served and roofline_hbm objects out of the default line")
    ap.add_argument("--extra-batch", type=int, default=16, help="RVEs of the default line's batched object")
    ap.add_argument("--extra-requests", type=int, default=16, help="requests of the default line's served object")
    ap.add_argument("--extra-rate", type=float, default=2.0, help="request rate of the served object (1/s)")
    ap.add_argument("--extra-sides", default="256,512",
                    help="grid sides of the batched and served objects (the batched workload's distribution "
                         "restricted to these sides so that both fit the default run)")
    ap.add_argument("--extra-niter", type=int, default=1_000_000, help="NITER of the batched and served objects")
    ap.add_argument("--hbm-iters", type=int, default=5000, help="iterations timed for roofline_hbm")
    ap.add_argument("--e2e-solves", type=int, default=1,
                    help="complete converged solves timed end to end through the C ABI (0: skip)")
    args = ap.parse_args()
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "residency":
        return run_residency(args)
    if args.workload == "precision":
        return run_precision(args)
    if args.workload == "serve":
        return run_serve(args)
    w = WORKLOADS[args.workload]
    if args.side and (args.kernel_only or args.solve_only):
        w = dict(w, n=args.side)
    if args.kernel_only:
        return run_kernel_only(args, w)
    if args.solve_only:
        return run_solve_only(args, w)
    if args.impl == "reference":
        return run_reference(args, w)
    return run_ours(args, w)


if __name__ == "__main__":
    sys.exit(main())
