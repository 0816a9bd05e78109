"""bench.py's reference arm runs on the host cores only, so its JSON line can be checked
without a GPU: the keys and types the bench contract requires, and the rank rule under a
multi-rank launch (rank 0 alone measures and prints; the others exit 0 without work).
The steps are shortened through the environment so the test takes seconds."""
import json
import os
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def run_reference_arm(extra_env, steps=1):
    env = dict(os.environ, EP2D_REF_STEP_ITERS="3", EP2D_CPU_SAMPLE_1T_S="0.2", **extra_env)
    return subprocess.run([sys.executable, "bench.py", "--impl", "reference", "--steps", str(steps), "--warmup", "0"],
                          cwd=ROOT, env=env, capture_output=True, text=True, timeout=300)


def test_reference_arm_line():
    import bench

    t = time.perf_counter()
    r = run_reference_arm({}, steps=2)
    wall = time.perf_counter() - t
    assert r.returncode == 0, r.stderr
    line = json.loads(r.stdout.strip().splitlines()[-1])
    for key in ("impl", "metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step", "higher_is_better",
                "scaling", "vs_baseline", "dtype", "data", "config", "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["metric"] == "converged RVE solves/s"
    assert line["value"] > 0 and line["higher_is_better"] is True and line["dtype"] == "f64"
    assert line["config"]["workload"] == "cfg2"
    # the same config object as the device arm prints for the same workload and ranks
    ips = bench.iterations_per_solve("cfg2")
    assert line["config"] == bench.bench_config(bench.WORKLOADS["cfg2"], "cfg2", 1, ips)
    # ms_per_step is the time of a step it ran: the timed steps fit in the run
    assert line["steps"] == 2 and 0 < line["steps"] * line["ms_per_step"] / 1000.0 < wall
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    assert cb["single_thread"]["cores"] == 1 and cb["single_thread"]["value"] > 0
    e2e = line["e2e"]
    assert (e2e["value"], e2e["unit"], e2e["h2d_bytes_per_step"], e2e["d2h_bytes_per_step"]) == \
        (line["value"], line["unit"], 0, 0)


def test_reference_arm_other_ranks_exit_quietly():
    r = run_reference_arm({"RANK": "1", "LOCAL_RANK": "1", "WORLD_SIZE": "2"})
    assert r.returncode == 0, r.stderr
    assert r.stdout.strip() == ""
