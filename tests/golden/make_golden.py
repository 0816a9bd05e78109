"""Generate the golden fixtures of tests/golden/ by running the UNMODIFIED reference.

Runs on a machine with a CUDA GPU, using the reference binaries that oracle/Makefile
builds from the reference's own sources into oracle/_ref/ (`make -C oracle ref`):

  harness_kernels   kernel-level: seeded states -> N iterations of the reference's
                    ComputeStress/ComputeJ2/ComputePlasticity/ComputeDisp sequence
  harness_<cfg>     EffPlast2D(nTimeSteps).ComputeEffModuli(...) with the records and
                    all device fields dumped at full precision
  cli_<cfg>         the reference's own main.cu (stdout at 17 digits, EffPlast2D.log,
                    data/*.dat outputs)

Usage: python tests/golden/make_golden.py [out_dir] [--only name,...] [--with-cfg2]
Writes <name>.npz (+ .json metadata) per case into out_dir (default golden_out/ at the repository root).
"""
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
import oracle  # noqa: E402  (pa derivation only: get_sigma_2D.m restatement)

REF = os.path.join(ROOT, "oracle", "_ref")

FIELDS = {  # name -> (width(nx), height(ny))
    "P": (0, 0), "tauXX": (0, 0), "tauYY": (0, 0), "tauXY": (-1, -1), "tauXYav": (0, 0), "J2": (0, 0),
    "J2XY": (-1, -1), "Ux": (1, 0), "Uy": (0, 1), "Vx": (1, 0), "Vy": (0, 1), "K": (0, 0), "G": (0, 0),
}

# kernel-level cases: name, nx, ny, nl, n_pores, porosity, Y, iterations, seed
KERNEL_CASES = [
    ("k32_nl1_it1", 32, 32, 1, 1, 0.02, 2e-5, 1, 11),
    ("k32_nl3_it1", 32, 32, 3, 1, 0.02, 2e-5, 1, 12),
    ("k64x32_nl2_it1", 64, 32, 2, 2, 0.03, 2e-5, 1, 13),
    ("k64_nl3_it100", 64, 64, 3, 3, 0.02, 1e-5, 100, 14),
    ("k32x64_nl1_it100", 32, 64, 1, 2, 0.02, 1.0, 100, 15),
]

# full-chain cases: name, binary suffix, n, n_pores, porosity, G0, Y, load, load type, nTimeSteps
CHAIN_CASES = [
    ("c32_nl1", "g32_nl1", 32, 1, 0.005, 0.5, 1.0, -4e-5, (1.0, 1.0, 0.0), 1),
    ("c64_nl2", "g64_nl2", 64, 2, 0.02, 0.5, 1e-5, -6e-5, (1.0, 1.0, 0.0), 2),
    ("c64_nl3", "g64_nl3", 64, 1, 0.01, 0.5, 1e-5, -5e-5, (1.0, 1.0, 0.5), 1),
    ("c96_nl3", "g96_nl3", 96, 3, 0.02, 0.5, 1e-5, -6e-5, (1.0, 0.8, 0.3), 2),
    ("cfg1", "cfg1", 128, 1, 0.005, 0.5, 1.0, -4e-5, (1.0, 1.0, 0.0), 1),
    # damping mode (ComputeEffDamping, NL >= 4): preload, then 4 sinusoidal increments
    ("c64_nl5", "g64_nl5", 64, 2, 0.02, 0.5, 1e-5, -6e-5, (1.0, 1.0, 0.2), 1),
]
CFG2 = ("cfg2", "cfg2", 1024, 3, 0.01, 0.5, 1e-5, -6e-5, (1.0, 1.0, 0.0), 2)

# the reference builds' macros (oracle/Makefile), recorded with each fixture
MACROS = {
    "g32_nl1": dict(NGRID=1, NL=1, NITER=100000, EITER=1e-9),
    "g64_nl2": dict(NGRID=2, NL=2, NITER=20000, EITER=1e-9),
    "g64_nl3": dict(NGRID=2, NL=3, NITER=20000, EITER=1e-9),
    "g96_nl3": dict(NGRID=3, NL=3, NITER=30000, EITER=1e-9),
    "cfg1": dict(NGRID=4, NL=1, NITER=100000, EITER=1e-9),
    "cfg2": dict(NGRID=32, NL=2, NITER=5000000, EITER=1e-9),
    "g64_nl5": dict(NGRID=2, NL=5, NITER=20000, EITER=1e-9),
}


def dims(name, nx, ny):
    dw, dh = FIELDS[name]
    return nx + dw, ny + dh


def read_field(d, name, nx, ny):
    w, h = dims(name, nx, ny)
    return np.fromfile(os.path.join(d, name + ".bin"), dtype="<f8").reshape(h, w)


def random_state(nx, ny, seed):
    rng = np.random.default_rng(seed)
    dx = 20.0 / (nx - 1)
    xi = -0.5 * dx * nx + dx * np.arange(nx + 1)
    yj = -0.5 * dx * (ny - 1) + dx * np.arange(ny)
    ux = 6e-5 * (-xi[None, :] + 0.3 * yj[:, None]) + 2e-6 * rng.standard_normal((ny, nx + 1))
    xi2 = -0.5 * dx * (nx - 1) + dx * np.arange(nx)
    yj2 = -0.5 * dx * ny + dx * np.arange(ny + 1)
    uy = 6e-5 * (-0.8 * yj2[:, None] + 0.3 * xi2[None, :]) + 2e-6 * rng.standard_normal((ny + 1, nx))
    vx = 1e-7 * rng.standard_normal((ny, nx + 1))
    vy = 1e-7 * rng.standard_normal((ny + 1, nx))
    vx[:, 0] = vx[:, -1] = 0.0
    vx[0, :] = vx[-1, :] = 0.0
    vy[0, :] = vy[-1, :] = 0.0
    vy[:, 0] = vy[:, -1] = 0.0
    return {"Ux": ux, "Uy": uy, "Vx": vx, "Vy": vy}


def run(cmd, cwd=None, timeout=3600):
    t = time.time()
    r = subprocess.run(cmd, cwd=cwd, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("%s failed (%d): %s %s" % (cmd, r.returncode, r.stdout[-2000:], r.stderr[-2000:]))
    return r.stdout, time.time() - t


def kernel_case(out, case):
    name, nx, ny, nl, npores, phi, Y, iters, seed = case
    pa = oracle.make_pa(20.0, 20.0, nx, ny, g0=0.5, yield_stress=Y, porosity=phi, n_pores=npores)
    with oracle.Oracle(nx, ny, pa, nl=nl) as o:
        K, G = o.get("K"), o.get("G")
    st = random_state(nx, ny, seed)
    tin = tempfile.mkdtemp()
    tout = tempfile.mkdtemp()
    np.asarray(pa, dtype="<f8").tofile(os.path.join(tin, "pa.bin"))
    for k, v in dict(st, K=K, G=G).items():
        np.ascontiguousarray(v, dtype="<f8").tofile(os.path.join(tin, k + ".bin"))
    _, dt = run([os.path.join(REF, "harness_kernels"), "kernels", tin, tout, str(nx), str(ny), str(nl), str(iters)])
    res = {"in_" + k: v for k, v in st.items()}
    res["pa"] = np.asarray(pa)
    res["K"], res["G"] = K, G
    for f in FIELDS:
        res["out_" + f] = read_field(tout, f, nx, ny)
    np.savez_compressed(os.path.join(out, name + ".npz"), **res)
    meta = dict(kind="kernels", nx=nx, ny=ny, nl=nl, n_pores=npores, porosity=phi, Y=Y, iterations=iters,
                seed=seed, binary="harness_kernels", seconds=dt)
    json.dump(meta, open(os.path.join(out, name + ".json"), "w"), indent=1)
    shutil.rmtree(tin)
    shutil.rmtree(tout)
    print(name, "%.1fs" % dt, flush=True)


def parse_records(path):
    recs, mod = {}, {}
    head = {}
    for line in open(path):
        p = line.split()
        if len(p) == 2:
            head[p[0]] = p[1]
            continue
        key, s, t = p[0], int(p[1]), int(p[2])
        vals = [float(v) for v in p[3:]]
        if key.startswith("moduli_"):
            mod[key[len("moduli_"):]] = vals
        else:
            recs.setdefault("%d_%d" % (s, t), {})[key] = vals
    return head, recs, mod


def chain_case(out, case, fields_keep=None, with_cli=True):
    name, cfg, n, npores, phi, g0, Y, load, lt, nts = case
    pa = oracle.make_pa(20.0, 20.0, n, n, g0=g0, yield_stress=Y, porosity=phi, n_pores=npores)
    args = ["%.17g" % load, "%.17g" % lt[0], "%.17g" % lt[1], "%.17g" % lt[2], str(nts), "%.17g" % (0.1 * load)]
    meta = dict(kind="chain", n=n, n_pores=npores, porosity=phi, G0=g0, Y=Y, load=load, load_type=list(lt),
                n_time_steps=nts, macros=MACROS[cfg], pa=list(pa), argv=args)
    res = {"pa": np.asarray(pa)}
    # 1) harness: full-precision records and device fields
    work = tempfile.mkdtemp()
    os.makedirs(os.path.join(work, "data"))
    np.asarray(pa, dtype="<f8").tofile(os.path.join(work, "data", "pa.dat"))
    dump = os.path.join(work, "dump")
    os.makedirs(dump)
    stdout_h, dt = run([os.path.join(REF, "harness_" + cfg), "moduli", dump] + args, cwd=work, timeout=7200)
    head, recs, mod = parse_records(os.path.join(dump, "records.txt"))
    meta["records"] = recs
    meta["moduli"] = mod
    meta["harness_seconds"] = dt
    keep = fields_keep or list(FIELDS)
    for f in keep:
        res["f_" + f] = read_field(dump, f, n, n)
    if with_cli:
        shutil.rmtree(work)
        # 2) the reference CLI itself: stdout (17 digits), EffPlast2D.log, data/*.dat
        work = tempfile.mkdtemp()
        os.makedirs(os.path.join(work, "data"))
        np.asarray(pa, dtype="<f8").tofile(os.path.join(work, "data", "pa.dat"))
        stdout_c, dt2 = run([os.path.join(REF, "cli_" + cfg)] + args, cwd=work, timeout=7200)
    else:
        # the harness ran the same ComputeEffModuli in `work`: its stdout (6 digits),
        # EffPlast2D.log and data/*.dat are the reference's outputs of this case
        stdout_c, dt2 = stdout_h, 0.0
    meta["cli_seconds"] = dt2
    meta["cli_stdout"] = stdout_c
    # iterations of the whole solve: the converged checkpoint, or NITER when a time step
    # ends on the iteration cap (EffPlast2D.cu:389-428)
    total, last = 0, 0
    for line in stdout_c.splitlines():
        if line.strip().startswith("Iteration "):
            last = int(line.split()[1].rstrip(":"))
        elif line.startswith("Number of iterations is"):
            total += int(line.split()[-1])
            last = 0
        elif line.startswith("WARNING: Maximum number of iterations"):
            total += MACROS[cfg]["NITER"]
            last = 0
    meta["total_iterations"] = total
    meta["cli_log"] = open(os.path.join(work, "EffPlast2D.log")).read()
    dats = sorted(os.listdir(os.path.join(work, "data")))
    meta["cli_dat_files"] = dats
    for dname in dats:
        if dname == "pa.dat":
            continue
        arr = np.fromfile(os.path.join(work, "data", dname), dtype="<f8")
        if fields_keep is None or dname.startswith(("Pc_", "tauXXc_")):
            res["dat_" + dname] = arr
    shutil.rmtree(work)
    np.savez_compressed(os.path.join(out, name + ".npz"), **res)
    json.dump(meta, open(os.path.join(out, name + ".json"), "w"), indent=1)
    print(name, "harness %.1fs cli %.1fs" % (dt, dt2), flush=True)


def reduce_fixture(path_in, path_out, stride=8):
    """Shrink a full-size fixture for the repository: every `stride`-th row and column of
    each field, its full middle row and column, and its sum and sum of squares."""
    z = np.load(path_in)
    out = {"pa": z["pa"], "stride": np.array(stride)}
    for k in z.files:
        if k == "pa":
            continue
        a = z[k]
        if a.ndim == 1:  # .dat files: square n x n fields
            n = int(round(a.size ** 0.5))
            a = a.reshape(n, n)
        out[k + "__sub"] = a[::stride, ::stride]
        out[k + "__midrow"] = a[a.shape[0] // 2, :]
        out[k + "__midcol"] = a[:, a.shape[1] // 2]
        out[k + "__sums"] = np.array([a.sum(), (a * a).sum()])
    np.savez_compressed(path_out, **out)


def main():
    argv = sys.argv[1:]
    out = os.path.join(ROOT, "golden_out")
    only = None
    with_cfg2 = False
    rest = []
    i = 0
    while i < len(argv):
        if argv[i] == "--only":
            only = set(argv[i + 1].split(","))
            i += 2
            continue
        if argv[i] == "--with-cfg2":
            with_cfg2 = True
        else:
            rest.append(argv[i])
        i += 1
    if rest:
        out = rest[0]
    os.makedirs(out, exist_ok=True)
    for c in KERNEL_CASES:
        if only is None or c[0] in only:
            kernel_case(out, c)
    for c in CHAIN_CASES:
        if only is None or c[0] in only:
            chain_case(out, c)
    if with_cfg2 or (only and "cfg2" in only):
        chain_case(out, CFG2, fields_keep=["P", "tauXX", "tauXY", "Ux", "Uy"], with_cli=False)
        full = os.path.join(out, "cfg2.npz")
        reduce_fixture(full, os.path.join(out, "cfg2_reduced.npz"))


if __name__ == "__main__":
    main()
