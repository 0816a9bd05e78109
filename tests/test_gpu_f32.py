"""The FP32 stencil bulk (EP2D_F32_BULK).

Each time step starts in FP32 -- arithmetic, velocities and the displacement
perturbation about the affine preload field -- and returns to FP64 displacements and
arithmetic once its checkpoint residual stops falling fast; only FP64 checkpoints decide
convergence.  The checks here: the FP32 phase runs and tracks the FP64 iteration to FP32
accuracy while it does; the hand-back leaves a state the FP64 path converges from; and the
moduli of whole ComputeEffModuli chains stay within the stated tolerance of the plain
FP64 path (EffPlast2D.cu:179-229), with the error of each modulus printed.
"""
import math

import numpy as np
import pytest

import effplast2d_b200 as ep

pytestmark = pytest.mark.gpu


def solver(n, prec, niter, ce, nl=2, n_pores=3, Y=1e-5, phi=0.02, kernel=ep.KERNEL_AUTO):
    pa = ep.make_pa(20.0, 20.0, n, n, g0=0.5, yield_stress=Y, porosity=phi, n_pores=n_pores)
    return ep.Solver(n, n, pa, nl=nl, niter=niter, eiter=1e-9, check_every=ce, precision=prec, kernel=kernel)


def test_f32_phase_tracks_fp64_iteration():
    # one time step of 3 x 1000 iterations: the first two intervals in FP32 (the residual
    # falls fast after a preload), the last one in FP64 by construction
    n, ce = 128, 1000
    out = {}
    for name, prec in (("fp64", ep.FP64), ("f32", ep.F32_BULK)):
        s = solver(n, prec, 3 * ce, ce)
        s.solve_step(0, -6e-5, [1.0, 0.8, 0.3], 1)
        out[name] = {f: s.get(f) for f in ("Ux", "Uy", "Vx", "Vy", "P", "tauXY")}
        out[name + "_f32"] = s.stats()["f32_iterations"]
        s.close()
    assert out["fp64_f32"] == 0
    assert out["f32_f32"] >= ce  # the FP32 form ran
    for f in ("Ux", "Uy", "P", "tauXY"):
        a, b = out["f32"][f], out["fp64"][f]
        err = float(np.max(np.abs(a - b)) / np.max(np.abs(b)))
        print("%s: max rel diff FP32 bulk vs FP64 %.2e" % (f, err))
        assert err < 1e-4, (f, err)
    for f in ("Vx", "Vy"):  # velocities: relative to their own scale, which decays
        a, b = out["f32"][f], out["fp64"][f]
        assert float(np.max(np.abs(a - b))) <= 0.05 * float(np.max(np.abs(b))), f


@pytest.mark.parametrize("n,nl,lt", [(96, 2, (1.0, 1.0, 0.0)), (128, 3, (1.0, 0.7, 0.3))])
def test_f32_bulk_chain_moduli(n, nl, lt):
    ce = 1000
    res = {}
    for name, prec in (("fp64", ep.FP64), ("f32", ep.F32_BULK)):
        s = solver(n, prec, 400_000, ce, nl=nl)
        r = s.compute_eff_moduli(-6e-5, list(lt), 1)
        res[name] = (r, s.stats()["f32_iterations"])
        s.close()
    r64, _ = res["fp64"]
    r32, it32 = res["f32"]
    assert r64["all_converged"] and r32["all_converged"]
    assert it32 > 0
    keys = ["kphi", "kd"] + (["g"] if nl == 3 else [])
    for k in keys:
        a, b = r32["num"][k], r64["num"][k]
        if not math.isfinite(b):
            continue
        err = abs(a - b) / abs(b)
        print("n=%d nl=%d %s: FP32 bulk %.10g FP64 %.10g rel err %.2e (FP32 iterations %d of %d)"
              % (n, nl, k, a, b, err, it32, r32["total_iterations"]))
        assert err < 1e-3, (k, a, b)


def test_f32_bulk_rejected_by_batches():
    from effplast2d_b200 import batch as B

    pa = ep.make_pa(20.0, 20.0, 64, 64, g0=0.5, yield_stress=1e-5, porosity=0.02, n_pores=2)
    with pytest.raises(ep.EP2DError) as e:
        B.batch_solve([B.spec(64, pa, 2, 1, -6e-5, (1.0, 1.0, 0.0))], niter=2000, check_every=1000,
                      precision=ep.F32_BULK)
    assert e.value.status == ep.ERR_ARG


def test_f32_round_trip_keeps_displacements():
    # zero FP32 iterations: U -> u' = U - Ua (float) -> U = Ua + u' changes U only by the
    # float rounding of the perturbation, never by the affine part
    n = 96
    s = solver(n, ep.F32_BULK, 2000, 1000)
    s.solve_step(0, -6e-5, [1.0, 0.8, 0.3], 1)
    before = {f: s.get(f) for f in ("Ux", "Uy")}
    s.iterate_f32(0)
    for f in ("Ux", "Uy"):
        after = s.get(f)
        # the perturbation is at most |U| here; its float rounding is 2^-24 of it
        assert np.max(np.abs(after - before[f])) <= 2.0 ** -23 * np.max(np.abs(before[f])), f
    f0 = s.stats()["f32_iterations"]  # the solve step's own FP32 phase
    s.iterate_f32(500)
    assert s.stats()["f32_iterations"] == f0 + 500
    s.close()
    with pytest.raises(ep.EP2DError) as e:  # FP64 handles have no FP32 form
        s64 = solver(n, ep.FP64, 2000, 1000)
        try:
            s64.iterate_f32(10)
        finally:
            s64.close()
    assert e.value.status == ep.ERR_STATE
