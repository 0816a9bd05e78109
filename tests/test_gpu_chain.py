"""Load-step chain parity (ComputeEffParams / ComputeEffModuli) against the CPU oracle.

The GPU path runs preload, averaging, boundary sums, hole area and moduli on the
device + host exactly as the reference orders them; the oracle restates the reference
sequentially.  Sums are reduced in a different order on the GPU (deterministic tree),
so scalars agree to rounding: tolerance 1e-9 relative on every record value and on the
moduli (the parity bar is 1e-5 on K_d, K_phi, G).
"""
import math

import numpy as np
import pytest

import effplast2d_b200 as ep
import oracle

pytestmark = pytest.mark.gpu

SCALARS = ["delta_p", "delta_p_per", "tau_infty", "hole_area_pi", "internal_hole_area_pi", "phi0", "phi",
           "phi_per", "dphi", "dphi_per", "kphi_exact_elast", "kd_exact_elast", "kphi_exact_plast",
           "kd_exact_plast", "kphi_exact_plast_per", "kd_exact_plast_per", "g_exact_elast", "g_exact_plast",
           "g_exact_plast_per", "error"]
VECTORS = ["macro_strain", "sigma", "sigma_per", "eps_per"]


STRESS_LIKE = {"delta_p", "delta_p_per", "tau_infty", "sigma", "sigma_per"}


def close(a, b, tol, atol=0.0):
    if a == b:
        return True
    if isinstance(a, float) and (math.isnan(a) or math.isnan(b)):
        return math.isnan(a) and math.isnan(b)
    return abs(a - b) <= tol * abs(b) + atol


def compare_records(rg, ro, tol):
    """Values that are rounding noise (tau_infty under a hydrostatic load, ~1e-21; the
    error of a converged state, ~1e-16) get absolute floors: 1e-9 of the record's stress
    scale for stress-like values, 1e-13 for the convergence error."""
    for k in ("iterations", "converged", "n_checks", "step", "time_step"):
        assert rg[k] == ro[k], k
    scale = max([abs(v) for v in ro["sigma"]] + [abs(ro["delta_p"])]) or 1.0
    strain = max(abs(v) for v in ro["macro_strain"]) or 1.0
    for k in SCALARS:
        atol = 1e-9 * scale if k in STRESS_LIKE else (1e-13 if k == "error" else 0.0)
        assert close(rg[k], ro[k], tol, atol), (k, rg[k], ro[k])
    for k in VECTORS:
        atol = 1e-9 * scale if k in STRESS_LIKE else 1e-9 * strain
        for a, b in zip(rg[k], ro[k]):
            assert close(a, b, tol, atol), (k, rg[k], ro[k])


CASES = [
    # nx, nl, n_pores, porosity, Y, load, load_type, n_time_steps, niter, check_every
    (48, 1, 1, 0.005, 1.0, -4e-5, [1.0, 1.0, 0.0], 1, 20000, 1000),
    (64, 2, 2, 0.02, 1e-5, -6e-5, [1.0, 1.0, 0.0], 2, 6000, 1000),
    (96, 3, 3, 0.02, 1e-5, -6e-5, [1.0, 0.8, 0.3], 2, 4000, 1000),
    (64, 3, 1, 0.01, 1e-5, -5e-5, [1.0, 1.0, 0.5], 1, 3000, 500),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "n%d_nl%d_N%d" % (c[0], c[1], c[2]))
def test_eff_moduli_chain(case):
    nx, nl, n_pores, phi, Y, load, lt, nts, niter, ce = case
    pa = oracle.make_pa(20.0, 20.0, nx, nx, g0=0.5, yield_stress=Y, porosity=phi, n_pores=n_pores)
    g = ep.Solver(nx, nx, pa, nl=nl, niter=niter, eiter=1e-9, check_every=ce)
    o = oracle.Oracle(nx, nx, pa, nl=nl, niter=niter, eiter=1e-9, check_every=ce)
    rg = g.compute_eff_moduli(load, lt, nts)
    ro = o.compute_eff_moduli(load, lt, nts)
    for s in range(nl):
        for t in range(nts if s == 0 else 1):
            compare_records(g.record(s, t), o.record(s, t), 1e-9)
            eg, eo = g.check_errors(s, t), o.check_errors(s, t)
            assert len(eg) == len(eo)
            assert np.allclose(eg, eo, rtol=1e-8, atol=1e-13)
    for kind in ("num", "num_per", "an", "an_per"):
        keys = ["kphi", "kd"] + (["g"] if nl == 3 else [])
        for k in keys:
            a, b = rg[kind][k], ro[kind][k]
            if not math.isfinite(b):
                # a load type with equal xx and yy parts leaves G's denominator exactly
                # zero; the quotient is +-inf or nan by the sign of rounding noise
                assert not math.isfinite(a), (kind, k, a, b)
                continue
            assert close(a, b, 1e-8), (kind, k, a, b)
    assert rg["total_iterations"] == ro["total_iterations"]
    # final fields
    for f in ("P", "tauXX", "tauYY", "tauXY", "Ux", "Uy"):
        a, b = g.get(f), o.get(f)
        assert np.max(np.abs(a - b)) <= 1e-9 * np.max(np.abs(b)), f


def test_niter_not_multiple_of_check_every():
    # the loop may end between checkpoints: the last iteration still records stresses
    nx = 64
    pa = oracle.make_pa(20.0, 20.0, nx, nx, g0=0.5, yield_stress=1e-5, porosity=0.02, n_pores=2)
    g = ep.Solver(nx, nx, pa, nl=2, niter=1234, eiter=1e-30, check_every=500)
    o = oracle.Oracle(nx, nx, pa, nl=2, niter=1234, eiter=1e-30, check_every=500)
    rg = g.solve_step(0, -6e-5, [1, 1, 0], 1)[0]
    ro = o.solve_step(0, -6e-5, [1, 1, 0], 1)[0]
    assert rg["iterations"] == ro["iterations"] == 1234
    assert rg["converged"] == ro["converged"] == 0
    assert rg["n_checks"] == ro["n_checks"] == 2
    compare_records(rg, ro, 1e-9)


def test_static_fields():
    nx = 64
    pa = oracle.make_pa(20.0, 20.0, nx, nx, g0=0.5, yield_stress=1e-5, porosity=0.01, n_pores=1)
    g = ep.Solver(nx, nx, pa, nl=2, niter=3000, eiter=1e-9, check_every=1000)
    o = oracle.Oracle(nx, nx, pa, nl=2, niter=3000, eiter=1e-9, check_every=1000)
    g.compute_eff_moduli(-6e-5, [1, 1, 0], 1)
    o.compute_eff_moduli(-6e-5, [1, 1, 0], 1)
    sg = g.static_fields()
    r0 = o.record(0, 0)
    so = o.static_fields(r0["delta_p"], r0["tau_infty"])
    for k in ("UnuAbs", "J1nu", "J2nu"):
        assert np.max(np.abs(sg[k] - so[k])) <= 1e-9 * np.max(np.abs(so[k])), k


@pytest.mark.parametrize("lt", [[1.0, 1.0, 0.0], [1.0, 0.7, 0.2]], ids=["hydrostatic", "shear"])
def test_analytic_fields(lt):
    # SaveAnStatic2D's analytic part (one pore): device complex FP64 vs the oracle's C99
    # complex restatement.  Different complex-function implementations: agree to 1e-10.
    nx = 64
    pa = oracle.make_pa(20.0, 20.0, nx, nx, g0=0.5, yield_stress=1e-5, porosity=0.01, n_pores=1)
    g = ep.Solver(nx, nx, pa, nl=2, niter=3000, eiter=1e-9, check_every=1000)
    o = oracle.Oracle(nx, nx, pa, nl=2, niter=3000, eiter=1e-9, check_every=1000)
    g.compute_eff_moduli(-6e-5, lt, 1)
    o.compute_eff_moduli(-6e-5, lt, 1)
    r0 = o.record(0, 0)
    ga = g.analytic_fields(r0["delta_p"], r0["tau_infty"])
    oa = o.static_fields(r0["delta_p"], r0["tau_infty"])
    for k in ("UanAbs", "J1an", "J2an"):
        assert np.max(np.abs(ga[k] - oa[k])) <= 1e-10 * np.max(np.abs(oa[k])), k
    for k in ("errorUabs", "errorJ1", "errorJ2"):
        assert np.max(np.abs(ga[k] - oa[k])) <= 1e-7, k
    assert np.allclose(ga["stats"], oa["stats"], rtol=1e-7, atol=0)


def test_increment_before_preload_is_rejected():
    nx = 32
    pa = oracle.make_pa(20.0, 20.0, nx, nx)
    g = ep.Solver(nx, nx, pa, nl=2)
    with pytest.raises(ep.EP2DError) as ei:
        g.solve_step(1, -1e-7, [1, 1, 0], 1)
    assert ei.value.status == 4
