"""Kernel-level parity: the fused sm_100a iteration kernel against the CPU oracle.

Both sides start from the same seeded state and run the same number of iterations of
the reference's sequence ComputeStress -> [ComputeJ2 -> ComputePlasticity] ->
ComputeDisp (EffPlast2D.cu:389-399).  The GPU contracts multiply-adds (as the
reference's own CUDA build does); the oracle does not.  Tolerance: every field within
1e-11 of its max-abs after one iteration and 1e-9 after hundreds (bar for fields:
1e-6).  Both kernel forms are checked: the tile form (CTA per tile, halos in shared
memory) and the stream form (warp per strip segment, neighbours by shuffles), the
latter with segments of 16 rows too, so that grids hold several segments, a ragged
last segment and a ragged last strip, and the resident form (the tile form's CTAs kept
resident across iterations, one cooperative launch per run of plain iterations).
"""
import numpy as np
import pytest

import effplast2d_b200 as ep
import oracle

pytestmark = pytest.mark.gpu

FIELDS = ["P", "tauXX", "tauYY", "tauXY", "Ux", "Uy", "Vx", "Vy"]
PLASTIC_FIELDS = ["tauXYav", "J2", "J2XY"]
FORMS = [(ep.KERNEL_TILE, 16), (ep.KERNEL_STREAM, 16), (ep.KERNEL_STREAM, 64), (ep.KERNEL_RESIDENT, 16)]
FORM_IDS = ["tile16", "stream16", "stream64", "resident16"]


def _pa(n_x, n_y, n_pores=1, porosity=0.01, yield_stress=1.0, g0=0.5):
    return oracle.make_pa(20.0, 20.0, n_x, n_y, g0=g0, yield_stress=yield_stress, porosity=porosity,
                          n_pores=n_pores)


def _random_state(nx, ny, seed, strain=6e-5, noise=2e-6, vnoise=1e-7):
    """affine strain field plus seeded noise; V random; boundary faces of V zero"""
    rng = np.random.default_rng(seed)
    dx = 20.0 / (nx - 1)
    xi = -0.5 * dx * nx + dx * np.arange(nx + 1)
    yj = -0.5 * dx * (ny - 1) + dx * np.arange(ny)
    ux = strain * (xi[None, :] * -1.0 + 0.3 * yj[:, None]) + noise * rng.standard_normal((ny, nx + 1))
    xi2 = -0.5 * dx * (nx - 1) + dx * np.arange(nx)
    yj2 = -0.5 * dx * ny + dx * np.arange(ny + 1)
    uy = strain * (yj2[:, None] * -0.8 + 0.3 * xi2[None, :]) + noise * rng.standard_normal((ny + 1, nx))
    vx = vnoise * rng.standard_normal((ny, nx + 1))
    vy = vnoise * rng.standard_normal((ny + 1, nx))
    vx[:, 0] = vx[:, -1] = 0.0
    vx[0, :] = vx[-1, :] = 0.0
    vy[0, :] = vy[-1, :] = 0.0
    vy[:, 0] = vy[:, -1] = 0.0
    return {"Ux": ux, "Uy": uy, "Vx": vx, "Vy": vy}


def _pair(nx, ny, pa, nl, form=(ep.KERNEL_AUTO, 0)):
    return ep.Solver(nx, ny, pa, nl=nl, kernel=form[0], rows=form[1]), oracle.Oracle(nx, ny, pa, nl=nl)


@pytest.mark.parametrize("nx,ny,n_pores", [(64, 64, 1), (96, 96, 3), (64, 96, 2), (40, 56, 1), (129, 71, 2)])
def test_materials_and_masks(nx, ny, n_pores):
    pa = _pa(nx, ny, n_pores=n_pores, porosity=0.03)
    g, o = _pair(nx, ny, pa, 1)
    for f in ("K", "G"):
        assert np.array_equal(g.get(f), o.get(f)), f
    st = _random_state(nx, ny, 1)
    for k, v in st.items():
        g.set(k, v)
        o.set(k, v)
    g.iterate(1)
    node, corner = o.masks()
    assert node.sum() > 0 and corner.sum() > 0
    # generic random strains: P == 0 and tauXY == 0 exactly where the kernel masks are
    assert np.array_equal(g.get("P") == 0.0, node.astype(bool))
    assert np.array_equal(g.get("tauXY") == 0.0, corner.astype(bool))


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
@pytest.mark.parametrize("nl", [1, 2, 3])
@pytest.mark.parametrize("nx,ny,n_pores", [(64, 64, 1), (96, 64, 3), (40, 56, 2), (33, 65, 1)])
def test_one_iteration_random_state(nl, nx, ny, n_pores, form, rel):
    # Y small enough that a good part of the grid yields
    pa = _pa(nx, ny, n_pores=n_pores, porosity=0.02, yield_stress=2e-5)
    g, o = _pair(nx, ny, pa, nl, form)
    st = _random_state(nx, ny, 7 + nl)
    for k, v in st.items():
        g.set(k, v)
        o.set(k, v)
    g.iterate(1)
    o.iterate(1)
    fields = FIELDS + (PLASTIC_FIELDS if nl > 1 else [])
    for f in fields:
        assert rel(g.get(f), o.get(f)) < 1e-11, f
    if nl > 1:
        j2 = o.get("J2XY")
        assert (j2 > pa[8]).mean() > 0.05  # the return map is exercised


@pytest.mark.parametrize("form", FORMS, ids=FORM_IDS)
@pytest.mark.parametrize("nl", [1, 3])
def test_many_iterations(nl, form, rel):
    nx = ny = 96
    pa = _pa(nx, ny, n_pores=3, porosity=0.02, yield_stress=1e-5)
    g, o = _pair(nx, ny, pa, nl, form)
    st = _random_state(nx, ny, 3, noise=0.0, vnoise=0.0)
    for k, v in st.items():
        g.set(k, v)
        o.set(k, v)
    for n in (1, 63, 64, 200):  # direct launches and captured graphs, both parities
        g.iterate(n)
        o.iterate(n)
    for f in FIELDS + (PLASTIC_FIELDS if nl > 1 else []):
        assert rel(g.get(f), o.get(f)) < 1e-9, f


def test_zero_state_stays_zero():
    nx = ny = 64
    g = ep.Solver(nx, ny, _pa(nx, ny), nl=3)
    g.iterate(10)
    for f in FIELDS:
        assert not np.any(g.get(f)), f


def test_homogeneous_affine_is_equilibrium():
    # no pores (rad = 0): an affine field is in equilibrium, V stays 0 (up to rounding)
    nx = ny = 64
    pa = _pa(nx, ny)
    pa[9] = 0.0
    g = ep.Solver(nx, ny, pa, nl=1)
    st = _random_state(nx, ny, 0, noise=0.0, vnoise=0.0)
    g.set("Ux", st["Ux"])
    g.set("Uy", st["Uy"])
    g.iterate(50)
    assert np.max(np.abs(g.get("Vx"))) < 1e-16  # rounding of the affine differences only
    P = g.get("P")
    assert np.allclose(P, P[1, 1], rtol=1e-12, atol=0)


@pytest.mark.parametrize("grid", [(301, 203), (242, 130)], ids=["301x203", "242x130"])
@pytest.mark.parametrize("rows", [4, 8, 12, 16, 64, 256])
def test_stream_form_matches_tile_form(rows, grid):
    # Both forms evaluate the same explicitly rounded per-cell formulas, so they agree
    # bit for bit.  The grids are wider and taller than several strips and segments,
    # ragged in both, so interior and edge segments both run; the last strip holds 21
    # (301) and 18 (242) columns of the grid.
    nx, ny = grid
    pa = _pa(nx, ny, n_pores=4, porosity=0.03, yield_stress=1e-5)
    st = _random_state(nx, ny, 11)
    out = []
    for kernel, r in ((ep.KERNEL_TILE, 16), (ep.KERNEL_STREAM, rows)):
        g = ep.Solver(nx, ny, pa, nl=3, kernel=kernel, rows=r)
        for k, v in st.items():
            g.set(k, v)
        g.iterate(1)
        g.iterate(300)
        out.append({f: g.get(f) for f in FIELDS + PLASTIC_FIELDS})
    for f in FIELDS + PLASTIC_FIELDS:
        assert np.array_equal(out[1][f], out[0][f]), (f, float(np.max(np.abs(out[1][f] - out[0][f]))))


def test_full_size_2048_against_oracle_and_tile_form(rel):
    # The 2048^2 grid of the 4x4-pore, porosity-0.02, Y = 1e-5 workload at full size: the
    # library's default shape there (stream form, 64-row segments: one wave of 2368 warps,
    # interior and edge segments), 20 iterations from a seeded state that yields widely,
    # bit for bit against the tile form and to 1e-9 against the oracle.
    n = 2048
    pa = _pa(n, n, n_pores=4, porosity=0.02, yield_stress=1e-5)
    st = _random_state(n, n, 5)
    g = ep.Solver(n, n, pa, nl=3)
    assert g.kernel_shape() == (ep.KERNEL_STREAM, 64)
    t = ep.Solver(n, n, pa, nl=3, kernel=ep.KERNEL_TILE, rows=16)
    o = oracle.Oracle(n, n, pa, nl=3)
    for k, v in st.items():
        g.set(k, v)
        t.set(k, v)
        o.set(k, v)
    for it in (1, 19):
        g.iterate(it)
        t.iterate(it)
        o.iterate(it)
    assert (o.get("J2XY") > pa[8]).mean() > 0.05  # the return map is exercised
    for f in FIELDS + PLASTIC_FIELDS:
        a = g.get(f)
        assert np.array_equal(a, t.get(f)), f
        assert rel(a, o.get(f)) < 1e-9, f
