"""The resident form of the iteration kernel (EP2D_KERNEL_RESIDENT).

The reference runs one launch sequence per pseudo-time iteration with a device-wide
synchronisation after each kernel (EffPlast2D.cu:386-428).  The resident form runs all
the plain iterations between two checkpoints in one cooperative launch: the tile form's
CTAs stay resident, own fixed tiles, and meet at a grid-wide barrier after every
iteration.  Per tile it runs the tile form's code, so every field must equal the tile
form's bit for bit (and, through it, the oracle's: test_gpu_kernels.py runs the resident
form against the oracle too).  The barrier's failure path is checked without a fault:
CTAs that never arrive make the others' bounded waits run out, the error flag is set,
and the context stays usable.
"""
import numpy as np
import pytest

import effplast2d_b200 as ep
from test_gpu_kernels import FIELDS, PLASTIC_FIELDS, _pa, _random_state

pytestmark = pytest.mark.gpu


def _run(nx, ny, pa, nl, kernel, rows, st, counts, precision=ep.FP64):
    g = ep.Solver(nx, ny, pa, nl=nl, kernel=kernel, rows=rows, precision=precision)
    assert g.kernel_shape() == (kernel, rows)
    for k, v in st.items():
        g.set(k, v)
    for n in counts:
        g.iterate(n)
    out = {f: g.get(f) for f in FIELDS + (PLASTIC_FIELDS if nl > 1 else [])}
    stats = g.stats()
    g.close()
    return out, stats


@pytest.mark.parametrize("rows", [8, 16, 32])
@pytest.mark.parametrize("grid,nl", [((301, 203), 3), ((256, 256), 3), ((96, 64), 1), ((40, 56), 2)],
                         ids=["301x203-nl3", "256-nl3", "96x64-nl1", "40x56-nl2"])
def test_resident_matches_tile_form(grid, nl, rows):
    # 1 (a single recording tile launch), then resident runs of odd and even length
    nx, ny = grid
    pa = _pa(nx, ny, n_pores=3, porosity=0.03, yield_stress=1e-5)
    st = _random_state(nx, ny, 17)
    counts = (1, 300, 64, 2, 3)
    a, sa = _run(nx, ny, pa, nl, ep.KERNEL_TILE, rows, st, counts)
    b, sb = _run(nx, ny, pa, nl, ep.KERNEL_RESIDENT, rows, st, counts)
    for f in a:
        assert np.array_equal(b[f], a[f]), (f, float(np.max(np.abs(b[f] - a[f]))))
    assert sb["cell_updates"] == sa["cell_updates"]
    # five recording launches, one resident launch for each run of 299, 63 and 2 plain
    # iterations, one tile launch for the run of 1
    assert sb["launches"] == 9


def test_resident_mixed_precision_matches_tile_form():
    nx, ny = 200, 150
    pa = _pa(nx, ny, n_pores=2, porosity=0.02, yield_stress=1e-5)
    st = _random_state(nx, ny, 23)
    a, _ = _run(nx, ny, pa, 3, ep.KERNEL_TILE, 16, st, (500,), precision=ep.MIXED)
    b, _ = _run(nx, ny, pa, 3, ep.KERNEL_RESIDENT, 16, st, (500,), precision=ep.MIXED)
    for f in a:
        assert np.array_equal(b[f], a[f]), f


def test_resident_more_tiles_than_resident_ctas():
    # 1024^2 in 32 x 8 tiles: 4096 tiles, more than fit on the GPU at once, so every CTA
    # walks several tiles per iteration
    n = 1024
    pa = _pa(n, n, n_pores=3, porosity=0.01, yield_stress=1e-5)
    st = _random_state(n, n, 29)
    a, _ = _run(n, n, pa, 3, ep.KERNEL_TILE, 8, st, (1, 40))
    b, _ = _run(n, n, pa, 3, ep.KERNEL_RESIDENT, 8, st, (1, 40))
    for f in a:
        assert np.array_equal(b[f], a[f]), f


def test_resident_chain_equals_tile_chain():
    # a whole ComputeEffModuli chain (EffPlast2D.cu:179-229): checkpoints, time steps and
    # moduli identical, with far fewer iteration launches
    n = 128
    pa = _pa(n, n, n_pores=2, porosity=0.02, yield_stress=1e-5)
    res = {}
    for kernel in (ep.KERNEL_TILE, ep.KERNEL_RESIDENT):
        s = ep.Solver(n, n, pa, nl=3, niter=200_000, eiter=1e-9, check_every=1000, kernel=kernel, rows=16)
        r = s.compute_eff_moduli(-6e-5, [1.0, 0.7, 0.3], 1)
        res[kernel] = (r, s.stats())
        s.close()
    (rt, st), (rr, sr) = res[ep.KERNEL_TILE], res[ep.KERNEL_RESIDENT]
    assert rr["all_converged"] == rt["all_converged"]
    assert rr["total_iterations"] == rt["total_iterations"]
    for k in ("kphi", "kd", "g"):
        assert rr["num"][k] == rt["num"][k] or (np.isnan(rr["num"][k]) and np.isnan(rt["num"][k])), k
    assert sr["launches"] * 100 < st["launches"]


def test_grid_barrier_completes():
    passed, flag = ep.check_grid_barrier(blocks=296, missing=0, rounds=200, timeout_ns=2_000_000_000)
    assert (passed, flag) == (296, 0)


def test_grid_barrier_wait_runs_out_and_context_survives():
    # one CTA never arrives: the others give up after 1 ms each and set the flag
    passed, flag = ep.check_grid_barrier(blocks=64, missing=1, rounds=3, timeout_ns=1_000_000)
    assert (passed, flag) == (0, 1)
    # the context is still usable: a resident solve right after still equals the tile form
    nx = ny = 96
    pa = _pa(nx, ny, n_pores=1, porosity=0.02, yield_stress=1e-5)
    st = _random_state(nx, ny, 31)
    a, _ = _run(nx, ny, pa, 3, ep.KERNEL_TILE, 16, st, (100,))
    b, _ = _run(nx, ny, pa, 3, ep.KERNEL_RESIDENT, 16, st, (100,))
    for f in a:
        assert np.array_equal(b[f], a[f]), f


def test_barrier_check_arguments():
    for kw in (dict(blocks=0), dict(blocks=4, missing=5), dict(blocks=4, rounds=-1),
               dict(blocks=4, rounds=2_000_000), dict(blocks=4, timeout_ns=20_000_000_000)):
        with pytest.raises(ep.EP2DError) as e:
            ep.check_grid_barrier(**kw)
        assert e.value.status == ep.ERR_ARG
