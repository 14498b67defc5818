"""The launch shape is a pure performance choice: packets in flight and traversal blocks change
how packets are grouped into waves, not their numbers (each packet's random stream is keyed by
its index), so the frames agree up to the summation order of the FP64 atomics.  The autotuner
picks among such shapes by timing trial phases."""
import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import autotune, models, runtime

from helpers import cell_center_density

pytestmark = pytest.mark.gpu


def test_pool_and_blocks_do_not_change_results():
    m = models.oligo_disk(N=(40, 40, 20))
    m.rho = cell_center_density(m)
    ctx = runtime.Context(m)
    frames = []
    for pool, blocks, refill in ((1 << 12, 148, 4), (1 << 16, 296, 16), (1 << 20, 0, 0), (1 << 18, 0, 32)):
        ctx.reset_tallies()
        ctx.run_phase(A.PHASE_STELLAR, [0], 60000, 0, 60000, seed=5, pool=pool, blocks=blocks, refill=refill)
        ctx.sync()
        frames.append(ctx.read_instrument(0)[0].copy())
        ev, tr, waves = ctx.phase_times()
        assert waves > 1 and tr > 0 and ev > 0
    for f in frames[1:]:
        assert np.allclose(f, frames[0], rtol=1e-11, atol=1e-13 * frames[0].max())
    # reading into caller-owned host arrays gives the same tallies
    cube, sed = ctx.read_instrument(0)
    c2, s2 = ctx.read_instrument(0, out=(np.empty(cube.size), np.empty(sed.size)))
    assert np.array_equal(c2, cube) and np.array_equal(s2, sed)
    res = autotune.tune(ctx, A.PHASE_STELLAR, [0], 60000, sample=20000, pools=[1 << 12, 1 << 14], refills=(4, 8),
                        blocks=[148, 296])
    assert res["pool"] in (1 << 12, 1 << 14) and res["blocks"] in (148, 296) and res["refill"] in (4, 8)
    assert len(res["trials"]) == 4                      # the start, then one coordinate at a time
    assert res["ms"] == min(t["ms"] for t in res["trials"])
    assert autotune.tune(ctx, A.PHASE_STELLAR, [0], 60000) is res          # cached per workload class
    ctx.close()


@pytest.mark.parametrize("grid", ["cartesian", "octree"])
def test_tail_pass_does_not_change_results(grid, monkeypatch):
    """The tail pass (one thread per remaining packet runs the rest of its life at once) uses the
    same random streams, samplers and tallies as the waves: a phase ending in waves only, in the
    tail pass from the default threshold, or handing nearly all its work to the tail pass (which
    then launches the remaining packets itself) gives the same frames and absorbed luminosities up
    to the summation order of the FP64 atomics, and the same counts."""
    m = models.oligo_disk(N=(40, 40, 20))
    if grid == "octree":
        from skirt7_b200.scene import KPC
        ext = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)
        m.dustGrid = runtime.build_tree(m, A.GRID_OCTREE, ext, minLevel=2, maxLevel=6, maxMassFraction=1e-4)
        m.rho = None
    else:
        m.rho = cell_center_density(m)
    ctx = runtime.Context(m)
    res = []
    for div in ("0", "16", "1"):
        monkeypatch.setenv("SKG_TAIL_DIV", div)
        ctx.reset_tallies()
        ctx.run_phase(A.PHASE_STELLAR, [0], 200000, 0, 200000, seed=7, pool=1 << 16)
        ctx.sync()
        c = ctx.counters()
        res.append((ctx.read_instrument(0)[0].copy(), ctx.read_absorption()[0].copy(), c))
    f0, l0, c0 = res[0]
    assert c0["errors"] == 0 and c0["packets"] == 200000
    for f, l, c in res[1:]:
        assert np.allclose(f, f0, rtol=1e-10, atol=1e-12 * f0.max())
        assert np.allclose(l, l0, rtol=1e-10, atol=1e-12 * l0.max())
        for k in ("packets", "scatterings", "peeloffs", "traversals", "errors"):
            assert c[k] == c0[k], (k, c[k], c0[k])
    ctx.close()
