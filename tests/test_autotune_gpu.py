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
    for pool, blocks in ((1 << 12, 148), (1 << 16, 296), (1 << 20, 0)):
        ctx.reset_tallies()
        ctx.run_phase(A.PHASE_STELLAR, [0], 60000, 0, 60000, seed=5, pool=pool, blocks=blocks)
        ctx.sync()
        frames.append(ctx.read_instrument(0)[0].copy())
        ev, tr, waves = ctx.phase_times()
        assert waves > 1 and tr > 0 and ev > 0
    for f in frames[1:]:
        assert np.allclose(f, frames[0], rtol=1e-11, atol=1e-13 * frames[0].max())
    res = autotune.tune(ctx, A.PHASE_STELLAR, [0], 60000, sample=20000, pools=[1 << 12, 1 << 14], blocks=[148, 296])
    assert res["pool"] in (1 << 12, 1 << 14) and res["blocks"] in (148, 296) and len(res["trials"]) == 4
    assert autotune.tune(ctx, A.PHASE_STELLAR, [0], 60000) is res          # cached per workload class
    ctx.close()
