"""The multi-GPU split on one device: distributed.run_phase_sharded runs each rank's packet range
(MonteCarloSimulation.cpp:98-104) in a context of its own, as separate ranks would; the sum of the
ranks' frames, SEDs and absorbed luminosities equals the single-context run of all packets (every
packet draws from a stream keyed by its id), up to the order of the FP64 atomic additions."""
import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import distributed, models, runtime

from helpers import cell_center_density

pytestmark = pytest.mark.gpu


def _read(ctx):
    cube, _ = ctx.read_instrument(0)
    _, sed = ctx.read_instrument(1)
    return cube, sed, ctx.read_absorption()[0]


@pytest.mark.parametrize("world", [2, 3, 4])
def test_sharded_phase_sums_to_the_full_run(world):
    m = models.oligo_disk(N=(40, 40, 20), npix=60)
    m.rho = cell_center_density(m)
    npp, seed = 300001, 17                      # not a multiple of the rank count
    full = runtime.Context(m)
    distributed.run_phase_sharded(full, A.PHASE_STELLAR, [0], npp, seed, 0, 1)
    ref = _read(full)
    full.close()
    parts = []
    covered = 0
    for rank in range(world):
        ctx = runtime.Context(m)
        first, count = distributed.run_phase_sharded(ctx, A.PHASE_STELLAR, [0], npp, seed, rank, world)
        covered += count
        parts.append(_read(ctx))
        assert ctx.counters()["packets"] == count
        ctx.close()
    assert covered == npp
    for k in range(3):
        got = sum(p[k] for p in parts)
        assert ref[k].sum() > 0
        assert np.allclose(got, ref[k], rtol=1e-9, atol=1e-12 * np.abs(ref[k]).max()), k
