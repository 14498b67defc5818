"""Batched launches: several simulations (FitSKIRT-style parameter variants of the oligochromatic
disk on Cartesian grids of different sizes) in one persistent launch give each simulation the
same tallies as running it alone -- up to the summation order of the FP64 atomics -- with and
without CUDA-graph replay, and packet slices spread over several launches add up to one launch."""
import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import models, runtime
from skirt7_b200.scene import DEG, KPC

from helpers import cell_center_density

pytestmark = pytest.mark.gpu


def variants():
    out = []
    for (hR, hz, tau, inc, bf, N) in [(3, 0.1, 0.2, 80, 0.0, 20), (6, 0.3, 1.5, 85, 0.3, 32), (9, 0.5, 4.0, 90, 0.5, 24)]:
        m = models.fit_variant((hR * KPC, hz * KPC, tau, inc * DEG, bf), N, npix=64)
        m.rho = cell_center_density(m)
        out.append(m)
    return out


def read(ctx):
    return [ctx.read_instrument(0)[0].copy()]


def test_alone_equals_mixed():
    ms = variants()
    ctxs = [runtime.Context(m) for m in ms]
    ells = [0, 1, 2]
    npps = [30000, 50000, 20000]
    alone = []
    for c, n, s in zip(ctxs, npps, (11, 22, 33)):
        c.run_phase(A.PHASE_STELLAR, ells, n, 0, n, seed=s)
        c.sync()
        alone.append(read(c))
        c.reset_tallies()
    b = runtime.Batch(max_slots=8, max_items=16, max_ells=64)
    for graph in (False, True):
        for c in ctxs:
            c.reset_tallies()
            c.sync()
        b.run(A.PHASE_STELLAR, [(c, ells, n, 0, n, s) for c, n, s in zip(ctxs, npps, (11, 22, 33))], graph=graph)
        b.sync()
        for c, a in zip(ctxs, alone):
            got = read(c)
            assert np.allclose(got[0], a[0], rtol=1e-12, atol=1e-300 + 1e-14 * a[0].max()), (graph, np.abs(got[0] - a[0]).max())
        cnt = b.counters()
        assert cnt["errors"] == 0
    # slices over several launches (and a replayed graph) add up to the single launch
    for c in ctxs:
        c.reset_tallies()
        c.sync()
    for k in range(4):
        sl = []
        for c, n, s in zip(ctxs, npps, (11, 22, 33)):
            per = -(-n // 4)
            first = k * per
            sl.append((c, ells, n, first, max(0, min(n, first + per) - first), s))
        b.run(A.PHASE_STELLAR, sl, graph=True)
        b.sync()
    for c, a in zip(ctxs, alone):
        got = read(c)
        assert np.allclose(got[0], a[0], rtol=1e-12, atol=1e-14 * a[0].max())
    b.close()
    for c in ctxs:
        c.close()
