"""Checkpointed re-walks.  After a packet's path has been walked (optical depth, absorption), the
interaction point is found by walking the path again up to the sampled optical depth
(DustGridPath::pathlength, DustGridPath.cpp:162-173).  The FP32 walks store a checkpoint of their
state every few cell steps, and the re-walk starts at the last one below the interaction optical
depth: the cells and segments it walks are those a re-walk from the start would walk, and only the
path length carried to the checkpoint is rounded differently (float against a sum of doubles).
So frames and absorbed luminosities agree with full re-walks (SKG_CKPT=0) to FP32 rounding, with
fewer cell steps.  (The Voronoi walk resumes by default; the Cartesian and tree walks when built
with SKG_CKPT_CART=1 / SKG_CKPT_TREE=1.)"""
import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import models, runtime
from skirt7_b200.scene import KPC

from helpers import cell_center_density

pytestmark = pytest.mark.gpu


def _model(grid):
    m = models.oligo_disk(N=(40, 40, 20))
    ext = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)
    if grid == "octree":
        m.dustGrid = runtime.build_tree(m, A.GRID_OCTREE, ext, minLevel=2, maxLevel=7, maxMassFraction=2e-5)
        m.rho = None
    elif grid == "voronoi":
        from test_voronoi_gpu import as_grid, build_mesh, voronoi_sites
        m.dustGrid = as_grid(build_mesh(voronoi_sites(30000, seed=3)))
        m.rho = None
    else:
        m.rho = cell_center_density(m)
    return m


@pytest.mark.parametrize("grid", ["voronoi"])
def test_checkpointed_rewalk_matches_full_rewalk(grid, monkeypatch):
    ctx = runtime.Context(_model(grid))
    res = []
    for ck in ("0", "1"):
        monkeypatch.setenv("SKG_CKPT", ck)
        ctx.reset_tallies()
        ctx.run_phase(A.PHASE_STELLAR, [0], 200000, 0, 200000, seed=11, precision=A.PREC_FP32, pool=1 << 16)
        ctx.sync()
        res.append((ctx.read_instrument(0)[0].copy(), ctx.read_absorption()[0].copy(), ctx.counters()))
    (f0, l0, c0), (f1, l1, c1) = res
    assert c0["errors"] == 0 and c1["errors"] == 0 and c0["packets"] == c1["packets"] == 200000
    # the same random numbers drive both: event counts agree but for packets whose termination test
    # sits within rounding of its threshold
    for k in ("scatterings", "peeloffs", "traversals"):
        assert abs(c1[k] - c0[k]) <= 1e-4 * c0[k] + 2, (k, c1[k], c0[k])
    assert c1["steps"] < c0["steps"]
    # totals to FP32 rounding; pixels and cells up to the rare packet that lands across an edge
    assert abs(f1.sum() - f0.sum()) <= 1e-5 * f0.sum()
    assert abs(l1.sum() - l0.sum()) <= 1e-5 * l0.sum()
    fd = np.abs(f1 - f0) > 1e-4 * np.abs(f0) + 1e-9 * f0.max()
    ld = np.abs(l1 - l0) > 1e-4 * np.abs(l0) + 1e-9 * l0.max()
    assert fd.mean() < 2e-3 and ld.mean() < 2e-3, (fd.mean(), ld.mean())
    ctx.close()
