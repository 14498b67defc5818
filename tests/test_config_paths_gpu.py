"""Bit-exact traversal gates at the configurations' own sizes (DustGrid::path on 10^6 seeded rays):

  * configuration 2's octree (max level 10, mass fraction 1e-6: 2,986,747 leaves), built by the
    device builder (the same tree as the restated subdivision, test_grid_setup_gpu): the FP64
    walk with the Neighbor search on 10^6 rays, TopDown and Bookkeeping on 10^5, against the
    oracle's TreeDustGrid::path (TreeDustGrid.cpp:371-643): identical cell sequences and
    segment lengths;
  * configuration 3's Voronoi grid (10^6 sites, 80 % disk + 20 % uniform), tessellated on the
    device: the FP64 walk on 10^6 rays against the oracle's VoronoiMesh::path
    (VoronoiMesh.cpp:778-873).

Rays: origins uniform in the domain (10 % outside it, to exercise the entry) and a third drawn
from the stellar disk, isotropic directions, Philox-free numpy seed.  The FP32 production walks
are compared on the same rays: the fraction of rays whose FP32 cell sequence differs from the
FP64 one (a wall crossed in a different order at a near-tie) is bounded here and stated in the
design notes."""
import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import runtime
from skirt7_b200.scene import KPC

import os, sys
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import scenes  # noqa: E402
from helpers import seeded_rays  # noqa: E402

pytestmark = pytest.mark.gpu
EXT = scenes.EXT
CHUNK = 100000


def seq_mismatch(o1, c1, o2, c2):
    """Number of rays whose cell sequences differ (length or any cell)."""
    n1, n2 = np.diff(o1), np.diff(o2)
    same = n1 == n2
    idx = np.flatnonzero(same & (n1 > 0))
    lens = n1[idx]
    rep = np.repeat(np.arange(len(idx)), lens)
    off = np.arange(lens.sum()) - np.repeat(np.cumsum(lens) - lens, lens)
    eq = c1[np.repeat(o1[idx], lens) + off] == c2[np.repeat(o2[idx], lens) + off]
    bad = np.bincount(rep, ~eq, len(idx)) > 0
    return int((~same).sum() + bad.sum())


def _gate(ctx, model, orc, r, k, fp32=True):
    """FP64 device == oracle on every chunk; returns the FP32 mismatch count."""
    mism = 0
    for i in range(0, len(r), CHUNK):
        rr, kk = r[i:i + CHUNK], k[i:i + CHUNK]
        og, cg, dg = ctx.trace_paths(rr, kk, A.PREC_FP64)
        oo, co, do = orc.trace_paths(model, rr, kk)
        assert np.array_equal(og, oo), "segment counts differ in chunk %d" % (i // CHUNK)
        assert np.array_equal(cg, co), "cell sequences differ in chunk %d" % (i // CHUNK)
        assert np.array_equal(dg, do), "segment lengths differ in chunk %d" % (i // CHUNK)
        if fp32:
            o32, c32, _ = ctx.trace_paths(rr, kk, A.PREC_FP32)
            mism += seq_mismatch(og, cg, o32, c32)
    return mism


@pytest.fixture(scope="module")
def cfg2_octree():
    m = scenes.octree_pan_model()
    s = scenes.OCTREE
    m.dustGrid = runtime.build_tree(m, s["gtype"], EXT, minLevel=s["minLevel"], maxLevel=s["maxLevel"],
                                    maxMassFraction=s["maxMassFraction"], sampleCount=s["samples"], seed=s["seed"])
    m.rho = np.full((1, m.dustGrid.ncells), 1e-21)
    return m


def test_cfg2_octree_neighbor_search_bit_exact_on_1e6_rays(orc, cfg2_octree):
    m = cfg2_octree
    assert m.dustGrid.ncells == 2986747
    ctx = runtime.Context(m)
    r, k = seeded_rays(1000000, EXT, seed=20, disk=(4 * KPC, 0.35 * KPC))
    mism = _gate(ctx, m, orc, r, k)
    ctx.close()
    print("octree cfg2: FP32 cell sequences differing from FP64 on %d of %d rays (%.4f %%)"
          % (mism, len(r), 100.0 * mism / len(r)))
    assert mism < 0.01 * len(r)


@pytest.mark.parametrize("search", [A.SEARCH_TOPDOWN, A.SEARCH_BOOKKEEPING])
def test_cfg2_octree_other_searches_bit_exact(orc, cfg2_octree, search):
    m = cfg2_octree
    saved = m.dustGrid.searchMethod
    m.dustGrid.searchMethod = search
    try:
        ctx = runtime.Context(m)
        r, k = seeded_rays(100000, EXT, seed=21 + search, disk=(4 * KPC, 0.35 * KPC))
        _gate(ctx, m, orc, r, k, fp32=False)
        ctx.close()
    finally:
        m.dustGrid.searchMethod = saved


def test_cfg3_voronoi_bit_exact_on_1e6_rays(orc):
    m = scenes.voronoi_clumpy_model()
    m.dustGrid = runtime.build_voronoi(scenes.voronoi_sites(), EXT)
    assert m.dustGrid.ncells == scenes.VORONOI_SITES
    m.rho = np.full((1, m.dustGrid.ncells), 1e-21)
    ctx = runtime.Context(m)
    r, k = seeded_rays(1000000, EXT, seed=30, disk=(4 * KPC, 0.35 * KPC))
    mism = _gate(ctx, m, orc, r, k)
    ctx.close()
    print("voronoi cfg3: FP32 cell sequences differing from FP64 on %d of %d rays (%.4f %%)"
          % (mism, len(r), 100.0 * mism / len(r)))
    assert mism < 0.02 * len(r)
