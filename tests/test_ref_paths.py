"""The oracle's restated grid walks against the reference's own compiled ones (TEST INFRASTRUCTURE
pins, CPU only): CartesianDustGrid::path (CartesianDustGrid.cpp:136-283), TreeDustGrid::path
(TreeDustGrid.cpp:371-643, all three search methods, on trees the reference's node classes build)
and VoronoiMesh::path (VoronoiMesh.cpp:778-873, on the mesh VoronoiMesh builds itself with Voro++,
its block lists and kd-trees) are compiled unmodified from the reference's sources into oracle/_ref
(oracle/Makefile, Qt-lite shims for the simulation-item headers).  On the same rays the cell sequences and segment
lengths are identical, so the GPU's bit-exact agreement with the oracle (test_paths_gpu,
test_voronoi_gpu, test_config_paths_gpu) is agreement with the reference's code."""
import numpy as np
import pytest

from skirt7_b200 import models
from skirt7_b200.scene import KPC, CartesianDustGrid

from helpers import axis_rays, seeded_rays

EXT = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)


@pytest.fixture(scope="module")
def R(orc):
    R = orc.ref()
    if R is None or not hasattr(R, "ref_cartesian_paths"):
        pytest.skip("the reference's grid classes are not built (oracle/_ref)")
    return R


def _same(a, b):
    (oa, ca, da), (ob, cb, db) = a, b
    assert np.array_equal(oa, ob), "segment counts differ"
    assert np.array_equal(ca, cb), "cell sequences differ"
    assert np.array_equal(da, db), "segment lengths differ"


@pytest.mark.parametrize("planes", ["linear", "random"])
def test_cartesian_restatement_is_the_reference_walk(R, orc, planes):
    m = models.oligo_disk()                        # configuration 1: 100 x 100 x 50 cells
    if planes == "random":                         # non-uniform planes (any MoveableMesh)
        rng = np.random.default_rng(3)
        g = m.dustGrid
        pts = lambda n, lo, hi: np.concatenate([[lo], np.sort(rng.uniform(lo, hi, n - 1)), [hi]])
        m.dustGrid = CartesianDustGrid(g.minX, g.maxX, g.minY, g.maxY, g.minZ, g.maxZ, 37, 29, 23,
                                       pts(37, g.minX, g.maxX), pts(29, g.minY, g.maxY), pts(23, g.minZ, g.maxZ))
    m.rho = np.full((1, m.dustGrid.pointsX * m.dustGrid.pointsY * m.dustGrid.pointsZ), 1e-21)
    r, k = seeded_rays(100000, EXT, seed=12, disk=(4 * KPC, 0.35 * KPC))
    r1, k1 = axis_rays(EXT, m.dustGrid.xv)
    r = np.concatenate([r1, r]); k = np.concatenate([k1, k])
    _same(orc.trace_paths(m, r, k), orc.ref_cartesian_paths(m.dustGrid, r, k))


def test_voronoi_restatement_is_the_reference_walk(R, orc):
    import os, sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import scenes
    sites = scenes.voronoi_sites(20000, seed=5)
    m = models.oligo_disk()
    m.dustGrid = orc.voronoi_mesh(sites, EXT)
    m.rho = np.full((1, m.dustGrid.ncells), 1e-21)
    r, k = seeded_rays(20000, EXT, seed=13, disk=(4 * KPC, 0.35 * KPC))
    r1, k1 = axis_rays(EXT)
    r = np.concatenate([r1, r]); k = np.concatenate([k1, k])
    o, c, d = orc.ref_voronoi_paths(sites, EXT, r, k)
    # VoronoiMesh::buildMesh numbers its cells in the order of the sites sorted on x (the sort that
    # looks for nearby sites, VoronoiMesh.cpp:300-327); the library and the oracle keep the input
    # order: the same cells under another numbering
    order = np.argsort(sites[:, 0], kind="stable")
    c = np.where(c >= 0, order[np.maximum(c, 0)], c).astype(np.int32)
    _same(orc.trace_paths(m, r, k), (o, c, d))


def _random_splits(gtype, maxlevel, minlevel, p, seed):
    rng = np.random.default_rng(seed)
    levels, split, l = [0], [], 0
    nch = 8 if gtype == 1 else 2
    while l < len(levels):
        do = levels[l] < minlevel or (levels[l] < maxlevel and rng.random() < p)
        split.append(1 if do else 0)
        if do:
            levels += [levels[l] + 1] * nch
        l += 1
    return np.array(split, dtype=np.uint8)


@pytest.mark.parametrize("gtype,search", [(1, 0), (1, 1), (1, 2), (2, 0), (2, 1)])
def test_tree_restatement_is_the_reference_walk(R, orc, gtype, search):
    from skirt7_b200 import _abi as A, runtime
    split = _random_splits(gtype, 7, 2, 0.35, 4) if gtype == 1 else _random_splits(gtype, 20, 6, 0.6, 4)
    tree = runtime.tree_from_splits(A.GRID_OCTREE if gtype == 1 else A.GRID_BINTREE, EXT, split, search)
    assert tree.ncells > 1000
    m = models.oligo_disk()
    m.dustGrid = tree
    m.rho = np.full((1, tree.ncells), 1e-21)
    r, k = seeded_rays(30000 if search else 10000, EXT, seed=14 + search, disk=(4 * KPC, 0.35 * KPC))
    r1, k1 = axis_rays(EXT)
    r = np.concatenate([r1, r]); k = np.concatenate([k1, k])
    _same(orc.trace_paths(m, r, k), orc.ref_tree_paths(gtype, EXT, split, search, r, k))


def test_cfg2_octree_restatement_is_the_reference_walk(R, orc):
    """Configuration 2's octree (max level 10, mass fraction 1e-6: 2,986,747 leaves), subdivided by
    the oracle's restatement, built and walked (Neighbor search) by the reference's own classes."""
    import os, sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import scenes
    m = scenes.octree_pan_model()
    s = scenes.OCTREE
    grid, split, _ = orc.tree_build(m, s["gtype"], EXT, s["minLevel"], s["maxLevel"], s["maxMassFraction"],
                                    s["samples"], s["seed"], sampler=1)
    assert grid.ncells == 2986747
    m.dustGrid = grid
    m.rho = np.full((1, grid.ncells), 1e-21)
    r, k = seeded_rays(20000, EXT, seed=16, disk=(4 * KPC, 0.35 * KPC))
    _same(orc.trace_paths(m, r, k), orc.ref_tree_paths(1, EXT, split, 1, r, k))
