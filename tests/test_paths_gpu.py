"""DustGrid::path on the device against the oracle: identical cell sequences and bit-identical
segment lengths for the FP64 traversal on 10^6 seeded rays (CartesianDustGrid.cpp:136-283,
TreeDustGrid.cpp:371-643), plus edge cases; the FP32 production traversal agrees to 1e-6
relative in path length and optical depth."""
import math

import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import models, runtime
from skirt7_b200.scene import KPC, CartesianDustGrid

from helpers import axis_rays, cell_center_density, seeded_rays

pytestmark = pytest.mark.gpu


def _cfg1_model(N=(100, 100, 50)):
    m = models.oligo_disk(N=N)
    m.rho = cell_center_density(m)
    return m


def _compare(o1, c1, d1, o2, c2, d2):
    assert np.array_equal(o1, o2), "segment counts differ"
    assert np.array_equal(c1, c2), "cell sequences differ"
    assert np.array_equal(d1, d2), "segment lengths differ (max rel %g)" % (
        np.max(np.abs(d1 - d2) / np.maximum(np.abs(d2), 1e-300)))


def test_cartesian_fp64_bit_exact_1e6_rays(orc):
    m = _cfg1_model()
    ctx = runtime.Context(m)
    ext = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)
    r, k = seeded_rays(10 ** 6, ext, seed=0, disk=(4 * KPC, 0.35 * KPC))
    og, cg, dg = ctx.trace_paths(r, k, A.PREC_FP64)
    oo, co, do = orc.trace_paths(m, r, k)
    assert og[-1] > 2 * 10 ** 7     # tens of segments per ray on average
    _compare(og, cg, dg, oo, co, do)
    ctx.close()


def test_cartesian_edge_cases_and_nonuniform_mesh(orc):
    m = _cfg1_model(N=(16, 12, 8))
    # power-law planes (PowMesh-like): non-uniform spacing
    g = m.dustGrid
    t = np.linspace(-1, 1, 17)
    xv = np.sign(t) * np.abs(t) ** 1.7 * 20 * KPC
    m.dustGrid = CartesianDustGrid(g.minX, g.maxX, g.minY, g.maxY, g.minZ, g.maxZ, xv=xv, yv=g.yv, zv=g.zv)
    m.rho = cell_center_density(m)
    ext = (g.minX, g.minY, g.minZ, g.maxX, g.maxY, g.maxZ)
    r1, k1 = axis_rays(ext, planes_x=xv)
    r2, k2 = seeded_rays(20000, ext, seed=5, frac_outside=0.5)
    r = np.concatenate([r1, r2]); k = np.concatenate([k1, k2])
    ctx = runtime.Context(m)
    og, cg, dg = ctx.trace_paths(r, k, A.PREC_FP64)
    oo, co, do = orc.trace_paths(m, r, k)
    _compare(og, cg, dg, oo, co, do)
    # rays starting outside and pointing away give empty paths
    assert (np.diff(og)[: len(r1)] == 0).any()
    ctx.close()


def test_cartesian_fp32_against_fp64():
    m = _cfg1_model()
    ctx = runtime.Context(m)
    ext = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)
    r, k = seeded_rays(200000, ext, seed=1)
    o64, c64, d64 = ctx.trace_paths(r, k, A.PREC_FP64)
    o32, c32, d32 = ctx.trace_paths(r, k, A.PREC_FP32)
    L64 = np.add.reduceat(d64, o64[:-1][np.diff(o64) > 0])
    L32 = np.add.reduceat(d32, o32[:-1][np.diff(o32) > 0])
    same = np.array_equal(o64, o32)
    if same:
        mism = np.mean(c64 != c32)
        assert mism < 1e-3, mism
    # total path length per ray
    assert len(L64) == len(L32)
    diag = np.sqrt(40.0 ** 2 + 40.0 ** 2 + 4.0 ** 2) * KPC
    err = np.abs(L32 - L64)
    # FP32 positions carry ~1e-7 of the domain size; grazing and corner rays may differ more
    assert np.mean(err < 1e-6 * diag + 1e-5 * L64) > 0.999
    assert np.max(err) < 1e-4 * diag
    assert np.median(err / L64) < 1e-6
    tau64 = ctx.optical_depth(r, k, 0, A.PREC_FP64)
    tau32 = ctx.optical_depth(r, k, 0, A.PREC_FP32)
    ok = tau64 > 1e-3
    rel = np.abs(tau32[ok] - tau64[ok]) / tau64[ok]
    # FP32 positions carry ~6e-8 of the 20 kpc half-width, i.e. ~1.5e-5 of an 80 pc z-cell, and a
    # plane crossing of a ray at small |k_z| is uncertain by that over |k_z|: each crossing moves
    # a sliver of path between two cells whose densities differ by tens of percent.  Stated error
    # of the FP32 optical depth against FP64: below 1e-4 relative on 99.9% of the rays, below 1e-2
    # on all of them, and the summed optical depth of all rays within 1e-6.
    assert np.mean(rel < 1e-4) > 0.999 and np.max(rel) < 1e-2, (np.mean(rel < 1e-4), np.max(rel))
    assert abs(tau32[ok].sum() / tau64[ok].sum() - 1) < 1e-6
    ctx.close()


def test_optical_depth_fp64_matches_oracle_exactly(orc):
    m = _cfg1_model()
    ctx = runtime.Context(m)
    ext = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)
    r, k = seeded_rays(50000, ext, seed=2)
    tg = ctx.optical_depth(r, k, 0, A.PREC_FP64)
    to = orc.optical_depth(m, r, k, 0)
    assert np.array_equal(tg, to)
    # face-on optical depth (FaceOnDustCompNormalization.cpp:67-74): tau_V = 1 through the centre of
    # the continuous disk; a column through the cell centred at R_c sees exp(-R_c/h_R) of it, up to
    # the z discretisation of the cell-centre densities (< 1 %)
    tz = ctx.optical_depth(np.array([[1e-3 * KPC, 1e-3 * KPC, -3 * KPC]]), np.array([[0, 0, 1.0]]), 0, A.PREC_FP64)
    Rc = 0.2 * math.sqrt(2.0) * KPC
    assert abs(tz[0] / math.exp(-Rc / (6 * KPC)) - 1.0) < 0.01, tz
    ctx.close()


def _random_splits(gtype, maxlevel, lmin, p, seed=0):
    """Reproducible random subdivision decisions in creation (breadth-first) order."""
    rng = np.random.default_rng(seed)
    levels = [0]
    split = []
    l = 0
    nch = 8 if gtype == A.GRID_OCTREE else 2
    while l < len(levels):
        lev = levels[l]
        do = lev < lmin or (lev < maxlevel and rng.random() < p)
        split.append(1 if do else 0)
        if do:
            levels += [lev + 1] * nch
        l += 1
    return np.array(split, dtype=np.uint8)


def _octree_splits(ext, maxlevel, gtype):
    """Deterministic subdivision: split nodes whose box comes within 1.5 box-widths of the disk
    mid-plane centre, down to maxlevel (creation order = breadth first)."""
    boxes = [np.array(ext, dtype=np.float64)]
    levels = [0]
    split = []
    nch = 8 if gtype == A.GRID_OCTREE else 2
    l = 0
    while l < len(boxes):
        b, lev = boxes[l], levels[l]
        c = 0.5 * (b[:3] + b[3:])
        w = b[3:] - b[:3]
        half = 0.5 * (np.array(ext[3:]) - np.array(ext[:3]))
        rr = np.linalg.norm(c / half)
        lmin = 2 if gtype == A.GRID_OCTREE else 6
        do = lev < lmin or (lev < maxlevel and rr < 0.9 * 0.8 ** (lev - lmin))
        split.append(1 if do else 0)
        if do:
            if gtype == A.GRID_OCTREE:
                for o in range(8):
                    lo = np.where([o & 1, o & 2, o & 4], c, b[:3])
                    hi = np.where([o & 1, o & 2, o & 4], b[3:], c)
                    boxes.append(np.concatenate([lo, hi])); levels.append(lev + 1)
            else:
                dd = lev % 3
                b0 = b.copy(); b1 = b.copy()
                b0[dd + 3] = c[dd]; b1[dd] = c[dd]
                boxes += [b0, b1]; levels += [lev + 1, lev + 1]
        l += 1
    return np.array(split, dtype=np.uint8)


@pytest.mark.parametrize("gtype,search", [(A.GRID_OCTREE, A.SEARCH_NEIGHBOR), (A.GRID_OCTREE, A.SEARCH_TOPDOWN),
                                          (A.GRID_OCTREE, A.SEARCH_BOOKKEEPING),
                                          (A.GRID_BINTREE, A.SEARCH_NEIGHBOR), (A.GRID_BINTREE, A.SEARCH_TOPDOWN)])
def test_tree_fp64_bit_exact(orc, gtype, search):
    ext = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)
    if gtype == A.GRID_OCTREE:
        split = _random_splits(gtype, 7, 2, 0.35)
    else:
        split = _random_splits(gtype, 22, 6, 0.62)
    tree = runtime.tree_from_splits(gtype, ext, split, search)
    assert tree.ncells > 1000
    m = models.oligo_disk()
    m.dustGrid = tree
    m.rho = np.full((1, tree.ncells), 1e-21)
    n = 300000 if search != A.SEARCH_TOPDOWN else 100000
    r, k = seeded_rays(n, ext, seed=3, disk=(4 * KPC, 0.35 * KPC))
    r1, k1 = axis_rays(ext)
    r = np.concatenate([r1, r]); k = np.concatenate([k1, k])
    ctx = runtime.Context(m)
    og, cg, dg = ctx.trace_paths(r, k, A.PREC_FP64)
    oo, co, do = orc.trace_paths(m, r, k)
    _compare(og, cg, dg, oo, co, do)
    # FP32 traversal: same total path lengths to 1e-5
    o32, c32, d32 = ctx.trace_paths(r, k, A.PREC_FP32)
    nz = np.diff(og) > 0
    L64 = np.add.reduceat(dg, og[:-1][nz])
    nz32 = np.diff(o32) > 0
    assert np.array_equal(nz, nz32)
    L32 = np.add.reduceat(d32, o32[:-1][nz32])
    diag = np.sqrt(40.0 ** 2 + 40.0 ** 2 + 4.0 ** 2) * KPC
    err = np.abs(L32 - L64)
    assert np.mean(err < 2e-6 * diag + 1e-5 * L64) > 0.999
    assert np.max(err) < 1e-4 * diag
    ctx.close()


@pytest.mark.parametrize("gtype", [A.GRID_OCTREE, A.GRID_BINTREE])
def test_tree_fp32_lattice_records_against_rope_records(gtype, monkeypatch):
    """The FP32 walk on 32-byte lattice leaf records (walls computed from integer centre codes)
    against the walk on 64-byte records holding the FP32-rounded FP64 boxes: the walls differ by at
    most an FP32 rounding, so cell sequences agree except at near-ties and path lengths and optical
    depths agree to FP32 resolution."""
    ext = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)
    split = _random_splits(gtype, 7, 2, 0.35, seed=1) if gtype == A.GRID_OCTREE else _random_splits(gtype, 22, 6, 0.62, seed=1)
    tree = runtime.tree_from_splits(gtype, ext, split, A.SEARCH_NEIGHBOR)
    assert tree.ncells > 3000
    m = models.oligo_disk()
    m.dustGrid = tree
    m.rho = np.random.default_rng(4).uniform(0.5e-21, 2e-21, (1, tree.ncells))
    r, k = seeded_rays(200000, ext, seed=8, disk=(4 * KPC, 0.35 * KPC))
    monkeypatch.setenv("SKG_TREE_RECORDS", "rope")
    ctx_rope = runtime.Context(m)
    monkeypatch.delenv("SKG_TREE_RECORDS")
    ctx_lat = runtime.Context(m)
    oa, ca, da = ctx_rope.trace_paths(r, k, A.PREC_FP32)
    ob, cb, db = ctx_lat.trace_paths(r, k, A.PREC_FP32)
    assert not (np.array_equal(oa, ob) and np.array_equal(da, db)), "both contexts walked the same records"
    # rays with identical cell sequences
    na, nb = np.diff(oa), np.diff(ob)
    same = na == nb
    ids = np.flatnonzero(same & (na > 0))
    seq_ok = np.array([np.array_equal(ca[oa[i]:oa[i + 1]], cb[ob[i]:ob[i + 1]]) for i in ids[:20000]])
    assert np.mean(same) > 0.999 and np.mean(seq_ok) > 0.999, (np.mean(same), np.mean(seq_ok))
    nz = na > 0
    assert np.array_equal(nz, nb > 0)
    La = np.add.reduceat(da, oa[:-1][nz])
    Lb = np.add.reduceat(db, ob[:-1][nz])
    diag = np.sqrt(40.0 ** 2 + 40.0 ** 2 + 4.0 ** 2) * KPC
    assert np.max(np.abs(La - Lb)) < 1e-5 * diag
    ta = ctx_rope.optical_depth(r, k, 0, A.PREC_FP32)
    tb = ctx_lat.optical_depth(r, k, 0, A.PREC_FP32)
    ok = ta > 1e-3
    rel = np.abs(ta[ok] - tb[ok]) / ta[ok]
    assert np.mean(rel < 1e-5) > 0.999 and abs(tb[ok].sum() / ta[ok].sum() - 1) < 1e-6
    ctx_rope.close()
    ctx_lat.close()
