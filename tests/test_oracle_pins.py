"""Pins the oracle (and the library's host-side tree builder) against the reference's own
translation units, compiled in place from the SKIRT7 sources into oracle/_ref by oracle/Makefile:
DustGridPath::pathlength/moveInside, SpecialFunctions::LambertW1, SersicFunction, and the
octree / k-d tree node classes' neighbour lists including their order."""
import ctypes as C
import math

import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import runtime

dp = C.POINTER(C.c_double)


@pytest.fixture(scope="module")
def ref(orc):
    R = orc.ref()
    if R is None:
        pytest.skip("oracle/_ref not built (the reference sources are absent)")
    return R


def _arr(a):
    a = np.ascontiguousarray(a, dtype=np.float64)
    return a, a.ctypes.data_as(dp)


def test_pathlength_matches_reference(orc, ref):
    rng = np.random.default_rng(0)
    L = orc.lib()
    for trial in range(3000):
        n = int(rng.integers(1, 40))
        ds = rng.exponential(1.0, n) * 10 ** rng.uniform(15, 20)
        kr = rng.exponential(1.0, n) * 10 ** rng.uniform(-21, -18)
        kr[rng.random(n) < 0.3] = 0.0              # empty cells (equal cumulative tau)
        ds[rng.random(n) < 0.05] = 0.0             # dropped segments (addSegment ignores ds <= 0)
        tot = float(np.sum(ds * kr))
        for tau in (rng.uniform(0, 1.2) * tot, 0.0, tot, 1e-3 * tot, 2 * tot + 1e-300):
            a, pa = _arr(ds)
            b, pb = _arr(kr)
            x = L.orc_pathlength(pa, pb, n, tau)
            y = ref.ref_pathlength(pa, pb, n, tau)
            assert x == y or (math.isnan(x) and math.isnan(y)), (trial, tau, x, y)


def test_moveinside_matches_reference(orc, ref):
    rng = np.random.default_rng(1)
    box, pbox = _arr([-2.0, -3.0, -1.0, 2.0, 3.0, 1.0])
    L = orc.lib()
    for i in range(20000):
        r = rng.uniform(-6, 6, 3)
        if i % 7 == 0:
            r[rng.integers(0, 3)] = box[rng.integers(0, 6)]   # on a wall
        k = rng.normal(size=3)
        if i % 11 == 0:
            k[rng.integers(0, 3)] = 0.0
        k /= np.linalg.norm(k)
        ra, pr = _arr(r)
        ka, pk = _arr(k)
        o1, po1 = _arr(np.zeros(3)); o2, po2 = _arr(np.zeros(3))
        s1, ps1 = _arr(np.zeros(3)); s2, ps2 = _arr(np.zeros(3))
        n1 = L.orc_moveinside(pbox, 1e-9, pr, pk, po1, ps1)
        n2 = ref.ref_moveinside(pbox, 1e-9, pr, pk, po2, ps2)
        assert n1 == n2
        if n1 >= 0:
            assert np.array_equal(o1, o2) and np.array_equal(s1[:n1], s2[:n1])


def test_lambertw1_matches_reference(orc, ref):
    z = -np.exp(-1.0) * np.concatenate([np.linspace(1e-12, 1.0, 2001)[::-1], 10 ** np.linspace(-300, -1, 300)])
    L = orc.lib()
    for v in z:
        a, b = L.orc_lambertw1(float(v)), ref.ref_lambertw1(float(v))
        assert abs(a - b) <= 1e-12 * abs(b), (v, a, b)


@pytest.mark.parametrize("n", [1.0, 2.5, 4.0, 8.0])
def test_sersic_tables_match_reference(orc, ref, n):
    s, ps = _arr(10 ** np.linspace(-7, 5, 400))
    X, pX = _arr(np.concatenate([[0.0, 1e-12], np.linspace(1e-6, 1 - 1e-9, 500), [1.0]]))
    out = {}
    for who, f in (("orc", orc.lib().orc_sersic), ("ref", ref.ref_sersic)):
        S, pS = _arr(np.zeros(len(s))); M, pM = _arr(np.zeros(len(s))); I, pI = _arr(np.zeros(len(X)))
        f(n, ps, len(s), pS, pM, pX, len(X), pI)
        out[who] = (S, M, I)
    # the profile's normalisation uses Gamma(2n+1): the reference's own SpecialFunctions::gamma
    # against std::tgamma here, a constant factor within 1e-9; the normalised mass and its inverse
    # (what the launch sampler uses) agree to 1e-12.  Below M(s_1) both return NaN: log10 of the
    # zero first mass entry (SersicFunction.cpp:116-121).
    for (a, b), tol in zip(zip(out["orc"], out["ref"]), (1e-9, 1e-12, 1e-12)):
        assert np.allclose(a, b, rtol=tol, atol=0, equal_nan=True)


def _splits(ext, gtype, maxlevel, lmin, seed):
    """Random but reproducible subdivision decisions in creation order."""
    rng = np.random.default_rng(seed)
    levels = [0]
    split = []
    l = 0
    nch = 8 if gtype == A.GRID_OCTREE else 2
    while l < len(levels):
        lev = levels[l]
        do = lev < lmin or (lev < maxlevel and rng.random() < 0.35)
        split.append(1 if do else 0)
        if do:
            levels += [lev + 1] * nch
        l += 1
    return np.array(split, dtype=np.uint8)


@pytest.mark.parametrize("gtype,seed", [(A.GRID_OCTREE, 0), (A.GRID_OCTREE, 1), (A.GRID_BINTREE, 2),
                                        (A.GRID_BINTREE, 3)])
def test_tree_neighbour_lists_match_reference(lib, ref, gtype, seed):
    ext = (-20.0, -20.0, -2.0, 20.0, 20.0, 2.0)
    split = _splits(ext, gtype, 6 if gtype == A.GRID_OCTREE else 14, 2 if gtype == A.GRID_OCTREE else 5, seed)
    tree = runtime.tree_from_splits(gtype, ext, split)
    n = tree.nnodes
    boxes = np.zeros(6 * n)
    off = np.zeros(6 * n + 1, dtype=np.int64)
    cap = int(tree.nbr_offsets[-1]) + 10
    ids = np.zeros(cap, dtype=np.int32)
    e, pe = _arr(ext)
    sp = np.ascontiguousarray(split)
    got = ref.ref_tree_neighbors(1 if gtype == A.GRID_OCTREE else 2, pe, sp.ctypes.data_as(C.POINTER(C.c_uint8)),
                                 len(sp), n, boxes.ctypes.data_as(dp), off.ctypes.data_as(C.POINTER(C.c_int64)),
                                 ids.ctypes.data_as(C.POINTER(C.c_int32)), cap)
    assert got == n
    assert np.array_equal(boxes, tree.node_box)
    # leaves: identical lists in identical order (TreeNode::whichnode(wall, r) takes the first match)
    leaves = np.nonzero(tree.node_cell >= 0)[0]
    assert len(leaves) == tree.ncells > 50
    for l in leaves:
        for w in range(6):
            a = ids[off[6 * l + w]: off[6 * l + w + 1]]
            b = tree.nbr_ids[tree.nbr_offsets[6 * l + w]: tree.nbr_offsets[6 * l + w + 1]]
            assert np.array_equal(a, b), (l, w, a, b)
