"""Voronoi grid: the device tessellation against Voro++ (the reference's vendored library, built in
oracle/_ref) -- identical neighbour sets, volumes and boxes -- and VoronoiMesh::path on the device
against the oracle: bit-identical FP64 cell sequences and segment lengths
(VoronoiMesh.cpp:778-873)."""
import ctypes as C

import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import models, runtime
from skirt7_b200.scene import KPC, VoronoiDustGrid

from helpers import axis_rays, seeded_rays

pytestmark = pytest.mark.gpu

EXT = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)
dp = C.POINTER(C.c_double)


def voronoi_sites(n, seed=0, frac_uniform=0.2):
    """Sites drawn from an exponential disk plus a uniform background (the Voronoi workload's
    80 % density-sampled + 20 % uniform mix)."""
    rng = np.random.default_rng(seed)
    nu = int(frac_uniform * n)
    lo, hi = np.array(EXT[:3]), np.array(EXT[3:])
    u = lo + rng.random((nu, 3)) * (hi - lo)
    nd = n - nu
    R = 6 * KPC * rng.gamma(2.0, 1.0, 3 * nd)
    ph = rng.uniform(0, 2 * np.pi, 3 * nd)
    z = rng.laplace(0, 0.25 * KPC, 3 * nd)
    d = np.stack([R * np.cos(ph), R * np.sin(ph), z], 1)
    inside = np.all((d > lo) & (d < hi), axis=1)
    d = d[inside][:nd]
    return np.ascontiguousarray(np.concatenate([u, d]))


def build_mesh(sites):
    lib = A.load()
    h = C.c_void_p()
    s = np.ascontiguousarray(sites, dtype=np.float64)
    A.check(lib.skg_voronoi_build(s.ctypes.data_as(dp), len(s), *EXT, 0, C.byref(h)))
    n, nn, nb, nbid = C.c_int32(), C.c_int64(), C.c_int32(), C.c_int64()
    lib.skg_voronoi_sizes(h, C.byref(n), C.byref(nn), C.byref(nb), C.byref(nbid))
    n = n.value
    out = dict(sites=np.zeros((n, 3)), off=np.zeros(n + 1, dtype=np.int64), ids=np.zeros(nn.value, dtype=np.int32),
               vol=np.zeros(n), cen=np.zeros((n, 3)), bbox=np.zeros((n, 6)),
               boff=np.zeros(nb.value ** 3 + 1, dtype=np.int64), bids=np.zeros(nbid.value, dtype=np.int32))
    lib.skg_voronoi_arrays(h, out["sites"].ctypes.data_as(dp), out["off"].ctypes.data_as(A.i64p),
                           out["ids"].ctypes.data_as(A.i32p), out["vol"].ctypes.data_as(dp),
                           out["cen"].ctypes.data_as(dp), out["bbox"].ctypes.data_as(dp),
                           out["boff"].ctypes.data_as(A.i64p), out["bids"].ctypes.data_as(A.i32p))
    lib.skg_voronoi_destroy(h)
    out["nb"] = nb.value
    return out


def as_grid(m):
    return VoronoiDustGrid(EXT, m["sites"], m["off"], m["ids"], m["nb"], m["boff"], m["bids"], m["vol"], m["bbox"])


def test_tessellation_matches_voropp(orc):
    R = orc.ref()
    if R is None:
        pytest.skip("oracle/_ref (Voro++) not built")
    sites = voronoi_sites(20000, seed=1)
    m = build_mesh(sites)
    n = len(m["sites"])
    assert n == len(sites)
    assert abs(m["vol"].sum() / np.prod(np.array(EXT[3:]) - np.array(EXT[:3])) - 1) < 1e-9
    nb = m["nb"]
    off = np.zeros(n + 1, dtype=np.int64)
    cap = 40 * n
    ids = np.zeros(cap, dtype=np.int32)
    vol, cen, bb = np.zeros(n), np.zeros(3 * n), np.zeros(6 * n)
    e = np.ascontiguousarray(EXT, dtype=np.float64)
    s = np.ascontiguousarray(m["sites"])
    q = R.ref_voronoi(s.ctypes.data_as(dp), n, e.ctypes.data_as(dp), nb, off.ctypes.data_as(A.i64p),
                      ids.ctypes.data_as(A.i32p), cap, vol.ctypes.data_as(dp), cen.ctypes.data_as(dp),
                      bb.ctypes.data_as(dp))
    assert q > 0
    assert np.allclose(vol, m["vol"], rtol=1e-9, atol=0)
    assert np.allclose(bb.reshape(n, 6), m["bbox"], rtol=0, atol=1e-9 * 40 * KPC)
    assert np.allclose(cen.reshape(n, 3), m["cen"], rtol=0, atol=1e-9 * 40 * KPC)
    for i in range(n):
        a = set(ids[off[i]:off[i + 1]].tolist())
        b = set(m["ids"][m["off"][i]:m["off"][i + 1]].tolist())
        assert a == b, (i, a ^ b)


def test_voronoi_paths_fp64_bit_exact(orc):
    m = build_mesh(voronoi_sites(50000, seed=2))
    grid = as_grid(m)
    model = models.oligo_disk()
    model.dustGrid = grid
    model.rho = np.full((1, grid.ncells), 1e-21)
    ctx = runtime.Context(model)
    r, k = seeded_rays(200000, EXT, seed=4, disk=(4 * KPC, 0.35 * KPC))
    r1, k1 = axis_rays(EXT)
    r = np.concatenate([r1, r]); k = np.concatenate([k1, k])
    og, cg, dg = ctx.trace_paths(r, k, A.PREC_FP64)
    oo, co, do = orc.trace_paths(model, r, k)
    assert np.array_equal(og, oo) and np.array_equal(cg, co) and np.array_equal(dg, do)
    # FP32 traversal (precomputed bisector planes): total lengths
    o32, c32, d32 = ctx.trace_paths(r, k, A.PREC_FP32)
    nz = np.diff(og) > 0
    nz32 = np.diff(o32) > 0
    assert np.mean(nz == nz32) > 0.999
    both = nz & nz32
    L64 = np.add.reduceat(dg, og[:-1][nz])[both[nz]]
    L32 = np.add.reduceat(d32, o32[:-1][nz32])[both[nz32]]
    diag = np.sqrt(40.0 ** 2 + 40.0 ** 2 + 4.0 ** 2) * KPC
    err = np.abs(L32 - L64)
    assert np.mean(err < 2e-6 * diag + 1e-5 * L64) > 0.999
    # optical depth in FP64 through the library and the oracle agree exactly
    tg = ctx.optical_depth(r[:20000], k[:20000], 0, A.PREC_FP64)
    to = orc.optical_depth(model, r[:20000], k[:20000], 0)
    assert np.array_equal(tg, to)
    ctx.close()
