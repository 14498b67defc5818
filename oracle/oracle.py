"""TEST INFRASTRUCTURE ONLY -- ctypes wrapper of the CPU oracle (oracle/liboracle.so).

The oracle is a scalar FP64 restatement of SKIRT7's packet life cycle (oracle/oracle.cpp).  It
takes the same scene structs as the CUDA library (include/skirt_b200.h) and is used by tests/,
by __graft_entry__.smoke() as the checker and by bench.py as the CPU baseline; the product never
imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
SRC = os.path.join(HERE, "oracle.cpp")
HDR = os.path.join(HERE, "..", "include", "skirt_b200.h")

dp = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)


class Stats(C.Structure):
    _fields_ = [("packets", C.c_int64), ("steps", C.c_int64), ("traversals", C.c_int64),
                ("scatterings", C.c_int64), ("fallbacks", C.c_int64), ("npp", C.c_uint64), ("chunks", C.c_uint64),
                ("seconds", C.c_double)]


def build():
    """Compiles the oracle with the reference's floating-point semantics (no FMA contraction)."""
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= max(os.path.getmtime(SRC), os.path.getmtime(HDR)):
        return LIB
    subprocess.check_call(["g++", "-O2", "-std=c++20", "-ffp-contract=off", "-fPIC", "-shared", "-o", LIB, SRC,
                           "-lpthread"])
    return LIB


_lib = None
_ref = None
REF_LIB = os.path.join(HERE, "_ref", "libskirt_ref.so")


def ref():
    """The reference's own translation units (oracle/_ref), or None when they were not built."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB):
        R = C.CDLL(REF_LIB)
        R.ref_pathlength.restype = C.c_double
        R.ref_pathlength.argtypes = [dp, dp, C.c_int, C.c_double]
        R.ref_moveinside.argtypes = [dp, C.c_double, dp, dp, dp, dp]
        R.ref_tree_neighbors.restype = C.c_int64
        R.ref_tree_neighbors.argtypes = [C.c_int, dp, C.POINTER(C.c_uint8), C.c_int64, C.c_int64, dp, i64p, i32p,
                                         C.c_int64]
        R.ref_voronoi.restype = C.c_int64
        R.ref_voronoi.argtypes = [dp, C.c_int, dp, C.c_int, i64p, i32p, C.c_int64, dp, dp, dp]
        R.ref_lambertw1.restype = C.c_double
        R.ref_lambertw1.argtypes = [C.c_double]
        R.ref_sersic.argtypes = [C.c_double, dp, C.c_int, dp, dp, dp, C.c_int, dp]
        if hasattr(R, "ref_cartesian_paths"):
            R.ref_cartesian_paths.restype = C.c_int64
            R.ref_cartesian_paths.argtypes = [dp, dp, C.c_int, dp, C.c_int, dp, C.c_int, dp, dp, C.c_int64, i32p, dp,
                                              i64p, C.c_int64]
            R.ref_tree_paths.restype = C.c_int64
            R.ref_tree_paths.argtypes = [C.c_int, dp, C.POINTER(C.c_uint8), C.c_int64, C.c_int, dp, dp, C.c_int64,
                                         i32p, dp, i64p, C.c_int64]
            R.ref_voronoi_paths.restype = C.c_int64
            R.ref_voronoi_paths.argtypes = [dp, C.c_int, dp, dp, dp, C.c_int64, i32p, dp, i64p, C.c_int64]
        _ref = R
    return _ref


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.orc_trace_paths.argtypes = [C.c_void_p, dp, dp, C.c_int64, i32p, dp, i64p, C.c_int64, i64p, C.c_int]
        L.orc_optical_depth.argtypes = [C.c_void_p, dp, dp, C.c_int64, C.c_int, dp]
        L.orc_pathlength.restype = C.c_double
        L.orc_pathlength.argtypes = [dp, dp, C.c_int, C.c_double]
        L.orc_moveinside.argtypes = [dp, C.c_double, dp, dp, dp, dp]
        L.orc_sersic.argtypes = [C.c_double, dp, C.c_int, dp, dp, dp, C.c_int, dp]
        L.orc_lambertw1.restype = C.c_double
        L.orc_lambertw1.argtypes = [C.c_double]
        L.orc_sample_positions.argtypes = [C.c_void_p, C.c_int64, C.c_uint64, dp]
        L.orc_density.argtypes = [C.c_void_p, dp, C.c_int64, dp]
        L.orc_sample_density.argtypes = [C.c_void_p, C.c_int, C.c_uint64, dp]
        L.orc_chunk_params.argtypes = [C.c_double, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint64),
                                       C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]
        L.orc_simulate_packets.argtypes = [C.c_void_p, C.c_uint64, C.c_uint64, C.c_uint64, C.c_int, C.c_uint64, i32p,
                                           C.c_int, C.POINTER(dp), C.POINTER(dp), dp, C.POINTER(Stats)]
        L.orc_tree_build.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_uint64, C.c_int,
                                     C.c_int, C.c_int64, C.POINTER(C.c_uint8), dp, i32p, i32p, i32p,
                                     C.POINTER(C.c_int8), i32p, i64p]
        L.orc_simulate.argtypes = [C.c_void_p, C.c_double, C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_int, C.c_int64, i32p,
                                   C.c_int,
                                   C.POINTER(dp), C.POINTER(dp), dp, dp, dp, C.POINTER(Stats)]
        _lib = L
    return _lib


def _tallies(model):
    nl = model.wavelengthGrid.Nlambda
    cubes, seds = [], []
    for ins in model.instruments:
        nc = 1 if ins.type != 3 else 6 + ins.scatteringLevels
        if ins.type == 1 and getattr(ins, "writeStellarComps", False):
            nc = 1 + len(model.stellarComps)
        cubes.append(None if ins.type == 0 else np.zeros((nc, nl, ins.pixelsY, ins.pixelsX)))
        seds.append(np.zeros((nc, nl)))
    ni = len(model.instruments)
    cp = (dp * max(ni, 1))()
    sp = (dp * max(ni, 1))()
    for i in range(ni):
        cp[i] = cubes[i].ctypes.data_as(dp) if cubes[i] is not None else None
        sp[i] = seds[i].ctypes.data_as(dp)
    return cubes, seds, cp, sp


def simulate_packets(model, npp, first, count, nthreads=8, seed=4357, ells=None):
    """The stellar phase for packets [first, first+count) of a simulation of npp packets per
    wavelength, every packet on its own counter-based stream (orc_simulate_packets): tallies of
    disjoint ranges sum to those of their union.  Needs model.rho."""
    assert model.rho is not None
    sc, keep = model.lower()
    cubes, seds, cp, sp = _tallies(model)
    nl = model.wavelengthGrid.Nlambda
    labs = np.zeros(model.dustGrid.ncells * nl)
    ev = np.ascontiguousarray(ells if ells is not None else [], dtype=np.int32)
    st = Stats()
    assert lib().orc_simulate_packets(C.byref(sc), int(npp), int(first), int(count), nthreads, seed,
                                      ev.ctypes.data_as(i32p) if len(ev) else None, len(ev), cp, sp,
                                      labs.ctypes.data_as(dp), C.byref(st)) == 0
    return dict(cubes=cubes, seds=seds, labs_stel=labs.reshape(-1, nl),
                stats={n: getattr(st, n) for n, _ in Stats._fields_})


def trace_paths(model, r, k, nthreads=None):
    """DustGrid::path for every ray: (offsets, cells, ds), segments of ray i at
    offsets[i]..offsets[i+1]-1; traced by nthreads threads (default: all cores)."""
    nthreads = nthreads or os.cpu_count() or 1
    sc, keep = model.lower()
    r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
    k = np.ascontiguousarray(k, dtype=np.float64).reshape(-1, 3)
    n = len(r)
    off = np.zeros(n + 1, dtype=np.int64)
    fb = np.zeros(1, dtype=np.int64)
    cap = 0
    cells = np.zeros(1, dtype=np.int32)
    ds = np.zeros(1)
    L = lib()
    rc = L.orc_trace_paths(C.byref(sc), r.ctypes.data_as(dp), k.ctypes.data_as(dp), n, cells.ctypes.data_as(i32p),
                           ds.ctypes.data_as(dp), off.ctypes.data_as(i64p), cap, fb.ctypes.data_as(i64p), nthreads)
    if rc == 8:
        cap = int(off[n])
        cells = np.zeros(max(cap, 1), dtype=np.int32)
        ds = np.zeros(max(cap, 1))
        rc = L.orc_trace_paths(C.byref(sc), r.ctypes.data_as(dp), k.ctypes.data_as(dp), n,
                               cells.ctypes.data_as(i32p), ds.ctypes.data_as(dp), off.ctypes.data_as(i64p), cap,
                               fb.ctypes.data_as(i64p), nthreads)
    assert rc == 0
    tot = int(off[n])
    return off, cells[:tot], ds[:tot]


def optical_depth(model, r, k, ell=0):
    sc, keep = model.lower()
    r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
    k = np.ascontiguousarray(k, dtype=np.float64).reshape(-1, 3)
    tau = np.zeros(len(r))
    assert lib().orc_optical_depth(C.byref(sc), r.ctypes.data_as(dp), k.ctypes.data_as(dp), len(r), ell,
                                   tau.ctypes.data_as(dp)) == 0
    return tau


def sample_density(model, nthreads=8, seed=99):
    sc, keep = model.lower()
    rho = np.zeros(len(model.dustComps) * model.dustGrid.ncells)
    lib().orc_sample_density(C.byref(sc), nthreads, seed, rho.ctypes.data_as(dp))
    return rho.reshape(len(model.dustComps), -1)


def simulate(model, packages, nthreads=8, seed=4357, selfabs_cycles=0, dust_emission_phase=False, max_packets=0,
             ells=None, selfabs_staged=False):
    """Runs the restated life cycle; returns dict(cubes, seds, labs_stel, labs_dust, T, stats).
    ells: run the stellar phase for these wavelength indices only (default: all).  selfabs_cycles
    self-absorption cycles at `packages`, or with selfabs_staged in each of the reference's three
    stages (1/10, 1/3 and 1 times the packages)."""
    sc, keep = model.lower()
    nl = model.wavelengthGrid.Nlambda
    ncomp = []
    cubes, seds = [], []
    for ins in model.instruments:
        nc = 1 if ins.type != 3 else 6 + ins.scatteringLevels
        if ins.type == 1 and getattr(ins, "writeStellarComps", False):
            nc = 1 + len(model.stellarComps)
        ncomp.append(nc)
        if ins.type == 0:
            cubes.append(None)
        else:
            cubes.append(np.zeros((nc, nl, ins.pixelsY, ins.pixelsX)))
        seds.append(np.zeros((nc, nl)))
    ni = len(model.instruments)
    cp = (dp * max(ni, 1))()
    sp = (dp * max(ni, 1))()
    for i in range(ni):
        cp[i] = cubes[i].ctypes.data_as(dp) if cubes[i] is not None else None
        sp[i] = seds[i].ctypes.data_as(dp)
    ncells = model.dustGrid.ncells if model.dustGrid is not None else 0
    ls = np.zeros(ncells * nl)
    ld = np.zeros(ncells * nl)
    T = np.zeros(max(ncells, 1))
    st = Stats()
    ev = np.ascontiguousarray(ells if ells is not None else [], dtype=np.int32)
    assert lib().orc_simulate(C.byref(sc), float(packages), nthreads, seed, selfabs_cycles, int(selfabs_staged),
                              int(dust_emission_phase),
                              int(max_packets), ev.ctypes.data_as(i32p) if len(ev) else None, len(ev), cp, sp, ls.ctypes.data_as(dp), ld.ctypes.data_as(dp),
                              T.ctypes.data_as(dp), C.byref(st)) == 0
    stats = {n: getattr(st, n) for n, _ in Stats._fields_}
    return dict(cubes=cubes, seds=seds, labs_stel=ls.reshape(ncells, nl), labs_dust=ld.reshape(ncells, nl),
                T=T[:ncells], stats=stats)


def tree_build(model, gtype, extent, minLevel=2, maxLevel=6, maxMassFraction=1e-6, samples=100, seed=4357,
               sampler=0, nthreads=8, neighbors=True):
    """TreeDustGrid construction restated on the CPU (oracle.cpp: orc_tree_build, following
    TreeDustGrid.cpp:80-230).  sampler 0 draws node samples from the reference's MT19937
    (Random::position); sampler 1 from the counter-based streams of the library's device builder.
    With neighbors=True the neighbour lists come from the reference's own node classes compiled
    in oracle/_ref (ref_tree_neighbors, OctTreeNode/BinTreeNode::addneighbors + sortneighbors),
    given the split decisions.  Returns (TreeDustGrid, split flags, levels)."""
    import sys
    sys.path.insert(0, os.path.join(HERE, ".."))
    from skirt7_b200.scene import CartesianDustGrid, TreeDustGrid
    from skirt7_b200 import _abi as A
    model.normalise()
    saved = model.dustGrid
    x0, y0, z0, x1, y1, z1 = extent
    model.dustGrid = CartesianDustGrid(x0, x1, y0, y1, z0, z1, 1, 1, 1)   # only the extent is read
    sc, keep = model.lower()
    model.dustGrid = saved
    L = lib()
    nn = C.c_int64(0)
    cap = 1
    while True:
        split = np.zeros(cap, dtype=np.uint8)
        box = np.zeros(6 * cap)
        child, father, cell, lev = (np.zeros(cap, dtype=np.int32) for _ in range(4))
        d = np.zeros(cap, dtype=np.int8)
        rc = L.orc_tree_build(C.byref(sc), gtype, minLevel, maxLevel, maxMassFraction, samples, seed, sampler, nthreads,
                              cap, split.ctypes.data_as(C.POINTER(C.c_uint8)), box.ctypes.data_as(dp),
                              child.ctypes.data_as(i32p), father.ctypes.data_as(i32p), cell.ctypes.data_as(i32p),
                              d.ctypes.data_as(C.POINTER(C.c_int8)), lev.ctypes.data_as(i32p), C.byref(nn))
        if rc == 0:
            break
        assert rc == 8, rc
        cap = nn.value
    n = nn.value
    off = np.zeros(6 * n + 1, dtype=np.int64)
    ids = np.zeros(1, dtype=np.int32)
    search = A.SEARCH_TOPDOWN
    if neighbors:
        R = ref()
        if R is None:
            raise RuntimeError("neighbour lists need the reference's node classes (oracle/_ref)")
        t = 1 if gtype == A.GRID_OCTREE else 2
        ex = np.array(extent, dtype=np.float64)
        rbox = np.zeros(6 * n)
        maxids = 16 * n
        while True:
            ids = np.zeros(maxids, dtype=np.int32)
            q = R.ref_tree_neighbors(t, ex.ctypes.data_as(dp), split.ctypes.data_as(C.POINTER(C.c_uint8)), n, n,
                                     rbox.ctypes.data_as(dp), off.ctypes.data_as(i64p), ids.ctypes.data_as(i32p),
                                     maxids)
            if q >= 0:
                break
            maxids = -q
        assert q == n and np.array_equal(rbox, box[: 6 * n]), "reference node boxes differ from the restated ones"
        ids = ids[: off[-1]]
        search = A.SEARCH_NEIGHBOR
    grid = TreeDustGrid(gtype, tuple(extent), box[: 6 * n], child[:n], father[:n], cell[:n], d[:n], off, ids, search)
    return grid, split[:n], lev[:n]


def voronoi_mesh(sites, extent):
    """The tessellation by Voro++ (oracle/_ref) with the block lists of VoronoiMesh::buildMesh
    (VoronoiMesh.cpp:330-395: nb = max(3, min(1000, 3 N^(1/3))) blocks per axis, each listing the
    cells whose box, widened by eps, overlaps it)."""
    import sys
    sys.path.insert(0, os.path.join(HERE, ".."))
    from skirt7_b200 import _abi as A
    from skirt7_b200.scene import VoronoiDustGrid
    EXT = tuple(extent)
    R = ref()
    assert R is not None, "Voro++ (oracle/_ref) not built"
    n = len(sites)
    nb = max(3, min(1000, int(3.0 * n ** (1.0 / 3.0))))
    e = np.ascontiguousarray(EXT, dtype=np.float64)
    s = np.ascontiguousarray(sites, dtype=np.float64)
    off = np.zeros(n + 1, dtype=np.int64)
    vol, cen, bb = np.zeros(n), np.zeros(3 * n), np.zeros(6 * n)
    cap = 20 * n
    while True:
        ids = np.zeros(cap, dtype=np.int32)
        q = R.ref_voronoi(s.ctypes.data_as(dp), n, e.ctypes.data_as(dp), nb, off.ctypes.data_as(A.i64p),
                          ids.ctypes.data_as(A.i32p), cap, vol.ctypes.data_as(dp), cen.ctypes.data_as(dp),
                          bb.ctypes.data_as(dp))
        if q >= 0:
            break
        cap = -q
    ids = ids[: off[-1]]
    bb = bb.reshape(n, 6)
    lo, hi = np.array(EXT[:3]), np.array(EXT[3:])
    eps = 1e-12 * np.linalg.norm(hi - lo)

    def idx(p):   # Box::cellindices (Box.hpp:120-125)
        return np.clip((nb * (p - lo) / (hi - lo)).astype(np.int64), 0, nb - 1)

    i1, i2 = idx(bb[:, :3] - eps), idx(bb[:, 3:] + eps)
    span = i2 - i1 + 1
    cnt = span.prod(1)
    cell = np.repeat(np.arange(n), cnt)
    t = np.arange(cnt.sum()) - np.repeat(np.cumsum(cnt) - cnt, cnt)
    sy, sz = np.repeat(span[:, 1], cnt), np.repeat(span[:, 2], cnt)
    bi = np.repeat(i1[:, 0], cnt) + t // (sy * sz)
    bj = np.repeat(i1[:, 1], cnt) + (t // sz) % sy
    bk = np.repeat(i1[:, 2], cnt) + t % sz
    block = (bi * nb + bj) * nb + bk
    order = np.argsort(block, kind="stable")
    boff = np.zeros(nb ** 3 + 1, dtype=np.int64)
    boff[1:] = np.cumsum(np.bincount(block, minlength=nb ** 3))
    return VoronoiDustGrid(EXT, s, off, ids, nb, boff, cell[order].astype(np.int32), vol, bb)


def _ref_trace(call, r, k):
    r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
    k = np.ascontiguousarray(k, dtype=np.float64).reshape(-1, 3)
    n = len(r)
    off = np.zeros(n + 1, dtype=np.int64)
    cap = 64 * max(n, 1)
    while True:
        cells, ds = np.zeros(cap, dtype=np.int32), np.zeros(cap)
        tot = call(r.ctypes.data_as(dp), k.ctypes.data_as(dp), n, cells.ctypes.data_as(i32p), ds.ctypes.data_as(dp),
                   off.ctypes.data_as(i64p), cap)
        if tot <= cap:
            return off, cells[:tot], ds[:tot]
        cap = int(tot)


def ref_cartesian_paths(grid, r, k):
    """CartesianDustGrid::path of the reference itself (compiled in oracle/_ref) on a grid's planes."""
    R = ref()
    ext = np.ascontiguousarray([grid.minX, grid.minY, grid.minZ, grid.maxX, grid.maxY, grid.maxZ], dtype=np.float64)
    xv, yv, zv = (np.ascontiguousarray(v, dtype=np.float64) for v in (grid.xv, grid.yv, grid.zv))
    return _ref_trace(lambda rp, kp, n, c, d, o, cap: R.ref_cartesian_paths(
        ext.ctypes.data_as(dp), xv.ctypes.data_as(dp), len(xv) - 1, yv.ctypes.data_as(dp), len(yv) - 1,
        zv.ctypes.data_as(dp), len(zv) - 1, rp, kp, n, c, d, o, cap), r, k)


def ref_voronoi_paths(sites, extent, r, k):
    """VoronoiMesh::path of the reference itself on the mesh it builds from the sites (Voro++,
    its block lists and kd-trees)."""
    R = ref()
    s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
    ext = np.ascontiguousarray(extent, dtype=np.float64)
    return _ref_trace(lambda rp, kp, n, c, d, o, cap: R.ref_voronoi_paths(
        s.ctypes.data_as(dp), len(s), ext.ctypes.data_as(dp), rp, kp, n, c, d, o, cap), r, k)


def ref_tree_paths(gtype, extent, split, search, r, k):
    """TreeDustGrid::path of the reference itself (compiled in oracle/_ref) on the octree
    (gtype 1) or k-d tree (2) that its node classes build from the split decisions."""
    R = ref()
    ext = np.ascontiguousarray(extent, dtype=np.float64)
    sp = np.ascontiguousarray(split, dtype=np.uint8)
    return _ref_trace(lambda rp, kp, n, c, d, o, cap: R.ref_tree_paths(
        int(gtype), ext.ctypes.data_as(dp), sp.ctypes.data_as(C.POINTER(C.c_uint8)), len(sp), int(search), rp, kp, n,
        c, d, o, cap), r, k)
