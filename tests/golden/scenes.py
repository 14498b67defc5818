"""TEST INFRASTRUCTURE: the deterministic scenes of the tracer-parity fixtures.

Each scene is one of the benchmark configurations at its own size -- the panchromatic octree disk
(max level 10, mass fraction 1e-6: 2,986,747 leaves), the k-d tree disk with a central point
source (config 5's grid, ~4*10^6 leaves) and the clumpy disk on a 10^6-site Voronoi grid (tau_V 5)
-- with inputs that both sides rebuild identically:

  * tree grids come from the subdivision restated in the oracle with the device builder's
    counter-based node sampler (identical decisions; the GPU test builds the same tree on the
    device and checks its hash against the fixture's);
  * Voronoi sites from a seeded generator, the tessellation from Voro++ (the reference's own
    library, oracle/_ref) or the device builder (equal neighbour sets and volumes; checked by
    counts against the fixture);
  * cell densities are the dust density at the cell centre (trees) or at the generator site
    (Voronoi), evaluated by the oracle's restated geometries: deterministic on any machine, so
    both sides trace the same medium.

Only tests/ and the fixture generator import this module."""
import ctypes as C
import hashlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import oracle  # noqa: E402
from skirt7_b200 import _abi as A  # noqa: E402
from skirt7_b200 import models  # noqa: E402
from skirt7_b200.scene import KPC, MICRON, TreeDustGrid, VoronoiDustGrid  # noqa: E402

EXT = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)
dp = C.POINTER(C.c_double)

# the octree of the panchromatic disk
OCTREE = dict(gtype=A.GRID_OCTREE, minLevel=2, maxLevel=10, maxMassFraction=1e-6, samples=100, seed=4357)
OCTREE_ELLS = [8, 20, 36]            # 0.21, 0.65 and 2.9 micron of the 50-point grid
# the k-d tree of the dust-emission disk (configuration 5)
KDTREE = dict(gtype=A.GRID_BINTREE, minLevel=6, maxLevel=30, maxMassFraction=3e-7, samples=100, seed=4357)
KDTREE_ELLS = [10, 25, 45]           # 0.25, 1.02 and 6.4 micron of the 100-point grid
# the clumpy Voronoi disk (configuration 3)
VORONOI_SITES = 1000000
VORONOI_SEED = 77


def tree_hash(grid):
    h = hashlib.sha256()
    for a in (grid.node_box, grid.node_child, grid.node_cell):
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()[:16]


def voronoi_signature(grid):
    deg = np.diff(grid.vnbr_offsets)
    return {"ncells": int(grid.ncells), "nnbr": int(grid.vnbr_offsets[-1]), "deg2": int((deg.astype(np.int64) ** 2).sum())}


def geometry_density(model, pts):
    """sum_h norm_h * rho_h(r) at the given points (the oracle's restated geometries)."""
    model.normalise()
    pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    L = oracle.lib()
    out = np.zeros(len(pts))
    tmp = np.zeros(len(pts))
    for d in model.dustComps:
        g = A.Geometry()
        d.geometry.lower(g)
        L.orc_density(C.byref(g), pts.ctypes.data_as(dp), len(pts), tmp.ctypes.data_as(dp))
        out += d.norm * tmp
    return out


def cell_centres(grid):
    if isinstance(grid, VoronoiDustGrid):
        return grid.sites
    b = grid.node_box.reshape(-1, 6)
    leaf = grid.node_cell >= 0
    order = np.argsort(grid.node_cell[leaf])
    bl = b[leaf][order]
    return 0.5 * (bl[:, :3] + bl[:, 3:])


def centre_density(model):
    return geometry_density(model, cell_centres(model.dustGrid)).reshape(1, -1)


def tree_grid(model, spec, nthreads=None):
    """The restated subdivision with the device builder's sampler (neighbour lists from the
    reference's node classes)."""
    grid, _, _ = oracle.tree_build(model, spec["gtype"], EXT, spec["minLevel"], spec["maxLevel"],
                                   spec["maxMassFraction"], spec["samples"], spec["seed"], sampler=1,
                                   nthreads=nthreads or os.cpu_count() or 1)
    return grid


def octree_pan_model():
    return models.pan_disk(nlambda=50, inclinations=(0, 60, 88), npix=512)


def kdtree_point_model():
    return models.pan_disk(nlambda=100, lmin=0.1 * MICRON, lmax=1000 * MICRON, inclinations=(60,), npix=512,
                           point_fraction=0.1, write_absorption=True)


def voronoi_sites(n=VORONOI_SITES, seed=VORONOI_SEED):
    """80 % of the sites from the smooth dust disk, 20 % uniform in the domain (configuration 3)."""
    rng = np.random.default_rng(seed)
    lo, hi = np.array(EXT[:3]), np.array(EXT[3:])
    nd = int(0.8 * n)
    d = np.zeros((0, 3))
    while len(d) < nd:
        R = 6 * KPC * rng.gamma(2.0, 1.0, n)
        ph = rng.uniform(0, 2 * np.pi, n)
        z = rng.laplace(0, 0.25 * KPC, n)
        q = np.stack([R * np.cos(ph), R * np.sin(ph), z], 1)
        d = np.concatenate([d, q[np.all((q > lo) & (q < hi), axis=1)]])
    u = lo + rng.random((n - nd, 3)) * (hi - lo)
    return np.ascontiguousarray(np.concatenate([d[:nd], u]))


def voronoi_clumpy_model():
    return models.clumpy_disk(tauV=5.0)


def voropp_mesh(sites):
    """The tessellation by Voro++ (oracle/_ref) with the block lists of VoronoiMesh::buildMesh
    (VoronoiMesh.cpp:330-395: nb = max(3, min(1000, 3 N^(1/3))) blocks per axis, each listing the
    cells whose box, widened by eps, overlaps it)."""
    R = oracle.ref()
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


def block_sums(frame, f=32):
    ny, nx = frame.shape[-2:]
    return frame.reshape(frame.shape[:-2] + (ny // f, f, nx // f, f)).sum((-3, -1))


def labs_groups(grid, labs, nr=8, nz=4):
    """Absorbed luminosity [cells][ells] summed over groups of cells by the radius (nr bins out to
    20 kpc) and height (nz bins out to 2 kpc) of the cell centre."""
    c = cell_centres(grid)
    R = np.hypot(c[:, 0], c[:, 1])
    ir = np.clip((R / (20 * KPC) * nr).astype(int), 0, nr - 1)
    iz = np.clip((np.abs(c[:, 2]) / (2 * KPC) * nz).astype(int), 0, nz - 1)
    g = ir * nz + iz
    out = np.zeros((nr * nz, labs.shape[1]))
    np.add.at(out, g, labs)
    return out
