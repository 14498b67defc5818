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

# the octree of the panchromatic disk (configuration 2: max level 10, cell mass fraction 1e-6)
OCTREE = dict(gtype=A.GRID_OCTREE, minLevel=2, maxLevel=10, maxMassFraction=1e-6, samples=100, seed=4357)
OCTREE_ELLS = [8, 20, 36]            # 0.21, 0.65 and 2.9 micron of the 50-point grid
# the k-d tree of the dust-emission disk (configuration 5)
KDTREE = dict(gtype=A.GRID_BINTREE, minLevel=6, maxLevel=30, maxMassFraction=3e-7, samples=100, seed=4357)
KDTREE_ELLS = [10, 25, 45]           # 0.25, 1.02 and 6.4 micron of the 100-point grid
# the clumpy Voronoi disk (configuration 3)
VORONOI_SITES = 1000000
VORONOI_SEED = 77


class SubsetWavelengthGrid:
    """Some wavelengths of a grid, with their own bin widths."""

    def __init__(self, lambdav, dlambdav):
        self.lambdav = np.ascontiguousarray(lambdav, dtype=np.float64)
        self.dlambdav = np.ascontiguousarray(dlambdav, dtype=np.float64)

    @property
    def Nlambda(self):
        return len(self.lambdav)


def wavelength_subset(model, ells):
    """The same simulation restricted to the wavelengths ells: stellar luminosities, mix tables and
    bin widths of those wavelengths, the dust normalisation of the full model (its face-on optical
    depth is defined at 0.55 micron of the full grid).  Packets of one wavelength never touch
    another in the stellar phase, so these wavelengths of the full run and of this run have the
    same expectation."""
    import copy
    from skirt7_b200.scene import DustComp, DustMix, StellarComp
    model.normalise()
    ells = list(ells)
    sub = copy.copy(model)
    wl = model.wavelengthGrid
    sub.wavelengthGrid = SubsetWavelengthGrid(wl.lambdav[ells], wl.dlambdav[ells])
    sub.stellarComps = [StellarComp(c.geometry, np.asarray(c.luminosities)[ells]) for c in model.stellarComps]
    sub.dustComps = [DustComp(d.geometry, DustMix(np.asarray(d.mix.kappaext)[ells], np.asarray(d.mix.albedo)[ells],
                                                  np.asarray(d.mix.asymmpar)[ells]), None, d.norm)
                     for d in model.dustComps]
    sub.instruments = list(model.instruments)
    return sub


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
    """Configuration 2's panchromatic disk: 50 wavelengths 0.1-10 micron, three 512x512 frames."""
    return models.pan_disk(nlambda=50, inclinations=(0, 60, 88), npix=512)


def kdtree_point_model():
    """Configuration 5's disk with a central point source (10 % of the luminosity): 100
    wavelengths 0.1-1000 micron, a 512x512 frame at 60 degrees, absorption tallies kept."""
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
    """The tessellation by Voro++ (oracle/_ref) with VoronoiMesh's block lists."""
    return oracle.voronoi_mesh(sites, EXT)


def block_sums(frame, fmax=32):
    """Sums over square blocks of pixels: the largest block size up to fmax that divides the frame
    (32 for 512x512, 30 for 300x300)."""
    ny, nx = frame.shape[-2:]
    f = next(d for d in range(fmax, 0, -1) if ny % d == 0 and nx % d == 0)
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
