"""Grid set-up on the device against the oracle.

P18 -- tree subdivision (TreeDustGrid.cpp:80-230): the device builder samples node masses with
counter-based streams; the oracle restates the subdivision and can draw the same samples, so at
the benchmark sizes (configuration 2's octree, configuration 5's k-d tree) both make identical
decisions and produce identical trees, with the leaf neighbour lists of the reference's own node
classes (order included).  With the reference's own sampler (MT19937 Random::position) the
decisions differ only near the threshold: leaf counts per level agree within sampling noise.

P17 -- cell densities (DustSystem::setSampleDensityBody, DustSystem.cpp:145-172): the device's
per-cell averages of 100 random samples against two independent oracle runs -- per slab the mean
difference within the noise the oracle runs show between themselves, the same scatter, and the
total dust mass in the domain equal to the analytic mass of the exponential disk in the box
(DustComp::mass, ExpDiskGeometry density normalisation ExpDiskGeometry.cpp:24-40)."""
import math

import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import models, runtime
from skirt7_b200.scene import KPC

import sys, os
sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import scenes  # noqa: E402

pytestmark = pytest.mark.gpu
EXT = scenes.EXT


def _leaf_lists(tree):
    """Per (leaf, wall) list lengths and the concatenated ids of the leaves' lists."""
    leaf = tree.node_cell >= 0
    cnt = np.diff(tree.nbr_offsets).reshape(-1, 6)
    owner = np.repeat(np.repeat(leaf, 6), np.diff(tree.nbr_offsets))
    return cnt[leaf], tree.nbr_ids[owner]


@pytest.mark.parametrize("spec,model", [(scenes.OCTREE, scenes.octree_pan_model),
                                        (scenes.KDTREE, scenes.kdtree_point_model)],
                         ids=["octree_cfg2", "kdtree_cfg5"])
def test_device_tree_is_the_restated_subdivision(orc, spec, model):
    m = model()
    dev = runtime.build_tree(m, spec["gtype"], EXT, minLevel=spec["minLevel"], maxLevel=spec["maxLevel"],
                             maxMassFraction=spec["maxMassFraction"], sampleCount=spec["samples"], seed=spec["seed"])
    ref = scenes.tree_grid(m, spec)
    assert dev.ncells == ref.ncells and dev.nnodes == ref.nnodes, (dev.ncells, ref.ncells)
    assert dev.ncells > (2_500_000 if spec["gtype"] == A.GRID_OCTREE else 3_000_000)
    for a in ("node_box", "node_child", "node_father", "node_cell", "node_dir"):
        assert np.array_equal(getattr(dev, a), getattr(ref, a)), a
    # the leaves' neighbour lists equal the reference node classes' lists, in order
    cd, idd = _leaf_lists(dev)
    cr, idr = _leaf_lists(ref)
    assert np.array_equal(cd, cr) and np.array_equal(idd, idr)


def test_subdivision_with_the_reference_sampler_agrees_within_noise(orc):
    """Device tree against the oracle's subdivision with the reference's MT19937 sampler
    (maximum level 8, mass fraction 1e-5: ~3*10^5 leaves): the same leaves per level within
    4 sigma of the counting noise plus 0.5 %, and the total within 0.2 %."""
    m = scenes.octree_pan_model()
    dev = runtime.build_tree(m, A.GRID_OCTREE, EXT, minLevel=2, maxLevel=8, maxMassFraction=1e-5, sampleCount=100,
                             seed=4357)
    ref, _, lev = orc.tree_build(m, A.GRID_OCTREE, EXT, 2, 8, 1e-5, 100, 4357, sampler=0, neighbors=False)
    levels = lambda t: np.bincount(np.log2(
        (EXT[3] - EXT[0]) / (t.node_box.reshape(-1, 6)[t.node_cell >= 0, 3] - t.node_box.reshape(-1, 6)[t.node_cell >= 0, 0])
    ).round().astype(int), minlength=9)
    a, b = levels(dev), levels(ref)
    assert abs(dev.ncells / ref.ncells - 1) < 2e-3, (dev.ncells, ref.ncells)
    assert np.all(np.abs(a - b) <= 4 * np.sqrt(np.maximum(a, b)) + 5e-3 * np.maximum(a, b) + 2), (a, b)


def _expdisk_box_mass_fraction(hR, hz, a, zmax):
    """Fraction of an untruncated exponential disk's mass inside |x|,|y| <= a, |z| <= zmax:
    rho0 = 1/(4 pi hR^2 hz); the z integral is 2 hz (1 - e^(-zmax/hz)); the square is eight
    times the wedge 0 <= phi <= pi/4, R <= a/cos(phi), whose radial integral is
    hR^2 (1 - e^-u (1 + u)), u = a/(hR cos phi)."""
    from scipy.integrate import quad

    def wedge(phi):
        u = a / (hR * math.cos(phi))
        return hR * hR * (1.0 - math.exp(-u) * (1.0 + u))
    ixy = 8.0 * quad(wedge, 0.0, math.pi / 4, epsabs=0, epsrel=1e-13, limit=200)[0]
    iz = 2.0 * hz * -math.expm1(-zmax / hz)
    return ixy * iz / (4.0 * math.pi * hR * hR * hz)


def _density_checks(d, o1, o2, vol, groups, mass_exact):
    """d: device densities; o1, o2: two oracle runs; groups: group index per cell."""
    diff, noise = d - o1, o2 - o1
    ng = groups.max() + 1
    num = np.bincount(groups, diff, ng)
    den = np.sqrt(np.bincount(groups, noise ** 2, ng))
    ok = den > 0
    z = num[ok] / den[ok]
    assert np.max(np.abs(z)) < 4.5, np.max(np.abs(z))
    ratio = (diff ** 2).sum() / (noise ** 2).sum()
    assert 0.9 < ratio < 1.1, ratio
    # total mass: sum of density x volume, against the analytic mass in the box
    sig = math.sqrt(float(((vol * noise) ** 2).sum()) / 2.0)
    for est in (d, o1):
        zm = ((est * vol).sum() - mass_exact) / sig
        assert abs(zm) < 5, zm
    assert sig / mass_exact < 1e-3


def test_cartesian_density_sampling_matches_oracle(orc):
    m = models.oligo_disk()                      # configuration 1: 100x100x50 cells over 40x40x4 kpc
    m.rho = None
    ctx = runtime.Context(m)
    d = ctx.density()[0]
    ctx.close()
    o1 = orc.sample_density(m, seed=1000)[0]
    o2 = orc.sample_density(m, seed=2000)[0]
    g = m.dustGrid
    vol = (np.diff(g.xv)[:, None, None] * np.diff(g.yv)[None, :, None] * np.diff(g.zv)[None, None, :]).reshape(-1)
    slabs = np.arange(d.size) // (g.pointsY * g.pointsZ)  # cells of one x index (m = k + nz j + nz ny i)
    dc = m.dustComps[0]
    frac = _expdisk_box_mass_fraction(dc.geometry.radialScale, dc.geometry.axialScale, 20 * KPC, 2 * KPC)
    _density_checks(d, o1, o2, vol, slabs, dc.norm * frac)


def test_tree_density_sampling_matches_oracle(orc):
    m = scenes.octree_pan_model()
    m.dustGrid = runtime.build_tree(m, A.GRID_OCTREE, EXT, minLevel=2, maxLevel=8, maxMassFraction=1e-5)
    m.rho = None
    ctx = runtime.Context(m)
    d = ctx.density()[0]
    ctx.close()
    o1 = orc.sample_density(m, seed=3000)[0]
    o2 = orc.sample_density(m, seed=4000)[0]
    b = m.dustGrid.node_box.reshape(-1, 6)[m.dustGrid.node_cell >= 0]
    b = b[np.argsort(m.dustGrid.node_cell[m.dustGrid.node_cell >= 0])]
    vol = np.prod(b[:, 3:] - b[:, :3], axis=1)
    c = 0.5 * (b[:, :3] + b[:, 3:])
    groups = np.clip((np.hypot(c[:, 0], c[:, 1]) / (20 * KPC) * 40).astype(int), 0, 39)   # 40 radial rings
    dc = m.dustComps[0]
    frac = _expdisk_box_mass_fraction(dc.geometry.radialScale, dc.geometry.axialScale, 20 * KPC, 2 * KPC)
    _density_checks(d, o1, o2, vol, groups, dc.norm * frac)
