"""The device's stellar emission phase against the oracle's restated life cycle
(MonteCarloSimulation.cpp:259-543) on the configurations' own grids, through committed fixtures
(tests/golden/tracer_<scene>.npz, written by tests/golden/make_tracer_fixtures.py on the same
deterministic scenes, tests/golden/scenes.py):

  * configuration 2's octree (2,986,747 leaves) with its panchromatic disk, three 512x512 frames
    at 0/60/88 degrees, at 0.21, 0.65 and 2.9 micron;
  * configuration 5's k-d tree (4,243,844 leaves) with the central point source, a 512x512 frame
    at 60 degrees and the absorbed luminosity per cell, at 0.25, 1.0 and 6.4 micron;
  * configuration 3's clumpy disk (tau_V 5, 10^4 clumps) on a 10^6-site Voronoi grid, a 300x300
    frame at 88 degrees.

The tolerances are the parity target's: every frame's 32x32-pixel blocks and every group of cells within
3 sigma of the combined Monte Carlo noise (z of the batch means: at most 1 % of the elements plus
two beyond 3 sigma, none beyond 5), and the total flux of every frame at every wavelength within
0.3 % (the fixtures' standard errors are about 0.1 % or less, so 0.3 % is resolved), with
|z| < 4.  The production FP32 geometry is compared; on the octree the FP32 total flux is also
compared with the FP64 walk's on the same packets: within 0.1 %."""
import json
import os
import sys

import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import runtime

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
import scenes  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


def fixture(name):
    return np.load(os.path.join(GOLDEN, "tracer_%s.npz" % name))


def device_scene(name, fx):
    """The scene of the fixture, its grid built on the device (identical to the oracle's)."""
    sig = json.loads(str(fx["signature"]))
    if name == "voronoi_clumpy":
        full = scenes.voronoi_clumpy_model()
        full.dustGrid = runtime.build_voronoi(scenes.voronoi_sites(), scenes.EXT)
        assert scenes.voronoi_signature(full.dustGrid) == sig, "the device tessellation is not the fixture's"
        ells = [0]
    else:
        spec = scenes.OCTREE if name == "octree_pan" else scenes.KDTREE
        full = scenes.octree_pan_model() if name == "octree_pan" else scenes.kdtree_point_model()
        full.dustGrid = runtime.build_tree(full, spec["gtype"], scenes.EXT, minLevel=spec["minLevel"],
                                           maxLevel=spec["maxLevel"], maxMassFraction=spec["maxMassFraction"],
                                           sampleCount=spec["samples"], seed=spec["seed"])
        assert scenes.tree_hash(full.dustGrid) == sig["tree_hash"], "the device tree is not the fixture's"
        ells = list(fx["ells"])
    m = scenes.wavelength_subset(full, ells)
    m.rho = scenes.centre_density(m)
    return m


def device_stats(ctx, m, e, packets, B, precision=A.PREC_FP32, seed0=1):
    frames = [i for i, ins in enumerate(m.instruments) if ins.type != 0]
    npp = int(packets / B)
    tot, blk, lab, labt = [], [], [], []
    for b in range(B):
        ctx.reset_tallies()
        ctx.run_phase(A.PHASE_STELLAR, [e], npp, 0, npp, seed=seed0 + 1000 * b + e, precision=precision)
        ctx.sync()
        cubes = [ctx.read_instrument(i)[0][0, e] for i in frames]
        tot.append([c.sum() for c in cubes])
        blk.append([scenes.block_sums(c) for c in cubes])
        if m.writeAbsorption:
            la = ctx.read_absorption()[0][:, e:e + 1]
            lab.append(scenes.labs_groups(m.dustGrid, la)[:, 0])
            labt.append(la.sum())
        assert ctx.counters()["errors"] == 0
    out = {}
    for key, val in (("tot", tot), ("blk", blk), ("lab", lab), ("labtot", labt)):
        if len(val):
            x = np.asarray(val)
            out[key] = (x.mean(0), x.std(0, ddof=1) / np.sqrt(B))
    return out


def zcheck(what, mg, sg, mo, so, keep=None):
    s = np.sqrt(sg ** 2 + so ** 2)
    ok = s > 0
    if keep is not None:
        ok &= keep
    z = np.abs((mg - mo)[ok] / s[ok])
    assert z.size > 0, what
    assert z.max() < 5, "%s: max |z| %.2f" % (what, z.max())
    n3 = int((z > 3).sum())
    assert n3 <= 0.01 * z.size + 2, "%s: %d of %d beyond 3 sigma" % (what, n3, z.size)
    return z


def compare(name, fx, G, e):
    # total flux of every frame
    mo, so = fx["tot_mean_%d" % e], fx["tot_sem_%d" % e]
    mg, sg = G["tot"]
    rel = mg / mo - 1
    z = (mg - mo) / np.sqrt(sg ** 2 + so ** 2)
    print("%s ell %d: total flux device/oracle - 1 = %s, z = %s, oracle standard error %s" %
          (name, int(fx["ells"][e]), np.array2string(rel, precision=5), np.array2string(z, precision=2),
           np.array2string(so / mo, precision=5)))
    assert np.all(so / mo < 1.5e-3), "fixture too noisy to resolve 0.3 %"
    assert np.all(np.abs(rel) < 3e-3), "%s ell %d: total flux off by %s" % (name, e, rel)
    assert np.all(np.abs(z) < 4), "%s ell %d: total flux z %s" % (name, e, z)
    # blocks of every frame that hold at least 0.1 % of the frame's flux
    mo, so = fx["blk_mean_%d" % e], fx["blk_sem_%d" % e]
    mg, sg = G["blk"]
    keep = mo > 1e-3 * mo.sum(axis=(-2, -1), keepdims=True)
    zcheck("%s ell %d blocks" % (name, e), mg, sg, mo, so, keep)
    if "lab" in G:
        mo, so = fx["lab_mean_%d" % e], fx["lab_sem_%d" % e]
        mg, sg = G["lab"]
        zcheck("%s ell %d absorbed luminosity groups" % (name, e), mg, sg, mo, so, mo > 1e-3 * mo.sum())
        mo, so = fx["labtot_mean_%d" % e], fx["labtot_sem_%d" % e]
        mg, sg = G["labtot"]
        assert abs(mg / mo - 1) < 3e-3 and abs((mg - mo) / np.hypot(sg, so)) < 4, (mg / mo - 1)


# packets per wavelength on the device: ten times the fixture's, so the combined noise is the
# oracle's to within 5 %
@pytest.mark.parametrize("name", ["octree_pan", "kdtree_point", "voronoi_clumpy"])
def test_stellar_phase_matches_oracle_fixture(name):
    fx = fixture(name)
    m = device_scene(name, fx)
    ctx = runtime.Context(m)
    for e in range(len(fx["ells"])):
        G = device_stats(ctx, m, e, 10 * float(fx["packets"][e]), 10)
        compare(name, fx, G, e)
    ctx.close()


def test_octree_fp32_total_flux_against_fp64():
    """The same packets (random streams keyed by packet) with the FP32 and the FP64 walk on
    configuration 2's octree: every frame's total flux at every wavelength within 0.1 %."""
    fx = fixture("octree_pan")
    m = device_scene("octree_pan", fx)
    ctx = runtime.Context(m)
    for e in range(len(fx["ells"])):
        t = {}
        for prec in (A.PREC_FP32, A.PREC_FP64):
            G = device_stats(ctx, m, e, 4e6, 2, precision=prec, seed0=77)
            t[prec] = G["tot"][0]
        rel = t[A.PREC_FP32] / t[A.PREC_FP64] - 1
        print("octree cfg2 ell %d: FP32/FP64 total flux - 1 = %s" % (int(fx["ells"][e]), rel))
        assert np.all(np.abs(rel) < 1e-3), rel
    ctx.close()
