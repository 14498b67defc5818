"""The persistent tracer (stellar emission phase) against the oracle's restated life cycle
(MonteCarloSimulation.cpp:259-543): frames, SEDs, FullInstrument components and per-cell
absorbed luminosity agree within the combined Monte Carlo noise (batch standard errors),
for the FP32 production traversal and the FP64 one."""
import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import models, runtime
from skirt7_b200.scene import DEG, MPC, KPC, FullInstrument, SimpleInstrument, FrameInstrument

from helpers import block_sum, cell_center_density, zscores

pytestmark = pytest.mark.gpu


def small_model(N=(40, 40, 20), npix=60):
    m = models.oligo_disk(N=N, npix=npix)
    fov = 40 * KPC
    m.instruments.append(FullInstrument(scatteringLevels=3, distance=10 * MPC, inclination=30 * DEG, pixelsX=npix,
                                        pixelsY=npix, fieldOfViewX=fov, fieldOfViewY=fov, instrumentName="full"))
    m.instruments.append(SimpleInstrument(distance=10 * MPC, inclination=88 * DEG, pixelsX=npix, pixelsY=npix,
                                          fieldOfViewX=fov, fieldOfViewY=fov, instrumentName="simple"))
    m.rho = cell_center_density(m)
    return m


def gpu_batches(m, B, npp, precision):
    ctx = runtime.Context(m)
    out = []
    for b in range(B):
        ctx.reset_tallies()
        ctx.run_phase(A.PHASE_STELLAR, [0], npp, 0, npp, seed=1000 + b, precision=precision)
        ctx.sync()
        res = {"inst": [ctx.read_instrument(i) for i in range(len(m.instruments))]}
        res["labs"] = ctx.read_absorption()[0][:, 0]
        res["counters"] = ctx.counters()
        out.append(res)
    ctx.close()
    return out


def oracle_batches(orc, m, B, npp):
    out = []
    for b in range(B):
        r = orc.simulate(m, npp, nthreads=8, seed=77 + 13 * b)
        out.append({"inst": list(zip(r["cubes"], r["seds"])), "labs": r["labs_stel"][:, 0], "stats": r["stats"]})
    return out


def _well_sampled(zok, O, f):
    """Restricts a z-test to elements holding at least 0.2 % of the total: elements fed by a few
    rare high-weight packets per batch have skewed batch means and unreliable variances."""
    z, ok = zok
    mean = np.mean([f(o) for o in O], axis=0)
    return z, ok & (mean > 2e-3 * mean.sum())


def _check(z, ok, what, zmax=5.0, frac=0.03):
    """z of batch means (16 + 16 batches: Student-t tails, P(|z| > 3) about 0.5 %); the oracle's
    batches vary from run to run (its threads take chunks dynamically, as the reference's do), so
    the count beyond 3 sigma gets two elements of slack above frac of the elements tested."""
    zz = np.abs(z[ok])
    assert zz.size > 0, what
    assert zz.max() < zmax, "%s: max |z| = %.2f" % (what, zz.max())
    nbeyond = int(np.sum(zz > 3))
    assert nbeyond <= frac * zz.size + 2, "%s: %d of %d elements beyond 3 sigma" % (what, nbeyond, zz.size)


@pytest.mark.parametrize("precision", [A.PREC_FP32, A.PREC_FP64])
def test_stellar_phase_matches_oracle(orc, precision):
    m = small_model()
    G = gpu_batches(m, 16, 200000, precision)
    O = oracle_batches(orc, m, 16, 8000)
    # frame (instrument 0): 60x60 -> 10x10 blocks of 6x6 pixels
    ff = lambda r: block_sum(r["inst"][0][0][0, 0], 6)
    zf, ok = _well_sampled(zscores([ff(g) for g in G], [ff(o) for o in O]), O, ff)
    _check(zf, ok, "frame")
    # SED (instrument 1)
    zs, ok = zscores([g["inst"][1][1][0] for g in G], [o["inst"][1][1][0] for o in O])
    _check(zs, ok, "sed", frac=1.0)
    # FullInstrument: every component's SED and the total/direct/scattered frames
    zfs, ok = zscores([g["inst"][2][1][:, 0] for g in G], [o["inst"][2][1][:, 0] for o in O])
    _check(zfs, ok, "full sed components", frac=0.2)
    for c in (A.FULL_TOT, A.FULL_TRA, A.FULL_STRDIR, A.FULL_STRSCA):
        fc = lambda r, c=c: block_sum(r["inst"][2][0][c, 0], 6)
        z, ok = _well_sampled(zscores([fc(g) for g in G], [fc(o) for o in O]), O, fc)
        _check(z, ok, "full frame component %d" % c)
    # SimpleInstrument shares the 88-degree direction group with the frame: the same frame up to
    # the summation order of the FP64 atomics
    for g in G:
        assert np.allclose(g["inst"][3][0][0, 0], g["inst"][0][0][0, 0], rtol=1e-12, atol=0)
    # absorbed luminosity per cell, summed over slabs of constant x index (40 slabs)
    nx = 40
    fl = lambda r: r["labs"].reshape(nx, -1).sum(1)
    zl, ok = _well_sampled(zscores([fl(g) for g in G], [fl(o) for o in O]), O, fl)
    _check(zl, ok, "absorbed luminosity")
    # total flux of the frame and absorbed luminosity agree within 3 combined sigma
    for key, gf, of in (("frame", lambda g: g["inst"][0][0].sum(), lambda o: o["inst"][0][0].sum()),
                        ("labs", lambda g: g["labs"].sum(), lambda o: o["labs"].sum())):
        z, ok = zscores([gf(g) for g in G], [of(o) for o in O])
        assert abs(float(z)) < 3.5, (key, float(z))
    c = G[0]["counters"]
    assert c["packets"] == 200000 and c["errors"] == 0
    assert c["steps"] > 0 and c["scatterings"] > 0


def test_transparent_flux_and_energy_budget():
    """FullInstrument's transparent flux sums the launch luminosities (FullInstrument.cpp:120-124):
    it estimates the emitted luminosity without dust; the scattered + direct + absorbed
    luminosity cannot exceed the emitted one."""
    m = small_model()
    ctx = runtime.Context(m)
    npp = 400000
    ctx.run_phase(A.PHASE_STELLAR, [0], npp, 0, npp, seed=9)
    ctx.sync()
    cube, sed = ctx.read_instrument(2)
    Lem = sum(s.luminosities[0] for s in m.stellarComps)
    tra = sed[A.FULL_TRA, 0]
    assert abs(tra / Lem - 1) < 0.01, tra / Lem
    labs = ctx.read_absorption()[0].sum()
    assert 0 < labs < Lem
    ctx.close()


@pytest.mark.parametrize("gtype", [A.GRID_OCTREE, A.GRID_BINTREE])
def test_fp32_geometry_total_flux_against_fp64(gtype):
    """The production FP32 tree walk (lattice records) against the FP64 walk on a panchromatic disk
    with a tree grid, with the same packets (each packet's random stream is keyed by its index, so
    the two runs differ by geometry precision alone): the total flux of every frame at every
    wavelength within 0.1 %, and the frames pixel by pixel within the Monte Carlo noise of a run."""
    from skirt7_b200.scene import KPC as _K
    m = models.pan_disk(nlambda=8, inclinations=(0, 60, 88), npix=64)
    ext = (-20 * _K, -20 * _K, -2 * _K, 20 * _K, 20 * _K, 2 * _K)
    if gtype == A.GRID_OCTREE:
        m.dustGrid = runtime.build_tree(m, gtype, ext, minLevel=2, maxLevel=7, maxMassFraction=1e-4)
    else:
        m.dustGrid = runtime.build_tree(m, gtype, ext, minLevel=6, maxLevel=21, maxMassFraction=1e-4)
    assert m.dustGrid.ncells > 2000
    ctx = runtime.Context(m)
    out = {}
    for prec in (A.PREC_FP32, A.PREC_FP64):
        ctx.reset_tallies()
        ctx.run_phase(A.PHASE_STELLAR, list(range(8)), 100000, 0, 100000, seed=31, precision=prec)
        ctx.sync()
        out[prec] = [ctx.read_instrument(i)[0][0] for i in range(3)]
        assert ctx.counters()["errors"] == 0
    for f32, f64 in zip(out[A.PREC_FP32], out[A.PREC_FP64]):
        t32, t64 = f32.sum(axis=(1, 2)), f64.sum(axis=(1, 2))
        assert np.all(np.abs(t32 / t64 - 1) < 1e-3), t32 / t64
        # 8x8-pixel blocks: paired runs differ far less than independent ones
        b32 = np.array([block_sum(f32[e], 8) for e in range(8)])
        b64 = np.array([block_sum(f64[e], 8) for e in range(8)])
        big = b64 > 1e-3 * b64.sum(axis=(1, 2), keepdims=True)
        assert np.median(np.abs(b32[big] / b64[big] - 1)) < 1e-3
    ctx.close()


def test_frames_per_stellar_component(orc):
    """A frame instrument that also writes one frame per stellar component (the frames FitSKIRT
    fits, MultiFrameInstrument::writeStellarComps): the component frames add up to the total frame
    (every stellar packet comes from one component) and each agrees with the oracle's."""
    m = models.oligo_disk(N=(40, 40, 20), npix=60)
    fov = 40 * KPC
    m.instruments = [FrameInstrument(distance=10 * MPC, inclination=80 * DEG, pixelsX=60, pixelsY=60,
                                     fieldOfViewX=fov, fieldOfViewY=fov, instrumentName="comps",
                                     writeStellarComps=True)]
    m.rho = cell_center_density(m)
    assert len(m.stellarComps) == 2
    G = gpu_batches(m, 12, 200000, A.PREC_FP32)
    O = oracle_batches(orc, m, 12, 8000)
    for g in G:
        cube = g["inst"][0][0]
        assert cube.shape[0] == 3
        assert np.allclose(cube[1] + cube[2], cube[0], rtol=1e-10, atol=1e-12 * cube[0].max())
        assert cube[1].sum() > 0 and cube[2].sum() > 0
    for c in (1, 2):
        fc = lambda r, c=c: block_sum(r["inst"][0][0][c, 0], 6)
        z, ok = _well_sampled(zscores([fc(g) for g in G], [fc(o) for o in O]), O, fc)
        _check(z, ok, "stellar component frame %d" % c)
