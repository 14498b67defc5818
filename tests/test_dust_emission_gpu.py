"""Panchromatic dust emission on the device against the oracle: the stellar phase storing absorbed
luminosities, one dust self-absorption cycle and the dust emission phase with peel-off
(PanMonteCarloSimulation.cpp:106-346), with grey-body equilibrium temperatures
(DustMix.cpp:674-697, GreyBodyDustEmissivity.cpp:21-45).  Frames at far-infrared wavelengths, the
absorbed luminosities and the temperatures agree within the combined Monte Carlo noise."""
import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import models, runtime
from skirt7_b200.scene import KPC, MICRON, CartesianDustGrid

from helpers import block_sum, cell_center_density, zscores

pytestmark = pytest.mark.gpu


def pan_model():
    m = models.pan_disk(nlambda=16, lmin=0.1 * MICRON, lmax=1000 * MICRON, inclinations=(60,), npix=40,
                        dust_emission=True, tauV=2.0)
    m.dustGrid = CartesianDustGrid(-20 * KPC, 20 * KPC, -20 * KPC, 20 * KPC, -2 * KPC, 2 * KPC, 20, 20, 10)
    m.rho = cell_center_density(m)
    return m


def gpu_run(m, npp, seed):
    ctx = runtime.Context(m)
    nl = ctx.nlambda
    ells = np.arange(nl)
    ctx.run_phase(A.PHASE_STELLAR, ells, npp, 0, npp, seed=seed)
    ctx.sync()
    ctx.calc_dust_emission()
    ctx.reset_dust_absorption()
    ctx.run_phase(A.PHASE_DUST_SELFABS, ells, npp, 0, npp, seed=seed + 1)
    ctx.sync()
    T = ctx.calc_dust_emission()
    ctx.run_phase(A.PHASE_DUST_EMISSION, ells, npp, 0, npp, seed=seed + 2)
    ctx.sync()
    cube, sed = ctx.read_instrument(0)
    ls, ld = ctx.read_absorption()
    c = ctx.counters()
    ctx.close()
    return dict(cube=cube[0], ls=ls, ld=ld, T=T, c=c)


def test_dust_emission_matches_oracle(orc):
    m = pan_model()
    # Both sides run the same packets per wavelength: the temperatures, hence the dust emission,
    # are a nonlinear function of the noisy absorbed luminosities, so batches of different sizes
    # have different expectations (with 10x more packets on one side the 1-14 micron dust
    # self-absorption differed by up to 90 % and the mean cell temperature by 1.3 %; with equal
    # sizes they agree to 0.1 %).
    G = [gpu_run(m, 4000, 100 + 10 * b) for b in range(24)]
    O = []
    for b in range(12):
        r = orc.simulate(m, 4000, nthreads=8, seed=500 + b, selfabs_cycles=1, dust_emission_phase=True)
        O.append(dict(cube=r["cubes"][0][0], ls=r["labs_stel"], ld=r["labs_dust"], T=r["T"]))
    assert all(g["c"]["errors"] == 0 for g in G)
    # stellar absorption per wavelength (summed over cells) and dust self-absorption.  The standard
    # errors come from 24 and 12 batches (about 20 degrees of freedom, heavier tails than a normal
    # z), and the oracle batches carry a few percent of noise each: bound the largest of the 16
    # |z| by 5 and their median by 1.5
    z, ok = zscores([g["ls"].sum(0) for g in G], [o["ls"].sum(0) for o in O])
    assert np.max(np.abs(z[ok])) < 5.0 and np.median(np.abs(z[ok])) < 1.5, z
    z, ok = zscores([g["ld"].sum() for g in G], [o["ld"].sum() for o in O])
    assert abs(float(z)) < 4.0, z
    # equilibrium temperatures of the cells holding most of the dust
    rho = m.rho[0]
    big = rho > np.percentile(rho, 90)
    Tg = np.mean([g["T"][big] for g in G], 0)
    To = np.mean([o["T"][big] for o in O], 0)
    assert np.all(Tg > 3) and np.all(To > 3)
    assert abs(np.median(Tg / To) - 1) < 0.02, np.median(Tg / To)
    # frames: the far-infrared (dust-emission dominated) wavelengths, 8x8 blocks
    for ell in (11, 13):
        f = lambda r, e=ell: block_sum(r["cube"][e], 5)
        z, ok = zscores([f(g) for g in G], [f(o) for o in O])
        mean = np.mean([f(o) for o in O], 0)
        ok &= mean > 2e-3 * mean.sum()
        zz = np.abs(z[ok])
        assert zz.max() < 5.0 and np.sum(zz > 3) <= max(1, 0.05 * zz.size), (ell, np.sort(zz)[-5:])
