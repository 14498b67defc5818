"""Dust self-absorption (PanMonteCarloSimulation::rundustselfabsorption, :106-187) through the
library's MonteCarloSimulation driver -- three stages with 1/10, 1/3 and 1 times the packages, a
fixed cycle count per stage, dust emission spectra recomputed before every cycle -- followed by the
dust emission phase, against the oracle's restatement of the same schedule.  Both sides run the
same packets per wavelength (the temperatures are a nonlinear function of the noisy absorbed
luminosities).  The absorbed dust luminosity, the temperatures of the dense cells and the
far-infrared frames agree within the combined Monte Carlo noise; the logged cycles show the
absorbed dust luminosity of every cycle."""
import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import runtime

from helpers import block_sum, zscores
from test_dust_emission_gpu import pan_model

pytestmark = pytest.mark.gpu
NPP = 4000


def gpu_run(m, seed):
    sim = runtime.MonteCarloSimulation(m, NPP, seed=seed, selfAbsorption=True, cycles=1).run()
    ctx = sim.ctx
    cube, _ = ctx.read_instrument(0)
    ls, ld = ctx.read_absorption()
    T = ctx.calc_dust_emission()
    out = dict(cube=cube[0], ls=ls, ld=ld, T=T, c=ctx.counters(), log=sim.selfabs_log)
    ctx.close()
    return out


def test_staged_self_absorption_matches_oracle(orc):
    m = pan_model()
    G = [gpu_run(m, 300 + 17 * b) for b in range(24)]
    assert all(len(g["log"]) == 3 for g in G)                 # one cycle in each of the three stages
    assert all(g["c"]["errors"] == 0 for g in G)
    O = []
    for b in range(12):
        r = orc.simulate(m, NPP, nthreads=8, seed=9000 + 101 * b, selfabs_cycles=1, selfabs_staged=True,
                         dust_emission_phase=True)
        O.append(dict(cube=r["cubes"][0][0], ls=r["labs_stel"], ld=r["labs_dust"], T=r["T"]))
    # absorbed dust luminosity after the last self-absorption cycle, in total and per wavelength
    z, ok = zscores([g["ld"].sum() for g in G], [o["ld"].sum() for o in O])
    assert abs(float(z)) < 4.0, z
    z, ok = zscores([g["ld"].sum(0) for g in G], [o["ld"].sum(0) for o in O])
    assert np.max(np.abs(z[ok])) < 5.0 and np.median(np.abs(z[ok])) < 1.5, z
    # temperatures of the cells holding most of the dust (the spectra of the dust emission phase)
    rho = m.rho[0]
    big = rho > np.percentile(rho, 90)
    Tg = np.mean([g["T"][big] for g in G], 0)
    To = np.mean([o["T"][big] for o in O], 0)
    assert abs(np.median(Tg / To) - 1) < 0.02, np.median(Tg / To)
    # far-infrared frames
    for ell in (11, 13):
        f = lambda r, e=ell: block_sum(r["cube"][e], 5)
        z, ok = zscores([f(g) for g in G], [f(o) for o in O])
        mean = np.mean([f(o) for o in O], 0)
        ok &= mean > 2e-3 * mean.sum()
        zz = np.abs(z[ok])
        assert zz.max() < 5.0 and np.sum(zz > 3) <= max(1, 0.05 * zz.size), (ell, np.sort(zz)[-5:])
