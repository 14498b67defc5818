"""FitSKIRT on the device: candidates simulated together in one batched launch with one frame per
stellar component, PSF convolution and luminosity fits on the device, the genetic algorithm over
the geometric parameters (OligoFitScheme.cpp:117-149, Optimization.cpp:26-187)."""
import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import fitskirt as F
from skirt7_b200 import models, runtime
from skirt7_b200.scene import DEG, KPC

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def _build(p):
    hRd, tau = p
    m = models.oligo_disk(N=(32, 32, 16), npix=64, tauV=tau, hRd=hRd, inclination=85 * DEG, with_sed=False,
                          write_absorption=False)
    m.instruments[0].writeStellarComps = True
    return m


def test_fit_scheme_prefers_the_truth_and_never_loses_its_best():
    truth = (6 * KPC, 1.0)
    ctx = runtime.Context(_build(truth))
    ctx.run_phase(A.PHASE_STELLAR, [0], 1000000, 0, 1000000, seed=99)
    cube, _ = ctx.read_instrument(0)
    ctx.close()
    assert cube.shape[0] == 3
    kern = F.gaussian_kernel(2.0, 7)
    # the "observed" image: both components at luminosity factor 1, seen through the PSF
    ref = F.convolve(torch.tensor(cube[1, 0] + cube[2, 0]), kern).numpy()
    img = F.ReferenceImage(ref, kern, [0.2, 0.2], [5.0, 5.0])
    scheme = F.OligoFitScheme(build=_build, lo=[3 * KPC, 0.2], hi=[9 * KPC, 4.0], images=[img],
                              optim=F.Optimization(popsize=8, generations=3, replacement=0.5, seed=5),
                              packets=100000)
    scores, lums = scheme.evaluate([truth, (3 * KPC, 3.5), (9 * KPC, 0.3)], seed=1)
    assert scores[0] < scores[1] and scores[0] < scores[2], scores
    # the truth's luminosity factors come back to within the Monte Carlo noise of 10^5 packets
    assert np.allclose(lums[0][0], [1.0, 1.0], rtol=0.15), lums[0]
    best, chi, bl = scheme.run()
    h = scheme.history
    assert len(h) == 4 and all(b <= a for a, b in zip(h, h[1:])), h
    assert np.all(best >= np.array(scheme.lo)) and np.all(best <= np.array(scheme.hi))
    assert chi == h[-1] and len(bl) == 1 and len(bl[0]) == 2
