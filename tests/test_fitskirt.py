"""FitSKIRT pieces that need no GPU: the PSF kernel and convolution against the reference's nested
loop (Convolution.cpp:80-100, GaussianKernel.cpp:18-45), the luminosity fits on images with known
luminosities (GoldenSection.cpp:83-122, LumSimplex.cpp:272-330), and the genetic operators."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from skirt7_b200 import fitskirt as F


def _nested_loop(image, kernel):
    """Convolution::nested_loop restated pixel by pixel (the checker for the FFT version)."""
    ny, nx = image.shape
    ky, kx = kernel.shape
    out = np.zeros_like(image)
    for yi in range(ny):
        for xi in range(nx):
            sx, sy = xi - (kx - 1) // 2, yi - (ky - 1) // 2
            for yk in range(ky):
                for xk in range(kx):
                    if 0 <= sx + xk < nx and 0 <= sy + yk < ny:
                        out[sy + yk, sx + xk] += image[yi, xi] * kernel[yk, xk]
    return out


def test_gaussian_kernel_and_convolution():
    k = F.gaussian_kernel(3.0, 7)
    assert k.shape == (7, 7) and abs(k.sum() - 1) < 1e-12 and k[3, 3] == k.max()
    assert np.allclose(k, k.T) and np.allclose(k, k[::-1, ::-1])
    rng = np.random.default_rng(1)
    img = rng.random((13, 17))
    got = F.convolve(torch.tensor(img), k).numpy()
    assert np.allclose(got, _nested_loop(img, k), rtol=1e-12, atol=1e-14)
    # an asymmetric kernel fixes the orientation
    ka = rng.random((5, 3))
    assert np.allclose(F.convolve(torch.tensor(img), ka).numpy(), _nested_loop(img, ka), rtol=1e-12, atol=1e-14)


def test_luminosity_fits_recover_known_luminosities():
    rng = np.random.default_rng(2)
    f1 = torch.tensor(rng.random((20, 20)) + 0.1)
    f2 = torch.tensor(np.outer(np.hanning(20), np.hanning(20)) + 0.05)
    ref = 2.5 * f1
    ref[0, 0] = 0.0                                   # a masked pixel
    lum, chi = F.golden_section(ref, f1, 0.1, 10.0)
    # the reference's stopping rule ends the search once the best point repeats after 20
    # reductions (golden section reuses one interior point), so its precision is the interval
    # left then: 9.9 x 0.618^20 = 6.6e-4 at most
    assert abs(lum / 2.5 - 1) < 3e-4 and chi < 1e-5
    ref2 = 1.3 * f1 + 0.7 * f2
    lums, chi2 = F.simplex2(ref2, torch.stack([f1, f2]), [0.1, 0.1], [5.0, 5.0])
    assert np.allclose(lums, [1.3, 0.7], rtol=1e-3) and chi2 < 1e-5
    # bounds are respected: a best fit outside the box lands on its edge
    lums, _ = F.simplex2(ref2, torch.stack([f1, f2]), [0.1, 0.9], [5.0, 5.0])
    assert lums[1] >= 0.9 - 1e-12


def test_steady_state_ga_operators():
    opt = F.Optimization(popsize=16, generations=0, pmut=0.5, pcross=0.9, replacement=0.5, seed=3)
    ga = F.SteadyStateGA([0.0, -1.0], [1.0, 1.0], opt)
    pop = ga.initial()
    assert pop.shape == (16, 2) and np.all(pop >= ga.lo) and np.all(pop <= ga.hi)
    target = np.array([0.3, 0.2])
    score = lambda P: ((P - target) ** 2).sum(axis=1)
    s = score(pop)
    best = [s.min()]
    for _ in range(30):
        kids = ga.offspring(pop, s)
        assert len(kids) == 8 and np.all(kids >= ga.lo) and np.all(kids <= ga.hi)
        pop, s = ga.replace(pop, s, kids, score(kids))
        best.append(s.min())
    assert all(b2 <= b1 for b1, b2 in zip(best, best[1:]))      # the best member is never lost
    assert best[-1] < 0.2 * best[0]
