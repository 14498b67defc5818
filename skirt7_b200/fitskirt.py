"""FitSKIRT on the device tracer: fits the free parameters of a model to reference images.

The reference's fit loop (FitSKIRTcore) is a genetic algorithm over the geometric parameters of a
ski file (OligoFitScheme, Optimization.cpp:26-187: GAlib's steady-state GA on a real genome with
uniform initialisation, Gaussian mutation, uniform crossover and sigma-truncation scaling).  Each
candidate is one simulation of the adjusted ski file (AdjustableSkirtSimulation::performWith) that
writes one frame per stellar component (MultiFrameInstrument::writeStellarComps); for every
reference image the component frames are convolved with the image's PSF (Convolution.cpp:70-100,
GaussianKernel.cpp:18-45) and the component luminosities are fitted to the image by minimising

    chi2 = sum over pixels with ref != 0 of (ref - sum_c L_c frame_c)^2 / (|ref| + sum_c L_c frame_c)

(GoldenSection.cpp:57-122 for one component, LumSimplex.cpp:97-330 for two); the candidate's
score is the sum of the images' minima (ReferenceImages::chi2).

Here the candidates of a generation are simulated together: every child of a generation is a
context of one batched launch (skg_batch_run), so the GA's evaluations overlap on the device the
way the serving loop's requests do; the convolutions and the luminosity fits run on the device
with torch.  The genetic operators are restated from their published definitions (below), not
from GAlib's code.
"""
import math
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from . import runtime


# ---------------------------------------------------------------------------------------------
# point spread function and convolution

def gaussian_kernel(fwhm, dimension):
    """GaussianKernel (GaussianKernel.cpp:18-45) normalised to unit sum
    (ConvolutionKernel.cpp:27): exp(-(X^2 + Y^2) / (2 sigma^2)), sigma = FWHM / 2.3548, pixel
    offsets X, Y from the kernel centre (dimension + 1) / 2."""
    if fwhm <= 0 or dimension <= 0:
        raise ValueError("FWHM and dimension must be positive")
    sigma = fwhm / 2.3548
    c = (dimension + 1) // 2
    off = c - np.arange(1, dimension + 1)
    k = np.exp(-(off[None, :] ** 2 + off[:, None] ** 2) / (2 * sigma * sigma))
    return k / k.sum()


def convolve(image, kernel):
    """Convolution::nested_loop (Convolution.cpp:80-100): each pixel spreads over the kernel
    footprint centred on it, contributions falling off the frame are dropped; computed as a
    zero-padded FFT convolution of the same result.  image: torch tensor [..., ny, nx]."""
    import torch
    ky, kx = kernel.shape
    ny, nx = image.shape[-2:]
    py, px = ny + ky - 1, nx + kx - 1
    k = torch.as_tensor(kernel, dtype=image.dtype, device=image.device)
    F = torch.fft.rfft2(image, s=(py, px)) * torch.fft.rfft2(k, s=(py, px))
    full = torch.fft.irfft2(F, s=(py, px))
    oy, ox = (ky - 1) // 2, (kx - 1) // 2
    return full[..., oy:oy + ny, ox:ox + nx]


# ---------------------------------------------------------------------------------------------
# luminosity fits

def chi2(ref, frames, lums):
    """The chi2 of GoldenSection::function / LumSimplex::function for component luminosities
    lums[..., c] (any leading batch shape) against ref; pixels where ref is 0 are masked."""
    import torch
    sim = torch.einsum("...c,cyx->...yx", lums, frames)
    mask = ref != 0
    sig2 = ref.abs() + sim
    r = torch.where(mask, (ref - sim) ** 2 / torch.where(mask, sig2, torch.ones_like(sig2)), torch.zeros_like(sim))
    return r.sum(dim=(-2, -1))


def golden_section(ref, frame, lmin, lmax):
    """GoldenSection::optimize (GoldenSection.cpp:83-122): the luminosity in [lmin, lmax] that
    minimises chi2 for one component; at most 300 interval reductions, stopping once the best
    value changes by at most 1e-8 relative after 20 of them.  Returns (lum, chi2)."""
    import torch
    G = 0.3819660113
    a0, b0 = float(lmin), float(lmax)
    frames = frame[None]
    lum, prev, chi = 1.0, 1.0, 1.0
    for j in range(300):
        d = (b0 - a0) * G
        a1, b1 = a0 + d, b0 - d
        c = chi2(ref, frames, torch.tensor([[a1], [b1]], dtype=ref.dtype, device=ref.device)).tolist()
        if c[0] < c[1]:
            b0, lum, chi = b1, a1, c[0]
        else:
            a0, lum, chi = a1, b1, c[1]
        if j >= 20 and abs(prev - lum) / max(abs(lum), 1e-300) <= 1e-8:
            break
        prev = lum
    return lum, chi


def simplex2(ref, frames, lo, hi, iters=200):
    """Two luminosities by the Nelder-Mead simplex (reflection 1, contraction 0.5, expansion 2,
    shrink 0.5: the coefficients LumSimplex::optimize uses, LumSimplex.cpp:272-330) on the box
    [lo, hi], the vertices kept inside it; stops when the vertices agree to 1e-6 of the box.
    Returns (lums, chi2)."""
    import torch
    lo = np.asarray(lo, dtype=float)
    hi = np.asarray(hi, dtype=float)
    span = hi - lo

    def f(P):
        P = np.clip(np.atleast_2d(P), lo, hi)
        return chi2(ref, frames, torch.tensor(P, dtype=ref.dtype, device=ref.device)).cpu().numpy()

    V = np.array([lo + 0.5 * span, lo + np.array([0.75, 0.5]) * span, lo + np.array([0.5, 0.75]) * span])
    FV = f(V)
    for _ in range(iters):
        o = np.argsort(FV)
        V, FV = V[o], FV[o]
        if np.all(np.abs(V - V[0]).sum(axis=0) <= 1e-6 * span):
            break
        c = V[:2].mean(axis=0)
        r = np.clip(c + (c - V[2]), lo, hi)
        fr = f(r)[0]
        if FV[0] <= fr < FV[1]:
            V[2], FV[2] = r, fr
        elif fr < FV[0]:
            e = np.clip(c + 2.0 * (c - V[2]), lo, hi)
            fe = f(e)[0]
            V[2], FV[2] = (e, fe) if fe < fr else (r, fr)
        else:
            k = np.clip(c + 0.5 * (V[2] - c), lo, hi)
            fk = f(k)[0]
            if fk < FV[2]:
                V[2], FV[2] = k, fk
            else:
                V[1:] = V[0] + 0.5 * (V[1:] - V[0])
                FV[1:] = f(V[1:])
    i = int(np.argmin(FV))
    return V[i], float(FV[i])


@dataclass
class ReferenceImage:
    """An observed image at one wavelength (ReferenceImage.cpp): its data, its PSF and the bounds
    of each stellar component's luminosity factor."""
    data: np.ndarray
    kernel: np.ndarray
    min_lum: list
    max_lum: list

    def fit(self, frames, device="cuda"):
        """Convolves the component frames [c, ny, nx] and fits their luminosities
        (ReferenceImage::chi2, ReferenceImage.cpp:95-140).  Returns (lums, chi2)."""
        import torch
        ref = torch.as_tensor(self.data, dtype=torch.float64, device=device)
        fr = convolve(torch.as_tensor(frames, dtype=torch.float64, device=device), self.kernel)
        if fr.shape[0] == 1:
            lum, c = golden_section(ref, fr[0], self.min_lum[0], self.max_lum[0])
            return [lum], c
        if fr.shape[0] == 2:
            lums, c = simplex2(ref, fr, self.min_lum, self.max_lum)
            return list(lums), c
        raise NotImplementedError("luminosity fits of more than two stellar components")


# ---------------------------------------------------------------------------------------------
# the genetic algorithm

@dataclass
class Optimization:
    """Steady-state GA settings (Optimization.cpp:26-80): population size, generations,
    mutation and crossover probabilities; `replacement` is the fraction of the population
    replaced by offspring each generation."""
    popsize: int = 20
    generations: int = 10
    pmut: float = 0.03
    pcross: float = 0.65
    replacement: float = 0.25
    seed: int = 4357


class SteadyStateGA:
    """A steady-state genetic algorithm on a real genome within bounds, minimising a score.

    Published operators: uniform random initialisation inside the bounds; sigma-truncation
    scaling (Goldberg 1989) of the raw scores, f' = max(0, (s_mean - s) + 2 sigma) for minimisation,
    with roulette-wheel selection on f'; uniform crossover (each gene from either parent with
    probability 1/2) applied with probability pcross; Gaussian mutation of each gene with
    probability pmut (a normal step of a tenth of the gene's range, kept inside the bounds); each
    generation the offspring replace the worst members of the population."""

    def __init__(self, lo, hi, opt: Optimization):
        self.lo = np.asarray(lo, dtype=float)
        self.hi = np.asarray(hi, dtype=float)
        self.opt = opt
        self.rng = np.random.default_rng(opt.seed)

    def initial(self):
        n = self.opt.popsize
        return self.lo + self.rng.random((n, len(self.lo))) * (self.hi - self.lo)

    def _select(self, scores, k):
        s = np.asarray(scores, dtype=float)
        f = np.maximum(0.0, (s.mean() - s) + 2.0 * s.std())
        if f.sum() <= 0:
            f = np.ones_like(s)
        return self.rng.choice(len(s), size=k, p=f / f.sum())

    def offspring(self, pop, scores):
        n = max(2, int(round(self.opt.replacement * len(pop))))
        kids = []
        while len(kids) < n:
            a, b = pop[self._select(scores, 2)]
            if self.rng.random() < self.opt.pcross:
                take = self.rng.random(len(a)) < 0.5
                c1, c2 = np.where(take, a, b), np.where(take, b, a)
            else:
                c1, c2 = a.copy(), b.copy()
            for c in (c1, c2):
                m = self.rng.random(len(c)) < self.opt.pmut
                c[m] += self.rng.normal(0.0, 0.1, m.sum()) * (self.hi - self.lo)[m]
                kids.append(np.clip(c, self.lo, self.hi))
        return np.array(kids[:n])

    @staticmethod
    def replace(pop, scores, kids, kid_scores):
        allp = np.concatenate([pop, kids])
        alls = np.concatenate([scores, kid_scores])
        keep = np.argsort(alls)[:len(pop)]
        return allp[keep], alls[keep]


# ---------------------------------------------------------------------------------------------
# the fit scheme

@dataclass
class OligoFitScheme:
    """OligoFitScheme (OligoFitScheme.cpp:117-149): a model builder that maps a parameter vector
    to a model whose first instrument is a frame writing one frame per stellar component at each of
    the reference images' wavelengths (the ski file with its [label:default] fields substituted,
    AdjustableSkirtSimulation.cpp:145-194), the parameter bounds, the reference images (one per
    wavelength), the GA settings and the packets per wavelength of each candidate."""
    build: object
    lo: list
    hi: list
    images: list
    optim: Optimization = field(default_factory=Optimization)
    packets: int = 100000
    device: int = 0
    history: list = field(default_factory=list)

    def simulate(self, params_list, seed):
        """Simulates the candidates together in one batched launch; returns each candidate's
        component frames [nimages][ncomp, ny, nx]."""
        ctxs = [runtime.Context(self.build(p), device=self.device) for p in params_list]
        try:
            batch = runtime.Batch(device=self.device, max_slots=max(len(ctxs), 1), max_items=max(len(ctxs), 1),
                                  max_ells=max(1, sum(c.nlambda for c in ctxs)))
            try:
                slices = [(c, list(range(c.nlambda)), self.packets, 0, self.packets, seed + 7919 * i)
                          for i, c in enumerate(ctxs)]
                batch.run(A.PHASE_STELLAR, slices)
                batch.sync()
            finally:
                batch.close()
            out = []
            for c in ctxs:
                cube, _ = c.read_instrument(0)
                if cube.shape[0] < 2:
                    raise ValueError("the fit instrument must write one frame per stellar component")
                out.append([cube[1:, e] for e in range(len(self.images))])
            return out
        finally:
            for c in ctxs:
                c.close()

    def score(self, frames_per_image):
        """ReferenceImages::chi2: the sum over the images of the fitted minimum, with the fitted
        luminosities."""
        total, lums = 0.0, []
        for img, fr in zip(self.images, frames_per_image):
            l, c = img.fit(fr)
            total += c
            lums.append(l)
        return total, lums

    def evaluate(self, params_list, seed):
        frames = self.simulate(params_list, seed)
        res = [self.score(f) for f in frames]
        return np.array([r[0] for r in res]), [r[1] for r in res]

    def run(self):
        """The GA: an initial population, then `generations` rounds of offspring evaluated
        together and put in place of the worst members.  Returns (best parameters, best chi2,
        best luminosities); `history` keeps the best chi2 after each generation."""
        ga = SteadyStateGA(self.lo, self.hi, self.optim)
        pop = ga.initial()
        scores, lums = self.evaluate(pop, seed=self.optim.seed)
        best = {tuple(p): l for p, l in zip(pop, lums)}
        self.history = [float(scores.min())]
        for gen in range(self.optim.generations):
            kids = ga.offspring(pop, scores)
            ks, kl = self.evaluate(kids, seed=self.optim.seed + 104729 * (gen + 1))
            best.update({tuple(p): l for p, l in zip(kids, kl)})
            pop, scores = ga.replace(pop, scores, kids, ks)
            self.history.append(float(scores[0]))
        i = int(np.argmin(scores))
        return pop[i], float(scores[i]), best[tuple(pop[i])]
