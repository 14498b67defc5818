"""The synthetic disk-galaxy workloads (stars: exponential disk + Sersic bulge; dust: exponential
disk), in the classes of skirt7_b200.scene.  Shapes, sizes and value ranges follow the
benchmark configurations: the oligochromatic Cartesian run, the panchromatic octree run, the
clumpy Voronoi run, the served fit variants and the dust-emission k-d tree run.

Luminosities: the reference scales oligochromatic luminosities by the solar SED read from
dat/SED/Sun/SunSED.dat (OligoStellarComp.cpp:39-75); that table is not shipped here, so the
solar spectrum is a 5772 K black body normalised to L_sun.  Only the absolute flux scale of
the outputs depends on it.
"""
import math

import numpy as np

from . import _abi as A
from .scene import (DEG, KPC, LSUN, MICRON, MPC, PC, CartesianDustGrid, ClumpyGeometryDecorator, DustComp,
                    DustMix, ExpDiskGeometry, FaceOnDustCompNormalization, FrameInstrument, LogWavelengthGrid,
                    OligoWavelengthGrid, PointGeometry, SceneModel, SEDInstrument, SersicGeometry, StellarComp)

H, CL, KB = 6.62606957e-34, 2.99792458e8, 1.3806488e-23
SIGMA_SB = 2 * math.pi ** 5 * KB ** 4 / (15 * CL ** 2 * H ** 3)


def planck(lam, T):
    """PlanckFunction (PlanckFunction.cpp:24-33), W/m2/m/sr."""
    x = H * CL / (lam * KB * T)
    return 2.0 * H * CL * CL / lam ** 5 / np.expm1(x)


def sun_Llambda(lam):
    """Solar monochromatic luminosity (W/m) as a 5772 K black body normalised to L_sun."""
    T = 5772.0
    return LSUN * math.pi * planck(np.asarray(lam), T) / (SIGMA_SB * T ** 4)


def synthetic_mix(lambdav, albedoV=0.6, gV=0.6, kappaV=2600.0):
    """A smooth interstellar-like dust mix: kappa_ext ~ lambda^-1.2 steepening to lambda^-2 in the
    far infrared, albedo and g peaking in the optical/UV.  At 0.55 micron it has the given
    albedo and g."""
    lam = np.asarray(lambdav, dtype=np.float64)
    x = lam / (0.55 * MICRON)
    ke = kappaV * x ** -1.2 / (1.0 + (lam / (10 * MICRON)) ** 0.8) * (1.0 + (0.55 / 10.0) ** 0.8)
    la = np.log(lam / (0.45 * MICRON))
    alb = 0.05 + (albedoV - 0.05) * np.exp(-la ** 2 / (2 * 1.3 ** 2)) / math.exp(-math.log(0.55 / 0.45) ** 2 / (2 * 1.3 ** 2))
    alb = np.clip(alb, 0.0, 0.95)
    lg = np.log(lam / (0.35 * MICRON))
    g = 0.1 + (gV - 0.1) * np.exp(-lg ** 2 / (2 * 1.6 ** 2)) / math.exp(-math.log(0.55 / 0.35) ** 2 / (2 * 1.6 ** 2))
    g = np.clip(g, 0.0, 0.9)
    return DustMix(ke, alb, g)


def _stars(wl, Ltot_sun=1e10, bulge_fraction=0.3, Tdisk=None, Tbulge=None, hR=4 * KPC, hz=0.35 * KPC,
           reff=1.5 * KPC, n=4.0):
    lam, dl = wl.lambdav, wl.dlambdav
    if Tdisk is None:
        # oligochromatic: luminosities in solar units times the solar SED times the bin width
        Ld = (1 - bulge_fraction) * Ltot_sun * sun_Llambda(lam) * dl
        Lb = bulge_fraction * Ltot_sun * sun_Llambda(lam) * dl
    else:
        def sed(T, Lbol):
            return Lbol * math.pi * planck(lam, T) / (SIGMA_SB * T ** 4) * dl
        Ld = sed(Tdisk, (1 - bulge_fraction) * Ltot_sun * LSUN)
        Lb = sed(Tbulge, bulge_fraction * Ltot_sun * LSUN)
    comps = [StellarComp(ExpDiskGeometry(hR, hz), Ld)]
    if bulge_fraction > 0:
        comps.append(StellarComp(SersicGeometry(n, reff), Lb))
    return comps


def oligo_disk(N=(100, 100, 50), packages=1e6, tauV=1.0, albedo=0.6, g=0.6, hRd=6 * KPC, hzd=0.25 * KPC,
               inclination=88 * DEG, npix=300, wavelengths=(0.55 * MICRON,), bulge_fraction=0.3,
               extent=(20 * KPC, 20 * KPC, 2 * KPC), with_sed=True, write_absorption=True,
               hR=4 * KPC, hz=0.35 * KPC):
    """Plain oligochromatic run: exponential stellar disk (h_R 4 kpc, h_z 0.35 kpc) plus a Sersic
    n=4 bulge (R_e 1.5 kpc, 30 % of the light); exponential dust disk (h_R 6 kpc, h_z 0.25 kpc)
    with face-on V optical depth 1, albedo 0.6, g 0.6 on a 100x100x50 Cartesian grid over
    40x40x4 kpc; a 300x300 frame at 88 degrees plus an SED instrument."""
    wl = OligoWavelengthGrid(list(wavelengths))
    nl = wl.Nlambda
    mix = DustMix(np.full(nl, KAPPA_V_DEFAULT), np.full(nl, albedo), np.full(nl, g))
    dgeom = ExpDiskGeometry(hRd, hzd)
    dust = DustComp(dgeom, mix, FaceOnDustCompNormalization(wl.lambdav[len(wl.lambdav) // 2], tauV))
    ex, ey, ez = extent
    grid = CartesianDustGrid(-ex, ex, -ey, ey, -ez, ez, *N)
    instr = [FrameInstrument(10 * MPC, inclination, npix, npix, 2 * ex, 2 * ex, instrumentName="frame")]
    if with_sed:
        instr.append(SEDInstrument(10 * MPC, inclination, instrumentName="sed"))
    return SceneModel(wl, _stars(wl, bulge_fraction=bulge_fraction, hR=hR, hz=hz), grid, [dust], instr,
                      writeAbsorption=write_absorption)


KAPPA_V_DEFAULT = 2600.0


def pan_disk(nlambda=50, lmin=0.1 * MICRON, lmax=10 * MICRON, tauV=1.0, inclinations=(0, 60, 88), npix=512,
             extent=(20 * KPC, 20 * KPC, 2 * KPC), point_fraction=0.0, dust_emission=False,
             write_absorption=False):
    """Panchromatic disk galaxy on a log wavelength grid with a synthetic dust mix; stellar SEDs
    are black bodies (disk 6000 K, bulge 4000 K, optional central point source 20000 K)."""
    wl = LogWavelengthGrid(lmin, lmax, nlambda)
    mix = synthetic_mix(wl.lambdav)
    dust = DustComp(ExpDiskGeometry(6 * KPC, 0.25 * KPC), mix, FaceOnDustCompNormalization(0.55 * MICRON, tauV))
    stars = _stars(wl, Ltot_sun=1e10 * (1 - point_fraction), Tdisk=6000.0, Tbulge=4000.0)
    if point_fraction > 0:
        T = 20000.0
        Lp = point_fraction * 1e10 * LSUN * math.pi * planck(wl.lambdav, T) / (SIGMA_SB * T ** 4) * wl.dlambdav
        stars.append(StellarComp(PointGeometry(), Lp))
    ex, ey, ez = extent
    instr = [FrameInstrument(10 * MPC, inc * DEG, npix, npix, 2 * ex, 2 * ex, instrumentName="i%02d" % inc)
             for inc in inclinations]
    return SceneModel(wl, stars, None, [dust], instr, dustEmission=dust_emission,
                      writeAbsorption=write_absorption)


def clumpy_disk(tauV=5.0, clumps=10000, sigma=50 * PC, fraction=0.25, seed=1234, wavelengths=(0.55 * MICRON,),
                npix=300, extent=(20 * KPC, 20 * KPC, 2 * KPC)):
    """Clumpy dust disk: 10^4 clumps holding 25 % of the dust mass.  The reference has cubic-spline
    and uniform clump kernels only (SKIRTcore/*SmoothingKernel*); a Gaussian of sigma 50 pc is
    stood in for by a cubic spline of support h = 2.5 sigma (the same half-mass radius to ~5 %)."""
    wl = OligoWavelengthGrid(list(wavelengths))
    nl = wl.Nlambda
    mix = DustMix(np.full(nl, KAPPA_V_DEFAULT), np.full(nl, 0.6), np.full(nl, 0.6))
    base = ExpDiskGeometry(6 * KPC, 0.25 * KPC)
    rng = np.random.default_rng(seed)
    cl = sample_expdisk(base, clumps, rng)
    geom = ClumpyGeometryDecorator(base, fraction, clumps, 2.5 * sigma, True, A.KERNEL_CUBICSPLINE, cl)
    dust = DustComp(geom, mix, FaceOnDustCompNormalization(wl.lambdav[0], tauV))
    ex, ey, ez = extent
    instr = [FrameInstrument(10 * MPC, 88 * DEG, npix, npix, 2 * ex, 2 * ex, instrumentName="frame")]
    return SceneModel(wl, _stars(wl), None, [dust], instr)


def sample_expdisk(geom: ExpDiskGeometry, n, rng):
    """Positions from an exponential disk: R from the Gamma(2) radial mass profile, phi uniform,
    z Laplace (the distributions ExpDiskGeometry::randomR/randomz sample, ExpDiskGeometry.cpp:133-161)."""
    R = geom.radialScale * rng.gamma(2.0, 1.0, n)
    phi = rng.uniform(0, 2 * math.pi, n)
    z = rng.laplace(0.0, geom.axialScale, n)
    return np.ascontiguousarray(np.stack([R * np.cos(phi), R * np.sin(phi), z], axis=1).reshape(-1))


def fit_variant(params, N, wavelengths=(0.45 * MICRON, 0.55 * MICRON, 0.65 * MICRON), npix=256):
    """One FitSKIRT-style parameter variant of the oligochromatic disk: dust h_R, h_z, tau_V,
    inclination and bulge fraction substituted (AdjustableSkirtSimulation.cpp:145-194)."""
    hR, hz, tau, inc, bf = params
    m = oligo_disk(N=(N, N, N), tauV=tau, hRd=hR, hzd=hz, inclination=inc, npix=npix, wavelengths=wavelengths,
                   bulge_fraction=bf, with_sed=False, write_absorption=False)
    return m
