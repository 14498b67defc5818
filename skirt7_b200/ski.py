"""Reading ski files: SKIRT7's XML simulation descriptions, run unchanged on the device.

A ski file is the XML serialisation of a SimulationItem hierarchy (Discover/XmlHierarchyCreator.cpp):
the root element `skirt-simulation-hierarchy` holds one element named after the simulation class;
an item's scalar properties are XML attributes ("4 kpc", "88 deg", "1e6", "yes"), and each compound
property is a child element named after the property whose children are the item(s) it holds,
named after their classes.  Physical values carry an optional unit; without one they are in the
default unit of the simulation's units system (ExtragalacticUnits unless the ski file names another;
SKIRTcore/Units.cpp:50-181, ExtragalacticUnits.cpp, StellarUnits.cpp, SIUnits.cpp).

This module builds the hot path's host items (skirt7_b200.scene) from such a file, with the
reference's property names and defaults (the Q_CLASSINFO blocks of the reference headers), and
`SkiSimulation.run()` drives the phases of OligoMonteCarloSimulation::runSelf or
PanMonteCarloSimulation::runSelf on the device.  Classes outside the hot path's scope raise
SkiError naming the class.  Items that read the reference's resource tables (dat/DustMix, dat/SED)
need the directory of those tables (`resources=`), as the reference does through FilePaths::resource.
"""
import math
import os
import xml.etree.ElementTree as ET
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .scene import (LSUN, MICRON, CartesianDustGrid, ClumpyGeometryDecorator, DustComp, DustMix,
                    ExpDiskGeometry, FaceOnDustCompNormalization, FrameInstrument, LogWavelengthGrid,
                    OligoWavelengthGrid, PlummerGeometry, PointGeometry, SceneModel, SEDInstrument, SersicGeometry,
                    StellarComp, FullInstrument, SimpleInstrument)


class SkiError(ValueError):
    """A ski file that cannot be run (the reference raises FatalError at the same points)."""


# ---------------------------------------------------------------------------------------------
# units (SKIRTcore/Units.cpp:17-181)

_PC = 3.08567758e16
_AU = 1.49597871e11
_MSUN = 1.9891e30
_LSUN = 3.839e26
_ARCSEC = math.pi / (180.0 * 3600.0)

_FACTORS = {
    "length": {"m": 1.0, "cm": 1e-2, "km": 1e3, "AU": _AU, "pc": _PC, "kpc": 1e3 * _PC, "Mpc": 1e6 * _PC},
    "distance": {"m": 1.0, "cm": 1e-2, "km": 1e3, "AU": _AU, "pc": _PC, "kpc": 1e3 * _PC, "Mpc": 1e6 * _PC},
    "wavelength": {"m": 1.0, "cm": 1e-2, "mm": 1e-3, "micron": 1e-6, "nm": 1e-9, "A": 1e-10},
    "mass": {"kg": 1.0, "g": 1e-3, "Msun": _MSUN},
    "opacity": {"m2/kg": 1.0},
    "bolluminosity": {"W": 1.0, "Lsun": _LSUN},
    "monluminosity": {"W/m": 1.0, "W/micron": 1e6, "Lsun/micron": _LSUN * 1e6},
    "temperature": {"K": 1.0},
    "angle": {"rad": 1.0, "deg": math.pi / 180.0, "arcsec": _ARCSEC},
    "posangle": {"rad": 1.0, "deg": math.pi / 180.0},
}

_UNIT_SYSTEMS = {
    "ExtragalacticUnits": {"length": "pc", "distance": "Mpc", "wavelength": "micron", "mass": "Msun",
                           "opacity": "m2/kg", "bolluminosity": "Lsun", "monluminosity": "Lsun/micron",
                           "temperature": "K", "angle": "arcsec", "posangle": "deg"},
    "StellarUnits": {"length": "AU", "distance": "pc", "wavelength": "micron", "mass": "Msun", "opacity": "m2/kg",
                     "bolluminosity": "Lsun", "monluminosity": "Lsun/micron", "temperature": "K",
                     "angle": "arcsec", "posangle": "deg"},
    "SIUnits": {"length": "m", "distance": "m", "wavelength": "m", "mass": "kg", "opacity": "m2/kg",
                "bolluminosity": "W", "monluminosity": "W/m", "temperature": "K", "angle": "rad",
                "posangle": "rad"},
}


def to_si(text, quantity, units="ExtragalacticUnits"):
    """DoublePropertyHandler::convertStringtoDouble (DoublePropertyHandler.cpp:169-200): "value
    [unit]" in SI; a value without unit is in the units system's default unit for the quantity."""
    parts = str(text).split()
    if not parts or len(parts) > 2:
        raise SkiError("invalid value '%s'" % text)
    v = float(parts[0])
    if quantity is None:
        if len(parts) != 1:
            raise SkiError("dimensionless value with a unit: '%s'" % text)
        return v
    table = _FACTORS[quantity]
    unit = parts[1] if len(parts) == 2 else _UNIT_SYSTEMS[units][quantity]
    if unit not in table:
        raise SkiError("unknown %s unit '%s'" % (quantity, unit))
    return v * table[unit]


# ---------------------------------------------------------------------------------------------
# the generic item tree

@dataclass
class Item:
    cls: str
    attrs: dict
    props: dict = field(default_factory=dict)     # compound property name -> list of Items
    line: int = 0

    def one(self, name, default=None):
        v = self.props.get(name)
        if not v:
            if default is None:
                raise SkiError("%s: missing property '%s'" % (self.cls, name))
            return Item(default, {})
        if len(v) != 1:
            raise SkiError("%s: property '%s' holds %d items, expected one" % (self.cls, name, len(v)))
        return v[0]

    def many(self, name):
        return self.props.get(name, [])


def _item(el):
    it = Item(el.tag, dict(el.attrib))
    for prop in el:
        it.props[prop.tag] = [_item(c) for c in prop]
    return it


def parse(source):
    """The item tree of a ski file (path or XML text); returns the simulation Item."""
    if isinstance(source, str) and source.lstrip().startswith("<"):
        root = ET.fromstring(source)
    else:
        root = ET.parse(source).getroot()
    if root.tag != "skirt-simulation-hierarchy":
        raise SkiError("root element is '%s' rather than 'skirt-simulation-hierarchy'" % root.tag)
    kids = list(root)
    if len(kids) != 1:
        raise SkiError("the root element must hold exactly one simulation")
    return _item(kids[0])


# ---------------------------------------------------------------------------------------------
# builders

class _Ctx:
    def __init__(self, units, resources):
        self.units = units
        self.resources = resources

    def d(self, item, name, quantity=None, default=None):
        if name in item.attrs:
            return to_si(item.attrs[name], quantity, self.units)
        if default is None:
            raise SkiError("%s: missing attribute '%s'" % (item.cls, name))
        return to_si(default, quantity, self.units) if isinstance(default, str) else float(default)

    def dl(self, item, name, quantity=None):
        if name not in item.attrs:
            raise SkiError("%s: missing attribute '%s'" % (item.cls, name))
        return [to_si(s.strip(), quantity, self.units) for s in item.attrs[name].split(",") if s.strip()]

    @staticmethod
    def i(item, name, default):
        return int(float(item.attrs.get(name, default)))

    @staticmethod
    def b(item, name, default):
        v = str(item.attrs.get(name, default)).strip().lower()
        return v in ("yes", "true", "1")

    @staticmethod
    def s(item, name, default):
        return item.attrs.get(name, default)


def _geometry(c, it):
    k = it.cls
    if k == "ExpDiskGeometry":
        return ExpDiskGeometry(c.d(it, "radialScale", "length"), c.d(it, "axialScale", "length"),
                               c.d(it, "radialTrunc", "length", 0), c.d(it, "axialTrunc", "length", 0),
                               c.d(it, "innerRadius", "length", 0))
    if k == "SersicGeometry":
        return SersicGeometry(c.d(it, "index", None, 1), c.d(it, "radius", "length"))
    if k == "PointGeometry":
        return PointGeometry()
    if k == "PlummerGeometry":
        return PlummerGeometry(c.d(it, "scale", "length"))
    if k == "ClumpyGeometryDecorator":
        kern = it.one("kernel", "CubicSplineSmoothingKernel").cls
        if kern not in ("CubicSplineSmoothingKernel", "UniformSmoothingKernel"):
            raise SkiError("unsupported smoothing kernel " + kern)
        return ClumpyGeometryDecorator(_geometry(c, it.one("geometry")), c.d(it, "clumpFraction"),
                                       c.i(it, "clumpCount", 0), c.d(it, "clumpRadius", "length"),
                                       c.b(it, "cutoff", "no"),
                                       A.KERNEL_CUBICSPLINE if kern.startswith("Cubic") else A.KERNEL_UNIFORM)
    raise SkiError("geometry class %s is not supported" % k)


def _mesh(c, it, lo, hi):
    """Mesh::numBins and the mesh points mapped to [lo, hi] (CartesianDustGrid.cpp:27-41)."""
    n = c.i(it, "numBins", 100)
    if it.cls in ("LinMesh", "Mesh"):
        t = np.arange(n + 1) / n
    elif it.cls == "PowMesh":                      # NR::powgrid (Fundamentals/NR.hpp:189-204)
        r = c.d(it, "ratio", None, 1)
        if n <= 1 or abs(r - 1.0) < 1e-3:
            t = np.arange(n + 1) / n
        else:
            q = r ** (1.0 / (n - 1))
            t = np.array([(1.0 - q ** i) / (1.0 - q ** n) for i in range(n + 1)])
    elif it.cls == "SymPowMesh":                   # NR::sympowgrid (NR.hpp:225-261)
        r = c.d(it, "ratio", None, 1)
        if n <= 2 or abs(r - 1.0) < 1e-3:
            t = np.arange(n + 1) / n
        else:
            t = np.empty(n + 1)
            if n % 2 == 0:
                M = n // 2
                q = r ** (1.0 / (M - 1.0))
                qM = q ** M
                t[M] = 0.5
                for i in range(1, M + 1):
                    dx = (1.0 - q ** i) / (1.0 - qM) * 0.5
                    t[M + i], t[M - i] = 0.5 + dx, 0.5 - dx
            else:
                M = (n + 1) // 2
                q = r ** (1.0 / (M - 1.0))
                qM = q ** M
                for i in range(1, M + 1):
                    dx = (0.5 + 0.5 * q - q ** i) / (0.5 + 0.5 * q - qM) * 0.5
                    t[M - 1 + i], t[M - i] = 0.5 + dx, 0.5 - dx
    else:
        raise SkiError("mesh class %s is not supported" % it.cls)
    return t * (hi - lo) + lo


@dataclass
class TreeGridSpec:
    """OctTreeDustGrid / BinTreeDustGrid: built on the device when the simulation is set up."""
    gtype: int
    extent: tuple
    minLevel: int
    maxLevel: int
    maxMassFraction: float
    sampleCount: int
    searchMethod: int


@dataclass
class VoronoiGridSpec:
    """VoronoiDustGrid with generated sites: built on the device when the simulation is set up."""
    extent: tuple
    numParticles: int
    distribution: str


def _grid(c, it):
    k = it.cls
    ext = tuple(c.d(it, n, "length") for n in ("minX", "minY", "minZ", "maxX", "maxY", "maxZ"))
    x0, y0, z0, x1, y1, z1 = ext
    if k == "CartesianDustGrid":
        xv = _mesh(c, it.one("meshX", "LinMesh"), x0, x1)
        yv = _mesh(c, it.one("meshY", "LinMesh"), y0, y1)
        zv = _mesh(c, it.one("meshZ", "LinMesh"), z0, z1)
        return CartesianDustGrid(x0, x1, y0, y1, z0, z1, xv=xv, yv=yv, zv=zv)
    if k in ("OctTreeDustGrid", "BinTreeDustGrid"):
        if k == "OctTreeDustGrid" and c.b(it, "barycentric", "no"):
            raise SkiError("OctTreeDustGrid barycentric subdivision is not supported")
        if k == "BinTreeDustGrid" and c.s(it, "directionMethod", "Alternating") != "Alternating":
            raise SkiError("BinTreeDustGrid direction method %s is not supported" % c.s(it, "directionMethod", ""))
        if c.d(it, "maxOpticalDepth", None, 0) > 0 or c.d(it, "maxDensDispFraction", None, 0) > 0:
            raise SkiError("tree subdivision criteria other than maxMassFraction are not supported")
        search = {"TopDown": A.SEARCH_TOPDOWN, "Neighbor": A.SEARCH_NEIGHBOR,
                  "Bookkeeping": A.SEARCH_BOOKKEEPING}[c.s(it, "searchMethod", "Neighbor")]
        return TreeGridSpec(A.GRID_OCTREE if k == "OctTreeDustGrid" else A.GRID_BINTREE, ext,
                            c.i(it, "minLevel", 2), c.i(it, "maxLevel", 6), c.d(it, "maxMassFraction", None, 1e-6),
                            c.i(it, "sampleCount", 100), search)
    if k == "VoronoiDustGrid":
        dist = c.s(it, "distribution", "DustDensity")
        if dist not in ("Uniform", "DustDensity"):
            raise SkiError("VoronoiDustGrid distribution %s is not supported" % dist)
        return VoronoiGridSpec(ext, c.i(it, "numParticles", 500), dist)
    raise SkiError("dust grid class %s is not supported" % k)


def _read_interstellar_mix(resources):
    """The tables InterstellarDustMix::setupSelfBefore reads (InterstellarDustMix.cpp): 1064 rows of
    (lambda [micron], albedo, g, C_ext, kappa_abs [cm2/g], <cos^2>) after '#' comment lines, in
    decreasing wavelength."""
    if not resources:
        raise SkiError("InterstellarDustMix needs the reference's resource tables (resources=<SKIRT dat dir>)")
    path = os.path.join(resources, "DustMix", "InterstellarDustMix.dat")
    rows = []
    with open(path) as f:
        for line in f:
            if line.startswith("#") or not line.strip():
                continue
            rows.append([float(v) for v in line.split()[:6]])
    t = np.array(rows[:1064])[::-1]
    lam = t[:, 0] * 1e-6
    kabs = t[:, 4] * 1e-1
    ksca = kabs * t[:, 1] / (1.0 - t[:, 1])
    return lam, kabs, ksca, t[:, 2]


def _mix(c, it, lam):
    k = it.cls
    nl = len(lam)
    if k == "SimpleOligoDustMix":
        op = c.dl(it, "opacities", "opacity")
        al = c.dl(it, "albedos")
        g = c.dl(it, "asymmetryParameters") if "asymmetryParameters" in it.attrs else [0.0] * len(op)
        if not (len(op) == len(al) == len(g) == nl):
            raise SkiError("SimpleOligoDustMix needs one value per wavelength")
        return DustMix(np.array(op), np.array(al), np.array(g))
    if k == "InterstellarDustMix":
        tl, kabs, ksca, g = _read_interstellar_mix(c.resources)
        # values at the simulation wavelengths: log-log in the opacities, linear in g
        la = np.exp(np.interp(np.log(lam), np.log(tl), np.log(kabs)))
        ls = np.exp(np.interp(np.log(lam), np.log(tl), np.log(ksca)))
        gg = np.interp(np.log(lam), np.log(tl), g)
        return DustMix(la + ls, ls / (la + ls), gg)
    raise SkiError("dust mix class %s is not supported" % k)


def _norm(c, it, lam):
    if it.cls == "FaceOnDustCompNormalization":
        return FaceOnDustCompNormalization(c.d(it, "wavelength", "wavelength"), c.d(it, "opticalDepth"))
    raise SkiError("dust normalization class %s is not supported" % it.cls)


def _stellar(c, it, wl, pan):
    from .models import planck, sun_Llambda, SIGMA_SB
    geom = _geometry(c, it.one("geometry", "PointGeometry"))
    lam, dlam = wl.lambdav, wl.dlambdav
    if it.cls == "OligoStellarComp":
        # luminosities in solar units times the solar spectrum over each bin (OligoStellarComp.cpp:39-75)
        lum = c.dl(it, "luminosities")
        if len(lum) != len(lam):
            raise SkiError("OligoStellarComp needs one luminosity per wavelength")
        return StellarComp(geom, np.array(lum) * sun_Llambda(lam) * dlam)
    if it.cls == "PanStellarComp":
        sed = it.one("sed")
        if sed.cls == "BlackBodySED":
            T = c.d(sed, "temperature", "temperature")
            shape = math.pi * planck(lam, T) / (SIGMA_SB * T ** 4)        # per unit bolometric luminosity
        elif sed.cls == "SunSED":
            shape = sun_Llambda(lam) / LSUN
        else:
            raise SkiError("stellar SED class %s is not supported" % sed.cls)
        nm = it.one("normalization")
        if nm.cls == "BolLuminosityStellarCompNormalization":
            Lbol = c.d(nm, "luminosity") * _LSUN
            return StellarComp(geom, Lbol * shape * dlam)
        if nm.cls == "SpectralLuminosityStellarCompNormalization":
            l0 = c.d(nm, "wavelength", "wavelength")
            L0 = c.d(nm, "luminosity", "monluminosity")
            s0 = float(np.interp(l0, lam, shape))
            return StellarComp(geom, L0 / s0 * shape * dlam)
        raise SkiError("stellar normalization class %s is not supported" % nm.cls)
    raise SkiError("stellar component class %s is not supported" % it.cls)


def _instrument(c, it):
    k = it.cls
    kw = dict(instrumentName=c.s(it, "instrumentName", ""))
    dist = c.d(it, "distance", "distance")
    inc = c.d(it, "inclination", "posangle", 0)
    az = c.d(it, "azimuth", "posangle", 0)
    pa = c.d(it, "positionAngle", "posangle", 0)
    if k == "SEDInstrument":
        return SEDInstrument(dist, inc, az, pa, **kw)
    if k == "MultiFrameInstrument":
        # one InstrumentFrame per wavelength (MultiFrameInstrument.hpp:25-38, InstrumentFrame.hpp:26-60);
        # supported when all frames share one geometry, as one frame instrument whose cube holds the
        # total (writeTotal) and, with writeStellarComps, one frame per stellar component
        geo = []
        for f in it.many("frames"):
            geo.append(dict(pixelsX=c.i(f, "pixelsX", 250), pixelsY=c.i(f, "pixelsY", 250),
                            fieldOfViewX=c.d(f, "fieldOfViewX", "length"),
                            fieldOfViewY=c.d(f, "fieldOfViewY", "length"),
                            centerX=c.d(f, "centerX", "length", 0), centerY=c.d(f, "centerY", "length", 0)))
        if not geo or any(g != geo[0] for g in geo):
            raise SkiError("MultiFrameInstrument: frames of different sizes are not supported")
        return FrameInstrument(distance=dist, inclination=inc, azimuth=az, positionAngle=pa,
                               writeStellarComps=c.b(it, "writeStellarComps", "no"), **geo[0], **kw)
    frame = dict(distance=dist, inclination=inc, azimuth=az, positionAngle=pa,
                 pixelsX=c.i(it, "pixelsX", 250), pixelsY=c.i(it, "pixelsY", 250),
                 fieldOfViewX=c.d(it, "fieldOfViewX", "length"), fieldOfViewY=c.d(it, "fieldOfViewY", "length"),
                 centerX=c.d(it, "centerX", "length", 0), centerY=c.d(it, "centerY", "length", 0), **kw)
    if k == "FrameInstrument":
        return FrameInstrument(**frame)
    if k == "SimpleInstrument":
        return SimpleInstrument(**frame)
    if k == "FullInstrument":
        return FullInstrument(scatteringLevels=c.i(it, "scatteringLevels", 0), **frame)
    raise SkiError("instrument class %s is not supported" % k)


@dataclass
class SkiSimulation:
    """A simulation read from a ski file: the host items plus the run parameters."""
    kind: str                       # "oligo" or "pan"
    model: SceneModel
    packages: float
    seed: int
    selfAbsorption: bool = False
    cycles: int = 0
    emissionBoost: float = 1.0
    grid_spec: object = None        # a tree or Voronoi grid still to build on the device
    instrument_names: list = field(default_factory=list)

    def setup_grid(self, device=0):
        """Builds a tree or Voronoi grid on the device (TreeDustGrid::setupSelfBefore,
        VoronoiDustGrid::setupSelfBefore); a Cartesian grid needs nothing."""
        from . import runtime
        spec = self.grid_spec
        if isinstance(spec, TreeGridSpec):
            self.model.dustGrid = runtime.build_tree(self.model, spec.gtype, spec.extent, spec.minLevel, spec.maxLevel,
                                                     spec.maxMassFraction, spec.sampleCount, self.seed, device,
                                                     spec.searchMethod)
        elif isinstance(spec, VoronoiGridSpec):
            self.model.dustGrid = runtime.build_voronoi(_voronoi_sites(self.model, spec, self.seed), spec.extent,
                                                        device)
        self.grid_spec = None
        return self

    def simulation(self, device=0, precision=A.PREC_FP32, threads=1, autotune=False):
        from . import runtime
        self.setup_grid(device)
        return runtime.MonteCarloSimulation(self.model, self.packages, seed=self.seed, precision=precision,
                                            device=device, selfAbsorption=self.selfAbsorption, cycles=self.cycles,
                                            emissionBoost=self.emissionBoost, threads=threads, autotune=autotune)

    def emulate(self):
        """The reference's emulation mode (-e, SkirtCommandLineHandler.cpp:270-284): one photon
        package per wavelength and no dust self-absorption -- the simulation is set up in full (grid,
        densities, tables on the device) and its phases run with a single packet."""
        self.packages = 1
        self.selfAbsorption = False
        return self

    def run(self, device=0, precision=A.PREC_FP32, threads=1, autotune=False):
        return self.simulation(device, precision, threads, autotune).run()


def _voronoi_sites(model, spec, seed):
    """Generator points: uniform in the domain, or drawn from the dust density (VoronoiDustGrid.cpp,
    distributions Uniform and DustDensity); points outside the domain are redrawn."""
    from .models import sample_expdisk
    rng = np.random.default_rng(seed)
    lo, hi = np.array(spec.extent[:3]), np.array(spec.extent[3:])
    n = spec.numParticles
    if spec.distribution == "Uniform":
        return lo + rng.random((n, 3)) * (hi - lo)
    geoms = [d.geometry for d in model.dustComps]
    if len(geoms) != 1:
        raise SkiError("DustDensity Voronoi sites need exactly one dust component")
    g = geoms[0]
    base = g.geometry if isinstance(g, ClumpyGeometryDecorator) else g
    if not isinstance(base, ExpDiskGeometry):
        raise SkiError("DustDensity Voronoi sites are supported for exponential-disk dust")
    out = np.zeros((0, 3))
    while len(out) < n:
        p = sample_expdisk(base, 2 * n, rng).reshape(-1, 3)
        out = np.concatenate([out, p[np.all((p > lo) & (p < hi), axis=1)]])
    return out[:n]


def load(source, resources=None):
    """Reads a ski file (path or XML text) into a SkiSimulation."""
    sim = parse(source)
    if sim.cls not in ("OligoMonteCarloSimulation", "PanMonteCarloSimulation"):
        raise SkiError("simulation class %s is not supported" % sim.cls)
    pan = sim.cls == "PanMonteCarloSimulation"
    units = sim.one("units", "ExtragalacticUnits").cls
    if units not in _UNIT_SYSTEMS:
        raise SkiError("units system %s is not supported" % units)
    c = _Ctx(units, resources)
    if c.b(sim, "continuousScattering", "no"):
        raise SkiError("continuous scattering is not supported")
    seed = c.i(sim.one("random", "Random"), "seed", 4357)

    wg = sim.one("wavelengthGrid", "LogWavelengthGrid" if pan else "OligoWavelengthGrid")
    if wg.cls == "OligoWavelengthGrid":
        wl = OligoWavelengthGrid(c.dl(wg, "wavelengths", "wavelength"))
    elif wg.cls == "LogWavelengthGrid":
        wl = LogWavelengthGrid(c.d(wg, "minWavelength", "wavelength"), c.d(wg, "maxWavelength", "wavelength"),
                               c.i(wg, "points", 25))
    else:
        raise SkiError("wavelength grid class %s is not supported" % wg.cls)
    lam = wl.lambdav

    ss = sim.one("stellarSystem")
    stars = [_stellar(c, s, wl, pan) for s in ss.many("components")]
    if not stars:
        raise SkiError("the stellar system has no components")

    ds = sim.props.get("dustSystem")
    dust, grid, spec = [], None, None
    sampleCount, selfabs, cycles, boost, dust_emission, write_abs, em_bias = 100, False, 0, 1.0, False, False, 0.5
    if ds:
        ds = ds[0]
        sampleCount = c.i(ds, "sampleCount", 100)
        dd = ds.one("dustDistribution", "CompDustDistribution")
        if dd.cls != "CompDustDistribution":
            raise SkiError("dust distribution class %s is not supported" % dd.cls)
        for comp in dd.many("components"):
            dust.append(DustComp(_geometry(c, comp.one("geometry")), _mix(c, comp.one("mix"), lam),
                                 _norm(c, comp.one("normalization"), lam)))
        g = _grid(c, ds.one("dustGrid"))
        if isinstance(g, (TreeGridSpec, VoronoiGridSpec)):
            spec = g
        else:
            grid = g
        if ds.cls == "OligoDustSystem":
            write_abs = c.b(ds, "writeMeanIntensity", "no")
        elif ds.cls == "PanDustSystem":
            emis = ds.props.get("dustEmissivity")
            dust_emission = bool(emis)
            if emis and emis[0].cls != "GreyBodyDustEmissivity":
                raise SkiError("dust emissivity class %s is not supported" % emis[0].cls)
            lib = ds.props.get("dustLib")
            if lib and lib[0].cls != "AllCellsDustLib":
                raise SkiError("dust library class %s is not supported" % lib[0].cls)
            em_bias = c.d(ds, "emissionBias", None, 0.5)
            boost = c.d(ds, "emissionBoost", None, 1)
            selfabs = c.b(ds, "selfAbsorption", "no")
            cycles = c.i(ds, "cycles", 0)
            write_abs = dust_emission
        else:
            raise SkiError("dust system class %s is not supported" % ds.cls)

    instr = [_instrument(c, i) for i in sim.one("instrumentSystem", "InstrumentSystem").many("instruments")]
    model = SceneModel(wl, stars, grid, dust, instr,
                       emissionBias=c.d(ss, "emissionBias", None, 0.5),
                       minWeightReduction=c.d(sim, "minWeightReduction", None, 1e4),
                       minScattEvents=c.i(sim, "minScattEvents", 0),
                       scattBias=c.d(sim, "scattBias", None, 0.5),
                       writeAbsorption=write_abs, dustEmission=dust_emission, dustEmissionBias=em_bias,
                       densitySamples=sampleCount)
    # clump centres are drawn from the wrapped geometry at set-up (ClumpyGeometryDecorator.cpp:52-63)
    from .models import sample_expdisk
    rng = np.random.default_rng(seed)
    for d in model.dustComps:
        g = d.geometry
        if isinstance(g, ClumpyGeometryDecorator) and g.clumps is None:
            if not isinstance(g.geometry, ExpDiskGeometry):
                raise SkiError("clumps are drawn for exponential-disk geometries only")
            g.clumps = sample_expdisk(g.geometry, g.clumpCount, rng)
    return SkiSimulation("pan" if pan else "oligo", model, c.d(sim, "packages", None, 1e6), seed, selfabs, cycles,
                         boost, spec, [getattr(i, "instrumentName", "") for i in instr])
