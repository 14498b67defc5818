"""Host-side simulation items, named and parameterised as SKIRT7's SimulationItem classes.

Each class holds the properties of the reference class it is named after (the Q_CLASSINFO
"Property" blocks of the reference headers) and knows how to lower itself into the flat C
structs of include/skirt_b200.h.  All values are SI, as inside the reference
(SKIRTcore/Units.cpp:17-30); the helpers below convert the usual ski units.
"""
import ctypes as C
import math
from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

from . import _abi as A

# physical constants and units (SKIRTcore/Units.cpp:17-30,51-79)
PC = 3.08567758e16
KPC = 1e3 * PC
MPC = 1e6 * PC
MICRON = 1e-6
LSUN = 3.839e26
DEG = math.pi / 180.0
KAPPA_V = 2600.0


def _dptr(a):
    return a.ctypes.data_as(A.dp) if a is not None else None


# --------------------------------------------------------------------------------------------
# wavelength grids

class OligoWavelengthGrid:
    """OligoWavelengthGrid: a few sorted wavelengths, bins 0.001*lambda wide (OligoWavelengthGrid.cpp:21-27)."""

    def __init__(self, wavelengths):
        self.lambdav = np.sort(np.asarray(wavelengths, dtype=np.float64))
        self.dlambdav = 0.001 * self.lambdav

    @property
    def Nlambda(self):
        return len(self.lambdav)


class LogWavelengthGrid:
    """LogWavelengthGrid: NR::loggrid over [min, max] (LogWavelengthGrid.cpp:20-34); bin widths
    from the geometric midpoints (PanWavelengthGrid.cpp:29-37, WavelengthGrid.cpp:85-95)."""

    def __init__(self, minWavelength, maxWavelength, points):
        n = points - 1
        logmin = math.log10(minWavelength)
        dlog = math.log10(maxWavelength / minWavelength) / n
        lam = np.array([10 ** (logmin + i * dlog) for i in range(n + 1)])
        self.lambdav = lam
        lo = np.empty_like(lam)
        hi = np.empty_like(lam)
        lo[0] = lam[0]
        lo[1:] = np.sqrt(lam[:-1] * lam[1:])
        hi[-1] = lam[-1]
        hi[:-1] = np.sqrt(lam[:-1] * lam[1:])
        self.dlambdav = hi - lo

    @property
    def Nlambda(self):
        return len(self.lambdav)


# --------------------------------------------------------------------------------------------
# geometries

@dataclass
class ExpDiskGeometry:
    radialScale: float
    axialScale: float
    radialTrunc: float = 0.0
    axialTrunc: float = 0.0
    innerRadius: float = 0.0

    def lower(self, g: A.Geometry):
        g.type = A.GEOM_EXPDISK
        for i, v in enumerate((self.radialScale, self.axialScale, self.radialTrunc, self.axialTrunc, self.innerRadius)):
            g.p[i] = v

    def SigmaZ(self):
        """ExpDiskGeometry::SigmaZ (ExpDiskGeometry.cpp:176-186) with rho0 from :24-40."""
        hR, hz, Rmax, zmax, Rmin = (self.radialScale, self.axialScale, self.radialTrunc, self.axialTrunc,
                                    self.innerRadius)
        intz = -2.0 * hz * math.expm1(-zmax / hz) if zmax > 0 else 2.0 * hz
        tmin = math.exp(-Rmin / hR) * (1.0 + Rmin / hR) if Rmin > 0 else 1.0
        tmax = math.exp(-Rmax / hR) * (1.0 + Rmax / hR) if Rmax > 0 else 0.0
        rho0 = 1.0 / (hR * hR * (tmin - tmax) * 2.0 * math.pi * intz)
        if Rmin > 0:
            return 0.0
        if zmax > 0:
            return -2.0 * rho0 * hz * math.expm1(-zmax / hz)
        return 2.0 * rho0 * hz


@dataclass
class SersicGeometry:
    index: float
    radius: float

    def lower(self, g):
        g.type = A.GEOM_SERSIC
        g.p[0] = self.index
        g.p[1] = self.radius


@dataclass
class PointGeometry:
    def lower(self, g):
        g.type = A.GEOM_POINT


@dataclass
class PlummerGeometry:
    scale: float

    def lower(self, g):
        g.type = A.GEOM_PLUMMER
        g.p[0] = self.scale


@dataclass
class ClumpyGeometryDecorator:
    """ClumpyGeometryDecorator (ClumpyGeometryDecorator.cpp).  Clump centres are drawn from the
    wrapped geometry at set-up (:52-63); pass them explicitly or let `draw_clumps` sample them."""
    geometry: object
    clumpFraction: float
    clumpCount: int
    clumpRadius: float
    cutoff: bool = True
    kernel: int = A.KERNEL_CUBICSPLINE
    clumps: Optional[np.ndarray] = None

    def lower(self, g):
        self.geometry.lower(g)
        if self.clumps is None:
            raise ValueError("clump positions not set (call draw_clumps)")
        g.clump_fraction = self.clumpFraction
        g.clump_count = self.clumpCount
        g.clump_radius = self.clumpRadius
        g.clump_cutoff = int(self.cutoff)
        g.clump_kernel = self.kernel
        g.clump_pos = _dptr(self.clumps)

    def SigmaZ(self):
        return self.geometry.SigmaZ()


# --------------------------------------------------------------------------------------------
# stellar components, dust

@dataclass
class StellarComp:
    """A geometric stellar component with a luminosity (W) per wavelength bin
    (GeometricStellarComp / OligoStellarComp / PanStellarComp)."""
    geometry: object
    luminosities: np.ndarray


@dataclass
class DustMix:
    """Per-wavelength extinction coefficient (m2/kg), albedo and HG asymmetry parameter --
    the single-population tables of SimpleOligoDustMix (SimpleOligoDustMix.cpp:22-51) or of a
    tabulated panchromatic mix."""
    kappaext: np.ndarray
    albedo: np.ndarray
    asymmpar: np.ndarray

    def kappaext_at(self, lam, lambdav):
        return float(np.interp(lam, lambdav, self.kappaext))


@dataclass
class FaceOnDustCompNormalization:
    """tau / (SigmaZ * kappa_ext(lambda)) (FaceOnDustCompNormalization.cpp:67-74)."""
    wavelength: float
    opticalDepth: float

    def factor(self, geometry, mix, lambdav):
        return self.opticalDepth / (geometry.SigmaZ() * mix.kappaext_at(self.wavelength, lambdav))


@dataclass
class DustComp:
    geometry: object
    mix: DustMix
    normalization: object
    norm: float = 0.0


# --------------------------------------------------------------------------------------------
# dust grids

@dataclass
class CartesianDustGrid:
    """CartesianDustGrid with linear meshes (LinMesh) or explicit plane arrays."""
    minX: float
    maxX: float
    minY: float
    maxY: float
    minZ: float
    maxZ: float
    pointsX: int = 0
    pointsY: int = 0
    pointsZ: int = 0
    xv: Optional[np.ndarray] = None
    yv: Optional[np.ndarray] = None
    zv: Optional[np.ndarray] = None

    def __post_init__(self):
        # CartesianDustGrid::setupSelfAfter: mesh*(max-min)+min (CartesianDustGrid.cpp:27-41);
        # LinMesh::mesh is i/N (LinMesh.cpp)
        if self.xv is None:
            self.xv = np.arange(self.pointsX + 1) / self.pointsX * (self.maxX - self.minX) + self.minX
        if self.yv is None:
            self.yv = np.arange(self.pointsY + 1) / self.pointsY * (self.maxY - self.minY) + self.minY
        if self.zv is None:
            self.zv = np.arange(self.pointsZ + 1) / self.pointsZ * (self.maxZ - self.minZ) + self.minZ
        self.xv = np.ascontiguousarray(self.xv, dtype=np.float64)
        self.yv = np.ascontiguousarray(self.yv, dtype=np.float64)
        self.zv = np.ascontiguousarray(self.zv, dtype=np.float64)

    @property
    def ncells(self):
        return (len(self.xv) - 1) * (len(self.yv) - 1) * (len(self.zv) - 1)

    def lower(self, g: A.Grid):
        g.type = A.GRID_CARTESIAN
        g.xmin, g.ymin, g.zmin, g.xmax, g.ymax, g.zmax = self.minX, self.minY, self.minZ, self.maxX, self.maxY, self.maxZ
        g.nx, g.ny, g.nz = len(self.xv) - 1, len(self.yv) - 1, len(self.zv) - 1
        g.xv, g.yv, g.zv = _dptr(self.xv), _dptr(self.yv), _dptr(self.zv)


class TreeDustGrid:
    """An octree (OctTreeDustGrid) or k-d tree (BinTreeDustGrid, alternating directions) held as
    flat arrays.  Build it with skirt7_b200.grids.build_tree (device-sampled subdivision) or from
    explicit split decisions."""

    def __init__(self, gtype, extent, node_box, node_child, node_father, node_cell, node_dir,
                 nbr_offsets, nbr_ids, searchMethod=A.SEARCH_NEIGHBOR):
        self.type = gtype
        self.extent = tuple(float(v) for v in extent)
        self.node_box = np.ascontiguousarray(node_box, dtype=np.float64)
        self.node_child = np.ascontiguousarray(node_child, dtype=np.int32)
        self.node_father = np.ascontiguousarray(node_father, dtype=np.int32)
        self.node_cell = np.ascontiguousarray(node_cell, dtype=np.int32)
        self.node_dir = np.ascontiguousarray(node_dir, dtype=np.int8)
        self.nbr_offsets = np.ascontiguousarray(nbr_offsets, dtype=np.int64)
        self.nbr_ids = np.ascontiguousarray(nbr_ids, dtype=np.int32)
        self.searchMethod = searchMethod

    @property
    def nnodes(self):
        return len(self.node_child)

    @property
    def ncells(self):
        return int((self.node_cell >= 0).sum())

    def lower(self, g: A.Grid):
        g.type = self.type
        g.xmin, g.ymin, g.zmin, g.xmax, g.ymax, g.zmax = self.extent
        g.nnodes = self.nnodes
        g.node_box = _dptr(self.node_box)
        g.node_child = self.node_child.ctypes.data_as(A.i32p)
        g.node_father = self.node_father.ctypes.data_as(A.i32p)
        g.node_cell = self.node_cell.ctypes.data_as(A.i32p)
        g.node_dir = self.node_dir.ctypes.data_as(A.i8p)
        g.nbr_offsets = self.nbr_offsets.ctypes.data_as(A.i64p)
        g.nbr_ids = self.nbr_ids.ctypes.data_as(A.i32p)
        g.search_method = self.searchMethod


class VoronoiDustGrid:
    """A Voronoi tessellation held as flat arrays (sites, CSR neighbour lists with walls -1..-6,
    block lists, cell volumes and bounding boxes)."""

    def __init__(self, extent, sites, vnbr_offsets, vnbr_ids, nb, block_offsets, block_ids,
                 volume=None, bbox=None):
        self.extent = tuple(float(v) for v in extent)
        self.sites = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
        self.vnbr_offsets = np.ascontiguousarray(vnbr_offsets, dtype=np.int64)
        self.vnbr_ids = np.ascontiguousarray(vnbr_ids, dtype=np.int32)
        self.nb = int(nb)
        self.block_offsets = np.ascontiguousarray(block_offsets, dtype=np.int64)
        self.block_ids = np.ascontiguousarray(block_ids, dtype=np.int32)
        self.volume = None if volume is None else np.ascontiguousarray(volume, dtype=np.float64)
        self.bbox = None if bbox is None else np.ascontiguousarray(bbox, dtype=np.float64)

    @property
    def ncells(self):
        return len(self.sites)

    def lower(self, g: A.Grid):
        g.type = A.GRID_VORONOI
        g.xmin, g.ymin, g.zmin, g.xmax, g.ymax, g.zmax = self.extent
        g.nsites = len(self.sites)
        g.sites = _dptr(self.sites)
        g.vnbr_offsets = self.vnbr_offsets.ctypes.data_as(A.i64p)
        g.vnbr_ids = self.vnbr_ids.ctypes.data_as(A.i32p)
        g.nb = self.nb
        g.block_offsets = self.block_offsets.ctypes.data_as(A.i64p)
        g.block_ids = self.block_ids.ctypes.data_as(A.i32p)
        g.cell_volume = _dptr(self.volume)
        g.cell_bbox = _dptr(self.bbox)


# --------------------------------------------------------------------------------------------
# instruments

@dataclass
class SEDInstrument:
    distance: float
    inclination: float = 0.0
    azimuth: float = 0.0
    positionAngle: float = 0.0
    instrumentName: str = "sed"
    type: int = A.INSTR_SED

    def lower(self, I: A.Instrument):
        I.type = self.type
        I.distance, I.inclination, I.azimuth, I.position_angle = (self.distance, self.inclination, self.azimuth,
                                                                  self.positionAngle)


@dataclass
class FrameInstrument:
    distance: float
    inclination: float
    pixelsX: int
    pixelsY: int
    fieldOfViewX: float
    fieldOfViewY: float
    azimuth: float = 0.0
    positionAngle: float = 0.0
    centerX: float = 0.0
    centerY: float = 0.0
    instrumentName: str = "frame"
    type: int = A.INSTR_FRAME
    scatteringLevels: int = 0
    writeStellarComps: bool = False   # FRAME: one more frame per stellar component (MultiFrameInstrument)

    def lower(self, I: A.Instrument):
        I.type = self.type
        I.distance, I.inclination, I.azimuth, I.position_angle = (self.distance, self.inclination, self.azimuth,
                                                                  self.positionAngle)
        I.nxp, I.nyp = self.pixelsX, self.pixelsY
        I.fovx, I.fovy, I.xc, I.yc = self.fieldOfViewX, self.fieldOfViewY, self.centerX, self.centerY
        I.nscatt_levels = self.scatteringLevels
        I.stellar_comps = int(bool(self.writeStellarComps) and self.type == A.INSTR_FRAME)


def SimpleInstrument(**kw):
    return FrameInstrument(type=A.INSTR_SIMPLE, **kw)


def FullInstrument(scatteringLevels=0, **kw):
    return FrameInstrument(type=A.INSTR_FULL, scatteringLevels=scatteringLevels, **kw)


# --------------------------------------------------------------------------------------------
# the simulation description

@dataclass
class SceneModel:
    """Everything below MonteCarloSimulation that the packet loop touches."""
    wavelengthGrid: object
    stellarComps: List[StellarComp]
    dustGrid: object = None
    dustComps: List[DustComp] = field(default_factory=list)
    instruments: list = field(default_factory=list)
    emissionBias: float = 0.5
    minWeightReduction: float = 1e4
    minScattEvents: int = 0
    scattBias: float = 0.5
    writeAbsorption: bool = False
    dustEmission: bool = False
    dustEmissionBias: float = 0.5
    densitySamples: int = 100
    rho: Optional[np.ndarray] = None

    def normalise(self):
        lam = self.wavelengthGrid.lambdav
        for d in self.dustComps:
            if d.normalization is not None:
                d.norm = d.normalization.factor(d.geometry, d.mix, lam)
        return self

    def lower(self):
        """Returns (Scene struct, keep-alive list)."""
        self.normalise()
        keep = []
        sc = A.Scene()
        if self.dustGrid is not None:
            self.dustGrid.lower(sc.grid)
        wl = self.wavelengthGrid
        lam = np.ascontiguousarray(wl.lambdav, dtype=np.float64)
        dl = np.ascontiguousarray(wl.dlambdav, dtype=np.float64)
        keep += [lam, dl]
        sc.nlambda = len(lam)
        sc.lambda_ = _dptr(lam)
        sc.dlambda = _dptr(dl)
        nd = len(self.dustComps)
        sc.ncomp = nd
        if nd:
            darr = (A.DustComp * nd)()
            for i, d in enumerate(self.dustComps):
                d.geometry.lower(darr[i].geometry)
                ke = np.ascontiguousarray(d.mix.kappaext, dtype=np.float64)
                al = np.ascontiguousarray(d.mix.albedo, dtype=np.float64)
                gg = np.ascontiguousarray(d.mix.asymmpar, dtype=np.float64)
                keep += [ke, al, gg]
                darr[i].norm = d.norm
                darr[i].kappaext, darr[i].albedo, darr[i].asymmpar = _dptr(ke), _dptr(al), _dptr(gg)
            keep.append(darr)
            sc.dust = darr
        if self.rho is not None:
            rho = np.ascontiguousarray(self.rho, dtype=np.float64)
            keep.append(rho)
            sc.rho = _dptr(rho)
        sc.density_samples = self.densitySamples
        ns = len(self.stellarComps)
        sarr = (A.StellarComp * ns)()
        for i, s in enumerate(self.stellarComps):
            s.geometry.lower(sarr[i].geometry)
            L = np.ascontiguousarray(s.luminosities, dtype=np.float64)
            keep.append(L)
            sarr[i].luminosity = _dptr(L)
        keep.append(sarr)
        sc.nstellar = ns
        sc.stellar = sarr
        sc.emission_bias = self.emissionBias
        ni = len(self.instruments)
        if ni:
            iarr = (A.Instrument * ni)()
            for i, ins in enumerate(self.instruments):
                ins.lower(iarr[i])
            keep.append(iarr)
            sc.instr = iarr
        sc.ninstr = ni
        sc.min_weight_reduction = self.minWeightReduction
        sc.min_scatt_events = self.minScattEvents
        sc.scatt_bias = self.scattBias
        sc.store_absorption = int(self.writeAbsorption)
        sc.dust_emission = int(self.dustEmission)
        sc.dust_emission_bias = self.dustEmissionBias
        # clump arrays etc. referenced from geometries
        for s in self.stellarComps:
            if isinstance(s.geometry, ClumpyGeometryDecorator):
                keep.append(s.geometry.clumps)
        for d in self.dustComps:
            if isinstance(d.geometry, ClumpyGeometryDecorator):
                keep.append(d.geometry.clumps)
        keep.append(self)
        return sc, keep
