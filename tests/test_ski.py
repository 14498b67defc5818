"""Ski files: the loader reads SKIRT7's XML format (property names, defaults and units of the
reference's SimulationItem classes) into the same host items the workloads build in code."""
import math
import os

import numpy as np
import pytest

from skirt7_b200 import _abi as A
from skirt7_b200 import models, ski
from skirt7_b200.scene import KPC, MPC, PC

HERE = os.path.dirname(os.path.abspath(__file__))
CFG1 = os.path.join(HERE, "golden", "oligo_disk_cartesian.ski")


def test_units_follow_the_reference_tables():
    assert ski.to_si("4 kpc", "length") == 4e3 * PC
    assert ski.to_si("4000", "length") == 4000 * PC                       # ExtragalacticUnits: pc
    assert ski.to_si("10", "distance") == 10 * MPC
    assert ski.to_si("10", "distance", "StellarUnits") == 10 * PC
    assert ski.to_si("88 deg", "posangle") == 88 * math.pi / 180
    assert ski.to_si("0.55", "wavelength") == 0.55e-6
    assert ski.to_si("2 Msun", "mass") == 2 * 1.9891e30
    with pytest.raises(ski.SkiError):
        ski.to_si("3 furlong", "length")


def test_ski_file_gives_the_coded_workload():
    s = ski.load(CFG1)
    m = models.oligo_disk()
    assert s.kind == "oligo" and s.packages == 1e6 and s.seed == 4357
    assert np.array_equal(s.model.wavelengthGrid.lambdav, m.wavelengthGrid.lambdav)
    assert len(s.model.stellarComps) == len(m.stellarComps) == 2
    for a, b in zip(s.model.stellarComps, m.stellarComps):
        assert type(a.geometry) is type(b.geometry)
        assert a.geometry == b.geometry
        assert np.allclose(a.luminosities, b.luminosities, rtol=1e-14)
    (da,), (db,) = s.model.dustComps, m.dustComps
    assert da.geometry == db.geometry
    for f in ("kappaext", "albedo", "asymmpar"):
        assert np.array_equal(getattr(da.mix, f), getattr(db.mix, f))
    assert da.normalization == db.normalization
    ga, gb = s.model.dustGrid, m.dustGrid
    for f in ("xv", "yv", "zv"):
        assert np.allclose(getattr(ga, f), getattr(gb, f), rtol=0, atol=1e-6 * KPC)
    assert [type(i) for i in s.model.instruments] == [type(i) for i in m.instruments]
    for a, b in zip(s.model.instruments, m.instruments):
        for f in ("distance", "inclination", "type"):
            assert getattr(a, f) == pytest.approx(getattr(b, f), rel=1e-15)
    assert s.model.writeAbsorption


def test_meshes_and_defaults():
    xml = open(CFG1).read().replace('<LinMesh numBins="100"/>', '<PowMesh numBins="10" ratio="5"/>', 1)
    xml = xml.replace(' minScattEvents="0"', "")
    s = ski.load(xml)
    xv = s.model.dustGrid.xv
    assert len(xv) == 11 and xv[0] == -20 * KPC and xv[-1] == pytest.approx(20 * KPC)
    w = np.diff(xv)
    assert w[-1] / w[0] == pytest.approx(5.0, rel=1e-12)                   # outermost / innermost bin
    assert s.model.minScattEvents == 0                                      # the property's default


def test_tree_grid_and_unsupported_classes():
    xml = open(CFG1).read()
    i, j = xml.index("<CartesianDustGrid"), xml.index("</CartesianDustGrid>") + len("</CartesianDustGrid>")
    tree = ('<OctTreeDustGrid minX="-20 kpc" maxX="20 kpc" minY="-20 kpc" maxY="20 kpc" minZ="-2 kpc" maxZ="2 kpc" '
            'minLevel="2" maxLevel="8" searchMethod="Bookkeeping" sampleCount="100" maxMassFraction="1e-5"/>')
    s = ski.load(xml[:i] + tree + xml[j:])
    assert isinstance(s.grid_spec, ski.TreeGridSpec)
    assert (s.grid_spec.gtype, s.grid_spec.maxLevel, s.grid_spec.searchMethod) == (A.GRID_OCTREE, 8, A.SEARCH_BOOKKEEPING)
    assert s.grid_spec.maxMassFraction == 1e-5
    with pytest.raises(ski.SkiError, match="TorusGeometry"):
        ski.load(xml.replace("SersicGeometry index=\"4\" radius=\"1.5 kpc\"", "TorusGeometry"))
    with pytest.raises(ski.SkiError, match="resource"):
        ski.load(xml.replace('<SimpleOligoDustMix opacities="2600 m2/kg" albedos="0.6" asymmetryParameters="0.6"/>',
                             "<InterstellarDustMix/>"))


def test_fits_round_trip_and_calibration(tmp_path):
    from skirt7_b200 import output
    cube = np.arange(2 * 3 * 4, dtype=np.float64).reshape(2, 3, 4) * 1.5e-3
    p = str(tmp_path / "x_frame_total.fits")
    output.write_fits(p, cube, [("BUNIT", "W/m2/arcsec2", "")])
    back, hdr = output.read_fits(p)
    assert np.array_equal(back, cube) and hdr["BUNIT"] == "W/m2/arcsec2"
    assert os.path.getsize(p) % 2880 == 0
    # a point source of luminosity L in one pixel: the surface brightness summed over the pixel
    # solid angle and multiplied by 4 pi d^2 dlambda / lambda gives L back
    lam, dlam, d, s = np.array([0.55e-6]), np.array([0.55e-9]), 10 * MPC, 40 * KPC / 300
    f = np.zeros((1, 3, 3))
    f[0, 1, 1] = 1e30
    sb = output.calibrate_frame(f, lam, dlam, d, s, s)
    area = (2 * math.atan(s / (2 * d))) ** 2
    L = sb[0, 1, 1] / ((math.pi / 648000) ** 2) * area * 4 * math.pi * d * d * dlam[0] / lam[0]
    assert L == pytest.approx(1e30, rel=1e-12)


def test_multiframe_instrument_for_fitskirt():
    """MultiFrameInstrument (one InstrumentFrame per wavelength, writeStellarComps for FitSKIRT)
    maps onto a frame instrument with one frame per stellar component when its frames share one
    geometry; frames of different sizes are refused by name."""
    frame = ('<InstrumentFrame fieldOfViewX="40 kpc" pixelsX="64" centerX="0 pc" fieldOfViewY="40 kpc" '
             'pixelsY="64" centerY="0 pc"/>')
    multi = ('<MultiFrameInstrument instrumentName="fit" distance="10 Mpc" inclination="85 deg" azimuth="0 deg" '
             'positionAngle="0 deg" writeTotal="true" writeStellarComps="true"><frames>%s</frames>'
             '</MultiFrameInstrument>' % frame)
    xml = open(CFG1).read()
    i0 = xml.index("<FrameInstrument ")
    i1 = xml.index("/>", i0) + 2
    s = ski.load(xml[:i0] + multi + xml[i1:])
    ins = s.model.instruments[0]
    assert ins.type == A.INSTR_FRAME and ins.writeStellarComps and ins.pixelsX == 64
    assert ins.inclination == pytest.approx(85 * np.pi / 180)
    other = frame.replace('pixelsX="64"', 'pixelsX="32"')
    bad = multi.replace("</frames>", other + "</frames>")
    with pytest.raises(ski.SkiError, match="different sizes"):
        ski.load(xml[:i0] + bad + xml[i1:])


def test_command_line_ski_lookup_and_refused_options(tmp_path, capsys):
    """SkirtCommandLineHandler::skifilesFor (SkirtCommandLineHandler.cpp:191-254): a missing .ski
    extension is added; wildcards match in the file's directory, -r also in its subdirectories,
    sorted by name ignoring case; -l and -x are refused as in a reference build without them."""
    from skirt7_b200.__main__ import main, skifiles_for
    (tmp_path / "sub").mkdir()
    for f in ("b.ski", "A.ski", "c.txt", "sub/d.ski"):
        (tmp_path / f).write_text("<skirt-simulation-hierarchy/>")
    assert skifiles_for(str(tmp_path / "b"), False) == [str(tmp_path / "b.ski")]
    assert skifiles_for(str(tmp_path / "nope"), False) == []
    assert skifiles_for(str(tmp_path / "*.ski"), False) == [str(tmp_path / "A.ski"), str(tmp_path / "b.ski")]
    assert skifiles_for(str(tmp_path / "*.ski"), True) == [str(tmp_path / "A.ski"), str(tmp_path / "b.ski"),
                                                            str(tmp_path / "sub" / "d.ski")]
    assert main(["-l", "1", str(tmp_path / "b.ski")]) == 1
    assert main(["-x"]) == 1
    assert main([str(tmp_path / "nope.ski")]) == 1
    assert "does not exist" in capsys.readouterr().err
