"""A ski file runs unchanged on the device: the oligochromatic Cartesian disk read from its ski file
gives, packet for packet, the frame of the same workload built in code (same seed, same packets;
only the summation order of the FP64 tally atomics differs)."""
import os

import numpy as np
import pytest

from skirt7_b200 import models, runtime, ski

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
CFG1 = os.path.join(HERE, "golden", "oligo_disk_cartesian.ski")


def test_ski_run_matches_coded_workload():
    xml = open(CFG1).read().replace('packages="1e6"', 'packages="2e4"')
    xml = xml.replace('<LinMesh numBins="100"/>', '<LinMesh numBins="40"/>').replace(
        '<LinMesh numBins="50"/>', '<LinMesh numBins="20"/>')
    sim = ski.load(xml).run()
    cube, sed = sim.ctx.read_instrument(0)
    m = models.oligo_disk(N=(40, 40, 20))
    ref = runtime.MonteCarloSimulation(m, packages=2e4, seed=4357).run()
    cube2, sed2 = ref.ctx.read_instrument(0)
    assert cube.sum() > 0
    assert np.allclose(cube, cube2, rtol=1e-10, atol=1e-12 * cube2.max())
    s1, s2 = sim.ctx.read_instrument(1)[1], ref.ctx.read_instrument(1)[1]
    assert np.allclose(s1, s2, rtol=1e-10)
    sim.ctx.close()
    ref.ctx.close()


def test_ski_octree_builds_on_the_device():
    xml = open(CFG1).read().replace('packages="1e6"', 'packages="1e4"')
    i, j = xml.index("<CartesianDustGrid"), xml.index("</CartesianDustGrid>") + len("</CartesianDustGrid>")
    tree = ('<OctTreeDustGrid minX="-20 kpc" maxX="20 kpc" minY="-20 kpc" maxY="20 kpc" minZ="-2 kpc" maxZ="2 kpc" '
            'minLevel="2" maxLevel="7" searchMethod="Neighbor" sampleCount="100" maxMassFraction="1e-4"/>')
    sim = ski.load(xml[:i] + tree + xml[j:]).run()
    assert sim.ctx.ncells > 1000
    cube, _ = sim.ctx.read_instrument(0)
    assert cube.sum() > 0 and sim.ctx.counters()["errors"] == 0
    sim.ctx.close()


def test_command_line_modes(tmp_path, capsys):
    """The skirt command's modes (SkirtCommandLineHandler.cpp): -e sets the simulation up and runs
    one package per wavelength; -t sets the chunking, so the packets run are the reference's
    totalChunks * chunksize for that thread count; -k with -o writes next to the ski file; --autotune
    picks launch choices before the first phase (results do not depend on them)."""
    from skirt7_b200.__main__ import main
    xml = open(CFG1).read().replace('packages="1e6"', 'packages="12345"')
    xml = xml.replace('<LinMesh numBins="100"/>', '<LinMesh numBins="20"/>').replace(
        '<LinMesh numBins="50"/>', '<LinMesh numBins="10"/>')
    d = tmp_path / "runs"
    d.mkdir()
    f = d / "disk.ski"
    f.write_text(xml)
    assert main(["-e", str(f)]) == 0
    out = capsys.readouterr().out
    assert "emulation" in out and "device memory" in out
    assert main(["-k", "-o", "out", "-t", "4", str(f)]) == 0
    assert (d / "out").is_dir() and any(p.name.startswith("disk_") for p in (d / "out").iterdir())
    # -t 4: 40 chunks of 309 packets (MonteCarloSimulation.cpp:86-94)
    s = ski.load(str(f))
    sim = s.run(threads=4, autotune=True)
    assert sim.ctx.counters()["packets"] == 40 * 309
    assert set(sim.launch) >= {"pool", "refill", "blocks"}
    sim.ctx.close()
