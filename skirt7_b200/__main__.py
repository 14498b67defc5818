"""Command line: run ski files on the device, as the `skirt` command does
(SkirtCommandLineHandler.cpp: -i input path, -o output path, -k/-t are accepted and ignored).

    python -m skirt7_b200 [-i inpath] [-o outpath] [-r resources] [-d device] [--fp64] file.ski ...

Each ski file runs its simulation's phases and writes every instrument's frames (FITS) and SED
(text) named <ski base name>_<instrument>_<component>, as the reference does.
"""
import argparse
import os
import sys
import time

from . import _abi as A
from . import output, ski


def main(argv=None):
    p = argparse.ArgumentParser(prog="python -m skirt7_b200")
    p.add_argument("ski", nargs="+")
    p.add_argument("-i", dest="inpath", default="")
    p.add_argument("-o", dest="outpath", default="")
    p.add_argument("-r", dest="resources", default=None, help="the reference's resource tables (dat directory)")
    p.add_argument("-d", dest="device", type=int, default=0)
    p.add_argument("-t", dest="threads", type=int, default=0, help="accepted for compatibility; unused")
    p.add_argument("-k", dest="keep", action="store_true", help="accepted for compatibility; unused")
    p.add_argument("--fp64", action="store_true", help="FP64 traversal geometry (default FP32)")
    a = p.parse_args(argv)
    rc = 0
    for name in a.ski:
        path = os.path.join(a.inpath, name)
        if not path.endswith(".ski"):
            path += ".ski"
        prefix = os.path.splitext(os.path.basename(path))[0]
        try:
            t0 = time.time()
            s = ski.load(path, resources=a.resources)
            sim = s.run(device=a.device, precision=A.PREC_FP64 if a.fp64 else A.PREC_FP32)
            units = ski.parse(path).one("units", "ExtragalacticUnits").cls
            files = output.write_instruments(sim.ctx, s.model, a.outpath or os.path.dirname(path) or ".", prefix,
                                             units)
            print("%s: %s simulation, %g packages, %d cells; %s; %.2f s; wrote %d files" %
                  (prefix, s.kind, s.packages, sim.ctx.ncells,
                   ", ".join("%s %.1f ms" % kv for kv in sim.phase_ms.items()), time.time() - t0, len(files)))
            sim.ctx.close()
        except (ski.SkiError, A.SkirtError, OSError) as e:
            print("%s: error: %s" % (prefix, e), file=sys.stderr)
            rc = 1
    return rc


if __name__ == "__main__":
    sys.exit(main())
