"""Command line: run ski files on the device, with the options of the `skirt` command
(SkirtCommandLineHandler.cpp:40-360).

    python -m skirt7_b200 [-t threads] [-s parallel] [-e] [-k] [-i inpath] [-o outpath] [-r]
                          [-b] [-v] [-m] [-d] [--resources dir] [--device n] [--fp64] [--autotune [file]]
                          file.ski ...

  -t N   the host thread count the reference would use: it sets the chunking, hence the packet count
         actually run (totalChunks * chunksize >= packages, MonteCarloSimulation.cpp:68-114)
  -s N   simulations run at once when several ski files are given (each on its own context and
         stream of the one device)
  -e     emulation: one photon package per wavelength, no dust self-absorption (:270-284); the
         simulation is set up in full and its device footprint reported
  -k     -i and -o are relative to the ski file's directory instead of the current one (:295-297)
  -i/-o  input and output paths
  -r     look for matching ski files recursively (file names may hold wildcards; :191-254)
  -b     brief console output; -v verbose; -m report the device memory with each message
  -d     data-parallel mode of a multi-process run: accepted, the ranks run packet ranges
  -l     memory (de)allocation logging: refused, as in a reference build without BUILDING_MEMORY
  -x     the SMILE schema export: not provided (the ski editor is out of scope)
Each ski file runs its simulation's phases and writes every instrument's frames (FITS) and SED
(text) named <ski base name>_<instrument>_<component>, as the reference does.
"""
import argparse
import fnmatch
import os
import sys
import threading
import time
from concurrent.futures import ThreadPoolExecutor

from . import _abi as A
from . import output, ski


def skifiles_for(filepath, recursive):
    """SkirtCommandLineHandler::skifilesFor (SkirtCommandLineHandler.cpp:191-254): a single file
    (the .ski extension added when missing), or with -r / wildcards every matching file of the
    directory, recursively with -r, sorted by name ignoring case."""
    name = os.path.basename(filepath)
    if not recursive and "?" not in name and "*" not in name:
        if not os.path.exists(filepath) and not filepath.lower().endswith(".ski"):
            filepath += ".ski"
        return [filepath] if os.path.exists(filepath) else []
    out = []

    def scan(d):
        try:
            entries = sorted(os.listdir(d), key=str.lower)
        except OSError:
            return
        out.extend(os.path.join(d, e) for e in entries
                   if fnmatch.fnmatch(e, name) and os.path.isfile(os.path.join(d, e)))
        if recursive:
            for e in entries:
                if os.path.isdir(os.path.join(d, e)):
                    scan(os.path.join(d, e))
    scan(os.path.abspath(os.path.dirname(filepath) or "."))
    return out


def main(argv=None):
    p = argparse.ArgumentParser(prog="python -m skirt7_b200")
    p.add_argument("ski", nargs="*")
    p.add_argument("-t", dest="threads", type=int, default=0)
    p.add_argument("-s", dest="parallel", type=int, default=1)
    p.add_argument("-e", dest="emulate", action="store_true")
    p.add_argument("-k", dest="skirel", action="store_true")
    p.add_argument("-i", dest="inpath", default="")
    p.add_argument("-o", dest="outpath", default="")
    p.add_argument("-r", dest="recursive", action="store_true")
    p.add_argument("-b", dest="brief", action="store_true")
    p.add_argument("-v", dest="verbose", action="store_true")
    p.add_argument("-m", dest="memory", action="store_true")
    p.add_argument("-d", dest="dataparallel", action="store_true")
    p.add_argument("-l", dest="alloclog", type=float, default=None)
    p.add_argument("-x", dest="schema", action="store_true")
    p.add_argument("--resources", default=None, help="the reference's resource tables (dat directory)")
    p.add_argument("--device", type=int, default=0)
    p.add_argument("--fp64", action="store_true", help="FP64 traversal geometry (default FP32)")
    p.add_argument("--autotune", nargs="?", const=True, default=False,
                   help="tune the launch choices before the first phase (optionally cached in a JSON file)")
    a = p.parse_args(argv)
    if a.alloclog is not None:
        print("error: Enable BUILDING_MEMORY in the build options to use the -l option", file=sys.stderr)
        return 1
    if a.schema:
        print("error: the SMILE schema export (-x) belongs to the ski editor, which this build does not provide",
              file=sys.stderr)
        return 1
    if not a.ski:
        p.print_help()
        return 1
    files, rc = [], 0
    for name in a.ski:
        found = skifiles_for(name, a.recursive)
        if not found:
            print("error: %s: %s" % ("No ski file matches the pattern" if (a.recursive or "*" in name or "?" in name)
                                     else "This ski file does not exist", name), file=sys.stderr)
            rc = 1
        files += found
    if rc or not files:
        return 1
    lock = threading.Lock()

    def say(msg, level=1):
        if level == 0 or (not a.brief and (level == 1 or a.verbose)):
            with lock:
                print(msg, flush=True)

    def one(path):
        prefix = os.path.splitext(os.path.basename(path))[0]
        base = os.path.dirname(os.path.abspath(path)) if a.skirel else os.getcwd()
        inpath = a.inpath if os.path.isabs(a.inpath) else os.path.join(base, a.inpath)
        outpath = a.outpath if os.path.isabs(a.outpath) else os.path.join(base, a.outpath)
        try:
            t0 = time.time()
            say("Constructing a simulation from ski file '%s'..." % path, 2)
            s = ski.load(path, resources=a.resources or (inpath if a.inpath else None))
            if a.emulate:
                s.emulate()
            sim = s.run(device=a.device, precision=A.PREC_FP64 if a.fp64 else A.PREC_FP32,
                        threads=a.threads or 1, autotune=a.autotune)
            mem = " (device memory %.3f GB)" % (sim.ctx.device_bytes / 1e9) if (a.memory or a.emulate) else ""
            if a.emulate:
                say("%s: emulation: %s simulation, %d cells, set up and run with one package per wavelength%s" %
                    (prefix, s.kind, sim.ctx.ncells, mem), 0)
            else:
                units = ski.parse(path).one("units", "ExtragalacticUnits").cls
                os.makedirs(outpath, exist_ok=True)
                files = output.write_instruments(sim.ctx, s.model, outpath, prefix, units)
                say("%s: %s simulation, %g packages, %d cells; %s; %.2f s; wrote %d files%s" %
                    (prefix, s.kind, s.packages, sim.ctx.ncells,
                     ", ".join("%s %.1f ms" % kv for kv in sim.phase_ms.items()), time.time() - t0, len(files), mem),
                    0)
            if sim.launch:
                say("%s: launch choices %s" % (prefix, {k: sim.launch[k] for k in ("pool", "refill", "blocks")}), 2)
            sim.ctx.close()
            return 0
        except (ski.SkiError, A.SkirtError, OSError) as e:
            say("%s: error: %s" % (prefix, e), 0)
            return 1

    if len(files) > 1 and a.parallel > 1:
        with ThreadPoolExecutor(max_workers=a.parallel) as ex:
            rcs = list(ex.map(one, files))
    else:
        rcs = [one(f) for f in files]
    return 1 if any(rcs) else 0


if __name__ == "__main__":
    sys.exit(main())
