"""The C ABI: the library loads without a GPU, exports every function include/skirt_b200.h
declares, its struct layouts match the ctypes mirror, and the host-only entry points behave
like the reference (chunk parameters, tree topology, error reporting)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from skirt7_b200 import _abi as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HDR = os.path.join(ROOT, "include", "skirt_b200.h")


def declared_functions():
    txt = open(HDR).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(skg_[a-z0-9_]+)\s*\(", txt)))


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 30
    out = subprocess.run(["nm", "-D", "--defined-only", A.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(l.split()[-1] for l in out.splitlines() if l.strip())
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    # the ctypes mirror binds each of them
    assert set(names) == set(A.FUNCS), set(names) ^ set(A.FUNCS)


def test_struct_layout_matches_header():
    structs = {"skg_grid": A.Grid, "skg_geometry": A.Geometry, "skg_stellar_comp": A.StellarComp,
               "skg_dust_comp": A.DustComp, "skg_instrument": A.Instrument, "skg_scene": A.Scene,
               "skg_run_opts": A.RunOpts, "skg_counters": A.Counters, "skg_server_opts": A.ServerOpts,
               "skg_request": A.Request, "skg_work": A.Work}
    src = '#include "%s"\n#include <stdio.h>\n#include <stddef.h>\nint main(){\n' % HDR
    for n in structs:
        src += 'printf("%s %%zu\\n", sizeof(%s));\n' % (n, n)
    for f, _ in A.Scene._fields_:
        cf = "lambda" if f == "lambda_" else f
        src += 'printf("skg_scene.%s %%zu\\n", offsetof(skg_scene, %s));\n' % (f, cf)
    src += "return 0;}\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.check_call(["gcc", "-o", exe, c])
        out = subprocess.check_output([exe], text=True)
    got = dict(l.rsplit(" ", 1) for l in out.splitlines())
    for n, S in structs.items():
        assert int(got[n]) == C.sizeof(S), n
    for f, _ in A.Scene._fields_:
        assert int(got["skg_scene." + f]) == getattr(A.Scene, f).offset, f


def test_version_and_no_device_errors(lib):
    assert lib.skg_version() == 1
    n = C.c_int(-1)
    rc = lib.skg_device_count(C.byref(n))
    assert rc in (0, A.SKG_ERR_NO_DEVICE)


@pytest.mark.parametrize("packages,threads,procs,nl", [(1e6, 1, 1, 1), (1e6, 8, 1, 1), (1e7, 8, 1, 50),
                                                       (12345, 4, 3, 3), (5e8, 96, 1, 100), (0, 8, 1, 1)])
def test_chunk_params_match_oracle(lib, orc, packages, threads, procs, nl):
    a = [C.c_uint64() for _ in range(3)]
    b = [C.c_uint64() for _ in range(3)]
    lib.skg_chunk_params(packages, threads, procs, nl, *[C.byref(x) for x in a])
    orc.lib().orc_chunk_params(packages, threads, procs, nl, *[C.byref(x) for x in b])
    assert [x.value for x in a] == [x.value for x in b]
    if packages > 0:
        assert a[2].value >= packages   # Npp = totalChunks*chunksize >= packages


def test_invalid_scene_is_reported_not_thrown(lib):
    sc = A.Scene()   # empty scene: no wavelengths
    h = C.c_void_p()
    rc = lib.skg_ctx_create(C.byref(sc), 0, C.byref(h))
    assert rc in (A.SKG_ERR_INVALID, A.SKG_ERR_NO_DEVICE)
    assert h.value is None
    assert lib.skg_last_error(None)


def test_scene_tally_sizes_and_server_without_device(lib):
    """skg_scene_tally_sizes gives the tally lengths of a scene's instruments before any context
    exists (the serving caller's result buffers); without a device the server is refused cleanly."""
    from skirt7_b200 import models
    from skirt7_b200.scene import DEG, KPC, MPC, FullInstrument, FrameInstrument
    m = models.oligo_disk(N=(8, 8, 4), npix=10, wavelengths=(0.45e-6, 0.55e-6))
    m.instruments.append(FullInstrument(scatteringLevels=2, distance=10 * MPC, inclination=30 * DEG, pixelsX=6,
                                        pixelsY=7, fieldOfViewX=40 * KPC, fieldOfViewY=40 * KPC, instrumentName="f"))
    m.instruments.append(FrameInstrument(10 * MPC, 80 * DEG, 5, 4, 40 * KPC, 40 * KPC, instrumentName="c",
                                         writeStellarComps=True))
    sc, keep = m.lower()
    want = [(1 * 2 * 10 * 10, 2), (0, 2), ((6 + 2) * 2 * 6 * 7, (6 + 2) * 2), (3 * 2 * 5 * 4, 3 * 2)]
    for i, (c, s) in enumerate(want):
        cl, sl = C.c_int64(), C.c_int64()
        assert lib.skg_scene_tally_sizes(C.byref(sc), i, C.byref(cl), C.byref(sl)) == 0
        assert (cl.value, sl.value) == (c, s), i
    assert lib.skg_scene_tally_sizes(C.byref(sc), 4, None, None) == A.SKG_ERR_INVALID
    from skirt7_b200 import runtime
    if runtime.device_count() == 0:
        h = C.c_void_p()
        assert lib.skg_server_create(0, None, C.byref(h)) != 0 and not h.value
