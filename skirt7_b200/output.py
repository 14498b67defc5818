"""Output files of the instruments, in the reference's calibration, units and names.

SingleFrameInstrument::calibrateAndWriteDataCubes (SingleFrameInstrument.cpp:151-226) turns the
tallied luminosity per pixel and wavelength bin into surface brightness: divide by the bin width,
by the pixel's solid angle (2 atan(size / 2d) on each axis) and by 4 pi d^2, then express it in the
units system's output style (Neutral by default: lambda f_lambda, in W/m2/arcsec2 for
ExtragalacticUnits and StellarUnits, W/m2/sr for SIUnits; Units.cpp:1033-1041).  The frame goes to
a FITS image <prefix>_<instrument>_<component>.fits (x fastest, then y, then wavelength).
DistantInstrument::calibrateAndWriteSEDs (DistantInstrument.cpp:131-183) divides the SED by the bin
width and 4 pi d^2 and writes <prefix>_<instrument>_sed.dat: a '# column k: ...' header and one
row per wavelength, in micron and W/m2 (Neutral style).
"""
import math
import os

import numpy as np

from . import _abi as A

_ARCSEC2 = (math.pi / (180.0 * 3600.0)) ** 2

# frame components of FullInstrument (FullInstrument.cpp:269-292) in the device tally order
_FULL_FRAMES = [("total", A.FULL_TOT), ("transparent", A.FULL_TRA), ("direct", A.FULL_STRDIR),
                ("scattered", A.FULL_STRSCA)]
_FULL_SEDS = ["total flux", "direct stellar flux", "scattered stellar flux", "total dust emission flux",
              "dust emission scattered flux", "transparent flux"]


def _sb_out(units):
    """Output factor and unit string of neutral surface brightness."""
    return (1.0, "W/m2/sr") if units == "SIUnits" else (_ARCSEC2, "W/m2/arcsec2")


def calibrate_frame(f, lam, dlam, distance, xpsiz, ypsiz, units="ExtragalacticUnits"):
    """f [nlambda, ny, nx] luminosity per pixel -> neutral surface brightness."""
    f = np.asarray(f, dtype=np.float64) / np.asarray(dlam)[:, None, None]
    area = 2.0 * math.atan(xpsiz / (2.0 * distance)) * 2.0 * math.atan(ypsiz / (2.0 * distance))
    f = f / area / (4.0 * math.pi * distance * distance)
    fac, _ = _sb_out(units)
    return np.asarray(lam)[:, None, None] * f * fac


def calibrate_sed(F, lam, dlam, distance):
    """F [nlambda] luminosity -> neutral flux density lambda F_lambda (W/m2)."""
    return np.asarray(lam) * np.asarray(F) / np.asarray(dlam) / (4.0 * math.pi * distance * distance)


def write_fits(path, cube, header=()):
    """A primary-HDU FITS image of 64-bit floats (NAXIS1 = x, NAXIS2 = y, NAXIS3 = wavelength)."""
    cube = np.asarray(cube, dtype=np.float64)
    if cube.ndim == 2:
        cube = cube[None]
    nl, ny, nx = cube.shape
    cards = [("SIMPLE", True, "conforms to FITS standard"), ("BITPIX", -64, "IEEE double"), ("NAXIS", 3, ""),
             ("NAXIS1", nx, ""), ("NAXIS2", ny, ""), ("NAXIS3", nl, "")] + list(header)

    def card(k, v, c):
        if isinstance(v, bool):
            s = "%20s" % ("T" if v else "F")
        elif isinstance(v, (int, np.integer)):
            s = "%20d" % v
        elif isinstance(v, float):
            s = "%20.12E" % v
        else:
            s = "'%-8s'" % str(v).replace("'", "''")
        line = "%-8s= %s / %s" % (k, s, c) if c else "%-8s= %s" % (k, s)
        return line[:80].ljust(80)

    text = "".join(card(*c) for c in cards) + "END".ljust(80)
    text += " " * (-len(text) % 2880)
    data = cube.astype(">f8").tobytes()
    data += b"\0" * (-len(data) % 2880)
    with open(path, "wb") as f:
        f.write(text.encode("ascii"))
        f.write(data)


def read_fits(path):
    """Reads back what write_fits wrote (for checks)."""
    with open(path, "rb") as f:
        raw = f.read()
    hdr = {}
    i = 0
    while True:
        c = raw[i:i + 80].decode("ascii")
        i += 80
        if c.startswith("END"):
            break
        if c[8:10] == "= ":
            v = c[10:].strip()
            if v.startswith("'"):
                v = v[1:v.index("'", 1)]
            else:
                v = v.split("/")[0]
            hdr[c[:8].strip()] = v.strip()
    i += -i % 2880
    nx, ny, nl = int(hdr["NAXIS1"]), int(hdr["NAXIS2"]), int(hdr["NAXIS3"])
    return np.frombuffer(raw[i:i + 8 * nx * ny * nl], dtype=">f8").reshape(nl, ny, nx), hdr


def write_instruments(ctx, model, outdir, prefix, units="ExtragalacticUnits"):
    """Writes every instrument's frames and SED; returns the paths written."""
    os.makedirs(outdir, exist_ok=True)
    lam, dlam = model.wavelengthGrid.lambdav, model.wavelengthGrid.dlambdav
    _, sbu = _sb_out(units)
    paths = []
    for i, ins in enumerate(model.instruments):
        name = getattr(ins, "instrumentName", "instrument%d" % i)
        cube, sed = ctx.read_instrument(i)
        d = ins.distance
        if ins.type == A.INSTR_FULL:
            frames = list(_FULL_FRAMES)
            if model.dustEmission:
                frames += [("dust", None), ("dustscattered", A.FULL_DUSSCA)]
            frames += [("scatteringlevel%d" % (n + 1), A.FULL_NBASE + n) for n in range(ins.scatteringLevels)]
            seds = [sed[A.FULL_TOT], sed[A.FULL_STRDIR], sed[A.FULL_STRSCA], sed[A.FULL_DUSDIR] + sed[A.FULL_DUSSCA],
                    sed[A.FULL_DUSSCA], sed[A.FULL_TRA]]
            seds += [sed[A.FULL_NBASE + n] for n in range(ins.scatteringLevels)]
            snames = _FULL_SEDS + ["%d-times scattered flux" % (n + 1) for n in range(ins.scatteringLevels)]
        else:
            frames = [("total", 0)] if cube is not None else []
            seds = [sed[0]] if ins.type in (A.INSTR_SED, A.INSTR_SIMPLE) else []
            snames = ["total flux"] * len(seds)
        if cube is not None:
            xps, yps = ins.fieldOfViewX / ins.pixelsX, ins.fieldOfViewY / ins.pixelsY
            for fname, comp in frames:
                f = cube[A.FULL_DUSDIR] + cube[A.FULL_DUSSCA] if comp is None else cube[comp]
                sb = calibrate_frame(f, lam, dlam, d, xps, yps, units)
                p = os.path.join(outdir, "%s_%s_%s.fits" % (prefix, name, fname))
                write_fits(p, sb, [("BUNIT", sbu, "neutral surface brightness"),
                                   ("CDELT1", xps / 3.08567758e16, "pixel size (pc)"),
                                   ("CDELT2", yps / 3.08567758e16, "pixel size (pc)")])
                paths.append(p)
        if seds:
            p = os.path.join(outdir, "%s_%s_sed.dat" % (prefix, name))
            with open(p, "w") as f:
                f.write("# column 1: lambda (micron)\n")
                for k, n in enumerate(snames):
                    f.write("# column %d: %s; lambda*F_lambda (W/m2)\n" % (k + 2, n))
                cols = [calibrate_sed(s, lam, dlam, d) for s in seds]
                for ell in range(len(lam)):
                    f.write(" ".join(["%.8e" % (lam[ell] * 1e6)] + ["%.8e" % c[ell] for c in cols]) + "\n")
            paths.append(p)
    return paths
