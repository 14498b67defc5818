"""Shared test utilities: seeded rays, deterministic cell densities, statistical comparison."""
import math

import numpy as np

from skirt7_b200 import _abi as A
from skirt7_b200.scene import CartesianDustGrid


def seeded_rays(n, extent, seed=0, frac_outside=0.1, disk=None):
    """Rays with origins uniform in the box (and a fraction outside it, to exercise the entry
    logic), or drawn from a stellar disk, and isotropic directions."""
    rng = np.random.default_rng(seed)
    ex = np.array(extent, dtype=np.float64)
    lo, hi = ex[:3], ex[3:]
    r = lo + rng.random((n, 3)) * (hi - lo)
    nout = int(frac_outside * n)
    if nout:
        c = 0.5 * (lo + hi)
        r[:nout] = c + (rng.random((nout, 3)) - 0.5) * 3.0 * (hi - lo)
    if disk is not None:
        hR, hz = disk
        nd = n // 3
        R = hR * rng.gamma(2.0, 1.0, nd)
        ph = rng.uniform(0, 2 * math.pi, nd)
        z = rng.laplace(0, hz, nd)
        r[nout:nout + nd] = np.stack([R * np.cos(ph), R * np.sin(ph), z], 1)
    cost = rng.uniform(-1, 1, n)
    phi = rng.uniform(0, 2 * math.pi, n)
    st = np.sqrt(1 - cost ** 2)
    k = np.stack([st * np.cos(phi), st * np.sin(phi), cost], 1)
    return np.ascontiguousarray(r), np.ascontiguousarray(k)


def axis_rays(extent, planes_x=None):
    """Edge cases: axis-aligned directions, origins on cell planes, corners, grazing rays."""
    xmin, ymin, zmin, xmax, ymax, zmax = extent
    rs, ks = [], []
    dirs = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1),
            (1 / math.sqrt(2), 1 / math.sqrt(2), 0), (1 / math.sqrt(3),) * 3]
    origins = [(0, 0, 0), (xmin, 0, 0), (xmax, ymax, zmax), (xmin * 2, 0.1 * ymax, 0.1 * zmax),
               (0.3 * xmax, 0.7 * ymin, 0.2 * zmin), (xmin, ymin, zmin)]
    if planes_x is not None:
        origins.append((planes_x[len(planes_x) // 3], 0.01 * ymax, 0.02 * zmax))
    for o in origins:
        for d in dirs:
            for sgn in (1, -1):
                rs.append(o)
                ks.append(tuple(sgn * v for v in d))
    return np.array(rs, dtype=np.float64), np.array(ks, dtype=np.float64)


def cell_center_density(model):
    """Deterministic densities: the dust density at the centre of each Cartesian cell."""
    g = model.dustGrid
    assert isinstance(g, CartesianDustGrid)
    xc = 0.5 * (g.xv[1:] + g.xv[:-1])
    yc = 0.5 * (g.yv[1:] + g.yv[:-1])
    zc = 0.5 * (g.zv[1:] + g.zv[:-1])
    X, Y, Z = np.meshgrid(xc, yc, zc, indexing="ij")   # cell m = k + nz*j + nz*ny*i
    model.normalise()
    rho = np.zeros((len(model.dustComps), X.size))
    for h, d in enumerate(model.dustComps):
        geo = d.geometry
        hR, hz = geo.radialScale, geo.axialScale
        rho0 = 1.0 / (hR * hR * 2.0 * math.pi * 2.0 * hz)
        R = np.sqrt(X ** 2 + Y ** 2)
        rho[h] = (d.norm * rho0 * np.exp(-R / hR) * np.exp(-np.abs(Z) / hz)).reshape(-1)
    return rho


def block_sum(img, f):
    ny, nx = img.shape[-2:]
    return img[..., : ny // f * f, : nx // f * f].reshape(img.shape[:-2] + (ny // f, f, nx // f, f)).sum((-3, -1))


def zscores(a_batches, b_batches):
    """Per-element z of the difference of two batch means (standard errors from the batches)."""
    a = np.asarray(a_batches)
    b = np.asarray(b_batches)
    ma, mb = a.mean(0), b.mean(0)
    va = a.var(0, ddof=1) / len(a)
    vb = b.var(0, ddof=1) / len(b)
    s = np.sqrt(va + vb)
    ok = s > 0
    z = np.zeros_like(ma)
    z[ok] = (ma[ok] - mb[ok]) / s[ok]
    return z, ok
