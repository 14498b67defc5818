"""TEST INFRASTRUCTURE: writes tests/golden/tracer_<scene>.npz, the oracle's stellar emission phase
(the restated life cycle, oracle/oracle.cpp, MonteCarloSimulation.cpp:259-543) on the
deterministic scenes of scenes.py, as batch statistics the device is compared against
(tests/test_config_tracer_gpu.py).

Per wavelength the oracle runs B independent batches (seeds far apart: its threads seed their
streams seed + thread) with packet counts chosen so that the standard error of every frame total
is about 0.1 % or less -- small enough to resolve the 0.3 % total-flux tolerance.  Stored per
wavelength: the mean and standard error of the batch means of every frame's total, of every
frame's 32x32-pixel block sums, and (when the scene keeps absorption) of the absorbed luminosity
summed over groups of cells; plus the grid's signature, the packet counts and the oracle's time.

Usage: python tests/golden/make_tracer_fixtures.py [octree_pan] [kdtree_point] [voronoi_clumpy]
       [--threads N] [--scale F]   (F scales every packet count; default 1)
"""
import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import scenes  # noqa: E402
import oracle  # noqa: E402  (put on the path by scenes)

# packets per wavelength over all batches (index of the wavelength in the scene's subset)
SCENES = {
    "octree_pan": dict(model=scenes.octree_pan_model, spec=scenes.OCTREE, ells=scenes.OCTREE_ELLS,
                       packets=[4.4e6, 1.2e6, 3.0e5], batches=20),
    "kdtree_point": dict(model=scenes.kdtree_point_model, spec=scenes.KDTREE, ells=scenes.KDTREE_ELLS,
                         packets=[3.0e6, 4.0e5, 4.0e5], batches=20),
    "voronoi_clumpy": dict(model=scenes.voronoi_clumpy_model, spec=None, ells=[0], packets=[4.8e6], batches=20),
}


def build(name, threads):
    cfg = SCENES[name]
    full = cfg["model"]()
    if cfg["spec"] is not None:
        full.dustGrid = scenes.tree_grid(full, cfg["spec"], nthreads=threads)
        sig = {"tree_hash": scenes.tree_hash(full.dustGrid), "ncells": int(full.dustGrid.ncells)}
    else:
        full.dustGrid = scenes.voropp_mesh(scenes.voronoi_sites())
        sig = scenes.voronoi_signature(full.dustGrid)
    m = scenes.wavelength_subset(full, cfg["ells"])
    m.rho = scenes.centre_density(m)
    return m, sig


def stats(x):
    x = np.asarray(x, dtype=np.float64)
    return x.mean(0), x.std(0, ddof=1) / np.sqrt(len(x))


def run(name, threads, scale):
    cfg = SCENES[name]
    t0 = time.time()
    m, sig = build(name, threads)
    frames = [i for i, ins in enumerate(m.instruments) if ins.type != 0]
    out = {"signature": json.dumps(sig), "ells": np.array(cfg["ells"]), "batches": cfg["batches"]}
    secs, pk = 0.0, []
    for e in range(len(cfg["ells"])):
        B = cfg["batches"]
        npp = int(cfg["packets"][e] * scale / B)
        tot, blk, lab, labt = [], [], [], []
        for b in range(B):
            r = oracle.simulate(m, npp, nthreads=threads, seed=7000003 * (b + 1) + 1009 * e, ells=[e])
            secs += r["stats"]["seconds"]
            cubes = [r["cubes"][i][0, e] for i in frames]
            tot.append([c.sum() for c in cubes])
            blk.append([scenes.block_sums(c) for c in cubes])
            if m.writeAbsorption:
                la = r["labs_stel"][:, e:e + 1]
                lab.append(scenes.labs_groups(m.dustGrid, la)[:, 0])
                labt.append(la.sum())
            npp_run = int(r["stats"]["npp"])
        pk.append(npp_run * B)
        for key, val in (("tot", tot), ("blk", blk), ("lab", lab), ("labtot", labt)):
            if len(val):
                mu, se = stats(val)
                out["%s_mean_%d" % (key, e)] = mu
                out["%s_sem_%d" % (key, e)] = se
        rel = out["tot_sem_%d" % e] / out["tot_mean_%d" % e]
        print("%s ell %d: %d packets, frame-total standard errors %s" %
              (name, cfg["ells"][e], pk[-1], np.array2string(rel, precision=5)), flush=True)
    out["packets"] = np.array(pk)
    out["oracle_seconds"] = secs
    out["threads"] = threads
    np.savez_compressed(os.path.join(HERE, "tracer_%s.npz" % name), **out)
    print("%s: %.0f s of packet loops, %.0f s in all" % (name, secs, time.time() - t0), flush=True)


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("scenes", nargs="*", default=list(SCENES))
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--scale", type=float, default=1.0)
    a = ap.parse_args()
    for s in a.scenes:
        run(s, a.threads, a.scale)
