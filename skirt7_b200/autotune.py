"""Launch-shape autotuner for the wavefront tracer.

Two choices set how a phase maps onto the device:
  pool    packets in flight per wave: more packets fill the traversal pass with more jobs per lane
          (fewer partly idle waves at the tail of the phase) but cost pool and job memory and a
          longer event pass;
  blocks  traversal blocks per wave: resident blocks per SM times the SM count (persistent lanes).
The tuner times short trial phases of the caller's own workload (a slice of its packets, same
wavelengths and seed stream) for each candidate on the device, keeps the fastest, and caches the
choice per workload class (grid type, cell-count decade, wavelengths, instruments, phase) for
the process, optionally in a JSON file.
"""
import json
import math
import os

from . import _abi as A

_CACHE = {}


def workload_key(ctx, phase, nell):
    m = ctx.model
    g = m.dustGrid
    gtype = type(g).__name__ if g is not None else "none"
    return "%s|c%d|l%d|i%d|p%d" % (gtype, int(math.log10(max(ctx.ncells, 1))), nell, len(m.instruments), phase)


def tune(ctx, phase, ells, npp, seed=777, precision=A.PREC_FP32, sample=None, pools=None, blocks=None,
         path=None, sms=148):
    """Returns {'pool': P, 'blocks': B, 'ms': t, 'trials': [...]} for the phase of `ctx`; the
    result is cached per workload class.  sample: packets per wavelength of each trial (default
    npp/8, at least 2^14)."""
    key = workload_key(ctx, phase, len(ells))
    if key in _CACHE:
        return _CACHE[key]
    if path and os.path.exists(path):
        with open(path) as f:
            disk = json.load(f)
        if key in disk:
            _CACHE[key] = disk[key]
            return disk[key]
    sample = int(sample or max(1 << 14, npp // 8))
    total = sample * len(ells)
    pools = pools or sorted({min(total, p) for p in (1 << 18, 1 << 19, 1 << 20, 1 << 21)})
    blocks = blocks or [2 * sms, 3 * sms]
    trials = []
    for P in pools:
        for B in blocks:
            ctx.reset_tallies()
            ctx.run_phase(phase, ells, npp, 0, sample, seed=seed, precision=precision, blocks=B, pool=P)
            ctx.sync()
            ms = ctx.last_phase_ms()
            trials.append((ms, P, B))
    ctx.reset_tallies()
    ms, P, B = min(trials)
    res = {"pool": int(P), "blocks": int(B), "ms": ms, "sample": sample,
           "trials": [{"ms": t, "pool": p, "blocks": b} for t, p, b in trials]}
    _CACHE[key] = res
    if path:
        disk = {}
        if os.path.exists(path):
            with open(path) as f:
                disk = json.load(f)
        disk[key] = res
        with open(path, "w") as f:
            json.dump(disk, f, indent=1)
    return res
