"""Launch autotuner for the wavefront tracer.

Four choices set how a phase maps onto the device:
  pool     packets in flight per wave: more packets fill the traversal pass with more jobs per lane
           and need fewer waves (fewer partly idle wave tails) but cost pool and job memory;
  refill   packets per warp refill: how many lanes of a traversal warp wait for a new job before
           the warp takes new jobs -- one job fetch and start per group of lanes instead of one per
           lane, against lanes idling until the group is complete;
  blocks   traversal blocks per wave: resident blocks per SM times the SM count (persistent lanes);
  records  grid-node layout of a tree grid: 32-byte lattice leaf records (trees split at
           midpoints) or 64-byte rope records holding the FP32 boxes.
The tuner times short trial phases of the caller's own workload (a slice of its packets, same
wavelengths and seed stream) on the device, coordinate by coordinate from the library's defaults,
keeps the fastest, and caches the choice per workload class (grid type, cell-count decade,
wavelengths, instruments, phase) for the process, optionally in a JSON file.  Every choice
leaves the results unchanged (each packet's random stream is keyed by the packet, not by where
it runs): only the time changes.
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


def _trial(ctx, phase, ells, npp, sample, seed, precision, launch):
    ctx.reset_tallies()
    ctx.run_phase(phase, ells, npp, 0, sample, seed=seed, precision=precision, launch=launch)
    ctx.sync()
    return ctx.last_phase_ms()


def tune(ctx, phase, ells, npp, seed=777, precision=A.PREC_FP32, sample=None, pools=None, refills=(4, 8, 16),
         blocks=None, path=None, sms=148, records=False):
    """Returns {'pool': P, 'refill': R, 'blocks': B, 'ms': t, 'trials': [...]} (and 'records' when
    records=True on a tree grid) for the phase of `ctx`; the result is cached per workload class.
    sample: packets per wavelength of each trial (default npp/8, at least 2^14, at most npp)."""
    key = workload_key(ctx, phase, len(ells))
    if key in _CACHE:
        return _CACHE[key]
    if path and os.path.exists(path):
        with open(path) as f:
            disk = json.load(f)
        if key in disk:
            _CACHE[key] = disk[key]
            return disk[key]
    sample = int(min(npp, sample or max(1 << 14, npp // 8)))
    total = sample * len(ells)
    pools = pools or sorted({min(total, p) for p in (1 << 21, 1 << 22, 1 << 23)})
    blocks = blocks or [0, 3 * sms]
    best = {"pool": pools[0], "refill": 8 if 8 in refills else refills[0], "blocks": blocks[0]}
    trials = []

    def run(launch):
        ms = _trial(ctx, phase, ells, npp, sample, seed, precision, launch)
        trials.append(dict(launch, ms=ms))
        return ms

    best_ms = run(best)
    for name, values in (("pool", pools), ("refill", refills), ("blocks", blocks)):
        start = best[name]                       # timed already (with the other coordinates as now)
        for v in values:
            if v == start:
                continue
            cand = dict(best, **{name: v})
            ms = run(cand)
            if ms < best_ms:
                best, best_ms = cand, ms
    res = dict(best, ms=best_ms, sample=sample, trials=trials)
    if records and type(ctx.model.dustGrid).__name__ == "TreeDustGrid":
        res["records"] = tune_records(ctx.model, phase, ells, npp, sample, seed, precision, best, best_ms,
                                      ctx_device=getattr(ctx, "device", 0))
    ctx.reset_tallies()
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


def tune_records(model, phase, ells, npp, sample, seed, precision, launch, lattice_ms, ctx_device=0):
    """Times the same trial on a context whose tree uses the 64-byte rope records; returns the
    faster layout's name ('lattice' or 'rope')."""
    from . import runtime
    old = os.environ.get("SKG_TREE_RECORDS")
    os.environ["SKG_TREE_RECORDS"] = "rope"
    try:
        ctx = runtime.Context(model, device=ctx_device)
    finally:
        if old is None:
            os.environ.pop("SKG_TREE_RECORDS", None)
        else:
            os.environ["SKG_TREE_RECORDS"] = old
    try:
        ms = _trial(ctx, phase, ells, npp, sample, seed, precision, launch)
    finally:
        ctx.close()
    return "rope" if ms < lattice_ms else "lattice"
