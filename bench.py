"""Benchmark: photon packets/s of SKIRT7's packet life cycle on the device.

Default workload (the headline): the stellar-emission phase of the panchromatic octree disk galaxy
(50 log-spaced wavelengths 0.1-10 micron, octree max level 10 with cell mass fraction < 1e-6,
three 512x512 frames at 0/60/88 degrees, FP32 geometry with FP64 tallies).  --workload selects the
other configurations of the hot path with the same machinery:
  cartesian_oligo   oligochromatic disk on a 100x100x50 Cartesian grid, 300x300 frame + SED at 88 deg
  voronoi_clumpy    clumpy dust disk (10^4 clumps, 25 % of the mass) on a 10^6-site Voronoi grid
  kdtree_dust       panchromatic disk + point source on a k-d tree, 100 wavelengths 0.1-1000 micron,
                    one step = stellar phase with absorption tallies, two dust self-absorption
                    cycles and the dust-emission phase (emission spectra recomputed before
                    each dust phase)

One step = the workload's phases (a sequence of waves: an event pass and a traversal pass each)
over all wavelengths with --packets packets per wavelength per GPU (by default the
configuration's count: 10^7, 10^8 for the Voronoi workload).  A step ends when its phases have finished (the host has seen the last
wave's counters), so every step times exactly its own waves.  Ranks (one process per GPU; with
--gpus N and no torchrun environment the script starts the N ranks itself) run disjoint packet
ranges of one simulation and all-reduce the frames over NCCL at the end of each step (weak
scaling: the packets per GPU are fixed).  `value` is device-timed; `e2e` is the same metric
through the C ABI with the tallies read back into host memory every step.

--impl reference times the reference's algorithm on the host cores: the oracle (a scalar FP64
restatement of the reference's life cycle, oracle/oracle.cpp) with all host threads on a
bounded sample of the same workload.  Its inputs are built on the host alone -- the tree by the
oracle's restated subdivision with the reference's node classes (oracle/_ref), the Voronoi grid
by Voro++, the cell densities by the oracle's DustSystem sampling -- so that arm loads none of
this repository's device code.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MEASURED = os.path.join(ROOT, "MEASURED_PEAKS.json")
WORKLOADS = ("octree_pan", "cartesian_oligo", "voronoi_clumpy", "kdtree_dust")


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=3)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="octree_pan", choices=WORKLOADS)
    p.add_argument("--packets", type=float, default=None,
                   help="packets per wavelength per GPU per step (default: the configuration's, 10^7; "
                        "10^8 for voronoi_clumpy)")
    p.add_argument("--e2e-steps", type=int, default=5, help="steps of the end-to-end leg (at most --steps)")
    p.add_argument("--plain-packets", type=float, default=1e6,
                   help="packets per wavelength of the plain-GPU leg (one thread per packet; 0 = skip)")
    p.add_argument("--no-autotune", action="store_true",
                   help="run with the library's default launch choices instead of the autotuner's (set-up, untimed)")
    p.add_argument("--max-level", type=int, default=10)
    p.add_argument("--mass-fraction", type=float, default=1e-6)
    p.add_argument("--nlambda", type=int, default=50)
    p.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    p.add_argument("--cpu-seconds", type=float, default=15.0, help="target duration of the CPU baseline sample")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--tree-cache", default=os.path.join(ROOT, ".bench_cache", "octree.npz"),
                   help="cache of the headline octree between runs of the same size (git-ignored)")
    p.add_argument("--serving", type=int, default=256,
                   help="requests of the fit-variant serving leg (Poisson 20/s; 0 = skip)")
    p.add_argument("--serving-rates", type=lambda v: [float(x) for x in v.split(",") if x], default=[10.0],
                   help="further arrival rates (per s) of the same requests, comma-separated ('' = none)")
    p.add_argument("--serving-impl", default="native", choices=["native", "python"],
                   help="the serving loop: the C ABI server (skg_submit/skg_poll) or the Python one")
    p.add_argument("--phase-only", action="store_true",
                   help="run one stellar phase of the workload (--packets per wavelength, the library's default "
                        "launch choices) and print its counters and pass times: the program the ncu captures "
                        "of a phase run")
    a = p.parse_args()
    if a.packets is None:
        a.packets = WORKLOAD_PACKETS[a.workload]
    return a


# packets per wavelength of a step: the configurations' counts (the Cartesian workload runs 10
# times configuration 1's 10^6 so that the device is filled)
WORKLOAD_PACKETS = {"octree_pan": 1e7, "cartesian_oligo": 1e7, "voronoi_clumpy": 1e8, "kdtree_dust": 1e7}


def peaks():
    try:
        with open(MEASURED) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons during the timed region."""

    def __init__(self, index=0):
        self.samples = []
        self.index = index
        self._stop = threading.Event()
        self._t = None

    def start(self):
        def run():
            q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap")
            while not self._stop.is_set():
                try:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), "--query-gpu=" + q,
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5).stdout.strip()
                    if out:
                        self.samples.append([s.strip() for s in out.split(",")])
                except Exception:
                    pass
                self._stop.wait(0.2)
        self._t = threading.Thread(target=run, daemon=True)
        self._t.start()

    def stop(self):
        self._stop.set()
        if self._t:
            self._t.join(timeout=10)
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 3 + i and "Active" in s[3 + i]
                          and "Not" not in s[3 + i]})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


# ---------------------------------------------------------------------------------------------
# workloads

KDTREE_MASS_FRACTION = 3e-7     # the k-d tree workload's cell mass fraction: ~4.2*10^6 leaves


class Workload:
    """A configuration: its scene, the phases of one step and the algorithmic bytes of its
    traversal pass.  host=True builds the grid on the host alone (the reference arm: the oracle's
    restated tree subdivision with the device builder's node sampler, so the tree is the same;
    Voro++ for the Voronoi grid); otherwise on the device."""

    def __init__(self, args, device, host=False):
        from skirt7_b200 import _abi as A
        from skirt7_b200 import models
        from skirt7_b200.scene import KPC
        self.name = args.workload
        self.grid_s = 0.0
        self.dust_phase = False
        self.selfabs_cycles = 0
        ext = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)
        t0 = time.time()
        if self.name == "octree_pan":
            self.model = models.pan_disk(nlambda=args.nlambda, inclinations=(0, 60, 88), npix=512)
            self.model.dustGrid, self.grid_s = get_tree(args, self.model, device, host)
            self.metric = "photon packets/s (stellar emission, octree pan disk)"
            self.desc = ("panchromatic octree disk galaxy: %d wavelengths 0.1-10 micron, octree max level %d, mass "
                         "fraction %g (%d leaves), 3 frames 512x512 at 0/60/88 deg" %
                         (args.nlambda, args.max_level, args.mass_fraction, self.model.dustGrid.ncells))
        elif self.name == "cartesian_oligo":
            self.model = models.oligo_disk()
            self.metric = "photon packets/s (oligochromatic disk, Cartesian grid)"
            self.desc = ("oligochromatic disk galaxy at 0.55 micron: 100x100x50 Cartesian grid, tau_V 1, "
                         "300x300 frame + SED at 88 deg")
        elif self.name == "voronoi_clumpy":
            import numpy as np
            self.model = models.clumpy_disk()
            rng = np.random.default_rng(77)
            n = 1000000
            lo, hi = np.array(ext[:3]), np.array(ext[3:])
            base = self.model.dustComps[0].geometry.geometry
            d = np.zeros((0, 3))
            while len(d) < int(0.8 * n):
                q = models.sample_expdisk(base, n, rng).reshape(-1, 3)
                d = np.concatenate([d, q[np.all((q > lo) & (q < hi), axis=1)]])
            sites = np.concatenate([d[: int(0.8 * n)], lo + rng.random((n - int(0.8 * n), 3)) * (hi - lo)])
            if host:
                self.model.dustGrid = _oracle().voronoi_mesh(sites, ext)
            else:
                from skirt7_b200 import runtime
                self.model.dustGrid = runtime.build_voronoi(sites, ext, device)
            self.grid_s = time.time() - t0
            self.metric = "photon packets/s (clumpy disk, Voronoi grid)"
            self.desc = ("clumpy dust disk at 0.55 micron (tau_V 5, 10^4 cubic-spline clumps with 25 %% of the "
                         "mass): Voronoi grid of %d sites (80 %% from the disk density, 20 %% uniform), 300x300 "
                         "frame at 88 deg" % self.model.dustGrid.ncells)
        else:
            self.model = models.pan_disk(nlambda=100, lmin=0.1e-6, lmax=1000e-6, inclinations=(60,), npix=512,
                                         point_fraction=0.1, dust_emission=True, write_absorption=True)
            if host:
                self.model.dustGrid, _, _ = _oracle().tree_build(self.model, A.GRID_BINTREE, ext, 6, 30,
                                                                 KDTREE_MASS_FRACTION, 100, 4357, sampler=1,
                                                                 nthreads=os.cpu_count() or 1)
            else:
                from skirt7_b200 import runtime
                self.model.dustGrid = runtime.build_tree(self.model, A.GRID_BINTREE, ext, minLevel=6, maxLevel=30,
                                                         maxMassFraction=KDTREE_MASS_FRACTION, sampleCount=100,
                                                         seed=4357, device=device)
            self.grid_s = time.time() - t0
            self.dust_phase = True
            self.selfabs_cycles = 2
            self.metric = "photon packets/s (stellar + dust self-absorption + dust emission, k-d tree pan disk)"
            self.desc = ("panchromatic disk + point source (10 %% of L) with grey-body dust emission: k-d tree "
                         "(alternating, %d leaves), 100 wavelengths 0.1-1000 micron, 512x512 frame at 60 deg; "
                         "a step is the stellar phase, 2 dust self-absorption cycles and the dust-emission phase "
                         "(dust emission spectra recomputed before each dust phase)" % self.model.dustGrid.ncells)
        self.model.rho = None
        self.gtype = type(self.model.dustGrid).__name__

    def alg_bytes(self, c, fp32):
        """Algorithmic bytes of the traversal pass from the exact counters.  Per cell step: tree --
        the leaf box (24 B) and density (4 B), plus the followed rope (4 B); Cartesian -- the crossed
        plane (4 B) and the density (4 B); Voronoi -- the density (4 B) plus, per neighbour entry
        tested, its bisector plane (16 B) and id (4 B).  Per absorption tally 8 B.  The FP64 walk
        doubles the box, plane and density words."""
        f = 1 if fp32 else 2
        if self.gtype == "CartesianDustGrid":
            b = c["steps"] * 8 * f
        elif self.gtype == "VoronoiDustGrid":
            b = c["steps"] * 4 * f + c["nbr_scanned"] * (16 * f + 4)
        else:
            b = c["steps"] * 28 * f + c["nbr_scanned"] * 4
        return b + 8 * c["absorb_adds"]

    # DRAM bytes per cell step of the headline traversal pass (FP32 walk), from one ncu capture
    # (dram__bytes_read.sum + dram__bytes_write.sum over the traversal launches of a stellar phase
    # of this workload, divided by that phase's cell steps); roofline.traffic scales it by a
    # launch's cell steps, and says so.  Other workloads report no traffic.
    NCU_DRAM_BYTES_PER_STEP = {"octree_pan": 11.76}

    def frames(self):
        from skirt7_b200 import _abi as A
        return [i for i, ins in enumerate(self.model.instruments) if ins.type != A.INSTR_SED]


def _oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def get_tree(args, model, device, host=False):
    """The octree of the headline workload: built on the device (device-sampled subdivision), or
    on the host by the oracle's restated subdivision with the same node sampler (the same tree);
    cached across runs of the same size."""
    import numpy as np
    from skirt7_b200 import _abi as A
    from skirt7_b200.scene import KPC, TreeDustGrid
    ext = (-20 * KPC, -20 * KPC, -2 * KPC, 20 * KPC, 20 * KPC, 2 * KPC)
    key = "L%d_f%g" % (args.max_level, args.mass_fraction)
    if os.path.exists(args.tree_cache):
        z = np.load(args.tree_cache)
        if str(z["key"]) == key:
            return TreeDustGrid(A.GRID_OCTREE, ext, z["box"], z["child"], z["father"], z["cell"], z["dir"],
                                z["off"], z["ids"]), 0.0
    t0 = time.time()
    if host:
        tree, _, _ = _oracle().tree_build(model, A.GRID_OCTREE, ext, 2, args.max_level, args.mass_fraction, 100, 4357,
                                          sampler=1, nthreads=os.cpu_count() or 1)
    else:
        from skirt7_b200 import runtime
        tree = runtime.build_tree(model, A.GRID_OCTREE, ext, minLevel=2, maxLevel=args.max_level,
                                  maxMassFraction=args.mass_fraction, sampleCount=100, seed=4357, device=device)
    dt = time.time() - t0
    try:
        os.makedirs(os.path.dirname(args.tree_cache), exist_ok=True)
        np.savez(args.tree_cache, key=key, box=tree.node_box, child=tree.node_child, father=tree.node_father,
                 cell=tree.node_cell, dir=tree.node_dir, off=tree.nbr_offsets, ids=tree.nbr_ids)
    except Exception:
        pass
    return tree, dt


# ---------------------------------------------------------------------------------------------
# the reference arm

def run_reference(args, rank, world):
    """The reference algorithm on the host cores (rank 0 only); everything on the host."""
    if rank != 0:
        return
    oracle = _oracle()
    oracle.build()
    threads = os.cpu_count() or 1
    wl = Workload(args, 0, host=True)
    model = wl.model
    t0 = time.time()
    model.rho = oracle.sample_density(model, nthreads=threads, seed=4357)   # DustSystem.cpp:145-172
    density_s = time.time() - t0
    kw = dict(dust_emission_phase=wl.dust_phase, selfabs_cycles=wl.selfabs_cycles)
    # calibrate the sample to about --cpu-seconds per step
    probe = oracle.simulate(model, args.packets * args.gpus, nthreads=threads, seed=1, max_packets=2000, **kw)
    rate = probe["stats"]["packets"] / max(probe["stats"]["seconds"], 1e-6)
    sample = int(max(1000, min(5e6, rate * args.cpu_seconds)))
    vals = []
    for s in range(args.warmup + args.steps):
        r = oracle.simulate(model, args.packets * args.gpus, nthreads=threads, seed=100 + s, max_packets=sample, **kw)
        if s >= args.warmup:
            vals.append(r["stats"]["packets"] / r["stats"]["seconds"])
    v = statistics.mean(vals)
    line = {"metric": wl.metric, "value": v, "unit": "packets/s",
            "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * sample / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": _config(args, wl),
            "setup": {"grid_build_s": wl.grid_s, "density_s": density_s, "grid": "host (oracle)"},
            "cpu_baseline": {"value": v, "unit": "packets/s", "cores": threads, "kind": "port",
                             "sample": "%d packets of the workload (all wavelengths%s) per step" %
                                       (sample, ", all phases" if wl.dust_phase else "")},
            "e2e": {"value": v, "unit": "packets/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "native_so_loaded": _native_libs()}
    print(json.dumps(line))


def _native_libs():
    """Shared objects of this repository mapped into the process (the reference arm must show
    oracle/ libraries only)."""
    libs = set()
    try:
        with open("/proc/self/maps") as f:
            for ln in f:
                p = ln.split()[-1] if ln.strip() else ""
                if p.endswith(".so") and p.startswith(ROOT):
                    libs.add(os.path.relpath(p, ROOT))
    except OSError:
        pass
    return sorted(libs)


def _config(args, wl):
    return {"workload": wl.desc, "name": wl.name,
            "packets_per_wavelength_per_gpu": args.packets, "nlambda": wl.model.wavelengthGrid.Nlambda,
            "cells": wl.model.dustGrid.ncells,
            "geometry_precision": args.precision, "tallies": "fp64",
            "l2": "L2 flushed between timed steps (a 256 MB write on the launching stream, outside the events)",
            "parallelism": "dp%d (packet ranges per GPU, NCCL all-reduce of frames per step)" % args.gpus}


# ---------------------------------------------------------------------------------------------
# the device arm

def spawn_ranks(args):
    """--gpus N without a torchrun environment: start the N ranks (one process per GPU) under
    torch.distributed.run on this node and return its exit status."""
    import socket
    sock = socket.socket()
    sock.bind(("127.0.0.1", 0))
    port = sock.getsockname()[1]
    sock.close()
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(args.gpus),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)

    import numpy as np
    import torch
    from skirt7_b200 import _abi as A
    from skirt7_b200 import runtime

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    wl = Workload(args, local)
    model = wl.model
    ctx = runtime.Context(model, device=local)
    nl = model.wavelengthGrid.Nlambda
    ells = np.arange(nl, dtype=np.int32)
    npp_rank = int(args.packets)
    Npp = npp_rank * world                      # the simulation's packets per wavelength
    first = rank * npp_rank
    prec = A.PREC_FP64 if args.precision == "fp64" else A.PREC_FP32
    # a dedicated stream: the launches, the events and the collective all go on it
    tstream = torch.cuda.Stream(device=local)
    handle = tstream.cuda_stream
    fr = wl.frames()
    sizes = [_tally_len(ctx, i) for i in fr]
    # per-rank frames handed to the all-reduce (Instrument::sumResults, Instrument.cpp:57-65)
    red = [torch.zeros(n, dtype=torch.float64, device="cuda") for n in sizes] if dist else None
    phases = ([A.PHASE_STELLAR] + [A.PHASE_DUST_SELFABS] * wl.selfabs_cycles +
              ([A.PHASE_DUST_EMISSION] if wl.dust_phase else []))
    if args.phase_only:
        ctx.run_phase(A.PHASE_STELLAR, ells, Npp, first, npp_rank, seed=5, precision=prec)
        ctx.sync()
        ev_ms, trav_ms, waves = ctx.phase_times()
        print(json.dumps({"workload": wl.name, "packets_per_wavelength": npp_rank, "counters": ctx.counters(),
                          "event_pass_ms": ev_ms, "traversal_pass_ms": trav_ms, "waves": waves}))
        ctx.close()
        return
    # launch choices (packets in flight, refill width, traversal blocks) from trial slices of the
    # stellar phase: set-up, not timed
    launch, tune_s = None, 0.0
    if not args.no_autotune:
        from skirt7_b200 import autotune
        t0 = time.time()
        launch = autotune.tune(ctx, A.PHASE_STELLAR, ells, Npp, precision=prec)
        tune_s = time.time() - t0

    def run_phases(seed, stream):
        ctx.run_phase(A.PHASE_STELLAR, ells, Npp, first, npp_rank, seed=seed, precision=prec, stream=stream,
                      launch=launch)
        if wl.dust_phase:
            # PanMonteCarloSimulation::rundustselfabsorption / rundustemission (:106-187, :191-346):
            # before each dust phase the emission spectra follow from the absorbed luminosity
            for c in range(wl.selfabs_cycles):
                ctx.calc_dust_emission()
                ctx.reset_dust_absorption()
                ctx.run_phase(A.PHASE_DUST_SELFABS, ells, Npp, first, npp_rank, seed=seed + 2 + c, precision=prec,
                              stream=stream, launch=launch)
            ctx.calc_dust_emission()            # PanDustSystem::calculatedustemission
            ctx.run_phase(A.PHASE_DUST_EMISSION, ells, Npp, first, npp_rank, seed=seed + 1, precision=prec,
                          stream=stream, launch=launch)

    def step(seed):
        # every step is a whole simulation from zero tallies: the dust phases' work depends on the
        # absorbed luminosities, which must not pile up over the steps
        ctx.reset_tallies()
        ctx.sync()
        run_phases(seed, handle)
        # the phase is finished: the host has seen its last wave's counters and enqueued every wave,
        # so the step's end event follows all of them
        ctx.sync()
        if dist:
            with torch.cuda.stream(tstream):
                for i, t in zip(fr, red):
                    ctx.read_instrument_device(i, t.data_ptr(), None, handle)
                    dist.all_reduce(t)

    ctx.reset_tallies()
    ctx.sync()
    for w in range(args.warmup):
        step(1000 + 10 * w)
    torch.cuda.synchronize()
    ctx.counters()   # also checks the error word

    # ---- device-timed steps (CUDA events on the launching stream), max over ranks
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")     # twice the 126 MB L2
    for s in range(args.steps):
        with torch.cuda.stream(tstream):
            flush.zero_()                          # L2 flushed between timed steps (outside the events)
        ev[s][0].record(tstream)
        step(2000 + 10 * s)
        ev[s][1].record(tstream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(ms)
    if dist:
        t = torch.tensor([total_ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms = float(t.item())
        dist.barrier()
    torch.cuda.synchronize()
    packets = Npp * nl * len(phases) * args.steps  # all ranks together
    value = packets / (total_ms / 1e3)

    # kernel times and counters of one more stellar phase for the roofline: the traversal pass is
    # the dominant kernel; its device time is summed over the waves of the phase (CUDA events
    # around each launch on the launching stream)
    ctx.reset_tallies()
    ctx.run_phase(A.PHASE_STELLAR, ells, Npp, first, npp_rank, seed=999, precision=prec, stream=handle, launch=launch)
    ctx.sync()
    kms = ctx.last_phase_ms()
    ev_ms, trav_ms, waves = ctx.phase_times()
    c = ctx.counters()
    alg_bytes = wl.alg_bytes(c, prec == A.PREC_FP32)
    bps = wl.NCU_DRAM_BYTES_PER_STEP.get(wl.name) if (prec == A.PREC_FP32 and args.nlambda == 50) else None
    traffic = bps * c["steps"] / max(waves, 1) if bps else None
    peak, peak_kind = peaks()
    achieved = alg_bytes / (trav_ms / 1e3) / 1e9 if trav_ms > 0 else 0.0

    # ---- end to end through the C ABI with host buffers: reset, run, read the frames to host
    cubes_bytes = 8 * sum(sizes)
    # page-locked host arrays for the frames, allocated once and reused every step (as a caller
    # keeps its output images)
    host = [torch.empty(n, dtype=torch.float64, pin_memory=True) for n in sizes]
    host_out = {i: (h.numpy(), np.empty(_tally_len(ctx, i, sed=True))) for i, h in zip(fr, host)}
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e2e_steps = max(1, min(args.steps, args.e2e_steps))
    t0 = time.perf_counter()
    for s in range(e2e_steps):
        ctx.reset_tallies()
        if dist:
            ctx.sync()
            step(3000 + 10 * s)
            if rank == 0:
                for h, t in zip(host, red):        # the reduced frames, device -> host
                    h.copy_(t)
            torch.cuda.synchronize()
        else:
            run_phases(3000 + 10 * s, None)
            for i in fr:
                ctx.read_instrument(i, out=host_out[i])   # synchronises, then device -> host
    e2e_s = time.perf_counter() - t0
    if dist:
        t = torch.tensor([e2e_s], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e = Npp * nl * len(phases) * e2e_steps / e2e_s

    # the plain GPU path of the same device code: one thread per packet runs its whole life (the
    # tail pass takes the phase over after its first wave: no wavefront, no job lists), on a
    # sample of the workload's packets
    plain = None
    if rank == 0 and world == 1 and args.plain_packets > 0:
        npl = int(args.plain_packets)
        os.environ["SKG_TAIL_DIV"] = "1"
        try:
            ctx.reset_tallies()
            ctx.run_phase(A.PHASE_STELLAR, ells, npl, 0, npl, seed=777, precision=prec, stream=handle)
            ctx.sync()
            pms = ctx.last_phase_ms()
        finally:
            del os.environ["SKG_TAIL_DIV"]
        plain = {"value": npl * nl / (pms / 1e3), "unit": "packets/s", "packets": npl * nl, "phase_ms": pms,
                 "how": "the stellar phase with one thread per packet for its whole life (the same device "
                        "functions in one persistent kernel after the first wave: no wavefront passes)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(args, wl, ctx)
    srv = None
    if rank == 0 and world == 1 and args.serving > 0 and args.workload == "octree_pan":
        srv = serving_leg(args, local)

    if rank == 0:
        line = {
            "metric": wl.metric,
            "value": value, "unit": "packets/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "ms_steps": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if prec == A.PREC_FP32 else "f64", "data": "synthetic",
            "config": _config(args, wl),
            "setup": {"grid_build_s": wl.grid_s, "grid": "device", "autotune_s": tune_s,
                      "launch": {k: launch[k] for k in ("pool", "refill", "blocks")} if launch else "library defaults",
                      "autotune_trials": launch["trials"] if launch else None},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
                         "traffic_basis": ("scaled, not measured in this run: ncu DRAM bytes per cell step of "
                                           "this workload's traversal pass (%.2f B, one capture of a stellar "
                                           "phase) x this launch's cell steps" % bps) if bps else None,
                         "kernel": "trav_kernel, path and peel-off instantiations (traversal pass of the stellar phase)",
                         "launch": "one traversal pass of a wave (its path-job and peel-off-job kernels)",
                         "algorithmic_bytes_per_launch": alg_bytes / max(waves, 1),
                         "kernel_ms_per_launch": trav_ms / max(waves, 1), "launches_per_phase": waves,
                         "phase_ms": kms, "event_pass_ms": ev_ms, "traversal_pass_ms": trav_ms},
            "e2e": {"value": e2e, "unit": "packets/s", "h2d_bytes_per_step": len(phases) * (4 * nl + 64),
                    "d2h_bytes_per_step": cubes_bytes, "steps": e2e_steps},
            # per wave: the event pass, the scatter-and-launch pass and the two traversal kernels
            # (path jobs, peel-off jobs)
            "gpu_launches": 4 * waves * len(phases) * args.steps,
            "clocks": clk,
            "counters_stellar_phase": c,
        }
        if plain:
            line["plain_gpu"] = plain
        if cpu:
            line["cpu_baseline"] = cpu
        if srv:
            line["serving"] = srv
        print(json.dumps(line))
    ctx.close()
    if dist:
        dist.destroy_process_group()


def _tally_len(ctx, i, sed=False):
    import ctypes as C
    cl, sl = C.c_int64(), C.c_int64()
    ctx.lib.skg_tally_sizes(ctx.h, i, C.byref(cl), C.byref(sl))
    return sl.value if sed else cl.value


def serving_leg(args, device):
    """Fit-variant requests (oligochromatic disk, 3 wavelengths, Cartesian N^3 with N in 32..128,
    packets per wavelength log-uniform in 1e5..1e7, one 256x256 frame) arriving as a Poisson stream,
    served by continuous batching: at the configured 20/s, then the same requests at each rate of
    --serving-rates; every request alone on the idle device (the plain single-simulation path); and
    the plain path serving the stream one request at a time.  Latency = result in host memory minus
    arrival."""
    import numpy as np
    from skirt7_b200 import serving

    def serve(rate):
        reqs = serving.fitskirt_requests(n=args.serving, rate=rate, seed=2024)
        t0 = time.perf_counter()
        if args.serving_impl == "native":
            done, nst = serving.serve_native(reqs, device=device, npix=256, max_slots=64)
            ticks, tick_s, admit_s, peak = nst["ticks"], nst["tick_device_s"], None, None
        else:
            srv = serving.Server(device=device, max_slots=64, npix=256)
            done = srv.serve(reqs, realtime=True)
            srv.close()
            ticks, tick_s, admit_s, peak = srv.ticks, srv.tick_gpu_s, srv.admit_s, srv.peak_resident
        wall = time.perf_counter() - t0
        return reqs, done, wall, ticks, tick_s, admit_s, peak

    reqs, done, wall, ticks, tick_s, admit_s, peak = serve(20.0)
    st = serving.latency_stats(done)
    # the same requests (the stream's parameters do not depend on the rate) alone on the idle device
    service = [serving.run_alone(r, device=device, npix=256)[1] for r in reqs]
    alone = sorted(service)
    a50, a99 = float(np.percentile(alone, 50)), float(np.percentile(alone, 99))

    def plain_fifo(rq):
        # the plain single-simulation path serving the stream: one request at a time in arrival
        # order, each taking its measured alone time (start = max(arrival, previous finish))
        finish, lat = 0.0, []
        for r, t in sorted(zip(rq, service), key=lambda q: q[0].arrival):
            finish = max(r.arrival, finish) + t
            lat.append(finish - r.arrival)
        return float(np.percentile(lat, 50)), float(np.percentile(lat, 99))

    f50, f99 = plain_fifo(reqs)
    packets = sum(3 * r.packets for r in reqs)
    out = {"impl": args.serving_impl, "requests": len(reqs), "arrival_rate_per_s": 20.0, "p50_s": st["p50_s"],
           "p99_s": st["p99_s"], "alone_p50_s": a50, "alone_p99_s": a99, "p99_over_alone_p99": st["p99_s"] / a99,
           "plain_fifo_p50_s": f50, "plain_fifo_p99_s": f99, "p99_over_plain_fifo_p99": st["p99_s"] / f99,
           "offered_packets_per_s": packets / max(r.arrival for r in reqs),
           "packets_per_s": packets / wall, "device_packets_per_s": packets / tick_s if tick_s else None,
           "makespan_s": wall, "ticks": ticks, "tick_device_s": tick_s, "admit_host_s": admit_s,
           "peak_resident": peak, "other_rates": []}
    for rate in args.serving_rates:
        rq, dn, wl_s, tk, ts, _, _ = serve(rate)
        s2 = serving.latency_stats(dn)
        p50, p99 = plain_fifo(rq)
        out["other_rates"].append({"arrival_rate_per_s": rate, "p50_s": s2["p50_s"], "p99_s": s2["p99_s"],
                                   "p99_over_alone_p99": s2["p99_s"] / a99, "plain_fifo_p99_s": p99,
                                   "offered_packets_per_s": packets / max(r.arrival for r in rq),
                                   "makespan_s": wl_s, "ticks": tk, "tick_device_s": ts})
    return out


def cpu_baseline(args, wl, ctx):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    oracle.build()
    model = wl.model
    model.rho = ctx.density()
    threads = os.cpu_count() or 1
    kw = dict(dust_emission_phase=wl.dust_phase, selfabs_cycles=wl.selfabs_cycles)
    probe = oracle.simulate(model, args.packets, nthreads=threads, seed=1, max_packets=2000, **kw)
    rate = probe["stats"]["packets"] / max(probe["stats"]["seconds"], 1e-6)
    sample = int(max(1000, min(5e6, rate * args.cpu_seconds)))
    r = oracle.simulate(model, args.packets, nthreads=threads, seed=2, max_packets=sample, **kw)
    model.rho = None
    return {"value": r["stats"]["packets"] / r["stats"]["seconds"], "unit": "packets/s", "cores": threads,
            "kind": "port", "sample": "%d packets over all %d wavelengths%s (%.1f s of packet loops)" %
                                      (r["stats"]["packets"], model.wavelengthGrid.Nlambda,
                                       ", all phases" if wl.dust_phase else "", r["stats"]["seconds"])}


if __name__ == "__main__":
    main()
