"""A request loop for FitSKIRT-style parameter variants: continuous batching on one device.

FitSKIRT evaluates many variants of one ski file, each with a few parameters substituted
(AdjustableSkirtSimulation.cpp:145-194), and waits for each variant's frames.  Here the variants
arrive as requests; the loop

  * admits an arrived request as soon as a batch slot is free and its context fits the device
    memory budget (the context's grid, densities and frames stay resident until its result is
    read: admission by HBM footprint);
  * runs *ticks*: one batched launch that carries, for every admitted request, the next slice of
    its packets (skg_batch_run with one work item per request), so requests that arrive while
    others are on the device join at the next tick and their work overlaps on the device;
  * retires a request when its last slice has run: its frames are read and its context freed.

A request's packets carry the same numbers whichever tick runs them (the packet RNG is keyed by
the request's seed and the packet's index), so its result is the same alone and in the mix, up
to the summation order of the FP64 tally atomics.
"""
import math
import threading
import time
from concurrent.futures import Future, ThreadPoolExecutor
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from . import models, runtime
from .scene import DEG, KPC, MICRON


@dataclass
class Request:
    """One variant: (h_R, h_z, tau_V, inclination, bulge fraction), grid size N^3, packets per
    wavelength, and its arrival time (s, relative to the start of the run)."""
    rid: int
    params: tuple
    N: int
    packets: int
    arrival: float
    seed: int = 0
    # filled in by the server
    admitted: float = math.nan
    done: float = math.nan
    ticks: int = 0
    frame: np.ndarray = None
    _ctx: object = field(default=None, repr=False)
    _next: int = 0                 # first packet of the next slice
    _ran: int = 0                  # packets whose ticks have completed
    _reserved: int = 0             # device bytes reserved at admission

    @property
    def latency(self):
        return self.done - self.arrival


def fitskirt_requests(n=256, rate=20.0, seed=12345, packets=(1e5, 1e7), grid=(32, 128)):
    """The variant stream of a fit: parameters uniform in the fit ranges (dust h_R 3-9 kpc, h_z
    0.1-0.5 kpc, tau_V 0.2-4, inclination 80-90 deg, bulge fraction 0-0.5), Cartesian N^3 with N
    uniform in `grid`, packets per wavelength log-uniform in `packets`, Poisson arrivals at `rate`
    per second."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n)) if rate > 0 else np.zeros(n)
    out = []
    for i in range(n):
        p = (rng.uniform(3, 9) * KPC, rng.uniform(0.1, 0.5) * KPC, rng.uniform(0.2, 4.0),
             rng.uniform(80, 90) * DEG, rng.uniform(0.0, 0.5))
        N = int(rng.integers(grid[0], grid[1] + 1))
        npk = int(round(math.exp(rng.uniform(math.log(packets[0]), math.log(packets[1])))))
        out.append(Request(i, p, N, npk, float(t[i]), seed=1000 + i))
    return out


def build_model(req, npix=256):
    return models.fit_variant(req.params, req.N, npix=npix)


class Server:
    """Continuous batching over skg_batch on one device.

    hbm_budget   bytes of device memory the admitted contexts may hold together
    max_slots    simulations per launch (skg_batch slots)
    tick_packets packets per wavelength a request runs per tick at most; smaller ticks let
                 arrivals join sooner, larger ones amortise the launch and the drain of each tick
                 (the fit-variant stream of 256 requests: p99 6.9 s at 2^19 packets and a tick budget
                 of 6 2^20, 5.8 s at 2^20 / 12 2^20, 5.4 s at 2^21 / 24 2^20, 4.7 s at 2^22 / 48 2^20)
    policy       "fifo": a tick's packets go to the admitted requests in arrival order until
                 tick_budget packets (all wavelengths) are given out, so the oldest requests finish
                 first and the longest wait -- the p99 latency of a loaded loop -- is shortest;
                 "share": every admitted request runs a slice every tick (processor sharing)
    threads      build the contexts of admitted requests, and read and release those of retired
                 ones, on two host threads while the ticks run (False: between ticks)
    pipeline     ticks in flight at once (each on a batch of its own): the next tick is launched
                 while the previous one drains its last packets (2 measured no faster than 1 on
                 the fit-variant stream: the device is busy either way)
    """

    def __init__(self, device=0, hbm_budget=40 << 30, max_slots=64, tick_packets=1 << 22, npix=256,
                 precision=A.PREC_FP32, policy="fifo", tick_budget=48 << 20, threads=True, pipeline=1):
        self.device = device
        self.budget = hbm_budget
        self.max_slots = max_slots
        self.tick_packets = int(tick_packets)
        self.npix = npix
        self.precision = precision
        if policy not in ("fifo", "share"):
            raise ValueError("policy is 'fifo' or 'share'")
        self.policy = policy
        self.tick_budget = int(tick_budget)
        self.batches = [runtime.Batch(device=device, max_slots=max_slots, max_items=max_slots, max_ells=3 * max_slots)
                        for _ in range(max(1, int(pipeline)))]
        self.batch = self.batches[0]
        self.reserved = 0            # footprint bounds of the resident contexts (admission)
        self.in_use = 0              # their actual device bytes
        self.resident = 0            # resident contexts
        self.held = 0                # admitted requests whose reservation is not released yet
        self.peak_held = 0
        self.peak_resident = 0
        self.peak_in_use = 0
        self.ticks = 0
        self.tick_gpu_s = 0.0        # device time of the ticks, summed (CUDA events around each launch)
        self.admit_s = 0.0           # host time spent admitting (model and context set-up)
        self.threads = threads
        self._lock = threading.Lock()   # the counters above, shared with the set-up threads

    def close(self):
        for b in self.batches:
            b.close()

    def _admit(self, req):
        """Builds the request's model and context (its footprint is reserved already)."""
        t0 = time.perf_counter()
        m = build_model(req, self.npix)
        ctx = runtime.Context(m, device=self.device)
        req._ctx = ctx
        req._next = 0
        req._ran = 0
        with self._lock:
            self.in_use += ctx.device_bytes
            self.resident += 1
            self.peak_resident = max(self.peak_resident, self.resident)
            self.peak_in_use = max(self.peak_in_use, self.in_use)
            self.admit_s += time.perf_counter() - t0

    def _retire(self, req, t0):
        """Reads the request's frame (its result, at which its latency ends) and frees its context
        and reservation."""
        ctx = req._ctx
        cube, _ = ctx.read_instrument(0)
        req.frame = cube[0]
        req.done = time.perf_counter() - t0
        nbytes = ctx.device_bytes
        ctx.close()
        req._ctx = None
        with self._lock:
            self.in_use -= nbytes
            self.reserved -= req._reserved
            self.held -= 1
            self.resident -= 1

    def serve(self, requests, realtime=True, on_tick=None):
        """Runs the request stream to completion; returns the requests with their results and
        timings.  realtime: arrivals follow the wall clock (else all are present at t=0)."""
        pending = sorted(requests, key=lambda r: r.arrival)
        active = []          # in the running tick
        building = []        # (request, future): admitted, context being built
        releasing = []       # futures of retired requests' frame reads and releases
        finished = []
        t0 = time.perf_counter()
        i = 0
        if self.threads:
            setup, release = ThreadPoolExecutor(max_workers=1), ThreadPoolExecutor(max_workers=1)
        else:
            setup = release = _Inline()

        def admit(now, n_on_device):
            nonlocal i
            while i < len(pending) and (not realtime or pending[i].arrival <= now) and n_on_device < self.max_slots:
                fp = _footprint(pending[i], self.npix)
                # (contexts still being released hold their reservations)
                held = n_on_device or any(not f.done() for f in releasing)
                with self._lock:
                    if held and self.reserved + fp > self.budget:
                        break
                    self.reserved += fp
                    self.held += 1
                    self.peak_held = max(self.peak_held, self.held)
                r = pending[i]
                r._reserved = fp
                r.admitted = now
                building.append((r, setup.submit(self._admit, r)))
                n_on_device += 1
                i += 1

        def joined():
            """Requests whose context is built (in admission order)."""
            out = []
            while building and building[0][1].done():
                r, f = building.pop(0)
                f.result()
                out.append(r)
            return out

        inflight = []        # (batch, [(request, packets)]): launched ticks, oldest first
        free = list(self.batches)
        try:
            while i < len(pending) or active or building or inflight:
                active += joined()
                waiting = [r for r in active if r._next < r.packets]
                if waiting and free:
                    # one tick: the next slices of the admitted requests in one batched launch
                    slices, given = [], []
                    budget = self.tick_budget
                    for r in sorted(waiting, key=lambda q: q.arrival):
                        cnt = min(self.tick_packets, r.packets - r._next)
                        if self.policy == "fifo":
                            if budget <= 0:
                                break
                            cnt = max(1, min(cnt, budget // 3))
                            budget -= 3 * cnt
                        slices.append((r._ctx, [0, 1, 2], r.packets, r._next, cnt, r.seed))
                        given.append((r, cnt))
                        r._next += cnt
                    b = free.pop(0)
                    b.run(A.PHASE_STELLAR, slices, precision=self.precision)
                    inflight.append((b, given))
                    # arrivals are admitted while ticks run: their contexts are built (on their own
                    # streams) by the set-up thread and join a later tick
                    admit(time.perf_counter() - t0, len(active) + len(building))
                    continue
                if inflight:
                    admit(time.perf_counter() - t0, len(active) + len(building))
                    b, given = inflight.pop(0)
                    b.sync()
                    self.tick_gpu_s += b.last_ms() / 1e3
                    self.ticks += 1
                    free.append(b)
                    now = time.perf_counter() - t0
                    for r, cnt in given:
                        r._ran += cnt
                        r.ticks += 1
                        if r._ran >= r.packets:
                            finished.append(r)
                            releasing.append(release.submit(self._retire, r, t0))
                    active = [r for r in active if r._ran < r.packets]
                    if on_tick:
                        on_tick(self, now)
                    continue
                # nothing on the device and nothing admitted
                now = time.perf_counter() - t0
                admit(now, len(building))
                if building:
                    building[0][1].result()          # wait for the first context
                elif i < len(pending) and (not realtime or pending[i].arrival <= now):
                    for f in releasing:              # due, but over the budget: wait for a release
                        if not f.done():
                            f.result()
                            break
                elif i < len(pending):
                    time.sleep(max(0.0, min(0.01, pending[i].arrival - now)))
            for f in releasing:
                f.result()
        finally:
            if self.threads:
                setup.shutdown(wait=True)
                release.shutdown(wait=True)
        return finished


class _Inline:
    """An executor that runs each call at once (Server(threads=False))."""

    def submit(self, fn, *args):
        f = Future()
        try:
            f.set_result(fn(*args))
        except BaseException as e:   # surfaced by f.result(), as a thread pool does
            f.set_exception(e)
        return f


def _footprint(req, npix):
    """Device bytes of a variant's context, bounded from above before creating it: densities (FP64
    and FP32) with room for the set-up tables, the Cartesian planes, the frame cube (3 wavelengths)
    and a fixed allowance for the remaining tables."""
    nc = req.N ** 3
    return nc * 24 + 3 * (req.N + 1) * 12 + 3 * npix * npix * 8 + (4 << 20)


def run_alone(req, device=0, npix=256, precision=A.PREC_FP32):
    """The plain single-simulation GPU path for one request: create, run one phase, read the frame.
    Returns (frame, seconds until the frame is in host memory); the context is released after the
    clock stops, as the served requests' latencies end when their frames are read."""
    t0 = time.perf_counter()
    ctx = runtime.Context(build_model(req, npix), device=device)
    ctx.run_phase(A.PHASE_STELLAR, [0, 1, 2], req.packets, 0, req.packets, seed=req.seed, precision=precision)
    cube, _ = ctx.read_instrument(0)
    t = time.perf_counter() - t0
    ctx.close()
    return cube[0], t


def latency_stats(reqs):
    lat = np.array([r.latency for r in reqs])
    return {"p50_s": float(np.percentile(lat, 50)), "p99_s": float(np.percentile(lat, 99)),
            "mean_s": float(lat.mean()), "max_s": float(lat.max()), "n": len(lat)}


class NativeServer:
    """The continuous-batching server of the C ABI (skg_server: skg_submit / skg_poll), whose loop
    and context set-up run on native threads: the same admission, ticks and retirement as Server,
    for a host program that links the library directly (a C++ FitSKIRT)."""

    def __init__(self, device=0, hbm_budget=0, max_slots=0, tick_packets=0, tick_budget=0, precision=A.PREC_FP32):
        import ctypes as C
        self.lib = A.load()
        o = A.ServerOpts(int(hbm_budget), int(max_slots), int(tick_packets), int(tick_budget), precision)
        h = C.c_void_p()
        A.check(self.lib.skg_server_create(device, C.byref(o), C.byref(h)))
        self.h = h
        self._out = {}

    def submit(self, model, ells, packages, seed, instr=0):
        """Queues one simulation (the scene is copied); returns its id."""
        import ctypes as C
        sc, keep = model.lower()
        cl, sl = C.c_int64(), C.c_int64()
        A.check(self.lib.skg_scene_tally_sizes(C.byref(sc), instr, C.byref(cl), C.byref(sl)))
        cube = np.zeros(max(cl.value, 1))
        sed = np.zeros(max(sl.value, 1))
        e = np.ascontiguousarray(ells, dtype=np.int32)
        q = A.Request(C.pointer(sc), e.ctypes.data_as(A.i32p), len(e), int(packages), int(seed), instr,
                      cube.ctypes.data_as(A.dp) if cl.value else None, sed.ctypes.data_as(A.dp))
        rid = C.c_int64()
        A.check(self.lib.skg_submit(self.h, C.byref(q), C.byref(rid)))
        ins = model.instruments[instr]
        self._out[rid.value] = (cube, sed, cl.value, sl.value, model.wavelengthGrid.Nlambda, ins)
        return rid.value

    def poll(self, rid, timeout_ms=-1):
        """(cube [components, nlambda, ny, nx] or None, sed [components, nlambda], latency s) once
        request rid is done; raises SkirtError with SKG_ERR_TIMEOUT while it runs."""
        import ctypes as C
        lat = C.c_double()
        A.check(self.lib.skg_poll(self.h, rid, int(timeout_ms), C.byref(lat)))
        cube, sed, cl, sl, nl, ins = self._out.pop(rid)
        ncomp = sl // nl
        sed = sed[:sl].reshape(ncomp, nl)
        cube = cube.reshape(ncomp, nl, ins.pixelsY, ins.pixelsX) if cl else None
        return cube, sed, lat.value

    def stats(self):
        import ctypes as C
        t, c, p, ms = C.c_int64(), C.c_int64(), C.c_int64(), C.c_double()
        A.check(self.lib.skg_server_stats(self.h, C.byref(t), C.byref(c), C.byref(p), C.byref(ms)))
        return {"ticks": t.value, "completed": c.value, "packets": p.value, "tick_device_s": ms.value / 1e3}

    def close(self):
        if self.h:
            self.lib.skg_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve_native(requests, device=0, npix=256, realtime=True, **opts):
    """Runs the request stream through NativeServer: each request is submitted at its arrival time
    (realtime) and its frame polled; returns the requests with frame, admitted and done filled in
    (done = arrival + the server's submission-to-completion latency)."""
    srv = NativeServer(device=device, **opts)
    pending = sorted(requests, key=lambda r: r.arrival)
    ids = {}
    t0 = time.perf_counter()
    try:
        for r in pending:
            if realtime:
                dt = r.arrival - (time.perf_counter() - t0)
                if dt > 0:
                    time.sleep(dt)
            r.admitted = time.perf_counter() - t0
            ids[r.rid] = srv.submit(build_model(r, npix), [0, 1, 2], r.packets, r.seed)
        for r in pending:
            cube, _, lat = srv.poll(ids[r.rid])
            r.frame = cube[0]
            r.done = r.admitted + lat
        st = srv.stats()
    finally:
        srv.close()
    st["makespan_s"] = time.perf_counter() - t0
    return pending, st
