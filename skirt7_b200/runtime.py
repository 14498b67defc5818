"""Python host side over the C ABI: a device context for one scene, the grid builders, and the
MonteCarloSimulation phase driver (the reference's runSelf sequences)."""
import ctypes as C
import math

import numpy as np

from . import _abi as A
from .scene import SceneModel, TreeDustGrid


def device_count():
    n = C.c_int(0)
    rc = A.load().skg_device_count(C.byref(n))
    return n.value if rc == 0 else 0


def chunk_params(packages, nthreads=1, nprocs=1, nlambda=1):
    """MonteCarloSimulation::setChunkParams (MonteCarloSimulation.cpp:68-114)."""
    a, b, c = C.c_uint64(), C.c_uint64(), C.c_uint64()
    A.load().skg_chunk_params(float(packages), nthreads, nprocs, nlambda, C.byref(a), C.byref(b), C.byref(c))
    return a.value, b.value, c.value


class Context:
    """A scene resident on one device (skg_ctx)."""

    def __init__(self, model: SceneModel, device=0):
        self.lib = A.load()
        self.model = model
        self.device = device
        self.scene, self._keep = model.lower()
        h = C.c_void_p()
        A.check(self.lib.skg_ctx_create(C.byref(self.scene), device, C.byref(h)))
        self.h = h
        self.nlambda = model.wavelengthGrid.Nlambda
        nc, nb = C.c_int64(), C.c_int64()
        self.lib.skg_ctx_info(self.h, C.byref(nc), C.byref(nb))
        self.ncells, self.device_bytes = nc.value, nb.value

    def close(self):
        if self.h:
            self.lib.skg_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        return A.check(rc, self.h)

    # ---- traversal harness
    def trace_paths(self, r, k, precision=A.PREC_FP64):
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
        k = np.ascontiguousarray(k, dtype=np.float64).reshape(-1, 3)
        n = len(r)
        off = np.zeros(n + 1, dtype=np.int64)
        cap = 0
        cells = np.zeros(1, dtype=np.int32)
        ds = np.zeros(1, dtype=np.float64)
        rc = self.lib.skg_trace_paths(self.h, r.ctypes.data_as(A.dp),
                                      k.ctypes.data_as(A.dp), n, precision, cells.ctypes.data_as(A.i32p),
                                      ds.ctypes.data_as(A.dp), off.ctypes.data_as(A.i64p), cap)
        if rc == A.SKG_ERR_CAPACITY:
            cap = int(off[n])
            cells = np.zeros(max(cap, 1), dtype=np.int32)
            ds = np.zeros(max(cap, 1), dtype=np.float64)
            rc = self.lib.skg_trace_paths(self.h, r.ctypes.data_as(A.dp), k.ctypes.data_as(A.dp), n, precision,
                                          cells.ctypes.data_as(A.i32p), ds.ctypes.data_as(A.dp),
                                          off.ctypes.data_as(A.i64p), cap)
        self._ck(rc)
        tot = int(off[n])
        return off, cells[:tot], ds[:tot]

    NOALLOC_MAX_RAYS = 1048576

    def trace_paths_noalloc(self, d_r, d_k, n, d_cells, d_ds, d_offsets, capacity, precision=A.PREC_FP64,
                            stream=None):
        """skg_trace_paths_noalloc: device addresses (ints) in and out; enqueues on `stream` (a
        cudaStream_t as int, None = the context's stream) and returns without waiting.  The
        status of the device work is reported by sync() after that stream has completed."""
        self._ck(self.lib.skg_trace_paths_noalloc(self.h, d_r, d_k, n, precision, d_cells, d_ds, d_offsets,
                                                  capacity, stream))

    def optical_depth(self, r, k, ell=0, precision=A.PREC_FP64):
        r = np.ascontiguousarray(r, dtype=np.float64).reshape(-1, 3)
        k = np.ascontiguousarray(k, dtype=np.float64).reshape(-1, 3)
        tau = np.zeros(len(r))
        self._ck(self.lib.skg_optical_depth(self.h, r.ctypes.data_as(A.dp), k.ctypes.data_as(A.dp), len(r), ell,
                                            precision, tau.ctypes.data_as(A.dp)))
        return tau

    # ---- the packet loop
    def run_phase(self, phase, ells, npp, first=0, count=None, seed=4357, precision=A.PREC_FP32,
                  max_steps=0, max_scatt=0, blocks=0, pool=0, stream=None, refill=0, launch=None):
        """skg_run_phase.  pool: packets in flight per wave, blocks: traversal blocks, refill: lanes
        of a warp that wait before it takes new jobs (0 = the library's defaults); launch: a dict
        with any of these (an autotuner result) that takes their place."""
        if launch:
            pool, blocks, refill = launch.get("pool", pool), launch.get("blocks", blocks), launch.get("refill", refill)
        ells = np.ascontiguousarray(ells, dtype=np.int32)
        opts = A.RunOpts(precision, max_steps, max_scatt, blocks, refill, 1, pool)
        count = npp if count is None else count
        self._ck(self.lib.skg_run_phase(self.h, phase, ells.ctypes.data_as(A.i32p), len(ells), int(npp), int(first),
                                        int(count), int(seed), C.byref(opts), stream))

    def sync(self, timeout_ms=-1):
        return self._ck(self.lib.skg_sync(self.h, timeout_ms))

    def last_phase_ms(self):
        ms = C.c_float()
        self._ck(self.lib.skg_last_phase_ms(self.h, C.byref(ms)))
        return ms.value

    def phase_times(self):
        """(event_ms, traversal_ms, waves) of the last phase: summed device time of its two kernels."""
        a, b, w = C.c_float(), C.c_float(), C.c_int32()
        self._ck(self.lib.skg_phase_times(self.h, C.byref(a), C.byref(b), C.byref(w)))
        return a.value, b.value, w.value

    def reset_tallies(self):
        self._ck(self.lib.skg_reset_tallies(self.h))

    def read_instrument(self, i, out=None):
        """(cube, sed): cube shaped [components, nlambda, nyp, nxp] (None for SED instruments),
        sed shaped [components, nlambda].  out: (cube, sed) flat float64 host arrays of the
        instrument's tally sizes to read into (e.g. page-locked buffers reused every step)."""
        cl, sl = C.c_int64(), C.c_int64()
        self._ck(self.lib.skg_tally_sizes(self.h, i, C.byref(cl), C.byref(sl)))
        ins = self.model.instruments[i]
        ncomp = sl.value // self.nlambda
        if out is not None:
            cube, sed = out
            if sed is None or sed.dtype != np.float64 or not sed.flags.c_contiguous or sed.size != sl.value or \
                    (cl.value and (cube is None or cube.dtype != np.float64 or not cube.flags.c_contiguous or
                                   cube.size != cl.value)):
                raise ValueError("out: flat contiguous float64 arrays of the instrument's tally sizes")
            cube = cube if cl.value else None
        else:
            sed = np.zeros(sl.value)
            cube = np.zeros(cl.value) if cl.value else None
        self._ck(self.lib.skg_read_instrument(self.h, i, cube.ctypes.data_as(A.dp) if cube is not None else None,
                                              sed.ctypes.data_as(A.dp)))
        sed = sed.reshape(ncomp, self.nlambda)
        if cube is not None:
            cube = cube.reshape(ncomp, self.nlambda, ins.pixelsY, ins.pixelsX)
        return cube, sed

    def read_instrument_device(self, i, d_cube, d_sed=None, stream=None):
        """Copies instrument i's tallies into caller-owned device buffers (raw device pointers,
        e.g. torch tensor data_ptr()) on the given stream."""
        self._ck(self.lib.skg_read_instrument_device(self.h, i, d_cube, d_sed, stream))

    def read_absorption(self):
        ls = np.zeros(self.ncells * self.nlambda)
        ld = np.zeros(self.ncells * self.nlambda)
        self._ck(self.lib.skg_read_absorption(self.h, ls.ctypes.data_as(A.dp), ld.ctypes.data_as(A.dp)))
        return ls.reshape(self.ncells, self.nlambda), ld.reshape(self.ncells, self.nlambda)

    def counters(self):
        c = A.Counters()
        rc = self.lib.skg_read_counters(self.h, C.byref(c))
        if rc not in (0, A.SKG_ERR_STEP_BUDGET, A.SKG_ERR_NAN_TAU):
            self._ck(rc)
        return {n: getattr(c, n) for n, _ in A.Counters._fields_}

    def density(self):
        nd = len(self.model.dustComps)
        rho = np.zeros(max(nd, 1) * self.ncells)
        self._ck(self.lib.skg_read_density(self.h, rho.ctypes.data_as(A.dp)))
        return rho[: nd * self.ncells].reshape(nd, self.ncells)

    def calc_dust_emission(self):
        T = np.zeros(self.ncells)
        self._ck(self.lib.skg_calc_dust_emission(self.h, T.ctypes.data_as(A.dp)))
        return T

    def absorbed_totals(self):
        a, b = C.c_double(), C.c_double()
        self._ck(self.lib.skg_absorbed_totals(self.h, C.byref(a), C.byref(b)))
        return a.value, b.value

    def reset_dust_absorption(self):
        self._ck(self.lib.skg_reset_dust_absorption(self.h))


class Batch:
    """Staging for launches that carry slices of several simulations at once (skg_batch)."""

    def __init__(self, device=0, max_slots=64, max_items=256, max_ells=1024):
        self.lib = A.load()
        h = C.c_void_p()
        A.check(self.lib.skg_batch_create(device, max_slots, max_items, max_ells, C.byref(h)))
        self.h = h
        self._keep = []

    def run(self, phase, slices, precision=A.PREC_FP32, graph=False, stream=None, max_scatt=0, pool=0, refill=0):
        """slices: list of (Context, ells, npp, first, count, seed)."""
        n = len(slices)
        arr = (A.Work * max(n, 1))()
        keep = []
        for i, (ctx, ells, npp, first, count, seed) in enumerate(slices):
            e = np.ascontiguousarray(ells, dtype=np.int32)
            keep.append(e)
            arr[i] = A.Work(ctx.h.value, e.ctypes.data_as(A.i32p), len(e), int(npp), int(first), int(count), int(seed))
        opts = A.RunOpts(precision, 0, max_scatt, 0, refill, 1, pool)
        A.check(self.lib.skg_batch_run(self.h, phase, arr, n, C.byref(opts), A.BATCH_GRAPH if graph else 0, stream))
        self._keep = keep

    def sync(self, timeout_ms=-1):
        A.check(self.lib.skg_batch_sync(self.h, timeout_ms))

    def last_ms(self):
        ms = C.c_float()
        A.check(self.lib.skg_batch_last_ms(self.h, C.byref(ms)))
        return ms.value

    def counters(self):
        c = A.Counters()
        self.lib.skg_batch_counters(self.h, C.byref(c))
        return {n: getattr(c, n) for n, _ in A.Counters._fields_}

    def close(self):
        if self.h:
            self.lib.skg_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# --------------------------------------------------------------------------------------------
# grid builders

def _tree_from_handle(lib, h, gtype, extent, search):
    nn, nc, nnb = C.c_int32(), C.c_int32(), C.c_int64()
    lib.skg_tree_sizes(h, C.byref(nn), C.byref(nc), C.byref(nnb))
    n = nn.value
    box = np.zeros(6 * n)
    child = np.zeros(n, dtype=np.int32)
    father = np.zeros(n, dtype=np.int32)
    cell = np.zeros(n, dtype=np.int32)
    d = np.zeros(n, dtype=np.int8)
    off = np.zeros(6 * n + 1, dtype=np.int64)
    ids = np.zeros(max(nnb.value, 1), dtype=np.int32)
    lib.skg_tree_arrays(h, box.ctypes.data_as(A.dp), child.ctypes.data_as(A.i32p), father.ctypes.data_as(A.i32p),
                        cell.ctypes.data_as(A.i32p), d.ctypes.data_as(A.i8p), off.ctypes.data_as(A.i64p),
                        ids.ctypes.data_as(A.i32p))
    lib.skg_tree_destroy(h)
    return TreeDustGrid(gtype, extent, box, child, father, cell, d, off, ids[: nnb.value], search)


def build_tree(model: SceneModel, gtype, extent, minLevel=2, maxLevel=6, maxMassFraction=1e-6, sampleCount=100,
               seed=4357, device=0, searchMethod=A.SEARCH_NEIGHBOR):
    """TreeDustGrid set-up (TreeDustGrid.cpp:49-162) with device-sampled node masses."""
    lib = A.load()
    model.normalise()
    from .scene import CartesianDustGrid
    saved = model.dustGrid
    x0, y0, z0, x1, y1, z1 = extent
    model.dustGrid = CartesianDustGrid(x0, x1, y0, y1, z0, z1, 1, 1, 1)   # only the extent is used
    sc, keep = model.lower()
    model.dustGrid = saved
    h = C.c_void_p()
    A.check(lib.skg_tree_build(C.byref(sc), gtype, minLevel, maxLevel, maxMassFraction, sampleCount, seed, device,
                               C.byref(h)))
    return _tree_from_handle(lib, h, gtype, extent, searchMethod)


def build_voronoi(sites, extent, device=0):
    """VoronoiMesh::buildMesh (VoronoiMesh.cpp:297-405) on the device: the tessellation of the
    generator points inside the domain box, with the block lists of the cell search."""
    from .scene import VoronoiDustGrid
    lib = A.load()
    s = np.ascontiguousarray(sites, dtype=np.float64).reshape(-1, 3)
    h = C.c_void_p()
    A.check(lib.skg_voronoi_build(s.ctypes.data_as(A.dp), len(s), *[float(v) for v in extent], device, C.byref(h)))
    try:
        n, nn, nb, nbid = C.c_int32(), C.c_int64(), C.c_int32(), C.c_int64()
        A.check(lib.skg_voronoi_sizes(h, C.byref(n), C.byref(nn), C.byref(nb), C.byref(nbid)))
        n = n.value
        pos, off = np.zeros((n, 3)), np.zeros(n + 1, dtype=np.int64)
        ids, vol = np.zeros(nn.value, dtype=np.int32), np.zeros(n)
        cen, bbox = np.zeros((n, 3)), np.zeros((n, 6))
        boff, bids = np.zeros(nb.value ** 3 + 1, dtype=np.int64), np.zeros(nbid.value, dtype=np.int32)
        A.check(lib.skg_voronoi_arrays(h, pos.ctypes.data_as(A.dp), off.ctypes.data_as(A.i64p),
                                       ids.ctypes.data_as(A.i32p), vol.ctypes.data_as(A.dp), cen.ctypes.data_as(A.dp),
                                       bbox.ctypes.data_as(A.dp), boff.ctypes.data_as(A.i64p),
                                       bids.ctypes.data_as(A.i32p)))
    finally:
        lib.skg_voronoi_destroy(h)
    return VoronoiDustGrid(extent, pos, off, ids, nb.value, boff, bids, vol, bbox)


def tree_from_splits(gtype, extent, split, searchMethod=A.SEARCH_NEIGHBOR):
    lib = A.load()
    split = np.ascontiguousarray(split, dtype=np.uint8)
    h = C.c_void_p()
    A.check(lib.skg_tree_from_splits(gtype, *[float(v) for v in extent], split.ctypes.data_as(A.u8p), len(split),
                                     C.byref(h)))
    return _tree_from_handle(lib, h, gtype, extent, searchMethod)


# --------------------------------------------------------------------------------------------
# MonteCarloSimulation driver

class MonteCarloSimulation:
    """The phase sequence of OligoMonteCarloSimulation::runSelf (OligoMonteCarloSimulation.cpp:69-74)
    and PanMonteCarloSimulation::runSelf (PanMonteCarloSimulation.cpp:92-102), each phase one
    persistent device launch over all wavelengths."""

    def __init__(self, model: SceneModel, packages, seed=4357, precision=A.PREC_FP32, device=0,
                 selfAbsorption=False, cycles=0, emissionBoost=1.0, nprocs=1, rank=0, threads=1, autotune=False):
        """threads: the host thread count the reference would run with (its -t option): it sets the
        chunking, hence the packet count actually run, totalChunks * chunksize >= packages
        (MonteCarloSimulation.cpp:68-114).  autotune: before the first phase, time trial slices of
        the stellar phase for the launch choices of skirt7_b200.autotune (True, or the path of a
        JSON cache) and run every phase with the fastest."""
        self.model = model
        self.packages = packages
        self.seed = seed
        self.precision = precision
        self.device = device
        self.selfAbsorption = selfAbsorption
        self.cycles = cycles
        self.emissionBoost = emissionBoost
        self.nprocs, self.rank = nprocs, rank
        self.threads = max(1, int(threads))
        self.autotune = autotune
        self.launch = None
        self.ctx = None
        self.phase_ms = {}

    def setup(self):
        if self.ctx is None:
            self.ctx = Context(self.model, self.device)
        return self

    def tune(self):
        """The launch choices for this simulation's phases (skirt7_b200.autotune.tune on a slice of
        the stellar phase); a tree grid whose rope records walk faster is rebuilt with them."""
        from . import autotune
        ctx = self.ctx
        _, _, npp = chunk_params(self.packages, self.threads, self.nprocs, ctx.nlambda)
        path = self.autotune if isinstance(self.autotune, str) else None
        self.launch = autotune.tune(ctx, A.PHASE_STELLAR, np.arange(ctx.nlambda), npp, precision=self.precision,
                                    path=path, records=True)
        if self.launch.get("records") == "rope":
            import os
            ctx.close()
            old = os.environ.get("SKG_TREE_RECORDS")
            os.environ["SKG_TREE_RECORDS"] = "rope"
            try:
                self.ctx = Context(self.model, self.device)
            finally:
                if old is None:
                    os.environ.pop("SKG_TREE_RECORDS", None)
                else:
                    os.environ["SKG_TREE_RECORDS"] = old
        return self.launch

    def _packet_range(self, npp):
        # disjoint packet ranges per rank (MonteCarloSimulation.cpp:98-104 distributes chunks)
        per = -(-npp // self.nprocs)
        first = min(npp, self.rank * per)
        return first, max(0, min(npp, first + per) - first)

    def _run(self, phase, packages, seed):
        ctx = self.ctx
        _, _, npp = chunk_params(packages, self.threads, self.nprocs, ctx.nlambda)
        first, count = self._packet_range(npp)
        ctx.run_phase(phase, np.arange(ctx.nlambda), npp, first, count, seed, self.precision, launch=self.launch)
        ctx.sync()
        return ctx.last_phase_ms() if count else 0.0

    def runstellaremission(self):
        self.phase_ms["stellar"] = self._run(A.PHASE_STELLAR, self.packages, self.seed)

    def rundustselfabsorption(self):
        """Three stages of cycles with 1/10, 1/3 and 1 times the packages and convergence limits
        1%, 0.7%, 0.5% (PanMonteCarloSimulation.cpp:106-187); a fixed cycle count runs exactly
        that many cycles per stage."""
        ctx = self.ctx
        prev = 0.0
        factors, epsmax = (0.1, 1. / 3., 1.0), (0.010, 0.007, 0.005)
        self.selfabs_log = []
        for stage in range(3):
            ncmax = self.cycles if self.cycles else 100
            cycle, conv = 1, False
            while cycle <= ncmax and (not conv or self.cycles):
                ctx.calc_dust_emission()
                ctx.reset_dust_absorption()
                ms = self._run(A.PHASE_DUST_SELFABS, self.packages * factors[stage], self.seed + 1000 * stage + cycle)
                _, ldust = ctx.absorbed_totals()
                eps = abs((ldust - prev) / ldust) if ldust else 0.0
                prev = ldust
                self.selfabs_log.append((stage, cycle, ldust, eps, ms))
                if (stage < 2 or cycle > 1) and eps < epsmax[stage]:
                    conv = True
                cycle += 1

    def rundustemission(self):
        ctx = self.ctx
        ctx.calc_dust_emission()
        self.phase_ms["dustemission"] = self._run(A.PHASE_DUST_EMISSION, self.packages * self.emissionBoost,
                                                  self.seed + 7777)

    def run(self):
        self.setup()
        if self.autotune and self.launch is None:
            self.tune()
        self.runstellaremission()
        if self.model.dustEmission and self.model.dustComps:
            if self.selfAbsorption:
                self.rundustselfabsorption()
            self.rundustemission()
        return self
