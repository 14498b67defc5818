"""ctypes mirror of include/skirt_b200.h.

Struct layouts here must match the header field for field; tests/test_abi.py checks the
exported symbols and the struct sizes against a C compiler's view of the header.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libskirt_b200.so")

SKG_OK = 0
SKG_ERR_INVALID = 1
SKG_ERR_OOM = 2
SKG_ERR_CUDA = 3
SKG_ERR_STEP_BUDGET = 4
SKG_ERR_NAN_TAU = 5
SKG_ERR_TIMEOUT = 6
SKG_ERR_NO_DEVICE = 7
SKG_ERR_CAPACITY = 8
SKG_ERR_BAD_CELL = 9

GRID_CARTESIAN, GRID_OCTREE, GRID_BINTREE, GRID_VORONOI = 0, 1, 2, 3
SEARCH_TOPDOWN, SEARCH_NEIGHBOR, SEARCH_BOOKKEEPING = 0, 1, 2
GEOM_EXPDISK, GEOM_SERSIC, GEOM_POINT, GEOM_PLUMMER = 0, 1, 2, 3
KERNEL_CUBICSPLINE, KERNEL_UNIFORM = 0, 1
INSTR_SED, INSTR_FRAME, INSTR_SIMPLE, INSTR_FULL = 0, 1, 2, 3
PHASE_STELLAR, PHASE_DUST_SELFABS, PHASE_DUST_EMISSION = 0, 1, 2
PREC_FP32, PREC_FP64 = 0, 1
FULL_TOT, FULL_TRA, FULL_STRDIR, FULL_STRSCA, FULL_DUSDIR, FULL_DUSSCA, FULL_NBASE = range(7)

dp = C.POINTER(C.c_double)
i32p = C.POINTER(C.c_int32)
i64p = C.POINTER(C.c_int64)
i8p = C.POINTER(C.c_int8)
u8p = C.POINTER(C.c_uint8)


class Grid(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("xmin", C.c_double), ("ymin", C.c_double), ("zmin", C.c_double),
        ("xmax", C.c_double), ("ymax", C.c_double), ("zmax", C.c_double),
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("xv", dp), ("yv", dp), ("zv", dp),
        ("nnodes", C.c_int32),
        ("node_box", dp), ("node_child", i32p), ("node_father", i32p), ("node_cell", i32p),
        ("node_dir", i8p), ("nbr_offsets", i64p), ("nbr_ids", i32p),
        ("search_method", C.c_int32),
        ("nsites", C.c_int32),
        ("sites", dp), ("vnbr_offsets", i64p), ("vnbr_ids", i32p),
        ("nb", C.c_int32), ("block_offsets", i64p), ("block_ids", i32p),
        ("cell_volume", dp), ("cell_bbox", dp),
    ]


class Geometry(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("p", C.c_double * 6),
        ("clump_fraction", C.c_double),
        ("clump_count", C.c_int32),
        ("clump_radius", C.c_double),
        ("clump_cutoff", C.c_int32),
        ("clump_kernel", C.c_int32),
        ("clump_pos", dp),
    ]


class StellarComp(C.Structure):
    _fields_ = [("geometry", Geometry), ("luminosity", dp)]


class DustComp(C.Structure):
    _fields_ = [("geometry", Geometry), ("norm", C.c_double), ("kappaext", dp), ("albedo", dp), ("asymmpar", dp)]


class Instrument(C.Structure):
    _fields_ = [
        ("type", C.c_int32),
        ("distance", C.c_double), ("inclination", C.c_double), ("azimuth", C.c_double),
        ("position_angle", C.c_double),
        ("nxp", C.c_int32), ("nyp", C.c_int32),
        ("fovx", C.c_double), ("fovy", C.c_double), ("xc", C.c_double), ("yc", C.c_double),
        ("nscatt_levels", C.c_int32),
        ("stellar_comps", C.c_int32),
    ]


class Scene(C.Structure):
    _fields_ = [
        ("grid", Grid),
        ("nlambda", C.c_int32), ("lambda_", dp), ("dlambda", dp),
        ("ncomp", C.c_int32), ("dust", C.POINTER(DustComp)), ("rho", dp), ("density_samples", C.c_int32),
        ("nstellar", C.c_int32), ("stellar", C.POINTER(StellarComp)), ("emission_bias", C.c_double),
        ("ninstr", C.c_int32), ("instr", C.POINTER(Instrument)),
        ("min_weight_reduction", C.c_double), ("min_scatt_events", C.c_int32), ("scatt_bias", C.c_double),
        ("store_absorption", C.c_int32),
        ("dust_emission", C.c_int32), ("dust_emission_bias", C.c_double),
    ]


class RunOpts(C.Structure):
    _fields_ = [
        ("precision", C.c_int32), ("max_steps", C.c_int32), ("max_scatt", C.c_int32),
        ("blocks", C.c_int32), ("refill", C.c_int32), ("dedupe_peeloff", C.c_int32), ("pool", C.c_int32),
    ]


class Counters(C.Structure):
    _fields_ = [(n, C.c_uint64) for n in (
        "packets", "steps", "traversals", "scatterings", "peeloffs", "absorb_adds", "pixel_adds",
        "nbr_scanned", "fallbacks", "errors", "waves")]


class Work(C.Structure):
    _fields_ = [("ctx", C.c_void_p), ("ells", i32p), ("nell", C.c_int32), ("npp", C.c_uint64), ("first", C.c_uint64),
                ("count", C.c_uint64), ("seed", C.c_uint64)]


BATCH_GRAPH = 1


class ServerOpts(C.Structure):
    _fields_ = [("hbm_budget", C.c_int64), ("max_slots", C.c_int32), ("tick_packets", C.c_int64),
                ("tick_budget", C.c_int64), ("precision", C.c_int32)]


class Request(C.Structure):
    _fields_ = [("scene", C.POINTER(Scene)), ("ells", i32p), ("nell", C.c_int32), ("packages", C.c_uint64),
                ("seed", C.c_uint64), ("instr", C.c_int32), ("cube", dp), ("sed", dp)]

# exported functions: name -> (restype, argtypes)
FUNCS = {
    "skg_version": (C.c_int, []),
    "skg_last_error": (C.c_char_p, [C.c_void_p]),
    "skg_device_count": (C.c_int, [C.POINTER(C.c_int)]),
    "skg_ctx_create": (C.c_int, [C.POINTER(Scene), C.c_int, C.POINTER(C.c_void_p)]),
    "skg_ctx_destroy": (C.c_int, [C.c_void_p]),
    "skg_ctx_info": (C.c_int, [C.c_void_p, i64p, i64p]),
    "skg_read_density": (C.c_int, [C.c_void_p, dp]),
    "skg_trace_paths": (C.c_int, [C.c_void_p, dp, dp, C.c_int64, C.c_int, i32p, dp, i64p, C.c_int64]),
    "skg_trace_paths_noalloc": (C.c_int, [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int64, C.c_int, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_int64, C.c_void_p]),
    "skg_optical_depth": (C.c_int, [C.c_void_p, dp, dp, C.c_int64, C.c_int, C.c_int, dp]),
    "skg_chunk_params": (C.c_int, [C.c_double, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_uint64),
                                   C.POINTER(C.c_uint64), C.POINTER(C.c_uint64)]),
    "skg_run_phase": (C.c_int, [C.c_void_p, C.c_int, i32p, C.c_int, C.c_uint64, C.c_uint64, C.c_uint64,
                                C.c_uint64, C.POINTER(RunOpts), C.c_void_p]),
    "skg_reset_tallies": (C.c_int, [C.c_void_p]),
    "skg_batch_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.POINTER(C.c_void_p)]),
    "skg_batch_destroy": (C.c_int, [C.c_void_p]),
    "skg_batch_run": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(Work), C.c_int, C.POINTER(RunOpts), C.c_int,
                                C.c_void_p]),
    "skg_batch_sync": (C.c_int, [C.c_void_p, C.c_int]),
    "skg_batch_counters": (C.c_int, [C.c_void_p, C.POINTER(Counters)]),
    "skg_batch_last_ms": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "skg_tally_sizes": (C.c_int, [C.c_void_p, C.c_int, i64p, i64p]),
    "skg_read_instrument": (C.c_int, [C.c_void_p, C.c_int, dp, dp]),
    "skg_read_instrument_device": (C.c_int, [C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]),
    "skg_read_absorption": (C.c_int, [C.c_void_p, dp, dp]),
    "skg_read_counters": (C.c_int, [C.c_void_p, C.POINTER(Counters)]),
    "skg_sync": (C.c_int, [C.c_void_p, C.c_int]),
    "skg_last_phase_ms": (C.c_int, [C.c_void_p, C.POINTER(C.c_float)]),
    "skg_phase_times": (C.c_int, [C.c_void_p, C.POINTER(C.c_float), C.POINTER(C.c_float), i32p]),
    "skg_calc_dust_emission": (C.c_int, [C.c_void_p, dp]),
    "skg_absorbed_totals": (C.c_int, [C.c_void_p, dp, dp]),
    "skg_reset_dust_absorption": (C.c_int, [C.c_void_p]),
    "skg_tree_build": (C.c_int, [C.POINTER(Scene), C.c_int, C.c_int, C.c_int, C.c_double, C.c_int, C.c_uint64,
                                 C.c_int, C.POINTER(C.c_void_p)]),
    "skg_tree_from_splits": (C.c_int, [C.c_int, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                       C.c_double, u8p, C.c_int64, C.POINTER(C.c_void_p)]),
    "skg_tree_sizes": (C.c_int, [C.c_void_p, i32p, i32p, i64p]),
    "skg_tree_arrays": (C.c_int, [C.c_void_p, dp, i32p, i32p, i32p, i8p, i64p, i32p]),
    "skg_tree_grid": (C.c_int, [C.c_void_p, C.POINTER(Grid)]),
    "skg_tree_destroy": (C.c_int, [C.c_void_p]),
    "skg_voronoi_build": (C.c_int, [dp, C.c_int32, C.c_double, C.c_double, C.c_double, C.c_double, C.c_double,
                                    C.c_double, C.c_int, C.POINTER(C.c_void_p)]),
    "skg_voronoi_sizes": (C.c_int, [C.c_void_p, i32p, i64p, i32p, i64p]),
    "skg_voronoi_arrays": (C.c_int, [C.c_void_p, dp, i64p, i32p, dp, dp, dp, i64p, i32p]),
    "skg_voronoi_grid": (C.c_int, [C.c_void_p, C.POINTER(Grid)]),
    "skg_voronoi_destroy": (C.c_int, [C.c_void_p]),
    "skg_server_create": (C.c_int, [C.c_int, C.POINTER(ServerOpts), C.POINTER(C.c_void_p)]),
    "skg_submit": (C.c_int, [C.c_void_p, C.POINTER(Request), i64p]),
    "skg_poll": (C.c_int, [C.c_void_p, C.c_int64, C.c_int, dp]),
    "skg_server_stats": (C.c_int, [C.c_void_p, i64p, i64p, i64p, dp]),
    "skg_server_destroy": (C.c_int, [C.c_void_p]),
    "skg_scene_tally_sizes": (C.c_int, [C.POINTER(Scene), C.c_int, i64p, i64p]),
}

_lib = None


def load():
    """Loads the in-tree library; raises if it has not been built (there is no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libskirt_b200.so is not built; run python skirt7_b200/build.py")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in FUNCS.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


class SkirtError(RuntimeError):
    """A non-zero status of the C ABI (the reference raises FatalError at the same points)."""

    def __init__(self, code, msg):
        super().__init__("%s (status %d)" % (msg, code))
        self.code = code


def check(rc, ctx=None):
    if rc != SKG_OK:
        msg = load().skg_last_error(ctx)
        raise SkirtError(rc, msg.decode() if msg else "error")
    return rc
