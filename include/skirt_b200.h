/* skirt_b200.h -- C-ABI of the B200-native photon-packet life cycle.
 *
 * This is the drop-in boundary for SKIRT7's packet loop.  In the reference the
 * loop is a ParallelTarget body dispatched by
 *     Parallel::call(this, &MonteCarloSimulation::dostellaremissionchunk, Nlambda, Nchunks)
 * (SKIRTcore/MonteCarloSimulation.cpp:241-255, template at SKIRTcore/Parallel.hpp:109-121),
 * and per packet it calls the virtual plugin interfaces DustGrid::path (DustGrid.hpp:106),
 * DustSystem::fillOpticalDepth/opticaldepth/absorb (DustSystem.cpp:935-976),
 * Instrument::detect (Instrument.hpp:83) and StellarComp::launch (StellarComp.hpp:42).
 * A virtual call per packet per cell crossing cannot cross a C ABI efficiently, so
 * the library replaces the WHOLE chunk loop: one call per phase per batch.  A per-ray
 * path entry point (skg_trace_paths) exists for bit-exact traversal checks.
 *
 * Conventions
 *  - Nothing throws across this boundary.  Every function returns SKG_OK (0) or a
 *    SKG_ERR_* code; skg_last_error() gives the message.  A host shim turns a non-zero
 *    status into the reference's FatalError (SKIRTcore/FatalError.hpp:29-40).
 *  - All pointers are host pointers.  Inputs are copied during the call; the context
 *    owns every device buffer until skg_ctx_destroy().  No device pointer escapes.
 *  - Units are SI (m, W, kg), as in the reference's internal units (SKIRTcore/Units.cpp:17-30).
 *  - A context is externally synchronised: one host thread at a time.
 */
#ifndef SKIRT_B200_H
#define SKIRT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SKG_ABI_VERSION 1

/* ---- status codes ------------------------------------------------------------------ */
#define SKG_OK                 0
#define SKG_ERR_INVALID        1   /* invalid scene / argument (FatalError at setup in the reference) */
#define SKG_ERR_OOM            2   /* device allocation failed (the context or batch stays usable) */
#define SKG_ERR_CUDA           3   /* CUDA runtime error */
#define SKG_ERR_STEP_BUDGET    4   /* a packet exceeded its traversal-step or scattering budget */
#define SKG_ERR_NAN_TAU        5   /* optical depth along a path is not a positive number (DustSystem.cpp:953-955) */
#define SKG_ERR_TIMEOUT        6   /* a bounded host wait gave up */
#define SKG_ERR_NO_DEVICE      7   /* no CUDA device */
#define SKG_ERR_CAPACITY       8   /* an output buffer or a batch's tables are too small */
#define SKG_ERR_BAD_CELL       9   /* a cell index out of range was produced or given */

/* ---- enumerations ------------------------------------------------------------------ */
/* dust grid structure (SKIRTcore/CartesianDustGrid, OctTreeDustGrid, BinTreeDustGrid, VoronoiDustGrid) */
#define SKG_GRID_CARTESIAN     0
#define SKG_GRID_OCTREE        1
#define SKG_GRID_BINTREE       2
#define SKG_GRID_VORONOI       3

/* tree search method (SKIRTcore/TreeDustGrid.hpp:45-50) */
#define SKG_SEARCH_TOPDOWN     0
#define SKG_SEARCH_NEIGHBOR    1
#define SKG_SEARCH_BOOKKEEPING 2

/* geometries (SKIRTcore/ExpDiskGeometry, SersicGeometry, PointGeometry, PlummerGeometry) */
#define SKG_GEOM_EXPDISK       0
#define SKG_GEOM_SERSIC        1
#define SKG_GEOM_POINT         2
#define SKG_GEOM_PLUMMER       3

/* clump smoothing kernels (SKIRTcore/CubicSplineSmoothingKernel, UniformSmoothingKernel) */
#define SKG_KERNEL_CUBICSPLINE 0
#define SKG_KERNEL_UNIFORM     1

/* instruments (SKIRTcore/SEDInstrument, FrameInstrument, SimpleInstrument, FullInstrument) */
#define SKG_INSTR_SED          0
#define SKG_INSTR_FRAME        1
#define SKG_INSTR_SIMPLE       2
#define SKG_INSTR_FULL         3

/* phases (MonteCarloSimulation::runstellaremission, PanMonteCarloSimulation::rundustselfabsorption,
   ::rundustemission) */
#define SKG_PHASE_STELLAR      0
#define SKG_PHASE_DUST_SELFABS 1
#define SKG_PHASE_DUST_EMISSION 2

/* geometry precision of the traversal (tallies and cumulative optical depths are always FP64) */
#define SKG_PREC_FP32          0
#define SKG_PREC_FP64          1

/* FullInstrument flux components, in tally order (FullInstrument.cpp:109-177) */
#define SKG_FULL_TOT           0   /* total (what Frame/Simple/SED record)           */
#define SKG_FULL_TRA           1   /* transparent (dust-free) stellar flux            */
#define SKG_FULL_STRDIR        2   /* direct stellar flux                             */
#define SKG_FULL_STRSCA        3   /* scattered stellar flux                          */
#define SKG_FULL_DUSDIR        4   /* direct dust emission                            */
#define SKG_FULL_DUSSCA        5   /* scattered dust emission                         */
#define SKG_FULL_NBASE         6   /* followed by nscatt_levels single-level slices    */

/* ---- scene description ------------------------------------------------------------- */

/* Dust grid.  Extent fields always apply; the other blocks apply to one grid type. */
typedef struct skg_grid {
    int32_t type;                           /* SKG_GRID_* */
    double xmin, ymin, zmin, xmax, ymax, zmax;

    /* Cartesian: nx*ny*nz cells, planes xv[nx+1], yv[ny+1], zv[nz+1]; cell m = k + nz*j + nz*ny*i
       (CartesianDustGrid.cpp:326-329) */
    int32_t nx, ny, nz;
    const double* xv;
    const double* yv;
    const double* zv;

    /* Octree / k-d tree: nodes in creation order (node 0 = root, children consecutive),
       node_box[6*l] = xmin,ymin,zmin,xmax,ymax,zmax; node_child[l] = id of child 0 or -1 for a leaf;
       node_father[l] (-1 for the root); node_cell[l] = cell number of a leaf or -1;
       node_dir[l] = split direction of a binary node (0,1,2) or -1.
       Neighbour lists of each node wall in CSR form: nbr_offsets[6*l+w] .. nbr_offsets[6*l+w+1]
       index nbr_ids (wall order BACK,FRONT,LEFT,RIGHT,BOTTOM,TOP as TreeNode::Wall).  May be
       NULL unless search_method == SKG_SEARCH_NEIGHBOR. */
    int32_t nnodes;
    const double*  node_box;
    const int32_t* node_child;
    const int32_t* node_father;
    const int32_t* node_cell;
    const int8_t*  node_dir;
    const int64_t* nbr_offsets;
    const int32_t* nbr_ids;
    int32_t search_method;                  /* SKG_SEARCH_* */

    /* Voronoi: nsites generator points sites[3*m]; neighbour lists in CSR form
       (vnbr_offsets[nsites+1], vnbr_ids; walls are -1..-6 as in Voro++/VoronoiMesh.cpp:836-845);
       a uniform block grid of nb^3 blocks listing the cells whose bounding box overlaps each block
       (VoronoiMesh.cpp:334-404): block_offsets[nb^3+1], block_ids. */
    int32_t nsites;
    const double*  sites;
    const int64_t* vnbr_offsets;
    const int32_t* vnbr_ids;
    int32_t nb;
    const int64_t* block_offsets;
    const int32_t* block_ids;
    const double*  cell_volume;             /* [nsites] Voronoi cell volumes */
    const double*  cell_bbox;               /* [6*nsites] enclosing boxes (VoronoiMesh.cpp:44-52) */
} skg_grid;

/* A geometry, optionally wrapped by a ClumpyGeometryDecorator (clump_count > 0). */
typedef struct skg_geometry {
    int32_t type;                           /* SKG_GEOM_* */
    /* EXPDISK: p0=hR p1=hz p2=Rmax p3=zmax p4=Rmin (ExpDiskGeometry.cpp:24-40)
       SERSIC : p0=n  p1=reff                     (SersicGeometry.cpp:29-39)
       PLUMMER: p0=c (scale radius)                                        */
    double p[6];
    double clump_fraction;                  /* ClumpyGeometryDecorator::_f */
    int32_t clump_count;                    /* _N; 0 = no decorator */
    double clump_radius;                    /* _h */
    int32_t clump_cutoff;                   /* _cutoff */
    int32_t clump_kernel;                   /* SKG_KERNEL_* */
    const double* clump_pos;                /* 3*clump_count, any order (sorted on x internally) */
} skg_geometry;

typedef struct skg_stellar_comp {
    skg_geometry geometry;
    const double* luminosity;               /* [nlambda] bolometric luminosity per wavelength bin (W) */
} skg_stellar_comp;

typedef struct skg_dust_comp {
    skg_geometry geometry;                  /* density = norm * geometry density (DustComp.cpp:100-106) */
    double norm;                            /* normalisation factor _nf (kg) */
    const double* kappaext;                 /* [nlambda] m2/kg */
    const double* albedo;                   /* [nlambda] */
    const double* asymmpar;                 /* [nlambda] Henyey-Greenstein g */
} skg_dust_comp;

typedef struct skg_instrument {
    int32_t type;                           /* SKG_INSTR_* */
    double distance, inclination, azimuth, position_angle;   /* m, rad (DistantInstrument.cpp:24-50) */
    int32_t nxp, nyp;                       /* pixels (SingleFrameInstrument) */
    double fovx, fovy, xc, yc;              /* field of view and centre (m) */
    int32_t nscatt_levels;                  /* FullInstrument::_Nscatt */
    int32_t stellar_comps;                  /* FRAME: also one frame per stellar component, the
                                               peel-offs of the packets it launched (components
                                               1..nstellar after the total; the frames FitSKIRT fits,
                                               MultiFrameInstrument::writeStellarComps,
                                               MultiFrameInstrument.cpp:17-57) */
} skg_instrument;

typedef struct skg_scene {
    skg_grid grid;

    int32_t nlambda;
    const double* lambda;                   /* [nlambda] m */
    const double* dlambda;                  /* [nlambda] m */

    int32_t ncomp;                          /* dust components (<= 4); 0 = no dust system */
    const skg_dust_comp* dust;
    const double* rho;                      /* optional [ncomp][ncells] cell densities; NULL = sample them
                                               on the device (DustSystem::setSampleDensityBody) */
    int32_t density_samples;                /* DustSystem::_Nrandom (default 100) */

    int32_t nstellar;
    const skg_stellar_comp* stellar;
    double emission_bias;                   /* StellarSystem::_emissionBias (default 0.5) */

    int32_t ninstr;
    const skg_instrument* instr;

    double min_weight_reduction;            /* default 1e4 (MonteCarloSimulation.hpp:43-47) */
    int32_t min_scatt_events;               /* default 0 */
    double scatt_bias;                      /* xi, default 0.5 */
    int32_t store_absorption;               /* keep per-cell absorbed luminosity (writeMeanIntensity / dust emission) */

    /* dust emission (PanDustSystem with GreyBodyDustEmissivity + AllCellsDustLib) */
    int32_t dust_emission;
    double dust_emission_bias;              /* PanDustSystem::_emissionBias (default 0.5) */
} skg_scene;

/* Per-call launch controls. */
typedef struct skg_run_opts {
    int32_t precision;                      /* SKG_PREC_* for the traversal geometry */
    int32_t max_steps;                      /* per traversal cell-step budget (0 = default 1<<20) */
    int32_t max_scatt;                      /* per packet scattering budget (0 = default 100000) */
    int32_t blocks;                         /* traversal blocks per wave (0 = auto: resident blocks x SMs) */
    int32_t refill;                         /* traversal lanes of a warp that wait for a job before the warp
                                               takes new ones, 1..32 (0 = default 8; the autotuner's choice) */
    int32_t dedupe_peeloff;                 /* share one peel-off traversal among instruments that see
                                               the packet from the same direction (same tau; default 1) */
    int32_t pool;                           /* packets in flight per wave (0 = default: 2^21, or 2^23 for a
                                               skg_run_phase of at least 2^26 packets on a Cartesian or tree
                                               grid) */
} skg_run_opts;

/* Counters of one phase run (device side, exact). */
typedef struct skg_counters {
    uint64_t packets;                       /* packets launched */
    uint64_t steps;                         /* cell steps of all traversals */
    uint64_t traversals;                    /* traversals (main, interaction re-walk, peel-off) */
    uint64_t scatterings;                   /* scattering events */
    uint64_t peeloffs;                      /* peel-off detections */
    uint64_t absorb_adds;                   /* per-cell absorption tally updates */
    uint64_t pixel_adds;                    /* pixel tally updates */
    uint64_t nbr_scanned;                   /* neighbour-list entries scanned (tree/Voronoi) */
    uint64_t fallbacks;                     /* neighbour search fallbacks / re-locations */
    uint64_t errors;                        /* packets retired on a budget or NaN */
    uint64_t waves;                         /* waves (event pass + traversal pass) of the phase */
} skg_counters;

typedef struct skg_ctx skg_ctx;

/* ---- lifecycle --------------------------------------------------------------------- */
int         skg_version(void);
/* Message of the most recent error on this thread (ctx may be NULL). */
const char* skg_last_error(const skg_ctx* ctx);
int         skg_device_count(int* count);

/* Uploads the scene: grid (SoA, FP64 and FP32 copies), cell densities (given, or sampled on the
   device), mix tables, source samplers, instrument frames.  Replaces Simulation::setup
   (SimulationItem.cpp:18-31) for the items on the hot path. */
int  skg_ctx_create(const skg_scene* scene, int device, skg_ctx** out);
/* Waits for the context's own work and frees it.  Its device memory is stream-ordered (allocated
   and freed on the context's stream, from the device's default memory pool), so destroying a
   context does not synchronise the device: other contexts and batches keep running. */
int  skg_ctx_destroy(skg_ctx* ctx);
/* Number of dust cells, and the device bytes held by the context (admission by footprint). */
int  skg_ctx_info(const skg_ctx* ctx, int64_t* ncells, int64_t* device_bytes);

/* Per-cell densities actually used (after device sampling), [ncomp][ncells]. */
int  skg_read_density(skg_ctx* ctx, double* rho);

/* ---- bit-exact traversal harness (DustGrid::path) ------------------------------------ */
/* For n rays (r[3n], k[3n]) computes the path through the grid exactly as DustGrid::path:
   cells[] and ds[] receive the segments of ray i at offsets[i] .. offsets[i+1]-1
   (m = -1 for segments outside the grid).  capacity = length of cells/ds.  Returns
   SKG_ERR_CAPACITY (and the needed total in offsets[n]) when the buffers are too small,
   SKG_ERR_INVALID for a precision other than SKG_PREC_FP32 / SKG_PREC_FP64.  Synchronous. */
int  skg_trace_paths(skg_ctx* ctx, const double* r, const double* k, int64_t n, int precision,
                     int32_t* cells, double* ds, int64_t* offsets, int64_t capacity);

/* The same paths as skg_trace_paths for callers that cannot allocate device memory during a
   call (a serving loop or host framework that owns a fixed HBM budget; cudaMalloc would
   synchronise the device and can fail on a fragmented heap).  No counterpart in the reference:
   it exists only because of how this library is embedded.
   All pointers are DEVICE pointers: d_r[3n], d_k[3n] in; d_cells/d_ds (length capacity) and
   d_offsets (n+1) out, with the same layout and values as skg_trace_paths.  The call allocates
   nothing: its scratch (per-ray counts and scan totals, 8 MiB + 8 KiB) is a static device array
   of this library, so n is limited to SKG_NOALLOC_MAX_RAYS (larger n returns SKG_ERR_CAPACITY
   at once).  The device address of that array is looked up on the first call on each device;
   make that first call before any stream capture.  A phase still running on the context is
   finished first (as every other entry point does).  The work is enqueued on `stream` (NULL =
   the context's stream) and the call returns without waiting.  skg_sync(ctx, ...) waits for
   the end of this work on that stream (bounded by its timeout) and then reports, once,
   SKG_ERR_CAPACITY when the segments exceed `capacity` (d_offsets[n] then holds the needed
   total) or SKG_ERR_STEP_BUDGET; a caller that does not call skg_sync can compare d_offsets[n]
   with `capacity` itself.  These flags live in a word of the context that the phases do not
   use, so the call never clears a finished phase's flags.  Any precision other than
   SKG_PREC_FP32 / SKG_PREC_FP64 returns SKG_ERR_INVALID.  All calls on one device share the one
   scratch array: two calls whose work overlaps in time (different streams or threads, or
   different contexts on the same device) race and corrupt each other's results. */
#define SKG_NOALLOC_MAX_RAYS 1048576
int  skg_trace_paths_noalloc(skg_ctx* ctx, const double* d_r, const double* d_k, int64_t n, int precision,
                             int32_t* d_cells, double* d_ds, int64_t* d_offsets, int64_t capacity,
                             void* stream);

/* Optical depth from each r along k to the grid edge at wavelength ell (Instrument::opticalDepth ->
   DustSystem::opticaldepth, DustSystem.cpp:960-976). */
int  skg_optical_depth(skg_ctx* ctx, const double* r, const double* k, int64_t n, int ell,
                       int precision, double* tau);

/* ---- the packet loop ---------------------------------------------------------------- */
/* MonteCarloSimulation::setChunkParams (MonteCarloSimulation.cpp:68-114): packet count actually
   run per wavelength for `packages` requested, nthreads workers and nprocs processes. */
int  skg_chunk_params(double packages, int nthreads, int nprocs, int nlambda,
                      uint64_t* nchunks, uint64_t* chunksize, uint64_t* npp);

/* Runs one phase for the wavelength indices ells[0..nell-1] in one persistent launch.  npp is
   the definitive packet count per wavelength (each packet carries L/npp, as _Npp in the
   reference); this call runs the packets with ids [first_packet, first_packet+count) of every
   wavelength (count = npp on one device; ranks take disjoint ranges).  The stream is a
   cudaStream_t (NULL = the context's own stream).  Returns once the launch is enqueued; the
   skg_read_* functions synchronise. */
int  skg_run_phase(skg_ctx* ctx, int phase, const int32_t* ells, int nell, uint64_t npp,
                   uint64_t first_packet, uint64_t count, uint64_t seed, const skg_run_opts* opts,
                   void* stream);

/* ---- batched launches (many simulations in one persistent launch) ------------------------ */
/* A slice of one simulation: packets [first, first+count) of each listed wavelength, each carrying
   L/npp of the simulation. */
typedef struct skg_work {
    skg_ctx* ctx;
    const int32_t* ells;
    int32_t nell;
    uint64_t npp, first, count, seed;
} skg_work;
typedef struct skg_batch skg_batch;
/* Staging for batched launches on one device: up to max_slots distinct simulations, max_items
   slices and max_ells wavelength entries per launch. */
int  skg_batch_create(int device, int max_slots, int max_items, int max_ells, skg_batch** out);
int  skg_batch_destroy(skg_batch* b);
/* Runs the slices in ONE persistent launch (all contexts on the batch's device, same grid type).
   A packet's random stream depends only on (seed, packet id, wavelength, phase), so a
   simulation's tallies are the same alone and mixed with others, up to the summation order of the
   FP64 atomics.  With SKG_BATCH_GRAPH in `flags` the launch sequence (table uploads, counter
   reset, tracer) is captured once into a CUDA graph and replayed while the grid type and launch
   configuration stay the same.  Returns once enqueued on `stream` (NULL = the batch's own
   stream).  More work items, distinct simulations or wavelength entries than the batch was
   created for return SKG_ERR_CAPACITY. */
#define SKG_BATCH_GRAPH 1
int  skg_batch_run(skg_batch* b, int phase, const skg_work* work, int nwork, const skg_run_opts* opts,
                   int flags, void* stream);
int  skg_batch_sync(skg_batch* b, int timeout_ms);
int  skg_batch_counters(skg_batch* b, skg_counters* out);
int  skg_batch_last_ms(skg_batch* b, float* ms);

/* ---- serving: continuous batching of many simulations on one device --------------------- */
/* The request pattern of FitSKIRT (FitSKIRTcore/OligoFitScheme.cpp:123-149 runs one simulation per
   parameter set through AdjustableSkirtSimulation::performWith, AdjustableSkirtSimulation.cpp:
   145-194): many short simulations of one ski file with a few values substituted.  A server admits
   submitted requests in arrival order while a batch slot is free and the request's device-memory
   bound fits hbm_budget (admission by HBM footprint), builds their contexts on a host thread of
   its own, and runs ticks -- one batched launch (skg_batch_run) carrying the next packet slice of
   every admitted request, oldest first up to tick_budget packets -- so that requests arriving
   while others run join the next tick.  A request retires when all its packets have run: its
   instrument's tallies are copied into the caller's buffers and its context is freed by a third
   host thread, off the ticks' path.  skg_server_create raises the release threshold of the
   device's default memory pool (cudaMemPoolAttrReleaseThreshold) to at least hbm_budget for the
   process, so that freed context memory is kept for the next contexts instead of being unmapped
   at each synchronisation (contexts allocate stream-ordered from that pool).  Its
   packets draw from streams keyed by its seed and packet index, so its result equals the same
   simulation run alone (skg_run_phase with count = npp) up to the order of the FP64 tally
   additions.  The stellar emission phase is served. */
typedef struct skg_server skg_server;
typedef struct skg_server_opts {
    int64_t hbm_budget;                     /* device bytes the admitted requests may hold together (0: 40 GiB) */
    int32_t max_slots;                      /* requests per launch, 1..64 (0: 64) */
    int64_t tick_packets;                   /* packets per wavelength each ready request is given first in a tick
                                               (0: 2^23); budget left after that goes to the oldest requests */
    int64_t tick_budget;                    /* packets (all wavelengths) one tick hands out (0: 16 * 2^20) */
    int32_t precision;                      /* SKG_PREC_* of the traversal geometry */
} skg_server_opts;
typedef struct skg_request {
    const skg_scene* scene;                 /* copied by skg_submit, arrays included */
    const int32_t* ells;                    /* wavelength indices (1..64 of them) */
    int32_t nell;
    uint64_t packages;                      /* packets per wavelength (the simulation's Npp) */
    uint64_t seed;
    int32_t instr;                          /* the instrument whose tallies are the result */
    double* cube;                           /* host buffer of the cube length (skg_scene_tally_sizes), or NULL */
    double* sed;                            /* host buffer of the SED length, or NULL; both written by the
                                               server thread, and final once skg_poll returns SKG_OK */
} skg_request;
int  skg_server_create(int device, const skg_server_opts* opts, skg_server** out);
/* Queues a request; returns at once with its id. */
int  skg_submit(skg_server* s, const skg_request* req, int64_t* id);
/* Waits up to timeout_ms (-1: no limit) for request id: SKG_ERR_TIMEOUT while it runs, else its
   status (SKG_OK: the result is in its buffers), reported once; latency_s (optional) receives the
   time from submission to completion. */
int  skg_poll(skg_server* s, int64_t id, int timeout_ms, double* latency_s);
/* Ticks run, requests completed, packets run (all wavelengths) and the device time of the ticks. */
int  skg_server_stats(skg_server* s, int64_t* ticks, int64_t* completed, int64_t* packets, double* tick_ms);
/* Waits for a context being built, ends every unfinished request with SKG_ERR_INVALID (its buffers
   are not written), and frees the server. */
int  skg_server_destroy(skg_server* s);
/* Tally lengths of instrument instr of a scene (as skg_tally_sizes gives for its context). */
int  skg_scene_tally_sizes(const skg_scene* scene, int instr, int64_t* cube_len, int64_t* sed_len);

/* Zeroes all tallies (instrument cubes and SEDs, absorbed luminosity). */
int  skg_reset_tallies(skg_ctx* ctx);

/* Tally layout: for instrument i, cube[i] has ncomponents(i) x nlambda x nyp x nxp doubles
   (pixel index i + nxp*j within a slice, ParallelDataCube.cpp:80-91) and sed[i] has
   ncomponents(i) x nlambda doubles; ncomponents is 1 except for FullInstrument
   (SKG_FULL_NBASE + nscatt_levels).  SED instruments have no cube. */
int  skg_tally_sizes(const skg_ctx* ctx, int instr, int64_t* cube_len, int64_t* sed_len);
int  skg_read_instrument(skg_ctx* ctx, int instr, double* cube, double* sed);
/* Device-to-device copy of instrument instr's tallies into caller-owned DEVICE buffers, enqueued
   on `stream` (a cudaStream_t; NULL = the context stream) after the work already on it.  This is
   how ranks hand their frames to a collective (the reference's Instrument::sumResults,
   Instrument.cpp:57-65) without the tallies leaving the device. */
int  skg_read_instrument_device(skg_ctx* ctx, int instr, double* d_cube, double* d_sed, void* stream);
/* Absorbed luminosity [ncells][nlambda] (stellar and dust parts separately; either may be NULL). */
int  skg_read_absorption(skg_ctx* ctx, double* labs_stellar, double* labs_dust);
int  skg_read_counters(skg_ctx* ctx, skg_counters* out);
/* Finishes the running phase and waits for the context stream (and for the last
   skg_trace_paths_noalloc call on its caller's stream) with a bounded wait: SKG_ERR_TIMEOUT
   after timeout_ms (-1 = no limit; a later call waits again).  Then reports the flags of the
   last phase (SKG_ERR_NAN_TAU, SKG_ERR_STEP_BUDGET, SKG_ERR_CAPACITY; they stay until the next
   phase starts) and of the last no-alloc path call (reported once). */
int  skg_sync(skg_ctx* ctx, int timeout_ms);
/* Device time (ms) of the last skg_run_phase launch (CUDA events on the launching stream). */
int  skg_last_phase_ms(skg_ctx* ctx, float* ms);
/* The last phase split by kernel: summed device time (ms) of its event passes (launch, detection,
   scattering) and of its traversal passes, and its number of waves (each wave is one launch of
   each).  Finishes the phase first. */
int  skg_phase_times(skg_ctx* ctx, float* event_ms, float* traversal_ms, int32_t* waves);

/* ---- dust emission (PanDustSystem::calculatedustemission / DustLib::calculate) --------- */
/* From the absorbed luminosity held in the context computes, per cell, the mean intensity
   (DustSystem::meanintensityv, DustSystem.cpp:911-931), the equilibrium temperature
   (DustMix::equilibrium, DustMix.cpp:689-697) and the normalised grey-body emission spectrum
   (GreyBodyDustEmissivity.cpp:21-45, DustLib.cpp:89-153).  Temperatures optional. */
int  skg_calc_dust_emission(skg_ctx* ctx, double* temperature);
/* Total absorbed luminosity (stellar, dust) for the self-absorption convergence test. */
int  skg_absorbed_totals(skg_ctx* ctx, double* labs_stellar_tot, double* labs_dust_tot);
/* PanDustSystem::rebootLabsdust */
int  skg_reset_dust_absorption(skg_ctx* ctx);

/* ---- grid construction ---------------------------------------------------------------- */
/* Builds an octree (type SKG_GRID_OCTREE) or k-d tree (SKG_GRID_BINTREE, alternating split
   directions) over the extent in `grid` by the subdivision rules of TreeDustGrid::subdivide
   (TreeDustGrid.cpp:166-230) using the dust densities of `scene` (mass fraction criterion,
   sampled with `samples` random points per node on the device), then the neighbour lists
   (OctTreeNode.cpp:67-180, BinTreeNode.cpp:75-320) sorted by decreasing overlap
   (TreeNode.cpp:151-158).  The result is held in an opaque builder; its arrays are copied
   out with skg_tree_arrays. */
typedef struct skg_tree skg_tree;
int  skg_tree_build(const skg_scene* scene, int type, int min_level, int max_level,
                    double max_mass_fraction, int samples, uint64_t seed, int device, skg_tree** out);
/* Builds a tree from explicit subdivision decisions: split[l] != 0 for nodes to subdivide,
   visited in creation order (for checks against the reference's node classes). */
int  skg_tree_from_splits(int type, double xmin, double ymin, double zmin, double xmax, double ymax,
                          double zmax, const uint8_t* split, int64_t nsplit, skg_tree** out);
int  skg_tree_sizes(const skg_tree* t, int32_t* nnodes, int32_t* ncells, int64_t* nnbr);
int  skg_tree_arrays(const skg_tree* t, double* node_box, int32_t* node_child, int32_t* node_father,
                     int32_t* node_cell, int8_t* node_dir, int64_t* nbr_offsets, int32_t* nbr_ids);
/* Fills grid fields from the builder (pointers stay valid until skg_tree_destroy). */
int  skg_tree_grid(const skg_tree* t, skg_grid* grid);
int  skg_tree_destroy(skg_tree* t);

/* Builds the Voronoi tessellation of `nsites` points clipped to the given extent
   (VoronoiMesh::buildMesh, VoronoiMesh.cpp:297-405): sites outside the extent and sites within
   1e-12 of the extent diagonal of another are dropped as the reference does; per kept site the
   neighbour list with the wall ids -1..-6, the cell volume, centroid and bounding box, and the
   nb^3 block lists.  Cells are computed on the device by clipping against nearby bisector planes. */
typedef struct skg_voronoi skg_voronoi;
int  skg_voronoi_build(const double* sites, int32_t nsites, double xmin, double ymin, double zmin,
                       double xmax, double ymax, double zmax, int device, skg_voronoi** out);
int  skg_voronoi_sizes(const skg_voronoi* v, int32_t* nsites, int64_t* nnbr, int32_t* nb,
                       int64_t* nblockids);
int  skg_voronoi_arrays(const skg_voronoi* v, double* sites, int64_t* vnbr_offsets, int32_t* vnbr_ids,
                        double* volume, double* centroid, double* bbox,
                        int64_t* block_offsets, int32_t* block_ids);
int  skg_voronoi_grid(const skg_voronoi* v, skg_grid* grid);
int  skg_voronoi_destroy(skg_voronoi* v);

#ifdef __cplusplus
}
#endif
#endif /* SKIRT_B200_H */
